"""Host logic of the GPU mat-vec: the restricted transforms that operator.py builds for every mode reproduce the
reference's FFT operator (golden mat-vecs). The contraction is emulated here in NumPy with the same stage order
as csrc/matvec.cu (contract the last axis, move the new axis to the front), so the schedule is checked on CPU too."""
import numpy as np
import pytest

from conftest import golden
from golden_cases import MATVEC_SPECS
from blml_b200 import operator as op_mod
from blml_b200.spec import parse_modes


def emulate(freqs, W, shape, x):
    """The stage schedule of csrc/matvec.cu in NumPy: x (nb, *shape) -> S x."""
    d = len(shape)
    cur = np.asarray(x, complex).reshape((x.shape[0],) + tuple(shape))
    V = [np.exp(2j * np.pi * np.outer(np.arange(m), f)) for m, f in zip(shape, freqs)]
    for s in range(d):                       # forward: contract last axis with conj(V_a), move to front
        a = d - 1 - s
        cur = np.moveaxis(np.tensordot(cur, np.conj(V[a]), axes=([-1], [0])), -1, 1)
    cur = cur * W[None]
    for s in range(d):                       # inverse: contract last axis with V_a^T
        a = d - 1 - s
        cur = np.moveaxis(np.tensordot(cur, V[a].T, axes=([-1], [0])), -1, 1)
    return cur


@pytest.mark.parametrize('name', list(MATVEC_SPECS))
def test_transform_reproduces_reference(name):
    g = golden('matvec.npz')[name]
    shape, modes, h = MATVEC_SPECS[name]
    d = len(shape)
    specs, _ = parse_modes(modes, d)
    hv = np.full(d, h)
    pad = op_mod.pad_rule(shape, hv, specs)
    assert tuple(pad) == tuple(g['pad'])
    E, U = g['E'], g['U']
    for k, sp in enumerate(specs):
        freqs, W = op_mod.mode_transform(sp, shape, hv, pad)
        assert abs(op_mod.kernel_at_zero(sp, d) - float(g['s'][k])) <= 1e-14 * abs(float(g['s'][k]))
        y = emulate(freqs, W, shape, E[k][None])[0]
        if not np.iscomplexobj(E):
            assert np.abs(y.imag).max() <= 1e-12 * np.abs(y).max()
            y = y.real
        assert np.abs(y - U[k]).max() <= 1e-12 * np.abs(U[k]).max(), name


def test_pball_circular_is_band_mask():
    """On a circular lattice the pball transform is the kernel's DFT mask: 5,621 harmonics at fc 0.33 on 256^2."""
    specs, _ = parse_modes([{(0, 1): dict(kind='pball', fc=0.33, period=[256.0, 256.0])}], 2)
    freqs, W = op_mod.mode_transform(specs[0], (256, 256), np.ones(2), (256, 256))
    assert [len(f) for f in freqs] == [85, 85]
    assert int((W > 0).sum()) == 5621


GRAD_OPS = [((40,), [{0: dict(kind='sinc', fc=0.35)}], 1.0),
            ((64,), [{0: dict(kind='slits', fc=0.3, fill=0.4)}], 1.0),
            ((24, 24), [{0: dict(kind='sinc', fc=0.4), 1: dict(kind='sinc', fc=0.3)}], 1.0),
            ((20, 20), [{(0, 1): dict(kind='ball', fc=0.45)}], 1.0),
            ((16, 12), [{0: dict(kind='dirichlet', fc=0.3, period=16.0), 1: dict(kind='sinc', fc=0.8)}], 0.5)]


@pytest.mark.parametrize('case', range(len(GRAD_OPS)))
def test_dlog_transforms_reproduce_oracle(case):
    """dS/dlog fc_u of every unit (blml_binned.py:92-101): the plane-wave forms of operator.mode_transform_dlog through
    the mat-vec's stage schedule equal the oracle's padded-FFT convolution with the dK/dlog fc table; integer units
    have none."""
    import blml_oracle as bo
    import grad_oracle as go
    shape, modes, h = GRAD_OPS[case]
    d = len(shape)
    specs, _ = parse_modes(modes, d)
    ospecs = bo.parse_modes(modes, d)
    hv = np.full(d, h)
    pad = op_mod.pad_rule(shape, hv, specs)
    rng = np.random.default_rng(case)
    x = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    fit = type('F', (), {})()
    fit.op = bo.Operator(ospecs, shape, hv)
    dks = go.dK_spectra(ospecs[0], shape, hv, fit.op.pad)
    units = op_mod.units_of(specs[0]['kinds'])
    assert len(dks) == len(units)
    for u, dK in enumerate(dks):
        tr = op_mod.mode_transform_dlog(specs[0], shape, hv, pad, u)
        assert (tr is None) == (dK is None)
        if tr is None:
            continue
        y = emulate(tr[0], tr[1], shape, x[None])[0]
        ref = go._apply(fit, dK, x)
        assert np.abs(y - ref).max() <= 1e-11 * np.abs(ref).max(), (case, u)
