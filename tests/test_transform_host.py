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
