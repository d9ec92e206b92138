"""The FFT route of the mat-vec (row / column FFTs of a DFT-mask kernel, csrc/fft_matvec.cu) against the restricted
transforms of the same plan and against the oracle's padded-FFT operator (the reference's own arithmetic,
blml_binned.py:156-168): single plans over one or two lattices, real and complex input, float64 and float32; the
grouped launch over every lattice of the 64-fit benchmark sweep, with a subset and a live mask; kernels without a
DFT-mask form keep the contraction route."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

SHAPES = [((64, 64), 0.33), ((96, 384), 0.45), ((384, 384), 0.2), ((192, 128), 0.05), ((256, 256), 0.33),
          ((128, 96), 0.12), ((384, 64), 0.4)]


def _plan(shape, fc, code):
    from blml_b200 import operator as op_mod, _lib, workloads
    from blml_b200.spec import parse_modes
    sp, _ = parse_modes(workloads.pball_modes(shape, fc), 2)
    return op_mod.Plan(*op_mod.mode_transform(sp[0], shape, np.ones(2), shape), shape, code, _lib.ENGINE_SIMT)


@pytest.mark.parametrize('dt', [np.float64, np.float32])
@pytest.mark.parametrize('shape,fc', SHAPES)
def test_fft_route_equals_contraction(cuda_device, dt, shape, fc):
    from blml_b200 import _lib
    code = _lib.F64 if dt == np.float64 else _lib.F32
    ct, rt = (torch.complex128, torch.float64) if dt == np.float64 else (torch.complex64, torch.float32)
    tol = 1e-12 if dt == np.float64 else 2e-6
    p = _plan(shape, fc, code)
    assert p.route == _lib.ROUTE_FFT
    st = torch.cuda.current_stream().cuda_stream
    g = torch.Generator(device='cuda').manual_seed(3)
    for xc in (True, False):
        for nb in (1, 2):
            x = torch.randn((nb,) + shape, dtype=ct if xc else rt, device='cuda', generator=g)
            y_fft, y_con = torch.empty_like(x), torch.empty_like(x)
            p.route = _lib.ROUTE_FFT
            p.apply(x, y_fft, nb, xc, st)
            p.route = _lib.ROUTE_CONTRACT
            p.apply(x, y_con, nb, xc, st)
            p.route = _lib.ROUTE_AUTO
            err = (y_fft - y_con).abs().max().item()
            assert err <= tol * y_con.abs().max().item(), (xc, nb, err)


@pytest.mark.parametrize('shape,fc', SHAPES[:4])
def test_fft_route_matches_oracle(cuda_device, shape, fc):
    import blml_oracle as bo
    from blml_b200 import _lib, workloads
    p = _plan(shape, fc, _lib.F64)
    rng = np.random.default_rng(11)
    e = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    x = torch.as_tensor(e).to('cuda')
    y = torch.empty_like(x)
    p.apply(x, y, 1, True, torch.cuda.current_stream().cuda_stream)
    ref = bo.Operator(bo.parse_modes(workloads.pball_modes(shape, fc), 2), shape, np.ones(2)).S(0, e)
    assert np.abs(y.cpu().numpy() - ref).max() <= 1e-12 * np.abs(ref).max()


@pytest.mark.parametrize('dt', [np.float64, np.float32])
def test_grouped_fft_route_over_the_benchmark_sweep(cuda_device, dt):
    """Every lattice of the 64-fit sweep (sides 64..384, fc 0.05..0.45) in one grouped launch: FFT route = the
    contraction route; then a masked launch over a subset with one problem off leaves that problem untouched."""
    from blml_b200.sweep import _Group
    from blml_b200 import _lib, workloads
    from blml_b200._lib import call
    code = _lib.F64 if dt == np.float64 else _lib.F32
    ct, rt = (torch.complex128, torch.float64) if dt == np.float64 else (torch.complex64, torch.float32)
    tol = 1e-12 if dt == np.float64 else 2e-6
    fits = workloads.cutoff_sweep(0)
    plans, offs, tot = [], [0], 0
    for f in fits:
        plans.append(_plan(f['shape'], f['fc'], code))
        tot += f['shape'][0] * f['shape'][1]; offs.append(tot)
    st = torch.cuda.current_stream().cuda_stream
    for xc in (True, False):
        x = torch.randn(tot, dtype=ct if xc else rt, device='cuda')
        y_fft, y_con = torch.empty_like(x), torch.empty_like(x)
        grp = _Group(plans, x, offs[:-1], y_fft, offs[:-1], xc)
        assert grp.route == _lib.ROUTE_FFT
        grp(st)
        gc = _Group(plans, x, offs[:-1], y_con, offs[:-1], xc)
        gc.route = _lib.ROUTE_CONTRACT
        gc(st)
        for g in range(len(plans)):
            a, b = y_fft[offs[g]:offs[g + 1]], y_con[offs[g]:offs[g + 1]]
            err = (a - b).abs().max().item()
            assert err <= tol * b.abs().max().item(), (g, xc, err)
    x = torch.randn(tot, dtype=ct, device='cuda')
    y = torch.zeros_like(x)
    grp = _Group(plans, x, offs[:-1], y, offs[:-1], True)
    subset = torch.arange(3, 40, dtype=torch.int32, device='cuda')
    live = torch.ones(len(plans), dtype=torch.int32, device='cuda'); live[5] = 0
    call('blml_group_matvec_masked', grp._h, subset.data_ptr(), int(subset.numel()), live.data_ptr(), st)
    for g in range(len(plans)):
        seg = y[offs[g]:offs[g + 1]]
        if g < 3 or g >= 40 or g == 5:
            assert seg.abs().max().item() == 0.0, g
        else:
            ref = torch.empty_like(seg)
            plans[g].apply(x[offs[g]:offs[g + 1]].contiguous(), ref, 1, True, st)
            assert (seg - ref).abs().max().item() <= tol * ref.abs().max().item(), g


def test_kernels_without_a_dft_mask_keep_the_contraction(cuda_device):
    from blml_b200 import operator as op_mod, _lib, make_modes
    from blml_b200.spec import parse_modes
    sp, _ = parse_modes(make_modes([0.2, 0.3], ['sinc', 'sinc']), 2)
    shape = (64, 48)
    h = np.ones(2)
    p = op_mod.Plan(*op_mod.mode_transform(sp[0], shape, h, op_mod.pad_rule(shape, h, sp)), shape, _lib.F64,
                    _lib.ENGINE_SIMT)
    assert p.route == _lib.ROUTE_CONTRACT
    with pytest.raises(_lib.BLMLError):
        p.route = _lib.ROUTE_FFT
    # a side with a prime factor 5 has no mixed-radix plan here: the contraction route
    assert _plan((80, 64), 0.3, _lib.F64).route == _lib.ROUTE_CONTRACT
