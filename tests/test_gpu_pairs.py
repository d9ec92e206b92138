"""GPU pair accumulation (rows / cols) against the reference's golden outputs: binning and pair indices bit-exact,
float64 sums to 1e-12 of the largest entry, float32 tables to 2e-4 (the reference's own f32 bar,
results/gpu_kernels_check.py)."""
import numpy as np
import pytest
import torch

from conftest import golden

pytestmark = pytest.mark.gpu


def test_rows_cols_5d(cuda_device):
    from blml_b200.local_gpu import ProductKernel, rows, cols, rank_coords
    p = golden('pairs.npz')['p5']
    u, cnt = p['bins'], p['counts']
    pk = ProductKernel(['sinc'] * 5, [None] * 5)
    tab = pk.tables(p['fc'], [None] * 5, p['h'], u)
    s, _ = rows(u, u, cnt, tab)
    scale = np.abs(p['rows']).max()
    assert np.abs(s - p['rows']).max() <= 1e-12 * scale
    s32, _ = rows(u, u, cnt, tab, f32=True)
    assert np.abs(s32 - p['rows']).max() <= 2e-4 * scale
    A = torch.as_tensor(rank_coords(u[:300], tab)).cuda(); B = torch.as_tensor(rank_coords(u[:200], tab)).cuda()
    out = torch.empty((300, 200), dtype=torch.float64, device='cuda')
    cols(A, B, tab, out)
    assert np.abs(out.cpu().numpy() - p['cols']).max() <= 1e-14
    assert np.abs(out.cpu().numpy() - p['gram']).max() <= 1e-13


def test_rows_torus_with_derivatives(cuda_device):
    from blml_b200.local_gpu import ProductKernel, rows, cols, rank_coords
    t = golden('pairs.npz')['pt']
    kinds, per = ['pball:0-1', 'pball:0-1', 'sinc'], [31.0, 31.0, None]
    fc, h = np.array([0.33, 0.33, 0.2]), np.array([1.0, 1.0, 0.7])
    pk = ProductKernel(kinds, per, fold=[True] * 3)
    want = [(1, ('shift', 0)), (1, ('shift', 1)), (0, 'fc')]
    tab = pk.tables(fc, per, h, np.r_[t['ZA'], t['ZB']], want=want)
    s, ds = rows(t['ZA'], t['ZB'], t['w'], tab, grad=True)
    assert np.abs(s - t['rows']).max() <= 1e-12
    assert np.abs(ds - t['drows']).max() <= 1e-12
    A = torch.as_tensor(rank_coords(t['ZA'], tab)).cuda(); B = torch.as_tensor(rank_coords(t['ZB'], tab)).cuda()
    out = torch.empty((len(t['ZA']), len(t['ZB'])), dtype=torch.float64, device='cuda')
    cols(A, B, tab, out)
    assert np.abs(out.cpu().numpy() - t['cols']).max() <= 1e-12


def test_stale_tables_are_an_error(cuda_device):
    """Coordinates outside the tables' span raise instead of reading out of range."""
    from blml_b200.local_gpu import ProductKernel, rows
    from blml_b200._lib import BLMLError
    Z = np.array([[0, 0], [3, 4], [6, 1]], np.int64)
    pk = ProductKernel(['sinc', 'sinc'])
    tab = pk.tables([0.3, 0.3], [None, None], [1.0, 1.0], Z)
    far = np.array([[40, 0]], np.int64)
    with pytest.raises(RuntimeError):                 # a rank column: the host rank lookup refuses it
        rows(far, Z, np.ones(3), tab)
    Zw = np.array([[0, 0], [3, 4], [6, 1], [1, 1], [2, 5]], np.int64)
    tab = ProductKernel(['sinc', 'sinc']).tables([0.3, 0.3], [None, None], [1.0, 1.0], Zw, )
    assert all(v is None for v in tab['vals'])        # offset rows only
    far_dev = torch.as_tensor([[400, 0]], dtype=torch.int64, device='cuda')
    with pytest.raises(BLMLError):                    # offset rows: the device extent check refuses it
        rows(far_dev, torch.as_tensor(Zw).cuda(), np.ones(5), tab)


def test_empty_inputs(cuda_device):
    from blml_b200.local_gpu import ProductKernel, rows
    Z = np.array([[0, 0], [3, 4]], np.int64)
    tab = ProductKernel(['sinc', 'sinc']).tables([0.3, 0.3], [None, None], [1.0, 1.0], Z)
    s, _ = rows(Z, Z[:0], np.zeros(0), tab)
    assert np.array_equal(s, np.zeros(2))
    s, _ = rows(Z[:0], Z, np.ones(2), tab)
    assert s.shape == (0,)


@pytest.mark.parametrize('case,masks', [('p5', (0b00101, 0b10000)), ('pt', (0b100, 0b001))])
def test_cols_joint_and_marginal(cuda_device, case, masks):
    """cols with depmask (blml_local_gpu.py:320-361): out = the joint block, out_m = the block of the product kernel
    over the columns outside the mask (a radial group dep when one of its columns is), both against the reference's
    own CPU blocks (tests/golden/cols_dep.npz); the pball group case masks the sinc column, then the group."""
    from blml_b200.local_gpu import ProductKernel, cols, rank_coords
    c = golden('cols_dep.npz')[case]
    p = golden('pairs.npz')[case]
    if case == 'p5':
        ZA, ZB = p['bins'][:300], p['bins'][:200]
        kinds, per, fc, h = ['sinc'] * 5, [None] * 5, p['fc'], p['h']
    else:
        ZA, ZB = p['ZA'], p['ZB']
        kinds, per = ['pball:0-1', 'pball:0-1', 'sinc'], [31.0, 31.0, None]
        fc, h = np.array([0.33, 0.33, 0.2]), np.array([1.0, 1.0, 0.7])
    pk = ProductKernel(kinds, per, fold=[True] * len(kinds))
    tab = pk.tables(fc, per, h, np.r_[ZA, ZB])
    A = torch.as_tensor(rank_coords(ZA, tab)).cuda(); B = torch.as_tensor(rank_coords(ZB, tab)).cuda()
    for mask in masks:
        out = torch.empty((len(ZA), len(ZB)), dtype=torch.float64, device='cuda')
        out_m = torch.empty_like(out)
        cols(A, B, tab, out, out_m=out_m, depmask=mask)
        assert np.abs(out.cpu().numpy() - c['joint']).max() <= 1e-13 * np.abs(c['joint']).max()
        marg = c[f'marg{mask}']
        assert np.abs(out_m.cpu().numpy() - marg).max() <= 1e-13 * np.abs(marg).max(), mask


def test_rows_plan_equals_rows(cuda_device):
    """The validated-once rows plan (the block coordinate descent's passes) gives blml_rows' sums, bit for bit, on
    the 5-D bins against a block of them and against all of them."""
    import ctypes as C
    from blml_b200.local_gpu import ProductKernel, rows_dev, rank_coords, dev_tab, _struct
    from blml_b200 import _lib
    from blml_b200._lib import call
    p = golden('pairs.npz')['p5']
    u, cnt = p['bins'], p['counts']
    pk = ProductKernel(['sinc'] * 5, [None] * 5)
    tab = pk.tables(p['fc'], [None] * 5, p['h'], u)
    Z = torch.as_tensor(rank_coords(u, tab)).cuda()
    B = Z.shape[0]
    st = torch.cuda.current_stream().cuda_stream
    plan = C.c_void_p()
    call('blml_rows_plan_create', _struct(tab, dev_tab(tab, 'cuda'), False, False), Z.data_ptr(), B, st, C.byref(plan))
    try:
        idx = torch.as_tensor(np.random.default_rng(1).permutation(B)[:257]).cuda()
        for ZB in (Z[idx].contiguous(), Z):
            w = torch.as_tensor(np.random.default_rng(2).standard_normal(ZB.shape[0])).cuda()
            ref = rows_dev(Z, ZB, w, tab)[0]
            ws = torch.empty(int(_lib.lib().blml_rows_plan_workspace(plan, B, ZB.shape[0])), dtype=torch.uint8,
                             device='cuda')
            out = torch.empty(B, dtype=torch.float64, device='cuda')
            call('blml_rows_plan_run', plan, Z.data_ptr(), B, ZB.data_ptr(), ZB.shape[0], w.data_ptr(), out.data_ptr(),
                 ws.data_ptr(), ws.numel(), st)
            assert torch.equal(out, ref)
    finally:
        _lib.lib().blml_rows_plan_destroy(plan)


@pytest.mark.parametrize('case', ['p5', 'pt'])
@pytest.mark.parametrize('f32', [False, True])
def test_rows_multi_matches_reference(cuda_device, case, f32):
    """The fused rows of several densities (blml_local.py:282-286, FusedFit's joint and marginals in one pass) against
    the reference's own values (tests/golden/rows_multi.npz): the 5-D sinc bins with two marginals, the pball torus
    group with a sinc column and each unit alone. float64 tables to 1e-12 of the largest row, float32 to 2e-4; and the
    joint density equals the single-density rows kernel."""
    from blml_b200.local_gpu import ProductKernel, rows_multi, rows
    g = golden('rows_multi.npz')[case]
    if case == 'p5':
        p = golden('pairs.npz')['p5']
        kinds, per, fc, h = ['sinc'] * 5, [None] * 5, p['fc'], p['h']
        tab = ProductKernel(kinds, per).tables(fc, per, h, g['ZB'])
    else:
        kinds, per = ['pball:0-1', 'pball:0-1', 'sinc'], [31.0, 31.0, None]
        fc, h = np.array([0.33, 0.33, 0.2]), np.array([1.0, 1.0, 0.7])
        tab = ProductKernel(kinds, per, fold=[True] * 3).tables(fc, per, h, np.r_[g['ZA'], g['ZB']])
    s, _ = rows_multi(g['ZA'], g['ZB'], g['W'], tab, g['umask'], f32=f32)
    ref = g['s']
    tol = 2e-4 if f32 else 1e-12
    assert s.shape == ref.shape
    assert np.abs(s - ref).max() <= tol * np.abs(ref).max(), np.abs(s - ref).max() / np.abs(ref).max()
    joint, _ = rows(g['ZA'], g['ZB'], g['W'][:, 0], tab, f32=f32)
    assert np.abs(joint - s[:, 0]).max() <= tol * np.abs(joint).max()
