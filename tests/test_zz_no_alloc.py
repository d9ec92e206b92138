"""blml_rows_noalloc, the pair-accumulation entry point that allocates nothing.

Some callers of this library cannot allocate device memory: processes whose device memory another allocator
reserves up front, and embedded hosts that forbid allocation after start-up. For them blml_rows_noalloc keeps its scratch in a fixed
device array inside the library. This test calls it through the C ABI and checks it against blml_rows on the same
inputs (the same deterministic arithmetic: equal to 1e-12 of the largest sum), on two calls in a row, since every
call reuses the one array. The file is named to run last."""
import numpy as np
import pytest
import torch

from conftest import golden

pytestmark = pytest.mark.gpu


def _noalloc(tab, ZA, ZB, w, f32=False):
    from blml_b200 import _lib
    from blml_b200.local_gpu import dev_tab, _struct
    t = dev_tab(tab, ZA.device)
    s = torch.full((ZA.shape[0],), float('nan'), dtype=torch.float64, device=ZA.device)
    st = _struct(tab, t, False, f32)
    _lib.call('blml_rows_noalloc', st, ZA.data_ptr(), ZA.shape[0], ZB.data_ptr(), ZB.shape[0], w.data_ptr(),
              s.data_ptr(), torch.cuda.current_stream().cuda_stream)
    return s


def _cases():
    from blml_b200.local_gpu import ProductKernel, rank_coords
    p = golden('pairs.npz')['p5']
    tab = ProductKernel(['sinc'] * 5).tables(p['fc'], [None] * 5, p['h'], p['bins'])
    u = torch.as_tensor(rank_coords(p['bins'], tab)).cuda()
    yield tab, u, u, torch.as_tensor(p['counts']).cuda()
    t = golden('pairs.npz')['pt']
    kinds, per = ['pball:0-1', 'pball:0-1', 'sinc'], [31.0, 31.0, None]
    tab2 = ProductKernel(kinds, per).tables([0.33, 0.33, 0.2], per, [1.0, 1.0, 0.7], np.r_[t['ZA'], t['ZB']])
    yield (tab2, torch.as_tensor(rank_coords(t['ZA'], tab2)).cuda(), torch.as_tensor(rank_coords(t['ZB'], tab2)).cuda(),
           torch.as_tensor(t['w']).cuda())


@pytest.mark.parametrize('f32', [False, True])
def test_rows_noalloc_equals_rows_twice(cuda_device, f32):
    from blml_b200.local_gpu import rows_dev
    for tab, A, B, w in _cases():
        ref, _ = rows_dev(A, B, w, tab, f32=f32)
        scale = ref.abs().max().item()
        for _ in range(2):                                   # the second call reuses the scratch the first left
            s = _noalloc(tab, A, B, w, f32=f32)
            torch.cuda.synchronize()
            assert (s - ref).abs().max().item() <= 1e-12 * scale


def test_rows_noalloc_rejects_rows_beyond_its_scratch(cuda_device):
    from blml_b200._lib import BLMLError
    from blml_b200.local_gpu import ProductKernel
    Z = np.array([[0, 0], [3, 4], [6, 1], [1, 1], [2, 5]], np.int64)
    tab = ProductKernel(['sinc', 'sinc']).tables([0.3, 0.3], [None, None], [1.0, 1.0], Z)
    big = torch.zeros((600_000, 2), dtype=torch.int64, device='cuda')
    with pytest.raises(BLMLError, match='fixed scratch'):
        _noalloc(tab, big, torch.as_tensor(Z).cuda(), torch.ones(5, dtype=torch.float64, device='cuda'))
