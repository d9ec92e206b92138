"""The complex64-history scan (blml_seg_dots2_h32: the certified rounds' L-BFGS history products, the quantities the
reference reads pair by pair at blml_binned.py:297-313) against float64 sums of the same stored values on the host.
Its blocks are shared out among the fits in proportion to their sizes (a split computed on the device), so the cases
cover what that split must get right: an empty fit (B = 0), fits smaller than one 128-element tile, sizes that are not
multiples of a tile, fits hundreds of times larger than the others, one fit alone, more fits than the split has
blocks to share, fewer than 20 stored vectors and no third vector."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _scan(dev, B, K, np_, with_x, seed):
    import torch
    from blml_b200 import _lib
    from blml_b200._lib import call, ptrs
    from blml_b200.sweep import _Seg
    rng = np.random.default_rng(seed)
    B = np.asarray(B, np.int64)
    F = len(B)
    n_f = K * B
    off = np.concatenate([[0], np.cumsum(n_f)])
    boff = np.concatenate([[0], np.cumsum(B)])
    segs = (_Seg * F)(*[_Seg(int(off[f]), int(boff[f]), int(B[f]), int(K[f]), 0) for f in range(F)])
    st_t = torch.frombuffer(bytearray(segs), dtype=torch.uint8).to(dev)
    n = max(int(off[-1]), 1)

    def c64():
        return (rng.standard_normal(n) + 1j * rng.standard_normal(n)).astype(np.complex64)

    def c128():
        return rng.standard_normal(n) + 1j * rng.standard_normal(n)
    a = [c64() for _ in range(np_)]
    b0, b1, x = c64(), c128(), c128()
    da = [torch.from_numpy(v).to(dev) for v in a]
    db0, db1, dx = (torch.from_numpy(v).to(dev) for v in (b0, b1, x))
    part = torch.full((43 * (_lib.SEG_SPLIT_BLOCKS + F),), np.nan, dtype=torch.float64, device=dev)
    split = torch.empty(int(_lib.lib().blml_seg_split_ints(F)), dtype=torch.int32, device=dev)
    out = torch.full((F * (2 * np_ + 3),), np.nan, dtype=torch.float64, device=dev)
    st = torch.cuda.current_stream(dev).cuda_stream
    call('blml_seg_dots2_h32', F, st_t.data_ptr(), split.data_ptr(), np_, ptrs(da), db0.data_ptr(), db1.data_ptr(),
         dx.data_ptr() if with_x else C.c_void_p(0), part.data_ptr(), out.data_ptr(), st)
    torch.cuda.synchronize(dev)
    _check_split(split.cpu().numpy(), n_f)
    got = out.cpu().numpy().reshape(F, 2 * np_ + 3)

    def rdot(u, v):                         # Re(conj(u) v) summed in float64: the scan's real inner product
        u = u.astype(np.complex128)
        return float(np.sum(u.real * v.real + u.imag * v.imag))
    want = np.zeros_like(got)
    for f in range(F):
        s = slice(int(off[f]), int(off[f + 1]))
        y0 = b0[s].astype(np.complex128)
        for q in range(np_):
            want[f, q] = rdot(a[q][s], y0)
            want[f, np_ + q] = rdot(a[q][s], b1[s])
        want[f, 2 * np_] = rdot(y0, y0)
        want[f, 2 * np_ + 1] = rdot(b1[s], b1[s])
        want[f, 2 * np_ + 2] = rdot(x[s], x[s]) if with_x else 0.0
    return got, want, n_f


def _check_split(split, n_f):
    """The device's block split against its rule: fit f gets min(ceil(G n_f / N), ceil(n_f / 1024)) of the G blocks
    (none without elements), bstart is their exclusive prefix sum and fit_of names each block's fit (-1 past the
    last); integer work, so exact."""
    from blml_b200 import _lib
    G, F = _lib.SEG_SPLIT_BLOCKS, len(n_f)
    N = int(n_f.sum())
    nb = np.array([0 if n == 0 else min(-(-G * int(n) // N), -(-int(n) // 1024)) for n in n_f], np.int64)
    bstart = np.concatenate([[0], np.cumsum(nb)])
    fit_of = np.full(G + F, -1, np.int64)
    fit_of[:bstart[-1]] = np.repeat(np.arange(F), nb)
    assert len(split) == 2 * F + 1 + G
    np.testing.assert_array_equal(split[:F + 1], bstart)
    np.testing.assert_array_equal(split[F + 1:], fit_of)


CASES = {
    # the sweep's spread: small and large lattices, one empty fit, ragged sizes
    'mixed': ([4096, 0, 147456, 37, 1, 9000, 128, 129, 65536, 4097], [4, 2, 4, 1, 3, 2, 1, 1, 2, 4], 20, True),
    'one_fit': ([300001], [1], 20, True),
    'tiny_only': ([1, 2, 127, 128, 5], [1, 1, 1, 1, 3], 7, False),
    # more fits than the split's 2048 blocks: every fit with work still gets one
    'many_fits': (list(np.random.default_rng(3).integers(0, 600, 2500)), [1] * 2500, 3, True),
}


@pytest.mark.parametrize('case', sorted(CASES))
def test_history_scan_matches_host_sums(cuda_device, case):
    B, K, np_, with_x = CASES[case]
    got, want, n_f = _scan(cuda_device, B, np.asarray(K, np.int64), np_, with_x, seed=len(B))
    assert np.all(np.isfinite(got))
    # float64 sums of up to ~6e5 products in another order: a few 1e-16 relative to the sum of |products|
    scale = np.maximum(np.abs(want), np.sqrt(np.maximum(n_f, 1))[:, None])
    err = np.abs(got - want) / scale
    assert err.max() < 1e-12, (case, err.max())
    assert np.all(got[n_f == 0] == 0.0)


def _lincomb(dev, B, K, nt, f32mask, out_f32, inplace, seed):
    import torch
    from blml_b200 import _lib
    from blml_b200._lib import call, ptrs
    from blml_b200.sweep import _Seg
    rng = np.random.default_rng(seed)
    B = np.asarray(B, np.int64)
    F = len(B)
    n_f = K * B
    off = np.concatenate([[0], np.cumsum(n_f)])
    boff = np.concatenate([[0], np.cumsum(B)])
    segs = (_Seg * F)(*[_Seg(int(off[f]), int(boff[f]), int(B[f]), int(K[f]), 0) for f in range(F)])
    st_t = torch.frombuffer(bytearray(segs), dtype=torch.uint8).to(dev)
    n = max(int(off[-1]), 1)
    is32 = [bool((f32mask >> q) & 1) for q in range(nt)]
    v = [(rng.standard_normal(n) + 1j * rng.standard_normal(n)).astype(np.complex64 if w else np.complex128)
         for w in is32]
    coef = rng.standard_normal((F, nt))
    coef[rng.random((F, nt)) < 0.2] = 0.0                # skipped terms
    dv = [torch.from_numpy(x).to(dev) for x in v]
    if inplace:                                          # out is the last term (complex64 when out_f32)
        assert is32[-1] == out_f32
        dout = dv[-1]
    else:
        dout = torch.full((n,), np.nan, dtype=torch.complex64 if out_f32 else torch.complex128, device=dev)
    split = torch.empty(int(_lib.lib().blml_seg_split_ints(F)), dtype=torch.int32, device=dev)
    dcoef = torch.from_numpy(coef.ravel()).to(dev)
    st = torch.cuda.current_stream(dev).cuda_stream
    call('blml_seg_lincomb_h32', F, st_t.data_ptr(), split.data_ptr(), dout.data_ptr(), int(out_f32), nt,
         dcoef.data_ptr(), ptrs(dv), f32mask, st)
    torch.cuda.synchronize(dev)
    got = dout.cpu().numpy().astype(np.complex128)
    want = np.zeros(n, np.complex128)
    for f in range(F):
        s = slice(int(off[f]), int(off[f + 1]))
        for q in range(nt):
            want[s] += coef[f, q] * v[q][s].astype(np.complex128)
    scale = sum(np.abs(x.astype(np.complex128)) for x in v) * np.abs(coef).max() + 1e-300
    return got[:int(off[-1])], want[:int(off[-1])], scale[:int(off[-1])]


LINCOMB = {
    # the direction: one complex128 gradient and 40 complex64 history vectors into complex128
    'direction': ('mixed', 41, ((1 << 40) - 1) << 1, False, False),
    # the history update in place: complex128 q and the complex64 slot itself into that slot
    'slot_inplace': ('mixed', 2, 0b10, True, True),
    # complex128 terms after complex64 ones in the term list
    'interleaved': ('tiny_only', 6, 0b010101, False, False),
    'many_fits': ('many_fits', 5, 0b11110, False, False),
}


@pytest.mark.parametrize('case', sorted(LINCOMB))
def test_history_lincomb_matches_host_sums(cuda_device, case):
    geo, nt, mask, out_f32, inplace = LINCOMB[case]
    B, K, _, _ = CASES[geo]
    got, want, scale = _lincomb(cuda_device, B, np.asarray(K, np.int64), nt, mask, out_f32, inplace, seed=nt)
    err = np.abs(got - want) / scale
    # float64 sums of nt terms (complex64 output rounds to float32: 2^-24 of the terms' scale)
    assert err.max() < (1e-7 if out_f32 else 1e-14), (case, err.max())
