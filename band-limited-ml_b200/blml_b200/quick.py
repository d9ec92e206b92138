"""BLML on counts at occupied lattice bins (the fixed-lattice entry of BLMLQuick, rahuljhu/band-limited-ml
blml_trivial.py:2705-2732, 3516-3598, and its GPU solver blml_gpu.py:61-520), real rank 1, on one B200.

    q = BLMLQuickLattice(tol=1e-7, dtype=np.float32).fit(Zc, with_lattice(modes, h), sample_weight=w)
    q.e_hat_, q.density_ (f at the bins), q.loglik_

The bins are Zi = round(Zc / h) (round half to even in float64, on the GPU, bit-exact with np.round); bins with
zero weight are dropped; bin order is the caller's. The operator over the B occupied bins is S e = rows(Z, Z, e):
one pair-accumulation pass over the B^2 bin pairs from the kernel's value tables in shared memory -- the
reference's block-Jacobi sweep materialises B x 4096 Gram blocks and multiplies them with cuBLAS; here the block
never exists. The solver is the binned fit's Jacobi coordinate update with Anderson mixing and the merit safeguard
(convex for real rank 1, so it reaches the reference's optimum). State float32 or float64, pair products in the
tables' precision (f32 tables for float32, as the reference's GPU engine), every sum in float64."""
import numpy as np
import torch

from . import _lib
from ._lib import call
from .binned import BLMLBinned, _Red, _device
from .spec import parse_modes, modes_lattice
from .local_gpu import ProductKernel, rows_dev


def lattice_coords(Z, h, device=None):
    """Integer lattice coordinates round(Z / h) of bin centres (float64, round half to even) on the GPU."""
    device = torch.device(device or 'cuda')
    Zt = torch.as_tensor(np.ascontiguousarray(Z, np.float64)).to(device)
    ht = torch.as_tensor(np.ascontiguousarray(np.broadcast_to(np.asarray(h, float), (Zt.shape[1],)), np.float64)).to(device)
    out = torch.empty(Zt.shape, dtype=torch.int64, device=device)
    call('blml_lattice_coords', Zt.data_ptr(), Zt.shape[0], Zt.shape[1], ht.data_ptr(), out.data_ptr(),
         torch.cuda.current_stream(device).cuda_stream)
    return out


def bin_points(X, h, device=None):
    """Points to occupied bins: integer coordinates round(X / h) on the GPU, then the distinct rows in lexicographic
    order with their counts (the reference's np.unique(..., axis=0) order). Returns (bins (B, d) int64, counts (B,))."""
    Zi = lattice_coords(X, h, device)
    u, cnt = torch.unique(Zi, dim=0, return_counts=True)
    return u, cnt.to(torch.float64)


class BLMLQuickLattice(BLMLBinned):
    """Real rank-1 BLML on counts at occupied lattice bins (see the module docstring)."""

    def __init__(self, tol=1e-4, max_sweeps=None, anderson=5, dtype=np.float32, seed=0, verbose=False, stall=1000,
                 device=None):
        super().__init__(tol=tol, max_sweeps=max_sweeps, anderson=anderson, dtype=dtype, seed=seed, verbose=verbose,
                         stall=stall, device=device)

    def fit(self, X, modes, sample_weight=None, init=None):
        Xn = X.detach().cpu().numpy() if isinstance(X, torch.Tensor) else np.asarray(X, np.float64)
        Xn = np.atleast_2d(Xn)
        d = Xn.shape[1]
        h = modes_lattice(modes, d)
        if h is None:
            raise ValueError("BLMLQuickLattice fits counts on a fixed lattice: give modes with_lattice(modes, h)")
        w = np.ones(len(Xn)) if sample_weight is None else np.asarray(sample_weight, float)
        if w.shape != (len(Xn),) or not np.all(w >= 0):
            raise ValueError("sample_weight: (n,) non-negative counts")
        specs, dep = parse_modes(modes, d)
        if dep is not None or len(specs) != 1:
            raise ValueError("BLMLQuickLattice: one real mode (rank 1) without dep columns")
        self.dev_ = _device(self.device)
        keep = w > 0
        Zi = lattice_coords(Xn[keep], h, self.dev_)
        self.Zi_t_ = Zi; self.h_ = h; self.specs_ = specs; self.d_ = d
        self.n_ = float(w[keep].sum())
        if not self.n_ > 0:
            raise ValueError("sample_weight: no observations")
        f32 = self.dtype == np.float32
        self._code = _lib.F32 if f32 else _lib.F64
        self.rdt_ = np.float32 if f32 else np.float64
        self._rt = torch.float32 if f32 else torch.float64
        self._ct = torch.complex64 if f32 else torch.complex128
        self._red = _Red(self.dev_)
        B = Zi.shape[0]
        self.B_ = B; self.shape_ = (B,); self.K_ = 1
        sp = specs[0]
        self.pk_ = ProductKernel(sp['kinds'], sp['periods'])
        Zh = Zi.cpu().numpy()
        self.tab_ = self.pk_.tables(sp['fc'], sp['periods'], h, Zh)
        from .local_gpu import rank_coords
        self._Z = torch.as_tensor(rank_coords(Zh, self.tab_)).to(self.dev_)
        self.s_ = np.array([self.pk_.k0(sp['fc'], sp['periods'])[1]])
        self.shared_ = True
        self.w_t_ = torch.as_tensor(w[keep], dtype=self._rt).to(self.dev_)
        self.c_t_ = self._lin([(self.n_, self.w_t_)])
        self.sg_t_ = torch.ones(B, dtype=self._rt, device=self.dev_)
        self.complex_g_ = False; self.psd_ = False
        if init is not None and getattr(init, 'e_hat_t_', None) is not None and init.B_ == B:
            E = init.e_hat_t_.to(self._rt).reshape(1, B).clone()
        else:
            E = torch.empty((1, B), dtype=self._rt, device=self.dev_)
            call('blml_start_root', self._code, B, self.c_t_.data_ptr(), self.sg_t_.data_ptr(), float(self.s_[0]),
                 E.data_ptr(), self._st)
        E, U = self._solve_cd(E, self.max_sweeps)
        # the solution's S e exactly (the solver's U is exact already: every U comes from a full pass)
        self._finish(E, U)
        return self

    def _Sall(self, E, out=None):
        """S E over the occupied bins: one pass of the pair kernel (float64 sums)."""
        w = E[0].to(torch.float64).contiguous()
        s, _ = rows_dev(self._Z, self._Z, w, self.tab_, grad=False, f32=self._code == _lib.F32)
        out = torch.empty_like(E) if out is None else out
        out[0].copy_(s.to(out.dtype))
        return out

    def _plan64(self):
        raise NotImplementedError("certificate on occupied bins: use a full-lattice fit")
