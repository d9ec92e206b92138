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
from ._lib import call, ptrs, dbl
from .binned import BLMLBinned, _Red, _device, point_cols
from .spec import parse_modes, modes_lattice, with_lattice, split_kind
from .local_gpu import ProductKernel, rows_dev, dev_tab, _struct


def lattice_coords(Z, h, device=None):
    """Integer lattice coordinates round(Z / h) of bin centres (float64, round half to even) on the GPU."""
    device = torch.device(device or 'cuda')
    Zt = torch.as_tensor(np.ascontiguousarray(Z, np.float64)).to(device)
    ht = torch.as_tensor(np.array(np.broadcast_to(np.asarray(h, float), (Zt.shape[1],)), np.float64)).to(device)
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
                 device=None, solver='jacobi'):
        super().__init__(tol=tol, max_sweeps=max_sweeps, anderson=anderson, dtype=dtype, seed=seed, verbose=verbose,
                         stall=stall, device=device)
        if solver not in ('block', 'jacobi'):
            raise ValueError("solver: 'block' (block coordinate descent) or 'jacobi' (Jacobi updates with Anderson)")
        self.cd_solver = solver

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
        if self.cd_solver == 'block':
            E, U = self._solve_block_cd(E, self.max_sweeps)
        else:
            E, U = self._solve_cd(E, self.max_sweeps)
        self._finish(E, U)
        return self

    def _solve_block_cd(self, E, max_sweeps):
        """Block coordinate descent (blml_trivial.py:2860-3035) from E: each sweep visits the bins in a seeded random
        order, in blocks of min(1024, max(32, B / 64)) bins; a block takes its coordinates' exact roots together and
        S e follows by one rows pass of every bin against the block (B x block pairs), so a sweep costs one full pass
        in total. Plain sweeps until one raises Phi = e'Se / 2 - sum c log e; that sweep is redone with the block
        safeguard (the largest t in 2^-k that does not raise Phi along the block's step), which stays on. Stops at
        max|rho| < tol (S e then recomputed exactly and the test repeated), or when the residual improved by less
        than 1% over 50 sweeps. State e and S e in float64, pair products in the tables' precision."""
        B, dev, n, st = self.B_, self.dev_, self.n_, self._st
        f32 = self._code == _lib.F32
        Bs = min(1024, max(32, B // 64), B)
        c64 = self.c_t_.to(torch.float64).contiguous()
        sg64 = torch.ones(B, dtype=torch.float64, device=dev)
        sbb = float(self.s_[0])
        red = self._red
        D = self._Z.shape[1]
        d = torch.empty(Bs, dtype=torch.float64, device=dev)
        Zb = torch.empty((Bs, D), dtype=torch.int64, device=dev)
        q = torch.empty(65, dtype=torch.float64, device=dev)
        v = torch.empty(B, dtype=torch.float64, device=dev)
        steps = 0.5 ** np.arange(31)
        rng = np.random.default_rng(self.seed)
        # every pass is bins against bins of the same coordinate set: the tables and extents are checked once here,
        # and the passes run with no host synchronisation or allocation
        import ctypes as C
        tstruct = _struct(self.tab_, dev_tab(self.tab_, dev), False, f32)
        rplan = C.c_void_p()
        call('blml_rows_plan_create', tstruct, self._Z.data_ptr(), B, st, C.byref(rplan))
        wsb = max(int(_lib.lib().blml_rows_plan_workspace(rplan, B, Bs)),
                  int(_lib.lib().blml_rows_plan_workspace(rplan, B, B)))
        rws = torch.empty(max(wsb, 8), dtype=torch.uint8, device=dev)

        def pass_rows(ZB, M, w, out):
            call('blml_rows_plan_run', rplan, self._Z.data_ptr(), B, ZB.data_ptr(), M, w.data_ptr(), out.data_ptr(),
                 rws.data_ptr(), rws.numel(), st)
            return out

        def exact_Se(e):
            return pass_rows(self._Z, B, e, torch.empty(B, dtype=torch.float64, device=dev))

        def phi(e, Se):
            call('blml_merit_terms', _lib.F64, 1, B, 0, 0, e.data_ptr(), Se.data_ptr(), c64.data_ptr(),
                 sg64.data_ptr(), red.part.data_ptr(), red.out.data_ptr(), st)
            a, b, _ = red.read(3)
            return (0.5 * a - b) / n

        def resid(e, Se):
            call('blml_resid', _lib.F64, 1, B, 0, e.data_ptr(), Se.data_ptr(), c64.data_ptr(), 1.0,
                 red.part.data_ptr(), red.out.data_ptr(), st)
            mx, nnan = red.read(2)
            return float('nan') if nnan > 0 else mx

        def sweep(e, Se, safeguard):
            perm = torch.as_tensor(rng.permutation(B)).to(dev)
            for s0 in range(0, B, Bs):
                I = perm[s0:s0 + Bs]
                m = int(I.numel())
                call('blml_block_root', m, I.data_ptr(), B, e.data_ptr(), Se.data_ptr(), c64.data_ptr(), sbb,
                     d.data_ptr(), st)
                call('blml_gather_rows_i64', m, D, self._Z.data_ptr(), I.data_ptr(), B, Zb.data_ptr(), st)
                pass_rows(Zb, m, d, v)
                t = 1.0
                if safeguard:
                    call('blml_block_search', m, I.data_ptr(), B, e.data_ptr(), d.data_ptr(), Se.data_ptr(),
                         v.data_ptr(), c64.data_ptr(), q.data_ptr(), st)
                    r = q.cpu().numpy()
                    lin, quad, npos, logs, bad = r[0], r[1], r[2], r[3:34], r[34:65]
                    if npos > 0:
                        ok = (steps * lin + 0.5 * steps ** 2 * quad - logs <= 0) & (bad == 0)
                        t = float(steps[np.argmax(ok)]) if ok.any() else 0.0
                if t != 0.0:
                    call('blml_block_apply', m, I.data_ptr(), B, d.data_ptr(), float(t), e.data_ptr(), st)
                    call('blml_lincomb', _lib.F64, B, Se.data_ptr(), 2, dbl([1.0, t]), ptrs([Se, v]), st)

        e = E[0].to(torch.float64).contiguous().clone()
        Se = exact_Se(e)
        safeguard = False
        obj_prev = phi(e, Se)
        hist, it, conv = [], 0, False
        res = resid(e, Se)
        self.stop_reason_ = 'stall'
        while True:
            if max_sweeps is not None and it >= max_sweeps:
                self.stop_reason_ = 'max_sweeps'
                break
            it += 1
            e_save, Se_save = e.clone(), Se.clone()
            sweep(e, Se, safeguard)
            obj_now = phi(e, Se)
            if not safeguard and obj_now > obj_prev + 1e-10 * abs(obj_prev):
                e, Se = e_save, Se_save
                safeguard = True
                sweep(e, Se, True)
                obj_now = phi(e, Se)
            obj_prev = obj_now
            res = resid(e, Se)
            if not np.isfinite(res):
                hist.append(np.inf)
                self.stop_reason_ = 'nan'
                break
            if res < self.tol:
                Se = exact_Se(e)
                res = resid(e, Se)
            hist.append(res)
            if self.verbose:
                print(f'  block sweep {it}: max|rho| {res:.2e} Phi/n {obj_now:.8f}', flush=True)
            if res < self.tol:
                conv = True
                self.stop_reason_ = 'tol'
                break
            if len(hist) > 50 and hist[-1] > 0.99 * min(hist[:-50]):
                break
        if not conv and max_sweeps is not None and np.isfinite(res):       # capped: normalise exactly
            Se = exact_Se(e)
            call('blml_dots', _lib.F64, B, 1, ptrs([e]), ptrs([Se]), red.part.data_ptr(), red.out.data_ptr(), st)
            ee = red.read(1)[0]
            sc = n / np.sqrt(max(ee, 1e-300))
            call('blml_lincomb', _lib.F64, B, e.data_ptr(), 1, dbl([sc]), ptrs([e]), st)
            call('blml_lincomb', _lib.F64, B, Se.data_ptr(), 1, dbl([sc]), ptrs([Se]), st)
            res = resid(e, Se)
            conv = res < self.tol
            hist.append(res)
        _lib.lib().blml_rows_plan_destroy(rplan)
        self.n_sweeps_, self.residual_, self.converged_ = it, res, conv
        self.rho_history_ = hist
        self.safeguard_ = safeguard
        return e.to(self._rt).reshape(1, B).contiguous(), Se.to(self._rt).reshape(1, B).contiguous()

    def _Sall(self, E, out=None):
        """S E over the occupied bins: one pass of the pair kernel (float64 sums)."""
        w = E[0].to(torch.float64).contiguous()
        s, _ = rows_dev(self._Z, self._Z, w, self.tab_, grad=False, f32=self._code == _lib.F32)
        out = torch.empty_like(E) if out is None else out
        out[0].copy_(s.to(out.dtype))
        return out

    def _plan64(self):
        raise NotImplementedError("certificate on occupied bins: use a full-lattice fit")


# ---------------------------------------------------------------------------------------------------- points path
def lattice_steps(kinds, periods, h_target):
    """The lattice steps for target widths (blml_kernels.py:57-68, the kernel classes' step rules,
    blml_trivial.py:399-400, 556-561): a dirichlet column (and a pball group's columns) tiles its period with whole
    bins, at least 8; every other column keeps its target width. Radial groups take their columns' finest target
    (lattice_target, blml_trivial.py:1333-1341)."""
    h_t = np.array(h_target, float)
    groups = {}
    for j, k in enumerate(kinds):
        if split_kind(k)[0] in ('ball', 'pball'):
            groups.setdefault(split_kind(k)[1], []).append(j)
    for dims in groups.values():
        h_t[dims] = h_t[dims].min()
    h = np.empty(len(kinds))
    for j, k in enumerate(kinds):
        if split_kind(k)[0] in ('dirichlet', 'pball'):
            P = float(periods[j])
            h[j] = P / max(8, int(np.ceil(P / h_t[j] - 1e-9)))
        else:
            h[j] = float(h_t[j])
    return h


def quantize_points(X, kinds, periods, h):
    """Bin centres of the points (blml_kernels.py:74-82; blml_trivial.py:402-403, 563-567): round(x / h) h, a periodic
    column wrapped into [0, P) first; -0.0 becomes +0.0 (bins are unique by their bytes)."""
    X = np.atleast_2d(np.asarray(X, float))
    Xq = np.empty_like(X)
    for j, k in enumerate(kinds):
        if split_kind(k)[0] in ('dirichlet', 'pball'):
            P = float(periods[j])
            Xq[:, j] = np.mod(np.round(np.mod(X[:, j], P) / h[j]) * h[j], P)
        else:
            Xq[:, j] = np.round(X[:, j] / h[j]) * h[j]
    return Xq + 0.0


def unique_bins(Xq, sample_weight=None):
    """The occupied bins in the reference's order (np.unique over each row's raw bytes, blml_trivial.py:2760-2765),
    their weights (counts, or the points' total weight) and each point's bin."""
    Xc = np.ascontiguousarray(Xq)
    vdt = np.dtype((np.void, Xc.dtype.itemsize * Xc.shape[1]))
    _, idx, inv, counts = np.unique(Xc.view(vdt), return_index=True, return_inverse=True, return_counts=True)
    inv = np.ravel(inv)
    w = counts.astype(float) if sample_weight is None else np.bincount(inv, weights=sample_weight, minlength=len(idx))
    return Xq[idx], w, inv




class BLMLQuick(BLMLQuickLattice):
    """The reference's BLMLQuick (engine='gpu', blml_trivial.py:2684-2800), real rank 1: points are snapped to a
    lattice of steps bin_scale n^-1/4 / fc (a periodic column tiled by whole bins), binned in the reference's order,
    and fitted as counts on the occupied bins by the pair operator of BLMLQuickLattice with the reference's block
    coordinate descent (_solve_block_cd); modes with h (with_lattice) are counts on that fixed lattice. predict / sqrt_density evaluate the exact kernel at any points on the GPU
    (blml_point_rows: sinc, slits and dirichlet columns)."""

    def __init__(self, tol=1e-4, batch_size=2000, seed=0, verbose=False, dtype=np.float32, bin_scale=0.1,
                 max_sweeps=None, engine='gpu', solver='cd', lbfgs_m=20, device=None):
        if solver not in ('cd', 'lbfgs'):
            raise ValueError("solver: 'cd' (block coordinate descent with Anderson mixing) or 'lbfgs'")
        if engine not in ('cpu', 'gpu'):
            raise ValueError(f"engine {engine!r}: 'cpu' or 'gpu'")
        super().__init__(tol=tol, max_sweeps=max_sweeps, dtype=dtype, seed=seed, verbose=verbose, device=device,
                         solver='block')
        self.batch_size, self.bin_scale, self.engine = batch_size, bin_scale, engine
        self.solver, self.lbfgs_m = solver, int(lbfgs_m)

    def fit(self, X, modes, init=None, rebin_tol=1.0, signs=None, complex_g=False, sample_weight=None):
        X = np.atleast_2d(np.asarray(X.detach().cpu().numpy() if isinstance(X, torch.Tensor) else X, np.float64))
        n_rows, d = X.shape
        if complex_g or signs is not None or init is not None:
            raise NotImplementedError("BLMLQuick on the GPU: real rank-1 fits without signs or warm starts")
        h_fixed = modes_lattice(modes, d)
        if h_fixed is not None:                           # counts on a fixed lattice: the occupied bins as given
            BLMLQuickLattice.fit(self, X, modes, sample_weight=sample_weight)
            keep = np.ones(n_rows, bool) if sample_weight is None else np.asarray(sample_weight, float) > 0
            self.Z_, self._h_vec = X[keep], np.asarray(h_fixed, float)
            self.n_bins_, self.dim_, self.n_samples_ = int(keep.sum()), d, self.n_
            self._pt_cols = None
            return self
        sw = None if sample_weight is None else np.asarray(sample_weight, np.float64)
        if sw is not None and (sw.shape != (n_rows,) or not np.all(sw > 0)):
            raise ValueError("sample_weight: (n,) positive weights")
        n = float(n_rows) if sw is None else float(sw.sum())
        specs, dep = parse_modes(modes, d)
        if dep is not None or len(specs) != 1:
            raise NotImplementedError("BLMLQuick on the GPU: one real mode (rank 1) without dep columns")
        sp = specs[0]
        h = lattice_steps(sp['kinds'], sp['periods'], self.bin_scale * n ** -0.25 / np.asarray(sp['fc'], float))
        Z, w, inv = unique_bins(quantize_points(X, sp['kinds'], sp['periods'], h), sw)
        BLMLQuickLattice.fit(self, Z, with_lattice(modes, h), sample_weight=w)
        self.Z_, self.w_pts_, self._h_vec, self.n_samples_ = Z, w, h, n
        self.n_bins_, self.dim_ = len(Z), d
        self._pt_cols = None
        return self

    # ---------------------------------------------------------------- at arbitrary points
    def _point_cols(self):
        if self._pt_cols is None:
            cols = point_cols(self.specs_[0], self.d_)
            self._pt_cols = cols
        return self._pt_cols

    def sqrt_density(self, Xq):
        """g(x) = (1/n) sum_b e_b K(x - z_b) at the points Xq, the exact kernel (blml_trivial.py:3307-3320)."""
        if getattr(self, 'Z_', None) is None:
            raise RuntimeError("Call fit() before sqrt_density().")
        Xq = np.asarray(Xq, float)
        Xq = Xq[:, None] if Xq.ndim == 1 else Xq
        if Xq.shape[1] != self.d_:
            raise ValueError(f"points: {self.d_} columns")
        dev = self.dev_
        Xt = torch.as_tensor(np.ascontiguousarray(Xq)).to(dev)
        Zt = torch.as_tensor(np.ascontiguousarray(self.Z_, np.float64)).to(dev)
        e = self.e_hat_t_[0].to(torch.float64).contiguous()
        g = torch.empty(len(Xq), dtype=torch.float64, device=dev)
        import ctypes as C
        call('blml_point_rows', len(Xq), self.d_, Xt.data_ptr(), len(self.Z_), Zt.data_ptr(), e.data_ptr(),
             C.cast(self._point_cols(), C.c_void_p), g.data_ptr(), self._st)
        return g.cpu().numpy() / self.n_samples_

    def predict(self, Xq):
        """f(x) = g(x)^2 at the points Xq (blml_trivial.py:3288-3305)."""
        return self.sqrt_density(Xq) ** 2
