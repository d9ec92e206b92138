"""BLMLBinned on one B200: the reference's binned fit (rahuljhu/band-limited-ml, blml_binned.py:104-645) with every
array operation on the GPU through libblml_b200 (restricted-transform mat-vecs, fused bin-wise kernels, float64
deterministic reductions). The host runs the solver's control flow and reads back only the scalars it branches on.

    m = BLMLBinned(tol=1e-6, solver='lbfgs', dtype=np.float32).fit(counts, modes, complex_g=True)
    m.density_, m.Se_, m.e_hat_, m.loglik_, m.certificate()

Same constructor keywords, fit signature, attributes, stop reasons and errors as the reference. Differences, by
design: the L-BFGS direction uses the compact (Byrd-Nocedal-Schnabel) form of the two-loop recursion (one pass over
the history instead of 2m sequential dots); line-search trials update U = S E linearly (U + t S q) and the gradient
is formed only at the accepted point; bin-wise arithmetic is float64 internally for both storage types. Arrays
(density_, e_hat_, Se_) are NumPy on the host, read back from the device on first access; the device copies are
density_t_, e_hat_t_, Se_t_ (torch)."""
import numpy as np
import torch

from . import _lib
from ._lib import call, ptrs, dbl
from .spec import parse_modes, spec_key, units_of
from .operator import pad_rule, mode_transform, mode_transform_dlog, kernel_at_zero, Plan


from collections import OrderedDict

_PLANS = OrderedDict()            # (kernel spec, lattice, h, dtype, engine, device) -> (Plan, K(0), transform)
_PLAN_CACHE_SIZE = 128


def _device(dev):
    if not torch.cuda.is_available():
        raise _lib.BLMLError('BLMLBinned needs a CUDA device (this engine has no CPU path)')
    return torch.device(dev if dev is not None else 'cuda')


class _Red:
    """Reduction workspace (block partials) and the device results of one fit."""

    def __init__(self, device):
        nb = _lib.lib().blml_reduce_blocks()
        self.part = torch.empty(64 * nb, dtype=torch.float64, device=device)
        self.out = torch.empty(64, dtype=torch.float64, device=device)
        self.host = torch.empty(64, dtype=torch.float64, pin_memory=True)

    def read(self, nq):
        self.host[:nq].copy_(self.out[:nq], non_blocking=True)
        torch.cuda.current_stream(self.out.device).synchronize()
        return self.host[:nq].tolist()


def point_cols(sp, d):
    """One mode's kernel as blml_point_col per column (include/blml_b200.h): sinc, slits and dirichlet columns, and
    ball groups (blml_trivial.py:580-591: prod fc p(||fc t||), p(0) the unit ball's volume pi^(D/2) (1/2)^D /
    Gamma(D/2 + 1), :135-143). Other kinds raise NotImplementedError."""
    from math import gamma, pi
    from .spec import split_kind, dirichlet_N, dirichlet_inner_M
    cols = (_lib.PointCol * d)()
    for kind, dims in units_of(sp['kinds']):
        name, tag = split_kind(kind)
        if name == 'ball':
            mask = sum(1 << j for j in dims)
            for j in dims:
                c = cols[j]
                c.kind, c.M, c.f, c.fi = _lib.PT_BALL, mask, float(sp['fc'][j]), 0.0
            lead, D = cols[min(dims)], len(dims)
            lead.fi = float(np.prod([float(sp['fc'][j]) for j in dims])); lead.Mi = D
            lead.P = pi ** (D / 2) * 0.5 ** D / gamma(D / 2 + 1)
            continue
        if name not in ('sinc', 'slits', 'dirichlet'):
            raise NotImplementedError(f"kernel at arbitrary points: kind {name!r} (sinc, slits, dirichlet, ball)")
        c = cols[dims[0]]
        c.kind = {'sinc': _lib.PT_SINC, 'slits': _lib.PT_SLITS, 'dirichlet': _lib.PT_DIRICHLET}[name]
        c.f = float(sp['fc'][dims[0]])
        if name == 'slits':
            c.fi = (1.0 - float(tag)) * c.f
        if name == 'dirichlet':
            c.P = float(sp['periods'][dims[0]]); c.M = 2 * dirichlet_N(c.f, c.P) + 1
            c.Mi = dirichlet_inner_M(c.f, c.P, float(tag) if tag else None)
    return cols


class BLMLBinned:
    """BLML on counts on a full regular lattice, fitted on the GPU (see the module docstring)."""

    def __init__(self, tol=1e-5, max_sweeps=None, anderson=5, engine='gpu', dtype=np.float64, phase_noise=0.1,
                 seed=0, workers=-1, verbose=False, stall=1000, ll_tol=None, ll_window=100, solver='cd', lbfgs_m=20,
                 device=None, matvec_engine='simt', matvec_route=0):
        if solver not in ('cd', 'lbfgs'):
            raise ValueError("solver: 'cd' (coordinate / Jacobi updates with Anderson mixing) or 'lbfgs'")
        if int(lbfgs_m) > 20:
            raise ValueError("lbfgs_m: at most 20 pairs (the history dots run in one 64-wide pass)")
        self.solver, self.lbfgs_m = solver, int(lbfgs_m)
        self.tol, self.max_sweeps, self.anderson = tol, max_sweeps, anderson
        self.engine, self.dtype, self.phase_noise, self.seed = engine, np.dtype(dtype), phase_noise, seed
        if self.dtype not in (np.float32, np.float64):
            raise ValueError("dtype: float64 or float32")
        self.workers, self.verbose, self.stall = workers, verbose, stall
        self.ll_tol, self.ll_window = ll_tol, ll_window
        self.device = device
        if matvec_engine not in ('simt', 'tc'):
            raise ValueError("matvec_engine: 'simt' or 'tc' (tcgen05, float32 only)")
        if matvec_engine == 'tc' and self.dtype != np.float32:
            raise ValueError("matvec_engine='tc' stores float32: use dtype=np.float32")
        self.matvec_engine = matvec_engine
        if matvec_route not in (_lib.ROUTE_AUTO, _lib.ROUTE_CONTRACT, _lib.ROUTE_FFT):
            raise ValueError("matvec_route: 0 (auto: FFTs where the kernel is a DFT mask), 1 (restricted transforms) "
                             "or 2 (FFTs)")
        self.matvec_route = matvec_route

    # ---------------------------------------------------------------- setup
    def _setup(self, counts, modes, h, origin):
        if isinstance(counts, torch.Tensor) and counts.is_cuda:
            # counts already in device memory: validated and cast there (one host read of the verdict)
            if counts.ndim < 1 or bool(((counts < 0) | ~torch.isfinite(counts)).any()):
                raise ValueError("counts: a non-negative finite array on the lattice, one axis per dimension")
            self.device = counts.device if self.device is None else self.device
        else:
            if isinstance(counts, torch.Tensor):
                counts = counts.detach().numpy()
            counts = np.asarray(counts.get() if hasattr(counts, 'get') else counts)
            if counts.ndim < 1 or np.any(counts < 0) or not np.all(np.isfinite(counts)):
                raise ValueError("counts: a non-negative finite array on the lattice, one axis per dimension")
        d = counts.ndim; shape = tuple(counts.shape)
        specs, dep = parse_modes(modes, d)
        if dep is not None:
            raise ValueError("BLMLBinned: conditional (dep) modes are not supported; fit the joint")
        self.h_ = np.broadcast_to(np.asarray(h, float), (d,)).copy()
        self.origin_ = np.broadcast_to(np.asarray(origin, float), (d,)).copy()
        self.pad_ = pad_rule(shape, self.h_, specs)
        self.shape_ = shape; self.d_ = d; self.specs_ = specs; self.modes_ = modes
        self.B_ = int(np.prod(shape))
        self.dev_ = _device(self.device)
        f32 = self.dtype == np.float32
        self._code = _lib.F32 if f32 else _lib.F64
        self.rdt_ = np.float32 if f32 else np.float64
        self.cdt_ = np.complex64 if f32 else np.complex128
        self._rt = torch.float32 if f32 else torch.float64
        self._ct = torch.complex64 if f32 else torch.complex128
        self._red = _Red(self.dev_)
        self._build_kernels()
        self.K_ = len(specs)
        return counts

    def _build_kernels(self):
        """One device plan per distinct mode kernel (modes with the same kernel share it), from a process-wide cache
        of recent plans (refits on the same lattice and kernel reuse their twiddles)."""
        eng = _lib.ENGINE_TC if self.matvec_engine == 'tc' and self.d_ == 2 and self.shape_[-1] % 4 == 0 \
            else _lib.ENGINE_SIMT
        self.kern_ = []
        mine = set()
        for sp in self.specs_:
            key = (spec_key(sp), self.shape_, tuple(np.round(self.h_, 15)), self._code, eng, str(self.dev_))
            hit = _PLANS.pop(key, None)
            if hit is None:
                freqs, W = mode_transform(sp, self.shape_, self.h_, self.pad_)
                with torch.cuda.device(self.dev_):
                    plan = Plan(freqs, W, self.shape_, self._code, eng)
                hit = (plan, kernel_at_zero(sp, self.d_), (freqs, W))
            _PLANS[key] = hit                         # most recent last
            mine.add(key)
            if eng == _lib.ENGINE_SIMT:
                hit[0].route = self.matvec_route          # a cached plan takes this fit's route
            self.kern_.append(hit)
        while len(_PLANS) > _PLAN_CACHE_SIZE:
            _PLANS.popitem(last=False)
        self.shared_ = len(mine) == 1
        self.s_ = np.array([kk[1] for kk in self.kern_])
        self._dplan_rows = None                          # derivative plans follow the kernels

    # ---------------------------------------------------------------- device helpers
    @property
    def _st(self):
        return torch.cuda.current_stream(self.dev_).cuda_stream

    def _Sall(self, E, out=None):
        """S_k E_k for every mode (modes sharing a plan in one batched call)."""
        out = torch.empty_like(E) if out is None else out
        K = E.shape[0]; k = 0
        while k < K:
            j = k + 1
            while j < K and self.kern_[j][0] is self.kern_[k][0]:
                j += 1
            self.kern_[k][0].apply(E[k:j], out[k:j], j - k, E.is_complex(), self._st)
            k = j
        return out

    def _nreal(self, x):
        return x.numel() * (2 if x.is_complex() else 1)

    def _dots(self, pairs):
        """Re <a, b> for a list of (a, b) tensor pairs, float64, one pass."""
        if not pairs:
            return []
        n = self._nreal(pairs[0][0])
        call('blml_dots', self._code, n, len(pairs), ptrs([p[0] for p in pairs]), ptrs([p[1] for p in pairs]),
             self._red.part.data_ptr(), self._red.out.data_ptr(), self._st)
        return self._red.read(len(pairs))

    def _lin(self, terms, out=None):
        """out = sum c_i v_i over (c_i, v_i) terms."""
        out = torch.empty_like(terms[0][1]) if out is None else out
        call('blml_lincomb', self._code, self._nreal(out), out.data_ptr(), len(terms), dbl([t[0] for t in terms]),
             ptrs([t[1] for t in terms]), self._st)
        return out

    def _scale_(self, x, sc):
        if sc != 1.0:
            self._lin([(sc, x)], out=x)
        return x

    # ---------------------------------------------------------------- merit, update, residual
    def _merit(self, E, U):
        """Larger is better. psd: scale-free log-likelihood / n; real rank 1: -Phi / n (blml_binned.py:171-182)."""
        call('blml_merit_terms', self._code, E.shape[0], self.B_, int(E.is_complex()), int(self.psd_), E.data_ptr(),
             U.data_ptr(), self.c_t_.data_ptr(), self.sg_t_.data_ptr(), self._red.part.data_ptr(),
             self._red.out.data_ptr(), self._st)
        a, b, bad = self._red.read(3)
        n = self.n_
        if self.psd_:
            if not b > 0:
                return -np.inf
            return a / n - n * np.log(b)
        if bad > 0:
            return -np.inf
        return -(0.5 * a - b) / n

    def _update(self, E, U):
        out = torch.empty_like(E)
        call('blml_jacobi_update', self._code, E.shape[0], self.B_, int(E.is_complex()), int(self.psd_),
             dbl(self.s_[:E.shape[0]]), E.data_ptr(), U.data_ptr(), self.c_t_.data_ptr(), self.sg_t_.data_ptr(),
             out.data_ptr(), self._st)
        return out

    def _Q(self, E, U):
        return self._dots([(E, U)])[0]

    def _rescale(self, E, U, Q=None):
        """In place: E, U scaled so that Q = e^H S e = n^2 (blml_binned.py:211-214)."""
        Q = self._Q(E, U) if Q is None else Q
        sc = float(self.n_ / np.sqrt(Q)) if Q > 0 else 1.0
        return self._scale_(E, sc), self._scale_(U, sc)

    def _resid(self, E, U, scale=1.0):
        call('blml_resid', self._code, E.shape[0], self.B_, int(E.is_complex()), E.data_ptr(), U.data_ptr(),
             self.c_t_.data_ptr(), float(scale), self._red.part.data_ptr(), self._red.out.data_ptr(), self._st)
        mx, nnan = self._red.read(2)
        return float('nan') if nnan > 0 else mx

    # ---------------------------------------------------------------- CD solver
    def _solve(self, E, max_sweeps):
        if self.solver == 'lbfgs' and self.psd_:
            return self._solve_lbfgs(E, max_sweeps)
        return self._solve_cd(E, max_sweeps)

    def _solve_cd(self, E, max_sweeps):
        """Jacobi coordinate updates + Anderson mixing + merit safeguard (blml_binned.py:223-276)."""
        E = E.clone()
        U = self._Sall(E); self._rescale(E, U)
        cur = self._merit(E, U); mA = self.anderson
        hist_ = _Anderson(self, mA)
        n_and = n_damp = n_grad = 0; it = 0; res = self._resid(E, U); hist = [res]
        cap = np.inf if max_sweeps is None else max_sweeps
        best_res, best_it, best_m = res, 0, cur
        mhist = [cur]; self.stop_reason_ = 'tol'
        while res >= self.tol and it < cap:
            if it - best_it >= self.stall:
                self.stop_reason_ = 'stall'; break
            if self.ll_tol is not None and len(mhist) > self.ll_window and \
                    (mhist[-1] - mhist[-1 - self.ll_window]) / self.n_ < self.ll_tol:
                self.stop_reason_ = 'll_tol'; break
            it += 1
            EJ0 = self._update(E, U); UJ0 = self._Sall(EJ0); mJ0 = self._merit(EJ0, UJ0)
            EJ, UJ, mJ = EJ0, UJ0, mJ0
            if mA:
                f = self._lin([(1.0, EJ0), (-1.0, E)])
                EA = hist_.step(E, f)
                if EA is not None:
                    UA = self._Sall(EA); mAc = self._merit(EA, UA)
                    if mAc > mJ:
                        EJ, UJ, mJ = EA, UA, mAc; n_and += 1
            if mJ < cur - 1e-12 * abs(cur):                # no ascent: damp the Jacobi step
                hist_.reset(); n_damp += 1
                EP, UP = EJ0, UJ0
                a = 0.5; found = False
                while a > 1e-8:
                    ET = self._lin([(1.0 - a, E), (a, EP)]); UT = self._lin([(1.0 - a, U), (a, UP)])
                    mJ = self._merit(ET, UT)
                    if mJ >= cur:
                        found = True; break
                    a *= 0.5
                if found:
                    EJ, UJ = ET, UT
                else:
                    EJ, UJ, mJ = E, U, cur
                    if self.psd_:
                        EJ, UJ, mJ = self._grad_steps(E, U, cur); n_grad += 1
            E, U = EJ, UJ
            self._rescale(E, U)
            cur = mJ if self.psd_ else self._merit(E, U); mhist.append(cur)
            res = self._resid(E, U); hist.append(res)
            if res < 0.9 * best_res or cur > best_m + 1e-13 * abs(best_m):
                best_res, best_it, best_m = min(res, best_res), it, max(cur, best_m)
            if self.verbose and it % 100 == 0:
                print(f'  sweep {it}: max|rho|={res:.2e} merit={cur:.9f} anderson={n_and} damped={n_damp} '
                      f'gradient={n_grad}', flush=True)
        if res >= self.tol and self.stop_reason_ == 'tol':
            self.stop_reason_ = 'max_sweeps'
        self.n_sweeps_, self.residual_, self.converged_ = it, res, res < self.tol
        self.merit_history_ = mhist
        self.rho_history_, self.n_anderson_, self.n_damped_, self.n_gradient_ = hist, n_and, n_damp, n_grad
        return E, U

    def _grad_weights(self, U, vscale=1.0):
        """V = vscale w / F U on occupied bins and sum_occ w log F."""
        V = torch.empty_like(U)
        call('blml_lgrad_weights', self._code, U.shape[0], self.B_, int(U.is_complex()), U.data_ptr(),
             self.w_t_.data_ptr(), float(vscale), V.data_ptr(), self._red.part.data_ptr(), self._red.out.data_ptr(),
             self._st)
        return V, self._red.read(1)[0]

    def _grad_finish(self, SV, U, nq):
        g = torch.empty_like(U)
        call('blml_lgrad_finish', self._code, U.shape[0], self.B_, int(U.is_complex()), SV.data_ptr(), U.data_ptr(),
             self.w_t_.data_ptr(), float(nq), g.data_ptr(), self._st)
        return g

    def _grad_steps(self, E, U, cur, steps=5):
        """Steepest ascent on L with Armijo backtracking (blml_binned.py:357-380)."""
        for _ in range(steps):
            Q = self._Q(E, U)
            V, _ = self._grad_weights(U)
            G = self._grad_finish(self._Sall(V), U, self.n_ / Q)
            self._scale_(G, 0.5)                         # _grad_finish returns 2 (S V - n U / Q) on occupied bins
            SG = self._Sall(G)
            g2, e2 = self._dots([(G, G), (E, E)])
            if not g2 > 0:
                break
            a = getattr(self, '_gstep', None) or 1e-3 * np.sqrt(e2 / g2)
            ok = False
            for _ in range(40):
                En = self._lin([(1.0, E), (a, G)]); Un = self._lin([(1.0, U), (a, SG)])
                mn = self._merit(En, Un)
                if mn > cur:
                    ok = True; break
                a *= 0.5
            if not ok:
                break
            E, U, cur = En, Un, mn; self._gstep = 2 * a
        return E, U, cur

    # ---------------------------------------------------------------- L-BFGS
    def _lgrad(self, E, U):
        """(L, g, Q): L = sum w log F - n log Q and its gradient 2 (S (w U / F) - n U / Q) on occupied bins."""
        Q = self._Q(E, U)
        if not Q > 0:
            return -np.inf, None, Q
        V, Lw = self._grad_weights(U)
        g = self._grad_finish(self._Sall(V), U, self.n_ / Q)
        return Lw - self.n_ * np.log(Q), g, Q

    def _solve_lbfgs(self, E, max_iter):
        """L-BFGS ascent of L on the coefficients with Armijo backtracking (blml_binned.py:290-355), the direction in
        compact form: H g = gamma g + S p - gamma Y t with R t = S^T g (R the upper triangle of S^T Y) and
        R^T p = (D + gamma Y^T Y) t - gamma Y^T g."""
        n = self.n_; m_ = self.lbfgs_m
        E = E.clone()
        U = self._Sall(E); self._rescale(E, U)
        L, g, Q = self._lgrad(E, U)
        Sh, Yh = [], []; SY = np.zeros((0, 0)); YY = np.zeros((0, 0))
        it = 0
        res = self._resid(E, U, self.n_ / np.sqrt(Q) if Q > 0 else 1.0); hist = [res]; mhist = [L / n]
        cap = np.inf if max_iter is None else max_iter; self.stop_reason_ = 'tol'; reset = False
        ftol, fwin = (self.ll_tol if self.ll_tol is not None else 1e-11), 10
        while res >= self.tol and it < cap:
            if len(mhist) > fwin and mhist[-1] - mhist[-1 - fwin] < ftol:
                self.stop_reason_ = 'll_tol'; break
            it += 1
            m = len(Sh)
            vals = self._dots([(s, g) for s in Sh] + [(y, g) for y in Yh] + [(g, g), (E, E)])
            a_, b_ = np.array(vals[:m]), np.array(vals[m:2 * m]); gg, ee = vals[2 * m], vals[2 * m + 1]
            first = 1e-3 * np.sqrt(ee / max(gg, 1e-300))
            if m:
                gam = SY[-1, -1] / YY[-1, -1]
                R = np.triu(SY)
                t_ = _solve_tri(R, a_, upper=True)
                p_ = _solve_tri(R.T, (np.diag(np.diag(SY)) + gam * YY) @ t_ - gam * b_, upper=False)
                q = self._lin([(gam, g)] + [(float(p_[i]), Sh[i]) for i in range(m)] +
                              [(float(-gam * t_[i]), Yh[i]) for i in range(m)])
                slope = gam * gg + float(a_ @ p_) - gam * float(b_ @ t_)
            else:
                q = self._lin([(first, g)]); slope = first * gg
            if not slope > 0:
                Sh, Yh = [], []; SY = np.zeros((0, 0)); YY = np.zeros((0, 0))
                q = self._lin([(first, g)]); slope = first * gg
            Sq = self._Sall(q)
            t = 1.0; ok = False
            En = torch.empty_like(E); Un = torch.empty_like(U)
            for _ in range(40):
                call('blml_lbfgs_trial', self._code, E.shape[0], self.B_, int(E.is_complex()), E.data_ptr(),
                     q.data_ptr(), U.data_ptr(), Sq.data_ptr(), self.w_t_.data_ptr(), t, En.data_ptr(), Un.data_ptr(),
                     self._red.part.data_ptr(), self._red.out.data_ptr(), self._st)
                Lw, Qn = self._red.read(2)
                Ln = Lw - n * np.log(Qn) if Qn > 0 else -np.inf
                if Ln >= L + 1e-4 * t * slope:
                    ok = True; break
                t *= 0.5
            if not ok:
                if reset or not Sh:
                    self.stop_reason_ = 'stall'; break
                Sh, Yh = [], []; SY = np.zeros((0, 0)); YY = np.zeros((0, 0)); reset = True; continue
            reset = False
            # the accepted point's U exactly: U + t S q equals S(E + t q) only up to rounding, and a drifting U lets
            # the ascent move e along the near-null directions of S (which change Q = <E, U> through the drift alone)
            self._Sall(En, out=Un)
            Qn = self._Q(En, Un)
            V, Lwn = self._grad_weights(Un)
            Ln = Lwn - n * np.log(Qn) if Qn > 0 else -np.inf
            gn = self._grad_finish(self._Sall(V), Un, n / Qn)
            s_ = self._lin([(t, q)]); y_ = self._lin([(1.0, g), (-1.0, gn)])
            vals = self._dots([(s_, y_), (s_, s_), (y_, y_)] + [(s, y_) for s in Sh] + [(y, y_) for y in Yh])
            sy, ss, yy = vals[:3]
            if sy > 1e-12 * np.sqrt(ss * yy):
                m = len(Sh)
                SYn = np.zeros((m + 1, m + 1)); SYn[:m, :m] = SY; SYn[:m, m] = vals[3:3 + m]; SYn[m, m] = sy
                YYn = np.zeros((m + 1, m + 1)); YYn[:m, :m] = YY; YYn[:m, m] = YYn[m, :m] = vals[3 + m:3 + 2 * m]
                YYn[m, m] = yy
                Sh.append(s_); Yh.append(y_); SY, YY = SYn, YYn
                if len(Sh) > m_:
                    Sh.pop(0); Yh.pop(0); SY = SY[1:, 1:]; YY = YY[1:, 1:]
            E, U, L, g, Q = En, Un, Ln, gn, Qn
            res = self._resid(E, U, self.n_ / np.sqrt(Q)); hist.append(res); mhist.append(L / n)
            if self.verbose and it % 100 == 0:
                print(f'  lbfgs {it}: max|rho|={res:.2e} L/n={L / n:.9f}', flush=True)
        if res >= self.tol and self.stop_reason_ == 'tol':
            self.stop_reason_ = 'max_sweeps'
        # the canonical form e_k = (Q / n) (w / F) u_k on occupied bins (blml_binned.py:342-350)
        Qc = self._Q(E, U)
        Ec, _ = self._grad_weights(U, vscale=Qc / n)
        Uc = self._Sall(Ec)
        _, Lwc = self._grad_weights(Uc)
        Qcc = self._Q(Ec, Uc)
        Lc = Lwc - n * np.log(Qcc) if Qcc > 0 else -np.inf
        if Lc >= L - 1e-9 * n:
            E, U = Ec, Uc
        self._rescale(E, U); res = self._resid(E, U)
        self.n_sweeps_, self.residual_ = it, res
        self.converged_ = res < self.tol or self.stop_reason_ == 'll_tol'
        self.merit_history_ = mhist; self.rho_history_ = hist
        self.n_anderson_ = self.n_damped_ = self.n_gradient_ = 0
        return E, U

    # ---------------------------------------------------------------- fit
    def fit(self, counts, modes, h=1.0, origin=0.0, complex_g=False, signs=None, init=None):
        """counts: (m_1, ..., m_d) histogram on the lattice origin + h * index. modes: the model (make_modes);
        rank K = len(modes). complex_g: complex g_k. signs: real rank 1 only, sign of g per bin (array shaped like
        counts, or a callable of the (B, d) bin centres). init: a previous fit on the same lattice (warm start)."""
        counts = self._setup(counts, modes, h, origin)
        dev = self.dev_
        if isinstance(counts, torch.Tensor):
            self.w_t_ = counts.reshape(-1).to(self._rt).contiguous()
            self.n_ = float(counts.sum(dtype=torch.float64))
        else:
            w = np.asarray(counts, float)
            self.n_ = float(w.sum(dtype=np.float64))
            self.w_t_ = torch.as_tensor(w.ravel(), dtype=self._rt).to(dev)
        if not self.n_ > 0:
            raise ValueError("counts: no observations")
        self.c_t_ = self._lin([(self.n_, self.w_t_)])
        self._occ_t = None
        self.complex_g_ = bool(complex_g); self.psd_ = bool(complex_g) or self.K_ > 1
        if signs is not None and self.psd_:
            raise ValueError("complex_g / rank > 1 estimate the phases; do not pass signs as well")
        sg = np.ones(self.shape_) if signs is None else (
            np.sign(signs(self.centres())).reshape(self.shape_) if callable(signs) else np.sign(np.asarray(signs, float)))
        if signs is not None and np.any(sg.ravel()[self.w_t_.cpu().numpy() > 0] == 0):
            raise ValueError("signs: nonzero on every occupied bin")
        self.sg_t_ = torch.as_tensor(np.ascontiguousarray(sg, float).ravel(), dtype=self._rt).to(dev)
        self.signs_ = None if signs is None else sg
        et = self._ct if self.complex_g_ else self._rt
        if init is not None and getattr(init, 'e_hat_', None) is not None and tuple(init.shape_) == tuple(self.shape_):
            E0 = getattr(init, 'e_hat_t_', None)
            E0 = torch.as_tensor(np.asarray(init.e_hat_)).to(dev) if E0 is None else E0.to(dev)
            E0 = E0.reshape(E0.shape[0], -1)
            E = torch.zeros((self.K_, self.B_), dtype=et, device=dev)
            kk = min(self.K_, E0.shape[0])
            E[:kk] = (E0[:kk] if self.complex_g_ else (E0[:kk].real if E0.is_complex() else E0[:kk])).to(et)
            occm = (self.w_t_ > 0).to(self._rt)
            call('blml_mul_bins', self._code, self.K_, self.B_, int(E.is_complex()), E.data_ptr(), occm.data_ptr(),
                 E.data_ptr(), self._st)
            E = self._fill_modes(E, kk, phases=False)
        else:
            E = self._start(et)
        E, U = self._solve(E, self.max_sweeps)
        self._finish(E, U)
        return self

    def _start(self, et):
        """Real positive root of mode 0 (one convex solve), then small phases / small other modes. For float32 fits
        the convex start is solved in float64: its merit safeguard needs more than float32 resolution below
        max|rho| ~ 1e-2, where a float32 solve stalls."""
        e0 = torch.empty((1, self.B_), dtype=self._rt, device=self.dev_)
        call('blml_start_root', self._code, self.B_, self.c_t_.data_ptr(), self.sg_t_.data_ptr(), float(self.s_[0]),
             e0.data_ptr(), self._st)
        if not self.psd_:
            return e0
        if self._code == _lib.F32:
            er = self._start_f64()
        else:
            save = (self.psd_, self.K_, self.kern_, self.s_)
            self.psd_, self.K_, self.kern_, self.s_ = False, 1, self.kern_[:1], self.s_[:1]
            try:
                er, _ = self._solve(e0, self.max_sweeps)
            finally:
                self.psd_, self.K_, self.kern_, self.s_ = save
        E = torch.zeros((self.K_, self.B_), dtype=et, device=self.dev_)
        E[0] = er[0].to(et)
        return self._fill_modes(E, 1)

    def _start_f64(self):
        """The real rank-1 start under mode 0, solved by a float64 twin of this fit (same counts, solver settings)."""
        twin = BLMLBinned(tol=self.tol, max_sweeps=self.max_sweeps, anderson=self.anderson, dtype=np.float64,
                          phase_noise=self.phase_noise, seed=self.seed, stall=self.stall, ll_tol=self.ll_tol,
                          ll_window=self.ll_window, solver='cd', device=self.dev_)
        twin._setup(self.w_t_.reshape(self.shape_).to(torch.float64), self.modes_[:1], self.h_, self.origin_)
        twin.n_ = self.n_
        twin.w_t_ = self.w_t_.to(torch.float64)
        twin.c_t_ = twin._lin([(self.n_, twin.w_t_)])
        twin.sg_t_ = self.sg_t_.to(torch.float64)
        twin.complex_g_ = False; twin.psd_ = False
        e0 = torch.empty((1, self.B_), dtype=torch.float64, device=self.dev_)
        call('blml_start_root', _lib.F64, self.B_, twin.c_t_.data_ptr(), twin.sg_t_.data_ptr(), float(twin.s_[0]),
             e0.data_ptr(), self._st)
        er, _ = twin._solve(e0, self.max_sweeps)
        self.start_sweeps_ = twin.n_sweeps_
        return er

    def _fill_modes(self, E, kk, phases=True):
        """The reference's seeded start noise (blml_binned.py:429-436): the normals are drawn on the host with the same
        generator and order, then applied on the device."""
        rng = np.random.default_rng(self.seed); sh = self.shape_
        draws = []
        if self.complex_g_ and phases:
            draws.append(rng.standard_normal(sh).ravel())
        for _ in range(kk, self.K_):
            draws.append(rng.standard_normal(sh).ravel())
            if self.complex_g_:
                draws.append(rng.standard_normal(sh).ravel())
        if not draws:
            return E
        z = torch.as_tensor(np.concatenate(draws), dtype=torch.float64).to(self.dev_)
        call('blml_fill_modes', self._code, self.K_, self.B_, int(E.is_complex()), int(kk), int(phases),
             float(self.phase_noise), z.data_ptr(), E.data_ptr(), self._st)
        return E

    def _finish(self, E, U):
        self.e_hat_t_, self.Se_t_ = E, U
        dens = torch.empty(self.B_, dtype=self._rt, device=self.dev_)
        call('blml_finish', self._code, E.shape[0], self.B_, int(U.is_complex()), U.data_ptr(), self.w_t_.data_ptr(),
             1.0 / self.n_ ** 2, dens.data_ptr(), self._red.part.data_ptr(), self._red.out.data_ptr(), self._st)
        self.density_t_ = dens
        self.loglik_ = self._red.read(1)[0] / self.n_
        self.n_samples_ = self.n_
        self._host = {}

    # ---------------------------------------------------------------- outputs
    def _np(self, name, t, shape):
        if name not in self._host:
            self._host[name] = t.detach().cpu().numpy().reshape(shape)
        return self._host[name]

    @property
    def density_(self):
        return self._np('density', self.density_t_, self.shape_)

    @property
    def e_hat_(self):
        return self._np('e_hat', self.e_hat_t_, (self.K_,) + tuple(self.shape_))

    @property
    def Se_(self):
        return self._np('Se', self.Se_t_, (self.K_,) + tuple(self.shape_))

    @property
    def w_(self):
        return self.w_t_.cpu().numpy().reshape(self.shape_)

    @property
    def c_(self):
        return self.c_t_.cpu().numpy().reshape(self.shape_)

    @property
    def occ_(self):
        return (self.w_t_ > 0).cpu().numpy().reshape(self.shape_)

    def centres(self):
        g = np.meshgrid(*[self.origin_[j] + self.h_[j] * np.arange(m) for j, m in enumerate(self.shape_)], indexing='ij')
        return np.stack([x.ravel() for x in g], 1)

    def log_density(self, counts, eps=0.0):
        """Mean over counts m on the lattice of log(f_b + eps), f = F / Q (blml_binned.py:630-637)."""
        U = self.Se_t_
        Z = self._Q(self.e_hat_t_, U)
        m = torch.as_tensor(np.asarray(counts, float).ravel(), dtype=self._rt).to(self.dev_)
        call('blml_log_score', self._code, U.shape[0], self.B_, int(U.is_complex()), U.data_ptr(), m.data_ptr(),
             1.0 / Z, float(eps), self._red.part.data_ptr(), self._red.out.data_ptr(), self._st)
        s, tot = self._red.read(2)
        return s / tot

    def _val_score(self, counts):
        return self.log_density(counts)

    def certificate(self, k=1, tol=1e-6):
        """lambda_max(D^1/2 S D^1/2) / n, D_b = ||e_b||^2 / w_b (shared kernel), by float64 Lanczos on the GPU
        (blml_binned.py:501-518). <= 1 (+ solver tolerance): the fit solves the convex lift."""
        if not self.shared_:
            raise ValueError("certificate: shared kernel only (per-mode kernels: no convex lift)")
        from .certificate import lanczos_max
        E = self.e_hat_t_
        dh = torch.empty(self.B_, dtype=torch.float64, device=self.dev_)
        call('blml_cert_weights', self._code, E.shape[0], self.B_, int(E.is_complex()), E.data_ptr(),
             self.w_t_.data_ptr(), dh.data_ptr(), self._st)
        plan = self._plan64()
        return lanczos_max(plan, dh, self._red, self._st, tol=tol, seed=self.seed) / self.n_

    def _plan64(self):
        if self._code == _lib.F64 and self.matvec_engine == 'simt':
            return self.kern_[0][0]
        if getattr(self, '_p64', None) is None:
            freqs, W = self.kern_[0][2]
            self._p64 = Plan(freqs, W, self.shape_, _lib.F64, _lib.ENGINE_SIMT)
        return self._p64

    # ---------------------------------------------------------------- at arbitrary points
    def _mode_at_points(self, k, X):
        """sum_b e_kb K_k(x - z_b) at the points X (m, d) on the device, complex128 (m,). Units of sinc / slits /
        dirichlet / ball kind: the exact kernels per (point, bin) pair over the occupied bins (blml_point_rows).
        Harmonic kernels (pball groups with dirichlet columns): the band's spectrum C = W (v^H e) and the plane-wave
        sum over it (blml_spectrum, blml_planewave_points), exact since the kernel is that sum."""
        from .spec import split_kind
        import ctypes as C
        sp = self.specs_[k]
        names = [split_kind(kd)[0] for kd, _ in units_of(sp['kinds'])]
        e = self.e_hat_t_[k].to(torch.complex128 if self.e_hat_t_.is_complex() else torch.float64).contiguous()
        Xt = torch.as_tensor(np.ascontiguousarray(X, np.float64)).to(self.dev_)
        m = len(X)
        if all(n in ('sinc', 'slits', 'dirichlet', 'ball') for n in names):
            cols = point_cols(sp, self.d_)
            occ = self.w_t_ > 0
            Z = torch.as_tensor(self.centres()).to(self.dev_)[occ].contiguous()
            parts = [e.real, e.imag] if e.is_complex() else [e]
            outs = []
            for part in parts:
                w = part[occ].contiguous()
                g = torch.empty(m, dtype=torch.float64, device=self.dev_)
                call('blml_point_rows', m, self.d_, Xt.data_ptr(), int(Z.shape[0]), Z.data_ptr(), w.data_ptr(),
                     C.cast(cols, C.c_void_p), g.data_ptr(), self._st)
                outs.append(g)
            return torch.complex(outs[0], outs[1]) if len(outs) == 2 else torch.complex(outs[0], torch.zeros_like(outs[0]))
        if not all(n in ('pball', 'dirichlet') for n in names) or self.d_ > 2:
            raise NotImplementedError("sqrt_density at arbitrary points: sinc / slits / dirichlet / ball units, or pball "
                                      "groups with dirichlet columns in 1-D / 2-D (a pball group times another unit "
                                      "is neither)")
        freqs, W = mode_transform(sp, self.shape_, self.h_, self.pad_)
        plan = Plan(freqs, W, self.shape_, _lib.F64, _lib.ENGINE_SIMT)
        ws = torch.empty(int(_lib.lib().blml_spectrum_workspace(plan._h, 1)), dtype=torch.uint8, device=self.dev_)
        spec = torch.empty(int(np.prod([len(f) for f in freqs])), dtype=torch.complex128, device=self.dev_)
        x = e if e.is_complex() else e.to(torch.complex128)
        call('blml_spectrum', plan._h, x.data_ptr(), spec.data_ptr(), 1, 1, ws.data_ptr(), ws.numel(), self._st)
        U = (np.asarray(X, float) - self.origin_[None, :]) / self.h_[None, :]
        if self.d_ == 1:
            f1, f2, U2 = np.zeros(1), np.asarray(freqs[0], float), np.stack([np.zeros(m), U[:, 0]], 1)
        else:
            f1, f2, U2 = np.asarray(freqs[0], float), np.asarray(freqs[1], float), U
        dev = self.dev_
        f1t, f2t = torch.as_tensor(f1).to(dev), torch.as_tensor(f2).to(dev)
        Ut = torch.as_tensor(np.ascontiguousarray(U2, np.float64)).to(dev)
        g = torch.empty(m, dtype=torch.complex128, device=dev)
        call('blml_planewave_points', len(f1), len(f2), f1t.data_ptr(), f2t.data_ptr(), spec.data_ptr(), m,
             Ut.data_ptr(), g.data_ptr(), self._st)
        return g

    def sqrt_density(self, X, chunk=65536):
        """g_k(x) = (1/n) sum_b e_bk K_k(x - z_b) at arbitrary points X (m, d) (blml_binned.py:451-465): (m,) for
        rank 1, else (m, K); complex for complex_g."""
        X = np.atleast_2d(np.asarray(X, float))
        if X.shape[1] != self.d_:
            X = X.reshape(-1, self.d_)
        out = np.zeros((len(X), self.K_), dtype=complex if self.complex_g_ else float)
        for i in range(0, len(X), chunk):
            for k in range(self.K_):
                g = self._mode_at_points(k, X[i:i + chunk]).cpu().numpy() / self.n_
                out[i:i + chunk, k] = g if self.complex_g_ else g.real
        return out[:, 0] if self.K_ == 1 else out

    def predict(self, X):
        """f(x) = sum_k |g_k(x)|^2 at arbitrary points (blml_binned.py:467-469)."""
        G = self.sqrt_density(X)
        return np.abs(G) ** 2 if G.ndim == 1 else (np.abs(G) ** 2).sum(1)

    def predict_grid(self, r):
        """f on the lattice refined r times per dim (from the origin in steps h / r; the last fine point is the last
        bin): shape ((m_j - 1) r + 1, ...) (blml_binned.py:471-500)."""
        r = int(r)
        fine = tuple((m - 1) * r + 1 for m in self.shape_)
        g = np.meshgrid(*[self.origin_[j] + (self.h_[j] / r) * np.arange(n) for j, n in enumerate(fine)], indexing='ij')
        X = np.stack([x.ravel() for x in g], 1)
        return self.predict(X).reshape(fine)

    # ---------------------------------------------------------------- fc gradients
    def _dplans(self):
        """Per mode, per kernel unit (units_of order): the device plan of dS/dlog fc_u, None for integer units
        (dirichlet, pball: fc moves in whole harmonics). Modes with one kernel share their plans."""
        key = (self._code, str(self.dev_))
        if getattr(self, '_dplan_key', None) != key or self._dplan_rows is None:
            rows, seen = [], {}
            for sp in self.specs_:
                k = spec_key(sp)
                if k not in seen:
                    row = []
                    for u in range(len(units_of(sp['kinds']))):
                        tr = mode_transform_dlog(sp, self.shape_, self.h_, self.pad_, u)
                        if tr is None:
                            row.append(None)
                        else:
                            with torch.cuda.device(self.dev_):
                                row.append(Plan(tr[0], tr[1], self.shape_, self._code, _lib.ENGINE_SIMT))
                    seen[k] = row
                rows.append(seen[k])
            self._dplan_rows, self._dplan_key = rows, key
        return self._dplan_rows

    def _dapply(self, plan, x):
        """dS x for one mode's coefficients x (1, B)."""
        y = torch.empty_like(x)
        plan.apply(x, y, 1, x.is_complex(), self._st)
        return y

    def _counts_t(self, counts):
        if isinstance(counts, torch.Tensor):
            return counts.reshape(-1).to(self.dev_, self._rt).contiguous()
        m = np.asarray(counts, float)
        if m.size != self.B_:
            raise ValueError("counts: one value per bin of the fitted lattice")
        return torch.as_tensor(m.ravel(), dtype=self._rt).to(self.dev_)

    def _score_weights(self, counts, eps):
        """(V = wn U, sum wn F / M, M, Z) of the score sum m log(F / Z + eps) / M (blml_binned.py:549-553)."""
        E, U = self.e_hat_t_, self.Se_t_
        m = self._counts_t(counts)
        Z = self._Q(E, U)
        V = torch.empty_like(U)
        call('blml_pgrad_weights', self._code, U.shape[0], self.B_, int(U.is_complex()), U.data_ptr(), m.data_ptr(),
             float(eps) * Z, V.data_ptr(), self._red.part.data_ptr(), self._red.out.data_ptr(), self._st)
        swf, M = self._red.read(2)
        if not M > 0:
            raise ValueError("counts: no observations")
        return V, swf / M, M, Z

    def param_grad(self, counts, eps=0.0):
        """d/dlog fc_u of sum_b m_b log(F_b / Z + eps) / sum m at the current coefficients (blml_binned.py:543-562),
        for counts m on the lattice (the training counts: fc_grad; a new batch: the prequential gradient). eps is in
        density units (f = F / Z). A list per mode of arrays, one entry per kernel unit (NaN for integer units)."""
        V, fz, M, Z = self._score_weights(counts, eps)
        E = self.e_hat_t_
        out = []
        for k, row in enumerate(self._dplans()):
            gk = []
            for plan in row:
                if plan is None:
                    gk.append(np.nan); continue
                dU = self._dapply(plan, E[k:k + 1])
                a, b = self._dots([(V[k:k + 1], dU), (E[k:k + 1], dU)])
                gk.append(2 * a / M - fz * b / Z)
            out.append(np.array(gk))
        return out

    def fc_grad(self):
        """d loglik_ / dlog fc of every (mode, unit) at the fitted coefficients (blml_binned.py:520-527: the envelope
        theorem, e stationary for the scale-free likelihood): param_grad of the training counts."""
        return self.param_grad(self.w_t_)

    def _occ_mask(self):
        if getattr(self, '_occ_t', None) is None:
            self._occ_t = (self.w_t_ > 0).to(self._rt)
        return self._occ_t

    def _mask_(self, x):
        call('blml_mul_bins', self._code, x.shape[0], self.B_, int(x.is_complex()), x.data_ptr(),
             self._occ_mask().data_ptr(), x.data_ptr(), self._st)
        return x

    def _hvp(self, D, Q):
        """The Hessian of the minimised objective times D (blml_binned.py:593-606): -L (psd) or Phi (real rank 1)."""
        E, U = self.e_hat_t_, self.Se_t_
        dU = self._Sall(D)
        out = torch.empty_like(D)
        if not self.psd_:
            call('blml_hvp_real1', self._code, self.B_, D.data_ptr(), E.data_ptr(), self.c_t_.data_ptr(),
                 dU.data_ptr(), out.data_ptr(), self._st)
            return out
        n = self.n_
        call('blml_hvp_inner', self._code, U.shape[0], self.B_, int(U.is_complex()), U.data_ptr(), dU.data_ptr(),
             self.w_t_.data_ptr(), out.data_ptr(), self._st)
        SI = self._Sall(out)
        dQ = 2 * self._dots([(U, D)])[0]
        return self._lin([(-2.0, SI), (2 * n / Q, dU), (-2 * n * dQ / Q ** 2, U)], out=out)

    def _mixed(self, k, plan, Q):
        """d(gradient of the minimised objective)/dlog fc for one unit of mode k at fixed coefficients
        (blml_binned.py:610-628)."""
        E, U = self.e_hat_t_, self.Se_t_
        n = self.n_
        dUk = self._dapply(plan, E[k:k + 1])
        if not self.psd_:
            return dUk
        dQ = self._dots([(E[k:k + 1], dUk)])[0]
        T = torch.empty_like(U); Wk = torch.empty_like(dUk)
        call('blml_mixed_terms', self._code, U.shape[0], self.B_, int(U.is_complex()), U.data_ptr(), int(k),
             dUk.data_ptr(), self.w_t_.data_ptr(), T.data_ptr(), Wk.data_ptr(), self._st)
        g = self._lin([(-2.0, self._Sall(T)), (-2 * n * dQ / Q ** 2, U)])
        dW = self._dapply(plan, Wk)
        self._lin([(1.0, g[k:k + 1]), (-2.0, dW), (2 * n / Q, dUk)], out=g[k:k + 1])
        return g

    def implicit_grad(self, counts, eps=0.0, tol=1e-6, maxit=300):
        """d/dlog fc_u of the same score as param_grad with the coefficients' response to the move included
        (blml_binned.py:565-628): dP/dtheta = dP/dtheta|_e - <v, d grad/dtheta>, H v = dP/de by conjugate gradients
        (blml_binned.py:1485-1496) on the occupied bins, Hessian-vector products by the mat-vec. Sets ift_iters_ and
        ift_res_ (the CG's iterations and relative residual)."""
        G = self.param_grad(counts, eps)
        V, fz, M, Q = self._score_weights(counts, eps)
        U = self.Se_t_
        b = self._mask_(self._lin([(2.0 / M, self._Sall(V)), (-2.0 * fz / Q, U)]))
        x = torch.zeros_like(b); r = b.clone(); p = r.clone()
        rs = self._dots([(r, r)])[0]; bn = np.sqrt(rs) or 1.0
        it, res = maxit, np.sqrt(rs) / bn
        for i in range(1, maxit + 1):
            Ap = self._mask_(self._hvp(p, Q))
            pAp = self._dots([(p, Ap)])[0]
            if not pAp > 0:
                it, res = i, np.sqrt(rs) / bn
                break
            a = rs / pAp
            self._lin([(1.0, x), (a, p)], out=x); self._lin([(1.0, r), (-a, Ap)], out=r)
            rs_new = self._dots([(r, r)])[0]
            if np.sqrt(rs_new) / bn < tol:
                it, res = i, np.sqrt(rs_new) / bn
                break
            self._lin([(1.0, r), (rs_new / rs, p)], out=p); rs = rs_new
            res = np.sqrt(rs) / bn
        self.ift_iters_, self.ift_res_ = it, res
        for k, row in enumerate(self._dplans()):
            for u, plan in enumerate(row):
                if plan is not None:
                    G[k][u] -= self._dots([(x, self._mask_(self._mixed(k, plan, Q)))])[0]
        return G


class _Anderson:
    """Anderson type-II history for the CD solver (blml_binned.py:239-250, 1463-1478): the differences dX, dF of the
    last m + 1 iterates and their float64 Gram matrix, kept up to date with one multi-dot pass per sweep."""

    def __init__(self, fit, m):
        self.fit, self.m = fit, m
        self.reset()

    def reset(self):
        self.pX = self.pF = None
        self.dX, self.dF = [], []
        self.G = np.zeros((0, 0))

    def step(self, E, f):
        """Record (E, f); return the mixed candidate E + f - sum g_i (dX_i + dF_i), or None (fewer than 3 iterates,
        or a singular / non-finite solve, which clears the history as the reference does)."""
        fit = self.fit
        if self.pX is not None:
            self.dX.append(fit._lin([(1.0, E), (-1.0, self.pX)]))
            self.dF.append(fit._lin([(1.0, f), (-1.0, self.pF)]))
            if len(self.dF) > self.m:
                self.dX.pop(0); self.dF.pop(0); self.G = self.G[1:, 1:]
        self.pX, self.pF = E.clone(), f.clone()
        if not self.dF:
            return None
        k = len(self.dF)
        pairs = [(self.dF[-1], self.dF[i]) for i in range(k)] + [(self.dF[i], f) for i in range(k)]
        vals = fit._dots(pairs)
        G = np.zeros((k, k)); G[:k - 1, :k - 1] = self.G
        G[k - 1, :] = G[:, k - 1] = vals[:k]
        self.G = G
        if k < 2:
            return None
        rhs = np.array(vals[k:2 * k])
        try:
            gam = np.linalg.solve(G + 1e-12 * np.trace(G) * np.eye(k), rhs)
            if not np.all(np.isfinite(gam)):
                raise np.linalg.LinAlgError
        except np.linalg.LinAlgError:
            self.reset()
            return None
        terms = [(1.0, E), (1.0, f)] + [(float(-gam[i]), self.dX[i]) for i in range(k)] + \
                [(float(-gam[i]), self.dF[i]) for i in range(k)]
        return fit._lin(terms)


def _solve_tri(A, b, upper):
    import scipy.linalg
    return scipy.linalg.solve_triangular(A, b, lower=not upper)
