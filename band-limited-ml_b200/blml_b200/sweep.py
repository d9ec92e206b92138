"""Many BLMLBinned fits in lockstep on one GPU: the cut-off sweep (selector._search, selector.py:488-553; the binned
sweeps of dslit_job.py:158-171 and results/p3_window_pball.py:27-30) and rolling windows run their fits one after
another through the reference's single-fit solver (blml_binned.py:223-355); here F fits of uneven lattice size and
cut-off advance together, every phase one launch over all fits (csrc/batched.cu, grouped mat-vecs in
csrc/matvec.cu). With control='device' (the default) the per-fit decisions (Anderson weights, the L-BFGS direction,
Armijo choices, stop rules) run as kernels too and each phase is a CUDA graph of a ring of iterations, replayed until
every fit has stopped (csrc/batch_runner.cu); control='host' makes the same decisions in vectorised NumPy with a few
host syncs per iteration.

    batch = BLMLBinnedBatch(tol=1e-6, dtype=np.float64)
    fits = batch.fit(counts_list, modes_list)              # complex_g, L-BFGS
    fits[i].loglik_, fits[i].density_, fits[i].n_sweeps_, fits[i].stop_reason_
    scores = batch.log_density(val_counts_list)            # held-out scores, one launch for all fits

Each fit is the reference's algorithm: the real rank-1 start under the fit's kernel by Jacobi coordinate updates
with Anderson mixing and the merit safeguard (in float64, see BLMLBinned._start), the seeded phases, L-BFGS ascent
of L = sum w log F - n log Q with Armijo backtracking (the first of t = 1, 1/2, ..., 2^-39 that passes; all forty
trials in one pass), memory 20, U = S E recomputed at every accepted step, the canonical form at the end. One mode
per fit (shared kernel), complex_g."""
import ctypes as C
from collections import OrderedDict

import numpy as np
import torch

from . import _lib
from ._lib import call, ptrs
from .spec import parse_modes, spec_key
from .operator import pad_rule, mode_transform, kernel_at_zero, Plan

NT = 40
_PLANS = OrderedDict()          # (kernel spec, lattice, dtype, device) -> (Plan, K(0))
_PLAN_CACHE_SIZE = 512
STOP_CODES = ('tol', 'll_tol', 'stall')


class _Seg(C.Structure):
    _fields_ = [('off', C.c_int64), ('boff', C.c_int64), ('B', C.c_int64), ('K', C.c_int32), ('pad', C.c_int32)]


class FitResult:
    """One fit of a batch: the attributes of a BLMLBinned fit (host NumPy)."""

    def __init__(self, **kw):
        self.__dict__.update(kw)

    @property
    def density_(self):
        return self._batch.density(self._f)


class _Group:
    """One grouped mat-vec: problem g applies plans[g] to nbatch[g] lattices from x_off[g] (default one each)."""

    def __init__(self, plans, x, x_off, y, y_off, x_complex, nbatch=None):
        G = len(plans)
        arr = (C.c_void_p * G)(*[p._h.value for p in plans])
        nb = np.ones(G, np.int32) if nbatch is None else np.ascontiguousarray(nbatch, np.int32)
        xo = np.ascontiguousarray(x_off, np.int64); yo = np.ascontiguousarray(y_off, np.int64)
        h = C.c_void_p()
        call('blml_group_create', G, C.cast(arr, C.c_void_p), nb.ctypes.data_as(C.c_void_p), int(x_complex),
             x.data_ptr(), xo.ctypes.data_as(C.c_void_p), y.data_ptr(), yo.ctypes.data_as(C.c_void_p), C.byref(h))
        self._h = h; self._keep = (plans, x, y)

    def __call__(self, stream):
        call('blml_group_matvec', self._h, stream)

    @property
    def route(self):
        return int(_lib.lib().blml_group_route(self._h))

    @route.setter
    def route(self, r):
        call('blml_group_set_route', self._h, int(r))

    def __del__(self):
        if getattr(self, '_h', None) is not None and self._h.value and _lib._lib is not None:
            _lib.lib().blml_group_destroy(self._h)


class BLMLBinnedBatch:
    """F independent complex one-mode BLMLBinned fits (L-BFGS) in lockstep; see the module docstring."""

    def __init__(self, tol=1e-5, max_sweeps=None, anderson=5, dtype=np.float64, phase_noise=0.1, seed=0, stall=1000,
                 ll_tol=None, ll_window=100, lbfgs_m=20, device=None, verbose=False, control='device'):
        self.tol, self.max_sweeps, self.anderson = tol, max_sweeps, anderson
        self.dtype = np.dtype(dtype); self.phase_noise, self.seed, self.stall = phase_noise, seed, stall
        self.ll_tol, self.ll_window, self.lbfgs_m = ll_tol, ll_window, int(lbfgs_m)
        self.device = torch.device(device or 'cuda'); self.verbose = verbose
        if self.lbfgs_m > 20:
            raise ValueError("lbfgs_m: at most 20")
        if control not in ('device', 'host'):
            raise ValueError("control: 'device' (per-fit decisions in kernels, CUDA graphs) or 'host'")
        if control == 'device' and not 0 <= anderson <= 8:
            raise ValueError("anderson: 0..8 with control='device'")
        self.control = control

    # ---------------------------------------------------------------- set-up
    def _plan(self, sp, shape, code):
        key = (spec_key(sp), tuple(shape), code, str(self.device))
        hit = _PLANS.pop(key, None)
        if hit is None:
            h = np.ones(2)
            freqs, W = mode_transform(sp, shape, h, pad_rule(shape, h, [sp]))
            with torch.cuda.device(self.device):
                hit = (Plan(freqs, W, shape, code, _lib.ENGINE_SIMT), kernel_at_zero(sp, 2))
        _PLANS[key] = hit                                   # most recent last
        while len(_PLANS) > _PLAN_CACHE_SIZE:
            _PLANS.popitem(last=False)
        return hit

    def _prepare(self, counts_list, modes_list):
        if not torch.cuda.is_available():
            raise _lib.BLMLError('BLMLBinnedBatch needs a CUDA device (no CPU path)')
        dev = self.device
        F = len(counts_list)
        if F < 1 or len(modes_list) != F:
            raise ValueError("one modes list per counts array")
        self.F = F
        f32 = self.dtype == np.float32
        self.code = _lib.F32 if f32 else _lib.F64
        self.rt = torch.float32 if f32 else torch.float64
        self.ct = torch.complex64 if f32 else torch.complex128
        shapes, specs, parts, Ks = [], [], [], []
        for counts, modes in zip(counts_list, modes_list):
            if isinstance(counts, torch.Tensor):            # counts already on the device stay there
                ct = counts.to(dev, torch.float64)
            else:
                ct = torch.as_tensor(np.asarray(counts, float)).to(dev)
            if ct.ndim != 2:
                raise ValueError("counts: non-negative finite 2-D arrays")
            sp, dep = parse_modes(modes, 2)
            if dep is not None or len(sp) < 1 or any(spec_key(x) != spec_key(sp[0]) for x in sp):
                raise ValueError("BLMLBinnedBatch fits K modes of one shared kernel per lattice")
            shapes.append(tuple(ct.shape)); specs.append(sp[0]); Ks.append(len(sp)); parts.append(ct.reshape(-1))
        w64 = torch.cat(parts)
        if bool(((w64 < 0) | ~torch.isfinite(w64)).any()):
            raise ValueError("counts: non-negative finite 2-D arrays")
        self.n = torch.stack([p.sum() for p in parts]).cpu().numpy()
        if not np.all(self.n > 0):
            raise ValueError("counts: no observations")
        self.shapes, self.specs = shapes, specs
        self.Kf = np.array(Ks, np.int64)
        self.B = np.array([a * b for a, b in shapes], np.int64)
        boff = np.concatenate([[0], np.cumsum(self.B)])
        self.boff = boff
        moff = np.concatenate([[0], np.cumsum(self.Kf * self.B)])     # mode arrays: fit f owns K_f lattices
        self.moff = moff
        self.Mtot = int(moff[-1])
        self.segs_all = [_Seg(int(moff[f]), int(boff[f]), int(self.B[f]), int(self.Kf[f]), 0) for f in range(F)]
        segs = (_Seg * F)(*self.segs_all)
        self.segs_t = torch.frombuffer(bytearray(segs), dtype=torch.uint8).to(dev)
        self.Btot = int(boff[-1])
        self.w64 = w64
        self.w = w64.to(self.rt)
        self.c64 = w64 * torch.as_tensor(np.repeat(self.n, self.B)).to(dev)
        self.c = self.c64.to(self.rt)
        self.sg64 = torch.ones(self.Btot, dtype=torch.float64, device=dev); self.sg = self.sg64.to(self.rt)
        nb = _lib.lib().blml_seg_blocks()
        self.part = torch.empty(48 * F * nb + 64, dtype=torch.float64, device=dev)
        self.out = torch.empty(48 * F + 64, dtype=torch.float64, device=dev)
        self.host = torch.empty(48 * F + 64, dtype=torch.float64, pin_memory=True)
        # plans (cached across batches): float64 for the start, the fit dtype for the L-BFGS
        self.p64, self.pfit, s0 = [], [], []
        for shape, sp in zip(shapes, specs):
            p64, k0 = self._plan(sp, shape, _lib.F64)
            self.p64.append(p64); s0.append(k0)
            self.pfit.append(p64 if not f32 else self._plan(sp, shape, _lib.F32)[0])
        self.s = np.array(s0)
        self.s_t = torch.as_tensor(self.s, dtype=torch.float64).to(dev)
        self.st = torch.cuda.current_stream(dev).cuda_stream

    # ---------------------------------------------------------------- device helpers
    def _read(self, nq):
        self.host[:nq * self.F].copy_(self.out[:nq * self.F], non_blocking=True)
        torch.cuda.current_stream(self.device).synchronize()
        return self.host[:nq * self.F].numpy().reshape(self.F, nq).copy()

    def _dots(self, code, cplx, pairs):
        call('blml_seg_dots', code, self.F, self.segs_t.data_ptr(), int(cplx), len(pairs), ptrs([p[0] for p in pairs]),
             ptrs([p[1] for p in pairs]), self.part.data_ptr(), self.out.data_ptr(), self.st)
        return self._read(len(pairs))

    def _lin(self, code, cplx, out, coef, vecs):
        """out = sum_i coef[:, i] v_i per fit (coef (F, nterms))."""
        cf = torch.as_tensor(np.ascontiguousarray(coef, np.float64)).to(self.device, non_blocking=True)
        call('blml_seg_lincomb', code, self.F, self.segs_t.data_ptr(), int(cplx), out.data_ptr(), len(vecs),
             cf.data_ptr(), ptrs(vecs), self.st)
        return out

    def _dev(self, a):
        return torch.as_tensor(np.ascontiguousarray(a, np.float64)).to(self.device, non_blocking=True)

    # ---------------------------------------------------------------- the real rank-1 start (float64)
    def _start(self):
        """Jacobi updates + Anderson (m = anderson) + the merit safeguard (blml_binned.py:223-276 with psd False),
        float64, every fit at once; returns the real roots E (flat float64)."""
        F, code, dev = self.F, _lib.F64, self.device
        E = torch.empty(self.Btot, dtype=torch.float64, device=dev)
        call('blml_seg_start_root', code, F, self.segs_t.data_ptr(), self.c64.data_ptr(), self.sg64.data_ptr(),
             self.s_t.data_ptr(), E.data_ptr(), self.st)
        U = torch.zeros_like(E)
        EJ, UJ, EA, UA, ET, UT, f = (torch.zeros_like(E) for _ in range(7))
        mA = self.anderson
        DX = [torch.zeros_like(E) for _ in range(mA)]; DF = [torch.zeros_like(E) for _ in range(mA)]
        pX, pF = torch.zeros_like(E), torch.zeros_like(E)
        g_EU = _Group(self.p64, E, self.boff[:-1], U, self.boff[:-1], False)
        g_J = _Group(self.p64, EJ, self.boff[:-1], UJ, self.boff[:-1], False)
        g_A = _Group(self.p64, EA, self.boff[:-1], UA, self.boff[:-1], False)
        n = self.n
        g_EU(self.st)

        def rescale(E_, U_, where=None):
            Q = self._dots(code, False, [(E_, U_)])[:, 0]
            sc = np.where(Q > 0, n / np.sqrt(np.maximum(Q, 1e-300)), 1.0)
            if where is not None:
                sc = np.where(where, sc, 1.0)
            self._lin(code, False, E_, sc[:, None], [E_]); self._lin(code, False, U_, sc[:, None], [U_])

        def merit(E_, U_):
            call('blml_seg_merit', code, F, self.segs_t.data_ptr(), 0, 0, E_.data_ptr(), U_.data_ptr(),
                 self.c64.data_ptr(), self.sg64.data_ptr(), self.part.data_ptr(), self.out.data_ptr(), self.st)
            r = self._read(3)
            m = -(0.5 * r[:, 0] - r[:, 1]) / n
            return np.where(r[:, 2] > 0, -np.inf, m)

        def resid(E_, U_):
            call('blml_seg_resid', code, F, self.segs_t.data_ptr(), 0, E_.data_ptr(), U_.data_ptr(),
                 self.c64.data_ptr(), self._dev(np.ones(F)).data_ptr(), self.part.data_ptr(), self.out.data_ptr(),
                 self.st)
            r = self._read(2)
            return np.where(r[:, 1] > 0, np.nan, r[:, 0])

        rescale(E, U)
        cur = merit(E, U); res = resid(E, U)
        active = res >= self.tol
        it = np.zeros(F, np.int64); best_res = res.copy(); best_it = np.zeros(F, np.int64); best_m = cur.copy()
        cap = np.inf if self.max_sweeps is None else self.max_sweeps
        valid = np.zeros((F, mA), bool); has_prev = np.zeros(F, bool)
        G = np.zeros((F, mA, mA))
        sweep = 0
        while active.any():
            stalled = active & (it - best_it >= self.stall)
            active &= ~stalled & (it < cap)
            if not active.any():
                break
            it += active
            call('blml_seg_update_real1', code, F, self.segs_t.data_ptr(), E.data_ptr(), U.data_ptr(),
                 self.c64.data_ptr(), self.sg64.data_ptr(), self.s_t.data_ptr(), EJ.data_ptr(), self.st)
            g_J(self.st)
            mJ = merit(EJ, UJ)
            take_A = np.zeros(F, bool)
            if mA:
                self._lin(code, False, f, np.tile([1.0, -1.0], (F, 1)), [EJ, E])
                p = sweep % mA
                # the new differences go to slot p for every fit (slots written before a fit's last reset are
                # invalid for it); the Anderson solve is invariant to the order of its columns
                self._lin(code, False, DX[p], np.tile([1.0, -1.0], (F, 1)), [E, pX])
                self._lin(code, False, DF[p], np.tile([1.0, -1.0], (F, 1)), [f, pF])
                valid[:, p] = has_prev & active
                vals = self._dots(code, False, [(DF[p], DF[q]) for q in range(mA)] + [(DF[q], f) for q in range(mA)])
                G[:, p, :] = vals[:, :mA]; G[:, :, p] = vals[:, :mA]
                rhs = vals[:, mA:]
                self._lin(code, False, pX, np.ones((F, 1)), [E]); self._lin(code, False, pF, np.ones((F, 1)), [f])
                has_prev |= active
                k = valid.sum(1)
                use = active & (k >= 2)
                gam = np.zeros((F, mA))
                for fi in np.where(use)[0]:
                    vv = np.where(valid[fi])[0]
                    Gs = G[fi][np.ix_(vv, vv)]
                    try:
                        gg = np.linalg.solve(Gs + 1e-12 * np.trace(Gs) * np.eye(len(vv)), rhs[fi, vv])
                        if not np.all(np.isfinite(gg)):
                            raise np.linalg.LinAlgError
                        gam[fi, vv] = gg
                    except np.linalg.LinAlgError:
                        valid[fi] = False; has_prev[fi] = False; use[fi] = False
                if use.any():
                    coef = np.concatenate([np.ones((F, 2)), -gam, -gam], 1)
                    coef[~use] = 0.0; coef[~use, 0] = 1.0          # fits without a mix: EA = E (unused)
                    self._lin(code, False, EA, coef, [E, f] + DX + DF)
                    g_A(self.st)
                    mAc = merit(EA, UA)
                    take_A = use & (mAc > mJ)
                    mJ = np.where(take_A, mAc, mJ)
            # candidate: the Anderson point where it won, else the Jacobi point
            ta = take_A.astype(float)
            self._lin(code, False, ET, np.stack([ta, 1 - ta], 1), [EA, EJ])
            self._lin(code, False, UT, np.stack([ta, 1 - ta], 1), [UA, UJ])
            damp = active & (mJ < cur - 1e-12 * np.abs(cur))
            if damp.any():                                   # no ascent: damp the Jacobi step, a = 0.5, 0.25, ...
                valid[damp] = False; has_prev[damp] = False
                a = np.where(damp, 0.5, 0.0); searching = damp.copy(); found = np.zeros(F, bool)
                while searching.any():
                    am = np.where(searching, a, 0.0)
                    self._lin(code, False, EA, np.stack([1 - am, am], 1), [E, EJ])
                    self._lin(code, False, UA, np.stack([1 - am, am], 1), [U, UJ])
                    mt = merit(EA, UA)
                    ok = searching & (mt >= cur)
                    sel = ok.astype(float)[:, None]
                    self._lin(code, False, ET, np.concatenate([sel, 1 - sel], 1), [EA, ET])
                    self._lin(code, False, UT, np.concatenate([sel, 1 - sel], 1), [UA, UT])
                    mJ = np.where(ok, mt, mJ); found |= ok
                    searching &= ~ok
                    a = a * 0.5
                    searching &= a > 1e-8
                stay = damp & ~found                         # no step found: the iterate stays (psd False: no gradient)
                st = stay.astype(float)[:, None]
                self._lin(code, False, ET, np.concatenate([st, 1 - st], 1), [E, ET])
                self._lin(code, False, UT, np.concatenate([st, 1 - st], 1), [U, UT])
                mJ = np.where(stay, cur, mJ)
            act = active.astype(float)[:, None]
            self._lin(code, False, E, np.concatenate([act, 1 - act], 1), [ET, E])
            self._lin(code, False, U, np.concatenate([act, 1 - act], 1), [UT, U])
            rescale(E, U, active)
            cur = np.where(active, merit(E, U), cur)
            r = resid(E, U)
            res = np.where(active, r, res)
            improved = active & ((res < 0.9 * best_res) | (cur > best_m + 1e-13 * np.abs(best_m)))
            best_res = np.where(improved, np.minimum(res, best_res), best_res)
            best_it = np.where(improved, it, best_it); best_m = np.where(improved, np.maximum(cur, best_m), best_m)
            active &= res >= self.tol
            sweep += 1
        self.start_sweeps_ = it
        return E

    def _start_device(self):
        """The same start with its per-fit decisions on the device (blml_start_batch_*: CUDA graphs of `anderson`
        sweeps replayed until every fit has stopped)."""
        F = self.F
        E = torch.empty(self.Btot, dtype=torch.float64, device=self.device)
        segs = (_Seg * F)(*self.segs_all)
        plans = (C.c_void_p * F)(*[p._h.value for p in self.p64])
        h = C.c_void_p()
        n = np.ascontiguousarray(self.n, np.float64); s0 = np.ascontiguousarray(self.s, np.float64)
        call('blml_start_batch_create', F, C.cast(segs, C.c_void_p), C.cast(plans, C.c_void_p), int(self.anderson),
             float(self.tol), -1 if self.max_sweeps is None else int(self.max_sweeps), int(self.stall),
             n.ctypes.data_as(C.c_void_p), s0.ctypes.data_as(C.c_void_p), self.c64.data_ptr(), self.sg64.data_ptr(),
             E.data_ptr(), C.byref(h))
        try:
            call('blml_start_batch_run', h, self.st)
            sweeps = np.zeros(F, np.int64)
            call('blml_start_batch_result', h, sweeps.ctypes.data_as(C.c_void_p), None)
            stats = np.zeros(4, np.int64)
            call('blml_start_batch_stats', h, stats.ctypes.data_as(C.c_void_p))
        finally:
            _lib.lib().blml_start_batch_destroy(h)
        self.start_sweeps_ = sweeps
        self.start_stats_ = dict(zip(('sweeps', 'replays', 'captures', 'kernels_per_replay'), stats.tolist()))
        return E

    def _lbfgs_device(self, E):
        """L-BFGS of every fit with its per-fit decisions on the device (blml_lbfgs_batch_*); returns U and the
        per-fit iterations, stop reasons, L and residuals."""
        F = self.F
        U = torch.zeros_like(E)
        segs = (_Seg * F)(*self.segs_all)
        plans = (C.c_void_p * F)(*[p._h.value for p in self.pfit])
        h = C.c_void_p()
        n = np.ascontiguousarray(self.n, np.float64)
        ftol = self.ll_tol if self.ll_tol is not None else 1e-11
        call('blml_lbfgs_batch_create', self.code, F, C.cast(segs, C.c_void_p), C.cast(plans, C.c_void_p),
             self.lbfgs_m, float(self.tol), float(ftol), -1 if self.max_sweeps is None else int(self.max_sweeps),
             n.ctypes.data_as(C.c_void_p), self.w.data_ptr(), self.c.data_ptr(), E.data_ptr(), U.data_ptr(),
             C.byref(h))
        try:
            if getattr(self, '_caps', None) is not None:
                caps = np.ascontiguousarray(self._caps, np.int64)
                call('blml_lbfgs_batch_set_caps', h, caps.ctypes.data_as(C.c_void_p))
            if getattr(self, '_history_f32', False):
                call('blml_lbfgs_batch_set_history', h, 1)
            call('blml_lbfgs_batch_run', h, self.st)
            it = np.zeros(F, np.int64); stop = np.zeros(F, np.int32); L = np.zeros(F); res = np.zeros(F)
            call('blml_lbfgs_batch_result', h, it.ctypes.data_as(C.c_void_p), stop.ctypes.data_as(C.c_void_p),
                 L.ctypes.data_as(C.c_void_p), None, res.ctypes.data_as(C.c_void_p))
            stats = np.zeros(4, np.int64)
            call('blml_lbfgs_batch_stats', h, stats.ctypes.data_as(C.c_void_p))
        finally:
            _lib.lib().blml_lbfgs_batch_destroy(h)
        self.lbfgs_stats_ = dict(zip(('iterations', 'replays', 'captures', 'kernels_per_replay'), stats.tolist()))
        return U, it, np.array(STOP_CODES, dtype=object)[stop], L, res

    # ---------------------------------------------------------------- fit
    def fit(self, counts_list, modes_list, init=None, caps=None):
        """init: None (the seeded start), or one complex start E0 per fit (arrays of the counts' shapes, host or
        device), e.g. from blml_b200.warmstart; the start phase is then skipped (blml_binned.py:403-408). caps: per-fit
        L-BFGS iteration caps (< 0: none but max_sweeps) in place of max_sweeps (device-side control)."""
        if caps is not None and self.max_sweeps is not None:
            caps = np.asarray(caps, np.int64)
            caps = np.where(caps < 0, int(self.max_sweeps), np.minimum(caps, int(self.max_sweeps)))
        self._caps = caps
        self._prepare(counts_list, modes_list)
        F, code, dev = self.F, self.code, self.device
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        ev[0].record()
        if init is not None:
            if len(init) != F:
                raise ValueError("init: one start per fit")
            parts = []
            for e0, shape, K in zip(init, self.shapes, self.Kf):
                t = e0 if isinstance(e0, torch.Tensor) else torch.as_tensor(np.asarray(e0, complex))
                if tuple(t.shape) not in ((int(K),) + tuple(shape),) + ((tuple(shape),) if K == 1 else ()):
                    raise ValueError("init: each start has its counts' shape, (K,) + shape for K modes")
                parts.append(t.to(dev, self.ct).reshape(-1))
            E = torch.cat(parts)
            # a start's coefficients on bins these counts leave empty are zeroed (blml_binned.py:403-408)
            occm = (self.w > 0).to(self.rt)
            if np.all(self.Kf == 1):
                call('blml_mul_bins', code, 1, self.Btot, 1, E.data_ptr(), occm.data_ptr(), E.data_ptr(), self.st)
            else:
                for f in range(F):
                    sg = self.segs_all[f]
                    Ef, of = E[sg.off:sg.off + sg.K * sg.B], occm[sg.boff:sg.boff + sg.B]
                    call('blml_mul_bins', code, int(sg.K), int(sg.B), 1, Ef.data_ptr(), of.data_ptr(), Ef.data_ptr(),
                         self.st)
            self.start_sweeps_ = np.zeros(F, np.int64)
        else:
            if np.any(self.Kf != 1):
                raise ValueError("fits of K > 1 modes start from init (e.g. a lower-rank fit and a new direction)")
            er = self._start_device() if self.control == 'device' else self._start()
            # complex start: the real root with the seeded phases exp(i pn N(0,1)) (blml_binned.py:429-436)
            E = torch.zeros(self.Btot, dtype=self.ct, device=dev)
            er_fit = er.to(self.rt)
            call('blml_seg_real_to_complex', code, F, self.segs_t.data_ptr(), self.segs_t.data_ptr(),
                 er_fit.data_ptr(), E.data_ptr(), self.st)
            z = np.concatenate([np.random.default_rng(self.seed).standard_normal(shape).ravel()
                                for shape in self.shapes])
            zt = torch.as_tensor(z, dtype=torch.float64).to(dev)
            call('blml_seg_phases', code, F, self.segs_t.data_ptr(), float(self.phase_noise), zt.data_ptr(),
                 E.data_ptr(), self.st)
        ev[1].record()
        if self.control == 'device':
            U, it, stop, L, res = self._lbfgs_device(E)
        else:
            U, it, stop, L, res = self._lbfgs(E)
        ev[2].record()
        out = self._finish(E, U, it, stop, L, res)
        ev[3].record(); ev[3].synchronize()
        self.timing_ = dict(start_s=ev[0].elapsed_time(ev[1]) / 1e3, lbfgs_s=ev[1].elapsed_time(ev[2]) / 1e3,
                            finish_s=ev[2].elapsed_time(ev[3]) / 1e3)
        return out

    def _lbfgs(self, E):
        """L-BFGS of every fit with the per-fit decisions on the host (vectorised NumPy, a few syncs per iteration);
        returns U and the per-fit iterations, stop reasons, L and residuals."""
        F, code, dev, n, m_ = self.F, self.code, self.device, self.n, self.lbfgs_m
        U, g, gn, q, Sq, V, SV = (torch.zeros_like(E) for _ in range(7))
        Sh = [torch.zeros_like(E) for _ in range(m_)]; Yh = [torch.zeros_like(E) for _ in range(m_)]
        off = self.moff[:-1]
        g_EU = _Group(self.pfit, E, off, U, off, True, self.Kf)
        g_q = _Group(self.pfit, q, off, Sq, off, True, self.Kf)
        g_V = _Group(self.pfit, V, off, SV, off, True, self.Kf)
        segs = self.segs_t.data_ptr()

        def Qdot(E_, U_):
            return self._dots(code, True, [(E_, U_)])[:, 0]

        def grad(Qv):
            """V = w / F U, S V, g = 2 (S V - n U / Q) for every fit; returns sum w log F per fit."""
            call('blml_seg_lgrad_weights', code, F, segs, 1, U.data_ptr(), self.w.data_ptr(),
                 self._dev(np.ones(F)).data_ptr(), V.data_ptr(), self.part.data_ptr(), self.out.data_ptr(), self.st)
            Lw = self._read(1)[:, 0]
            g_V(self.st)
            call('blml_seg_lgrad_finish', code, F, segs, 1, SV.data_ptr(), U.data_ptr(), self.w.data_ptr(),
                 self._dev(n / Qv).data_ptr(), gn.data_ptr(), self.st)
            return Lw

        def resid(Qv):
            call('blml_seg_resid', code, F, segs, 1, E.data_ptr(), U.data_ptr(), self.c.data_ptr(),
                 self._dev(np.where(Qv > 0, n / np.sqrt(np.maximum(Qv, 1e-300)), 1.0)).data_ptr(),
                 self.part.data_ptr(), self.out.data_ptr(), self.st)
            r = self._read(2)
            return np.where(r[:, 1] > 0, np.nan, r[:, 0])

        g_EU(self.st)
        Q = Qdot(E, U)
        sc = np.where(Q > 0, n / np.sqrt(np.maximum(Q, 1e-300)), 1.0)
        self._lin(code, True, E, sc[:, None], [E]); self._lin(code, True, U, sc[:, None], [U])
        Q = Q * sc * sc
        Lw = grad(Q)
        self._lin(code, True, g, np.ones((F, 1)), [gn])
        L = Lw - n * np.log(Q)
        res = resid(Q)
        stamp = np.full((F, m_), -1, np.int64)             # iteration at which each slot's pair entered (-1: empty)
        SY = np.zeros((F, m_, m_)); YY = np.zeros((F, m_, m_))
        it = np.zeros(F, np.int64); active = res >= self.tol
        reset = np.zeros(F, bool); stop = np.array(['tol'] * F, dtype=object)
        ftol, fwin = (self.ll_tol if self.ll_tol is not None else 1e-11), 10
        mhist = [L / n]
        cap = np.inf if self.max_sweeps is None else self.max_sweeps
        step = 0
        while active.any():
            if len(mhist) > fwin:
                lt = active & (mhist[-1] - mhist[-1 - fwin] < ftol)
                stop[lt] = 'll_tol'; active &= ~lt
            active &= it < cap
            if not active.any():
                break
            it += active
            # ---- direction (compact L-BFGS over each fit's chronologically ordered pairs)
            vals = self._dots(code, True, [(s, g) for s in Sh] + [(y, g) for y in Yh] + [(g, g), (E, E)])
            a_all, b_all = vals[:, :m_], vals[:, m_:2 * m_]; gg, ee = vals[:, 2 * m_], vals[:, 2 * m_ + 1]
            first = 1e-3 * np.sqrt(ee / np.maximum(gg, 1e-300))
            coef = np.zeros((F, 1 + 2 * m_)); slope = np.zeros(F)
            for fi in range(F):
                if not active[fi]:
                    continue
                occ = np.where(stamp[fi] >= 0)[0]
                if len(occ):
                    order = occ[np.argsort(stamp[fi, occ])]
                    R = np.triu(SY[fi][np.ix_(order, order)]); Yy = YY[fi][np.ix_(order, order)]
                    last = order[-1]
                    gam = SY[fi, last, last] / YY[fi, last, last]
                    a_, b_ = a_all[fi, order], b_all[fi, order]
                    try:
                        import scipy.linalg as sl
                        t_ = sl.solve_triangular(R, a_, lower=False)
                        p_ = sl.solve_triangular(R.T, (np.diag(np.diag(R)) + gam * Yy) @ t_ - gam * b_, lower=True)
                        coef[fi, 0] = gam; coef[fi, 1 + order] = p_; coef[fi, 1 + m_ + order] = -gam * t_
                        slope[fi] = gam * gg[fi] + a_ @ p_ - gam * b_ @ t_
                    except (np.linalg.LinAlgError, ValueError):
                        slope[fi] = -1.0
                if not len(occ) or not slope[fi] > 0:
                    if len(occ):
                        stamp[fi] = -1
                    coef[fi] = 0.0; coef[fi, 0] = first[fi]; slope[fi] = first[fi] * gg[fi]
            self._lin(code, True, q, coef, [g] + Sh + Yh)
            g_q(self.st)
            # ---- every fit's Armijo search in one pass
            call('blml_seg_trials', code, F, segs, 1, E.data_ptr(), q.data_ptr(), U.data_ptr(), Sq.data_ptr(),
                 self.w.data_ptr(), self.part.data_ptr(), self.out.data_ptr(), self.st)
            tr = self._read(NT + 3)
            ts = 0.5 ** np.arange(NT)
            Qt = Q[:, None] + ts[None, :] * (tr[:, NT] + tr[:, NT + 1])[:, None] + ts[None, :] ** 2 * tr[:, NT + 2][:, None]
            with np.errstate(invalid='ignore', divide='ignore'):
                Lt = np.where(Qt > 0, tr[:, :NT] - n[:, None] * np.log(np.where(Qt > 0, Qt, 1.0)), -np.inf)
            okt = Lt >= L[:, None] + 1e-4 * ts[None, :] * slope[:, None]
            ok = okt.any(1) & active
            j = np.argmax(okt, 1)
            t = np.where(ok, ts[j], 0.0)
            fail = active & ~ok
            stall = fail & (reset | (stamp < 0).all(1))
            stop[stall] = 'stall'; active &= ~stall
            retry = fail & ~stall
            stamp[retry] = -1; reset = np.where(retry, True, np.where(ok, False, reset))
            # ---- the accepted steps: E += t q, then U = S E exactly
            call('blml_seg_axpy2', code, F, segs, 1, E.data_ptr(), q.data_ptr(), U.data_ptr(), Sq.data_ptr(),
                 self._dev(t).data_ptr(), self.st)
            g_EU(self.st)
            Qn = Qdot(E, U)
            Lwn = grad(np.where(ok, Qn, Q))
            Ln = np.where(Qn > 0, Lwn - n * np.log(np.where(Qn > 0, Qn, 1.0)), -np.inf)
            # ---- the new pair (s, y) = (t q, g - g_new) into slot p of the fits that stepped
            p = step % m_
            okf = ok.astype(float)
            self._lin(code, True, Sh[p], np.stack([t, 1 - okf], 1), [q, Sh[p]])
            self._lin(code, True, Yh[p], np.stack([okf, -okf, 1 - okf], 1), [g, gn, Yh[p]])
            vals = self._dots(code, True, [(Sh[p], Yh[p]), (Sh[p], Sh[p]), (Yh[p], Yh[p])] +
                              [(s, Yh[p]) for s in Sh] + [(y, Yh[p]) for y in Yh])
            sy, ss, yy = vals[:, 0], vals[:, 1], vals[:, 2]
            enter = ok & (sy > 1e-12 * np.sqrt(np.maximum(ss * yy, 0.0)))
            stamp[ok, p] = -1
            stamp[enter, p] = step
            full = enter & ((stamp >= 0).sum(1) > m_)
            SY[enter, :, p] = vals[enter, 3:3 + m_]; SY[enter, p, p] = sy[enter]
            YY[enter, :, p] = vals[enter, 3 + m_:3 + 2 * m_]; YY[enter, p, :] = YY[enter, :, p]; YY[enter, p, p] = yy[enter]
            for fi in np.where(full)[0]:                   # more than m pairs: the oldest leaves
                live = np.where(stamp[fi] >= 0)[0]
                stamp[fi, live[np.argmin(stamp[fi, live])]] = -1
            # g = g_new on the fits that stepped
            self._lin(code, True, g, np.stack([okf, 1 - okf], 1), [gn, g])
            L = np.where(ok, Ln, L); Q = np.where(ok, Qn, Q)
            r = resid(Q)
            res = np.where(ok, r, res)
            mhist.append(np.where(active, L / n, mhist[-1]))
            conv = active & (res < self.tol)
            active &= ~conv
            step += 1
            if self.verbose and step % 100 == 0:
                print(f'  batch lbfgs {step}: active {int(active.sum())}/{F} max rho {np.nanmax(res):.2e}', flush=True)
        return U, it, stop, L, res

    def _finish(self, E, U, it, stop, L, res):
        """The canonical form per fit (kept unless it loses likelihood), the normalisation, the densities and the
        per-fit results (blml_trivial.py:2646-2650)."""
        F, code, dev, n = self.F, self.code, self.device, self.n
        segs = self.segs_t.data_ptr()
        stop = np.array(stop, dtype=object)
        stop[(stop == 'tol') & (res >= self.tol)] = 'max_sweeps'
        V, SV, tmp = (torch.zeros_like(E) for _ in range(3))
        g_V = _Group(self.pfit, V, self.moff[:-1], SV, self.moff[:-1], True, self.Kf)

        def Qdot(E_, U_):
            return self._dots(code, True, [(E_, U_)])[:, 0]

        Qc = Qdot(E, U)
        call('blml_seg_lgrad_weights', code, F, segs, 1, U.data_ptr(), self.w.data_ptr(), self._dev(Qc / n).data_ptr(),
             V.data_ptr(), self.part.data_ptr(), self.out.data_ptr(), self.st)
        self._read(1)
        g_V(self.st)                                       # SV = S Ec
        Qcc = self._dots(code, True, [(V, SV)])[:, 0]
        call('blml_seg_lgrad_weights', code, F, segs, 1, SV.data_ptr(), self.w.data_ptr(), self._dev(np.ones(F)).data_ptr(),
             tmp.data_ptr(), self.part.data_ptr(), self.out.data_ptr(), self.st)
        Lwc = self._read(1)[:, 0]
        Lc = np.where(Qcc > 0, Lwc - n * np.log(np.where(Qcc > 0, Qcc, 1.0)), -np.inf)
        keep = (Lc >= L - 1e-9 * n).astype(float)[:, None]
        self._lin(code, True, E, np.concatenate([keep, 1 - keep], 1), [V, E])
        self._lin(code, True, U, np.concatenate([keep, 1 - keep], 1), [SV, U])
        Q = Qdot(E, U)
        sc = np.where(Q > 0, n / np.sqrt(np.maximum(Q, 1e-300)), 1.0)
        self._lin(code, True, E, sc[:, None], [E]); self._lin(code, True, U, sc[:, None], [U])
        call('blml_seg_resid', code, F, segs, 1, E.data_ptr(), U.data_ptr(), self.c.data_ptr(),
             self._dev(np.ones(F)).data_ptr(), self.part.data_ptr(), self.out.data_ptr(), self.st)
        r = self._read(2)
        res = np.where(r[:, 1] > 0, np.nan, r[:, 0])
        dens = torch.empty(self.Btot, dtype=self.rt, device=dev)
        call('blml_seg_finish', code, F, segs, 1, U.data_ptr(), self.w.data_ptr(), self._dev(1.0 / n ** 2).data_ptr(),
             dens.data_ptr(), self.part.data_ptr(), self.out.data_ptr(), self.st)
        ll = self._read(1)[:, 0] / n
        self.E_t, self.U_t, self.dens_t = E, U, dens
        conv = (res < self.tol) | (stop == 'll_tol')
        self.results_ = [FitResult(loglik_=float(ll[f]), n_sweeps_=int(it[f]), stop_reason_=str(stop[f]),
                                   residual_=float(res[f]), converged_=bool(conv[f]), n_=float(n[f]),
                                   shape_=self.shapes[f], start_sweeps_=int(self.start_sweeps_[f]), _batch=self, _f=f)
                         for f in range(F)]
        return self.results_

    def field(self, f):
        """u = S e / n of fit f on the device (complex, the counts' shape; (K,) + shape for K modes): sum_k |u_k|^2
        is the density."""
        a, b = self.moff[f], self.moff[f + 1]
        shp = self.shapes[f] if self.Kf[f] == 1 else (int(self.Kf[f]),) + self.shapes[f]
        return (self.U_t[a:b] / float(self.n[f])).reshape(shp)

    def e_hat(self, f):
        """The coefficients of fit f on the device, (K,) + the counts' shape (blml_binned.py e_hat_)."""
        a, b = self.moff[f], self.moff[f + 1]
        return self.E_t[a:b].reshape((int(self.Kf[f]),) + self.shapes[f])

    def density(self, f):
        a, b = self.boff[f], self.boff[f + 1]
        return self.dens_t[a:b].cpu().numpy().reshape(self.shapes[f])

    # ---------------------------------------------------------------- certificate and certified fits
    def certificate(self, tol=1e-6, vectors=False, decide_above=None, max_basis=64, second=False):
        """lambda_max(D^1/2 S D^1/2) / n of every fit (blml_binned.py:501-518; D = sum_k |e_k|^2 / w on occupied
        bins), by float64 Lanczos over all fits at once. <= 1 (up to the solver's tolerance) when the fit is the
        optimum of the convex lift. With vectors: (certificates, dh, v), v the top eigenvectors (per bin).
        decide_above: a level (e.g. 1 + cert_tol) past which a fit's value need not be refined -- the Lanczos value is
        a lower bound, so the returned value is then a lower bound above that level. max_basis: the Lanczos basis
        before a restart. second (with vectors): v is a pair (top, second Ritz vectors), the second Ritz values in
        theta2_ (divided by n they compare with the certificate)."""
        from .certificate import lanczos_max_batched
        above = None if decide_above is None else decide_above * self.n
        theta, dh, v = lanczos_max_batched(self, tol=tol, seed=self.seed, vectors=vectors, above=above,
                                           max_basis=max_basis, second=second)
        cert = theta / self.n
        return (cert, dh, v) if vectors else cert

    def _grown_starts(self, grow, dh, v, step, v2=None, two=()):
        """Starts of rank K_f + 1 for the fits `grow` (indices into this batch): the K_f modes, then
        step * sqrt(sum |e|^2 / K_f) / |d| * d with d = dh v (device tensors, one (K_f + 1, M1, M2) start per fit).
        The fits in `two` take a second new mode the same way along d2 = dh v2 (rank K_f + 2)."""
        F, code, dev = self.F, self.code, self.device
        ee = self._dots(code, True, [(self.E_t, self.E_t)])[:, 0]
        segs1 = (_Seg * F)(*[_Seg(int(self.boff[f]), int(self.boff[f]), int(self.B[f]), 1, 0) for f in range(F)])
        s1 = torch.frombuffer(bytearray(segs1), dtype=torch.uint8).to(dev)

        def scales(vv):                                   # step * sqrt(sum |e|^2 / K) / |dh vv| per fit
            d = torch.empty(self.Btot, dtype=torch.float64, device=dev)
            call('blml_mul_bins', _lib.F64, 1, self.Btot, 0, vv.data_ptr(), dh.data_ptr(), d.data_ptr(), self.st)
            call('blml_seg_dots', _lib.F64, F, s1.data_ptr(), 0, 1, ptrs([d]), ptrs([d]), self.part.data_ptr(),
                 self.out.data_ptr(), self.st)
            dd = self._read(1)[:, 0]
            return step * np.sqrt(ee / self.Kf) / np.sqrt(np.maximum(dd, 1e-300))

        def append(old, add_v, sc):                       # old: [(seg into src)], returns (new segs, En)
            G = len(old)
            nB = np.array([o.B for o in old], np.int64); nK = np.array([o.K + 1 for o in old], np.int64)
            noff = np.concatenate([[0], np.cumsum(nB * nK)])
            new = [_Seg(int(noff[t]), int(old[t].boff), int(nB[t]), int(nK[t]), 0) for t in range(G)]
            return new, noff

        scale = scales(v)
        G = len(grow)
        old = [self.segs_all[j] for j in grow]
        new, noff = append(old, v, scale)
        o_t = torch.frombuffer(bytearray((_Seg * G)(*old)), dtype=torch.uint8).to(dev)
        n_t = torch.frombuffer(bytearray((_Seg * G)(*new)), dtype=torch.uint8).to(dev)
        En = torch.empty(int(noff[-1]), dtype=self.ct, device=dev)
        sc = self._dev(scale[np.asarray(grow)])
        call('blml_seg_append_mode', code, G, o_t.data_ptr(), n_t.data_ptr(), self.E_t.data_ptr(), dh.data_ptr(),
             v.data_ptr(), sc.data_ptr(), En.data_ptr(), self.st)
        starts = [En[noff[t]:noff[t + 1]].reshape((int(new[t].K),) + self.shapes[grow[t]]) for t in range(G)]
        sel = [t for t in range(G) if grow[t] in set(two)]
        if v2 is not None and sel:
            scale2 = scales(v2)
            old2 = [new[t] for t in sel]
            new2, noff2 = append(old2, v2, scale2)
            o2 = torch.frombuffer(bytearray((_Seg * len(sel))(*old2)), dtype=torch.uint8).to(dev)
            n2 = torch.frombuffer(bytearray((_Seg * len(sel))(*new2)), dtype=torch.uint8).to(dev)
            En2 = torch.empty(int(noff2[-1]), dtype=self.ct, device=dev)
            sc2 = self._dev(scale2[np.asarray([grow[t] for t in sel])])
            call('blml_seg_append_mode', code, len(sel), o2.data_ptr(), n2.data_ptr(), En.data_ptr(), dh.data_ptr(),
                 v2.data_ptr(), sc2.data_ptr(), En2.data_ptr(), self.st)
            for u, t in enumerate(sel):
                starts[t] = En2[noff2[u]:noff2[u + 1]].reshape((int(new2[u].K),) + self.shapes[grow[t]])
        return starts

    def fit_certified(self, counts_list, modes_list, cert_tol=1e-3, max_rank=8, step=0.1, init=None, grow_iters=300,
                      grow_margin=1.0, history_f32=True, ll_tol=None, lanczos_basis=64, grow_two_above=None):
        """Certified fits: each fit's one-mode kernel at rank K = 1 (the seeded start, or init), then rounds in one
        batch each: a fit whose certificate lambda_max(D^1/2 S D^1/2) / n exceeds 1 + cert_tol gets one more shared
        mode started along the certificate's top eigenvector, and a fit that meets it after a capped round is run on
        to tol at the same rank and checked again. Rounds before the last rank are capped at grow_iters L-BFGS
        iterations: at too low a rank the solver crawls along the lift's boundary, so those fits only have to show that
        they need another mode. A capped fit whose certificate is above the bar by less than grow_margin times
        cert_tol (default: none) is run on to tol at its rank before it may grow; on the benchmark sweep a margin of
        10 doubled the time, the polished fits crawling at too low a rank. The lift is convex: a fit that meets the certificate at tol is at its unique optimum
        (the reference computes the certificate, blml_binned.py:501-518; the rank growth is this engine's). Results
        carry rank_, certificate_ and rank_path_ [(K, loglik, certificate, iterations, capped), ...].
        history_f32: the L-BFGS history of every round in complex64 storage (the iterate, gradient and line search
        stay float64): the certified optimum does not depend on the path the solver takes to it. ll_tol: the rounds'
        L-BFGS stop on the gain of L / n over 10 iterations (None: the batch's own, 1e-11 by default). lanczos_basis:
        the certificate's Lanczos basis before a restart. grow_two_above: a fit whose certificate exceeds this level,
        and whose second Ritz value is above the bar too, takes two new modes at once (the top two Ritz vectors)."""
        F = len(counts_list)
        first_caps = np.full(F, grow_iters if max_rank > 1 else -1, np.int64)
        self._history_f32 = bool(history_f32)
        own_ll_tol = self.ll_tol
        if ll_tol is not None:
            self.ll_tol = ll_tol
        try:
            self.fit(counts_list, modes_list, init=init, caps=first_caps)
        finally:
            self._history_f32 = False
            self.ll_tol = own_ll_tol
        round_ll_tol = own_ll_tol if ll_tol is None else ll_tol
        final = [None] * F
        paths = [[] for _ in range(F)]
        cur, idx, capped = self, np.arange(F), first_caps >= 0
        self.certify_stats_ = dict(rounds=0, fits_per_round=[], lbfgs_iterations_max=[], seconds_certificate=0.0)
        while True:
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
            ev[0].record()
            two_ok = grow_two_above is not None
            cert, dh, v = cur.certificate(vectors=True, decide_above=1.0 + cert_tol, max_basis=lanczos_basis,
                                          second=two_ok)
            v2 = None
            if two_ok:
                v, v2 = v
                th2 = cur.theta2_ / cur.n
            ev[1].record(); ev[1].synchronize()
            st = self.certify_stats_
            st['seconds_certificate'] += ev[0].elapsed_time(ev[1]) / 1e3
            st['rounds'] += 1; st['fits_per_round'].append(len(idx))
            st['lbfgs_iterations_max'].append(int(max(r.n_sweeps_ for r in cur.results_)))
            st.setdefault('lbfgs_seconds', []).append(round(cur.timing_['lbfgs_s'] + cur.timing_['start_s'], 4))
            st.setdefault('lanczos', []).append(cur.lanczos_stats_)
            nxt_fits, nxt_starts, nxt_caps = [], [], []
            for j, i in enumerate(idx):
                r = cur.results_[j]
                K = int(cur.Kf[j])
                was_capped = bool(capped[j]) and r.stop_reason_ == 'max_sweeps'
                paths[i].append((K, float(r.loglik_), float(cert[j]), int(r.n_sweeps_), was_capped))
                r.certificate_, r.rank_, r.rank_path_ = float(cert[j]), K, paths[i]
                final[i] = r
                ok = cert[j] <= 1.0 + cert_tol
                near = cert[j] <= 1.0 + grow_margin * cert_tol
                if was_capped and (near or K >= max_rank):
                    nxt_fits.append((j, i, K)); nxt_caps.append(-1)            # run on to tol at this rank
                elif not ok and K < max_rank:
                    add = 2 if (two_ok and cert[j] > grow_two_above and th2[j] > 1.0 + cert_tol and
                                K + 2 <= max_rank) else 1
                    nxt_fits.append((j, i, K + add)); nxt_caps.append(grow_iters if K + add < max_rank else -1)
            if not nxt_fits:
                return final
            grow = [j for j, _, K1 in nxt_fits if K1 > int(cur.Kf[j])]
            two = [j for j, _, K1 in nxt_fits if K1 > int(cur.Kf[j]) + 1]
            st['two_mode_growths'] = st.get('two_mode_growths', 0) + len(two)
            grown = dict(zip(grow, cur._grown_starts(grow, dh, v, step, v2=v2, two=two))) if grow else {}
            starts = [grown[j] if j in grown else cur.e_hat(j) for j, _, _ in nxt_fits]
            nxt = BLMLBinnedBatch(tol=self.tol, max_sweeps=self.max_sweeps, anderson=self.anderson, dtype=self.dtype,
                                  phase_noise=self.phase_noise, seed=self.seed, stall=self.stall, ll_tol=round_ll_tol,
                                  ll_window=self.ll_window, lbfgs_m=self.lbfgs_m, device=self.device,
                                  verbose=self.verbose, control=self.control)
            mds = [[modes_list[i][0]] * K1 for _, i, K1 in nxt_fits]
            caps = np.array(nxt_caps, np.int64)
            nxt._history_f32 = bool(history_f32)
            nxt.fit([counts_list[i] for _, i, _ in nxt_fits], mds, init=starts, caps=caps)
            nxt._history_f32 = False
            cur, idx, capped = nxt, np.array([i for _, i, _ in nxt_fits]), caps >= 0

    def val_score(self, counts_list):
        """Per fit: the mean log-probability of the counts (validation counts on the fit's lattice) with bin
        probabilities p = f / sum f over every bin, f floored at 1e-300 (the cut-off search's objective,
        selector.py:712-716); one launch for all fits."""
        m = torch.cat([c.reshape(-1).to(self.device, self.rt) if isinstance(c, torch.Tensor) else
                       torch.as_tensor(np.asarray(c, float).ravel(), dtype=self.rt).to(self.device)
                       for c in counts_list])
        if m.numel() != self.Btot:
            raise ValueError("val_score: one lattice per fit, of the fit's shape")
        call('blml_seg_val_score', self.code, self.F, self.segs_t.data_ptr(), self.dens_t.data_ptr(), m.data_ptr(),
             self.part.data_ptr(), self.out.data_ptr(), self.st)
        r = self._read(3)
        with np.errstate(divide='ignore', invalid='ignore'):
            return (r[:, 1] - r[:, 2] * np.log(r[:, 0])) / r[:, 2]

    def log_density(self, counts_list, eps=0.0):
        """Per fit: mean over the counts of log(f_b + eps), f = F / Q (blml_binned.py:630-645), one launch for all."""
        m = torch.cat([c.reshape(-1).to(self.device, self.rt) if isinstance(c, torch.Tensor) else
                       torch.as_tensor(np.asarray(c, float).ravel(), dtype=self.rt).to(self.device)
                       for c in counts_list])
        Q = self._dots(self.code, True, [(self.E_t, self.U_t)])[:, 0]
        call('blml_seg_log_score', self.code, self.F, self.segs_t.data_ptr(), 1, self.U_t.data_ptr(), m.data_ptr(),
             self._dev(1.0 / Q).data_ptr(), float(eps), self.part.data_ptr(), self.out.data_ptr(), self.st)
        r = self._read(2)
        return r[:, 0] / r[:, 1]


def certified_log_density(results, counts_list, eps=0.0):
    """Per fit of BLMLBinnedBatch.fit_certified's results: the mean log density of counts_list[i] (held-out counts on
    fit i's lattice) under fit i (blml_binned.py:630-645); one launch per batch that holds a final fit."""
    groups = {}
    for i, r in enumerate(results):
        groups.setdefault(id(r._batch), (r._batch, []))[1].append(i)
    out = np.full(len(results), np.nan)
    for b, idx in groups.values():
        mine = {r._f: i for i, r in ((i, results[i]) for i in idx)}
        full = [counts_list[mine[f]] if f in mine else np.zeros(b.shapes[f]) for f in range(b.F)]
        with np.errstate(invalid='ignore', divide='ignore'):     # the batch's other fits score empty counts: 0 / 0
            sc = b.log_density(full, eps)
        for f, i in mine.items():
            out[i] = sc[f]
    return out


class BLMLBinnedRolling:
    """Rolling-window refits of many sequences at once (blml_rolling.py:40-155: BLMLRolling refits one estimator per
    window, each fit warm-started from the previous window's through init=). Each update(windows) takes the next count
    window of every sequence (one lattice per sequence), fits them all in one BLMLBinnedBatch call, each started from
    its sequence's previous fit (the first window from the seeded start), and keeps the new coefficients on the
    device for the next call. Complex one-mode fits (L-BFGS), as BLMLBinnedBatch runs them.

        roll = BLMLBinnedRolling([pball_modes(shape, fc) for shape, fc in zip(shapes, fcs)], tol=1e-6)
        for windows in stream_of_windows:            # one count array per sequence
            fits = roll.update(windows)              # FitResults, one per sequence
    """

    def __init__(self, modes_list, **batch_kw):
        self.modes_list = list(modes_list)
        self.batch_kw = dict(batch_kw)
        self.prev_ = None                             # per sequence: its last coefficients (device)
        self.n_updates_ = 0
        self.history_ = []

    def update(self, windows):
        if len(windows) != len(self.modes_list):
            raise ValueError("update: one window per sequence")
        batch = BLMLBinnedBatch(**self.batch_kw)
        init = None
        if self.prev_ is not None:
            init = []
            for e, w in zip(self.prev_, windows):
                if tuple(e.shape[-2:]) != tuple(np.shape(w)):
                    raise ValueError("update: a sequence's windows share its lattice")
                init.append(e)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        ev[0].record()
        res = batch.fit(list(windows), self.modes_list, init=init)
        ev[1].record(); ev[1].synchronize()
        self.prev_ = [batch.e_hat(f).clone() for f in range(batch.F)]
        self.n_updates_ += 1
        self.history_.append(dict(seconds=ev[0].elapsed_time(ev[1]) / 1e3,
                                  iterations=[r.n_sweeps_ for r in res], warm=init is not None))
        self.batch_ = batch
        return res
