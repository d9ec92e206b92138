"""Counts arriving in batches on one fixed lattice, with kernel-parameter learning (rahuljhu/band-limited-ml,
blml_binned.py:648-1112: _KernelLearner and BLMLBinnedStreaming), on the GPU engine of blml_b200.binned.

The state between batches is the fit's coefficients and S e in device memory. A batch is scored by the current model
(its prequential score, log_density), then its gradient of that score in log fc (implicit_grad / param_grad: the
derivative plans and Hessian-vector products of blml_b200.binned) is pooled, then it is added (held counts times
decay plus the batch) and the coefficients are warm-refitted. Every param_every learning batches the trainable
cut-offs take one Adam step on log fc (sinc / slits / ball) or one hill-climb step (dirichlet / pball harmonics, once
the pooled paired gain of the candidate on the batches exceeds z_se standard errors). fit(batches, epochs) revisits
held batches with leave-batch-out scores. An fc left out of the modes (NaN) is selected at the burn-in by the
selector's search (blml_b200.selector.search) on an 80/20 split of the held counts.

Every array operation runs in libblml_b200.so (the fit's kernels plus the bin-wise streaming kernels
blml_counts_axpy, blml_bin_ratio, blml_new_bins and blml_gain_sums); the host keeps the control flow, the pooled
gradients and the Adam / hill-climb state.
"""
import contextlib

import numpy as np
import torch

from ._lib import call
from .binned import BLMLBinned
from .spec import parse_modes, modes_fc, units_of, split_kind, with_fc
from . import selector as _sel

INTEGER_KINDS = ('dirichlet', 'pball')       # fc moves in whole harmonics: hill-climb, no gradient


def adam_log_step(value, grad, state, lr, betas):
    """One Adam ascent step on log(value) from grad = d/dlog value; state = [m, v, t] updated in place
    (blml_maps.py:19-36, the 'scale' parameter type)."""
    b1, b2 = betas
    state[2] += 1
    t = state[2]
    state[0] = b1 * state[0] + (1 - b1) * grad
    state[1] = b2 * state[1] + (1 - b2) * grad * grad
    step = lr * (state[0] / (1 - b1 ** t)) / (np.sqrt(state[1] / (1 - b2 ** t)) + 1e-12)
    return value * np.exp(step)


def batch_order(nb, groups, rng):
    """Batch indices in random group order (no groups: a random permutation), whole groups together
    (blml_binned.py:1022-1031)."""
    if groups is None:
        return list(rng.permutation(nb))
    u, inv = np.unique(np.asarray(groups), return_inverse=True)
    members = [[] for _ in u]
    for i, k in enumerate(np.ravel(inv)):
        members[k].append(i)
    return [i for k in rng.permutation(len(u)) for i in members[k]]


def _fill(F, free, v):
    F = F.copy()
    F[free] = np.asarray(v, float)
    return F


class BLMLBinnedStreaming(BLMLBinned):
    """BLMLBinned on counts arriving in batches (blml_binned.py:1034-1112); see the module docstring.

    partial_fit(counts) holds counts until burn_in, then adds each batch (the held counts times decay first) and
    refits warm from the current coefficients, to tol or for batch_sweeps sweeps. fit(batches, modes, epochs, ...)
    revisits the batches over epochs. preq_ / history_ record every batch; converged_, epochs_, residual_ the epochs."""

    def __init__(self, decay=1.0, batch_sweeps=None, burn_in=0, fc_update='adam', lr=0.1, betas=(0.9, 0.999),
                 step=1.05, z_se=1.0, param_every=3, grad_eps=1e-3, implicit_grad=True, search='shared', bcd_frac=1.0,
                 freeze_frac=0.0, trace_trainable=False, loo_sweeps=None, **kw):
        if 'implicit' in kw:
            implicit_grad = kw.pop('implicit')
        super().__init__(**kw)
        self._base_kw = dict(kw)
        self.decay, self.batch_sweeps, self.loo_sweeps = decay, batch_sweeps, loo_sweeps
        if fc_update not in (None, 'adam', 'hillclimb'):
            raise ValueError("fc_update: 'adam', 'hillclimb' or None")
        if search not in ('shared', 'refine'):
            raise ValueError("search: 'shared' or 'refine'")
        if not (0.0 < bcd_frac <= 1.0 and 0.0 <= freeze_frac < 1.0):
            raise ValueError("bcd_frac in (0, 1], freeze_frac in [0, 1)")
        self.burn_in, self.fc_update, self.lr, self.betas, self.step, self.z_se = \
            burn_in, fc_update, lr, betas, step, z_se
        self.param_every, self.grad_eps, self._implicit = max(1, int(param_every)), grad_eps, bool(implicit_grad)
        self.search, self.bcd_frac, self.freeze_frac = search, float(bcd_frac), float(freeze_frac)
        self.trace_trainable = trace_trainable
        self.preq_, self.history_ = [], []
        self._n_learn, self._pool, self._hc, self._adam, self._epoch_g = 0, [], {}, {}, []
        self._held, self._held_groups, self.n_batches_ = None, [], 0
        self.converged_ = self.epochs_ = self.residual_ = None

    @property
    def implicit(self):
        return self._implicit

    def _base(self):
        return BLMLBinned(**self._base_kw)

    # ---------------------------------------------------------------- device state
    def _set_weights(self, w):
        """The held counts w (device, fit dtype): n, c = n w and the occupied mask follow."""
        self.w_t_ = w
        self.n_ = float(w.sum(dtype=torch.float64))
        self.c_t_ = self._lin([(self.n_, w)])
        self._occ_t = None

    def _axpy(self, a, w, b, m, clamp=False):
        out = torch.empty_like(w)
        call('blml_counts_axpy', self._code, self.B_, float(a), w.data_ptr(), float(b), m.data_ptr(), int(clamp),
             out.data_ptr(), self._st)
        return out

    def _refresh(self):
        E = self.e_hat_t_.clone()
        U = self._Sall(E)
        E, U = self._rescale(E, U)
        self._finish(E, U)

    def _residual(self):
        return self._resid(self.e_hat_t_, self.Se_t_)

    def _hill_sweeps(self):
        return self.loo_sweeps if self.loo_sweeps is not None else self.max_sweeps

    def _candidate_refit(self):
        E, U = self._solve(self.e_hat_t_, self._hill_sweeps())
        self._finish(E, U)

    def _loo_enter(self, m):
        """The fit with batch m left out (blml_binned.py:1068-1080): each bin's coefficient scaled by its remaining
        share (w - m) / w, then a warm refit on the held counts less m (loo_sweeps: a cap on its sweeps)."""
        mt = self._counts_t(m)
        w = self._axpy(1.0, self.w_t_, -1.0, mt, clamp=True)
        if not float(w.sum(dtype=torch.float64)) > 0:
            return
        f = torch.empty_like(w)
        call('blml_bin_ratio', self._code, self.B_, w.data_ptr(), self.w_t_.data_ptr(), f.data_ptr(), self._st)
        self._set_weights(w)
        E = self.e_hat_t_
        Ef = torch.empty_like(E)
        call('blml_mul_bins', self._code, E.shape[0], self.B_, int(E.is_complex()), E.data_ptr(), f.data_ptr(),
             Ef.data_ptr(), self._st)
        E, U = self._solve(Ef, self._hill_sweeps())
        self._finish(E, U)

    # ---------------------------------------------------------------- parameters
    def _registry(self):
        reg = []
        if self.fc_update is None:
            return reg
        for k, sp in enumerate(self.specs_):
            for u, (kind, dims) in enumerate(units_of(sp['kinds'])):
                if not bool(sp['fc_trainable'][dims[0]]):
                    continue
                ptype = 'integer' if split_kind(kind)[0] in INTEGER_KINDS else 'scale'
                rule = 'adam' if ptype == 'scale' and self.fc_update == 'adam' else 'hill'
                reg.append(dict(mode=k, unit=u, dims=tuple(dims), ptype=ptype, rule=rule))
        return reg

    def _fc_now(self):
        return [np.array(sp['fc'], float) for sp in self.specs_]

    def _trainable_now(self):
        return {k: {'fc': [float(v) for v, t in zip(sp['fc'], sp['fc_trainable']) if t]}
                for k, sp in enumerate(self.specs_)}

    def _set_fc(self, k, dims, value):
        fc = np.array(self.specs_[k]['fc'], float)
        fc[list(dims)] = value
        self.specs_ = [dict(sp, fc=fc) if j == k else sp for j, sp in enumerate(self.specs_)]

    def _nyq(self, e):
        """The largest identifiable value: fc <= 0.5 / h (the lattice's Nyquist limit, blml_binned.py:772-775)."""
        return 0.5 / float(self.h_[e['dims'][0]])

    def _in_range(self, e, value):
        return 0.0 < value <= self._nyq(e) + 1e-12

    def _keep_pools(self, saved):
        pools = (self._pool, self._hc, self._adam, self._epoch_g)
        self.__dict__.clear()
        self.__dict__.update(saved)
        self._pool, self._hc, self._adam, self._epoch_g = pools

    def _candidate_fit(self, e, cand):
        """(density, scale) of the fit with e's parameter at cand: the kernel swapped and a warm refit of the held
        counts (blml_binned.py:777-789); F / Z = density * scale."""
        saved = dict(self.__dict__)
        try:
            self._set_fc(e['mode'], e['dims'], cand)
            self._build_kernels()
            self._candidate_refit()
            Z = self._Q(self.e_hat_t_, self.Se_t_)
            return self.density_t_, self.n_ ** 2 / Z
        finally:
            self._keep_pools(saved)

    def _learn(self, counts):
        """The batch's gradient (pooled) and hill-climb gains before it is added (blml_binned.py:737-770)."""
        m = np.asarray(counts, float)
        occ = m.ravel() > 0
        Z0 = self._Q(self.e_hat_t_, self.Se_t_)
        n2 = self.n_ ** 2
        eps = self.grad_eps * n2 * float(np.median(self.density_.ravel()[occ])) / Z0 if occ.any() else 0.0
        reg = self._registry()
        adam = [e for e in reg if e['rule'] == 'adam']
        if adam:
            G = self.implicit_grad(m, eps) if self._implicit else self.param_grad(m, eps)
            self._pool.append((float(m.sum()), [G[e['mode']][e['unit']] for e in adam]))
            self._epoch_g.append(self._pool[-1])
        hill = [e for e in reg if e['rule'] == 'hill']
        if not hill:
            return
        mt = self._counts_t(m)
        d0, s0 = self.density_t_, n2 / Z0
        for e in hill:
            k, dims = e['mode'], list(e['dims'])
            v = float(self.specs_[k]['fc'][dims[0]])
            for sgn in (+1, -1):
                if e['ptype'] == 'integer':       # one harmonic, N = floor(fc P / 2) +- 1, at its interval's middle
                    P = float(self.specs_[k]['periods'][dims[0]])
                    N = int(np.floor(v * P / 2.0)) + sgn
                    if N < 0:
                        continue
                    cand = (N + 0.5) * 2.0 / P
                else:
                    cand = v * self.step ** sgn
                if not self._in_range(e, cand):
                    continue
                dc, sc = self._candidate_fit(e, cand)
                call('blml_gain_sums', self._code, self.B_, dc.data_ptr(), float(sc), d0.data_ptr(), float(s0),
                     mt.data_ptr(), float(eps), self._red.part.data_ptr(), self._red.out.data_ptr(), self._st)
                s, ss, W = self._red.read(3)
                acc = self._hc.setdefault((k, e['unit'], sgn), dict(s=0.0, ss=0.0, W=0.0, cand=cand))
                acc['s'] += s; acc['ss'] += ss; acc['W'] += W; acc['cand'] = cand

    def _param_step(self):
        """Every param_every learning batches (blml_binned.py:791-815): Adam on the pooled, count-weighted
        gradients; a hill-climb move once its pooled gain exceeds z_se standard errors. Returns what moved."""
        reg = self._registry()
        moved = []
        adam = [e for e in reg if e['rule'] == 'adam']
        if adam and self._pool:
            Wt = sum(p[0] for p in self._pool)
            G = sum(p[0] * np.asarray(p[1], float) for p in self._pool) / Wt
            if not np.all(np.isfinite(G)):
                raise FloatingPointError(f"streaming: non-finite gradient {G}")
            for q, e in enumerate(adam):
                k, dims = e['mode'], e['dims']
                old = float(self.specs_[k]['fc'][dims[0]])
                st = self._adam.setdefault((k, e['unit']), [0.0, 0.0, 0])
                new = min(float(adam_log_step(old, G[q], st, self.lr, self.betas)), self._nyq(e))
                self._set_fc(k, dims, new)
                moved.append((k, e['unit'], round(float(np.log(new / old)), 5)))
        self._pool = []
        for e in (e for e in reg if e['rule'] == 'hill'):
            for sgn in (+1, -1):
                acc = self._hc.get((e['mode'], e['unit'], sgn))
                if not acc or acc['W'] <= 1:
                    continue
                mu = acc['s'] / acc['W']
                se = np.sqrt(max(acc['ss'] / acc['W'] - mu * mu, 0.0) / (acc['W'] - 1))
                if mu > 0 and mu > self.z_se * se:
                    self._set_fc(e['mode'], e['dims'], acc['cand'])
                    moved.append((e['mode'], e['unit'], sgn))
                    self._hc = {kk: v for kk, v in self._hc.items() if kk[:2] != (e['mode'], e['unit'])}
                    break
        if moved:
            self._build_kernels()
            self._refresh()
        return moved

    def _param_stationary(self):
        """Whether the epoch's parameters are stationary (blml_binned.py:817-842): each Adam parameter's
        count-weighted mean gradient within z_se standard errors of 0, or > 0 at the Nyquist cap, and no pending
        hill-climb move. Returns (bool, max |mean| / se)."""
        reg = self._registry()
        adam = [e for e in reg if e['rule'] == 'adam']
        zmax = 0.0
        if adam and self._epoch_g:
            W = np.array([p[0] for p in self._epoch_g])
            G = np.array([np.ravel(np.asarray(p[1], float)) for p in self._epoch_g])
            if len(W) < 2:
                return False, np.inf
            mu = (W[:, None] * G).sum(0) / W.sum()
            var = (W[:, None] * (G - mu) ** 2).sum(0) / W.sum()
            se = np.sqrt(var / (len(W) - 1))
            ok = True
            for q, e in enumerate(adam):
                at_cap = float(self.specs_[e['mode']]['fc'][e['dims'][0]]) >= self._nyq(e) - 1e-12
                z = abs(mu[q]) / se[q] if se[q] > 0 else (0.0 if mu[q] == 0 else np.inf)
                if not (z <= self.z_se or (at_cap and mu[q] > 0)):
                    ok = False
                    zmax = max(zmax, z)
        else:
            ok = not adam
        for acc in self._hc.values():
            if acc['W'] > 1:
                mu = acc['s'] / acc['W']
                se = np.sqrt(max(acc['ss'] / acc['W'] - mu * mu, 0.0) / (acc['W'] - 1))
                if mu > 0 and mu > self.z_se * se:
                    ok = False
        return ok, zmax

    # ---------------------------------------------------------------- one batch
    def _left_out(self, counts):
        """Context: the fit with counts' share of the held counts removed (None: unchanged), restored after; the
        gradients and gains gathered inside are kept (blml_binned.py:871-888)."""
        @contextlib.contextmanager
        def ctx():
            if counts is None:
                yield
                return
            saved = dict(self.__dict__)
            try:
                self._loo_enter(np.asarray(counts, float))
                yield
            finally:
                self._keep_pools(saved)
        return ctx()

    def _stream_step(self, counts, absorb, revisit=False, learn=True):
        """Score (leave-batch-out on a revisit) and learn after the burn-in, absorb, then a parameter step every
        param_every learning batches (blml_binned.py:850-868)."""
        burned = self.n_ >= self.burn_in
        do_learn = learn and burned and self.fc_update is not None
        with self._left_out(counts if revisit else None):
            preq = self.log_density(counts)
            if do_learn:
                self._learn(counts)
        if absorb is not None:
            absorb(burned)
        moved = []
        if do_learn:
            self._n_learn += 1
            if self._n_learn % self.param_every == 0:
                moved = self._param_step()
        self.preq_.append(preq)
        h = dict(n=self.n_, preq=preq, fc=[f.tolist() for f in self._fc_now()], moved=moved, revisit=bool(revisit))
        if self.trace_trainable:
            h['trainable'] = self._trainable_now()
        self.history_.append(h)

    # ---------------------------------------------------------------- burn-in
    def _hold(self, counts, modes, h, origin, complex_g, group):
        if self._held is None:
            if modes is None:
                raise ValueError("partial_fit: modes on the first call")
            self._modes_args = (modes, h, origin, complex_g)
            self._held = counts.copy()
            self._held_list = [counts]
        else:
            if counts.shape != self._held.shape:
                raise ValueError("partial_fit: the batch must be on the lattice of the first one")
            self._held = self._held + counts
            self._held_list.append(counts)
        self._held_groups.append(group)
        return float(self._held.sum()) >= self.burn_in

    def _select(self):
        """The selector's search for the fc entries the modes leave out (NaN), on the held counts: an 80/20 binomial
        split, or 20% of whole groups for validation (blml_binned.py:904-940)."""
        modes, h, origin, cg = self._modes_args
        F = modes_fc(modes)
        free = ~np.isfinite(F)
        if not free.any():
            return modes
        specs = parse_modes(modes, self._held.ndim, need_fc=False)[0]
        rng = np.random.default_rng(self.seed)
        groups = list(self._held_groups)
        if all(g is not None for g in groups):
            u = np.unique(groups)
            V = rng.choice(u, max(1, int(round(0.2 * len(u)))), replace=False)
            tr = sum((b for b, g in zip(self._held_list, groups) if g not in V), np.zeros(self._held.shape))
            va = sum((b for b, g in zip(self._held_list, groups) if g in V), np.zeros(self._held.shape))
        else:
            if not np.allclose(self._held, np.round(self._held)):
                raise ValueError("burn-in selection: integer counts for the binomial split (or pass split_groups)")
            tr = rng.binomial(np.round(self._held).astype(np.int64), 0.8).astype(float)
            va = self._held - tr
        idx = np.argwhere(free)
        kinds = [specs[k]['kinds'][j].split(':')[0] for k, j in idx]
        hh = np.broadcast_to(np.asarray(h, float), (self._held.ndim,))
        periods = [None if specs[k]['periods'][j] is None else specs[k]['periods'][j] / hh[j] for k, j in idx]

        def obj(v):
            if np.any(np.asarray(v) > 0.5 / hh[idx[:, 1]] + 1e-12):
                return -np.inf
            try:
                mm = self._base().fit(tr, with_fc(modes, _fill(F, free, v)), h=h, origin=origin, complex_g=cg)
            except (ValueError, FloatingPointError, np.linalg.LinAlgError):
                return -np.inf
            return mm._val_score(va)
        fc0 = 2.0 / (max(self._held.shape) * float(np.max(hh)))
        v, _ = _sel.search(obj, len(idx), kinds, periods, fc0=fc0, max_sweeps=0 if self.search == 'shared' else 6,
                           tag='burn-in', factors=(np.sqrt(2.0), 2.0 ** 0.25, 2.0 ** 0.125))
        return with_fc(modes, _fill(F, free, v))

    # ---------------------------------------------------------------- public
    def partial_fit(self, counts, modes=None, h=1.0, origin=0.0, complex_g=False, split_groups=None, _learn=True):
        counts = np.asarray(counts, float)
        if self.n_batches_ == 0:
            if not self._hold(counts, modes, h, origin, complex_g, split_groups):
                return self
            modes = self._select()
            _, h, origin, complex_g = self._modes_args
            cap = self.max_sweeps
            if self.batch_sweeps is not None and not self.burn_in:
                self.max_sweeps = self.batch_sweeps
            BLMLBinned.fit(self, self._held, modes, h, origin, complex_g)
            self.max_sweeps = cap
            self.n_batches_ = 1
            self._held_list = None
            self.history_.append(dict(n=self.n_, preq=np.nan, fc=[f.tolist() for f in self._fc_now()], moved=[],
                                      burn_in=True))
            self.preq_.append(np.nan)
            return self
        if counts.shape != self.shape_:
            raise ValueError("partial_fit: the batch must be on the lattice of the first one")

        def absorb(burned):
            mt = self._counts_t(counts)
            n_old = self.n_
            self._set_weights(self._axpy(self.decay, self.w_t_, 1.0, mt))
            E = self._mask_(self._lin([(self.n_ / n_old, self.e_hat_t_)]))     # same g; _solve rescales Q = n^2
            U = self._Sall(E)
            Eu = self._update(E, U)
            call('blml_new_bins', self._code, E.shape[0], self.B_, int(E.is_complex()), E.data_ptr(), Eu.data_ptr(),
                 self.w_t_.data_ptr(), E.data_ptr(), self._st)                 # newly occupied bins: their own root
            sweeps = self.batch_sweeps if (self.batch_sweeps is not None and burned) else self.max_sweeps
            E, U = self._solve(E, sweeps)
            self._finish(E, U)

        self._stream_step(counts, absorb, learn=_learn)
        self.n_batches_ += 1
        return self

    def _again(self, counts, learn=True):
        """A held batch revisited: scored leave-batch-out, its gradient pooled, the coefficients swept (not added)."""
        def absorb(burned):
            sweeps = self.batch_sweeps if (self.batch_sweeps is not None and burned) else self.max_sweeps
            E, U = self._solve(self.e_hat_t_, sweeps)
            self._finish(E, U)
        self._stream_step(counts, absorb, revisit=True, learn=learn)

    def fit(self, batches, modes=None, epochs=2, h=1.0, origin=0.0, complex_g=False, split_groups=None, on_epoch=None,
            tol=None, tol_check='running'):
        """batches: count arrays on one lattice. Epoch 1 adds them in random group order; later epochs revisit them
        (scored leave-batch-out, the coefficients swept, the parameters moving); tol stops after the first epoch
        whose fit meets the solver's residual test with the parameters stationary (blml_binned.py:942-1011)."""
        batches = [np.asarray(b, float) for b in batches]
        nb = len(batches)
        grp = None if split_groups is None else list(np.asarray(split_groups).tolist())
        if grp is not None and len(grp) != nb:
            raise ValueError("split_groups: one label per batch")
        if tol is not None and not tol > 0:
            raise ValueError("tol: None (fixed epochs) or > 0")
        if tol is not None and (self.bcd_frac < 1.0 or self.freeze_frac > 0.0):
            raise ValueError("tol needs bcd_frac = 1 and freeze_frac = 0")
        if tol_check not in ('running', 'exact'):
            raise ValueError("tol_check: 'running' or 'exact'")
        split = self.bcd_frac < 1.0
        if split:
            if not all(np.allclose(b, np.round(b)) for b in batches):
                raise ValueError("bcd_frac < 1: integer counts (the learn share is a binomial thinning)")
            r0 = np.random.default_rng([self.seed, 11])
            L = [r0.binomial(np.round(b).astype(np.int64), 1.0 - self.bcd_frac).astype(float) for b in batches]
        held, joined = [False] * nb, [False] * nb
        T_learn = int(round((1.0 - self.freeze_frac) * epochs * nb))
        t = 0
        self.converged_, self.epochs_, self.residual_ = None, 0, None
        first = dict(modes=modes, h=h, origin=origin, complex_g=complex_g)
        for ep in range(epochs):
            run_max = 0.0
            self._epoch_g = []
            for i in batch_order(nb, grp, np.random.default_rng(self.seed + ep)):
                frozen = t >= T_learn
                t += 1
                both = not split and not frozen
                Fi = batches[i] if (not split or frozen) else batches[i] - L[i]
                if not held[i]:
                    self.partial_fit(Fi, split_groups=None if grp is None else grp[i], _learn=both and not frozen,
                                     **first)
                    held[i] = True
                    first = {}
                elif self.n_batches_ > 0:
                    run_max = max(run_max, self._residual())
                    self._again(Fi, learn=both)
                if split and not frozen and self.n_batches_ > 0:
                    self._stream_step(L[i], None, learn=True)            # scored, gradient pooled, not added
                if split and frozen and not joined[i] and self.n_batches_ > 0:
                    self.partial_fit(L[i], _learn=False)
                    joined[i] = True
            if self.n_batches_ == 0:
                raise ValueError(f"fit: burn_in = {self.burn_in} exceeds the counts given "
                                 f"({sum(float(b.sum()) for b in batches):g})")
            self.epochs_ = ep + 1
            if tol is not None and (tol_check == 'exact' or ep > 0):
                self.residual_ = self._residual() if tol_check == 'exact' else run_max
                still, z = self._param_stationary() if self.fc_update is not None else (True, 0.0)
                self.converged_ = bool(self.residual_ < tol and still)
                self.history_.append(dict(epoch=ep + 1, residual=self.residual_, params_stationary=still, grad_z=z))
            if on_epoch is not None:
                on_epoch(ep, self)
            if tol is not None and self.converged_:
                break
        return self
