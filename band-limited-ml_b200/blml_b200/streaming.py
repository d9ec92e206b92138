"""Counts arriving in batches on one fixed lattice, with cut-off learning, on the GPU engine of blml_b200.binned.

Behaviour (rahuljhu/band-limited-ml, blml_binned.py:648-1112, _KernelLearner and BLMLBinnedStreaming): each batch is
scored by the current model before it is used (its prequential score), its gradient of that score in log fc is
pooled, then it joins the held counts (old counts times `decay`) and the coefficients are warm-refitted. Every
`param_every` learning batches the trainable cut-offs move: an Adam step on log fc for continuous bands (sinc,
slits, ball), or a one-harmonic hill-climb step (dirichlet, pball) once the pooled paired gain of a neighbouring
value exceeds z_se standard errors. `fit(batches, epochs)` revisits the held batches, scored with their own share left
out. An fc left out of the modes (NaN) is chosen at the burn-in by the selector's search (blml_b200.selector.search)
on an 80/20 split of the held counts.

Structure. The learner is its own object (`CutoffLearner`): a table of the trainable units and, per unit, array
state -- Adam moments, pooled gradient rows, paired-gain sums of the two neighbouring candidates -- so the fit object
never has to be snapshotted. Every what-if fit (a candidate cut-off, a batch left out) runs on a `probe`: a shallow
fork of the streaming fit with its own kernels and coefficients that shares the device counts and the learner, then
is dropped, so the stream's own state is never rewound. Every array operation runs in libblml_b200.so (the fit's
kernels and the bin-wise kernels blml_counts_axpy, blml_bin_ratio, blml_new_bins, blml_gain_sums).
"""
import copy

import numpy as np
import torch

from ._lib import call
from .binned import BLMLBinned
from .spec import parse_modes, modes_fc, units_of, split_kind, with_fc
from . import selector as _sel

HARMONIC_KINDS = ('dirichlet', 'pball')      # fc moves in whole harmonics: hill-climb, no gradient


def adam_log_step(value, grad, state, lr, betas):
    """One Adam ascent step on log(value) from grad = d/dlog value; state = [m, v, t] updated in place (the 'scale'
    parameter rule of blml_maps.py:19-36). Returns the new value."""
    b1, b2 = betas
    state[2] += 1
    state[0] = b1 * state[0] + (1 - b1) * grad
    state[1] = b2 * state[1] + (1 - b2) * grad * grad
    m_hat = state[0] / (1 - b1 ** state[2])
    v_hat = state[1] / (1 - b2 ** state[2])
    return value * np.exp(lr * m_hat / (np.sqrt(v_hat) + 1e-12))


def batch_order(nb, groups, rng):
    """The visiting order of nb batches: a random permutation, or (with group labels) the groups in random order,
    each group's batches together in their given order (blml_binned.py:1022-1031)."""
    if groups is None:
        return list(rng.permutation(nb))
    labels = np.asarray(groups)
    uniq, which = np.unique(labels, return_inverse=True)
    order = rng.permutation(len(uniq))
    return [int(i) for g in order for i in np.flatnonzero(np.ravel(which) == g)]


def _welford_free(s, ss, W):
    """(mean, standard error) of a weighted sample from its sums: sum x, sum x^2, total weight W > 1."""
    mu = s / W
    return mu, np.sqrt(max(ss / W - mu * mu, 0.0) / (W - 1))


class CutoffLearner:
    """The learning state of a stream. units: one row per trainable unit (mode k, unit u, its dims, whether fc moves
    by Adam or by hill-climb); per unit the Adam moments, and for hill-climb units the pooled paired-gain sums
    [s, ss, W] and candidate value of its two neighbours (index 0: up, 1: down). Gradients of the Adam units are
    pooled per batch (count weight, one value per unit) until the next move, and kept for the epoch's stationarity
    test."""

    def __init__(self, specs, fc_update):
        self.units = []
        if fc_update is not None:
            for k, sp in enumerate(specs):
                for u, (kind, dims) in enumerate(units_of(sp['kinds'])):
                    if bool(sp['fc_trainable'][dims[0]]):
                        harmonic = split_kind(kind)[0] in HARMONIC_KINDS
                        rule = 'adam' if (not harmonic and fc_update == 'adam') else 'hill'
                        self.units.append(dict(k=k, u=u, dims=tuple(dims), harmonic=harmonic, rule=rule))
        self.adam_idx = [i for i, e in enumerate(self.units) if e['rule'] == 'adam']
        self.hill_idx = [i for i, e in enumerate(self.units) if e['rule'] == 'hill']
        self.moments = np.zeros((len(self.units), 3))                 # Adam m, v, t
        self.gains = np.zeros((len(self.units), 2, 3))                 # hill-climb s, ss, W per neighbour
        self.cands = np.full((len(self.units), 2), np.nan)
        self.pool_w, self.pool_g = [], []                               # since the last move
        self.epoch_w, self.epoch_g = [], []                             # since the epoch began
        self.n_learned = 0

    def pool(self, weight, grads):
        self.pool_w.append(float(weight)); self.pool_g.append(np.asarray(grads, float))
        self.epoch_w.append(float(weight)); self.epoch_g.append(np.asarray(grads, float))

    def add_gain(self, i, side, s, ss, W, cand):
        self.gains[i, side] += (s, ss, W)
        self.cands[i, side] = cand

    def new_epoch(self):
        self.epoch_w, self.epoch_g = [], []

    def adam_moves(self, fc_of, cap_of, lr, betas):
        """New values of the Adam units from the pooled count-weighted mean gradient, capped at their Nyquist
        limit; clears the pool. Returns [(unit index, old, new)]."""
        if not self.adam_idx or not self.pool_w:
            self.pool_w, self.pool_g = [], []
            return []
        w = np.asarray(self.pool_w)
        G = (w[:, None] * np.stack(self.pool_g)).sum(0) / w.sum()
        self.pool_w, self.pool_g = [], []
        if not np.all(np.isfinite(G)):
            raise FloatingPointError(f"streaming: non-finite gradient {G}")
        out = []
        for q, i in enumerate(self.adam_idx):
            old = fc_of(i)
            new = min(float(adam_log_step(old, G[q], self.moments[i], lr, betas)), cap_of(i))
            out.append((i, old, new))
        return out

    def hill_moves(self, z_se):
        """The hill-climb units whose up or down neighbour's pooled gain is positive and beyond z_se standard
        errors (the up side looked at first); their gain sums restart. Returns [(unit index, side, value)]."""
        out = []
        for i in self.hill_idx:
            for side in (0, 1):
                s, ss, W = self.gains[i, side]
                if W <= 1:
                    continue
                mu, se = _welford_free(s, ss, W)
                if mu > 0 and mu > z_se * se:
                    out.append((i, side, float(self.cands[i, side])))
                    self.gains[i] = 0.0; self.cands[i] = np.nan
                    break
        return out

    def stationary(self, fc_of, cap_of, z_se):
        """Whether the epoch's parameters are stationary (blml_binned.py:817-842): every Adam unit's count-weighted
        mean gradient within z_se standard errors of zero (or positive at its cap) and no hill-climb move pending.
        Returns (bool, the largest |mean| / se among the units that fail)."""
        ok, zmax = True, 0.0
        if self.adam_idx:
            if not self.epoch_w:
                ok = False
            else:
                w = np.asarray(self.epoch_w)
                if len(w) < 2:
                    return False, np.inf
                G = np.stack([np.ravel(g) for g in self.epoch_g])
                mu = (w[:, None] * G).sum(0) / w.sum()
                se = np.sqrt((w[:, None] * (G - mu) ** 2).sum(0) / w.sum() / (len(w) - 1))
                for q, i in enumerate(self.adam_idx):
                    z = abs(mu[q]) / se[q] if se[q] > 0 else (0.0 if mu[q] == 0 else np.inf)
                    at_cap = fc_of(i) >= cap_of(i) - 1e-12
                    if not (z <= z_se or (at_cap and mu[q] > 0)):
                        ok = False; zmax = max(zmax, z)
        for i in self.hill_idx:
            for side in (0, 1):
                s, ss, W = self.gains[i, side]
                if W > 1:
                    mu, se = _welford_free(s, ss, W)
                    if mu > 0 and mu > z_se * se:
                        ok = False
        return ok, zmax


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
        self._fit_kw = dict(kw)
        if fc_update not in (None, 'adam', 'hillclimb'):
            raise ValueError("fc_update: 'adam', 'hillclimb' or None")
        if search not in ('shared', 'refine'):
            raise ValueError("search: 'shared' or 'refine'")
        if not (0.0 < bcd_frac <= 1.0 and 0.0 <= freeze_frac < 1.0):
            raise ValueError("bcd_frac in (0, 1], freeze_frac in [0, 1)")
        self.decay, self.batch_sweeps, self.loo_sweeps, self.burn_in = decay, batch_sweeps, loo_sweeps, burn_in
        self.fc_update, self.lr, self.betas, self.step, self.z_se = fc_update, lr, betas, step, z_se
        self.param_every, self.grad_eps, self._implicit = max(1, int(param_every)), grad_eps, bool(implicit_grad)
        self.search, self.bcd_frac, self.freeze_frac = search, float(bcd_frac), float(freeze_frac)
        self.trace_trainable = trace_trainable
        self.preq_, self.history_ = [], []
        self.learner_ = None
        self._buffer = None                   # burn-in: (held sum, list of batches, their group labels, fit args)
        self.n_batches_ = 0
        self.converged_ = self.epochs_ = self.residual_ = None

    @property
    def implicit(self):
        return self._implicit

    # ---------------------------------------------------------------- probes and device state
    def _probe(self):
        """A what-if copy of the fit: rebinding its attributes (kernels, specs, counts, coefficients) leaves this
        fit untouched; it shares the device counts, the reduction buffers and the learner."""
        return copy.copy(self)

    def _hold_weights(self, w):
        """The held counts w (device, fit dtype) with n, c = n w and the occupancy that follow."""
        self.w_t_ = w
        self.n_ = float(w.sum(dtype=torch.float64))
        self.c_t_ = self._lin([(self.n_, w)])
        self._occ_t = None

    def _blend(self, a, w, b, m, clamp=False):
        """a w + b m per bin (clamped at 0), a new device array."""
        out = torch.empty_like(w)
        call('blml_counts_axpy', self._code, self.B_, float(a), w.data_ptr(), float(b), m.data_ptr(), int(clamp),
             out.data_ptr(), self._st)
        return out

    def _refit(self, E, sweeps):
        if getattr(self, '_defer', None) is not None:        # BLMLBinnedStreamingBatch refits many streams at once
            self._defer.append((E, sweeps))
            return
        E, U = self._solve(E, sweeps)
        self._finish(E, U)

    def _what_if_sweeps(self):
        return self.loo_sweeps if self.loo_sweeps is not None else self.max_sweeps

    def _without(self, counts):
        """The probe with a batch's share taken out of the held counts (blml_binned.py:1068-1080): each bin's
        coefficients scaled by its remaining share (w - m) / w, then a warm refit (loo_sweeps caps it). The held
        counts unchanged when nothing would remain."""
        p = self._probe()
        m = p._counts_t(counts)
        rest = p._blend(1.0, p.w_t_, -1.0, m, clamp=True)
        if not float(rest.sum(dtype=torch.float64)) > 0:
            return p
        share = torch.empty_like(rest)
        call('blml_bin_ratio', p._code, p.B_, rest.data_ptr(), p.w_t_.data_ptr(), share.data_ptr(), p._st)
        p._hold_weights(rest)
        E = torch.empty_like(p.e_hat_t_)
        call('blml_mul_bins', p._code, E.shape[0], p.B_, int(E.is_complex()), p.e_hat_t_.data_ptr(), share.data_ptr(),
             E.data_ptr(), p._st)
        p._refit(E, p._what_if_sweeps())
        return p

    def _with_fc(self, k, dims, value):
        """The probe with mode k's fc on dims set to value, its kernels rebuilt and refitted warm."""
        p = self._probe()
        p._set_fc(k, dims, value)
        p._build_kernels()
        p._refit(p.e_hat_t_.clone(), p._what_if_sweeps())
        return p

    # ---------------------------------------------------------------- cut-off values
    def _set_fc(self, k, dims, value):
        fc = np.array(self.specs_[k]['fc'], float)
        fc[list(dims)] = value
        self.specs_ = [dict(sp, fc=fc) if j == k else sp for j, sp in enumerate(self.specs_)]

    def _fc_of(self, i):
        e = self.learner_.units[i]
        return float(self.specs_[e['k']]['fc'][e['dims'][0]])

    def _cap_of(self, i):
        """The largest identifiable cut-off of a unit: 0.5 / h, the lattice's Nyquist limit (blml_binned.py:772-775)."""
        return 0.5 / float(self.h_[self.learner_.units[i]['dims'][0]])

    def _neighbour(self, i, side):
        """The hill-climb candidate of unit i on one side (0 up, 1 down): one harmonic more / less, at the middle of
        its fc interval (N = floor(fc P / 2) +- 1, fc = (N + 1/2) 2 / P), or fc times step^+-1; None off range."""
        e = self.learner_.units[i]
        v = self._fc_of(i)
        sgn = 1 if side == 0 else -1
        if e['harmonic']:
            P = float(self.specs_[e['k']]['periods'][e['dims'][0]])
            N = int(np.floor(v * P / 2.0)) + sgn
            if N < 0:
                return None
            cand = (N + 0.5) * 2.0 / P
        else:
            cand = v * self.step ** sgn
        return cand if 0.0 < cand <= self._cap_of(i) + 1e-12 else None

    def _trainable_values(self):
        return {k: {'fc': [float(v) for v, t in zip(sp['fc'], sp['fc_trainable']) if t]}
                for k, sp in enumerate(self.specs_)}

    # ---------------------------------------------------------------- learning from one batch
    def _gather(self, counts):
        """The batch's contribution to the learner before it joins the held counts (blml_binned.py:737-770): the
        Adam units' score gradient (implicit or at fixed coefficients) pooled with the batch's count as weight, and
        for each hill-climb unit the paired gain of both neighbours' refits on the batch."""
        L = self.learner_
        m = np.asarray(counts, float)
        on = m.ravel() > 0
        Z0 = self._Q(self.e_hat_t_, self.Se_t_)
        nn = self.n_ ** 2
        eps = self.grad_eps * nn * float(np.median(self.density_.ravel()[on])) / Z0 if on.any() else 0.0
        if L.adam_idx:
            G = self.implicit_grad(m, eps) if self._implicit else self.param_grad(m, eps)
            L.pool(m.sum(), [G[L.units[i]['k']][L.units[i]['u']] for i in L.adam_idx])
        if not L.hill_idx:
            return
        mt = self._counts_t(m)
        for i in L.hill_idx:
            e = L.units[i]
            for side in (0, 1):
                cand = self._neighbour(i, side)
                if cand is None:
                    continue
                p = self._with_fc(e['k'], e['dims'], cand)
                zp = p._Q(p.e_hat_t_, p.Se_t_)
                call('blml_gain_sums', self._code, self.B_, p.density_t_.data_ptr(), float(p.n_ ** 2 / zp),
                     self.density_t_.data_ptr(), float(nn / Z0), mt.data_ptr(), float(eps), self._red.part.data_ptr(),
                     self._red.out.data_ptr(), self._st)
                L.add_gain(i, side, *self._red.read(3), cand)

    def _move(self):
        """A parameter step (blml_binned.py:791-815): the Adam units' new values, then at most one hill-climb move
        per unit; the kernels rebuilt and the fit refreshed when anything moved. Returns the moves as
        (mode, unit, log ratio) for Adam and (mode, unit, +-1) for hill-climb."""
        L = self.learner_
        moved = []
        for i, old, new in L.adam_moves(self._fc_of, self._cap_of, self.lr, self.betas):
            e = L.units[i]
            self._set_fc(e['k'], e['dims'], new)
            moved.append((e['k'], e['u'], round(float(np.log(new / old)), 5)))
        for i, side, value in L.hill_moves(self.z_se):
            e = L.units[i]
            self._set_fc(e['k'], e['dims'], value)
            moved.append((e['k'], e['u'], 1 if side == 0 else -1))
        if moved:
            self._build_kernels()
            E = self.e_hat_t_.clone()
            E, U = self._rescale(E, self._Sall(E))
            self._finish(E, U)
        return moved

    def _record(self, preq, moved, revisit):
        self.preq_.append(preq)
        entry = dict(n=self.n_, preq=preq, fc=[np.array(sp['fc'], float).tolist() for sp in self.specs_], moved=moved,
                     revisit=bool(revisit))
        if self.trace_trainable:
            entry['trainable'] = self._trainable_values()
        self.history_.append(entry)

    def _visit(self, counts, join, revisit=False, learn=True):
        """One batch after the burn-in (blml_binned.py:850-868): scored -- on a revisit by the fit without its own
        share -- and gathered for learning, then joined (join(burned) changes the fit), then a parameter step every
        param_every learning batches."""
        burned = self.n_ >= self.burn_in
        learning = learn and burned and self.fc_update is not None
        judge = self._without(counts) if revisit else self
        preq = judge.log_density(counts)
        if learning:
            judge._gather(counts)
        if join is not None:
            join(burned)
        moved = []
        if learning:
            self.learner_.n_learned += 1
            if self.learner_.n_learned % self.param_every == 0:
                moved = self._move()
        self._record(preq, moved, revisit)

    def _sweeps(self, burned):
        return self.batch_sweeps if (self.batch_sweeps is not None and burned) else self.max_sweeps

    def _join_new(self, counts):
        """Add a batch: held counts times decay plus the batch, the same roots rescaled to the new n, newly occupied
        bins given their own coordinate root, then the warm refit."""
        def join(burned):
            mt = self._counts_t(counts)
            n_was = self.n_
            self._hold_weights(self._blend(self.decay, self.w_t_, 1.0, mt))
            E = self._mask_(self._lin([(self.n_ / n_was, self.e_hat_t_)]))
            Eu = self._update(E, self._Sall(E))
            call('blml_new_bins', self._code, E.shape[0], self.B_, int(E.is_complex()), E.data_ptr(), Eu.data_ptr(),
                 self.w_t_.data_ptr(), E.data_ptr(), self._st)
            self._refit(E, self._sweeps(burned))
        return join

    def _join_again(self):
        """A held batch revisited: the coefficients swept again on the unchanged held counts."""
        def join(burned):
            self._refit(self.e_hat_t_, self._sweeps(burned))
        return join

    # ---------------------------------------------------------------- burn-in
    def _buffer_batch(self, counts, modes, h, origin, complex_g, group):
        """Keep a burn-in batch; True once the held counts reach burn_in."""
        if self._buffer is None:
            if modes is None:
                raise ValueError("partial_fit: modes on the first call")
            self._buffer = dict(total=counts.copy(), batches=[counts], groups=[group],
                                args=(modes, h, origin, complex_g))
        else:
            if counts.shape != self._buffer['total'].shape:
                raise ValueError("partial_fit: the batch must be on the lattice of the first one")
            self._buffer['total'] = self._buffer['total'] + counts
            self._buffer['batches'].append(counts); self._buffer['groups'].append(group)
        return float(self._buffer['total'].sum()) >= self.burn_in

    def _choose_missing_fc(self):
        """The selector's search for the fc entries the modes leave out (NaN) on the held counts (blml_binned.py:
        904-940): trained on 80% of them (a binomial split, or 80% of whole groups when every batch has a group) and
        scored on the rest."""
        buf = self._buffer
        modes, h, origin, cg = buf['args']
        fc_all = modes_fc(modes)
        missing = ~np.isfinite(fc_all)
        if not missing.any():
            return modes
        total = buf['total']
        specs = parse_modes(modes, total.ndim, need_fc=False)[0]
        rng = np.random.default_rng(self.seed)
        groups = buf['groups']
        if all(g is not None for g in groups):
            labels = np.unique(groups)
            held_out = rng.choice(labels, max(1, int(round(0.2 * len(labels)))), replace=False)
            train = np.zeros(total.shape); valid = np.zeros(total.shape)
            for b, g in zip(buf['batches'], groups):
                if g in held_out:
                    valid = valid + b
                else:
                    train = train + b
        else:
            if not np.allclose(total, np.round(total)):
                raise ValueError("burn-in selection: integer counts for the binomial split (or pass split_groups)")
            train = rng.binomial(np.round(total).astype(np.int64), 0.8).astype(float)
            valid = total - train
        where = np.argwhere(missing)
        kinds = [specs[k]['kinds'][j].split(':')[0] for k, j in where]
        hv = np.broadcast_to(np.asarray(h, float), (total.ndim,))
        periods = [None if specs[k]['periods'][j] is None else specs[k]['periods'][j] / hv[j] for k, j in where]
        caps = 0.5 / hv[where[:, 1]] + 1e-12

        def filled(v):
            out = fc_all.copy()
            out[missing] = np.asarray(v, float)
            return out

        def score(v):
            if np.any(np.asarray(v) > caps):
                return -np.inf
            try:
                f = BLMLBinned(**self._fit_kw).fit(train, with_fc(modes, filled(v)), h=h, origin=origin, complex_g=cg)
            except (ValueError, FloatingPointError, np.linalg.LinAlgError):
                return -np.inf
            return f._val_score(valid)

        start = 2.0 / (max(total.shape) * float(np.max(hv)))
        v, _ = _sel.search(score, len(where), kinds, periods, fc0=start, max_sweeps=0 if self.search == 'shared' else 6,
                           tag='burn-in', factors=(np.sqrt(2.0), 2.0 ** 0.25, 2.0 ** 0.125))
        return with_fc(modes, filled(v))

    def _first_fit(self):
        """The burn-in's end: the missing fc chosen, the fit of the held counts (capped at batch_sweeps when there
        is no burn-in), the learner set up on its modes."""
        modes = self._choose_missing_fc()
        _, h, origin, complex_g = self._buffer['args']
        cap, self.max_sweeps = self.max_sweeps, (self.batch_sweeps if (self.batch_sweeps is not None and
                                                                        not self.burn_in) else self.max_sweeps)
        try:
            BLMLBinned.fit(self, self._buffer['total'], modes, h, origin, complex_g)
        finally:
            self.max_sweeps = cap
        self.learner_ = CutoffLearner(self.specs_, self.fc_update)
        self._buffer = dict(args=self._buffer['args'])
        self.n_batches_ = 1
        self.history_.append(dict(n=self.n_, preq=np.nan, fc=[np.array(sp['fc'], float).tolist()
                                                              for sp in self.specs_], moved=[], burn_in=True))
        self.preq_.append(np.nan)

    # ---------------------------------------------------------------- public
    def partial_fit(self, counts, modes=None, h=1.0, origin=0.0, complex_g=False, split_groups=None, _learn=True):
        counts = np.asarray(counts, float)
        if self.n_batches_ == 0:
            if self._buffer_batch(counts, modes, h, origin, complex_g, split_groups):
                self._first_fit()
            return self
        if counts.shape != self.shape_:
            raise ValueError("partial_fit: the batch must be on the lattice of the first one")
        self._visit(counts, self._join_new(counts), learn=_learn)
        self.n_batches_ += 1
        return self

    def fit(self, batches, modes=None, epochs=2, h=1.0, origin=0.0, complex_g=False, split_groups=None, on_epoch=None,
            tol=None, tol_check='running'):
        """batches: count arrays on one lattice. Epoch 1 adds them in random group order; later epochs revisit them
        (scored leave-batch-out, the coefficients swept, the parameters moving); tol stops after the first epoch
        whose fit meets the solver's residual test with the parameters stationary (blml_binned.py:942-1011).
        bcd_frac < 1 keeps a binomial 1 - bcd_frac share of each batch for learning only (scored and gathered, not
        joined) until freeze_frac of the visits are done, when the shares join the fit."""
        batches = [np.asarray(b, float) for b in batches]
        nb = len(batches)
        labels = None if split_groups is None else list(np.asarray(split_groups).tolist())
        if labels is not None and len(labels) != nb:
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
            rs = np.random.default_rng([self.seed, 11])
            learn_part = [rs.binomial(np.round(b).astype(np.int64), 1.0 - self.bcd_frac).astype(float) for b in batches]
        added = np.zeros(nb, bool); shares_in = np.zeros(nb, bool)
        learn_visits = int(round((1.0 - self.freeze_frac) * epochs * nb))
        visit = 0
        self.converged_, self.epochs_, self.residual_ = None, 0, None
        first_args = dict(modes=modes, h=h, origin=origin, complex_g=complex_g)
        for ep in range(epochs):
            worst = 0.0
            if self.learner_ is not None:
                self.learner_.new_epoch()
            for i in batch_order(nb, labels, np.random.default_rng(self.seed + ep)):
                frozen = visit >= learn_visits
                visit += 1
                whole = not split and not frozen
                part = batches[i] if (not split or frozen) else batches[i] - learn_part[i]
                if not added[i]:
                    self.partial_fit(part, split_groups=None if labels is None else labels[i],
                                     _learn=whole, **first_args)
                    added[i] = True
                    first_args = {}
                elif self.n_batches_ > 0:
                    worst = max(worst, self._resid(self.e_hat_t_, self.Se_t_))
                    self._visit(part, self._join_again(), revisit=True, learn=whole)
                if split and not frozen and self.n_batches_ > 0:
                    self._visit(learn_part[i], None, learn=True)             # scored and gathered, not joined
                if split and frozen and not shares_in[i] and self.n_batches_ > 0:
                    self.partial_fit(learn_part[i], _learn=False)
                    shares_in[i] = True
            if self.n_batches_ == 0:
                raise ValueError(f"fit: burn_in = {self.burn_in} exceeds the counts given "
                                 f"({sum(float(b.sum()) for b in batches):g})")
            self.epochs_ = ep + 1
            if tol is not None and (tol_check == 'exact' or ep > 0):
                self.residual_ = self._resid(self.e_hat_t_, self.Se_t_) if tol_check == 'exact' else worst
                if self.fc_update is not None:
                    still, z = self.learner_.stationary(self._fc_of, self._cap_of, self.z_se)
                else:
                    still, z = True, 0.0
                self.converged_ = bool(self.residual_ < tol and still)
                self.history_.append(dict(epoch=ep + 1, residual=self.residual_, params_stationary=still, grad_z=z))
            if on_epoch is not None:
                on_epoch(ep, self)
            if tol is not None and self.converged_:
                break
        return self


class BLMLBinnedStreamingBatch:
    """Many count streams at once, each the reference's streaming fit with a fixed kernel (blml_binned.py:1034-1112
    with fc_update=None; complex_g, L-BFGS): partial_fit(batches) takes the next batch of every stream. Each stream
    scores and joins its batch as BLMLBinnedStreaming does (the prequential score under the current fit, the held
    counts times decay plus the batch, the roots rescaled to the new n, newly occupied bins given their coordinate
    root), then every stream's warm refit runs in one BLMLBinnedBatch lockstep from its joined coefficients, in place
    of one L-BFGS fit per stream. The first batch of a stream (its burn-in and first fit) runs on the stream itself.

        sb = BLMLBinnedStreamingBatch(len(streams), tol=1e-6, decay=0.95)
        for batches in zip(*streams):                  # one count array per stream
            sb.partial_fit(batches, modes_list)        # sb.streams[i].preq_, .loglik_, .e_hat_ ...
    """

    def __init__(self, n_streams, **kw):
        if kw.get('fc_update', 'adam') is not None:
            raise ValueError("BLMLBinnedStreamingBatch: fixed kernels (fc_update=None)")
        if kw.setdefault('solver', 'lbfgs') != 'lbfgs':
            raise ValueError("BLMLBinnedStreamingBatch: complex L-BFGS streams (solver='lbfgs')")
        self.streams = [BLMLBinnedStreaming(**kw) for _ in range(int(n_streams))]
        self.n_refits_ = 0

    def partial_fit(self, batches, modes_list=None, h=1.0, origin=0.0):
        from .sweep import BLMLBinnedBatch
        if len(batches) != len(self.streams):
            raise ValueError("partial_fit: one batch per stream")
        pend = []
        for i, (st, counts) in enumerate(zip(self.streams, batches)):
            if st.n_batches_ == 0 and st._buffer is None:
                if modes_list is None:
                    raise ValueError("partial_fit: the first batches need modes_list")
                st.partial_fit(counts, modes_list[i], h=h, origin=origin, complex_g=True)
                continue
            st._defer = []
            try:
                st.partial_fit(counts)
            finally:
                job, st._defer = st._defer, None
            if job:
                if st.d_ != 2 or not np.allclose(st.h_, 1.0):
                    raise NotImplementedError("BLMLBinnedStreamingBatch: 2-D lattices with unit steps (h = 1)")
                pend.append((st, job[-1]))
        if not pend:
            return self
        ref = pend[0][0]
        caps = np.array([-1 if sw is None else int(sw) for _, (_, sw) in pend], np.int64)
        b = BLMLBinnedBatch(tol=ref.tol, max_sweeps=None, anderson=ref.anderson, dtype=ref.dtype,
                            phase_noise=ref.phase_noise, seed=ref.seed, stall=ref.stall, ll_tol=ref.ll_tol,
                            ll_window=ref.ll_window, lbfgs_m=ref.lbfgs_m, device=ref.dev_)
        counts = [st.w_t_.reshape(st.shape_) for st, _ in pend]
        modes = [st.modes_ for st, _ in pend]
        init = [E.reshape((E.shape[0],) + tuple(st.shape_)) for st, (E, _) in pend]
        res = b.fit(counts, modes, init=init, caps=caps)
        for f, (st, _) in enumerate(pend):
            E = b.e_hat(f).reshape(st.e_hat_t_.shape).clone()
            a, z = b.moff[f], b.moff[f + 1]
            U = b.U_t[a:z].reshape(E.shape).clone()
            st._finish(E, U)
            r = res[f]
            st.n_sweeps_, st.stop_reason_, st.residual_, st.converged_ = (r.n_sweeps_, r.stop_reason_, r.residual_,
                                                                         r.converged_)
        self.n_refits_ += 1
        return self
