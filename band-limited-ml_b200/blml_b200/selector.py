"""The selector's cut-off search (rahuljhu/band-limited-ml, selector.py:58-82 `_blocks` / `_free_blocks`, :467-487
`_move`, :488-553 `_search`) with its candidate fits batched on the GPU.

The reference walks the search one candidate at a time: each candidate is one fit, and which candidate comes next
depends on whether the last one improved the validation score. Here the walk is a generator (`search_walk`) that
yields every candidate it has not scored yet and receives its score. The search's result depends on nothing but those
scores, so any driver that hands it the same scores returns the reference loop's (fc, best).

- `search` drives one walk with a scalar objective: the reference's call `_search(obj, d, kinds, periods_scaled, ...)`.
- `search_batched` drives many walks with a batched objective. Before each batch it replays every unfinished walk
  under hypothetical outcomes (improved / not improved) of its unscored candidates, breadth-first, and gathers the
  candidates those branches ask for. One batch of fits then scores the candidate each walk needs now together with
  the ones it is likely to need next. A branch not taken costs fits, never a different answer.
- `select_counts_batched` is the binned-counts use (dslit_job.py:158-171 `search_fc`, selector.py:695-732
  `select_counts`): fits on training counts by BLMLBinnedBatch, scored on validation counts, for many lattices (bead
  windows, rolling windows, frames) in one run.
"""
from collections import deque

import numpy as np

from .spec import is_group, split_kind, KINDS, make_modes

SQRT2 = float(np.sqrt(2.0))
SEARCH_FACTORS = (SQRT2, 2.0 ** 0.25, 2.0 ** 0.125)      # dslit_job.py:170 resolves fc to about 9 %


def _key(fc):
    """The search's memo key (selector.py:497): log fc rounded to 6 decimals."""
    return tuple(np.round(np.log(np.asarray(fc, float)), 6))


def blocks(kinds, d):
    """Search coordinates (selector.py:58-72): each radial group (ball / pball columns sharing a tag) moves as one
    block, placed at its first column; every other column is a block of its own."""
    if kinds is None:
        return [[k] for k in range(d)]
    groups, kind_of = {}, {}
    for k, kind in enumerate(kinds):
        name, tag = split_kind(kind)
        if name not in KINDS:
            raise ValueError(f"unknown kernel kind {kind!r}")
        if is_group(kind):
            if kind_of.setdefault(tag, name) != name:
                raise ValueError(f"radial group {tag!r} mixes kinds {kind_of[tag]!r} and {name!r}")
            groups.setdefault(tag, []).append(k)
    member = {k: tuple(g) for g in groups.values() for k in g}
    out = []
    for k in range(d):
        g = member.get(k)
        if g is None:
            out.append([k])
        elif g[0] == k:
            out.append(list(g))
    return out


def free_blocks(kinds, d, free):
    return [b for b in blocks(kinds, d) if all(free[b])]


def move(fc, block, factor, kinds, periods_scaled):
    """fc with the block's columns scaled by factor (selector.py:470-487). A lone dirichlet column only changes the
    fit when its harmonic count floor(fc P / 2) does, so a step that keeps the count goes on to the next count in
    that direction, at its centre (n + 1/2) 2 / P; None when that count would be negative."""
    new = fc.copy()
    new[block] *= factor
    if len(block) > 1:
        return new
    k = block[0]
    if kinds is not None and split_kind(kinds[k])[0] == 'dirichlet':
        P = periods_scaled[k]
        n0 = int(np.floor(fc[k] * P / 2.0))
        n1 = int(np.floor(new[k] * P / 2.0))
        if n1 == n0:
            n1 = n0 + 1 if factor > 1 else n0 - 1
            if n1 < 0:
                return None
            new[k] = (n1 + 0.5) * 2.0 / P
    return new


def search_walk(d, kinds, periods_scaled, fc0=0.2, patience=2, max_sweeps=6, factors=(SQRT2,), start=None,
                free=None):
    """The search of selector.py:488-553 as a generator.

    Yields (fc, best, stage) for each candidate not scored before, best being the score it is compared with (None
    for the first) and stage the step that proposes it ('double', 'volume' or 'refine'); receives the candidate's
    score; returns (fc, best, n_scored). Stage 1 doubles every growing column (free,
    without a start) until `patience` doublings in a row fail to improve, then walks the volume grid
    centre * 2^(j / dg) from the best doubling, up first and down only if no up-step improved. Stage 2 steps each free
    block by each factor (up, then down if up did not move), repeating full sweeps, at most `max_sweeps` per factor,
    until a sweep accepts nothing; a step must improve by more than 1e-6."""
    scored = {}

    def score(fc, best, stage):
        k = _key(fc)
        if k not in scored:
            scored[k] = yield fc, best, stage
        return scored[k]

    st = np.full(d, np.nan) if start is None else np.asarray(start, float)
    fr = np.ones(d, bool) if free is None else np.asarray(free, bool)
    grow = fr & ~np.isfinite(st)
    dg = int(grow.sum())
    fc = np.where(grow, float(fc0), st)
    best_fc = fc.copy()
    best = yield from score(fc, None, 'double')
    misses = 0
    while dg and misses <= patience:
        fc = np.where(grow, fc * 2.0, fc)
        v = yield from score(fc, best, 'double')
        if v > best:
            best, best_fc, misses = v, fc.copy(), 0
        else:
            misses += 1
    centre = best_fc.copy()
    for sign in (1, -1):
        took = False
        for j in range(1, dg):
            cand = np.where(grow, centre * 2.0 ** (sign * j / dg), centre)
            v = yield from score(cand, best, 'volume')
            if not v > best:
                break
            best, best_fc, took = v, cand, True
        if took:
            break
    fc = best_fc
    moving = free_blocks(kinds, d, fr)
    for factor in factors:
        for _ in range(max_sweeps):
            moved = False
            for blk in moving:
                for fac in (factor, 1.0 / factor):
                    stepped = False
                    cand = move(fc, blk, fac, kinds, periods_scaled)
                    while cand is not None:
                        v = yield from score(cand, best, 'refine')
                        if not v > best + 1e-6:
                            break
                        best, fc, moved, stepped = v, cand, True, True
                        cand = move(fc, blk, fac, kinds, periods_scaled)
                    if stepped:
                        break
            if not moved:
                break
    return fc, best, len(scored)


def search(obj, d, kinds, periods_scaled, fc0=0.2, patience=2, max_sweeps=6, tag='auto', factors=(SQRT2,),
           start=None, free=None, verbose=False):
    """The reference's `_search(obj, ...)` (selector.py:488): one walk, one candidate at a time; returns (fc, best).
    obj(fc) -> validation score (higher is better)."""
    walk = search_walk(d, kinds, periods_scaled, fc0, patience, max_sweeps, factors, start, free)
    try:
        fc = next(walk)[0]
        while True:
            fc = walk.send(float(obj(fc)))[0]
    except StopIteration as done:
        fc, best, n = done.value
    if verbose:
        print(f"  [{tag}] final fc={np.round(fc, 4)} ll={best:.4f} ({n} fits)", flush=True)
    return fc, best


class _Walk:
    """One search of a batched run: its walk's arguments, the scores known so far, host-side scores (bounds)."""

    def __init__(self, args, cheap=None):
        self.args, self.cheap, self.known = args, cheap, {}
        self.result = None

    def replay(self, hyp=()):
        """A fresh walk answered from the known scores and, for its unscored candidates in order, from hyp; returns
        (True, (fc, best, n)) when it finishes, else (False, (fc, best)) at the first candidate past hyp."""
        walk = search_walk(*self.args)
        i = 0
        try:
            fc, best, stage = next(walk)
            while True:
                k = _key(fc)
                v = self.known.get(k)
                if v is None and self.cheap is not None:
                    v = self.cheap(fc)
                    if v is not None:
                        v = self.known[k] = float(v)
                if v is None:
                    if i == len(hyp):
                        return False, (fc, best, stage)
                    v = hyp[i]
                    i += 1
                fc, best, stage = walk.send(v)
        except StopIteration as done:
            return True, done.value

    def frontier(self, cap, max_depth=24):
        """Up to cap unscored candidates: the one the walk needs now, then those of the hypothetical branches,
        breadth-first (an improving outcome before a failing one at each level)."""
        out, keys = [], set()
        queue, runs = deque([()]), 0
        while queue and len(out) < cap and runs < 16 * cap:
            hyp = queue.popleft()
            runs += 1
            finished, r = self.replay(hyp)
            if finished:
                if not hyp:
                    self.result = r
                continue
            fc, best, _ = r
            k = _key(fc)
            if k not in keys:
                keys.add(k)
                out.append(fc)
            if len(hyp) >= max_depth:
                continue
            if best is None:
                queue.append(hyp + (0.0,))
            else:
                queue.append(hyp + ((best + 1.0) if np.isfinite(best) else 0.0,))
                queue.append(hyp + (-np.inf,))
        return out


def search_batched(obj_batch, walks, batch=64, max_depth=24):
    """Many searches at once. walks: one dict per search with the keywords of `search_walk` (d, kinds,
    periods_scaled, fc0, patience, max_sweeps, factors, start, free) and optionally 'cheap', a host-side
    score fc -> float or None (e.g. -inf outside the allowed band, which costs no fit). obj_batch(requests) takes a
    list of (search index, fc) and returns their scores. Each round every unfinished search adds about
    batch / (unfinished searches) candidates, at least the one it needs now. Returns [(fc, best)] per search and the
    run's statistics (rounds, fits scored, fits the searches used)."""
    order = ('d', 'kinds', 'periods_scaled', 'fc0', 'patience', 'max_sweeps', 'factors', 'start', 'free')
    dflt = dict(fc0=0.2, patience=2, max_sweeps=6, factors=(SQRT2,), start=None, free=None)
    ws = []
    for w in walks:
        kw = {**dflt, **{k: v for k, v in w.items() if k != 'cheap'}}
        ws.append(_Walk(tuple(kw[k] for k in order), w.get('cheap')))
    rounds, fits, per_round = 0, 0, []
    while True:
        reqs = []
        active = [w for w in ws if w.result is None]
        cap = max(1, int(batch) // max(1, len(active)))
        for s, w in enumerate(ws):
            if w.result is None:
                reqs += [(s, fc) for fc in w.frontier(cap, max_depth)]
        if not reqs:
            break
        vals = obj_batch(reqs)
        if len(vals) != len(reqs):
            raise ValueError("obj_batch: one score per request")
        for (s, fc), v in zip(reqs, vals):
            ws[s].known[_key(fc)] = float(v)
        rounds += 1
        fits += len(reqs)
        per_round.append(len(reqs))
    res = [(w.result[0], w.result[1]) for w in ws]
    stats = dict(rounds=rounds, fits=fits, used=int(sum(w.result[2] for w in ws)), per_round=per_round)
    return res, stats


def select_counts_batched(train, val, kinds=('sinc', 'sinc'), periods=None, fc0=None, fc_min=None, fc_max=0.5,
                          factors=SEARCH_FACTORS, patience=2, max_sweeps=6, start=None, free=None, batch=64, tol=1e-6,
                          dtype=np.float64, max_fit_sweeps=None, device=None, return_stats=False, **fit_kw):
    """Cut-offs for many binned lattices at once. train / val: lists of 2-D count arrays (host or CUDA), one pair
    per search; the fit of a candidate fc is BLMLBinnedBatch's complex one-mode fit of make_modes(fc, kinds, periods)
    on the training counts (lattice units, h = 1), and its score the mean log-probability of the validation counts,
    p = f / sum f over the lattice (selector.py:712-716).

    fc0 defaults to 0.1 fc_max (selector.py:722). A candidate with a column above fc_max (the bin lattice's Nyquist
    0.5 by default, as dslit_job.py:165; select_counts caps at 1 / h) or below fc_min (default none; dslit_job.py uses
    2 / max(shape)) scores -inf without a fit. start / free as in the reference (per column; NaN where none).
    Returns [(modes, best)] per lattice (and the run's statistics with return_stats)."""
    import torch
    from .sweep import BLMLBinnedBatch
    if len(train) != len(val) or not train:
        raise ValueError("one validation lattice per training lattice")
    dev = torch.device(device or 'cuda')
    tr = [torch.as_tensor(np.asarray(t, float)) if not isinstance(t, torch.Tensor) else t for t in train]
    tr = [t.to(dev, torch.float64) for t in tr]
    va = [torch.as_tensor(np.asarray(v, float)) if not isinstance(v, torch.Tensor) else v for v in val]
    va = [v.to(dev, torch.float64) for v in va]
    for t, v in zip(tr, va):
        if t.ndim != 2 or tuple(t.shape) != tuple(v.shape):
            raise ValueError("train / val: 2-D lattices of equal shape")
    d = len(kinds)
    if d != 2:
        raise ValueError("select_counts_batched: two columns (2-D lattices)")
    hi = np.broadcast_to(np.asarray(fc_max, float), (d,))
    lo = np.broadcast_to(np.asarray(0.0 if fc_min is None else fc_min, float), (d,))
    f0 = float(fc0) if fc0 is not None else 0.1 * float(hi.min())
    per = list(periods) if periods is not None else [None] * d

    def cheap(fc):
        if np.any(fc > hi * (1 + 1e-9)) or np.any(fc < lo):
            return -np.inf
        return None

    def modes_of(fc):
        return make_modes(np.asarray(fc, float), list(kinds), per)

    def obj_batch(reqs):
        est = BLMLBinnedBatch(tol=tol, max_sweeps=max_fit_sweeps, dtype=dtype, device=dev, **fit_kw)
        est.fit([tr[s] for s, _ in reqs], [modes_of(fc) for _, fc in reqs])
        return est.val_score([va[s] for s, _ in reqs])

    walks = [dict(d=d, kinds=list(kinds), periods_scaled=per, fc0=f0, patience=patience, max_sweeps=max_sweeps,
                  factors=tuple(factors), start=start, free=free, cheap=cheap) for _ in tr]
    res, stats = search_batched(obj_batch, walks, batch=batch)
    out = [(modes_of(fc), best) for fc, best in res]
    return (out, stats) if return_stats else out


# ---------------------------------------------------------------------------------------------------- entry points
# The selector's public entry points (selector.py:617-732): select on points and select_counts on counts on a fixed
# lattice, both fitting BLMLQuick (here the GPU point / lattice fit of blml_b200.quick, real rank 1).

def _estimator_class(engine):
    """The point estimator for engine 'cpu' | 'gpu' (selector.py:113-118); this engine fits on the GPU for both."""
    if engine not in ('cpu', 'gpu'):
        raise ValueError(f"engine must be 'cpu' or 'gpu', got {engine}")
    from .quick import BLMLQuick
    return BLMLQuick


def _lattice_estimator(tol):
    """The fixed-lattice estimator of select_counts (selector.py:706-708), float64 state."""
    return _estimator_class('gpu')(dtype=np.float64, tol=tol)


def _wmean(v, w):
    return float(np.mean(v)) if w is None else float(np.average(v, weights=w))


def _wquantile(X, q, w):
    """Per-column quantiles q (%) of X weighted by w (selector.py:39-51): np.percentile's linear rule on the points
    repeated w times; constant or no weights: np.percentile itself."""
    if w is None or np.all(w == w[0]):
        return np.percentile(X, q, axis=0)
    out = np.empty((len(q), X.shape[1]))
    qs = np.asarray(q, float) / 100.0
    for j in range(X.shape[1]):
        o = np.argsort(X[:, j], kind='stable')
        xs = X[o, j]
        cw = np.cumsum(w[o])
        N = cw[-1]
        pos = qs * (N - 1)
        lo = np.floor(pos)
        hi = np.minimum(lo + 1, np.floor(N - 1))
        at = lambda k: xs[np.minimum(np.searchsorted(cw, k, side='right'), len(xs) - 1)]
        out[:, j] = at(lo) + (pos - lo) * (at(hi) - at(lo))
    return out


def _radial_groups(kinds):
    """[(name, [columns])] of the ball / pball groups in order of first appearance (blml_trivial.py:251-261)."""
    groups = {}
    for j, k in enumerate(kinds or []):
        if is_group(k):
            name, tag = split_kind(k)
            groups.setdefault(tag, (name, []))[1].append(j)
    return list(groups.values())


def _template(modes, d):
    """kinds, periods, dep, rank and fc (K, d; NaN where missing) of a modes template (selector.py:54-61)."""
    from .spec import parse_modes, modes_fc
    specs, dep = parse_modes(modes, d, need_fc=False)
    if any(sp['kinds'] != specs[0]['kinds'] or sp['periods'] != specs[0]['periods'] for sp in specs):
        raise ValueError("selector: modes must share kind, period and group per column (fc may differ)")
    return specs[0]['kinds'], specs[0]['periods'], dep, len(specs), modes_fc(modes)


def _start_free(start, free, iqr, d):
    """Scaled start (NaN where none), the trainable mask and the columns a shared bracket grows (selector.py:75-82)."""
    st = np.full(d, np.nan) if start is None else np.asarray(start, float) * iqr
    fr = np.ones(d, bool) if free is None else np.asarray(free, bool)
    if start is not None and np.any(~fr & ~np.isfinite(st)):
        raise ValueError("a fixed (non-trainable) fc needs a value")
    return st, fr, fr & ~np.isfinite(st)


def _tie(fc, kinds):
    """fc equalised within each radial group (geometric mean, selector.py:89-94)."""
    fc = np.array(fc, dtype=float)
    for _, dims in _radial_groups(kinds):
        fc[dims] = np.exp(np.log(fc[dims]).mean())
    return fc


def _split(Xtr, iqr, seed, X_val, sw=None, sw_val=None):
    """Training / validation points in scaled units (selector.py:126-135): X_val scaled by the training IQR, or a
    seeded 80/20 permutation split of the training points (their weights follow)."""
    if X_val is not None:
        return Xtr, np.asarray(X_val, dtype=float) / iqr, sw, sw_val
    rng = np.random.default_rng(seed)
    n = len(Xtr)
    idx = rng.permutation(n)
    n2 = int(0.8 * n)
    sub = lambda a, i: None if a is None else a[i]
    return Xtr[idx[:n2]], Xtr[idx[n2:]], sub(sw, idx[:n2]), sub(sw, idx[n2:])


def _scale_data(X, kinds, periods, sw=None):
    """(scaled points, scaled periods, IQR) (selector.py:137-159): each column divided by its (weighted) IQR, a radial
    group by its columns' geometric-mean IQR; dirichlet / pball periods scaled with their columns."""
    q75, q25 = _wquantile(np.asarray(X, float), [75, 25], sw)
    iqr = np.maximum(q75 - q25, 1e-10)
    for _, dims in _radial_groups(kinds):
        iqr[dims] = np.exp(np.log(iqr[dims]).mean())
    Xs = X / iqr
    per = None
    if periods is not None:
        per = [p / iqr[k] if (p is not None and kinds is not None and k < len(kinds) and
                              split_kind(kinds[k])[0] in ('dirichlet', 'pball')) else p
               for k, p in enumerate(periods)]
    return Xs, per, iqr


def _shared_step(shared_step, d):
    return 2.0 ** (1.0 / d) if shared_step == 'volume' else float(shared_step) if not isinstance(shared_step, str) \
        else 2.0


def _fit(Est, X, fc, kinds, periods, rank=1, complex_g=False, sw=None):
    """One fit at cut-offs fc with the template's kinds / periods (selector.py:30-34)."""
    kw = {} if sw is None else dict(sample_weight=sw)
    return Est().fit(X, make_modes(fc, kinds, periods, rank, d=X.shape[1]), complex_g=complex_g, **kw)


def _vll_fn(Est, Xa, Xb, kinds, periods_scaled, rank, complex_g, wa, wb, jac):
    def vll(fc):
        m = _fit(Est, Xa, fc, kinds, periods_scaled, rank, complex_g, sw=wa)
        return _wmean(np.log(np.maximum(m.predict(Xb).ravel(), 1e-300)), wb) - jac
    return vll


def _cond_vll_fn(Est, Xa, Xb, kinds, periods_scaled, dep, iqr, rank, complex_g, wa, wb):
    """The conditional validation score (selector.py:318-357, method 'ratio' with separate fits): the mean of
    log p_joint - log p_marginal over the validation points, the marginal fitted on the other columns with the same
    fc, less the dep columns' log IQR (original units)."""
    d = Xa.shape[1]
    dep_idx = sorted(set(int(i) for i in np.atleast_1d(dep)))
    if not dep_idx or any(i < 0 or i >= d for i in dep_idx):
        raise ValueError(f"dep indices {dep_idx} out of range for {d} dims")
    keep = [k for k in range(d) if k not in dep_idx]
    if not keep:
        raise ValueError("dep covers all dims; need at least one conditioning dim for the marginal")
    kinds_m = [kinds[k] for k in keep] if kinds else None
    per_m = [periods_scaled[k] for k in keep] if periods_scaled else None
    jac = np.log(iqr[dep_idx]).sum()

    def cvll(fc):
        fc = list(fc)
        mj = _fit(Est, Xa, fc, kinds, periods_scaled, rank, complex_g, sw=wa)
        mm = _fit(Est, Xa[:, keep], [fc[k] for k in keep], kinds_m, per_m, rank, complex_g, sw=wa)
        lj = np.log(np.maximum(mj.predict(Xb).ravel(), 1e-300))
        lm = np.log(np.maximum(mm.predict(Xb[:, keep]).ravel(), 1e-300))
        return _wmean(lj - lm, wb) - jac
    return cvll


def _objective(Est, Xa, Xb, kinds, per, rank, complex_g, wa, wb, iqr, dep):
    if dep is None:
        return _vll_fn(Est, Xa, Xb, kinds, per, rank, complex_g, wa, wb, np.log(iqr).sum())
    return _cond_vll_fn(Est, Xa, Xb, kinds, per, dep, iqr, rank, complex_g, wa, wb)


def _select_shared(X, kinds, periods, seed=0, engine='cpu', X_val=None, shared_step='double', complex_g=False,
                   rank=1, start=None, free=None, sw=None, sw_val=None, dep=None):
    """One fc for every growing scaled column, doubled from 0.2 until the validation score first drops; the peak
    (selector.py:162-195; conditional, dep given: :360-392). Returns (fc in data units, best)."""
    Est = _estimator_class(engine)
    Xs, per, iqr = _scale_data(X, kinds, periods, sw)
    Xa, Xb, wa, wb = _split(Xs, iqr, seed, X_val, sw, sw_val)
    step = _shared_step(shared_step, Xa.shape[1])
    vll = _objective(Est, Xa, Xb, kinds, per, rank, complex_g, wa, wb, iqr, dep)
    st, fr, grow = _start_free(start, free, iqr, Xa.shape[1])
    vec = lambda c: np.where(grow, c, st)
    fc = 0.2
    best = vll(vec(fc))
    if not grow.any():
        return vec(fc) / iqr, best
    prev = best
    while True:
        fc *= step
        v = vll(vec(fc))
        if v < prev:
            fc /= step
            break
        if v > best:
            best = v
        prev = v
    return vec(fc) / iqr, best


def _select_hillclimb(X, kinds, periods, seed=0, init_fc=None, engine='cpu', X_val=None, complex_g=False, rank=1,
                      start=None, free=None, sw=None, sw_val=None, dep=None):
    """Per-block doubling (x2 while it improves, else x0.5 while it improves), full sweeps until none moves
    (selector.py:197-247; conditional: :394-440, started at 0.2 in every scaled column). Returns (fc in data
    units, best)."""
    Est = _estimator_class(engine)
    Xs, per, iqr = _scale_data(X, kinds, periods, sw)
    Xa, Xb, wa, wb = _split(Xs, iqr, seed, X_val, sw, sw_val)
    n2, d = Xa.shape
    vll = _objective(Est, Xa, Xb, kinds, per, rank, complex_g, wa, wb, iqr, dep)
    if init_fc is not None:
        fc = np.array(init_fc, dtype=float)
    elif dep is not None:
        fc = np.full(d, 0.2)
    else:
        ranges = np.maximum(Xa.max(axis=0) - Xa.min(axis=0), 1e-10)
        fc = 0.5 * 0.1 * (n2 ** -0.25) / ranges
    st, fr, _ = _start_free(start, free, iqr, d)
    fc = _tie(np.where(np.isfinite(st), st, fc), kinds)
    best = vll(fc)
    while True:
        moved = False
        for k in free_blocks(kinds, d, fr):
            improved = False
            for factor, tried_up in ((2.0, False), (0.5, True)):
                if tried_up and improved:
                    break
                while True:
                    cand = fc.copy()
                    cand[k] *= factor
                    v = vll(cand)
                    if v > best:
                        best, fc, improved = v, cand, True
                    else:
                        break
            moved = moved or improved
        if not moved:
            break
    return fc / iqr, best


def _select_auto(X, kinds, periods, seed=0, engine='cpu', X_val=None, fc0=0.2, complex_g=False, rank=1,
                 factors=(SQRT2,), start=None, free=None, sw=None, sw_val=None, dep=None):
    """The volume-grid shared search and the harmonic-aware refinement (search) on the validation score, joint or
    conditional (selector.py:554-613, rank 1 / shared modes). Returns (fc in data units, best)."""
    X = np.asarray(X, dtype=float)
    Xs, per, iqr = _scale_data(X, kinds, periods, sw)
    Xa, Xb, wa, wb = _split(Xs, iqr, seed, X_val, sw, sw_val)
    d = Xa.shape[1]
    obj = _objective(_estimator_class(engine), Xa, Xb, kinds, per, rank, complex_g, wa, wb, iqr, dep)
    st = None if start is None else np.asarray(start, float) * iqr
    fc, best = search(obj, d, kinds, per, fc0=fc0, factors=factors, start=st, free=free)
    return fc / iqr, best


def select(Xtr_raw, modes, search='shared_hillclimb', seed=0, init_fc=None, engine='cpu', cond_method='ratio',
           X_val=None, shared_step='double', signs=None, complex_g=False, factors=(SQRT2,), separate_modes=False,
           sample_weight=None, val_weight=None):
    """fc for a modes template on points (selector.py:617-666): IQR-scaled columns, a validation split (or X_val), the
    search pattern 'shared_hillclimb' (default), 'shared', 'hillclimb' or 'auto', each candidate a BLMLQuick fit
    scored by the mean log density of the validation points (in data units); dep columns in the modes give the
    conditional score, mean log(p_joint / p_marginal), the marginal a second fit on the other columns with the same
    fc. Returns (modes with the selected fc, best). The GPU fits are real rank 1: signs, complex_g, rank > 1 and
    separate_modes raise NotImplementedError."""
    if search not in ('shared_hillclimb', 'shared', 'hillclimb', 'auto'):
        raise ValueError(f"search must be 'shared_hillclimb', 'shared', 'hillclimb' or 'auto', got {search}")
    if cond_method != 'ratio':
        raise ValueError(f"cond_method must be 'ratio', got {cond_method}")
    Xtr_raw = np.asarray(Xtr_raw, dtype=float)
    sw = None if sample_weight is None else np.asarray(sample_weight, float)
    sw_val = None if val_weight is None else np.asarray(val_weight, float)
    kinds, periods, dep, K, F = _template(modes, Xtr_raw.shape[1])
    if signs is not None and dep is not None:
        raise ValueError("signs with dep=... (the marginal's g has its own signs)")
    if signs is not None or complex_g or K > 1 or separate_modes:
        raise NotImplementedError("select on the GPU: real rank-1 fits (no signs, complex_g, rank > 1)")
    from .spec import modes_trainable, with_fc
    T = modes_trainable(modes)
    start, free = F[0], T[0]
    start = None if np.all(np.isnan(start)) else start
    free = None if np.all(free) else free
    sf = dict(start=start, free=free, sw=sw, sw_val=sw_val, dep=dep)
    if search == 'auto':
        fc, best = _select_auto(Xtr_raw, kinds, periods, seed, engine, X_val, factors=factors, **sf)
    elif search == 'shared':
        fc, best = _select_shared(Xtr_raw, kinds, periods, seed, engine, X_val, shared_step, **sf)
    elif search == 'hillclimb':
        fc, best = _select_hillclimb(Xtr_raw, kinds, periods, seed, init_fc, engine, X_val, **sf)
    else:
        fc_shared, _ = _select_shared(Xtr_raw, kinds, periods, seed, engine, X_val, shared_step, **sf)
        _, _, iqr = _scale_data(Xtr_raw, kinds, periods, sw)
        fc, best = _select_hillclimb(Xtr_raw, kinds, periods, seed, fc_shared * iqr, engine, X_val, free=free, sw=sw,
                                     sw_val=sw_val, dep=dep)
    return with_fc(modes, fc), best


def select_counts(Z, w_tr, w_va, h, modes, complex_g=False, separate_modes=False, fc0=None, fc_max=None, tag='counts',
                  factors=(SQRT2,), engine='cpu', **fit_kw):
    """fc for counts on a fixed lattice (selector.py:670-732): fit (Z, w_tr) with the modes on the lattice h, score
    the mean log-probability of the validation counts w_va with bin probabilities f(z_b) normalised over the bins
    given (Z should be the full grid, empty bins included); the search of `search` from fc0 (default 0.1 fc_max),
    fc capped at fc_max (default 1 / h per column). Returns (modes with the selected fc, best). Real rank 1 on the
    GPU: dep, complex_g, rank > 1 and separate_modes raise NotImplementedError."""
    from .spec import modes_trainable, with_fc, with_lattice
    Z = np.atleast_2d(np.asarray(Z, float))
    d = Z.shape[1]
    kinds, periods, dep, K, F = _template(modes, d)
    if dep is not None or complex_g or K > 1 or separate_modes:
        raise NotImplementedError("select_counts on the GPU: real rank-1 joint fits (no dep, complex_g, rank > 1)")
    T = modes_trainable(modes)
    start = None if np.all(np.isnan(F[0])) else np.asarray(F[0], float).ravel()
    free = None if np.all(T[0]) else np.asarray(T[0], bool).ravel()
    periods = list(periods) if periods is not None else [None] * d
    h_vec = np.broadcast_to(np.asarray(h, float), (d,)).copy()
    cap = np.broadcast_to(np.asarray(fc_max if fc_max is not None else 1.0 / h_vec, float), (d,))
    w_tr = np.asarray(w_tr, float).ravel()
    w_va = np.asarray(w_va, float).ravel()

    def obj(fcv):
        Fv = np.asarray(fcv, float).reshape(1, d)
        if np.any(Fv > cap[None] * (1 + 1e-9)):
            return -np.inf
        m = _lattice_estimator(fit_kw.get('tol', 1e-5))
        m.fit(Z, with_lattice(make_modes(Fv[0], kinds, periods, 1, d=d), h_vec), sample_weight=w_tr)
        P = np.maximum(m.predict(Z), 1e-300)
        P = P / P.sum()
        return float(w_va @ np.log(P) / w_va.sum())
    f0 = float(fc0) if fc0 is not None else 0.1 * float(cap.min())
    fc, best = search(obj, d, kinds, periods, fc0=f0, tag=tag, factors=factors, start=start, free=free)
    return with_fc(modes, fc), best
