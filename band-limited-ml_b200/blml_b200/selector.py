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


# ---------------------------------------------------------------------------------------------------- counts entry
def _lattice_estimator(tol):
    """The fixed-lattice fit that scores a select_counts candidate: blml_b200.quick.BLMLQuick on the GPU, float64."""
    from .quick import BLMLQuick
    return BLMLQuick(dtype=np.float64, tol=tol)


def select_counts(Z, w_tr, w_va, h, modes, complex_g=False, separate_modes=False, fc0=None, fc_max=None, tag='counts',
                  factors=(SQRT2,), engine='cpu', **fit_kw):
    """fc of a one-mode template for counts on a fixed lattice (the reference's entry, selector.py:716-732): the
    search of `search` over fc, each candidate a fit of the training counts w_tr at the lattice points Z (step h)
    scored by the mean log-probability of the validation counts w_va, bin probabilities being the fitted density
    normalised over the points given (so Z should hold the whole grid, empty bins included). The template's fc
    values start the search (NaN: from fc0, default a tenth of the cap) and its non-trainable columns stay fixed;
    no column goes above fc_max (default 1 / h). Returns (modes with the selected fc, best score). Real rank-1
    joint fits only: dep columns, complex_g, K > 1 and separate_modes raise NotImplementedError. `engine` is
    accepted for the reference's signature; the fits run on the GPU."""
    from .spec import parse_modes, modes_fc, modes_trainable, with_fc, with_lattice
    pts = np.atleast_2d(np.asarray(Z, float))
    d = pts.shape[1]
    specs, dep = parse_modes(modes, d, need_fc=False)
    if dep is not None or complex_g or len(specs) != 1 or separate_modes:
        raise NotImplementedError("select_counts on the GPU: real rank-1 joint fits (no dep, complex_g, rank > 1)")
    kinds, periods = specs[0]['kinds'], specs[0]['periods']
    fc_tpl = np.asarray(modes_fc(modes), float).reshape(-1, d)[0]
    train_mask = np.asarray(modes_trainable(modes), bool).reshape(-1, d)[0]
    step = np.ones(d) * np.asarray(h, float)
    ceiling = np.ones(d) * np.asarray(1.0 / step if fc_max is None else fc_max, float)
    train = np.asarray(w_tr, float).ravel()
    held = np.asarray(w_va, float).ravel()
    held_n = held.sum()
    tol = fit_kw.get('tol', 1e-5)

    def held_out_score(fc):
        fc = np.asarray(fc, float).ravel()
        if np.any(fc > ceiling * (1 + 1e-9)):
            return -np.inf
        est = _lattice_estimator(tol)
        est.fit(pts, with_lattice(make_modes(fc, kinds, periods, 1, d=d), step), sample_weight=train)
        p = np.maximum(est.predict(pts), 1e-300)
        return float(held @ np.log(p / p.sum()) / held_n)

    first = 0.1 * float(ceiling.min()) if fc0 is None else float(fc0)
    fc, best = search(held_out_score, d, kinds, list(periods), fc0=first, tag=tag, factors=factors,
                      start=None if np.all(np.isnan(fc_tpl)) else fc_tpl,
                      free=None if np.all(train_mask) else train_mask)
    return with_fc(modes, fc), best
