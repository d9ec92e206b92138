"""CPU oracle of the selector's cut-off search (TEST INFRASTRUCTURE ONLY: the product path never calls this).

A plain-loop restatement of rahuljhu/band-limited-ml selector.py: `_blocks` (:58-72), `_free_blocks` (:85-86),
`_harmonics` / `_move` (:467-487) and `_search` (:488-553), one objective call per uncached candidate, in the
reference's order. It is pinned by tests/golden/selector_search.json, which holds the reference's own request
sequences and results on deterministic objectives (tests/golden/make_selector_golden.py), and it checks the product's
generator walk and its batched driver (blml_b200/selector.py) on many more objectives than the fixtures hold.
"""
import numpy as np

RADIAL = ('ball', 'pball')


def _kind(k):
    return str(k).partition(':')


def blocks(kinds, d):
    """selector.py:58-72 (radial_groups: blml_trivial.py:251-261)."""
    groups = {}
    for k, kind in enumerate(kinds or []):
        name, _, tag = _kind(kind)
        if name in RADIAL:
            groups.setdefault(tag, []).append(k)
    out, seen = [], set()
    for k in range(d):
        g = next((dims for dims in groups.values() if k in dims), None)
        if g is None:
            out.append([k])
        elif g[0] not in seen:
            out.append(list(g))
            seen.add(g[0])
    return out


def harmonics(fc_s, Ps):
    return int(np.floor(fc_s * Ps / 2.0))


def move(fc, block, factor, kinds, periods_scaled):
    """selector.py:470-487."""
    new = fc.copy()
    new[block] *= factor
    if len(block) > 1:
        return new
    k = block[0]
    if kinds is not None and _kind(kinds[k])[0] == 'dirichlet':
        Ps = periods_scaled[k]
        a, b = harmonics(fc[k], Ps), harmonics(new[k], Ps)
        if a == b:
            b = a + 1 if factor > 1 else a - 1
            if b < 0:
                return None
            new[k] = (b + 0.5) * 2.0 / Ps
    return new


def search(obj, d, kinds, periods_scaled, fc0=0.2, patience=2, max_sweeps=6, factors=(np.sqrt(2.0),), start=None,
           free=None):
    """selector.py:488-553; returns (fc, best, calls) with calls the candidates obj was called on, in order."""
    cache, calls = {}, []

    def f(fc):
        key = tuple(np.round(np.log(fc), 6))
        if key not in cache:
            calls.append(np.array(fc, float))
            cache[key] = obj(fc)
        return cache[key]

    st = np.full(d, np.nan) if start is None else np.asarray(start, float)
    fr = np.ones(d, bool) if free is None else np.asarray(free, bool)
    grow = fr & ~np.isfinite(st)
    dg = int(grow.sum())
    fc = np.where(grow, float(fc0), st)
    best_fc, best = fc.copy(), f(fc)
    bad = 0
    while dg and bad <= patience:
        fc = np.where(grow, fc * 2.0, fc)
        ll = f(fc)
        if ll > best:
            best, best_fc, bad = ll, fc.copy(), 0
        else:
            bad += 1
    centre = best_fc.copy()
    for sign in (1, -1):
        improved = False
        for j in range(1, dg):
            cand = np.where(grow, centre * 2.0 ** (sign * j / dg), centre)
            ll = f(cand)
            if ll > best:
                best, best_fc, improved = ll, cand, True
            else:
                break
        if improved:
            break
    fc = best_fc
    fblocks = [b for b in blocks(kinds, d) if all(fr[b])]
    for factor in factors:
        for _ in range(max_sweeps):
            moved = False
            for blk in fblocks:
                for fac in (factor, 1.0 / factor):
                    stepped = False
                    while True:
                        cand = move(fc, blk, fac, kinds, periods_scaled)
                        if cand is None:
                            break
                        ll = f(cand)
                        if ll > best + 1e-6:
                            best, fc, moved, stepped = ll, cand, True, True
                        else:
                            break
                    if stepped:
                        break
            if not moved:
                break
    return fc, best, calls
