"""The cut-off search on the host: the oracle against the reference's own request sequences
(tests/golden/selector_search.json, made by tests/golden/make_selector_golden.py), the product's generator walk
against both, and the batched driver (speculative rounds over many searches) against the sequential search: the same
(fc, best) for every search, every candidate the sequential search scored among those the batched run scored, and
fewer rounds than sequential fits. Candidates are memoised on log fc rounded to 6 decimals (selector.py:497), so a
speculative branch may score another float representative of a candidate the sequential walk reaches: the batched
driver's best agrees to 1e-12 relative, its fc exactly."""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN
import selector_oracle as so
from selector_cases import CASES, bowl, hashed, R2, F3
from blml_b200 import selector as ps

with open(os.path.join(GOLDEN, 'selector_search.json')) as fh:
    GOLD = json.load(fh)


def _same_best(a, b):
    return a == b or (np.isnan(a) and np.isnan(b)) or abs(a - b) <= 1e-12 * abs(b)


def _args(c):
    return c['d'], c['kinds'], c['periods_scaled']


@pytest.mark.parametrize('name', sorted(CASES))
def test_oracle_matches_reference(name):
    c, g = CASES[name], GOLD[name]
    fc, best, calls = so.search(c['obj'], *_args(c), **c['kw'])
    assert len(calls) == len(g['calls'])
    for a, b in zip(calls, g['calls']):
        assert np.array_equal(a, np.array(b))
    assert np.array_equal(fc, g['fc']) and best == g['best']


@pytest.mark.parametrize('name', sorted(CASES))
def test_walk_matches_reference(name):
    c, g = CASES[name], GOLD[name]
    calls = []

    def obj(fc):
        calls.append(np.array(fc, float))
        return c['obj'](fc)
    fc, best = ps.search(obj, *_args(c), **c['kw'])
    assert len(calls) == len(g['calls'])
    for a, b in zip(calls, g['calls']):
        assert np.array_equal(a, np.array(b))
    assert np.array_equal(fc, g['fc']) and best == g['best']


def _batched(cases, batch, cheap=None):
    objs = [c['obj'] for c in cases]
    walks = [dict(d=c['d'], kinds=c['kinds'], periods_scaled=c['periods_scaled'], **c['kw']) for c in cases]
    if cheap is not None:
        for w in walks:
            w['cheap'] = cheap
    seen = [[] for _ in cases]

    def obj_batch(reqs):
        out = []
        for s, fc in reqs:
            seen[s].append(ps._key(fc))
            out.append(objs[s](fc))
        return out
    res, stats = ps.search_batched(obj_batch, walks, batch=batch)
    return res, stats, seen


@pytest.mark.parametrize('batch', [1, 4, 16, 64, 512])
def test_batched_matches_sequential(batch):
    names = sorted(CASES)
    res, stats, seen = _batched([CASES[n] for n in names], batch)
    for (fc, best), n, keys in zip(res, names, seen):
        g = GOLD[n]
        assert np.array_equal(fc, g['fc']) and _same_best(best, g['best'])
        assert {ps._key(np.array(x)) for x in g['calls']} <= set(keys)
        assert len(keys) == len(set(keys))                   # no candidate scored twice
    seq = sum(len(GOLD[n]['calls']) for n in names)
    assert stats['used'] == seq
    assert stats['rounds'] <= max(len(GOLD[n]['calls']) for n in names)
    if batch >= 64:
        assert stats['rounds'] < 0.6 * max(len(GOLD[n]['calls']) for n in names)


def test_single_search_speculation_saves_rounds():
    c = CASES['sinc2_fine']
    res, stats, _ = _batched([c], 32)
    assert np.array_equal(res[0][0], GOLD['sinc2_fine']['fc'])
    assert stats['rounds'] * 2 <= len(GOLD['sinc2_fine']['calls'])


def test_cheap_scores_cost_no_fit():
    """-inf outside the band comes from the host-side score, not from obj_batch."""
    c = dict(CASES['sinc3_rugged_cap'])
    cap = lambda fc: -np.inf if np.any(np.asarray(fc) > 0.5) else None
    res, stats, seen = _batched([c], 16, cheap=cap)
    assert np.array_equal(res[0][0], GOLD['sinc3_rugged_cap']['fc'])
    for k in seen[0]:
        assert np.all(np.exp(np.array(k)) <= 0.5 * (1 + 1e-6))


def _random_case(rng):
    d = int(rng.integers(1, 5))
    kinds = list(rng.choice(['sinc', 'dirichlet', 'pball'], d, p=[0.6, 0.2, 0.2]))
    if kinds.count('pball') == 1:
        kinds[kinds.index('pball')] = 'sinc'
    per = [float(rng.uniform(8, 64)) if k == 'dirichlet' else None for k in kinds]
    centre = np.exp(rng.uniform(np.log(0.01), np.log(0.45), d))
    for j, k in enumerate(kinds):
        if k == 'pball':
            centre[j] = centre[kinds.index('pball')]
    kw = dict(fc0=float(np.exp(rng.uniform(np.log(0.005), np.log(0.3)))), patience=int(rng.integers(0, 4)),
              max_sweeps=int(rng.integers(1, 7)), factors=[(R2,), (R2, 2.0 ** 0.25), F3][int(rng.integers(3))])
    if d > 1 and rng.uniform() < 0.3:
        st = np.full(d, np.nan); j = int(rng.integers(d))
        if kinds[j] != 'pball':
            st[j] = float(centre[j] * np.exp(rng.normal(0, 0.5)))
            kw['start'] = st
            if rng.uniform() < 0.5:
                fr = np.ones(d, bool); fr[j] = False; kw['free'] = fr
    if rng.uniform() < 0.5:
        obj = bowl(centre, cap=0.5 if rng.uniform() < 0.5 else None, ripple=float(rng.uniform(0, 0.1)),
                   freq=float(rng.uniform(3, 15)))
    else:
        obj = hashed(int(rng.integers(1 << 30)), float(rng.uniform(0.01, 1.0)))
    return dict(d=d, kinds=kinds, periods_scaled=per, kw=kw, obj=obj)


def test_batched_matches_oracle_on_random_searches():
    rng = np.random.default_rng(5)
    cases = [_random_case(rng) for _ in range(40)]
    want = [so.search(c['obj'], *_args(c), **c['kw']) for c in cases]
    for batch in (8, 96):
        res, stats, seen = _batched(cases, batch)
        for (fc, best), (wfc, wbest, calls), keys in zip(res, want, seen):
            assert np.array_equal(fc, wfc) and _same_best(best, wbest)
            assert {ps._key(x) for x in calls} <= set(keys)
        assert stats['used'] == sum(len(w[2]) for w in want)


def test_blocks_and_move_match_oracle():
    for kinds, d in ((['sinc', 'ball:a', 'sinc', 'ball:a'], 4), (['pball', 'pball', 'dirichlet'], 3),
                     (None, 3), (['ball:x', 'ball:y', 'ball:x', 'ball:y', 'slits:0.5'], 5)):
        assert ps.blocks(kinds, d) == so.blocks(kinds, d)
    fc = np.array([0.1, 0.2, 0.0625])
    for blk, fac in (([2], R2), ([2], 1 / R2), ([0, 1], 2.0), ([2], 0.5)):
        a = ps.move(fc, blk, fac, ['pball', 'pball', 'dirichlet'], [None, None, 16.0])
        b = so.move(fc, blk, fac, ['pball', 'pball', 'dirichlet'], [None, None, 16.0])
        assert (a is None and b is None) or np.array_equal(a, b)
    assert ps.move(np.array([0.05]), [0], 0.5, ['dirichlet'], [16.0]) is None
    with pytest.raises(ValueError):
        ps.blocks(['ball:a', 'pball:a'], 2)
    with pytest.raises(ValueError):
        ps.blocks(['gauss'], 1)
