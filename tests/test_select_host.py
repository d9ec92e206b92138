"""The selector's entry points on the host (blml_b200.selector.select / select_counts) against the reference's own
(tests/golden/select.json, made by tests/golden/make_select_golden.py): both run with the deterministic stand-in
estimator of tests/selector_cases.py (StubQuick) in place of BLMLQuick, so the IQR scaling, the validation split,
the search patterns (shared, shared with volume steps, hillclimb, shared_hillclimb, auto), weights, fixed columns,
radial groups and the counts objective must request the same fits, in the same order, and select the same fc."""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN
from selector_cases import StubQuick, SELECT_CASES, COUNTS_CASES, select_points, counts_lattice
from blml_b200 import selector as ps
from blml_b200.spec import modes_fc

with open(os.path.join(GOLDEN, 'select.json')) as fh:
    GOLD = json.load(fh)


@pytest.fixture
def stub(monkeypatch):
    monkeypatch.setattr(ps, '_estimator_class', lambda engine: StubQuick)
    monkeypatch.setattr(ps, '_lattice_estimator', lambda tol: StubQuick())
    StubQuick.calls = []
    yield StubQuick


def _check(name, m, best):
    g = GOLD[name]
    assert len(StubQuick.calls) == len(g['calls'])
    for a, b in zip(StubQuick.calls, g['calls']):
        assert np.array_equal(a, np.array(b)), (a, b)
    assert np.array_equal(modes_fc(m), np.array(g['fc'])) and best == g['best']


@pytest.mark.parametrize('name', list(SELECT_CASES))
def test_select_matches_reference(stub, name):
    n, seed, modes, kw, with_val, weighted = SELECT_CASES[name]
    X = select_points(n, seed)
    extra = {}
    if with_val:
        extra['X_val'] = select_points(n // 4, seed + 50)
    if weighted:
        r = np.random.default_rng(seed + 60)
        extra['sample_weight'] = r.integers(1, 4, n).astype(float)
        if with_val:
            extra['val_weight'] = r.integers(1, 4, n // 4).astype(float)
    m, best = ps.select(X, modes, **kw, **extra)
    _check(name, m, best)


@pytest.mark.parametrize('name', list(COUNTS_CASES))
def test_select_counts_matches_reference(stub, name):
    shape, seed, modes, kw = COUNTS_CASES[name]
    Z, w_tr, w_va, h = counts_lattice(shape, seed)
    m, best = ps.select_counts(Z, w_tr, w_va, h, modes, **kw)
    _check(name, m, best)


def test_weighted_quantile_repeats_points():
    rng = np.random.default_rng(0)
    X = rng.normal(size=(50, 2)); w = rng.integers(1, 5, 50).astype(float)
    rep = np.repeat(X, w.astype(int), axis=0)
    assert np.allclose(ps._wquantile(X, [25, 75], w), np.percentile(rep, [25, 75], axis=0))


def test_unsupported_options_raise(stub):
    X = select_points(100, 0)
    with pytest.raises(NotImplementedError):
        ps.select(X, [{0: dict(kind='sinc'), 1: dict(kind='sinc')}], complex_g=True)
    with pytest.raises(ValueError):
        ps.select(X, [{0: dict(kind='sinc'), 1: dict(kind='sinc')}], search='grid')
