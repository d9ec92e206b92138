"""The selector's counts entry point on the host (blml_b200.selector.select_counts) against the reference's own
(tests/golden/select.json, made by tests/golden/make_select_golden.py): both run with the deterministic stand-in
estimator of tests/selector_cases.py (StubQuick) in place of BLMLQuick, so the template handling, the cap, the start
and the counts objective must request the same fits, in the same order, and select the same fc."""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN
from selector_cases import StubQuick, COUNTS_CASES, counts_lattice
from blml_b200 import selector as ps
from blml_b200.spec import modes_fc

with open(os.path.join(GOLDEN, 'select.json')) as fh:
    GOLD = json.load(fh)


@pytest.fixture
def stub(monkeypatch):
    monkeypatch.setattr(ps, '_lattice_estimator', lambda tol: StubQuick())
    StubQuick.calls = []
    yield StubQuick


def _check(name, m, best):
    g = GOLD[name]
    assert len(StubQuick.calls) == len(g['calls'])
    for a, b in zip(StubQuick.calls, g['calls']):
        assert np.array_equal(a, np.array(b)), (a, b)
    assert np.array_equal(modes_fc(m), np.array(g['fc'])) and best == g['best']


@pytest.mark.parametrize('name', list(COUNTS_CASES))
def test_select_counts_matches_reference(stub, name):
    shape, seed, modes, kw = COUNTS_CASES[name]
    Z, w_tr, w_va, h = counts_lattice(shape, seed)
    m, best = ps.select_counts(Z, w_tr, w_va, h, modes, **kw)
    _check(name, m, best)


def test_unsupported_options_raise(stub):
    shape, seed, modes, kw = next(iter(COUNTS_CASES.values()))
    Z, w_tr, w_va, h = counts_lattice(shape, seed)
    with pytest.raises(NotImplementedError):
        ps.select_counts(Z, w_tr, w_va, h, modes, complex_g=True)
    with pytest.raises(NotImplementedError):
        ps.select_counts(Z, w_tr, w_va, h, list(modes) * 2)
