"""The batched cut-off search on the GPU: the validation-score kernel against NumPy on the fitted densities, and
select_counts_batched end to end on three lattices: its selected cut-offs are the ones the sequential search
(selector.py:488-553, one candidate at a time) picks from the same candidate scores, the selection is a local optimum
of the search's moves, and the speculative rounds are fewer than the candidates the searches used."""
import numpy as np
import pytest

from blml_b200 import workloads, make_modes

pytestmark = pytest.mark.gpu


def _split(c, seed):
    rng = np.random.default_rng(seed)
    tr = rng.binomial(c.astype(np.int64), 0.8).astype(float)
    return tr, c - tr


def test_val_score_matches_numpy(cuda_device):
    from blml_b200.sweep import BLMLBinnedBatch
    shapes, fcs = [(32, 32), (40, 48), (24, 24)], [(0.2, 0.3), (0.15, 0.15), (0.35, 0.25)]
    tr, va, modes = [], [], []
    for i, (sh, fc) in enumerate(zip(shapes, fcs)):
        t, v = _split(workloads.two_disk_field(sh, fc=0.3, N=3e4, seed=i), i)
        tr.append(t); va.append(v); modes.append(make_modes(list(fc), ['sinc', 'sinc']))
    for dt, tol in ((np.float64, 1e-12), (np.float32, 1e-5)):
        b = BLMLBinnedBatch(tol=1e-6, max_sweeps=300, dtype=dt)
        res = b.fit(tr, modes)
        got = b.val_score(va)
        for f, r in enumerate(res):
            p = np.maximum(r.density_.astype(np.float64), 1e-300)
            ref = float(np.sum(va[f] * np.log(p / p.sum())) / va[f].sum())
            assert abs(got[f] - ref) <= tol * abs(ref), (dt, f, got[f], ref)
        with pytest.raises(ValueError):
            b.val_score(va[:2])


def test_select_counts_batched(cuda_device):
    from blml_b200 import selector as ps
    tr, va = [], []
    for i, (sh, fc, N) in enumerate((((32, 32), 0.3, 4e4), ((40, 40), 0.2, 8e4), ((32, 48), 0.35, 2e4))):
        t, v = _split(workloads.two_disk_field(sh, fc=fc, N=N, seed=20 + i), i)
        tr.append(t); va.append(v)
    scores = [dict() for _ in tr]
    real = ps.search_batched

    def recording(obj_batch, walks, batch=64, max_depth=24):
        def rec(reqs):
            out = obj_batch(reqs)
            for (s, fc), v in zip(reqs, out):
                scores[s][ps._key(fc)] = float(v)
            return out
        return real(rec, walks, batch=batch, max_depth=max_depth)
    ps.search_batched = recording
    try:
        out, stats = ps.select_counts_batched(tr, va, fc0=0.05, factors=(ps.SQRT2,), batch=48, tol=1e-6,
                                              max_fit_sweeps=3000, return_stats=True)
    finally:
        ps.search_batched = real
    assert stats['rounds'] < stats['used'] <= stats['fits']
    for s, (modes, best) in enumerate(out):
        fc = np.array([modes[0][0]['fc'], modes[0][1]['fc']])
        assert np.all(fc <= 0.5) and np.isfinite(best)

        def lookup(c, s=s):
            c = np.asarray(c, float)
            if np.any(c > 0.5 * (1 + 1e-9)):
                return -np.inf
            return scores[s][ps._key(c)]
        sfc, sbest = ps.search(lookup, 2, ['sinc', 'sinc'], [None, None], fc0=0.05, factors=(ps.SQRT2,))
        assert np.array_equal(sfc, fc) and sbest == best
        for blk in ([0], [1]):                                 # no move of the last factor improves by > 1e-6
            for fac in (ps.SQRT2, 1 / ps.SQRT2):
                k = ps._key(ps.move(fc, blk, fac, ['sinc', 'sinc'], [None, None]))
                if k in scores[s]:
                    assert scores[s][k] <= best + 1e-6
