"""Streaming fits on the GPU (blml_b200.streaming.BLMLBinnedStreaming: warm refits per batch, prequential scores, fc
learning by Adam on the implicit / fixed-coefficient gradients and by hill-climbs, leave-batch-out epochs, burn-in
selection) against the reference's own streams (tests/golden/stream.npz, made by tests/golden/make_stream_golden.py).
The real rank-1 fits are convex, so the streams must agree closely: prequential scores and the final loglik to 1e-7
relative, every fc of the trajectory to 1e-6, the discrete moves (hill-climb, burn-in selection) exactly; the stream
whose refits are capped at 50 sweeps to 1e-5 (the capped iterate carries the solvers' rounding). The complex stream is
non-convex: a rounding-level change of trajectory can end at a nearby optimum, whose fc gradient differs, and Adam's
second step depends on the ratio of two pooled gradients. There the same moves must happen on the same batches, the
first step must agree to 1e-6 (one Adam step is lr times the gradient's sign), the prequential scores to 5e-3 and the
later fc to 5e-2 (a step is at most lr = 0.1 in log fc)."""
import numpy as np
import pytest

from conftest import golden
from golden_cases import STREAM_SPECS

pytestmark = pytest.mark.gpu

# (prequential scores and loglik, fc trajectory)
BARS = {'adam_real': (1e-7, 1e-6), 'adam_decay_capped': (1e-5, 1e-5), 'hill_dirichlet': (1e-7, 1e-6),
        'epochs_loo': (1e-7, 1e-6), 'burnin_select': (1e-7, 1e-6), 'complex_adam': (5e-3, 5e-2)}


def _run(name):
    from blml_b200.streaming import BLMLBinnedStreaming
    g = golden('stream.npz')[name]
    shape, modes, ckw, how, fkw, nb, per = STREAM_SPECS[name]
    m = BLMLBinnedStreaming(dtype=np.float64, **ckw)
    if how == 'partial':
        for b in g['batches']:
            m.partial_fit(b, modes, **fkw)
    else:
        m.fit(list(g['batches']), modes, epochs=how[1], **fkw)
    return g, m


@pytest.mark.parametrize('name', list(STREAM_SPECS))
def test_stream_matches_reference(cuda_device, name):
    g, m = _run(name)
    pbar, fbar = BARS[name]
    preq = np.array(m.preq_, float)
    assert preq.shape == g['preq'].shape and np.array_equal(np.isnan(preq), np.isnan(g['preq']))
    ok = ~np.isnan(preq)
    assert np.all(np.abs(preq[ok] - g['preq'][ok]) <= pbar * np.abs(g['preq'][ok])), (preq, g['preq'])
    fcs = np.array([h['fc'] for h in m.history_ if 'fc' in h], float)
    assert fcs.shape == g['fc_hist'].shape
    moved = np.array([len(h.get('moved', [])) for h in m.history_ if 'fc' in h])
    assert np.array_equal(moved, g['moved'])
    first = np.argmax(moved > 0) + 1 if (moved > 0).any() else len(moved)
    assert np.all(np.abs(fcs[:first] - g['fc_hist'][:first]) <= 1e-6 * np.abs(g['fc_hist'][:first]))
    assert np.all(np.abs(fcs - g['fc_hist']) <= fbar * np.abs(g['fc_hist'])), (fcs[:, 0, 0], g['fc_hist'][:, 0, 0])
    assert abs(m.loglik_ - float(g['loglik'])) <= pbar * abs(float(g['loglik']))


def test_stream_errors(cuda_device):
    from blml_b200.streaming import BLMLBinnedStreaming
    with pytest.raises(ValueError):
        BLMLBinnedStreaming(fc_update='sgd')
    m = BLMLBinnedStreaming(tol=1e-8)
    g = golden('stream.npz')['adam_real']
    with pytest.raises(ValueError):
        m.partial_fit(g['batches'][0])                      # modes on the first call
    m.partial_fit(g['batches'][0], STREAM_SPECS['adam_real'][1])
    with pytest.raises(ValueError):
        m.partial_fit(np.ones(10))                          # another lattice
