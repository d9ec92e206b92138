"""Rolling-window refits of many sequences in one batch (BLMLBinnedRolling; blml_rolling.py:40-155 refits each window
warm-started from the previous one): every sequence's fits equal the single-fit engine's fits of the same windows
with the same warm starts (init = the previous window's fit), within the batch-vs-single bar of the sweep tests."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_rolling_batch_equals_sequential_warm_fits(cuda_device):
    from blml_b200 import workloads
    from blml_b200.binned import BLMLBinned
    from blml_b200.sweep import BLMLBinnedRolling
    shapes, fcs = [(32, 32), (48, 32), (40, 40)], [0.3, 0.25, 0.35]
    seqs = []
    for s, (shape, fc) in enumerate(zip(shapes, fcs)):
        base = workloads.two_disk_field(shape, fc=fc, N=2e4, seed=100 + s)
        rng = np.random.default_rng(s)
        seqs.append([rng.poisson(base * 0.5).astype(float) + rng.poisson(0.2, base.shape) for _ in range(3)])
    modes = [workloads.pball_modes(shape, fc) for shape, fc in zip(shapes, fcs)]
    roll = BLMLBinnedRolling(modes, tol=1e-6, device='cuda')
    prev = [None] * len(seqs)
    for t in range(3):
        res = roll.update([seq[t] for seq in seqs])
        for i, seq in enumerate(seqs):
            m = BLMLBinned(tol=1e-6, solver='lbfgs', device='cuda').fit(seq[t], modes[i], complex_g=True,
                                                                         init=prev[i])
            prev[i] = m
            assert abs(res[i].loglik_ - m.loglik_) <= 1e-6 * abs(m.loglik_), (t, i, res[i].loglik_, m.loglik_)
    assert roll.n_updates_ == 3 and roll.history_[1]['warm']
