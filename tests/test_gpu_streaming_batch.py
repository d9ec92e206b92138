"""Many streams at once (BLMLBinnedStreamingBatch): each stream scores and joins its batches as the single-stream
class does (blml_binned.py:1034-1112, fc_update=None) and all streams' warm refits run in one BLMLBinnedBatch lockstep.
Against the same streams run one by one through BLMLBinnedStreaming: the prequential scores and the fits' logliks
agree within the batch-vs-single bar of the sweep tests (1e-6 relative)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _streams():
    from blml_b200 import workloads
    shapes, fcs = [(48, 48), (64, 48), (40, 40)], [0.3, 0.25, 0.35]
    out = []
    for s, (shape, fc) in enumerate(zip(shapes, fcs)):
        base = workloads.two_disk_field(shape, fc=fc, N=3e4, seed=200 + s)
        rng = np.random.default_rng(s)
        out.append([rng.poisson(base * 0.25).astype(float) + rng.poisson(0.1, base.shape) for _ in range(4)])
    return out, [workloads.pball_modes(shape, fc) for shape, fc in zip(shapes, fcs)]


def test_streams_in_one_batch_equal_streams_one_by_one(cuda_device):
    from blml_b200.streaming import BLMLBinnedStreaming, BLMLBinnedStreamingBatch
    streams, modes = _streams()
    kw = dict(tol=1e-6, decay=0.9, fc_update=None, solver='lbfgs', device='cuda')
    sb = BLMLBinnedStreamingBatch(len(streams), **kw)
    for t in range(4):
        sb.partial_fit([s[t] for s in streams], modes)
    assert sb.n_refits_ == 3
    for i, s in enumerate(streams):
        one = BLMLBinnedStreaming(**kw)
        for t in range(4):
            one.partial_fit(s[t], modes[i] if t == 0 else None, complex_g=True)
        got = sb.streams[i]
        assert len(got.preq_) == len(one.preq_) == 4            # the first batch has no fit to score it: NaN
        assert np.isnan(got.preq_[0]) and np.isnan(one.preq_[0])
        for a, b in zip(got.preq_[1:], one.preq_[1:]):
            assert abs(a - b) <= 1e-6 * abs(b), (i, got.preq_, one.preq_)
        assert abs(got.loglik_ - one.loglik_) <= 1e-6 * abs(one.loglik_), (i, got.loglik_, one.loglik_)
