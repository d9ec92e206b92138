"""The multi-stream class's host checks (no GPU): fixed kernels only, L-BFGS streams only, one batch per stream."""
import pytest


def test_multi_stream_arguments():
    from blml_b200.streaming import BLMLBinnedStreamingBatch
    with pytest.raises(ValueError):
        BLMLBinnedStreamingBatch(2)                                   # fc_update defaults to 'adam'
    with pytest.raises(ValueError):
        BLMLBinnedStreamingBatch(2, fc_update=None, solver='cd')
    sb = BLMLBinnedStreamingBatch(3, fc_update=None, tol=1e-6)
    assert len(sb.streams) == 3 and all(s.fc_update is None and s.solver == 'lbfgs' for s in sb.streams)
    with pytest.raises(ValueError):
        sb.partial_fit([None, None])
