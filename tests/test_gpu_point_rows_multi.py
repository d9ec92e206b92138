"""Point sums of several densities (blml_local.py:555-560, point_rows_multi: FusedFit's joint and marginals at
points) against the reference's own values (tests/golden/point_rows_multi.npz): sinc x sinc x dirichlet columns to
1e-12 of the largest sum; a 2-D ball group times a sinc column to 1e-5, the reference's radial profile being a
linearly interpolated table where this kernel evaluates the Bessel function; and the joint density equals the
single-density point kernel."""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu

CASES = {
    'ss': (['sinc', 'sinc', 'dirichlet'], [0.4, 0.3, 0.25], [None, None, 24.0], 1e-12),
    'bs': (['ball', 'ball', 'sinc'], [0.4, 0.4, 0.3], [None, None, None], 1e-5),
}


@pytest.mark.parametrize('case', sorted(CASES))
def test_point_rows_multi_matches_reference(cuda_device, case):
    from blml_b200.local_gpu import point_rows_multi
    g = golden('point_rows_multi.npz')[case]
    kinds, fc, per, tol = CASES[case]
    s, _ = point_rows_multi(g['A'], g['Bp'], g['W'], kinds, fc, per, g['umask'])
    ref = g['s']
    assert s.shape == ref.shape
    assert np.abs(s - ref).max() <= tol * np.abs(ref).max(), np.abs(s - ref).max() / np.abs(ref).max()
    joint, _ = point_rows_multi(g['A'], g['Bp'], g['W'][:, :1], kinds, fc, per, np.ones((1, g['umask'].shape[1])))
    assert np.abs(joint[:, 0] - s[:, 0]).max() <= 1e-13 * np.abs(s[:, 0]).max()
