"""The 5-D fixed-lattice fit at size (n = 2e5 points, B ~ 1.84e5 occupied bins, sinc columns at fc = 0.1 cycles per
bin) against the reference's own fit of the same bins (tests/golden/quick5d.npz, made by
tests/golden/make_quick5d_golden.py; blml_trivial.py:2860-3035). The objective is convex (real rank 1); both fits
stop at max|rho| < tol of the same optimum, so the GPU fit, run to a tighter tol, must land within the reference's
own stopping error: densities at the reference's 2,000 sampled bins within 2e-3 relative, the loglik within 1e-6
relative."""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


def test_quick5d_fit_matches_reference_at_size(cuda_device):
    from blml_b200 import workloads
    from blml_b200.quick import BLMLQuickLattice, bin_points
    from blml_b200.spec import make_modes, with_lattice
    g = golden('quick5d.npz')
    X = workloads.points_5d_mixture(seed=0)
    u, cnt = bin_points(X, 1 / 64, device='cuda')
    w = cnt.cpu().numpy()
    assert len(w) == int(g['bins']) and w.sum() == float(g['counts_sum']) and (w * w).sum() == float(g['counts_sq'])
    Zi = u.cpu().numpy()
    modes = with_lattice(make_modes(np.full(5, 0.1 * 64), ['sinc'] * 5), 1 / 64)
    m = BLMLQuickLattice(tol=1e-6, dtype=np.float64, device='cuda', solver='block').fit(Zi / 64.0, modes,
                                                                                         sample_weight=w)
    assert m.converged_
    ll = float(g['loglik'])
    assert abs(m.loglik_ - ll) <= 1e-6 * abs(ll), (m.loglik_, ll)
    row = {tuple(z): i for i, z in enumerate(map(tuple, Zi))}
    idx = np.array([row[tuple(z)] for z in map(tuple, g['sample_bins'])])
    f = np.asarray(m.density_)[idx]
    ref = g['sample_f']
    assert np.max(np.abs(f - ref) / ref) <= 2e-3, np.max(np.abs(f - ref) / ref)
