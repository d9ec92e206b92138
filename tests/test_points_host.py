"""The points path of BLMLQuick on the host: lattice steps, quantized bin centres, the bins in the reference's order
(np.unique over raw bytes) and their weights reproduce the reference's own fits bit for bit
(tests/golden/points.npz, made by tests/golden/make_points_golden.py)."""
import numpy as np
import pytest

from conftest import golden
from golden_cases import POINT_SPECS, point_cloud
from blml_b200.quick import lattice_steps, quantize_points, unique_bins
from blml_b200.spec import parse_modes


@pytest.mark.parametrize('name', list(POINT_SPECS))
def test_bins_match_reference(name):
    g = golden('points.npz')[name]
    modes, n, weighted, seed = POINT_SPECS[name]
    X = point_cloud(n, seed)
    assert np.array_equal(X, g['X'])
    sw = g['sw'] if weighted else None
    nn = float(n if sw is None else sw.sum())
    sp = parse_modes(modes, 2)[0][0]
    h = lattice_steps(sp['kinds'], sp['periods'], 0.1 * nn ** -0.25 / np.asarray(sp['fc'], float))
    assert np.array_equal(h, g['h'])
    Z, w, inv = unique_bins(quantize_points(X, sp['kinds'], sp['periods'], h), sw)
    assert np.array_equal(Z, g['Z']) and np.array_equal(w, g['w'])
    assert np.array_equal(Z[inv], quantize_points(X, sp['kinds'], sp['periods'], h))


def test_steps_tile_periods():
    h = lattice_steps(['dirichlet', 'pball:1-2', 'pball:1-2'], [1.0, 2.0, 3.0], [0.3, 0.01, 0.02])
    assert h[0] == 1.0 / 8                                     # at least 8 bins per period
    assert h[1] == 2.0 / 200 and h[2] == 3.0 / 300            # a group's columns take its finest target
