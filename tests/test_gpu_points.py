"""The points path of BLMLQuick on the GPU against the reference's own point fits (tests/golden/points.npz): the same
bins in the same order, the coefficients of the convex real rank-1 fit (both solved to max|rho| < 1e-8) within 1e-6 of
their largest, predict / sqrt_density at off-lattice query points within 1e-6 of the largest value; the point kernel
alone (blml_point_rows at the reference's coefficients) to 1e-11; float32 fits within 1e-3."""
import numpy as np
import pytest
import torch

from conftest import golden
from golden_cases import POINT_SPECS

pytestmark = pytest.mark.gpu


def _fit(name, dtype=np.float64):
    from blml_b200.quick import BLMLQuick
    g = golden('points.npz')[name]
    modes, n, weighted, seed = POINT_SPECS[name]
    m = BLMLQuick(dtype=dtype, tol=1e-8).fit(g['X'], modes, sample_weight=g['sw'] if weighted else None)
    return g, m


def _rel(a, b):
    return float(np.max(np.abs(np.ravel(a) - np.ravel(b))) / np.max(np.abs(b)))


@pytest.mark.parametrize('name', list(POINT_SPECS))
def test_point_fit_matches_reference(cuda_device, name):
    g, m = _fit(name)
    assert np.array_equal(m.Z_, g['Z']) and np.array_equal(m.w_pts_, g['w']) and np.array_equal(m._h_vec, g['h'])
    assert m.n_samples_ == float(g['n'])
    assert _rel(m.e_hat_, g['e_hat']) <= 1e-6
    assert _rel(m.predict(g['Xq']), g['predict']) <= 1e-6
    assert _rel(m.sqrt_density(g['Xq']), g['sqrt_density']) <= 1e-6


@pytest.mark.parametrize('name', list(POINT_SPECS))
def test_point_kernel_exact(cuda_device, name):
    g, m = _fit(name)
    m.e_hat_t_ = torch.as_tensor(np.ravel(g['e_hat'])[None]).to(m.dev_, torch.float64)
    assert _rel(m.sqrt_density(g['Xq']), g['sqrt_density']) <= 1e-11


def test_point_fit_float32(cuda_device):
    g, m = _fit('sinc_dirichlet', np.float32)
    assert _rel(m.predict(g['Xq']), g['predict']) <= 1e-3


def test_point_errors(cuda_device):
    from blml_b200.quick import BLMLQuick
    g = golden('points.npz')['sinc2']
    modes = POINT_SPECS['sinc2'][0]
    with pytest.raises(NotImplementedError):
        BLMLQuick().fit(g['X'], modes, complex_g=True)
    with pytest.raises(ValueError):
        BLMLQuick().fit(g['X'], modes, sample_weight=-np.ones(len(g['X'])))
    m = BLMLQuick(dtype=np.float64, tol=1e-6).fit(g['X'], modes)
    with pytest.raises(ValueError):
        m.predict(np.zeros((3, 3)))
