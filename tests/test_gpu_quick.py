"""The fixed-lattice pair path (5-D points -> occupied bins -> real rank-1 fit) on the GPU: binning and bin order
bit-exact with the reference; the fit at the reference BLMLQuick optimum (convex: unique), density within 1e-5
relative (float64) and loglik within 1e-7; at the full workload size (n = 2e5, B ~ 1.8e5 bins) the pair operator is
symmetric and linear (size-independent properties)."""
import numpy as np
import pytest
import torch

from conftest import golden

pytestmark = pytest.mark.gpu


def test_binning_bit_exact(cuda_device):
    from blml_b200.quick import lattice_coords, bin_points
    p = golden('pairs.npz')['p5']
    Zi = lattice_coords(p['X'], p['h']).cpu().numpy()
    assert np.array_equal(Zi, p['Zi'])
    u, cnt = bin_points(p['X'], p['h'])
    assert np.array_equal(u.cpu().numpy(), p['bins']) and np.array_equal(cnt.cpu().numpy(), p['counts'])


def test_round_half_to_even(cuda_device):
    from blml_b200.quick import lattice_coords
    Z = np.array([[0.5, 1.5, 2.5, -0.5, -1.5, 0.49999999999999994, 1e15 + 0.5]]).T
    got = lattice_coords(Z, [1.0]).cpu().numpy().ravel()
    assert np.array_equal(got, np.round(Z.ravel()).astype(np.int64))


@pytest.mark.parametrize('dt', ['f64', 'f32'])
def test_lattice_fit_matches_reference(cuda_device, dt):
    from blml_b200.quick import BLMLQuickLattice
    from blml_b200 import make_modes, with_lattice
    p = golden('pairs.npz')['p5']
    u, cnt, h = p['bins'], p['counts'], float(p['h'][0])
    modes = with_lattice(make_modes(p['fc'], ['sinc'] * 5), h)
    q = BLMLQuickLattice(tol=1e-7 if dt == 'f64' else 1e-5, dtype=np.float64 if dt == 'f64' else np.float32)
    q.fit(u * h, modes, sample_weight=cnt)
    f = q.density_
    ref = p['quick_f']
    if dt == 'f64':
        assert np.max(np.abs(f - ref) / ref) <= 1e-5
    else:
        assert np.max(np.abs(f - ref)) / ref.max() <= 1e-5
    assert abs(q.loglik_ - float(p['quick_ll'])) <= 1e-7 * abs(float(p['quick_ll']))


def test_full_size_pair_operator_properties(cuda_device):
    """n = 2e5 points of the 8-component 5-D mixture at step 1/64: <u, S w> = <w, S u> (symmetry) and
    S(a w + u) = a S w + S u (linearity), float64 tables, over all B^2 bin pairs."""
    from blml_b200 import workloads
    from blml_b200.quick import bin_points
    from blml_b200.local_gpu import ProductKernel, rows_dev
    X = workloads.points_5d_mixture(seed=0)
    u, cnt = bin_points(X, 1 / 64)
    B = u.shape[0]
    assert 1.7e5 < B < 2.0e5
    pk = ProductKernel(['sinc'] * 5)
    tab = pk.tables(np.full(5, 0.1 * 64), [None] * 5, np.full(5, 1 / 64), u.cpu().numpy())
    g = torch.Generator(device='cuda').manual_seed(0)
    w = torch.rand(B, dtype=torch.float64, device='cuda', generator=g)
    v = torch.rand(B, dtype=torch.float64, device='cuda', generator=g)
    Sw, _ = rows_dev(u, u, w, tab)
    Sv, _ = rows_dev(u, u, v, tab)
    a = (v @ Sw).item(); b = (w @ Sv).item()
    assert abs(a - b) <= 1e-10 * abs(a)
    Sc, _ = rows_dev(u, u, (2.5 * w + v).contiguous(), tab)
    assert (Sc - (2.5 * Sw + Sv)).abs().max().item() <= 1e-10 * Sc.abs().max().item()
