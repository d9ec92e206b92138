"""The fc gradients on the GPU (BLMLBinned.fc_grad / param_grad / implicit_grad through the C ABI: derivative plans
of the restricted transforms, csrc/solver_ops.cu's gradient kernels) at the reference's fitted coefficients against
the reference's own values (tests/golden/grads.npz): fixed-coefficient gradients to 1e-9 relative; the implicit
gradient to 1e-5 where the reference's conjugate gradients converged and 2e-3 where they stopped at 300 iterations
(there the value depends on the iteration's rounding path; the reference's own moves by ~1e-4 between caps). Also a
convex fit of the engine's own end to end."""
import types

import numpy as np
import pytest
import torch

from conftest import golden
from golden_cases import GRAD_SPECS

pytestmark = pytest.mark.gpu


def _close(a, b, rtol, atol=1e-12):
    a, b = np.asarray(a, float), np.asarray(b, float)
    assert np.array_equal(np.isnan(a), np.isnan(b))
    m = ~np.isnan(b)
    assert np.all(np.abs(a[m] - b[m]) <= rtol * np.abs(b[m]) + atol), (a, b)


def _at_reference(name, dtype=np.float64):
    from blml_b200.binned import BLMLBinned
    g = golden('grads.npz')[name]
    shape, modes, fkw, ckw = GRAD_SPECS[name]
    kw = {k: v for k, v in ckw.items() if k != 'max_sweeps'}
    m = BLMLBinned(dtype=dtype, max_sweeps=0, **kw).fit(
        g['counts'], modes, init=types.SimpleNamespace(e_hat_=g['e_hat'], shape_=tuple(shape)), **fkw)
    E = torch.as_tensor(np.asarray(g['e_hat'])).to(m.dev_, m.e_hat_t_.dtype).reshape(m.K_, -1).contiguous()
    m.e_hat_t_ = E                                       # the reference's coefficients exactly (no canonical step)
    m.Se_t_ = m._Sall(E)
    return g, m


@pytest.mark.parametrize('name', list(GRAD_SPECS))
def test_gradients_match_reference(cuda_device, name):
    g, m = _at_reference(name)
    eps = float(g['eps'])
    _close(np.array(m.fc_grad()), g['fc_grad'], 1e-9)
    _close(np.array(m.param_grad(g['val'], eps)), g['param_grad'], 1e-9)
    G = np.array(m.implicit_grad(g['val'], eps))
    converged = int(g['ift_iters']) < 300
    _close(G, g['implicit_grad'], 1e-5 if converged else 2e-3)
    if converged:
        assert abs(m.ift_iters_ - int(g['ift_iters'])) <= 1


def test_float32_gradients(cuda_device):
    """float32 state, float64 per-bin arithmetic and sums: fixed-coefficient gradients within 1e-3 relative (each is a
    difference of O(1) terms that leaves ~1e-2, so float32 rounding of U and dS E shows at ~1e-4 of it)."""
    g, m = _at_reference('g2_sinc_sinc_complex', np.float32)
    _close(np.array(m.fc_grad()), g['fc_grad'], 1e-3)
    _close(np.array(m.param_grad(g['val'], float(g['eps']))), g['param_grad'], 1e-3)


def test_own_convex_fit(cuda_device):
    """The real rank-1 sinc fit is convex: the engine's own fit (tol 1e-10) gives the reference's gradients (both
    fits stop at residual ~1e-10, which moves a gradient of ~2e-4 by ~1e-10)."""
    from blml_b200.binned import BLMLBinned
    g = golden('grads.npz')['g1_sinc_real']
    shape, modes, fkw, ckw = GRAD_SPECS['g1_sinc_real']
    m = BLMLBinned(dtype=np.float64, **ckw).fit(g['counts'], modes, **fkw)
    _close(np.array(m.fc_grad()), g['fc_grad'], 1e-4, atol=1e-9)
    _close(np.array(m.implicit_grad(g['val'], float(g['eps']))), g['implicit_grad'], 1e-4, atol=1e-9)


def test_counts_shape_checked(cuda_device):
    g, m = _at_reference('g1_sinc_real')
    with pytest.raises(ValueError):
        m.param_grad(np.ones(3))
