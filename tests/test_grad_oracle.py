"""The gradient oracle (oracle/grad_oracle.py) against the reference's own fc_grad / param_grad / implicit_grad at the
reference's fitted coefficients (tests/golden/grads.npz, made by tests/golden/make_grad_golden.py): the
fixed-coefficient gradients to 1e-12; the implicit gradient to 1e-6 where the reference's conjugate gradients
converged (tol 1e-6), and to 1e-3 where they stopped at their 300-iteration cap (the 2-D complex cases: there the
result depends on the iteration's rounding path, and the reference's own value moves by ~1e-4 between caps of 300,
1,000 and 3,000 iterations)."""
import types

import numpy as np
import pytest

from conftest import golden
from golden_cases import GRAD_SPECS
import blml_oracle as bo
import grad_oracle as go


def state(name):
    g = golden('grads.npz')[name]
    shape, modes, fkw, ckw = GRAD_SPECS[name]
    kw = {k: v for k, v in ckw.items() if k != 'max_sweeps'}
    f = bo.BinnedFit(max_sweeps=0, **kw).fit(g['counts'], modes,
                                             init=types.SimpleNamespace(e_hat=g['e_hat'], shape=tuple(shape)), **fkw)
    f.e_hat = np.asarray(g['e_hat']).astype(f.e_hat.dtype)          # the reference's coefficients exactly
    f.Se = f.Sall(f.e_hat)
    return g, f


def close(a, b, rtol, atol=1e-14):
    a, b = np.asarray(a, float), np.asarray(b, float)
    assert np.array_equal(np.isnan(a), np.isnan(b))
    m = ~np.isnan(b)
    assert np.all(np.abs(a[m] - b[m]) <= rtol * np.abs(b[m]) + atol), (a, b)


@pytest.mark.parametrize('name', list(GRAD_SPECS))
def test_gradients_match_reference(name):
    g, f = state(name)
    eps = float(g['eps'])
    close(np.array(go.fc_grad(f)), g['fc_grad'], 1e-12)
    close(np.array(go.param_grad(f, g['val'], eps)), g['param_grad'], 1e-12)
    G, iters, res = go.implicit_grad(f, g['val'], eps)
    converged = int(g['ift_iters']) < 300
    close(np.array(G), g['implicit_grad'], 1e-6 if converged else 1e-3)
    if converged:
        assert iters == int(g['ift_iters'])
