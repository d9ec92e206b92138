"""The oracle's certified fit (rank growth until the certificate is <= 1 + 1e-4) against the reference's own fits
(tests/golden/certified.npz, made by tests/golden/make_certified_golden.py): on three small fits of the benchmark
sweep, the reference's BLMLBinned started at the oracle's certified coefficients stays at the same loglik and its
own certificate() is <= 1 + 1e-4, so that loglik is the reference's optimum of the lift; the oracle's certified fit
(whatever rank its path ends at) reaches it to 1e-8."""
import numpy as np
import pytest

from conftest import golden


@pytest.mark.parametrize('i', [34, 48, 11])
def test_certified_fit_is_the_references_optimum(i):
    import blml_oracle as bo
    from blml_b200 import workloads
    g = golden('certified.npz')[f'f{i}']
    f = workloads.cutoff_sweep(0)[i]
    assert np.array_equal(f['train'], g['counts'])
    fit, path = bo.certified_fit(f['train'], workloads.pball_modes(f['shape'], f['fc'])[0], cert_tol=1e-4)
    assert float(g['certificate']) <= 1 + 1e-4 and path[-1][2] <= 1 + 1e-4
    # the rank the growth stops at depends on its path; the certified optimum of the convex lift does not
    assert abs(path[-1][1] - float(g['loglik'])) <= 1e-8 * abs(float(g['loglik'])), (path, float(g['loglik']))
