"""The headline's certification rule (bench.certified_mask): the certificate bar, the two-sided loglik bar where the
oracle certified its fit, and the one-sided bar where the oracle's rank growth stopped uncertified."""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), '..'))


def test_certified_mask():
    import bench
    ref = np.array([[-5.0, 1.00005],      # oracle certified: two-sided
                    [-5.0, 1.00005],
                    [-5.0, 1.00005],
                    [-5.0, 1.002],        # oracle uncertified at its last rank: one-sided
                    [-5.0, 1.002],
                    [-5.0, 1.00005]])
    ll = np.array([-5.0 - 4e-6, -5.0 + 1e-5, -5.0 - 1e-5, -5.0 + 1e-5, -5.0 - 1e-5, -5.0])
    cert = np.array([1.0005, 1.0005, 1.0005, 1.0005, 1.0005, 1.0011])
    ok, rel = bench.certified_mask(ll, cert, ref)
    assert ok.tolist() == [True, False, False, True, False, False]
    assert np.allclose(rel, (ll + 5.0) / 5.0)


def test_reference_arm_certifies_its_cheapest_fit():
    """The reference arm's worker (the port's certified fit of one sweep fit, with the main arm's procedure settings)
    runs on the host: sweep fit 34, the one the port certifies fastest."""
    import bench
    ll, cert = bench._port_certified_fit(34)
    assert cert <= 1 + bench.CERT_TOL and ll < 0
