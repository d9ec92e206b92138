"""The block coordinate descent restated in the oracle (oracle/quick_oracle.py, the solver BLMLQuick runs on the GPU)
against the reference's own point fits (tests/golden/points.npz): on the reference's bins it converges to max|rho| <
1e-8 in a few tens of sweeps and reaches the reference's coefficients within 1e-7 of their largest."""
import numpy as np
import pytest

from conftest import golden
from golden_cases import POINT_SPECS
import quick_oracle as qo


@pytest.mark.parametrize('name', list(POINT_SPECS))
def test_block_cd_reaches_reference(name):
    g = golden('points.npz')[name]
    G = qo.gram(g['Z'], g['h'], POINT_SPECS[name][0])
    e, sweeps, conv, res = qo.block_cd(G, g['w'], tol=1e-8)
    assert conv and res < 1e-8 and sweeps < 60
    ref = np.ravel(g['e_hat'])
    assert np.max(np.abs(e - ref)) <= 1e-7 * np.max(np.abs(ref))
