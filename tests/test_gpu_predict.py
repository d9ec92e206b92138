"""The binned fit at arbitrary points (BLMLBinned.sqrt_density / predict / predict_grid, blml_binned.py:451-500)
against the reference's own values at its own coefficients (tests/golden/predict.npz, made by
tests/golden/make_predict_golden.py): sinc, slits-free sinc rank 2 per mode, dirichlet, sinc x sinc, pball and pball
with a background pball, 2-D ball, 3-D ball (a half-integer Bessel order) and a 2-D ball group times a sinc column;
exact kernels for the interval and radial bands, the harmonic sums for the periodic ones (1e-10 of the largest
value)."""
import numpy as np
import pytest
import torch

from conftest import golden
from golden_cases import FIT_SPECS, PREDICT_EXTRA

pytestmark = pytest.mark.gpu

CASES = ('d1_sinc_real', 'd1_sinc_complex', 'd1_sinc_rank2_permode', 'd1_dir_circ_real', 'd2_sinc_sinc_real',
         'd2_pball_lbfgs', 'd2_pball_bg_lbfgs', 'd2_ball_real') + tuple(PREDICT_EXTRA)


@pytest.mark.parametrize('name', CASES)
def test_points_match_reference(cuda_device, name):
    from blml_b200.binned import BLMLBinned
    g = golden('predict.npz')[name]
    modes, fkw, ckw = PREDICT_EXTRA[name][1:] if name in PREDICT_EXTRA else FIT_SPECS[name]
    kw = dict(ckw); kw['max_sweeps'] = 0
    m = BLMLBinned(dtype=np.float64, device='cuda', **kw).fit(g['counts'], modes, **fkw)
    E = torch.as_tensor(g['e_hat']).reshape(g['e_hat'].shape[0], -1).to('cuda')
    m.e_hat_t_ = E if m.complex_g_ else E.real.contiguous() if E.is_complex() else E
    sd = m.sqrt_density(g['X'])
    ref = g['sqrt_density']
    assert sd.shape == ref.shape
    assert np.abs(sd - ref).max() <= 1e-10 * np.abs(ref).max(), np.abs(sd - ref).max()
    p = m.predict(g['X'])
    assert np.abs(p - g['predict']).max() <= 1e-10 * np.abs(g['predict']).max()
    gr = m.predict_grid(2)
    assert gr.shape == g['grid2'].shape
    assert np.abs(gr - g['grid2']).max() <= 1e-10 * np.abs(g['grid2']).max()
