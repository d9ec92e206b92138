"""The CPU oracle against the reference's own outputs (tests/golden, made by tests/golden/make_golden.py): the pin
that makes the oracle a valid checker for the GPU path."""
import numpy as np
import pytest

from conftest import golden
import blml_oracle as bo
import pairs_oracle as po


def test_kernel_values():
    g = golden('kernels.npz')
    t, t2 = g['t'], g['t2']
    assert np.abs(bo.unit_value('sinc', [0.35], [None], [t]) - g['sinc']).max() < 1e-14
    assert np.abs(bo.unit_value('slits:0.4', [0.3], [None], [t]) - g['slits']).max() < 1e-14
    assert np.abs(bo.unit_value('dirichlet', [0.3], [32.0], [t]) - g['dirichlet']).max() < 1e-13
    assert np.abs(bo.unit_value('dirichlet:0.5', [0.3], [50.0], [t]) - g['dirichlet_fill']).max() < 1e-13
    assert np.abs(bo.unit_value('pball:0-1', [0.33, 0.33], [31.0, 31.0], [t2[0], t2[1]]) - g['pball']).max() < 1e-12
    assert np.abs(bo.unit_value('pball:0-1', [0.2, 0.2], [24.0, 40.0], [t2[0], t2[1]]) - g['pball_rect']).max() < 1e-12
    assert np.abs(bo.unit_value('ball:0-1', [0.4, 0.4], [None, None], [t2[0], t2[1]]) - g['ball']).max() < 1e-13
    Kv, sc = bo.pball_harmonics(0.33, [256.0, 256.0])
    assert len(Kv) == int(g['pball256_nharm']) and sc == float(g['pball256_scale'])


MATVEC = ['d1_sinc40', 'd1_sinc1024', 'd1_slits64', 'd1_dir_circ32', 'd1_dir_long32', 'd2_pball64', 'd2_pball_rect',
          'd2_pball_linear', 'd2_sinc_dir', 'd2_ball', 'd2_ball_h', 'd3_sinc']


@pytest.mark.parametrize('name', MATVEC)
def test_matvec(name):
    from golden_cases import MATVEC_SPECS
    g = golden('matvec.npz')[name]
    shape, modes, h = MATVEC_SPECS[name]
    specs = bo.parse_modes(modes, len(shape))
    op = bo.Operator(specs, shape, np.full(len(shape), h))
    assert tuple(op.pad) == tuple(g['pad'])
    np.testing.assert_allclose(op.s, g['s'], rtol=1e-14)
    U = op.Sall(g['E'])
    scale = np.abs(g['U']).max()
    assert np.abs(U - g['U']).max() <= 1e-13 * scale


@pytest.mark.parametrize('name', ['real1', 'psd_eq', 'psd_sec'])
def test_updates(name):
    from golden_cases import UPDATE_MODES
    g = golden('updates.npz')[name]
    w = g['w']; shape = w.shape
    f = bo.BinnedFit()
    f.d = len(shape); f.shape = shape
    f.specs = bo.parse_modes(UPDATE_MODES[name], f.d)
    f.op = bo.Operator(f.specs, shape, np.ones(f.d)); f.s = f.op.s; f.K = len(f.specs)
    f.w = w; f.n = float(w.sum()); f.c = f.n * w; f.occ = w > 0
    f.complex_g = name != 'real1'; f.psd = f.complex_g or f.K > 1; f.sg = np.ones(shape)
    E, U = g['E'], g['U']
    np.testing.assert_allclose(f.update(E, U), g['update'], rtol=1e-12, atol=1e-12)
    assert abs(f.merit(E, U) - float(g['merit'])) <= 1e-12 * abs(float(g['merit']))
    assert abs(f.resid(E, U) - float(g['resid'])) <= 1e-12
    np.testing.assert_allclose(f.rescale(E, U)[0], g['rescaled_E'], rtol=1e-13)
    if f.psd:
        L, gr = f.lgrad(E, U)
        assert abs(L - float(g['lgrad_L'])) <= 1e-12 * abs(L)
        np.testing.assert_allclose(gr, g['lgrad_g'], rtol=1e-11, atol=1e-12 * np.abs(gr).max())


def test_secular_and_cd_root():
    g = golden('updates.npz')
    lam = bo.secular(g['secular']['R2'], g['secular']['s'], g['secular']['c'])
    np.testing.assert_allclose(lam, g['secular']['lam'], rtol=1e-14)
    t = bo.cd_root(g['cd_root']['b'], g['cd_root']['c'], 0.35)
    np.testing.assert_allclose(t, g['cd_root']['t'], rtol=1e-15)


FAST_FITS = ['d1_sinc_real', 'd1_sinc_rank2_real', 'd1_dir_circ_real', 'd2_sinc_sinc_real', 'd2_ball_real',
             'd2_pball_lbfgs', 'd2_pball_bg_lbfgs', 'c1_sinc1024']


@pytest.mark.parametrize('name', FAST_FITS)
def test_fit(name):
    """The oracle's fit retraces the reference's: loglik to 1e-9 relative, density to 1e-6 relative L-inf."""
    from golden_cases import FIT_SPECS
    g = golden('fits.npz')[name]
    modes, fkw, ckw = FIT_SPECS[name]
    f = bo.BinnedFit(**ckw).fit(g['counts'], modes, **fkw)
    assert abs(f.loglik - float(g['loglik'])) <= 1e-9 * abs(float(g['loglik']))
    occ = g['counts'] > 0
    assert np.max(np.abs(f.density[occ] - g['density'][occ]) / g['density'][occ]) < 1e-6
    assert f.stop_reason == str(g['stop'])
    if 'cert' in g:
        assert abs(f.certificate() - float(g['cert'])) < 1e-5 * max(1.0, abs(float(g['cert'])))


def test_certificate_dense_matches_lanczos():
    """certificate() (ARPACK on the FFT operator) equals the dense eigvalsh of D^1/2 S D^1/2 / n, as the reference
    checks it (results/binned_checks.py:50-53)."""
    from golden_cases import FIT_SPECS
    g = golden('fits.npz')['d2_sinc_sinc_real']
    modes, fkw, ckw = FIT_SPECS['d2_sinc_sinc_real']
    f = bo.BinnedFit(**ckw).fit(g['counts'], modes, **fkw)
    assert abs(f.certificate(tol=1e-10) - f.certificate_dense()) < 1e-8


def test_pairs_rows_cols():
    g = golden('pairs.npz')
    p = g['p5']
    Zi = po.bin_points(p['X'], p['h'])
    assert np.array_equal(Zi, p['Zi'])                           # bit-exact binning
    u, cnt = po.unique_bins(Zi)
    assert np.array_equal(u, p['bins']) and np.array_equal(cnt, p['counts'])
    kinds, per = ['sinc'] * 5, [None] * 5
    tab = po.build_tables(kinds, p['fc'], per, p['h'], u)
    s = po.rows(tab, u, u, cnt)
    np.testing.assert_allclose(s, p['rows'], rtol=1e-12, atol=1e-12 * np.abs(s).max())
    np.testing.assert_allclose(po.pair_values(tab, u[:300], u[:200]), p['cols'], rtol=1e-12, atol=1e-15)
    np.testing.assert_allclose(po.gram(u[:300], u[:200], kinds, p['fc'], per, p['h']), p['gram'], rtol=1e-12,
                               atol=1e-15)
    t = g['pt']
    kinds2, per2 = ['pball:0-1', 'pball:0-1', 'sinc'], [31.0, 31.0, None]
    fc2, h2 = np.array([0.33, 0.33, 0.2]), np.array([1.0, 1.0, 0.7])
    tab2 = po.build_tables(kinds2, fc2, per2, h2, np.r_[t['ZA'], t['ZB']])
    np.testing.assert_allclose(po.rows(tab2, t['ZA'], t['ZB'], t['w']), t['rows'], atol=1e-12)
    np.testing.assert_allclose(po.pair_values(tab2, t['ZA'], t['ZB']), t['cols'], atol=1e-12)
    np.testing.assert_allclose(po.gram(t['ZA'], t['ZB'], kinds2, fc2, per2, h2), t['gram'], atol=1e-12)
