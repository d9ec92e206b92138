"""The model specs behind the golden fixtures (shared by tests/golden/make_golden.py and the tests). Modes are plain
dicts in the reference's modes format, built with the oracle's make_modes restatement."""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, '..', 'oracle'))
sys.path.insert(0, os.path.join(HERE, '..', 'band-limited-ml_b200'))
from blml_oracle import make_modes          # noqa: E402
from blml_b200.workloads import pball_modes  # noqa: E402

# name: (shape, modes, h); the E / U arrays and the complex flag are in matvec.npz
MATVEC_SPECS = {
    'd1_sinc40': ((40,), make_modes([0.35], ['sinc']), 1.0),
    'd1_sinc1024': ((1024,), make_modes([0.05], ['sinc']), 1.0),
    'd1_slits64': ((64,), make_modes([0.3], ['slits:0.4']), 1.0),
    'd1_dir_circ32': ((32,), make_modes([0.3], ['dirichlet'], periods=[32.0]), 1.0),
    'd1_dir_long32': ((32,), make_modes([0.3], ['dirichlet'], periods=[50.0]), 1.0),
    'd2_pball64': ((64, 64), pball_modes((64, 64), 0.33, 3 / 64), 1.0),
    'd2_pball_rect': ((48, 80), pball_modes((48, 80), 0.25), 1.0),
    'd2_pball_linear': ((24, 24), [{(0, 1): dict(kind='pball', fc=0.33, period=[31.0, 31.0])}], 1.0),
    'd2_sinc_dir': ((24, 24), make_modes([0.4, 0.3], ['sinc', 'dirichlet'], periods=[None, 24.0]), 1.0),
    'd2_ball': ((24, 24), make_modes([0.4, 0.4], ['ball', 'ball']), 1.0),
    'd2_ball_h': ((24, 24), make_modes([0.8, 0.8], ['ball', 'ball']), 0.5),
    'd3_sinc': ((10, 10, 10), make_modes([0.5] * 3, ['sinc'] * 3), 1.0),
}
MATVEC_COMPLEX = {'d1_slits64', 'd1_dir_circ32', 'd2_pball64', 'd2_pball_rect', 'd2_pball_linear', 'd2_sinc_dir',
                  'd2_ball_h'}

UPDATE_MODES = {
    'real1': pball_modes((16, 16), 0.4),
    'psd_eq': make_modes([0.4, 0.4], ['sinc', 'sinc'], rank=2),
    'psd_sec': pball_modes((16, 16), 0.4, 0.2),
}

# name: (modes, fit kwargs, constructor kwargs); counts are in fits.npz
FIT_SPECS = {
    'd1_sinc_real': (make_modes([0.35], ['sinc']), {}, dict(tol=1e-9)),
    'd1_sinc_complex': (make_modes([0.35], ['sinc']), dict(complex_g=True), dict(tol=1e-9)),
    'd1_sinc_rank2_real': (make_modes([0.35], ['sinc'], rank=2), {}, dict(tol=1e-8)),
    'd1_sinc_rank2_permode': (make_modes([[0.35], [0.12]], ['sinc']), dict(complex_g=True), dict(tol=1e-8)),
    'd1_dir_circ_real': (make_modes([0.3], ['dirichlet'], periods=[32.0]), {}, dict(tol=1e-9)),
    'd2_sinc_sinc_real': (make_modes([0.4, 0.3], ['sinc', 'sinc']), {}, dict(tol=1e-9)),
    'd2_ball_real': (make_modes([0.4, 0.4], ['ball', 'ball']), {}, dict(tol=1e-9)),
    'd2_pball_lbfgs': (pball_modes((32, 32), 0.33), dict(complex_g=True), dict(tol=1e-8, solver='lbfgs', max_sweeps=3000)),
    'd2_pball_bg_lbfgs': (pball_modes((32, 32), 0.33, 3 / 32), dict(complex_g=True),
                          dict(tol=1e-8, solver='lbfgs', max_sweeps=3000)),
    'd2_pball_cd': (pball_modes((32, 32), 0.33), dict(complex_g=True), dict(tol=1e-7, max_sweeps=3000)),
    'c1_sinc1024': (make_modes([0.05], ['sinc']), {}, dict(tol=1e-7)),
}

# point-prediction cases beyond FIT_SPECS (tests/golden/make_predict_golden.py): name -> (shape, modes, fit kwargs,
# constructor kwargs), counts from extra_counts
PREDICT_EXTRA = {
    'd3_ball3_real': ((10, 10, 8), make_modes([0.45, 0.45, 0.45], ['ball', 'ball', 'ball']), {}, dict(tol=1e-9)),
    'd3_ball2_sinc_complex': ((12, 12, 6), make_modes([0.4, 0.4, 0.3], ['ball', 'ball', 'sinc']), dict(complex_g=True),
                              dict(tol=1e-8, solver='lbfgs', max_sweeps=3000)),
}


def extra_counts(name):
    """Seeded counts of a PREDICT_EXTRA case: 4,000 draws from a two-bump density on its lattice."""
    shape = PREDICT_EXTRA[name][0]

    def f(*g):
        c1 = [0.35 * m for m in shape]; c2 = [0.7 * m for m in shape]
        r1 = sum((x - a) ** 2 for x, a in zip(g, c1)) / (0.2 * max(shape)) ** 2
        r2 = sum((x - a) ** 2 for x, a in zip(g, c2)) / (0.15 * max(shape)) ** 2
        return np.exp(-r1) + 0.6 * np.exp(-r2) + 0.02
    return hist(np.random.default_rng(sum(shape)), shape, 4000, f)


def hist(rng, shape, n, f):
    g = np.meshgrid(*[np.arange(m, dtype=float) for m in shape], indexing='ij')
    p = f(*g); p = p / p.sum()
    return rng.multinomial(n, p.ravel()).reshape(shape).astype(float)

# the fc gradients (blml_binned.py:520-628): name -> (shape, modes, fit kwargs, constructor kwargs); counts, the
# reference's fitted coefficients and its fc_grad / param_grad / implicit_grad values are in grads.npz
GRAD_SPECS = {
    'g1_sinc_real': ((40,), make_modes([0.35], ['sinc']), {}, dict(tol=1e-10)),
    'g1_slits_complex': ((64,), make_modes([0.3], ['slits:0.4']), dict(complex_g=True),
                         dict(tol=1e-9, solver='lbfgs', max_sweeps=5000)),
    'g2_sinc_sinc_complex': ((24, 24), make_modes([0.4, 0.3], ['sinc', 'sinc']), dict(complex_g=True),
                             dict(tol=1e-9, solver='lbfgs', max_sweeps=5000)),
    'g2_ball_complex': ((20, 20), make_modes([0.45, 0.45], ['ball', 'ball']), dict(complex_g=True),
                        dict(tol=1e-9, solver='lbfgs', max_sweeps=5000)),
    'g2_dir_sinc_rank2': ((24, 24), make_modes([[0.3, 0.4], [0.3, 0.15]], ['dirichlet', 'sinc'],
                                               periods=[24.0, None]), dict(complex_g=True),
                          dict(tol=1e-8, solver='lbfgs', max_sweeps=5000)),
}


def grad_density(shape):
    """A smooth positive test density on the lattice (two bumps and a floor)."""
    def f(*g):
        c = [0.3 * m for m in shape]; c2 = [0.65 * m for m in shape]
        r1 = sum((x - a) ** 2 for x, a in zip(g, c)) / (0.12 * max(shape)) ** 2
        r2 = sum((x - a) ** 2 for x, a in zip(g, c2)) / (0.08 * max(shape)) ** 2
        return np.exp(-0.5 * r1) + 0.6 * np.exp(-0.5 * r2) + 0.02
    return f

# streaming fits (blml_binned.py:648-1112): name -> (shape, modes, constructor kwargs, how: 'partial' (partial_fit per
# batch) or ('fit', epochs), fit kwargs, number of batches, counts per batch); the batches, the reference's preq_, fc
# trajectory and final loglik are in stream.npz
STREAM_SPECS = {
    'adam_real': ((64,), make_modes([0.12], ['sinc']), dict(tol=1e-9, lr=0.1, param_every=2), 'partial', {}, 8, 500),
    'adam_decay_capped': ((64,), make_modes([0.3], ['sinc']),
                          dict(tol=1e-9, lr=0.1, param_every=1, implicit_grad=False, decay=0.95, batch_sweeps=50),
                          'partial', {}, 8, 500),
    'hill_dirichlet': ((40,), make_modes([0.3], ['dirichlet'], periods=[40.0]),
                       dict(tol=1e-9, param_every=2, z_se=0.5), 'partial', {}, 8, 500),
    'epochs_loo': ((48,), make_modes([0.15], ['sinc']), dict(tol=1e-9, lr=0.1, param_every=2), ('fit', 2), {}, 6, 500),
    'burnin_select': ((64,), [{0: dict(kind='sinc')}], dict(tol=1e-9, burn_in=1500, fc_update=None), 'partial', {},
                      6, 500),
    'complex_adam': ((48,), make_modes([0.2], ['sinc']),
                     dict(tol=1e-8, solver='lbfgs', max_sweeps=3000, lr=0.1, param_every=2), 'partial',
                     dict(complex_g=True), 6, 500),
}

# the points path of BLMLQuick (blml_trivial.py:2705-2800): name -> (modes, n points, sample weights?, seed); the points,
# the reference's bins (Z_ in its order), counts, steps, coefficients and predictions are in points.npz
POINT_SPECS = {
    'sinc2': (make_modes([3.0, 2.0], ['sinc', 'sinc']), 3000, False, 1),
    'sinc_dirichlet': (make_modes([3.0, 4.0], ['sinc', 'dirichlet'], periods=[None, 1.0]), 3000, False, 2),
    'sinc2_weighted': (make_modes([2.5, 2.5], ['sinc', 'sinc']), 2000, True, 3),
}


def point_cloud(n, seed):
    """Two Gaussian blobs in the unit square (the second column wraps into [0, 1))."""
    rng = np.random.default_rng(seed)
    comp = rng.uniform(size=n) < 0.6
    X = np.where(comp[:, None], rng.normal([0.35, 0.4], 0.08, (n, 2)), rng.normal([0.7, 0.75], 0.05, (n, 2)))
    X[:, 1] = np.mod(X[:, 1], 1.0)
    return X
