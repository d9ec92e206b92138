"""Generate the golden fixtures of the binned path by running the reference implementation itself
(rahuljhu/band-limited-ml, imported read-only from its checkout) on seeded inputs.

    python tests/golden/make_golden.py <reference checkout>

Writes tests/golden/*.npz. The fixtures pin the CPU oracle (oracle/) and the GPU path's parity tests; the
reference is never needed at test time.
"""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from _refpath import reference_checkout   # noqa: E402
REF = reference_checkout()
HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REF)
sys.path.insert(0, os.path.join(HERE, '..', '..', 'band-limited-ml_b200'))

import blml_trivial as bt                       # noqa: E402  (the reference)
from blml_binned import BLMLBinned              # noqa: E402
from blml_kernels import ProductKernel, BinnedGram, rank_coords   # noqa: E402
import blml_local                               # noqa: E402
from blml_b200 import workloads                 # noqa: E402
sys.path.insert(0, os.path.join(HERE, '..'))
from golden_cases import MATVEC_SPECS, MATVEC_COMPLEX, UPDATE_MODES, FIT_SPECS, hist   # noqa: E402


def save(name, **arrs):
    np.savez_compressed(os.path.join(HERE, name), **arrs)
    print('wrote', name, sum(np.asarray(v).nbytes for v in arrs.values()), 'bytes raw')


def kernels():
    rng = np.random.default_rng(10)
    t = rng.uniform(-40, 40, 400); t2 = rng.uniform(-40, 40, (2, 400))
    out = {}
    out['t'] = t; out['t2'] = t2
    out['sinc'] = bt.kernel_class('sinc').eval(dict(fc=[0.35]), [t])
    out['slits'] = bt.kernel_class('slits:0.4').eval(dict(fc=[0.3]), [t])
    out['dirichlet'] = bt.kernel_class('dirichlet').eval(dict(fc=[0.3], period=32.0), [t])
    out['dirichlet_fill'] = bt.kernel_class('dirichlet:0.5').eval(dict(fc=[0.3], period=50.0), [t])
    out['pball'] = bt.kernel_class('pball').eval(dict(fc=[0.33, 0.33], period=np.array([31.0, 31.0])), [t2[0], t2[1]])
    out['pball_rect'] = bt.kernel_class('pball').eval(dict(fc=[0.2, 0.2], period=np.array([24.0, 40.0])), [t2[0], t2[1]])
    out['ball'] = bt.kernel_class('ball').eval(dict(fc=[0.4, 0.4]), [t2[0], t2[1]])
    Kv, sc = bt.pball_harmonics(0.33, [256.0, 256.0])
    out['pball256_nharm'] = np.array(len(Kv)); out['pball256_scale'] = np.array(sc)
    save('kernels.npz', **out)


def matvec():
    rng = np.random.default_rng(11)
    out = {}
    for name, (shape, modes, h) in MATVEC_SPECS.items():
        cplx = name in MATVEC_COMPLEX
        counts = np.ones(shape)
        m = BLMLBinned(engine='cpu', dtype=np.float64)
        m._setup(counts, modes, h, 0.0)
        K = len(m.specs_)
        E = rng.standard_normal((K,) + shape)
        if cplx:
            E = E + 1j * rng.standard_normal((K,) + shape)
        U = m._Sall(E)
        out[f'{name}/E'] = E; out[f'{name}/U'] = U
        out[f'{name}/s'] = m.s_; out[f'{name}/pad'] = np.array(m.pad_)
    save('matvec.npz', **out)


def updates():
    """_update / _merit / _resid / _rescale of the reference on random states."""
    rng = np.random.default_rng(12)
    out = {}
    shape = (16, 16)
    w = rng.poisson(3.0, shape).astype(float); w[0, :3] = 0
    for name, modes in UPDATE_MODES.items():
        cplx = name != 'real1'
        m = BLMLBinned(engine='cpu', dtype=np.float64)
        m._setup(w, modes, 1.0, 0.0)
        m.w_ = w; m.n_ = float(w.sum()); m.c_ = m.n_ * w; m.occ_ = w > 0
        m.complex_g_ = cplx; m.psd_ = cplx or m.K_ > 1; m.sg_ = np.ones(shape)
        E = np.abs(rng.standard_normal((m.K_,) + shape)) + 0.1
        if cplx:
            E = E * np.exp(1j * rng.uniform(0, 2 * np.pi, E.shape))
        E[:, ~m.occ_] = 0
        U = m._Sall(E)
        out[f'{name}/w'] = w; out[f'{name}/E'] = E; out[f'{name}/U'] = U; out[f'{name}/s'] = m.s_
        out[f'{name}/update'] = m._update(E, U)
        out[f'{name}/merit'] = np.array(m._merit(E, U))
        out[f'{name}/resid'] = np.array(m._resid(E, U))
        Er, Ur = m._rescale(E, U)
        out[f'{name}/rescaled_E'] = Er
        if m.psd_:
            L, g = m._lgrad(E, U)
            out[f'{name}/lgrad_L'] = np.array(L); out[f'{name}/lgrad_g'] = g
    # secular root on its own
    R2 = rng.uniform(0, 2, (3, 200)); s = np.array([0.5, 0.3, 0.1])[:, None]; c = rng.uniform(0.1, 50, 200)
    from blml_binned import _secular
    out['secular/R2'] = R2; out['secular/s'] = s; out['secular/c'] = c; out['secular/lam'] = _secular(np, R2, s, c)
    b = rng.standard_normal(300) * 5; cc = rng.uniform(0, 20, 300)
    out['cd_root/b'] = b; out['cd_root/c'] = cc; out['cd_root/t'] = bt.cd_root(b, cc, 0.35)
    save('updates.npz', **out)


def fit_counts():
    """The counts of each fit case, drawn in a fixed order from default_rng(1)."""
    rng = np.random.default_rng(1)
    c1 = lambda x: np.exp(-0.5 * ((x - 14) / 3) ** 2) + 0.5 * np.exp(-0.5 * ((x - 27) / 2) ** 2) + 0.02
    c2 = lambda x, y: np.exp(-0.5 * (((x - 11) / 2.5) ** 2 + ((y - 13) / 3) ** 2)) + \
        0.4 * np.exp(-0.5 * (((x - 17) / 2) ** 2 + ((y - 6) / 2) ** 2)) + 0.01
    cp = lambda x: np.exp(np.cos(2 * np.pi * x / 32)) + 0.3 * np.exp(-0.5 * ((x - 5) / 1.5) ** 2)
    return {'d1_sinc_real': hist(rng, (40,), 3000, c1), 'd1_sinc_complex': hist(rng, (40,), 3000, c1),
            'd1_sinc_rank2_real': hist(rng, (40,), 3000, c1), 'd1_sinc_rank2_permode': hist(rng, (40,), 3000, c1),
            'd1_dir_circ_real': hist(rng, (32,), 3000, cp), 'd2_sinc_sinc_real': hist(rng, (24, 24), 8000, c2),
            'd2_ball_real': hist(rng, (24, 24), 8000, c2), 'd2_pball_lbfgs': hist(rng, (32, 32), 20000, c2),
            'd2_pball_bg_lbfgs': hist(rng, (32, 32), 20000, c2), 'd2_pball_cd': hist(rng, (32, 32), 20000, c2),
            'c1_sinc1024': workloads.lattice_1d_mixture(0)}


def fits():
    out = {}
    counts_of = fit_counts()
    for name, (modes, fkw, ckw) in FIT_SPECS.items():
        counts = counts_of[name]
        m = BLMLBinned(engine='cpu', dtype=np.float64, **ckw).fit(counts, modes, **fkw)
        out[f'{name}/counts'] = counts
        out[f'{name}/density'] = m.density_
        out[f'{name}/e_hat'] = m.e_hat_
        out[f'{name}/loglik'] = np.array(m.loglik_)
        out[f'{name}/n_sweeps'] = np.array(m.n_sweeps_)
        out[f'{name}/residual'] = np.array(m.residual_)
        out[f'{name}/stop'] = np.array(m.stop_reason_)
        if m.shared_:
            out[f'{name}/cert'] = np.array(m.certificate())
        print(f'{name}: ll {m.loglik_:.10f} sweeps {m.n_sweeps_} stop {m.stop_reason_} res {m.residual_:.2e}', flush=True)
    save('fits.npz', **out)


def pairs():
    """Binning and pair sums on a 5-D mixture subsample (sinc columns) and on a pball x sinc lattice."""
    out = {}
    X = workloads.points_5d_mixture(seed=3, n=4000)
    h = 1.0 / 64
    kinds, per = ['sinc'] * 5, [None] * 5
    pk = ProductKernel(kinds, per, fold=[True] * 5)
    Zi = pk.coords(X, np.full(5, h))
    out['p5/X'] = X; out['p5/Zi'] = Zi
    u, inv, cnt = np.unique(Zi, axis=0, return_inverse=True, return_counts=True)
    out['p5/bins'] = u; out['p5/counts'] = cnt.astype(float)
    fcv = np.full(5, 0.1 / h)                       # 0.1 cycles per bin
    tab = pk.tables(fcv, per, np.full(5, h), u)
    w = cnt.astype(float)
    s, _ = blml_local.rows(u, u, w, tab)
    out['p5/rows'] = s
    sub = u[:300]
    out['p5/cols'] = blml_local.cols(sub, u[:200], tab)
    out['p5/gram'] = BinnedGram(pk, fcv, np.full(5, h)).gram_int(sub, u[:200])
    out['p5/fc'] = fcv; out['p5/h'] = np.full(5, h)
    # pball torus group with a sinc column (the reference's own mixed case, results/pball_parity.py:43-81)
    rng = np.random.default_rng(0)
    P, fc = 31.0, 0.33
    kinds2, per2 = ['pball:0-1', 'pball:0-1', 'sinc'], [P, P, None]
    fc2, h2 = np.array([fc, fc, 0.2]), np.array([1.0, 1.0, 0.7])
    pk2 = ProductKernel(kinds2, per2, fold=[True] * 3)
    ZA = np.c_[rng.integers(0, 31, 60), rng.integers(0, 31, 60), rng.integers(-20, 20, 60)]
    ZB = np.c_[rng.integers(0, 31, 80), rng.integers(0, 31, 80), rng.integers(-20, 20, 80)]
    want = [(1, ('shift', 0)), (1, ('shift', 1)), (0, 'fc')]
    tab2 = pk2.tables(fc2, per2, h2, np.r_[ZA, ZB], want=want)
    w2 = rng.normal(size=80)
    s2, ds2 = blml_local.rows(ZA, ZB, w2, tab2, grad=True)
    out['pt/ZA'] = ZA; out['pt/ZB'] = ZB; out['pt/w'] = w2; out['pt/rows'] = s2; out['pt/drows'] = ds2
    out['pt/cols'] = blml_local.cols(ZA, ZB, tab2)
    out['pt/gram'] = BinnedGram(pk2, fc2, h2).gram_int(ZA, ZB)
    # a BLMLQuick fixed-lattice fit on the 5-D bins (convex: unique optimum)
    Zc = u * h
    q = bt.BLMLQuick(dtype=np.float64, tol=1e-7)
    modes = bt.with_lattice(bt.make_modes(fcv, ['sinc'] * 5), h)
    q.fit(Zc, modes, sample_weight=w)
    out['p5/quick_e'] = np.asarray(q.e_hat_); out['p5/quick_f'] = q.predict(Zc)
    out['p5/quick_ll'] = np.array(float(np.sum(w * np.log(q.predict(Zc))) / w.sum()))
    print('quick fit: sweeps', q.n_sweeps_, 'conv', q.converged_)
    save('pairs.npz', **out)


if __name__ == '__main__':
    which = sys.argv[2:] or ['kernels', 'matvec', 'updates', 'fits', 'pairs']
    for w in which:
        globals()[w]()
