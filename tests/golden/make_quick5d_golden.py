"""Generate tests/golden/quick5d.npz: the reference's own fixed-lattice fit (rahuljhu/band-limited-ml BLMLQuick,
blml_trivial.py:2860-3035, numba on the host cores; imported read-only from its checkout) of the 5-D workload at
size: n = 2e5 points of the 8-component mixture (blml_b200.workloads.points_5d_mixture(seed=0)), bins at 1/64 by
the reference's own binning, sinc columns at fc = 0.1 cycles per bin, float64, tol 1e-4 (its default). The fit is
convex (real rank 1), so its optimum is unique. Stored: the bin count, the counts' checksum, the loglik, sweeps and
seconds, and the coefficients and densities at 2,000 sampled bins of the fit (their lattice coordinates with them).

    python tests/golden/make_quick5d_golden.py <reference checkout>      (about four hours on 8 cores: the fit 2.2 h)
"""
import os
import sys
import time

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from _refpath import reference_checkout   # noqa: E402
REF = reference_checkout()
HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REF)
sys.path.insert(0, os.path.join(HERE, '..', '..', 'band-limited-ml_b200'))

import blml_trivial as bt                      # noqa: E402  (the reference)
from blml_kernels import ProductKernel         # noqa: E402  (the reference)
from blml_b200 import workloads                # noqa: E402


def main():
    X = workloads.points_5d_mixture(seed=0)
    h = 1.0 / 64
    pk = ProductKernel(['sinc'] * 5, [None] * 5, fold=[True] * 5)
    Zi = pk.coords(X, np.full(5, h))
    u, cnt = np.unique(Zi, axis=0, return_counts=True)
    w = cnt.astype(float)
    Zc = u * h
    modes = bt.with_lattice(bt.make_modes(np.full(5, 0.1 / h), ['sinc'] * 5), h)
    t0 = time.perf_counter()
    q = bt.BLMLQuick(dtype=np.float64, tol=1e-4).fit(Zc, modes, sample_weight=w)
    secs = time.perf_counter() - t0
    f = np.asarray(q.predict(Zc))
    ll = float(np.sum(w * np.log(f)) / w.sum())
    Zq = np.asarray(q._Zi)                      # the fit's own bins, in its coefficient order
    idx = np.sort(np.random.default_rng(0).choice(len(Zq), 2000, replace=False))
    row = {tuple(z): i for i, z in enumerate(map(tuple, u))}
    fi = np.array([row[tuple(z)] for z in map(tuple, Zq[idx])])
    np.savez_compressed(os.path.join(HERE, 'quick5d.npz'), bins=np.array(len(u)), counts_sum=w.sum(),
                        counts_sq=(w * w).sum(), loglik=np.array(ll), n_sweeps=np.array(int(q.n_sweeps_)),
                        converged=np.array(bool(q.converged_)), seconds=np.array(secs), cores=np.array(os.cpu_count()),
                        sample_bins=Zq[idx], sample_e=np.asarray(q.e_hat_)[idx],
                        sample_f=f[fi])
    print('bins', len(u), 'loglik', ll, 'sweeps', q.n_sweeps_, 'converged', q.converged_, 'seconds', secs)


if __name__ == '__main__':
    main()
