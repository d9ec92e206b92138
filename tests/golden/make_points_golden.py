"""Generate tests/golden/points.npz by running the reference's own point fits (rahuljhu/band-limited-ml, BLMLQuick,
blml_trivial.py:2705-2800 with engine='cpu', float64; imported read-only from its checkout) on the cases of
tests/golden_cases.py POINT_SPECS. Per case: the points (and weights), the reference's bins Z_ in its order, counts
w_, steps, coefficients e_hat_, its predict and sqrt_density at query points.

    python tests/golden/make_points_golden.py <reference checkout>
"""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from _refpath import reference_checkout   # noqa: E402
REF = reference_checkout()
HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REF)
sys.path.insert(0, os.path.join(HERE, '..'))

from blml_trivial import BLMLQuick              # noqa: E402  (the reference)
from golden_cases import POINT_SPECS, point_cloud   # noqa: E402


def main():
    out = {}
    for name, (modes, n, weighted, seed) in POINT_SPECS.items():
        X = point_cloud(n, seed)
        sw = np.random.default_rng(seed + 100).integers(1, 4, n).astype(float) if weighted else None
        m = BLMLQuick(engine='cpu', dtype=np.float64, tol=1e-8).fit(X, modes, sample_weight=sw)
        Xq = np.random.default_rng(seed + 200).uniform(0.05, 0.95, (400, 2))
        out[f'{name}/X'] = X
        if sw is not None:
            out[f'{name}/sw'] = sw
        out[f'{name}/Z'] = m.Z_
        out[f'{name}/w'] = np.asarray(m.w_, float)
        out[f'{name}/h'] = np.asarray(m._h_vec, float)
        out[f'{name}/e_hat'] = np.asarray(m.e_hat_, float)
        out[f'{name}/n'] = np.array(m.n_samples_)
        out[f'{name}/Xq'] = Xq
        out[f'{name}/predict'] = m.predict(Xq)
        out[f'{name}/sqrt_density'] = np.asarray(m.sqrt_density(Xq), float)
        out[f'{name}/converged'] = np.array(m.converged_)
        print(name, 'bins', m.n_bins_, 'h', m._h_vec, 'sweeps', m.n_sweeps_, 'conv', m.converged_,
              'res', m.residual_, flush=True)
    np.savez_compressed(os.path.join(HERE, 'points.npz'), **out)


if __name__ == '__main__':
    main()
