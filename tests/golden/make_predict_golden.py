"""Generate tests/golden/predict.npz: the reference's own sqrt_density, predict and predict_grid(2)
(rahuljhu/band-limited-ml blml_binned.py:451-500; imported read-only from its checkout) of its fits of the fit cases
in tests/golden/fits.npz (counts and the fit settings of tests/golden_cases.py FIT_SPECS): per case the fitted
coefficients e_hat, 300 query points inside the lattice's span (default_rng(7)), the amplitudes, densities and the
refined grid; and two 3-D ball cases on seeded counts of their own (EXTRA: a ball over all three columns -- a
half-integer Bessel order -- and a 2-D ball group times a sinc column).

    python tests/golden/make_predict_golden.py <reference checkout>
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
sys.path.insert(0, os.path.join(HERE, '..', '..', 'band-limited-ml_b200'))

from blml_binned import BLMLBinned              # noqa: E402  (the reference)
from golden_cases import FIT_SPECS, PREDICT_EXTRA, extra_counts     # noqa: E402

CASES = ('d1_sinc_real', 'd1_sinc_complex', 'd1_sinc_rank2_permode', 'd1_dir_circ_real', 'd2_sinc_sinc_real',
         'd2_pball_lbfgs', 'd2_pball_bg_lbfgs', 'd2_ball_real') + tuple(PREDICT_EXTRA)


def main():
    fits = np.load(os.path.join(HERE, 'fits.npz'))
    out = {}
    rng = np.random.default_rng(7)
    for name in CASES:
        if name in PREDICT_EXTRA:
            _, modes, fkw, ckw = PREDICT_EXTRA[name]
            counts = extra_counts(name)
        else:
            modes, fkw, ckw = FIT_SPECS[name]
            counts = fits[f'{name}/counts']
        m = BLMLBinned(engine='cpu', dtype=np.float64, **ckw).fit(counts, modes, **fkw)
        X = np.stack([rng.uniform(0.0, s - 1.0, 300) for s in counts.shape], 1)
        out[f'{name}/counts'] = counts
        out[f'{name}/e_hat'] = m.e_hat_
        out[f'{name}/X'] = X
        out[f'{name}/sqrt_density'] = m.sqrt_density(X)
        out[f'{name}/predict'] = m.predict(X)
        out[f'{name}/grid2'] = m.predict_grid(2)
        print(name, out[f'{name}/grid2'].shape, flush=True)
    np.savez_compressed(os.path.join(HERE, 'predict.npz'), **out)


if __name__ == '__main__':
    main()
