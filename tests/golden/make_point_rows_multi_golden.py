"""Generate tests/golden/point_rows_multi.npz: the reference's own point sums of several densities
(blml_local.point_rows_multi, blml_local.py:555-560 -- FusedFit's joint and marginals at points; imported read-only
from its checkout) on two seeded cases: sinc x sinc x dirichlet columns (the joint, the two sinc columns, the
dirichlet column) and a 2-D ball group times a sinc column (the joint, the ball alone, the sinc alone). The
reference evaluates radial profiles from a table by linear interpolation; the others exactly.

    python tests/golden/make_point_rows_multi_golden.py <reference checkout>
"""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from _refpath import reference_checkout   # noqa: E402
REF = reference_checkout()
HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REF)

import blml_local                               # noqa: E402  (the reference)

CASES = {
    'ss': (['sinc', 'sinc', 'dirichlet'], [0.4, 0.3, 0.25], [None, None, 24.0],
           [[1, 1, 1], [1, 1, 0], [0, 0, 1]]),
    'bs': (['ball', 'ball', 'sinc'], [0.4, 0.4, 0.3], [None, None, None],
           [[1, 1], [0, 1], [1, 0]]),                    # units: the sinc column, then the ball group
}


def main():
    rng = np.random.default_rng(5)
    out = {}
    for name, (kinds, fc, per, umask) in CASES.items():
        A = rng.uniform(0.0, 20.0, (50, 3))
        Bp = rng.uniform(0.0, 20.0, (300, 3))
        W = rng.standard_normal((300, 3))
        s, _ = blml_local.point_rows_multi(A, Bp, W, kinds, np.asarray(fc, float), per, np.asarray(umask, np.int64))
        out.update({f'{name}/A': A, f'{name}/Bp': Bp, f'{name}/W': W, f'{name}/s': s,
                    f'{name}/umask': np.asarray(umask, np.int64)})
    np.savez_compressed(os.path.join(HERE, 'point_rows_multi.npz'), **out)
    print({k: v.shape for k, v in out.items()})


if __name__ == '__main__':
    main()
