"""Generate tests/golden/rows_multi.npz: the reference's own fused rows of several densities (blml_local.rows_multi,
blml_local.py:282-286 -- FusedFit's joint and marginals in one pass; imported read-only from its checkout) on the two
cases of tests/golden/pairs.npz: the 5-D sinc bins (the joint and two marginals: units {0, 1} and {2, 3, 4}) and the
pball torus group with a sinc column (the joint, the group alone, the sinc column alone), seeded weights.

    python tests/golden/make_rows_multi_golden.py <reference checkout>
"""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from _refpath import reference_checkout   # noqa: E402
REF = reference_checkout()
HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REF)

from blml_kernels import ProductKernel          # noqa: E402  (the reference)
import blml_local                               # noqa: E402


def main():
    g = np.load(os.path.join(HERE, 'pairs.npz'))
    rng = np.random.default_rng(11)
    out = {}
    u = g['p5/bins']; fc = g['p5/fc']; h = g['p5/h']
    ZA, ZB = u[:400], u
    pk = ProductKernel(['sinc'] * 5, [None] * 5, fold=[True] * 5)
    tab = pk.tables(fc, [None] * 5, h, u)
    W = rng.standard_normal((len(ZB), 3))
    umask = np.array([[1, 1, 1, 1, 1], [1, 1, 0, 0, 0], [0, 0, 1, 1, 1]], np.int64)
    s, _ = blml_local.rows_multi(ZA, ZB, W, tab, umask)
    out.update({'p5/ZA': ZA, 'p5/ZB': ZB, 'p5/W': W, 'p5/umask': umask, 'p5/s': s})
    ZA, ZB = g['pt/ZA'], g['pt/ZB']
    P = 31.0
    kinds2, per2 = ['pball:0-1', 'pball:0-1', 'sinc'], [P, P, None]
    fc2, h2 = np.array([0.33, 0.33, 0.2]), np.array([1.0, 1.0, 0.7])
    pk2 = ProductKernel(kinds2, per2, fold=[True] * 3)
    tab2 = pk2.tables(fc2, per2, h2, np.r_[ZA, ZB])
    W2 = rng.standard_normal((len(ZB), 3))
    umask2 = np.array([[1, 1], [0, 1], [1, 0]], np.int64)        # units: the sinc column, then the pball group
    s2, _ = blml_local.rows_multi(ZA, ZB, W2, tab2, umask2)
    out.update({'pt/ZA': ZA, 'pt/ZB': ZB, 'pt/W': W2, 'pt/umask': umask2, 'pt/s': s2})
    np.savez_compressed(os.path.join(HERE, 'rows_multi.npz'), **out)
    print({k: v.shape for k, v in out.items()})


if __name__ == '__main__':
    main()
