"""Generate tests/golden/cols_dep.npz for the joint + marginal pass of the explicit Gram blocks (cols with depmask,
blml_local_gpu.py:320-361): the reference's CPU cols (blml_local.cols; imported read-only from its checkout) of the
product kernel over every column (the joint) and over the columns outside the dep mask only (the marginal; a radial
group counts as dep when one of its columns does), on the two cases of tests/golden/pairs.npz: the 5-D sinc bins and
the pball torus group with a sinc column.

    python tests/golden/make_cols_dep_golden.py <reference checkout>
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


def block(kinds, per, fc, h, ZA, ZB):
    pk = ProductKernel(kinds, per, fold=[True] * len(kinds))
    tab = pk.tables(np.asarray(fc, float), per, np.asarray(h, float), np.r_[ZA, ZB])
    return blml_local.cols(ZA, ZB, tab)


def main():
    g = np.load(os.path.join(HERE, 'pairs.npz'))
    out = {}
    u = g['p5/bins']; fc = g['p5/fc']; h = g['p5/h']
    ZA, ZB = u[:300], u[:200]
    kinds, per = ['sinc'] * 5, [None] * 5
    out['p5/joint'] = block(kinds, per, fc, h, ZA, ZB)
    for mask in (0b00101, 0b10000):
        keep = [k for k in range(5) if not (mask >> k) & 1]
        out[f'p5/marg{mask}'] = block([kinds[k] for k in keep], [per[k] for k in keep], fc[keep], h[keep],
                                      ZA[:, keep], ZB[:, keep])
    ZA, ZB = g['pt/ZA'], g['pt/ZB']
    P = 31.0
    kinds2, per2 = ['pball:0-1', 'pball:0-1', 'sinc'], [P, P, None]
    fc2, h2 = np.array([0.33, 0.33, 0.2]), np.array([1.0, 1.0, 0.7])
    out['pt/joint'] = block(kinds2, per2, fc2, h2, ZA, ZB)
    out['pt/marg4'] = block(kinds2[:2], per2[:2], fc2[:2], h2[:2], ZA[:, :2], ZB[:, :2])   # sinc column dep
    out['pt/marg1'] = block(kinds2[2:], per2[2:], fc2[2:], h2[2:], ZA[:, 2:], ZB[:, 2:])   # the group dep
    np.savez_compressed(os.path.join(HERE, 'cols_dep.npz'), **out)
    print({k: v.shape for k, v in out.items()})


if __name__ == '__main__':
    main()
