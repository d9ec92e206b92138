"""Generate tests/golden/stream_helpers.json from the reference's own streaming helpers (rahuljhu/band-limited-ml,
blml_maps.py:19-36 adam_step on a 'scale' parameter with dlog gradients, blml_binned.py:1022-1031 _batch_order;
imported read-only from its checkout): Adam trajectories of log fc for seeded gradient sequences of three magnitudes,
and batch orders with and without groups.

    python tests/golden/make_stream_helpers_golden.py <reference checkout>
"""
import json
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from _refpath import reference_checkout   # noqa: E402
REF = reference_checkout()
HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REF)

from blml_maps import adam_step                 # noqa: E402  (the reference)
from blml_binned import _batch_order            # noqa: E402


def main():
    out = {'adam': [], 'order': []}
    rng = np.random.default_rng(0)
    for case in range(6):
        v0 = float(rng.uniform(0.05, 0.4))
        grads = rng.normal(0, [1e-3, 1e-1, 1.0][case % 3], 8).tolist()
        st, v, traj = [0.0, 0.0, 0], v0, []
        for g in grads:
            v = float(adam_step(v, g, st, 'scale', 0.1, (0.9, 0.999), dlog=True))
            traj.append(v)
        out['adam'].append(dict(v0=v0, grads=grads, traj=traj))
    for nb, groups, seed in ((7, None, 0), (9, [0, 1, 1, 2, 0, 3, 3, 3, 1], 4), (5, ['a', 'b', 'a', 'c', 'b'], 9)):
        out['order'].append(dict(nb=nb, groups=groups, seed=seed,
                                 order=[int(i) for i in _batch_order(nb, groups, np.random.default_rng(seed))]))
    with open(os.path.join(HERE, 'stream_helpers.json'), 'w') as fh:
        json.dump(out, fh, indent=0)


if __name__ == '__main__':
    main()
