"""Generate tests/golden/select.json by running the reference's own selector entry points (rahuljhu/band-limited-ml
selector.py: select :617-666, select_counts :716-732 with their _select_* / _search; imported read-only from its
checkout) with the deterministic stand-in estimator of tests/selector_cases.py (StubQuick) in place of BLMLQuick, on
SELECT_CASES and COUNTS_CASES. Per case: every fit's fc in order, the selected fc and the best score.

    NUMBA_CACHE_DIR=/tmp/nb python tests/golden/make_select_golden.py /root/reference
"""
import contextlib
import io
import json
import os
import sys

import numpy as np

REF = sys.argv[1] if len(sys.argv) > 1 else '/root/reference'
HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REF)
sys.path.insert(0, os.path.join(HERE, '..'))
os.environ.setdefault('NUMBA_CACHE_DIR', '/tmp/nb')

import selector as sel                          # noqa: E402  (the reference)
from blml_trivial import modes_fc               # noqa: E402
from selector_cases import (StubQuick, SELECT_CASES, COUNTS_CASES, select_points,   # noqa: E402
                            counts_lattice)

sel._estimator_class = lambda engine: StubQuick
sel.BLMLQuick = StubQuick


def main():
    out = {}
    for name, (n, seed, modes, kw, with_val, weighted) in SELECT_CASES.items():
        X = select_points(n, seed)
        extra = {}
        if with_val:
            extra['X_val'] = select_points(n // 4, seed + 50)
        if weighted:
            r = np.random.default_rng(seed + 60)
            extra['sample_weight'] = r.integers(1, 4, n).astype(float)
            if with_val:
                extra['val_weight'] = r.integers(1, 4, n // 4).astype(float)
        StubQuick.calls = []
        with contextlib.redirect_stdout(io.StringIO()):
            m, best = sel.select(X, modes, **kw, **extra)
        out[name] = dict(calls=[c.tolist() for c in StubQuick.calls], fc=modes_fc(m).tolist(), best=float(best))
        print(name, len(StubQuick.calls), 'fits', np.round(modes_fc(m), 4).tolist(), best, flush=True)
    for name, (shape, seed, modes, kw) in COUNTS_CASES.items():
        Z, w_tr, w_va, h = counts_lattice(shape, seed)
        StubQuick.calls = []
        with contextlib.redirect_stdout(io.StringIO()):
            m, best = sel.select_counts(Z, w_tr, w_va, h, modes, **kw)
        out[name] = dict(calls=[c.tolist() for c in StubQuick.calls], fc=modes_fc(m).tolist(), best=float(best))
        print(name, len(StubQuick.calls), 'fits', np.round(modes_fc(m), 4).tolist(), best, flush=True)
    with open(os.path.join(HERE, 'select.json'), 'w') as fh:
        json.dump(out, fh, indent=0)


if __name__ == '__main__':
    main()
