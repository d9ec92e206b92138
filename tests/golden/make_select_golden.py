"""Generate tests/golden/select.json by running the reference's own selector entry points (rahuljhu/band-limited-ml
selector.py: select_counts :716-732 with its _select_counts_flat / _search; imported read-only from its checkout) with
the deterministic stand-in estimator of tests/selector_cases.py (StubQuick) in place of BLMLQuick, on COUNTS_CASES.
Per case: every fit's fc in order, the selected fc and the best score.

    python tests/golden/make_select_golden.py <reference checkout>
"""
import contextlib
import io
import json
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from _refpath import reference_checkout   # noqa: E402
REF = reference_checkout()
HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REF)
sys.path.insert(0, os.path.join(HERE, '..'))

import selector as sel                          # noqa: E402  (the reference)
from blml_trivial import modes_fc               # noqa: E402
from selector_cases import StubQuick, COUNTS_CASES, counts_lattice          # noqa: E402

sel._estimator_class = lambda engine: StubQuick
sel.BLMLQuick = StubQuick


def main():
    out = {}
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
