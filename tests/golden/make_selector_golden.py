"""Generate tests/golden/selector_search.json by running the reference's own cut-off search
(rahuljhu/band-limited-ml selector.py:488-553 `_search`, imported read-only from its checkout) on the deterministic
objectives of tests/selector_cases.py, recording every candidate it scores, in order, and its result.

    python tests/golden/make_selector_golden.py <reference checkout>
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
from selector_cases import CASES                # noqa: E402


def main():
    out = {}
    for name, c in CASES.items():
        calls = []

        def obj(fc, f=c['obj']):
            calls.append([float(x) for x in fc])
            return f(fc)
        kw = dict(c['kw'])
        with contextlib.redirect_stdout(io.StringIO()):
            fc, best = sel._search(obj, c['d'], c['kinds'], c['periods_scaled'], **kw)
        out[name] = dict(calls=calls, fc=[float(x) for x in fc], best=float(best))
        print(name, len(calls), 'candidates', np.round(fc, 4), best)
    with open(os.path.join(HERE, 'selector_search.json'), 'w') as fh:
        json.dump(out, fh, indent=0)


if __name__ == '__main__':
    main()
