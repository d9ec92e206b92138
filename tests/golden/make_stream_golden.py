"""Generate tests/golden/stream.npz by running the reference's own streaming fits (rahuljhu/band-limited-ml,
blml_binned.py:648-1112: BLMLBinnedStreaming with its _KernelLearner; imported read-only from its checkout) on the cases
of tests/golden_cases.py STREAM_SPECS. Per case: the batches, preq_ (NaN for burn-in entries), the fc of every
history entry (entries x modes x columns), the number of parameter moves per entry and the final loglik_.

    python tests/golden/make_stream_golden.py <reference checkout>
"""
import contextlib
import io
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from _refpath import reference_checkout   # noqa: E402
REF = reference_checkout()
HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REF)
sys.path.insert(0, os.path.join(HERE, '..'))

from blml_binned import BLMLBinnedStreaming     # noqa: E402  (the reference)
from golden_cases import STREAM_SPECS, grad_density, hist   # noqa: E402


def main():
    out = {}
    for i, (name, (shape, modes, ckw, how, fkw, nb, per)) in enumerate(STREAM_SPECS.items()):
        rng = np.random.default_rng(500 + i)
        batches = np.array([hist(rng, shape, per, grad_density(shape)) for _ in range(nb)])
        m = BLMLBinnedStreaming(engine='cpu', dtype=np.float64, **ckw)
        with contextlib.redirect_stdout(io.StringIO()):
            if how == 'partial':
                for b in batches:
                    m.partial_fit(b, modes, **fkw)
            else:
                m.fit(list(batches), modes, epochs=how[1], **fkw)
        fcs = np.array([h['fc'] for h in m.history_ if 'fc' in h], float)
        out[f'{name}/batches'] = batches
        out[f'{name}/preq'] = np.array(m.preq_, float)
        out[f'{name}/fc_hist'] = fcs
        out[f'{name}/loglik'] = np.array(m.loglik_)
        out[f'{name}/moved'] = np.array([len(h.get('moved', [])) for h in m.history_ if 'fc' in h])
        print(name, 'preq', np.round(m.preq_, 5).tolist(), 'fc', fcs[:, 0, 0].round(5).tolist(),
              'll', m.loglik_, flush=True)
    np.savez_compressed(os.path.join(HERE, 'stream.npz'), **out)


if __name__ == '__main__':
    main()
