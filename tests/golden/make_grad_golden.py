"""Generate tests/golden/grads.npz by running the reference's own fit and fc gradients (rahuljhu/band-limited-ml,
blml_binned.py:520-628: fc_grad, param_grad, implicit_grad; imported read-only from its checkout) on the cases of
tests/golden_cases.py GRAD_SPECS. Per case: the training and validation counts, the reference's fitted coefficients
e_hat, fc_grad(), param_grad(val, eps), implicit_grad(val, eps) (K x units, NaN for integer units) and eps.

    python tests/golden/make_grad_golden.py <reference checkout>
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

from blml_binned import BLMLBinned              # noqa: E402  (the reference)
from golden_cases import GRAD_SPECS, grad_density, hist   # noqa: E402


def main():
    out = {}
    for i, (name, (shape, modes, fkw, ckw)) in enumerate(GRAD_SPECS.items()):
        rng = np.random.default_rng(300 + i)
        n = 3000 if len(shape) == 1 else 8000
        counts = hist(rng, shape, n, grad_density(shape))
        val = hist(rng, shape, n // 4, grad_density(shape))
        m = BLMLBinned(engine='cpu', dtype=np.float64, **ckw).fit(counts, modes, **fkw)
        dens = np.asarray(m.density_)
        eps = 0.05 * float(np.median(dens[val > 0]))
        stack = lambda G: np.array([np.asarray(g, float) for g in G])
        out[f'{name}/counts'] = counts
        out[f'{name}/val'] = val
        out[f'{name}/e_hat'] = np.asarray(m.e_hat_)
        out[f'{name}/loglik'] = np.array(m.loglik_)
        out[f'{name}/eps'] = np.array(eps)
        out[f'{name}/fc_grad'] = stack(m.fc_grad())
        out[f'{name}/param_grad'] = stack(m.param_grad(val, eps))
        out[f'{name}/implicit_grad'] = stack(m.implicit_grad(val, eps))
        out[f'{name}/ift_iters'] = np.array(m.ift_iters_)
        print(name, 'll', m.loglik_, 'stop', m.stop_reason_, 'res', f'{m.residual_:.1e}', 'fc_grad',
              out[f'{name}/fc_grad'].tolist(), 'implicit', out[f'{name}/implicit_grad'].tolist(), 'cg', m.ift_iters_,
              flush=True)
    np.savez_compressed(os.path.join(HERE, 'grads.npz'), **out)


if __name__ == '__main__':
    main()
