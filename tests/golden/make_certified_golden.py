"""Generate tests/golden/certified.npz: certified fits of three small fits of the benchmark cut-off sweep pinned to the
reference itself (rahuljhu/band-limited-ml BLMLBinned, engine 'cpu', float64; imported read-only from its checkout).
For each fit the oracle's certified fit (oracle/blml_oracle.py certified_fit: rank growth until the certificate is
<= 1 + 1e-4) gives the rank K and its coefficients; the reference's own fit with K shared modes, started there
(init=, blml_binned.py:403-408) and run to tol 1e-6, gives the loglik and certificate() (blml_binned.py:501-518)
recorded here. A CPU test checks that the oracle's certified loglik is the reference's.

    python tests/golden/make_certified_golden.py <reference checkout>
"""
import os
import sys
from types import SimpleNamespace

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from _refpath import reference_checkout   # noqa: E402
REF = reference_checkout()
HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REF)
sys.path.insert(0, os.path.join(HERE, '..', '..', 'band-limited-ml_b200'))
sys.path.insert(0, os.path.join(HERE, '..', '..', 'oracle'))

from blml_binned import BLMLBinned              # noqa: E402  (the reference)
import blml_oracle as bo                        # noqa: E402
from blml_b200 import workloads                 # noqa: E402

FITS = (34, 48, 11)


def main():
    sweep = workloads.cutoff_sweep(0)
    out = {}
    for i in FITS:
        f = sweep[i]
        spec = workloads.pball_modes(f['shape'], f['fc'])[0]
        fit, path = bo.certified_fit(f['train'], spec, cert_tol=1e-4)
        K = path[-1][0]
        init = SimpleNamespace(e_hat_=fit.e_hat, shape_=f['train'].shape)
        m = BLMLBinned(engine='cpu', dtype=np.float64, solver='lbfgs', tol=1e-6).fit(f['train'], [spec] * K,
                                                                                    complex_g=True, init=init)
        cert = m.certificate()
        out[f'f{i}/counts'] = f['train']
        out[f'f{i}/rank'] = np.array(K)
        out[f'f{i}/loglik'] = np.array(m.loglik_)
        out[f'f{i}/certificate'] = np.array(cert)
        print(i, f['shape'], 'K', K, 'oracle', path[-1][1], 'reference', m.loglik_, 'cert', cert, flush=True)
    np.savez_compressed(os.path.join(HERE, 'certified.npz'), **out)


if __name__ == '__main__':
    main()
