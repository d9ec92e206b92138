"""Generate tests/golden/config2_256.npz: the reference's own fit (rahuljhu/band-limited-ml BLMLBinned, engine 'cpu',
float64, solver 'lbfgs', tol 1e-6; blml_binned.py:278-355, 383-445; imported read-only from its checkout) of the
256 x 256 complex two-mode pball workload: counts ~ Poisson(1e6 p) from two displaced disks (diameter 0.165,
shift +-0.0825 cycles/bin, inside the band) with a random relative phase and a 5% flat background
(blml_b200.workloads.two_disk_field, seed 0); modes: a pball of cut-off 0.33 and a background pball of cut-off 3 / 256,
both with the lattice as their period; complex_g. Stores the counts, e_hat_, density_, loglik_, the iterations, the
stop reason and the reference's fit time. About a minute on 8 cores.

    python tests/golden/make_config2_golden.py <reference checkout>
"""
import os
import sys
import time

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from _refpath import reference_checkout   # noqa: E402
REF = reference_checkout()
HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REF)
sys.path.insert(0, os.path.join(HERE, '..', '..', 'band-limited-ml_b200'))

from blml_binned import BLMLBinned              # noqa: E402  (the reference)
from blml_b200 import workloads                 # noqa: E402


def main():
    shape = (256, 256)
    counts = workloads.two_disk_field(shape, fc=0.33, N=1e6, seed=0)
    modes = workloads.pball_modes(shape, 0.33, bg_fc=3.0 / 256)
    t0 = time.perf_counter()
    m = BLMLBinned(engine='cpu', dtype=np.float64, solver='lbfgs', tol=1e-6).fit(counts, modes, complex_g=True)
    secs = time.perf_counter() - t0
    np.savez_compressed(os.path.join(HERE, 'config2_256.npz'), counts=counts, e_hat=m.e_hat_, density=m.density_,
                        loglik=np.array(m.loglik_), n_sweeps=np.array(m.n_sweeps_), stop=np.array(m.stop_reason_),
                        residual=np.array(m.residual_), seconds=np.array(secs), cores=np.array(os.cpu_count()))
    print(f'loglik {m.loglik_:.12f} iterations {m.n_sweeps_} stop {m.stop_reason_} residual {m.residual_:.2e} '
          f'{secs:.1f} s', flush=True)


if __name__ == '__main__':
    main()
