"""Run the CPU oracle (the float64 port of the reference's BLMLBinned) on every fit of the 64-fit cut-off sweep and
record, per fit, the start sweeps, L-BFGS iterations, stop reason, loglik and held-out score. TEST / MEASUREMENT
INFRASTRUCTURE: bench.py's reference arm reads the counts (its per-iteration costs are timed live on the host), and
the GPU tests compare the batched engine's logliks with these.

    python oracle/make_sweep_counts.py [processes]      ->  oracle/sweep64_counts.json
"""
import json
import os
import sys
import time
from multiprocessing import get_context

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.join(HERE, '..', 'band-limited-ml_b200'))


def one(i):
    os.environ.setdefault('OMP_NUM_THREADS', '1')
    import numpy as np
    import blml_oracle as bo
    from blml_b200 import workloads
    sweep = workloads.cutoff_sweep(seed=0, n_fits=64)
    f = sweep[i]
    modes = workloads.pball_modes(f['shape'], f['fc'])
    t0 = time.perf_counter()
    # the start alone (its sweep count), then the whole fit
    st = bo.BinnedFit(tol=1e-6, solver='cd').fit(f['train'], modes)
    fit = bo.BinnedFit(tol=1e-6, solver='lbfgs').fit(f['train'], modes, complex_g=True)
    F = np.abs(fit.Se[0]) ** 2
    val = f['val']
    score = float(np.sum(val[val > 0] * np.log(F[val > 0] / F.sum())) / val.sum())
    return dict(i=i, shape=list(f['shape']), fc=f['fc'], start_sweeps=int(st.n_sweeps), start_stop=st.stop_reason,
                lbfgs_its=int(fit.n_sweeps), stop=fit.stop_reason, loglik=float(fit.loglik), score=score,
                seconds=time.perf_counter() - t0)


if __name__ == '__main__':
    procs = int(sys.argv[1]) if len(sys.argv) > 1 else os.cpu_count()
    with get_context('spawn').Pool(procs) as pool:
        out = sorted(pool.map(one, range(64), chunksize=1), key=lambda r: r['i'])
    json.dump(out, open(os.path.join(HERE, 'sweep64_counts.json'), 'w'), indent=1)
    print('total CPU seconds', sum(r['seconds'] for r in out))
