"""Run the CPU oracle's certified fit (rank growth of the float64 port of the reference's BLMLBinned until the
certificate is <= 1 + 1e-4; ranks below the last capped at 300 L-BFGS iterations, the last one run to tol) on every
fit of the 64-fit cut-off sweep and record, per fit, the rank path (K, loglik, certificate, L-BFGS iterations, capped),
the certified loglik and the CPU seconds. TEST / MEASUREMENT INFRASTRUCTURE: the
certified-fit bar of bench.py and the GPU tests compares the engine's certified logliks with these (the convex lift's
optimum is unique, so the certified loglik does not depend on the path).

    python oracle/make_sweep_certified.py [processes]      ->  oracle/sweep64_certified.json
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
    import blml_oracle as bo
    from blml_b200 import workloads
    sweep = workloads.cutoff_sweep(seed=0, n_fits=64)
    f = sweep[i]
    spec = workloads.pball_modes(f['shape'], f['fc'])[0]
    t0 = time.perf_counter()
    fit, path = bo.certified_fit(f['train'], spec, cert_tol=1e-4)
    rec = dict(i=i, shape=list(f['shape']), fc=f['fc'], rank=path[-1][0], loglik=path[-1][1],
               certificate=path[-1][2], path=[list(p) for p in path], seconds=time.perf_counter() - t0)
    with open(os.path.join(HERE, f'.certified_{i}.json'), 'w') as fh:       # partial results survive a crash
        json.dump(rec, fh)
    return rec


if __name__ == '__main__':
    procs = int(sys.argv[1]) if len(sys.argv) > 1 else os.cpu_count()
    cost = json.load(open(os.path.join(HERE, 'sweep64_counts.json')))
    order = sorted(range(64), key=lambda i: -cost[i]['seconds'])          # longest first
    with get_context('spawn').Pool(procs) as pool:
        out = sorted(pool.map(one, order, chunksize=1), key=lambda r: r['i'])
    json.dump(out, open(os.path.join(HERE, 'sweep64_certified.json'), 'w'), indent=1)
    for i in range(64):
        p = os.path.join(HERE, f'.certified_{i}.json')
        if os.path.exists(p):
            os.remove(p)
    print('total CPU seconds', sum(r['seconds'] for r in out))
