"""Benchmark of the binned fitting path on B200 (one JSON line on rank 0).

Workload (N=1): the batched cut-off sweep -- 64 independent 2-D complex pball fits of uneven lattice size (sides from
{64, 96, 128, 192, 256, 384}) and cut-off (16-point log grid 0.05..0.45), counts ~ Poisson(N p) with N log-uniform
in 1e4..1e6 from a two-disk field with a 5% background, an 80/20 binomial held-out split. A step is the whole sweep
certified: every fit's complex L-BFGS fit (tol 1e-6, float64, the reference's seeded start), its certificate
lambda_max(D^1/2 S D^1/2) / n (blml_binned.py:501-518), and, while it exceeds 1 + 1e-3, one more shared mode started
along the certificate's top eigenvector and a refit (at most 8 modes), then the held-out scores. A fit is certified
when its certificate is <= 1 + 1e-3 and its loglik is within 1e-6 (relative, either side) of the FP64 oracle's
certified fit of the same counts (oracle/sweep64_certified.json): the convex lift has one optimum, so that loglik is
unique. Where the oracle's rank growth stops at 8 modes with its certificate above 1 + 1e-4, its loglik is only a lower
bound of the optimum, and the fit may not fall more than 1e-6 below it. value = certified fits/s with the counts in device memory; e2e = the same through the public API from host
counts (host->device copy of the counts, device->host read of every density and score inside each timed step).
plain_gpu = the same certification with one fit at a time (no batching, cold starts, every 4th fit); learned = the
learned warm start's rank-1 starts, then the same certification; same_sample_gpu = the reference arm's 8-fit sample
certified here in one batch (the same work as the reference arm's step).

Multi-GPU: the fits are independent (no exchange step): N ranks run N replicas of the sweep; value is all ranks'
certified fits over the slowest rank's time.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference] [--one-fit] [--matvec] [--pairs]
                    [--select] [--extras]
"""
import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, 'band-limited-ml_b200'))

N_FITS, TOL, CERT_TOL, MAX_RANK = 64, 1e-6, 1e-3, 8
METRIC = ('certified fits/s (certificate <= 1 + 1e-3 and |dloglik| <= 1e-6 rel of the FP64 oracle\'s certified fit; '
          'not below it where the oracle needs more than 8 modes), 64-fit 2-D pball cut-off sweep')
CONFIG = {'workload': '64-fit batched 2-D complex pball cut-off sweep: sides {64..384}^2, fc geomspace(0.05, 0.45, '
                      '16), N log-uniform 1e4..1e6, 80/20 held-out split, L-BFGS tol 1e-6, float64 state, '
                      'certified by rank growth',
          'fits': N_FITS, 'solver': 'lbfgs', 'state': 'float64',
          'certification': 'certificate lambda_max(D^1/2 S D^1/2)/n by batched float64 Lanczos; while > 1 + 1e-3 one '
                           'more shared mode along its top eigenvector and a refit, at most 8 modes; the rounds\' '
                           'L-BFGS stops when L / n gains < 1e-9 over 10 iterations; rounds below the last rank '
                           'capped at 150 iterations',
          'engine': 'batched lockstep, device-side control in CUDA-graph rings, grouped FFT mat-vecs; the certified '
                    'rounds keep their L-BFGS history (step and gradient-difference vectors) in complex64 storage',
          'l2': 'flushed between steps (256 MiB write)'}
REF_SAMPLE = 8                       # fits of the sweep in the reference arm's bounded sample (the cheapest on CPU)
LBFGS_M = 20                         # L-BFGS memory of the certified rounds (the certified optimum does not depend on it)
HISTORY_F32 = True                   # their L-BFGS history in complex64 storage (likewise path only)
PLAIN_SAMPLE = range(0, 64, 4)       # the fits the one-fit-at-a-time arm certifies
ROUND_LL_TOL = 1e-9                  # the certified rounds' L-BFGS stop on L / n gained over 10 iterations (plain fits: 1e-11)
GROW_ITERS, GROW_STEP = 150, 0.1     # L-BFGS cap of the rounds below the last rank; size of a new mode (x rms mode)
LANCZOS_BASIS = 32                   # the certificate's Lanczos basis before a restart
GROW_TWO_ABOVE = None                # a certificate above this level (and a second Ritz value above the bar): two modes


def workload(seed=0):
    from blml_b200 import workloads
    sweep = workloads.cutoff_sweep(seed=seed, n_fits=N_FITS)
    return sweep, [workloads.pball_modes(f['shape'], f['fc']) for f in sweep]


def peaks():
    try:
        return json.load(open(os.path.join(ROOT, 'MEASURED_PEAKS.json')))
    except Exception:
        return None


class Clocks:
    """nvidia-smi samples of SM clock and throttle reasons while the timed region runs."""
    Q = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,'
         'clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,'
         'clocks_event_reasons.sw_power_cap')

    def __init__(self, index):
        self.index = index; self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(['nvidia-smi', f'--id={self.index}', f'--query-gpu={self.Q}',
                                       '--format=csv,noheader,nounits', '-lms', '200'],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.p = None
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.p is not None:
            self.p.terminate()
            try:
                out, _ = self.p.communicate(timeout=5)
                self.lines = [l for l in out.splitlines() if l.strip()]
            except Exception:
                self.p.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        for l in getattr(self, 'lines', []):
            f = [x.strip() for x in l.split(',')]
            try:
                sm.append(float(f[1])); mx = float(f[2])
            except (ValueError, IndexError):
                continue
            for nm, v in zip(names, f[4:8]):
                if v.lower().startswith('active'):
                    reasons.add(nm)
        return {'sm_mhz': float(np.median(sm)) if sm else None, 'sm_max_mhz': mx, 'reasons': sorted(reasons),
                'samples': len(sm)}


def dist_init():
    import torch
    ws = int(os.environ.get('WORLD_SIZE', '1'))
    if ws > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group('nccl', timeout=timedelta(seconds=600))
        rank = dist.get_rank(); local = int(os.environ.get('LOCAL_RANK', rank))
        torch.cuda.set_device(local)
        return rank, ws, local
    return 0, 1, 0


def _red_device():
    """Where the process group reduces: the GPU under NCCL, the host under gloo (the CPU tests of the N > 1 path)."""
    import torch.distributed as dist
    return 'cuda' if dist.get_backend() == 'nccl' else 'cpu'


def barrier_sync(ws):
    import torch
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
    if torch.cuda.is_available():
        torch.cuda.synchronize()


def max_over_ranks(x, ws):
    import torch
    if ws == 1:
        return x
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=_red_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x, ws):
    import torch
    if ws == 1:
        return x
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=_red_device())
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def replica_value(certified, seconds, ws):
    """Whole-job certified fits/s of N replicas: every rank's certified fits over the slowest rank's time."""
    tmax = max_over_ranks(seconds, ws)
    return (sum_over_ranks(certified, ws) / tmax if tmax > 0 else 0.0), tmax


def grouped_matvec_roofline(batch, reps=20, route=0):
    """The dominant kernel chain of the sweep: one grouped mat-vec over all 64 fits (route 0: the group's own choice,
    the FFT route's 3 launches on these DFT-mask kernels; 1: the 4 restricted-transform stages), timed with CUDA
    events on the fits' stream; algorithmic bytes = read E + write U of every lattice (complex128)."""
    import torch
    from blml_b200.sweep import _Group
    st = torch.cuda.current_stream(batch.device)
    x = torch.randn(batch.Btot, dtype=torch.complex128, device=batch.device)
    y = torch.empty_like(x)
    off = batch.boff[:-1]
    grp = _Group(batch.p64, x, off, y, off, True)
    if route:
        grp.route = route
    for _ in range(3):
        grp(st.cuda_stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(reps):
        grp(st.cuda_stream)
    e1.record(st); torch.cuda.synchronize()
    t = e0.elapsed_time(e1) / 1e3 / reps
    nbytes = 2 * batch.Btot * 16
    flops = sum(p.flops_per_lattice for p in batch.p64)
    return t, nbytes, flops


def traffic_from_profiles():
    """Per-chain DRAM bytes of the grouped mat-vec from the committed ncu summary, if present."""
    try:
        return json.load(open(os.path.join(ROOT, 'profiles', 'grouped_matvec_sweep64_traffic.json'))).get(
            'dram_bytes_per_matvec')
    except Exception:
        return None


def scan_traffic(K, variant='c128'):
    """DRAM bytes of one history-scan launch at K modes per fit: the committed ncu capture (K = 1, the same 64 lattices)
    scaled by K -- the scan streams K-times-longer vectors, so its traffic grows in proportion. variant 'h32': the
    complex64-history scan."""
    try:
        t = json.load(open(os.path.join(ROOT, 'profiles', 'history_scan_sweep64_traffic.json')))
        b = t['dram_bytes_per_launch'] if variant == 'c128' else t['h32_dram_bytes_per_launch']
        return b * K / t['K']
    except Exception:
        return None


def _port_certified_fit(i):
    """Sweep fit i certified by the FP64 NumPy / SciPy port of the reference's algorithm (oracle/blml_oracle.py) on
    one host core: the same rank growth and certificate bar as the engine. Runs in a spawned worker."""
    os.environ['OMP_NUM_THREADS'] = '1'
    sys.path.insert(0, os.path.join(ROOT, 'oracle'))
    import blml_oracle as bo
    sweep, modes = workload(0)
    _, path = bo.certified_fit(sweep[i]['train'], modes[i][0], tol=TOL, cert_tol=CERT_TOL, max_rank=MAX_RANK,
                               ll_tol=ROUND_LL_TOL, grow_iters=GROW_ITERS, step=GROW_STEP)
    return path[-1][1], path[-1][2]


def port_sample():
    """The reference arm's bounded sample: the REF_SAMPLE sweep fits the port certifies fastest."""
    secs = [c['seconds'] for c in oracle_certified()]
    return sorted(range(N_FITS), key=lambda i: secs[i])[:REF_SAMPLE]


def port_step(pool, sample, ref):
    """One step of the CPU arm: every sample fit certified, one per worker process in parallel; returns (wall
    seconds, certified count) with the main arm's certification rule."""
    t0 = time.perf_counter()
    out = pool.map(_port_certified_fit, sample, chunksize=1)
    wall = time.perf_counter() - t0
    ll = np.array([o[0] for o in out]); cert = np.array([o[1] for o in out])
    return wall, int(certified_mask(ll, cert, ref[sample])[0].sum())


def port_pool():
    from multiprocessing import get_context
    procs = min(REF_SAMPLE, os.cpu_count() or 1)
    return get_context('spawn').Pool(procs), procs


def sample_desc(sample, procs):
    sw, _ = workload(0)
    shapes = [tuple(sw[i]['shape']) for i in sample]
    return (f'{len(sample)} whole sweep fits certified per step (the {len(sample)} the port certifies fastest, '
            f'lattices {shapes}), float64 NumPy/SciPy port of the reference\'s algorithm, one fit per process on '
            f'{procs} host cores; no extrapolation: a sample of the sweep\'s cheapest fits, so its fits/s exceeds '
            f'the whole sweep\'s')


def oracle_certified():
    """The FP64 oracle's certified fit of every sweep fit (oracle/make_sweep_certified.py): loglik, rank, seconds."""
    return json.load(open(os.path.join(ROOT, 'oracle', 'sweep64_certified.json')))


def oracle_ref():
    """(64, 2): the oracle's loglik and certificate per sweep fit."""
    return np.array([[c['loglik'], c['certificate']] for c in oracle_certified()])


ORACLE_CERT_TOL = 1e-4               # the oracle's own bar (oracle/make_sweep_certified.py)


def certified_mask(ll, cert, ref):
    """The certification rule: certificate <= 1 + CERT_TOL, and the loglik within 1e-6 (relative) of the oracle's
    where the oracle certified its fit within MAX_RANK modes (its loglik is then the lift's optimum); where it did
    not, its loglik is only a lower bound of the optimum and the fit may not fall more than 1e-6 below it."""
    ref, c_ref = ref[:, 0], ref[:, 1]
    rel = (np.asarray(ll) - ref) / np.abs(ref)
    pinned = c_ref <= 1.0 + ORACLE_CERT_TOL
    ok = (np.asarray(cert) <= 1.0 + CERT_TOL) & np.where(pinned, np.abs(rel) <= 1e-6, rel >= -1e-6)
    return ok, rel


def certify(res, ref):
    """(certified count, relative loglik differences, certificates) of fit_certified's results against the oracle's
    certified fits."""
    cert = np.array([r.certificate_ for r in res])
    ok, rel = certified_mask([r.loglik_ for r in res], cert, ref[:len(res)])
    return int(ok.sum()), rel, cert


def certified_sweep(dev, train, val, modes, init=None):
    """One step: the sweep's certified fits (rank growth) and their held-out scores."""
    from blml_b200.sweep import BLMLBinnedBatch, certified_log_density
    b = BLMLBinnedBatch(tol=TOL, dtype=np.float64, device=dev, lbfgs_m=LBFGS_M)
    res = b.fit_certified(train, modes, cert_tol=CERT_TOL, max_rank=MAX_RANK, init=init, history_f32=HISTORY_F32,
                          ll_tol=ROUND_LL_TOL, grow_iters=GROW_ITERS, step=GROW_STEP, lanczos_basis=LANCZOS_BASIS,
                          grow_two_above=GROW_TWO_ABOVE)
    return b, res, certified_log_density(res, val)


def learned_arm(dev, sweep, modes, train_dev, val_dev, ref, flush, ws, steps=2):
    """The learned warm start on the same sweep (the trained weights shipped with the package): network inference
    (one forward per lattice shape) for the rank-1 starts, then the same certification (rank growth, held-out
    scores), timed like the main arm. None when no weights ship."""
    import torch
    from blml_b200 import warmstart_job
    path = os.path.join(ROOT, 'band-limited-ml_b200', 'blml_b200', 'warmstart_weights.npz')
    if not os.path.exists(path):
        return None
    net = warmstart_job.load(path, device=dev)
    fcs = [f['fc'] for f in sweep]; kinds = ['pball'] * len(sweep)
    st = torch.cuda.current_stream(dev)
    certified_sweep(dev, train_dev, val_dev, modes, init=net.start(train_dev, fcs, kinds))      # warm-up
    tot = 0.0; cert = 0; rel = ranks = None
    for _ in range(steps):
        flush_l2(flush)
        barrier_sync(1)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        b, res, _ = certified_sweep(dev, train_dev, val_dev, modes, init=net.start(train_dev, fcs, kinds))
        e1.record(st); torch.cuda.synchronize()
        tot += e0.elapsed_time(e1) / 1e3
        c1, rel, _ = certify(res, ref)
        cert += c1; ranks = np.array([r.rank_ for r in res])
        its = np.array([r.rank_path_[0][3] for r in res])
    tmax = max_over_ranks(tot, ws)
    return {'value': sum_over_ranks(cert, ws) / tmax, 'unit': 'fits/s', 'ms_per_step': 1e3 * tmax / steps,
            'certified_per_step': cert / steps, 'rel_dloglik_max_abs': float(np.max(np.abs(rel))),
            'rank_mean': float(ranks.mean()), 'rank1_lbfgs_iterations_mean': float(its.mean()),
            'what': 'learned warm start (U-Net, tcgen05 BF16 kernels) for the rank-1 starts, then the same rank '
                    'growth and certificate as the main value'}


def pairs_bench(dev, reps=3):
    """The pair path at the 5-D workload (n = 2e5 points of an 8-component mixture binned at 1/64, B ~ 1.84e5
    occupied bins, sinc fc = 0.1 cycles per bin per column): one full rows pass s = S w over all B^2 bin pairs, float64
    and float32 tables (float64 sums), CUDA events; beside it the CPU oracle (NumPy, float64) on a bounded sample of
    rows against all B bins, scaled to pairs/s."""
    import torch
    from blml_b200 import workloads
    from blml_b200.quick import bin_points
    from blml_b200.local_gpu import ProductKernel, rows_dev
    X = workloads.points_5d_mixture(seed=0)
    u, cnt = bin_points(X, 1 / 64, device=dev)
    B = int(u.shape[0])
    tab = ProductKernel(['sinc'] * 5).tables(np.full(5, 0.1 * 64), [None] * 5, np.full(5, 1 / 64), u.cpu().numpy())
    w = cnt.to(dev)
    out = {'workload': '5-D pair rows: n = 2e5 points, 8-component mixture, bins at 1/64, sinc fc 0.1 / bin',
           'bins': B, 'pairs_per_pass': B * B}
    for name, f32 in (('f64_tables', False), ('f32_tables', True)):
        rows_dev(u, u, w, tab, f32=f32)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            rows_dev(u, u, w, tab, f32=f32)
        e1.record(); torch.cuda.synchronize()
        t = e0.elapsed_time(e1) / 1e3 / reps
        out[name] = {'seconds_per_pass': t, 'Gpair_per_s': B * B / t / 1e9}
    sys.path.insert(0, os.path.join(ROOT, 'oracle'))
    import pairs_oracle as po
    Z = u.cpu().numpy()
    otab = po.build_tables(['sinc'] * 5, np.full(5, 0.1 * 64), [None] * 5, np.full(5, 1 / 64), Z)
    R = 256
    t0 = time.perf_counter(); po.rows(otab, Z[:R], Z, cnt.cpu().numpy()); t = time.perf_counter() - t0
    out['cpu_oracle'] = {'Gpair_per_s': R * B / t / 1e9, 'sample': f'{R} rows x {B} bins in {t:.1f} s',
                         'cores': os.cpu_count(), 'kind': 'port'}
    return out


def segscan_bench(dev, K=4, m=20, reps=20):
    """The L-BFGS history kernels that dominate the certified sweep's GPU time, at its size: every sweep fit at K
    shared modes (complex128 vectors of sum K B elements), the history scan (blml_seg_dots2: m stored vectors against
    two shared ones) and the direction's linear combination (blml_seg_lincomb of 1 + 2 m vectors), and both with the
    certified rounds' complex64 history (blml_seg_dots2_h32, blml_seg_lincomb_h32). CUDA events; GB/s of the
    algorithmic bytes (each vector read once, the output written once)."""
    import ctypes as C
    import torch
    from blml_b200 import _lib
    from blml_b200._lib import call, ptrs
    from blml_b200.sweep import _Seg
    sweep, _ = workload(0)
    B = np.array([f['train'].size for f in sweep], np.int64)
    off = np.concatenate([[0], np.cumsum(K * B)]); boff = np.concatenate([[0], np.cumsum(B)])
    F = len(B)
    segs = (_Seg * F)(*[_Seg(int(off[f]), int(boff[f]), int(B[f]), K, 0) for f in range(F)])
    st_t = torch.frombuffer(bytearray(segs), dtype=torch.uint8).to(dev)
    n = int(off[-1])
    g = torch.Generator(device=dev).manual_seed(0)
    vecs = [torch.randn(n, dtype=torch.complex128, device=dev, generator=g) for _ in range(2 * m + 3)]
    part = torch.empty(max(48 * F * _lib.lib().blml_seg_blocks(), 43 * (_lib.SEG_SPLIT_BLOCKS + F)) + 64,
                       dtype=torch.float64, device=dev)
    out = torch.empty(48 * F + 64, dtype=torch.float64, device=dev)
    q = torch.empty_like(vecs[0])
    cf = torch.full((F, 1 + 2 * m), 0.5, dtype=torch.float64, device=dev)
    st = torch.cuda.current_stream(dev).cuda_stream
    vb = n * 16

    def dots2():
        call('blml_seg_dots2', _lib.F64, F, st_t.data_ptr(), 1, m, ptrs(vecs[:m]), vecs[2 * m].data_ptr(),
             vecs[2 * m + 1].data_ptr(), vecs[2 * m + 2].data_ptr(), part.data_ptr(), out.data_ptr(), st)

    def lincomb():
        call('blml_seg_lincomb', _lib.F64, F, st_t.data_ptr(), 1, q.data_ptr(), 1 + 2 * m, cf.data_ptr(),
             ptrs([vecs[2 * m]] + vecs[:2 * m]), st)
    hist32 = [v.to(torch.complex64) for v in vecs[:m + 1]]          # the certified rounds' complex64 history

    split = torch.empty(int(_lib.lib().blml_seg_split_ints(F)), dtype=torch.int32, device=dev)

    def dots2_h32():
        call('blml_seg_dots2_h32', F, st_t.data_ptr(), split.data_ptr(), m, ptrs(hist32[:m]), hist32[m].data_ptr(),
             vecs[2 * m + 1].data_ptr(), vecs[2 * m + 2].data_ptr(), part.data_ptr(), out.data_ptr(), st)
    hist32 += [v.to(torch.complex64) for v in vecs[m + 1:2 * m]]    # 2 m complex64 history vectors in all

    def lincomb_h32():                  # the certified rounds' direction: complex128 g and 2 m complex64 vectors
        call('blml_seg_lincomb_h32', F, st_t.data_ptr(), split.data_ptr(), q.data_ptr(), 0, 1 + 2 * m,
             cf.data_ptr(), ptrs([vecs[2 * m]] + hist32[:2 * m]), ((1 << (2 * m)) - 1) << 1, st)
    res = {'elements': n, 'vector_MB': vb / 1e6, 'K': K, 'm': m}
    for name, fn, nbytes in (('dots2', dots2, (m + 3) * vb), ('lincomb', lincomb, (2 * m + 2) * vb),
                             ('dots2_h32', dots2_h32, (m + 1) * vb // 2 + 2 * vb),
                             ('lincomb_h32', lincomb_h32, m * vb + 2 * vb)):
        for _ in range(3):
            fn()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record(); torch.cuda.synchronize()
        t = e0.elapsed_time(e1) / 1e3 / reps
        res[name] = {'us': t * 1e6, 'GB/s': nbytes / t / 1e9}
    return res


def tune_fft(dev, cta_kib=(24, 32, 48, 64, 72), max_cols=(1, 2, 4), reps=20):
    """The project's autotuner for the FFT route's launch shape: the grouped mat-vec over the 64 sweep lattices
    (complex float64, and real float64 as the start phase runs it) timed with CUDA events for every shared-memory
    budget per CTA and column-stage width; the fastest total is written to the package's fft_tuning.json, which the
    library applies at load. Returns every measurement."""
    import torch
    from blml_b200 import _lib
    from blml_b200.sweep import BLMLBinnedBatch, _Group
    import ctypes as C
    sweep, modes = workload(0)
    b = BLMLBinnedBatch(tol=TOL, dtype=np.float64, device=dev)
    b._prepare([f['train'] for f in sweep], modes)
    st = torch.cuda.current_stream(dev)
    off = b.boff[:-1]
    xc = torch.randn(b.Btot, dtype=torch.complex128, device=dev); yc = torch.empty_like(xc)
    xr = torch.randn(b.Btot, dtype=torch.float64, device=dev); yr = torch.empty_like(xr)
    L = _lib.lib()
    c0, m0 = C.c_int(), C.c_int()
    L.blml_fft_get_shape(C.byref(c0), C.byref(m0))
    rows = []
    try:
        for kib in cta_kib:
            for mc in max_cols:
                _lib.call('blml_fft_set_shape', kib * 1024, mc)
                t = {}
                for name, x, y, xcp in (('complex', xc, yc, True), ('real', xr, yr, False)):
                    g = _Group(b.p64, x, off, y, off, xcp)
                    for _ in range(3):
                        g(st.cuda_stream)
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record(st)
                    for _ in range(reps):
                        g(st.cuda_stream)
                    e1.record(st); torch.cuda.synchronize()
                    t[name] = e0.elapsed_time(e1) * 1e3 / reps
                    del g
                rows.append({'cta_bytes': kib * 1024, 'max_cols': mc, 'us_complex': t['complex'], 'us_real': t['real']})
    finally:
        L.blml_fft_set_shape(c0.value, m0.value)
    best = min(rows, key=lambda r: 2 * r['us_complex'] + r['us_real'])      # the L-BFGS runs two complex per real
    out = {'best': best, 'candidates': rows,
           'what': 'grouped FFT mat-vec over the 64 sweep lattices, float64, CUDA events, 20 launches each'}
    with open(os.path.join(ROOT, 'band-limited-ml_b200', 'blml_b200', 'fft_tuning.json'), 'w') as fh:
        json.dump({'cta_bytes': best['cta_bytes'], 'max_cols': best['max_cols'], 'measured': out}, fh, indent=1)
    return out


def config2_bench(dev, reps=50):
    """The 256 x 256 complex two-mode pball workload (pball 0.33 + background pball 3/256, L-BFGS tol 1e-6, float64,
    the reference's seeded start) through the public fit call, against the reference's own fit of the same counts
    (tests/golden/config2_256.npz holds its loglik, iterations and CPU seconds); and one mat-vec of each mode on every
    route: FFT float64, restricted transforms float64, tcgen05 split-TF32 float32 -- CUDA events, mat-vecs/s, GB/s of
    the algorithmic bytes (read E + write U, complex of the storage type) and the error against the FFT float64
    result."""
    import torch
    from blml_b200 import workloads, _lib
    from blml_b200.binned import BLMLBinned
    from blml_b200.operator import Plan, mode_transform, pad_rule
    from blml_b200.spec import parse_modes
    shape = (256, 256)
    counts = workloads.two_disk_field(shape, fc=0.33, N=1e6, seed=0)
    modes = workloads.pball_modes(shape, 0.33, bg_fc=3.0 / 256)
    g = np.load(os.path.join(ROOT, 'tests', 'golden', 'config2_256.npz'))
    out = {'workload': '256 x 256 complex pball 0.33 + background pball 3/256, L-BFGS tol 1e-6, float64'}
    BLMLBinned(dtype=np.float64, solver='lbfgs', tol=1e-6, device=dev).fit(counts, modes, complex_g=True)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    m = BLMLBinned(dtype=np.float64, solver='lbfgs', tol=1e-6, device=dev).fit(counts, modes, complex_g=True)
    torch.cuda.synchronize()
    t = time.perf_counter() - t0
    ref = float(g['loglik'])
    out['fit'] = {'seconds': t, 'iterations': int(m.n_sweeps_), 'loglik': float(m.loglik_),
                  'rel_dloglik_vs_reference': (float(m.loglik_) - ref) / abs(ref),
                  'reference_cpu_seconds': float(g['seconds']), 'reference_iterations': int(g['n_sweeps']),
                  'reference_cores': int(g['cores'])}
    specs, _ = parse_modes(modes, 2)
    h = np.ones(2)
    st = torch.cuda.current_stream(dev).cuda_stream
    rng = np.random.default_rng(3)
    for k, sp in enumerate(specs):
        tr = mode_transform(sp, shape, h, pad_rule(shape, h, specs))
        e = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
        ref = None
        row = {}
        for name, code, eng, route in (('fft_f64', _lib.F64, _lib.ENGINE_SIMT, _lib.ROUTE_FFT),
                                       ('contract_f64', _lib.F64, _lib.ENGINE_SIMT, _lib.ROUTE_CONTRACT),
                                       ('tcgen05_split_tf32_f32', _lib.F32, _lib.ENGINE_TC, None)):
            p = Plan(*tr, shape, code, eng)
            if route is not None:
                p.route = route
            x = torch.as_tensor(e).to(dev, torch.complex128 if code == _lib.F64 else torch.complex64)
            y = torch.empty_like(x)
            for _ in range(3):
                p.apply(x, y, 1, True, st)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(reps):
                p.apply(x, y, 1, True, st)
            e1.record(); torch.cuda.synchronize()
            tm = e0.elapsed_time(e1) / 1e3 / reps
            yy = y.cpu().numpy().astype(np.complex128)
            if ref is None:
                ref = yy
            nbytes = 2 * x.numel() * x.element_size()
            row[name] = {'us': tm * 1e6, 'matvecs_per_s': 1.0 / tm, 'GB_per_s': nbytes / tm / 1e9,
                         'rel_err_vs_fft_f64': float(np.abs(yy - ref).max() / np.abs(ref).max())}
        out[f'mode{k}_matvec'] = row
    return out


def quick5d_bench(dev, solvers=('block', 'jacobi')):
    """The 5-D fixed-lattice fit at size (n = 2e5 points of an 8-component mixture, bins at 1/64, B ~ 1.84e5 occupied
    bins, sinc fc = 0.1 cycles per bin per column; blml_trivial.py:2860-3035 through BLMLQuickLattice): float32 pair
    tables, float64 state and loglik, tol 1e-4 (BLMLQuick's default); wall time of the public fit call, sweeps, the
    final max|rho| (S e recomputed exactly at the stop) and the loglik. The objective is convex (real rank 1), so a fit
    that meets tol is at the unique optimum; solvers: the block coordinate descent and the Jacobi / Anderson sweep."""
    import torch
    from blml_b200 import workloads
    from blml_b200.quick import BLMLQuickLattice, bin_points
    from blml_b200.spec import make_modes, with_lattice
    X = workloads.points_5d_mixture(seed=0)
    u, cnt = bin_points(X, 1 / 64, device=dev)
    Zc = u.cpu().numpy() / 64.0
    w = cnt.cpu().numpy()
    modes = with_lattice(make_modes(np.full(5, 0.1 * 64), ['sinc'] * 5), 1 / 64)
    out = {'workload': '5-D fixed-lattice fit: n = 2e5 points, 8-component mixture, bins at 1/64, sinc fc 0.1 / bin',
           'bins': int(len(w))}
    for solver in solvers:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        m = BLMLQuickLattice(tol=1e-4, dtype=np.float32, device=dev, solver=solver).fit(Zc, modes, sample_weight=w)
        torch.cuda.synchronize()
        t = time.perf_counter() - t0
        out[solver] = {'seconds': t, 'sweeps': int(m.n_sweeps_), 'residual': float(m.residual_),
                       'converged': bool(m.converged_), 'loglik': float(m.loglik_), 'stop': m.stop_reason_,
                       'seconds_per_sweep': t / max(m.n_sweeps_, 1)}
    return out


def select_bench(dev, n_search=16, seq_sample=2, batch=256):
    """The cut-off search over many lattices (selector.py:488-553 `_search`, run on binned counts as
    dslit_job.py:158-171 does): 16 lattices of 64 x 64 from two-disk fields (band fc geomspace(0.08, 0.4, 16),
    N = 5e4, 80/20 binomial split), sinc x sinc cut-offs searched from fc0 = 0.02 with factors sqrt 2, 2^1/4, 2^1/8
    inside [2/64, 0.5]; each candidate a complex L-BFGS fit to tol 1e-6 (at most 3000 iterations, float64) scored on
    its validation counts. Batched: every search at once, speculative rounds of about `batch` fits. Sequential: the
    reference's order, one candidate after another through the single-fit GPU engine, on a sample of the searches."""
    import torch
    from blml_b200 import workloads, selector as ps, make_modes
    from blml_b200.binned import BLMLBinned
    tr, va = [], []
    for i, fc in enumerate(np.geomspace(0.08, 0.4, n_search)):
        c = workloads.two_disk_field((64, 64), fc=float(fc), N=5e4, seed=100 + i)
        t = np.random.default_rng(i).binomial(c.astype(np.int64), 0.8).astype(float)
        tr.append(t); va.append(c - t)
    kw = dict(fc0=0.02, fc_min=2 / 64, fc_max=0.5, factors=ps.SEARCH_FACTORS, tol=1e-6, max_fit_sweeps=3000)
    ps.select_counts_batched(tr[:2], va[:2], batch=32, **{**kw, 'factors': (ps.SQRT2,)})     # warm-up
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    out, stats = ps.select_counts_batched(tr, va, batch=batch, return_stats=True, **kw)
    torch.cuda.synchronize()
    t_b = time.perf_counter() - t0
    picks = [np.array([m[0][0]['fc'], m[0][1]['fc']]) for m, _ in out]
    seq_fits, same = 0, 0
    t0 = time.perf_counter()
    for s in range(seq_sample):
        trd = torch.as_tensor(tr[s]).to(dev)

        def obj(fc, s=s, trd=trd):
            nonlocal seq_fits
            if np.any(fc > 0.5 * (1 + 1e-9)) or np.any(fc < 2 / 64):
                return -np.inf
            seq_fits += 1
            m = BLMLBinned(tol=1e-6, max_sweeps=3000, solver='lbfgs', dtype=np.float64, device=dev).fit(
                trd, make_modes(list(fc), ['sinc', 'sinc']), complex_g=True)
            p = np.maximum(m.density_, 1e-300)
            return float(np.sum(va[s] * np.log(p / p.sum())) / va[s].sum())
        fc, _ = ps.search(obj, 2, ['sinc', 'sinc'], [None, None], fc0=kw['fc0'], factors=kw['factors'])
        same += int(np.array_equal(fc, picks[s]))
    torch.cuda.synchronize()
    t_s = (time.perf_counter() - t0) / seq_sample
    return {'workload': '16 cut-off searches (sinc x sinc, 3 refinement factors) on 64 x 64 two-disk lattices, '
                        'candidates = complex L-BFGS fits to tol 1e-6 (<= 3000 its), validation-scored',
            'batched': {'selections_per_s': n_search / t_b, 'seconds': t_b, 'rounds': stats['rounds'],
                        'fits': stats['fits'], 'fits_used': stats['used'], 'batch': batch},
            'sequential_single_fit_gpu': {'selections_per_s': 1.0 / t_s, 'seconds_per_selection': t_s,
                                          'sample': f'{seq_sample} searches, {seq_fits} fits',
                                          'same_pick_as_batched': f'{same}/{seq_sample}'},
            'speedup': t_s * n_search / t_b,
            'picks': [[round(float(x), 5) for x in p] for p in picks]}


def _timed(f, reps=1):
    import torch
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(reps):
        out = f()
    torch.cuda.synchronize()
    return (time.perf_counter() - t0) / reps, out


def extras_bench(dev):
    """The rows built around the fit, timed on the GPU (synchronised wall time of the public call) beside a bounded
    CPU-oracle sample where the oracle restates the row:
      gradients  fc_grad and implicit_grad (CG, at most 300 iterations) of a complex sinc x sinc fit on 128 x 128,
                 float64, against the oracle's NumPy / SciPy FFT restatement at the same coefficients;
      points     predict at 2e5 off-lattice points of a 2-D sinc x dirichlet point fit (n = 2e5 points, float32 state,
                 tol 1e-4 as the reference's defaults; float64 kernel), pairs/s, against the oracle's unit formulas in
                 NumPy on 1,000 of the points;
      streaming  partial_fit of a 96 x 96 complex stream in 12 batches (L-BFGS refits to tol 1e-6, implicit
                 gradients, an Adam step every 3 batches), batches/s; its parity anchor is the reference's own
                 streams, so no CPU restatement is timed."""
    import types
    import torch
    from blml_b200 import workloads, make_modes
    from blml_b200.binned import BLMLBinned
    from blml_b200.quick import BLMLQuick
    from blml_b200.streaming import BLMLBinnedStreaming
    sys.path.insert(0, os.path.join(ROOT, 'oracle'))
    import blml_oracle as bo
    import grad_oracle as go
    out = {}
    # ---- gradients
    c = workloads.two_disk_field((128, 128), fc=0.3, N=2e5, seed=7)
    rng = np.random.default_rng(7)
    tr = rng.binomial(c.astype(np.int64), 0.8).astype(float); va = c - tr
    modes = make_modes([0.3, 0.3], ['sinc', 'sinc'])
    m = BLMLBinned(tol=1e-6, solver='lbfgs', max_sweeps=3000, device=dev).fit(tr, modes, complex_g=True)
    m.fc_grad()
    t_fc, G0 = _timed(m.fc_grad, 3)
    t_ig, G1 = _timed(lambda: m.implicit_grad(va, 1e-3))
    f = bo.BinnedFit(max_sweeps=0, tol=1e-6, solver='lbfgs').fit(
        tr, modes, init=types.SimpleNamespace(e_hat=m.e_hat_, shape=tr.shape), complex_g=True)
    f.e_hat = np.asarray(m.e_hat_); f.Se = f.Sall(f.e_hat)
    t0 = time.perf_counter(); H0 = go.fc_grad(f); c_fc = time.perf_counter() - t0
    t0 = time.perf_counter(); H1, it_c, _ = go.implicit_grad(f, va, 1e-3); c_ig = time.perf_counter() - t0
    out['gradients'] = {'workload': 'complex sinc x sinc fit, 128 x 128, float64',
                        'fc_grad_ms': 1e3 * t_fc, 'implicit_grad_ms': 1e3 * t_ig, 'cg_iterations': int(m.ift_iters_),
                        'cpu_oracle': {'fc_grad_ms': 1e3 * c_fc, 'implicit_grad_ms': 1e3 * c_ig,
                                       'cg_iterations': int(it_c), 'cores': os.cpu_count(), 'kind': 'port'},
                        'fc_grad_rel_diff': float(np.max(np.abs(np.array(G0) - np.array(H0)) / np.abs(np.array(H0))))}
    # ---- points
    X = workloads.two_blob_points(200_000, seed=1)
    pm = make_modes([3.0, 4.0], ['sinc', 'dirichlet'], periods=[None, 1.0])
    t_fit, q = _timed(lambda: BLMLQuick(tol=1e-4, dtype=np.float32, device=dev).fit(X, pm))   # the reference's defaults
    Xq = np.random.default_rng(2).uniform(0.0, 1.0, (200_000, 2))
    q.predict(Xq[:1000])
    t_pr, P = _timed(lambda: q.predict(Xq))
    B = q.n_bins_
    R = 1000
    t0 = time.perf_counter()
    g = np.zeros(R)
    for s0 in range(0, B, 4096):
        Z = q.Z_[s0:s0 + 4096]
        K = bo.unit_value('sinc', [3.0], [None], [Xq[:R, 0, None] - Z[None, :, 0]]) * \
            bo.unit_value('dirichlet', [4.0], [1.0], [Xq[:R, 1, None] - Z[None, :, 1]])
        g += K @ np.ravel(q.e_hat_)[s0:s0 + 4096]
    c_pr = time.perf_counter() - t0
    ref = (g / q.n_samples_) ** 2
    out['points'] = {'workload': '2-D sinc x dirichlet point fit, n = 2e5 points, predict at 2e5 points',
                     'bins': int(B), 'fit_s': t_fit, 'fit_sweeps': int(q.n_sweeps_), 'fit_stop': q.stop_reason_,
                     'predict_s': t_pr, 'Gpair_per_s': 2e5 * B / t_pr / 1e9,
                     'cpu_oracle': {'Gpair_per_s': R * B / c_pr / 1e9, 'sample': f'{R} points x {B} bins',
                                    'cores': os.cpu_count(), 'kind': 'port'},
                     'predict_rel_diff': float(np.max(np.abs(P[:R] - ref)) / np.max(ref))}
    # ---- streaming
    full = workloads.two_disk_field((96, 96), fc=0.3, N=3e5, seed=9)
    parts = np.random.default_rng(9).multinomial(1, [1 / 12] * 12, size=int(full.sum()))
    idx = np.repeat(np.arange(full.size), full.astype(np.int64).ravel())
    batches = [np.bincount(idx[parts[:, j] > 0], minlength=full.size).reshape(full.shape).astype(float)
               for j in range(12)]
    sm = make_modes([0.25, 0.25], ['sinc', 'sinc'])
    st = BLMLBinnedStreaming(tol=1e-6, solver='lbfgs', max_sweeps=2000, param_every=3, device=dev)
    st.partial_fit(batches[0], sm, complex_g=True)
    t_st, _ = _timed(lambda: [st.partial_fit(b) for b in batches[1:]])
    out['streaming'] = {'workload': '96 x 96 complex stream, 12 batches, L-BFGS refits tol 1e-6, Adam every 3',
                        'batches_per_s': 11 / t_st, 'seconds': t_st,
                        'fc_final': [float(v) for v in st.specs_[0]['fc']]}
    return out


def flush_l2(buf):
    buf.add_(1.0)


def main():
    global LBFGS_M, MAX_RANK, HISTORY_F32, ROUND_LL_TOL, GROW_ITERS, GROW_STEP, LANCZOS_BASIS, GROW_TWO_ABOVE
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=3)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--impl', default='b200', choices=['b200', 'reference'])
    ap.add_argument('--one-fit', action='store_true', help='one batched sweep and exit (profiling runs)')
    ap.add_argument('--certify', action='store_true',
                    help='one certified sweep (rank growth) with its per-round statistics, and exit')
    ap.add_argument('--pairs', action='store_true',
                    help='the 5-D pair path: one full rows pass over all bin pairs, GPU and a CPU-oracle sample')
    ap.add_argument('--tune', action='store_true',
                    help="the FFT route's autotuner: time its launch shapes on the sweep, write the package's table")
    ap.add_argument('--config2', action='store_true',
                    help='the 256 x 256 complex two-mode pball fit and its mat-vec routes')
    ap.add_argument('--quick5d', action='store_true',
                    help='the 5-D fixed-lattice fit at size (B ~ 1.84e5 bins): block CD and Jacobi sweeps')
    ap.add_argument('--select', action='store_true',
                    help='the batched cut-off search over 16 lattices beside the sequential single-fit search')
    ap.add_argument('--extras', action='store_true',
                    help='the gradients, point predictions and streaming refits, each beside a CPU-oracle sample')
    ap.add_argument('--segscan', action='store_true',
                    help="the L-BFGS history scan and direction kernels at the sweep's size (--segscan-k modes per fit)")
    ap.add_argument('--segscan-k', type=int, default=4)
    ap.add_argument('--lbfgs-m', type=int, default=20, help='L-BFGS memory of the certified rounds (1..20)')
    ap.add_argument('--max-rank', type=int, default=MAX_RANK, help='most shared modes a certified fit grows to')
    ap.add_argument('--history-f64', action='store_true', help='certified rounds keep a complex128 L-BFGS history')
    ap.add_argument('--grow-iters', type=int, default=GROW_ITERS, help='L-BFGS cap of the rounds below the last rank')
    ap.add_argument('--grow-step', type=float, default=GROW_STEP, help='size of a new mode (x the rms mode)')
    ap.add_argument('--lanczos-basis', type=int, default=LANCZOS_BASIS, help="the certificate's Lanczos basis")
    ap.add_argument('--grow-two-above', type=float, default=GROW_TWO_ABOVE,
                    help='a certificate above this level grows two modes at once')
    ap.add_argument('--round-ll-tol', type=float, default=ROUND_LL_TOL,
                    help="the certified rounds' L-BFGS stop on L / n gained over 10 iterations")
    ap.add_argument('--matvec', action='store_true',
                    help="only the grouped mat-vec chain over the sweep's 64 lattices, 3 warm-up + 20 timed chains "
                         "(profiling runs)")
    args = ap.parse_args()
    LBFGS_M, MAX_RANK, HISTORY_F32 = args.lbfgs_m, args.max_rank, not args.history_f64
    ROUND_LL_TOL, GROW_ITERS, GROW_STEP = args.round_ll_tol, args.grow_iters, args.grow_step
    LANCZOS_BASIS, GROW_TWO_ABOVE = args.lanczos_basis, args.grow_two_above
    rank, ws, local = dist_init()
    if args.impl == 'reference':
        return reference_arm(args, rank, ws)
    import torch
    from blml_b200.sweep import BLMLBinnedBatch
    from blml_b200.binned import BLMLBinned
    from blml_b200 import _lib
    dev = torch.device('cuda', local)
    torch.cuda.set_device(dev)
    sweep, modes = workload(seed=0)                    # every rank runs a replica of the same sweep
    train = [f['train'] for f in sweep]; val = [f['val'] for f in sweep]
    if args.pairs:
        print(json.dumps(pairs_bench(dev)), flush=True)
        return
    if args.select:
        print(json.dumps(select_bench(dev)), flush=True)
        return
    if args.quick5d:
        print(json.dumps(quick5d_bench(dev)), flush=True)
        return
    if args.config2:
        print(json.dumps(config2_bench(dev)), flush=True)
        return
    if args.tune:
        print(json.dumps(tune_fft(dev)), flush=True)
        return
    if args.extras:
        print(json.dumps(extras_bench(dev)), flush=True)
        return
    if args.segscan:
        print(json.dumps(segscan_bench(dev, K=args.segscan_k)), flush=True)
        return
    if args.matvec:
        b = BLMLBinnedBatch(tol=TOL, dtype=np.float64, device=dev)
        b._prepare(train, modes)
        out = {}
        for name, route in (('auto', 0), ('contract', _lib.ROUTE_CONTRACT), ('fft', _lib.ROUTE_FFT)):
            t_mv, mv_bytes, mv_flops = grouped_matvec_roofline(b, route=route)
            out[name] = {'us_per_chain': t_mv * 1e6, 'bytes': mv_bytes, 'GB/s': mv_bytes / t_mv / 1e9}
        print(json.dumps(out))
        return
    if args.one_fit:
        b = BLMLBinnedBatch(tol=TOL, dtype=np.float64, device=dev)
        l0 = _lib.lib().blml_launch_count()
        res = b.fit(train, modes)
        torch.cuda.synchronize()
        print(json.dumps({'launches': int(_lib.lib().blml_launch_count() - l0), 'bins': int(b.Btot),
                          'iterations_max': max(r.n_sweeps_ for r in res),
                          'loglik_mean': float(np.mean([r.loglik_ for r in res])),
                          'start': getattr(b, 'start_stats_', None), 'lbfgs': getattr(b, 'lbfgs_stats_', None),
                          'phase_seconds': getattr(b, 'timing_', None)}))
        return
    train_dev = [torch.as_tensor(c).to(dev) for c in train]
    val_dev = [torch.as_tensor(c).to(dev) for c in val]
    if args.certify:
        l0 = _lib.lib().blml_launch_count()
        t0 = time.perf_counter()
        b, res, sc = certified_sweep(dev, train_dev, val_dev, modes)
        torch.cuda.synchronize()
        out = {'seconds': time.perf_counter() - t0, 'launches': int(_lib.lib().blml_launch_count() - l0),
               'stats': b.certify_stats_,
               'rank_path': [r.rank_path_ for r in res], 'scores': sc.tolist()}
        try:
            out['certified'] = certify(res, oracle_ref())[0]
        except FileNotFoundError:
            pass
        print(json.dumps(out), flush=True)
        return
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    ref = oracle_ref()
    # the plain engine: the same certification, one fit at a time (no batching), cold starts, on every 4th sweep fit
    # (16 fits spread over the lattice sizes and cut-offs) to keep the run short
    certified_sweep(dev, train_dev[:1], val_dev[:1], modes[:1])
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    plain_res = []
    for i in PLAIN_SAMPLE:
        plain_res += certified_sweep(dev, train_dev[i:i + 1], val_dev[i:i + 1], modes[i:i + 1])[1]
    torch.cuda.synchronize()
    t_plain = time.perf_counter() - t0
    plain_cert = int(certified_mask([r.loglik_ for r in plain_res], [r.certificate_ for r in plain_res],
                                    ref[list(PLAIN_SAMPLE)])[0].sum())
    del plain_res
    for _ in range(args.warmup):
        certified_sweep(dev, train_dev, val_dev, modes)
    st = torch.cuda.current_stream(dev)
    barrier_sync(ws)
    l0 = _lib.lib().blml_launch_count()
    tot = 0.0; certified = 0; rel = cert = ranks = None; stats = None
    with Clocks(local) as clk:
        for _ in range(args.steps):
            flush_l2(flush)
            barrier_sync(1)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            b, res, scores = certified_sweep(dev, train_dev, val_dev, modes)
            e1.record(st); torch.cuda.synchronize()
            tot += e0.elapsed_time(e1) / 1e3
            c1, rel, cert = certify(res, ref)
            certified += c1
            ranks = np.array([r.rank_ for r in res]); stats = b.certify_stats_
    launches = _lib.lib().blml_launch_count() - l0
    barrier_sync(ws)
    value, tmax = replica_value(certified, tot, ws)
    # end to end through the public API: host counts in, densities and held-out scores out, every step
    e2e_steps = min(args.steps, 5)
    e2e_t = 0.0; e2e_cert = 0; d2h = 0
    for _ in range(e2e_steps):
        flush_l2(flush)
        barrier_sync(1)
        t0 = time.perf_counter()
        _, res, sc = certified_sweep(dev, train, val, modes)
        dens = [r.density_ for r in res]
        torch.cuda.synchronize()
        e2e_t += time.perf_counter() - t0
        e2e_cert += certify(res, ref)[0]
        d2h = int(sum(d.nbytes for d in dens) + sc.nbytes)
    e2e_t = max_over_ranks(e2e_t, ws)
    e2e_value = sum_over_ranks(e2e_cert, ws) / e2e_t if e2e_t > 0 else 0.0
    learned = learned_arm(dev, sweep, modes, train_dev, val_dev, ref, flush, ws)
    # the reference arm's bounded sample (its 8 cheapest fits) certified here too, in one batch: the same work on both
    sample = port_sample()
    st_, sv_, sm_ = [train_dev[i] for i in sample], [val_dev[i] for i in sample], [modes[i] for i in sample]
    certified_sweep(dev, st_, sv_, sm_)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    _, sres, _ = certified_sweep(dev, st_, sv_, sm_)
    torch.cuda.synchronize()
    t_s = time.perf_counter() - t0
    s_cert = int(certified_mask([r.loglik_ for r in sres], [r.certificate_ for r in sres], ref[sample])[0].sum())
    same_sample = {'value': s_cert / t_s, 'unit': 'fits/s', 'certified': s_cert, 'fits': len(sample),
                   'seconds': t_s, 'what': "the reference arm's sample (its 8 cheapest fits) certified in one batch"}
    b1 = BLMLBinnedBatch(tol=TOL, dtype=np.float64, device=dev)
    b1._prepare(train, modes)
    t_mv, mv_bytes, mv_flops = grouped_matvec_roofline(b1)
    scan = segscan_bench(dev, K=4)
    pk = peaks()
    peak = pk['hbm_gbs'] if pk else 6650.0
    achieved = mv_bytes / t_mv / 1e9
    if rank == 0:
        cpu = None
        if ws == 1:
            sample = port_sample()
            pool, procs = port_pool()
            try:
                port_step(pool, sample, ref)                      # worker start-up and imports
                wall, nc = port_step(pool, sample, ref)
            finally:
                pool.terminate()
            cpu = {'value': nc / wall, 'unit': 'fits/s', 'cores': procs, 'kind': 'port',
                   'sample': sample_desc(sample, procs)}
        out = {'metric': METRIC, 'value': value, 'unit': 'fits/s', 'n_gpus': ws, 'steps': args.steps,
               'warmup': args.warmup, 'ms_per_step': 1e3 * tmax / args.steps, 'higher_is_better': True,
               'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f64', 'data': 'synthetic',
               'config': dict(CONFIG, e2e_steps=e2e_steps),
               'e2e': {'value': e2e_value, 'unit': 'fits/s',
                       'h2d_bytes_per_step': int(sum(c.nbytes for c in train) + sum(c.nbytes for c in val)),
                       'd2h_bytes_per_step': d2h},
               'gpu_launches': int(launches),
               'roofline': {'bound': 'hbm', 'achieved': scan['dots2_h32']['GB/s'], 'peak': peak, 'unit': 'GB/s',
                            'frac': scan['dots2_h32']['GB/s'] / peak, 'traffic': scan_traffic(4, 'h32'),
                            'kernel': f"k_seg_dots2_h32, the certified rounds' L-BFGS history scan (with the "
                                      f"direction's linear combination, the largest share of the certified sweep's "
                                      f"GPU time): the 20 stored complex64 vectors and the shared complex64 y and "
                                      f"complex128 g and E over the 64 sweep lattices at K = 4 modes, "
                                      f"{scan['elements']} elements: {21 * 8 * scan['elements'] + 32 * scan['elements']} "
                                      f"algorithmic bytes, {scan['dots2_h32']['us']:.1f} us per call (its block split, "
                                      f"the scan and the partials' sum: 3 launches)",
                            'peak_source': 'MEASURED_PEAKS.json hbm_gbs (of measured)' if pk else 'fallback'},
               'roofline_scan_c128': {'bound': 'hbm', 'achieved': scan['dots2']['GB/s'], 'peak': peak, 'unit': 'GB/s',
                                      'frac': scan['dots2']['GB/s'] / peak, 'traffic': scan_traffic(4),
                                      'kernel': f"k_seg_dots2_c128<double2, double2>, the complex128 history scan of "
                                                f"plain fits, {scan['dots2']['us']:.1f} us per launch"},
               'roofline_lincomb': {'bound': 'hbm', 'achieved': scan['lincomb']['GB/s'], 'peak': peak,
                                    'unit': 'GB/s', 'frac': scan['lincomb']['GB/s'] / peak,
                                    'kernel': f"k_seg_lincomb<double, double2>, the direction (41 vectors in, 1 out), "
                                              f"{scan['lincomb']['us']:.1f} us per launch"},
               'roofline_lincomb_h32': {'bound': 'hbm', 'achieved': scan['lincomb_h32']['GB/s'], 'peak': peak,
                                        'unit': 'GB/s', 'frac': scan['lincomb_h32']['GB/s'] / peak,
                                        'kernel': f"k_seg_lincomb_mixed<double2>, the certified rounds' direction "
                                                  f"(complex128 g and 40 complex64 vectors in, complex128 out), "
                                                  f"{scan['lincomb_h32']['us']:.1f} us per call (its block split and "
                                                  f"the combination: 2 launches)"},
               'roofline_matvec': {'bound': 'hbm', 'achieved': achieved, 'peak': peak, 'unit': 'GB/s',
                                   'frac': achieved / peak, 'traffic': traffic_from_profiles(),
                                   'kernel': f'grouped mat-vec over the 64 fits (FFT route: 3 grouped launches, '
                                             f'float64): {mv_bytes} algorithmic bytes (read E + write U, complex128), '
                                             f'{t_mv * 1e6:.1f} us per chain; latency bound'},
               'cpu_baseline': cpu, 'clocks': clk.summary(),
               'plain_gpu': {'value': plain_cert / t_plain, 'unit': 'fits/s', 'certified': plain_cert,
                             'fits': len(PLAIN_SAMPLE), 'seconds': t_plain,
                             'what': 'the same certification with one fit at a time (no batching), cold starts, '
                                     'on every 4th sweep fit'},
               'sweep': {'certified_per_step': certified / args.steps, 'rel_dloglik_max_abs': float(np.max(np.abs(rel))),
                         'rel_dloglik_median': float(np.median(rel)), 'certificate_max': float(np.max(cert)),
                         'rank_max': int(ranks.max()), 'rank_mean': float(ranks.mean()),
                         'rank_rounds': stats['rounds'], 'fits_per_round': stats['fits_per_round'],
                         'lbfgs_iterations_max_per_round': stats['lbfgs_iterations_max'],
                         'certificate_seconds': stats['seconds_certificate'], 'bins': int(b1.Btot)},
               'learned': learned, 'same_sample_gpu': same_sample}
        print(json.dumps(out), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.barrier(); dist.destroy_process_group()


def reference_arm(args, rank, ws):
    """The reference's algorithm on the host cores (the float64 NumPy / SciPy port, oracle/blml_oracle.py; the
    reference itself lives only in the build container): each step certifies a fixed bounded sample of the sweep's
    fits whole, one fit per process; value = certified fits / wall time of the sample."""
    if rank != 0:
        return
    ref = oracle_ref()
    sample = port_sample()
    pool, procs = port_pool()
    walls, ncs = [], []
    try:
        for i in range(args.warmup + args.steps):
            wall, nc = port_step(pool, sample, ref)
            if i >= args.warmup:
                walls.append(wall); ncs.append(nc)
    finally:
        pool.terminate()
    v = float(np.sum(ncs) / np.sum(walls))
    out = {'metric': METRIC, 'value': v, 'unit': 'fits/s', 'n_gpus': ws, 'steps': args.steps, 'warmup': args.warmup,
           'ms_per_step': 1e3 * float(np.mean(walls)), 'higher_is_better': True, 'scaling': 'weak',
           'vs_baseline': None, 'dtype': 'f64', 'data': 'synthetic', 'config': CONFIG, 'impl': 'reference',
           'cpu_baseline': {'value': v, 'unit': 'fits/s', 'cores': procs, 'kind': 'port',
                            'sample': sample_desc(sample, procs)},
           'e2e': {'value': v, 'unit': 'fits/s', 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0}}
    print(json.dumps(out), flush=True)


if __name__ == '__main__':
    main()
