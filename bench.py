"""Benchmark of the binned fitting path on B200 (one JSON line on rank 0).

Workload (N=1): the 2-D complex pball fit -- a 256 x 256 torus, counts ~ Poisson(1e6 p) from two displaced disks
in the band with a random relative phase and a 5% flat background, modes = signal pball (fc 0.33, period 256) +
background pball (fc 3/256), complex_g, L-BFGS to tol 1e-6, float32 state with float64 reductions. A step is one
whole fit. value = fits/s with the counts already in device memory; e2e = fits/s through the public API from host
counts (host->device copy of the counts and device->host read of density_ inside each timed step). Each fit is
certified against a float64 fit of the same counts: |loglik32 - loglik64| / |loglik64| <= 1e-6.

Multi-GPU: the path has no exchange step (independent fits), so N ranks run N replicas of the workload and value
is the total fits of all ranks over the slowest rank's time.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
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

SHAPE = (256, 256)
FC, BG_FC, NCOUNTS, TOL = 0.33, 3 / 256, 1e6, 1e-6
METRIC = 'certified fits/s (dloglik<=1e-6 vs float64), 2-D complex pball fit'
CONFIG = {'workload': '256x256 complex pball fit (signal fc 0.33 + background fc 3/256), L-BFGS tol 1e-6, '
                      'Poisson N=1e6 two-disk field', 'lattice': '256x256', 'modes': 2, 'solver': 'lbfgs',
          'state': 'float32 (float64 reductions)', 'l2': 'flushed between steps (256 MiB write)'}


def workload(seed=0):
    from blml_b200 import workloads
    counts = workloads.two_disk_field(SHAPE, fc=FC, N=NCOUNTS, seed=seed)
    return counts, workloads.pball_modes(SHAPE, FC, BG_FC)


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
        dist.init_process_group('nccl', timeout=timedelta(seconds=120))
        rank = dist.get_rank(); local = int(os.environ.get('LOCAL_RANK', rank))
        torch.cuda.set_device(local)
        return rank, ws, local
    return 0, 1, 0


def barrier_sync(ws):
    import torch
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()


def max_over_ranks(x, ws):
    import torch
    if ws == 1:
        return x
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device='cuda')
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def matvec_roofline(dev, reps=200):
    """Average duration of the signal mode's complex mat-vec (the dominant kernel chain) on the fit's stream with
    CUDA events, and its achieved GB/s against the algorithmic bytes (read E + write U, complex64)."""
    import torch
    from blml_b200.binned import BLMLBinned
    counts, modes = workload(0)
    m = BLMLBinned(dtype=np.float32, device=dev)
    m._setup(counts, modes, 1.0, 0.0)
    plan = m.kern_[0][0]
    x = torch.randn(SHAPE, dtype=torch.complex64, device=dev)
    y = torch.empty_like(x)
    st = torch.cuda.current_stream(dev)
    for _ in range(10):
        plan.apply(x, y, 1, True, st.cuda_stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(reps):
        plan.apply(x, y, 1, True, st.cuda_stream)
    e1.record(st); torch.cuda.synchronize()
    t = e0.elapsed_time(e1) / 1e3 / reps
    nbytes = 2 * x.numel() * x.element_size()
    return t, nbytes, plan.flops_per_lattice


def traffic_from_profiles():
    """Per-mat-vec DRAM bytes from the committed ncu summary, if present."""
    p = os.path.join(ROOT, 'profiles', 'matvec_pball256_traffic.json')
    try:
        return json.load(open(p)).get('dram_bytes_per_matvec')
    except Exception:
        return None


def cpu_port_rate(counts, modes, sample_iters, workers=-1):
    """The CPU port of the reference's algorithm (float64 NumPy/SciPy, FFT over every host core): seconds per L-BFGS
    iteration on this workload, timed over a bounded sample of iterations from the reference's own start."""
    sys.path.insert(0, os.path.join(ROOT, 'oracle'))
    import blml_oracle as bo
    f = bo.BinnedFit(tol=TOL, solver='lbfgs', max_sweeps=0)
    f.workers = workers
    f.fit(counts, modes, complex_g=True)          # set-up and the seeded start, no iterations
    E0 = f.e_hat.copy()
    t0 = time.perf_counter()
    f.solve_lbfgs(E0, sample_iters)
    t = time.perf_counter() - t0
    return t, f.n_sweeps


def flush_l2(buf):
    buf.add_(1.0)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=5)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--impl', default='b200', choices=['b200', 'reference'])
    ap.add_argument('--cpu-sample-iters', type=int, default=40)
    ap.add_argument('--one-fit', action='store_true', help='one fit of the workload and exit (profiling runs)')
    ap.add_argument('--engine', default='simt', choices=['simt', 'tc'], help='mat-vec engine of the float32 fits')
    args = ap.parse_args()
    rank, ws, local = dist_init()
    if args.impl == 'reference':
        return reference_arm(args, rank, ws)
    if args.one_fit:
        from blml_b200.binned import BLMLBinned
        counts, modes = workload(0)
        m = BLMLBinned(tol=TOL, solver='lbfgs', dtype=np.float32, matvec_engine=args.engine).fit(counts, modes,
                                                                                                complex_g=True)
        print(json.dumps({'loglik': m.loglik_, 'iterations': m.n_sweeps_, 'stop': m.stop_reason_}))
        return
    import torch
    from blml_b200.binned import BLMLBinned
    from blml_b200 import _lib
    dev = torch.device('cuda', local)
    torch.cuda.set_device(dev)
    counts, modes = workload(seed=rank)
    counts_dev = torch.as_tensor(counts).to(dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    kw = dict(tol=TOL, solver='lbfgs', dtype=np.float32, device=dev, matvec_engine=args.engine)
    CONFIG['matvec_engine'] = args.engine
    # certification reference: the float64 fit of the same counts
    ref64 = BLMLBinned(tol=TOL, solver='lbfgs', dtype=np.float64, device=dev).fit(counts_dev, modes, complex_g=True)
    for _ in range(args.warmup):
        BLMLBinned(**kw).fit(counts_dev, modes, complex_g=True)
    st = torch.cuda.current_stream(dev)
    barrier_sync(ws)
    l0 = _lib.lib().blml_launch_count()
    tot = 0.0; certified = 0; iters = []; lls = []
    with Clocks(local) as clk:
        for _ in range(args.steps):
            flush_l2(flush)
            barrier_sync(1)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            m = BLMLBinned(**kw).fit(counts_dev, modes, complex_g=True)
            e1.record(st); torch.cuda.synchronize()
            tot += e0.elapsed_time(e1) / 1e3
            iters.append(m.n_sweeps_); lls.append(m.loglik_)
            certified += abs(m.loglik_ - ref64.loglik_) <= 1e-6 * abs(ref64.loglik_)
    launches = _lib.lib().blml_launch_count() - l0
    barrier_sync(ws)
    tmax = max_over_ranks(tot, ws)
    value = certified * ws / tmax if tmax > 0 else 0.0
    # end to end through the public API: host counts in, density_ out, every step
    barrier_sync(ws)
    e2e_t = 0.0; e2e_cert = 0
    for _ in range(args.steps):
        flush_l2(flush)
        barrier_sync(1)
        t0 = time.perf_counter()
        m = BLMLBinned(**kw).fit(counts, modes, complex_g=True)
        dens = m.density_
        torch.cuda.synchronize()
        e2e_t += time.perf_counter() - t0
        e2e_cert += abs(m.loglik_ - ref64.loglik_) <= 1e-6 * abs(ref64.loglik_)
    e2e_t = max_over_ranks(e2e_t, ws)
    e2e_value = e2e_cert * ws / e2e_t if e2e_t > 0 else 0.0
    # dominant kernel: the restricted-transform mat-vec
    t_mv, mv_bytes, mv_flops = matvec_roofline(dev)
    pk = peaks()
    peak = pk['hbm_gbs'] if pk else 6650.0
    achieved = mv_bytes / t_mv / 1e9
    out = None
    if rank == 0:
        cpu = None
        if ws == 1:
            t_s, it_s = cpu_port_rate(counts, modes, args.cpu_sample_iters)
            full_iters = float(np.median(iters))
            per_it = t_s / max(it_s, 1)
            cpu = {'value': 1.0 / (per_it * full_iters), 'unit': 'fits/s', 'cores': os.cpu_count(), 'kind': 'port',
                   'sample': f'{it_s} L-BFGS iterations (from the seeded start; the start solve not timed) of the '
                             f'float64 NumPy/SciPy port with FFTs on every core '
                             f'on this workload in {t_s:.1f} s, scaled to the {full_iters:.0f} iterations of a full fit'}
        out = {'metric': METRIC, 'value': value, 'unit': 'fits/s', 'n_gpus': ws, 'steps': args.steps,
               'warmup': args.warmup, 'ms_per_step': 1e3 * tmax / args.steps, 'higher_is_better': True,
               'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f32', 'data': 'synthetic', 'config': CONFIG,
               'e2e': {'value': e2e_value, 'unit': 'fits/s', 'h2d_bytes_per_step': int(counts.nbytes),
                       'd2h_bytes_per_step': int(dens.nbytes) + 8},
               'gpu_launches': int(launches),
               'roofline': {'bound': 'hbm', 'achieved': achieved, 'peak': peak, 'unit': 'GB/s',
                            'frac': achieved / peak, 'traffic': traffic_from_profiles(),
                            'kernel': 'signal-mode complex mat-vec (4 k_contract stages), L2-resident, '
                                      f'{mv_bytes} algorithmic bytes, {mv_flops:.3e} flop, {t_mv * 1e6:.1f} us',
                            'peak_source': 'MEASURED_PEAKS.json hbm_gbs' if pk else 'fallback'},
               'cpu_baseline': cpu, 'clocks': clk.summary(),
               'fit': {'iterations': iters, 'loglik': lls, 'loglik_f64': ref64.loglik_,
                       'iterations_f64': ref64.n_sweeps_, 'certified': int(certified)}}
        print(json.dumps(out), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.barrier(); dist.destroy_process_group()


def reference_arm(args, rank, ws):
    """The reference's CPU implementation of the path (the float64 NumPy/SciPy port, every host core), each step a
    bounded sample of the same workload's fit, reported as fits/s extrapolated to a full fit's iterations."""
    if rank != 0:
        return
    counts, modes = workload(0)
    full_iters = 916.0          # iterations of the full float64 fit of this workload (reference CPU engine)
    rates = []
    for i in range(args.warmup + args.steps):
        t_s, it_s = cpu_port_rate(counts, modes, args.cpu_sample_iters)
        if i >= args.warmup:
            rates.append(1.0 / (t_s / max(it_s, 1) * full_iters))
    v = float(np.mean(rates))
    out = {'metric': METRIC, 'value': v, 'unit': 'fits/s', 'n_gpus': ws, 'steps': args.steps, 'warmup': args.warmup,
           'ms_per_step': 1e3 / v, 'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f64',
           'data': 'synthetic', 'config': CONFIG, 'impl': 'reference',
           'cpu_baseline': {'value': v, 'unit': 'fits/s', 'cores': os.cpu_count(), 'kind': 'port',
                            'sample': f'{args.cpu_sample_iters} L-BFGS iterations per step of the float64 port, '
                                      f'scaled to {full_iters:.0f} iterations'},
           'e2e': {'value': v, 'unit': 'fits/s', 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0}}
    print(json.dumps(out), flush=True)


if __name__ == '__main__':
    main()
