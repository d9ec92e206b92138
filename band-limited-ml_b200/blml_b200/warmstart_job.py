"""Training and evaluation of the learned warm start on one GPU (the engine makes its own training data).

    python -m blml_b200.warmstart_job train --fits 2048 --sweeps 8 --epochs 20 --out weights.npz
    python -m blml_b200.warmstart_job eval --weights weights.npz --fits 512 [--set sweep]
    python -m blml_b200.warmstart_job gemm [--mnk 262144,288,864]      # the BF16 tcgen05 product alone

train: fits of workloads.warm_start_set (128 x 128, two-disk pupils under a pball kernel or two-slit pupils under a
slits x sinc kernel, fc ~ U(0.1, 0.4), N = 10^U(4, 6)) plus cut-off sweeps of other seeds than the benchmark's
(workloads.cutoff_sweep: 2-D pball, sides 64..384) are fitted cold by the batched engine (float64, tol 1e-6); the
network learns their fields u = S e / n; weights are saved as BF16 bit patterns (.npz).
eval: fresh seeds, fitted cold (the seeded real start + L-BFGS) and warm (the network's start + L-BFGS) by the batched
engine: iterations, seconds, certified fraction (warm loglik >= cold loglik - 1e-6 relative). One JSON line."""
import argparse
import json
import time

import numpy as np
import torch

from . import workloads
from .sweep import BLMLBinnedBatch
from .warmstart import WarmStartNet, features, make_training_set

TRAIN_SEED, SWEEP_SEED, EVAL_SEED = 10_000, 20_000, 50_000
# iteration cap of every fit here (start sweeps and L-BFGS iterations each): the real rank-1 start of a slits x sinc
# kernel can creep (its merit keeps gaining a little, so the stall rule never fires), and the reference's own solver
# has no cap by default; the benchmark sweep's fits stay well below it (at most 1,295 start sweeps, ~3,300 L-BFGS
# iterations)
CAP = 5000


def engine_fields(fits, batch=64, tol=1e-6, cap=CAP):
    """Cold fits of `fits` (dicts with counts, modes) by the batched engine, grouped in batches; returns the fields
    (device complex tensors), the BLMLBinnedBatch results and the seconds spent."""
    fields, results, secs = [], [], 0.0
    for b0 in range(0, len(fits), batch):
        part = fits[b0:b0 + batch]
        t0 = time.perf_counter()
        b = BLMLBinnedBatch(tol=tol, dtype=np.float64, max_sweeps=cap)
        res = b.fit([f['counts'] for f in part], [f['modes'] for f in part])
        torch.cuda.synchronize()
        secs += time.perf_counter() - t0
        fields += [b.field(i).clone() for i in range(len(part))]
        results += res
        print(f'  engine fits {b0 + len(part)}/{len(fits)}: {time.perf_counter() - t0:.1f} s', flush=True)
    return fields, results, secs


def sweep_fits(n_sweeps, seed=SWEEP_SEED):
    out = []
    for s in range(n_sweeps):
        for f in workloads.cutoff_sweep(seed=seed + 64 * s, n_fits=64):
            out.append(dict(kind='pball', fc=f['fc'], N=f['N'], counts=f['train'],
                            modes=workloads.pball_modes(f['shape'], f['fc'])))
    return out


def train(args):
    fits = workloads.warm_start_set(args.fits, seed=TRAIN_SEED, shape=(128, 128)) + sweep_fits(args.sweeps)
    t0 = time.perf_counter()
    fields, _, fit_secs = engine_fields(fits, cap=args.data_cap)
    by_shape = {}
    for f, u in zip(fits, fields):
        by_shape.setdefault(tuple(np.shape(f['counts'])), []).append((f, u))
    net = WarmStartNet(seed=args.seed)
    hist = []
    # every epoch visits each lattice shape's samples (batch size scaled so a batch holds ~128^2 x 16 bins)
    datasets = {}
    for shape, items in by_shape.items():
        datasets[shape] = make_training_set([f for f, _ in items], [u for _, u in items])
    t1 = time.perf_counter()
    for ep in range(args.epochs):
        losses = []
        for shape, data in sorted(datasets.items()):
            bs = int(max(1, min(args.batch * 128 * 128 // (shape[0] * shape[1]), data['x'].shape[0])))
            h = net.train(data, epochs=1, batch=bs, lr=args.lr * (0.1 if ep >= int(0.8 * args.epochs) else 1.0),
                          seed=args.seed + ep)
            losses.append((h[0], data['x'].shape[0]))
        hist.append(sum(l * n for l, n in losses) / sum(n for _, n in losses))
        print(f'epoch {ep}: loss {hist[-1]:.4f} ({time.perf_counter() - t1:.1f} s)', flush=True)
    torch.cuda.synchronize()
    save_bf16(net.params_numpy(), args.out)
    print(json.dumps({'fits': len(fits), 'shapes': len(by_shape), 'fit_seconds': fit_secs,
                      'train_seconds': time.perf_counter() - t1, 'total_seconds': time.perf_counter() - t0,
                      'loss_first': hist[0], 'loss_last': hist[-1], 'loss_history': hist}))


def to_bf16_bits(a):
    """float32 -> BF16 bit patterns (round to nearest even), uint16."""
    u = np.ascontiguousarray(a, np.float32).view(np.uint32)
    return ((u + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint16)


def from_bf16_bits(b):
    return (np.asarray(b, np.uint32) << 16).view(np.float32)


def save_bf16(params, path):
    """The weights as BF16 bit patterns (what the network computes with), half the size of float32."""
    np.savez_compressed(path, **{k: to_bf16_bits(v) for k, v in params.items()})


def load(path, device='cuda'):
    z = np.load(path)
    p = {k: (from_bf16_bits(z[k]) if z[k].dtype == np.uint16 else z[k]) for k in z.files}
    return WarmStartNet(device=device, params=p)


def evaluate(net, fits, tol=1e-6, batch=64):
    """Cold vs warm on `fits` by the batched engine, in batches: per-fit iterations and loglik, seconds."""
    cold, warm = [], []
    t_cold = t_warm = 0.0
    for b0 in range(0, len(fits), batch):
        part = fits[b0:b0 + batch]
        counts = [f['counts'] for f in part]; modes = [f['modes'] for f in part]
        torch.cuda.synchronize(); t0 = time.perf_counter()
        rc = BLMLBinnedBatch(tol=tol, dtype=np.float64, max_sweeps=CAP).fit(counts, modes)
        torch.cuda.synchronize(); t_cold += time.perf_counter() - t0
        t0 = time.perf_counter()
        E0 = net.start(counts, [f['fc'] for f in part], [f['kind'] for f in part])
        rw = BLMLBinnedBatch(tol=tol, dtype=np.float64, max_sweeps=CAP).fit(counts, modes, init=E0)
        torch.cuda.synchronize(); t_warm += time.perf_counter() - t0
        cold += rc; warm += rw
    llc = np.array([r.loglik_ for r in cold]); llw = np.array([r.loglik_ for r in warm])
    rel = (llw - llc) / np.abs(llc)
    itc = np.array([r.start_sweeps_ + r.n_sweeps_ for r in cold]); itw = np.array([r.n_sweeps_ for r in warm])
    return dict(fits=len(fits), cold_seconds=t_cold, warm_seconds=t_warm, cold_fits_per_s=len(fits) / t_cold,
                warm_fits_per_s=len(fits) / t_warm, speedup=t_cold / t_warm,
                certified_warm=float(np.mean(rel >= -1e-6)), rel_dloglik_median=float(np.median(rel)),
                rel_dloglik_min=float(rel.min()), cold_iterations_mean=float(itc.mean()),
                cold_lbfgs_mean=float(np.mean([r.n_sweeps_ for r in cold])),
                warm_iterations_mean=float(itw.mean()), iteration_ratio=float(itc.mean() / max(itw.mean(), 1e-9)))


def gemm_bench(M, N, K, reps=10):
    """The network's BF16 tcgen05 product C = A B^T at one shape (random operands): TFLOP/s by CUDA events."""
    from ._lib import call
    g = torch.Generator(device='cuda').manual_seed(0)
    A = torch.randn(M, K, device='cuda', generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device='cuda', generator=g).to(torch.bfloat16)
    C = torch.empty(M, N, device='cuda'); err = torch.zeros(1, dtype=torch.int32, device='cuda')
    st = torch.cuda.current_stream().cuda_stream
    for _ in range(3):
        call('blml_nn_gemm_bf16', A.data_ptr(), B.data_ptr(), C.data_ptr(), M, N, K, 1, err.data_ptr(), st)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        call('blml_nn_gemm_bf16', A.data_ptr(), B.data_ptr(), C.data_ptr(), M, N, K, 1, err.data_ptr(), st)
    e1.record(); torch.cuda.synchronize()
    t = e0.elapsed_time(e1) / 1e3 / reps
    return dict(M=M, N=N, K=K, us=t * 1e6, tflops=2.0 * M * N * K / t / 1e12, err=int(err.item()))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('mode', choices=['train', 'eval', 'gemm'])
    ap.add_argument('--fits', type=int, default=2048)
    ap.add_argument('--sweeps', type=int, default=8)
    ap.add_argument('--epochs', type=int, default=20)
    ap.add_argument('--batch', type=int, default=16)
    ap.add_argument('--lr', type=float, default=1e-3)
    ap.add_argument('--seed', type=int, default=0)
    ap.add_argument('--out', default='warmstart_weights.npz')
    ap.add_argument('--weights', default='warmstart_weights.npz')
    ap.add_argument('--set', default='ws', choices=['ws', 'sweep'], help='eval on the warm-start set or the sweep')
    ap.add_argument('--data-cap', type=int, default=CAP, help='iteration cap of the training fits')
    ap.add_argument('--mnk', default='262144,288,864', help='gemm: M,N,K (the decoder product at 16 x 128^2)')
    args = ap.parse_args()
    if args.mode == 'train':
        return train(args)
    if args.mode == 'gemm':
        print(json.dumps(gemm_bench(*[int(v) for v in args.mnk.split(',')])), flush=True)
        return
    net = load(args.weights)
    if args.set == 'sweep':                         # the benchmark's 64-fit cut-off sweep (seed 0)
        fits = sweep_fits(1, seed=0)
        out = evaluate(net, fits)
        out['workload'] = '64-fit cut-off sweep of the benchmark (sides 64..384, pball)'
    else:
        fits = workloads.warm_start_set(args.fits, seed=EVAL_SEED, shape=(128, 128))
        out = evaluate(net, fits)
        out['workload'] = '128x128 warm-start set, fresh seeds'
    print(json.dumps(out), flush=True)


if __name__ == '__main__':
    main()
