"""The batched engine (many fits of uneven lattice size and cut-off in lockstep) against the single-fit engine on
the same counts: the same start and solver, so each fit lands on the single fit's likelihood (1e-6 relative, the
certification bar); the grouped mat-vec equals per-plan mat-vecs; held-out scores equal log_density."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _sweep(n=4, seed=7):
    from blml_b200 import workloads
    rng = np.random.default_rng(seed)
    sides = [(32, 32), (48, 64), (64, 48), (40, 40), (64, 64), (32, 48)]
    fcs = [0.33, 0.25, 0.4, 0.3, 0.2, 0.45]
    out = []
    for i in range(n):
        shape, fc = sides[i % len(sides)], fcs[i % len(fcs)]
        counts = workloads.two_disk_field(shape, fc=fc, N=float(rng.integers(5e3, 5e4)), seed=seed + i)
        out.append((counts, workloads.pball_modes(shape, fc)))
    return out


def test_grouped_matvec_equals_single(cuda_device):
    from blml_b200.sweep import _Group
    from blml_b200 import operator as op_mod, _lib
    from blml_b200.spec import parse_modes
    fits = _sweep(4)
    plans, offs, tot = [], [0], 0
    for counts, modes in fits:
        sp, _ = parse_modes(modes, 2)
        shape = counts.shape
        plans.append(op_mod.Plan(*op_mod.mode_transform(sp[0], shape, np.ones(2), shape), shape, _lib.F64,
                                 _lib.ENGINE_SIMT))
        tot += counts.size; offs.append(tot)
    x = torch.randn(tot, dtype=torch.complex128, device='cuda')
    y = torch.empty_like(x)
    _Group(plans, x, offs[:-1], y, offs[:-1], True)(torch.cuda.current_stream().cuda_stream)
    for g, (counts, _) in enumerate(fits):
        ref = torch.empty(counts.size, dtype=torch.complex128, device='cuda')
        plans[g].apply(x[offs[g]:offs[g + 1]].contiguous(), ref, 1, True, torch.cuda.current_stream().cuda_stream)
        assert (y[offs[g]:offs[g + 1]] - ref).abs().max().item() <= 1e-12 * ref.abs().max().item()


@pytest.mark.parametrize('dt', [np.float64, np.float32])
def test_batch_matches_single_fits(cuda_device, dt):
    from blml_b200.sweep import BLMLBinnedBatch
    from blml_b200.binned import BLMLBinned
    fits = _sweep(4)
    batch = BLMLBinnedBatch(tol=1e-6, dtype=dt)
    res = batch.fit([c for c, _ in fits], [m for _, m in fits])
    bar = 1e-6 if dt == np.float64 else 5e-5        # float32 state stops ~1e-5 short (test_gpu_binned)
    for (counts, modes), r in zip(fits, res):
        one = BLMLBinned(tol=1e-6, solver='lbfgs', dtype=np.float64).fit(counts, modes, complex_g=True)
        assert abs(r.loglik_ - one.loglik_) <= bar * abs(one.loglik_), (r.loglik_, one.loglik_, r.stop_reason_)
        assert r.density_.shape == counts.shape and np.all(np.isfinite(r.density_))


def test_batch_held_out_scores(cuda_device):
    from blml_b200.sweep import BLMLBinnedBatch
    fits = _sweep(3, seed=11)
    rng = np.random.default_rng(0)
    train = [rng.binomial(c.astype(np.int64), 0.8).astype(float) for c, _ in fits]
    val = [c - t for (c, _), t in zip(fits, train)]
    batch = BLMLBinnedBatch(tol=1e-5, dtype=np.float64)
    res = batch.fit(train, [m for _, m in fits])
    scores = batch.log_density(val)
    for f, r in enumerate(res):
        dens = r.density_
        ref = float(np.sum(val[f][val[f] > 0] * np.log(dens[val[f] > 0] / dens.sum())) / val[f].sum())
        assert abs(scores[f] - ref) <= 1e-6 * abs(ref)
