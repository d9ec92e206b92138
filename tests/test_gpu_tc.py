"""The tcgen05 engine of the mat-vec (split-TF32 operands, FP32 accumulation in tensor memory) against the reference's
golden mat-vecs and the float32 SIMT engine, on every 2-D case; one batched call equals per-lattice calls."""
import numpy as np
import pytest
import torch

from conftest import golden
from golden_cases import MATVEC_SPECS, MATVEC_COMPLEX

pytestmark = pytest.mark.gpu

CASES_2D = [n for n, (shape, _, _) in MATVEC_SPECS.items() if len(shape) == 2 and shape[-1] % 4 == 0]


def _plans(name, engine):
    from blml_b200 import operator as op_mod, _lib
    from blml_b200.spec import parse_modes
    shape, modes, h = MATVEC_SPECS[name]
    specs, _ = parse_modes(modes, 2)
    hv = np.full(2, h)
    pad = op_mod.pad_rule(shape, hv, specs)
    return [op_mod.Plan(*op_mod.mode_transform(sp, shape, hv, pad), shape, _lib.F32, engine) for sp in specs]


@pytest.mark.parametrize('name', CASES_2D)
def test_tc_matvec_matches_reference(cuda_device, name):
    from blml_b200 import _lib
    g = golden('matvec.npz')[name]
    cplx = name in MATVEC_COMPLEX
    st = torch.cuda.current_stream().cuda_stream
    for k, plan in enumerate(_plans(name, _lib.ENGINE_TC)):
        x = torch.as_tensor(g['E'][k]).to(cuda_device, torch.complex64 if cplx else torch.float32).contiguous()
        y = torch.full_like(x, float('nan'))
        plan.apply(x, y, 1, cplx, st)
        _lib.call('blml_plan_status', plan._h)
        ref = g['U'][k]
        err = np.abs(y.cpu().numpy().astype(ref.dtype) - ref).max() / np.abs(ref).max()
        assert err <= 1e-5, (name, k, err)


def test_tc_batched_equals_single(cuda_device):
    from blml_b200 import _lib
    plan = _plans('d2_pball64', _lib.ENGINE_TC)[0]
    x = torch.randn(5, 64, 64, dtype=torch.complex64, device=cuda_device)
    y = torch.empty_like(x); y1 = torch.empty_like(x)
    st = torch.cuda.current_stream().cuda_stream
    plan.apply(x, y, 5, True, st)
    for b in range(5):
        plan.apply(x[b], y1[b], 1, True, st)
    _lib.call('blml_plan_status', plan._h)
    assert torch.equal(y, y1)


def test_tc_matches_simt_at_256(cuda_device):
    """The bench workload's signal mode (256 x 256 torus, pball fc 0.33) on both float32 engines."""
    from blml_b200 import operator as op_mod, _lib, workloads
    from blml_b200.spec import parse_modes
    specs, _ = parse_modes(workloads.pball_modes((256, 256), 0.33), 2)
    args = op_mod.mode_transform(specs[0], (256, 256), np.ones(2), (256, 256))
    tc = op_mod.Plan(*args, (256, 256), _lib.F32, _lib.ENGINE_TC)
    simt64 = op_mod.Plan(*args, (256, 256), _lib.F64, _lib.ENGINE_SIMT)
    x = torch.randn(2, 256, 256, dtype=torch.complex128, device=cuda_device)
    y64 = torch.empty_like(x); y = torch.empty(2, 256, 256, dtype=torch.complex64, device=cuda_device)
    st = torch.cuda.current_stream().cuda_stream
    simt64.apply(x, y64, 2, True, st)
    tc.apply(x.to(torch.complex64), y, 2, True, st)
    _lib.call('blml_plan_status', tc._h)
    err = (y.to(torch.complex128) - y64).abs().max().item() / y64.abs().max().item()
    assert err <= 3e-5, err          # split-TF32 products, FP32 accumulation over K = 512: measured 1.2e-5


def test_tc_fit_matches_float64(cuda_device):
    """A whole complex pball fit with the tensor-core mat-vec lands on the float64 fit's likelihood."""
    from blml_b200.binned import BLMLBinned
    from blml_b200 import workloads
    counts = workloads.two_disk_field((64, 64), fc=0.33, N=2e5, seed=3)
    modes = workloads.pball_modes((64, 64), 0.33)
    m64 = BLMLBinned(tol=1e-6, solver='lbfgs', dtype=np.float64).fit(counts, modes, complex_g=True)
    mtc = BLMLBinned(tol=1e-6, solver='lbfgs', dtype=np.float32, matvec_engine='tc').fit(counts, modes, complex_g=True)
    assert abs(mtc.loglik_ - m64.loglik_) <= 5e-5 * abs(m64.loglik_)     # the float32-state floor (test_gpu_binned)
