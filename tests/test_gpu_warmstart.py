"""The learned warm start on the GPU: the tcgen05 BF16 GEMM against an FP32 product of the same BF16 operands, the
network's forward pass and every parameter gradient against the float64 CPU oracle (oracle/unet_oracle.py, itself
pinned by finite differences) at BF16 accuracy, and a short training run that lowers the loss and whose starts
converge."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize('M,N,K,splits', [(128, 32, 72, 1), (300, 64, 200, 1), (1000, 256, 864, 1),
                                          (64, 300, 512, 3), (32, 2304, 4096, 7), (513, 16, 8, 1),
                                          (200, 48, 512, 7), (262144 // 16, 288, 864, 1)])
def test_gemm_bf16_matches_fp32_product(cuda_device, M, N, K, splits):
    from blml_b200._lib import call
    g = torch.Generator(device='cuda').manual_seed(M + N + K)
    A = torch.randn(M, K, device='cuda', generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device='cuda', generator=g).to(torch.bfloat16)
    C = torch.empty(splits, M, N, device='cuda')
    err = torch.zeros(1, dtype=torch.int32, device='cuda')
    call('blml_nn_gemm_bf16', A.data_ptr(), B.data_ptr(), C.data_ptr(), M, N, K, splits, err.data_ptr(),
         torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    ref = A.double() @ B.double().T
    got = C.double().sum(0)
    assert (got - ref).abs().max().item() <= 1e-5 * ref.abs().max().item() + 1e-6


def _bf16(a):
    return torch.as_tensor(np.asarray(a, np.float32)).to(torch.bfloat16).float().double().numpy()


def test_forward_and_gradients_match_oracle(cuda_device):
    import unet_oracle as uo
    from blml_b200.warmstart import WarmStartNet
    rng = np.random.default_rng(0)
    p = uo.init_params(3)
    for k in p:
        if k.endswith('.b'):
            p[k] = 0.05 * rng.standard_normal(p[k].shape)
    N, H, W = 2, 16, 16
    x = rng.standard_normal((N, H, W, 8)); t = rng.standard_normal((N, H, W, 2))
    net = WarmStartNet(params=p)
    xb = torch.as_tensor(x, dtype=torch.float32).to('cuda', torch.bfloat16)
    u = net.forward(xb, N, H, W)
    ls, du = net.loss(u, torch.as_tensor(t, dtype=torch.float32, device='cuda'))
    net.backward(du)
    torch.cuda.synchronize(); net.check()
    # the oracle on the same BF16-rounded weights and input (convolution weights are BF16 on the GPU)
    po = {k: (_bf16(v) if k.endswith('.w') and not k.startswith('head') else np.asarray(v, np.float32).astype(float))
          for k, v in p.items()}
    # the oracle rounds every stored activation and the ReLU-masked gradient the GEMMs take to BF16, as the GPU does,
    # so what remains is FP32 (GPU) against FP64 (oracle) accumulation
    uo_, c = uo.forward(po, uo.bf16(x), store=uo.bf16)
    lo, duo = uo.loss(uo_, t)
    go = uo.backward(po, c, duo)
    ug = u.double().cpu().numpy()
    assert np.linalg.norm(ug - uo_) <= 1e-2 * np.linalg.norm(uo_), np.linalg.norm(ug - uo_) / np.linalg.norm(uo_)
    assert np.allclose(ls.cpu().numpy(), lo, rtol=1e-2)
    worst = {}
    for k in go:
        gg = net.g[k].double().cpu().numpy().reshape(go[k].shape)
        worst[k] = np.linalg.norm(gg - go[k]) / max(np.linalg.norm(go[k]), 1e-30)
    assert max(worst.values()) <= 2e-2, worst


@pytest.mark.timeout(600)
def test_short_training_lowers_loss_and_starts_converge(cuda_device):
    from blml_b200 import workloads
    from blml_b200.sweep import BLMLBinnedBatch
    from blml_b200.warmstart import WarmStartNet, make_training_set
    fits = workloads.warm_start_set(48, seed=100, shape=(32, 32))
    b = BLMLBinnedBatch(tol=1e-5, dtype=np.float64, max_sweeps=5000)
    b.fit([f['counts'] for f in fits], [f['modes'] for f in fits])
    data = make_training_set(fits, [b.field(i) for i in range(len(fits))])
    net = WarmStartNet(seed=1)
    hist = net.train(data, epochs=6, batch=8, lr=1e-3)
    assert hist[-1] < hist[0], hist
    test = workloads.warm_start_set(8, seed=900, shape=(32, 32))
    E0 = net.start([f['counts'] for f in test], [f['fc'] for f in test], [f['kind'] for f in test])
    res = BLMLBinnedBatch(tol=1e-5, dtype=np.float64, max_sweeps=5000).fit(
        [f['counts'] for f in test], [f['modes'] for f in test], init=E0)
    net.check()
    assert all(np.isfinite(r.loglik_) and r.start_sweeps_ == 0 for r in res)
