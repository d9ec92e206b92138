"""The learned warm start: a small convolutional U-Net maps (log counts, cut-off, kernel kind) on a lattice to the
field u = S e / n of the fit (|u|^2 is the density), trained on fits this engine produces; the fit then starts from
e0 = w / conj(u) on the occupied bins -- the stationarity condition e = (Q / n) (w / F) S e solved for e with the
predicted field -- and L-BFGS refines it to the same tolerance as a cold fit. The reference has no learned part: its
start is the real rank-1 solve with seeded phases (blml_binned.py:415-436), which a warm-started fit skips
(blml_binned.py:403-408 takes an `init`).

    net = WarmStartNet(device='cuda', seed=0)
    data = make_training_set(fits, batch)                  # the engine's fits of workloads.warm_start_set(...)
    net.train(data, epochs=20, batch=16, lr=1e-3)
    E0 = net.start(counts_list, fcs, kinds)               # one complex start per fit
    BLMLBinnedBatch(tol=1e-6).fit(counts_list, modes_list, init=E0)

The network (about 1.94e6 parameters): three encoder levels of two 3 x 3 convolutions + ReLU (32, 64, 128 channels)
with 2 x 2 average pooling, a 256-channel bottleneck, three decoder levels (nearest x2 upsampling, the skip
concatenated after the upsampled channels, two 3 x 3 convolutions + ReLU), a 1 x 1 head to (re, im). BF16 weights
and activations, FP32 accumulation, FP32 master weights and Adam state; every convolution is an im2col + tcgen05
GEMM of csrc/unet.cu, in forward and backward. Inputs: 8 channels per bin -- log1p(counts) / 8, 4 fc, the one-hot
kernel kind (pball, slits), log10(n) / 6, zeros. Lattice sides must be multiples of 8. The loss is the phase- and
conjugation-invariant distance of csrc/unet.cu (a fit's field is defined up to a global phase and conjugation)."""
import ctypes as C

import numpy as np
import torch

from . import _lib
from ._lib import call

ARCH = [('enc1a', 8, 32), ('enc1b', 32, 32), ('enc2a', 32, 64), ('enc2b', 64, 64), ('enc3a', 64, 128),
        ('enc3b', 128, 128), ('bot1', 128, 256), ('bot2', 256, 256), ('dec3a', 384, 128), ('dec3b', 128, 128),
        ('dec2a', 192, 64), ('dec2b', 64, 64), ('dec1a', 96, 32), ('dec1b', 32, 32)]
HEAD = (32, 2)
IN_CH = 8
KINDS = ('pball', 'slits')


def init_params(seed=0):
    """He-normal convolution weights, zero biases, a small head (float64 NumPy, [Cout, 9 Cin] layout)."""
    rng = np.random.default_rng(seed)
    p = {}
    for name, ci, co in ARCH:
        p[name + '.w'] = rng.standard_normal((co, 9 * ci)) * np.sqrt(2.0 / (9 * ci))
        p[name + '.b'] = np.zeros(co)
    p['head.w'] = rng.standard_normal((HEAD[1], HEAD[0])) * np.sqrt(1.0 / HEAD[0]) * 0.1
    p['head.b'] = np.zeros(HEAD[1])
    return p


def features(counts_list, fcs, kinds):
    """(N, H, W, 8) float32 inputs of the network (host NumPy)."""
    N = len(counts_list); H, W = np.shape(counts_list[0])
    x = np.zeros((N, H, W, IN_CH), np.float32)
    for s, (c, fc, kind) in enumerate(zip(counts_list, fcs, kinds)):
        c = np.asarray(c, float)
        if c.shape != (H, W):
            raise ValueError("features: one lattice shape per call")
        x[s, :, :, 0] = np.log1p(c) / 8.0
        x[s, :, :, 1] = 4.0 * fc
        x[s, :, :, 2 + KINDS.index(kind)] = 1.0
        x[s, :, :, 4] = np.log10(max(c.sum(), 1.0)) / 6.0
    return x


class WarmStartNet:
    """The U-Net on one GPU (see the module docstring)."""

    def __init__(self, device='cuda', seed=0, params=None):
        if not torch.cuda.is_available():
            raise _lib.BLMLError('WarmStartNet needs a CUDA device (no CPU path)')
        self.device = torch.device(device)
        p = init_params(seed) if params is None else params
        f32 = dict(dtype=torch.float32, device=self.device)
        self.p = {k: torch.as_tensor(np.asarray(v, np.float32)).to(self.device).contiguous() for k, v in p.items()}
        self.g = {k: torch.zeros_like(v) for k, v in self.p.items()}
        self.m = {k: torch.zeros_like(v) for k, v in self.p.items()}
        self.v = {k: torch.zeros_like(v) for k, v in self.p.items()}
        self.wb, self.wbt = {}, {}
        for name, ci, co in ARCH:
            self.wb[name] = torch.empty(co * 9 * ci, dtype=torch.bfloat16, device=self.device)
            self.wbt[name] = torch.empty(co * 9 * ci, dtype=torch.bfloat16, device=self.device)
        self.err = torch.zeros(1, dtype=torch.int32, device=self.device)
        self.gw_head = torch.zeros(HEAD[1] * (HEAD[0] + 1), **f32)
        self.ws, self.acts = {}, {}
        self.step_ = 0
        self._sync_bf16()

    # ---------------------------------------------------------------- buffers
    @property
    def st(self):
        return torch.cuda.current_stream(self.device).cuda_stream

    def _ws(self, key, n, dtype):
        t = self.ws.get(key)
        if t is None or t.numel() < n or t.dtype != dtype:
            t = torch.empty(max(int(n), 1), dtype=dtype, device=self.device)
            self.ws[key] = t
        return t

    def _act(self, key, n, dtype=torch.bfloat16):
        return self._ws('act.' + key, n, dtype)

    def _sync_bf16(self):
        for name, ci, co in ARCH:
            call('blml_nn_to_bf16', self.p[name + '.w'].data_ptr(), co * 9 * ci, self.wb[name].data_ptr(),
                 self.wbt[name].data_ptr(), co, 9 * ci, self.st)

    def params_numpy(self):
        return {k: v.detach().cpu().numpy().astype(np.float64) for k, v in self.p.items()}

    # ---------------------------------------------------------------- layers
    def _conv(self, name, X, Y, N, H, W, relu=True):
        """Y slice = act(conv3x3(X slice)); X, Y = (tensor, channel stride, offset, channels)."""
        xt, xcs, xc0, ci = X; yt, ycs, yc0, co = Y
        P = N * H * W; K9 = 9 * ci
        col = self._ws('col', P * K9, torch.bfloat16)
        call('blml_nn_im2col', xt.data_ptr(), N, H, W, xcs, xc0, ci, col.data_ptr(), 0, self.st)
        Cm = self._ws('C', P * co, torch.float32)
        call('blml_nn_gemm_bf16', col.data_ptr(), self.wb[name].data_ptr(), Cm.data_ptr(), P, co, K9, 1,
             self.err.data_ptr(), self.st)
        call('blml_nn_bias_act', Cm.data_ptr(), 1, P, co, self.p[name + '.b'].data_ptr(), int(relu), yt.data_ptr(),
             ycs, yc0, self.st)

    def _conv_bwd(self, name, X, Y, dY, dX, N, H, W):
        """Gradients of a conv + ReLU layer: weights and bias into self.g, the input's gradient into the dX slice
        (overwritten) unless dX is None. dY, dX = (tensor, channel stride, offset)."""
        xt, xcs, xc0, ci = X; yt, ycs, yc0, co = Y
        P = N * H * W; K9 = 9 * ci
        dpre = self._ws('dpre', P * co, torch.bfloat16); dpreT = self._ws('dpreT', P * co, torch.bfloat16)
        call('blml_nn_relu_bwd', dY[0].data_ptr(), dY[1], dY[2], yt.data_ptr(), ycs, yc0, P, co, dpre.data_ptr(),
             dpreT.data_ptr(), self.st)
        chunks = int(min(2048, max(1, P // 256)))     # ~256 rows per block
        part = self._ws('bpart', chunks * co, torch.float32)
        call('blml_nn_bias_grad', dY[0].data_ptr(), dY[1], dY[2], yt.data_ptr(), ycs, yc0, P, co, 1, chunks,
             part.data_ptr(), self.g[name + '.b'].data_ptr(), self.st)
        colT = self._ws('col', P * K9, torch.bfloat16)
        call('blml_nn_im2col', xt.data_ptr(), N, H, W, xcs, xc0, ci, colT.data_ptr(), 1, self.st)
        mt = (co + 127) // 128; nt = (K9 + 255) // 256; nkb = (P + 63) // 64
        splits = int(max(1, min(nkb, -(-296 // (mt * nt)))))
        Cp = self._ws('Cp', splits * co * K9, torch.float32)
        call('blml_nn_gemm_bf16', dpreT.data_ptr(), colT.data_ptr(), Cp.data_ptr(), co, K9, P, splits,
             self.err.data_ptr(), self.st)
        call('blml_nn_sum_splits', Cp.data_ptr(), splits, co * K9, self.g[name + '.w'].data_ptr(), self.st)
        if dX is not None:
            dcol = self._ws('dcol', P * K9, torch.float32)
            call('blml_nn_gemm_bf16', dpre.data_ptr(), self.wbt[name].data_ptr(), dcol.data_ptr(), P, K9, co, 1,
                 self.err.data_ptr(), self.st)
            call('blml_nn_col2im', dcol.data_ptr(), N, H, W, ci, dX[0].data_ptr(), dX[1], dX[2], self.st)

    # ---------------------------------------------------------------- forward / backward
    def forward(self, x, N, H, W):
        """x: BF16 (N, H, W, 8) on the device -> u FP32 (N, H, W, 2); keeps the activations for backward."""
        if H % 8 or W % 8:
            raise ValueError("WarmStartNet: lattice sides must be multiples of 8")
        self.shape_ = (N, H, W)
        P1, P2, P3, P4 = N * H * W, N * H * W // 4, N * H * W // 16, N * H * W // 64
        H2, W2, H4, W4, H8, W8 = H // 2, W // 2, H // 4, W // 4, H // 8, W // 8
        A = {k: self._act(k, n) for k, n in dict(a1=P1 * 32, cat1=P1 * 96, p1=P2 * 32, a2=P2 * 64, cat2=P2 * 192,
                                                   p2=P3 * 64, a3=P3 * 128, cat3=P3 * 384, p3=P4 * 128, b1=P4 * 256,
                                                   b2=P4 * 256, d3a=P3 * 128, d3=P3 * 128, d2a=P2 * 64, d2=P2 * 64,
                                                   d1a=P1 * 32, d1=P1 * 32).items()}
        A['x'] = x
        self.A = A
        st = self.st
        self._conv('enc1a', (x, 8, 0, 8), (A['a1'], 32, 0, 32), N, H, W)
        self._conv('enc1b', (A['a1'], 32, 0, 32), (A['cat1'], 96, 64, 32), N, H, W)
        call('blml_nn_pool_fwd', A['cat1'].data_ptr(), N, H, W, 96, 64, 32, A['p1'].data_ptr(), 32, 0, st)
        self._conv('enc2a', (A['p1'], 32, 0, 32), (A['a2'], 64, 0, 64), N, H2, W2)
        self._conv('enc2b', (A['a2'], 64, 0, 64), (A['cat2'], 192, 128, 64), N, H2, W2)
        call('blml_nn_pool_fwd', A['cat2'].data_ptr(), N, H2, W2, 192, 128, 64, A['p2'].data_ptr(), 64, 0, st)
        self._conv('enc3a', (A['p2'], 64, 0, 64), (A['a3'], 128, 0, 128), N, H4, W4)
        self._conv('enc3b', (A['a3'], 128, 0, 128), (A['cat3'], 384, 256, 128), N, H4, W4)
        call('blml_nn_pool_fwd', A['cat3'].data_ptr(), N, H4, W4, 384, 256, 128, A['p3'].data_ptr(), 128, 0, st)
        self._conv('bot1', (A['p3'], 128, 0, 128), (A['b1'], 256, 0, 256), N, H8, W8)
        self._conv('bot2', (A['b1'], 256, 0, 256), (A['b2'], 256, 0, 256), N, H8, W8)
        call('blml_nn_up_fwd', A['b2'].data_ptr(), N, H8, W8, 256, A['cat3'].data_ptr(), 384, 0, st)
        self._conv('dec3a', (A['cat3'], 384, 0, 384), (A['d3a'], 128, 0, 128), N, H4, W4)
        self._conv('dec3b', (A['d3a'], 128, 0, 128), (A['d3'], 128, 0, 128), N, H4, W4)
        call('blml_nn_up_fwd', A['d3'].data_ptr(), N, H4, W4, 128, A['cat2'].data_ptr(), 192, 0, st)
        self._conv('dec2a', (A['cat2'], 192, 0, 192), (A['d2a'], 64, 0, 64), N, H2, W2)
        self._conv('dec2b', (A['d2a'], 64, 0, 64), (A['d2'], 64, 0, 64), N, H2, W2)
        call('blml_nn_up_fwd', A['d2'].data_ptr(), N, H2, W2, 64, A['cat1'].data_ptr(), 96, 0, st)
        self._conv('dec1a', (A['cat1'], 96, 0, 96), (A['d1a'], 32, 0, 32), N, H, W)
        self._conv('dec1b', (A['d1a'], 32, 0, 32), (A['d1'], 32, 0, 32), N, H, W)
        u = self._act('u', P1 * 2, torch.float32)
        call('blml_nn_head_fwd', A['d1'].data_ptr(), P1, 32, self.p['head.w'].data_ptr(), self.p['head.b'].data_ptr(),
             2, u.data_ptr(), st)
        return u[:P1 * 2].view(N, H, W, 2)

    def backward(self, du):
        """Parameter gradients (self.g) from du = dL/du (FP32 (N, H, W, 2)) after forward."""
        N, H, W = self.shape_
        A, st = self.A, self.st
        P1, P2, P3, P4 = N * H * W, N * H * W // 4, N * H * W // 16, N * H * W // 64
        H2, W2, H4, W4, H8, W8 = H // 2, W // 2, H // 4, W // 4, H // 8, W // 8
        f = torch.float32
        D = {k: self._act('d' + k, n, f) for k, n in dict(d1=P1 * 32, d1a=P1 * 32, cat1=P1 * 96, d2=P2 * 64,
                                                           d2a=P2 * 64, cat2=P2 * 192, d3=P3 * 128, d3a=P3 * 128,
                                                           cat3=P3 * 384, b2=P4 * 256, b1=P4 * 256, p3=P4 * 128,
                                                           a3=P3 * 128, p2=P3 * 64, a2=P2 * 64, p1=P2 * 32,
                                                           a1=P1 * 32).items()}
        chunks = int(min(2048, max(1, P1 // 256)))
        part = self._ws('hpart', chunks * HEAD[1] * (HEAD[0] + 1), f)
        call('blml_nn_head_bwd', du.data_ptr(), A['d1'].data_ptr(), P1, 32, 2, self.p['head.w'].data_ptr(),
             D['d1'].data_ptr(), chunks, part.data_ptr(), self.gw_head.data_ptr(), st)
        gw = self.gw_head.view(HEAD[1], HEAD[0] + 1)
        self.g['head.w'].copy_(gw[:, :HEAD[0]]); self.g['head.b'].copy_(gw[:, HEAD[0]])
        cb = self._conv_bwd
        cb('dec1b', (A['d1a'], 32, 0, 32), (A['d1'], 32, 0, 32), (D['d1'], 32, 0), (D['d1a'], 32, 0), N, H, W)
        cb('dec1a', (A['cat1'], 96, 0, 96), (A['d1a'], 32, 0, 32), (D['d1a'], 32, 0), (D['cat1'], 96, 0), N, H, W)
        call('blml_nn_up_bwd', D['cat1'].data_ptr(), N, H2, W2, 96, 0, 64, D['d2'].data_ptr(), st)
        cb('dec2b', (A['d2a'], 64, 0, 64), (A['d2'], 64, 0, 64), (D['d2'], 64, 0), (D['d2a'], 64, 0), N, H2, W2)
        cb('dec2a', (A['cat2'], 192, 0, 192), (A['d2a'], 64, 0, 64), (D['d2a'], 64, 0), (D['cat2'], 192, 0),
           N, H2, W2)
        call('blml_nn_up_bwd', D['cat2'].data_ptr(), N, H4, W4, 192, 0, 128, D['d3'].data_ptr(), st)
        cb('dec3b', (A['d3a'], 128, 0, 128), (A['d3'], 128, 0, 128), (D['d3'], 128, 0), (D['d3a'], 128, 0),
           N, H4, W4)
        cb('dec3a', (A['cat3'], 384, 0, 384), (A['d3a'], 128, 0, 128), (D['d3a'], 128, 0), (D['cat3'], 384, 0),
           N, H4, W4)
        call('blml_nn_up_bwd', D['cat3'].data_ptr(), N, H8, W8, 384, 0, 256, D['b2'].data_ptr(), st)
        cb('bot2', (A['b1'], 256, 0, 256), (A['b2'], 256, 0, 256), (D['b2'], 256, 0), (D['b1'], 256, 0), N, H8, W8)
        cb('bot1', (A['p3'], 128, 0, 128), (A['b1'], 256, 0, 256), (D['b1'], 256, 0), (D['p3'], 128, 0), N, H8, W8)
        call('blml_nn_pool_bwd_add', D['p3'].data_ptr(), N, H4, W4, 128, D['cat3'].data_ptr(), 384, 256, st)
        cb('enc3b', (A['a3'], 128, 0, 128), (A['cat3'], 384, 256, 128), (D['cat3'], 384, 256), (D['a3'], 128, 0),
           N, H4, W4)
        cb('enc3a', (A['p2'], 64, 0, 64), (A['a3'], 128, 0, 128), (D['a3'], 128, 0), (D['p2'], 64, 0), N, H4, W4)
        call('blml_nn_pool_bwd_add', D['p2'].data_ptr(), N, H2, W2, 64, D['cat2'].data_ptr(), 192, 128, st)
        cb('enc2b', (A['a2'], 64, 0, 64), (A['cat2'], 192, 128, 64), (D['cat2'], 192, 128), (D['a2'], 64, 0),
           N, H2, W2)
        cb('enc2a', (A['p1'], 32, 0, 32), (A['a2'], 64, 0, 64), (D['a2'], 64, 0), (D['p1'], 32, 0), N, H2, W2)
        call('blml_nn_pool_bwd_add', D['p1'].data_ptr(), N, H, W, 32, D['cat1'].data_ptr(), 96, 64, st)
        cb('enc1b', (A['a1'], 32, 0, 32), (A['cat1'], 96, 64, 32), (D['cat1'], 96, 64), (D['a1'], 32, 0), N, H, W)
        cb('enc1a', (A['x'], 8, 0, 8), (A['a1'], 32, 0, 32), (D['a1'], 32, 0), None, N, H, W)

    def loss(self, u, t):
        """Per-sample loss (host) and du (device) for targets t (FP32 (N, H, W, 2))."""
        N, H, W = self.shape_
        stats = self._ws('stats', 6 * N, torch.float64); du = self._ws('du', N * H * W * 2, torch.float32)
        ls = self._ws('loss', N, torch.float64)
        call('blml_nn_phase_loss', u.data_ptr(), t.data_ptr(), H * W, N, stats.data_ptr(), du.data_ptr(),
             ls.data_ptr(), self.st)
        return ls[:N], du[:N * H * W * 2].view(N, H, W, 2)

    def adam(self, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
        self.step_ += 1
        for k, w in self.p.items():
            name = k.split('.')[0]
            conv_w = k.endswith('.w') and name in self.wb
            rows, cols = (w.shape[0], w.shape[1]) if conv_w else (0, 0)
            call('blml_nn_adam', w.data_ptr(), self.g[k].data_ptr(), self.m[k].data_ptr(), self.v[k].data_ptr(),
                 w.numel(), float(lr), float(b1), float(b2), float(eps), self.step_,
                 self.wb[name].data_ptr() if conv_w else None, self.wbt[name].data_ptr() if conv_w else None,
                 int(rows), int(cols), self.st)

    def check(self):
        """Raise when a tensor-core GEMM gave up on a bounded wait since the net was made."""
        if int(self.err.item()):
            raise _lib.BLMLError('warm-start GEMM: a bounded wait timed out (results invalid)')

    # ---------------------------------------------------------------- training and use
    def train(self, data, epochs=20, batch=16, lr=1e-3, seed=0, verbose=False):
        """data: dict(x BF16 (S, H, W, 8), t FP32 (S, H, W, 2)) on the device; returns the mean loss per epoch."""
        x, t = data['x'], data['t']
        S, H, W, _ = x.shape
        rng = np.random.default_rng(seed)
        hist = []
        for ep in range(epochs):
            order = rng.permutation(S)
            tot, nb = 0.0, 0
            lsum = torch.zeros((), dtype=torch.float64, device=self.device)
            for b0 in range(0, S - batch + 1, batch):
                idx = torch.as_tensor(order[b0:b0 + batch], device=self.device)
                xb = x.index_select(0, idx).contiguous(); tb = t.index_select(0, idx).contiguous()
                u = self.forward(xb, batch, H, W)
                ls, du = self.loss(u, tb)
                lsum += ls.sum()
                self.backward(du)
                self.adam(lr)
                nb += batch
            hist.append(float(lsum.item()) / max(nb, 1))
            self.check()
            if verbose:
                print(f'  warm-start epoch {ep}: loss {hist[-1]:.4f}', flush=True)
        return hist

    def predict(self, x, batch=16):
        """u (complex64, (S, H, W)) for BF16 inputs (S, H, W, 8): the head output / sqrt(H W)."""
        S, H, W, _ = x.shape
        out = torch.empty((S, H, W), dtype=torch.complex64, device=self.device)
        for b0 in range(0, S, batch):
            nb = min(batch, S - b0)
            u = self.forward(x[b0:b0 + nb].contiguous(), nb, H, W)
            out[b0:b0 + nb] = torch.view_as_complex(u.contiguous()) / float(np.sqrt(H * W))
        return out

    def start(self, counts_list, fcs, kinds, batch=16):
        """One complex start per fit: e0 = w / conj(u) on the occupied bins (w = counts), 0 elsewhere. Fits are
        grouped by lattice shape for the network."""
        out = [None] * len(counts_list)
        host = [c.detach().cpu().numpy() if isinstance(c, torch.Tensor) else np.asarray(c, float) for c in counts_list]
        by_shape = {}
        for i, c in enumerate(host):
            by_shape.setdefault(tuple(np.shape(c)), []).append(i)
        for shape, ids in by_shape.items():
            x = torch.as_tensor(features([host[i] for i in ids], [fcs[i] for i in ids],
                                         [kinds[i] for i in ids])).to(self.device, torch.bfloat16)
            u = self.predict(x, batch)
            for j, i in enumerate(ids):
                c = counts_list[i]
                w = (c if isinstance(c, torch.Tensor) else torch.as_tensor(host[i])).to(self.device, torch.float64)
                uc = u[j].to(torch.complex128)
                ok = (w > 0) & (uc.abs() > 0)
                e0 = torch.where(ok, w / torch.conj(torch.where(ok, uc, torch.ones_like(uc))), torch.zeros_like(uc))
                out[i] = e0
        return out


def make_training_set(fits, fields, device='cuda'):
    """Network inputs and targets from fits (workloads.warm_start_set entries) and their engine fields u (complex,
    from BLMLBinnedBatch.field): x BF16 (S, H, W, 8), t FP32 (S, H, W, 2) = u sqrt(H W) as (re, im)."""
    H, W = np.shape(fits[0]['counts'])
    x = torch.as_tensor(features([f['counts'] for f in fits], [f['fc'] for f in fits],
                                 [f['kind'] for f in fits])).to(device, torch.bfloat16)
    t = torch.stack([torch.view_as_real(u.to(torch.complex64)) for u in fields]).to(device) * float(np.sqrt(H * W))
    return dict(x=x, t=t.contiguous())
