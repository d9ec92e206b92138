"""CPU oracle of the warm-start network (TEST INFRASTRUCTURE ONLY: the GPU path never calls this).

A float64 NumPy restatement of the U-Net the warm start trains (blml_b200/warmstart.py runs it with the kernels of
csrc/unet.cu): NHWC activations, 3 x 3 convolutions with padding 1 written as im2col products with the weight layout
[Cout, (ky 3 + kx) Cin + c], ReLU, 2 x 2 average pooling, nearest x2 upsampling with the skip concatenated after the
upsampled channels, a 1 x 1 head to 2 channels (re, im), and the phase- and conjugation-invariant loss
    l_s = (|u|^2 + |t|^2 - 2 max(|<t, u>|, |<conj t, u>|)) / |t|^2,   mean over samples.
The network has no counterpart in the reference (its start is the real rank-1 solve, blml_binned.py:415-436); the
oracle pins the GPU forward / backward and is itself pinned by finite differences (tests/test_warmstart_oracle.py).
"""
import numpy as np

# (name, Cin, Cout) of the 3 x 3 convolutions in forward order
ARCH = [('enc1a', 8, 32), ('enc1b', 32, 32), ('enc2a', 32, 64), ('enc2b', 64, 64), ('enc3a', 64, 128),
        ('enc3b', 128, 128), ('bot1', 128, 256), ('bot2', 256, 256), ('dec3a', 384, 128), ('dec3b', 128, 128),
        ('dec2a', 192, 64), ('dec2b', 64, 64), ('dec1a', 96, 32), ('dec1b', 32, 32)]
HEAD = (32, 2)


def init_params(seed=0, scale=1.0):
    """He-normal convolution weights, zero biases, a small head (float64)."""
    rng = np.random.default_rng(seed)
    p = {}
    for name, ci, co in ARCH:
        p[name + '.w'] = rng.standard_normal((co, 9 * ci)) * np.sqrt(2.0 / (9 * ci)) * scale
        p[name + '.b'] = np.zeros(co)
    p['head.w'] = rng.standard_normal((HEAD[1], HEAD[0])) * np.sqrt(1.0 / HEAD[0]) * 0.1
    p['head.b'] = np.zeros(HEAD[1])
    return p


def im2col(x):
    """x (N, H, W, C) -> (N H W, 9 C), column (ky 3 + kx) C + c = x[n, y + ky - 1, x + kx - 1, c] (0 outside)."""
    N, H, W, C = x.shape
    xp = np.zeros((N, H + 2, W + 2, C), x.dtype)
    xp[:, 1:-1, 1:-1] = x
    cols = [xp[:, ky:ky + H, kx:kx + W] for ky in range(3) for kx in range(3)]
    return np.concatenate(cols, axis=3).reshape(N * H * W, 9 * C)


def col2im(dcol, shape):
    """The adjoint of im2col: (N H W, 9 C) -> (N, H, W, C)."""
    N, H, W, C = shape
    d = dcol.reshape(N, H, W, 9, C)
    dxp = np.zeros((N, H + 2, W + 2, C))
    for ky in range(3):
        for kx in range(3):
            dxp[:, ky:ky + H, kx:kx + W] += d[:, :, :, ky * 3 + kx]
    return dxp[:, 1:-1, 1:-1]


def conv(x, w, b):
    N, H, W, _ = x.shape
    return (im2col(x) @ w.T + b).reshape(N, H, W, -1)


def pool(x):
    N, H, W, C = x.shape
    return x.reshape(N, H // 2, 2, W // 2, 2, C).mean(axis=(2, 4))


def up(x):
    return x.repeat(2, axis=1).repeat(2, axis=2)


def bf16(a):
    """Round to the nearest BF16 value (ties to even), returned as float64: the storage rounding of the GPU path."""
    u = np.ascontiguousarray(a, np.float32).view(np.uint32)
    return (((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16).astype(np.uint32).view(np.float32).astype(np.float64)


def forward(p, x, store=None):
    """x (N, H, W, 8) -> (u (N, H, W, 2), cache). store: a rounding applied to every stored activation (bf16 to
    follow the GPU's BF16 activations exactly), identity by default."""
    st = store or (lambda v: v)
    c = {'x': x, 'store': store}
    r = lambda v: st(np.maximum(v, 0.0))
    h = x
    for lvl in (1, 2, 3):
        a = r(conv(h, p[f'enc{lvl}a.w'], p[f'enc{lvl}a.b'])); c[f'enc{lvl}a'] = a
        e = r(conv(a, p[f'enc{lvl}b.w'], p[f'enc{lvl}b.b'])); c[f'enc{lvl}b'] = e
        h = st(pool(e)); c[f'pool{lvl}'] = h
    b1 = r(conv(h, p['bot1.w'], p['bot1.b'])); c['bot1'] = b1
    h = r(conv(b1, p['bot2.w'], p['bot2.b'])); c['bot2'] = h
    for lvl in (3, 2, 1):
        cat = np.concatenate([up(h), c[f'enc{lvl}b']], axis=3); c[f'cat{lvl}'] = cat
        a = r(conv(cat, p[f'dec{lvl}a.w'], p[f'dec{lvl}a.b'])); c[f'dec{lvl}a'] = a
        h = r(conv(a, p[f'dec{lvl}b.w'], p[f'dec{lvl}b.b'])); c[f'dec{lvl}b'] = h
    u = h @ p['head.w'].T + p['head.b']
    return u, c


def loss(u, t):
    """Mean phase / conjugation-invariant loss and its gradient; u, t (N, H, W, 2) as (re, im)."""
    uc = u[..., 0] + 1j * u[..., 1]; tc = t[..., 0] + 1j * t[..., 1]
    N = u.shape[0]
    ls, du = np.zeros(N), np.zeros_like(u)
    for s in range(N):
        us, ts = uc[s].ravel(), tc[s].ravel()
        a = np.sum(np.conj(ts) * us); b = np.sum(ts * us)
        tt = np.sum(np.abs(ts) ** 2); uu = np.sum(np.abs(us) ** 2)
        cj = abs(b) > abs(a)
        m = abs(b) if cj else abs(a)
        ph = (b if cj else a) / m if m > 0 else 1.0
        tp = np.conj(ts) if cj else ts
        ls[s] = (uu + tt - 2 * m) / tt
        g = (2.0 / (tt * N)) * (us - tp * ph)
        du[s, ..., 0] = g.real.reshape(u.shape[1:3]); du[s, ..., 1] = g.imag.reshape(u.shape[1:3])
    return ls, du


def backward(p, c, du):
    """Gradients of the parameters given du = dL/du."""
    g = {}
    N, H, W, _ = du.shape
    d1 = c['dec1b']
    g['head.w'] = du.reshape(-1, 2).T @ d1.reshape(-1, d1.shape[3])
    g['head.b'] = du.reshape(-1, 2).sum(0)
    dh = du @ p['head.w']

    st = c.get('store') or (lambda v: v)

    def conv_bwd(name, x, y, dy, need_dx=True):
        dpre = dy * (y > 0)
        g[name + '.b'] = dpre.reshape(-1, dpre.shape[3]).sum(0)
        dpre = st(dpre)                                 # the GPU multiplies a BF16 copy
        g[name + '.w'] = dpre.reshape(-1, dpre.shape[3]).T @ im2col(x)
        if not need_dx:
            return None
        return col2im(dpre.reshape(-1, dpre.shape[3]) @ p[name + '.w'], x.shape)

    dskip = {}
    for lvl in (1, 2, 3):
        da = conv_bwd(f'dec{lvl}b', c[f'dec{lvl}a'], c[f'dec{lvl}b'], dh)
        dcat = conv_bwd(f'dec{lvl}a', c[f'cat{lvl}'], c[f'dec{lvl}a'], da)
        cu = dcat.shape[3] - c[f'enc{lvl}b'].shape[3]
        dskip[lvl] = dcat[..., cu:]
        dup = dcat[..., :cu]
        n_, h2, w2, cc = dup.shape
        dh = dup.reshape(n_, h2 // 2, 2, w2 // 2, 2, cc).sum(axis=(2, 4))
    db1 = conv_bwd('bot2', c['bot1'], c['bot2'], dh)
    dp = conv_bwd('bot1', c['pool3'], c['bot1'], db1)
    for lvl in (3, 2, 1):
        de = dskip[lvl] + 0.25 * up(dp)
        da = conv_bwd(f'enc{lvl}b', c[f'enc{lvl}a'], c[f'enc{lvl}b'], de)
        x_in = c[f'pool{lvl - 1}'] if lvl > 1 else c['x']
        dp = conv_bwd(f'enc{lvl}a', x_in, c[f'enc{lvl}a'], da, need_dx=lvl > 1)
    return g
