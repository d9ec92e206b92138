"""The CPU oracle of the warm-start network pinned by finite differences: its backward pass (convolutions through
im2col, ReLU, pooling, upsampling with skips, the 1 x 1 head) and the phase / conjugation-invariant loss give the
gradient of the loss to 1e-6 relative on sampled parameters of every layer; the loss is invariant to a global phase
and to conjugation of the target."""
import numpy as np
import pytest

import unet_oracle as uo


def _setup(seed=0, N=2, H=16, W=16):
    rng = np.random.default_rng(seed)
    p = uo.init_params(seed)
    for k in p:
        if k.endswith('.b'):
            p[k] = 0.05 * rng.standard_normal(p[k].shape)
    x = rng.standard_normal((N, H, W, 8))
    t = rng.standard_normal((N, H, W, 2))
    return p, x, t


def _loss(p, x, t):
    u, _ = uo.forward(p, x)
    return uo.loss(u, t)[0].mean()


def test_loss_invariances():
    rng = np.random.default_rng(1)
    u = rng.standard_normal((2, 8, 8, 2)); t = rng.standard_normal((2, 8, 8, 2))
    tc = t[..., 0] + 1j * t[..., 1]
    base = uo.loss(u, t)[0]
    rot = tc * np.exp(0.7j)
    assert np.allclose(uo.loss(u, np.stack([rot.real, rot.imag], -1))[0], base, rtol=1e-12)
    cj = np.conj(tc)
    assert np.allclose(uo.loss(u, np.stack([cj.real, cj.imag], -1))[0], base, rtol=1e-12)
    assert np.allclose(uo.loss(t, t)[0], 0.0, atol=1e-12)


@pytest.mark.parametrize('name', ['enc1a.w', 'enc2b.w', 'enc3a.b', 'bot1.w', 'bot2.w', 'dec3a.w', 'dec2a.b',
                                  'dec1a.w', 'dec1b.w', 'head.w', 'head.b'])
def test_oracle_gradient_matches_finite_differences(name):
    p, x, t = _setup()
    u, c = uo.forward(p, x)
    _, du = uo.loss(u, t)
    g = uo.backward(p, c, du)
    rng = np.random.default_rng(abs(hash(name)) % 2 ** 32)
    flat = p[name].reshape(-1)
    idx = rng.choice(flat.size, size=min(4, flat.size), replace=False)
    for i in idx:
        h = 1e-6 * max(1.0, abs(flat[i]))
        old = flat[i]
        flat[i] = old + h; lp = _loss(p, x, t)
        flat[i] = old - h; lm = _loss(p, x, t)
        flat[i] = old
        fd = (lp - lm) / (2 * h)
        an = g[name].reshape(-1)[i]
        assert abs(fd - an) <= 1e-6 * max(1.0, abs(fd)) + 1e-5 * abs(fd), (name, i, fd, an)
