"""CPU oracle of the fc gradients of a binned fit (TEST INFRASTRUCTURE ONLY: the product path never calls this).

A float64 NumPy restatement of rahuljhu/band-limited-ml blml_binned.py:520-628 on the oracle's FFT operator
(blml_oracle.Operator):

  * dK/dlog fc tables   one per scale unit, the unit's value replaced by its dlog form (blml_binned.py:92-101;
                        sinc f cos(pi f t), slits f cos(pi f t) - fi cos(pi fi t), ball prod fc (D p(s) + s p'(s)):
                        blml_trivial.py:372-377, 446-453, 593-600, 146-154); integer units (dirichlet, pball): None
  * param_grad          d/dlog fc_u of sum m log(F / Z + eps) / sum m at fixed coefficients (:543-562); fc_grad is
                        param_grad(w) (:520-527)
  * implicit_grad       the same with the coefficients' refit response: one CG solve H v = dP/de on the occupied
                        bins, H the Hessian of the minimised objective (:565-628, _icg :1485-1496)

Pinned by tests/golden/grads.npz (tests/golden/make_grad_golden.py runs the reference's own methods at its own
fitted coefficients).
"""
import numpy as np

from blml_oracle import ball_profile, split_kind, units_of, unit_value, rdot


def ball_profile_dlog(s, dg):
    """s p'(s) of the ball profile: -pi (1/2)^(dg/2) s^(1 - dg/2) J_{dg/2 + 1}(pi s), 0 at s = 0."""
    from scipy.special import jv
    s = np.asarray(s, float)
    out = np.zeros(s.shape)
    nz = s > 0
    out[nz] = -np.pi * 0.5 ** (dg / 2) * s[nz] ** (1 - dg / 2) * jv(dg / 2 + 1, np.pi * s[nz])
    return out


def unit_value_dlog(kind, fc, periods, diffs):
    """dK/dlog fc of one unit (its fc columns scaled together), or None for units whose fc moves in whole
    harmonics."""
    name, tag = split_kind(kind)
    if name == 'sinc':
        f = float(fc[0])
        return f * np.cos(np.pi * f * diffs[0])
    if name == 'slits':
        f = float(fc[0]); fi = (1.0 - float(tag)) * f
        return f * np.cos(np.pi * f * diffs[0]) - fi * np.cos(np.pi * fi * diffs[0])
    if name == 'ball':
        f = np.asarray(fc, float); D = len(f)
        s = np.sqrt(sum((fi * dk) ** 2 for fi, dk in zip(f, diffs)))
        return float(np.prod(f)) * (D * ball_profile(s, D) + ball_profile_dlog(s, D))
    if name in ('dirichlet', 'pball'):
        return None
    raise ValueError(f"unknown kernel kind {kind!r}")


def dK_spectra(spec, shape, h, pad):
    """rFFTs of dK/dlog fc_u on the padded lattice, one per unit (None: integer units)."""
    import scipy.fft as sfft
    d = len(shape)
    diffs, masks = [], []
    for j, (m, L) in enumerate(zip(shape, pad)):
        idx = np.arange(L)
        off = np.where(idx < (L + 1) // 2, idx, idx - L).astype(float)
        mk = np.ones(L) if L == m else (np.abs(off) <= m - 1).astype(float)
        sh = [1] * d; sh[j] = L
        diffs.append((off * h[j]).reshape(sh)); masks.append(mk.reshape(sh))
    units = units_of(spec['kinds'])
    out = []
    for u, (kind, dims) in enumerate(units):
        th = lambda kd, ds: (spec['fc'][ds], [spec['periods'][j] for j in ds], [diffs[j] for j in ds])
        if unit_value_dlog(kind, *th(kind, dims)) is None:
            out.append(None); continue
        T = 1.0
        for v, (kv, dv) in enumerate(units):
            fcv, per, dd = th(kv, dv)
            if v == u:
                T = T * unit_value_dlog(kv, fcv, per, dd)
            else:
                T = T * unit_value(kv, fcv, per, dd)
        for mk in masks:
            T = T * mk
        out.append(sfft.rfftn(np.broadcast_to(T, pad).astype(np.float64), s=pad))
    return out


def _apply(fit, Kf, e):
    import scipy.fft as sfft
    op = fit.op
    sl = tuple(slice(0, m) for m in op.shape)
    parts = [e.real, e.imag] if np.iscomplexobj(e) else [e]
    g = [sfft.irfftn(sfft.rfftn(p, s=op.pad) * Kf, s=op.pad)[sl] for p in parts]
    return g[0] + 1j * g[1] if len(g) == 2 else g[0]


def _dKf(fit):
    if getattr(fit, '_dKf', None) is None:
        fit._dKf = [dK_spectra(sp, fit.shape, fit.h, fit.op.pad) for sp in fit.specs]
    return fit._dKf


def param_grad(fit, counts, eps=0.0):
    """blml_binned.py:543-562: a list per mode of arrays (one entry per unit; NaN for integer units)."""
    E, U = fit.e_hat, fit.Se
    m = np.asarray(counts, float); M = float(m.sum())
    F = (np.abs(U) ** 2).sum(0); Z = rdot(E, U)
    wn = np.where(m > 0, m / np.maximum(F + eps * Z, 1e-300), 0.0)
    fz = float(np.sum(wn * F)) / M
    out = []
    for k, dks in enumerate(_dKf(fit)):
        gk = []
        for dKf in dks:
            if dKf is None:
                gk.append(np.nan); continue
            dU = _apply(fit, dKf, E[k])
            gk.append(2 * float(np.sum(wn * np.real(np.conj(U[k]) * dU))) / M - fz * rdot(E[k], dU) / Z)
        out.append(np.array(gk))
    return out


def fc_grad(fit):
    return param_grad(fit, fit.w)


def _icg(A, b, tol, maxit):
    x = np.zeros_like(b); r = b.copy(); p = r.copy(); rs = rdot(r, r); bn = np.sqrt(rs) or 1.0
    for it in range(1, maxit + 1):
        Ap = A(p); pAp = rdot(p, Ap)
        if not pAp > 0:
            return x, it, np.sqrt(rs) / bn
        a = rs / pAp; x = x + a * p; r = r - a * Ap; rs_new = rdot(r, r)
        if np.sqrt(rs_new) / bn < tol:
            return x, it, np.sqrt(rs_new) / bn
        p = r + (rs_new / rs) * p; rs = rs_new
    return x, maxit, np.sqrt(rs) / bn


def implicit_grad(fit, counts, eps=0.0, tol=1e-6, maxit=300):
    """blml_binned.py:565-628; returns (G, CG iterations, CG relative residual)."""
    G = param_grad(fit, counts, eps)
    E, U, w, n, occ = fit.e_hat, fit.Se, fit.w, fit.n, fit.occ
    F = (np.abs(U) ** 2).sum(0); Q = rdot(E, U); Fs = np.where(occ, F, 1.0)
    m = np.asarray(counts, float); M = float(m.sum())
    wn = m / np.maximum(F + eps * Q, 1e-300); fz = float(np.sum(wn * F)) / M
    b = 2 * fit.Sall((wn / M)[None] * U) - fz * 2 * U / Q
    mask = occ[None].astype(float)

    def hvp(D):
        dU = fit.Sall(D)
        if not fit.psd:
            return dU + np.where(occ, fit.c / np.where(occ, E[0] * E[0], 1.0), 0.0)[None] * D
        dF = 2 * np.real(np.conj(U) * dU).sum(0); dQ = 2 * rdot(U, D)
        inner = (w / Fs)[None] * dU - (w * dF / Fs ** 2)[None] * U
        return -2 * fit.Sall(np.where(occ[None], inner, 0)) + 2 * n * dU / Q - 2 * n * U * dQ / Q ** 2

    def mixed(k, dKf):
        dUk = _apply(fit, dKf, E[k])
        if not fit.psd:
            return dUk[None]
        dF = 2 * np.real(np.conj(U[k]) * dUk); dQ = rdot(E[k], dUk)
        ws = np.where(occ, w / Fs, 0.0); wd = np.where(occ, w * dF / Fs ** 2, 0.0)
        out = []
        for j in range(fit.K):
            t = -wd * U[j]
            if j == k:
                t = t + ws * dUk
            g = -2 * fit.op.S(j, t) - 2 * n * U[j] * dQ / Q ** 2
            if j == k:
                g = g - 2 * _apply(fit, dKf, ws * U[k]) + 2 * n * dUk / Q
            out.append(g)
        return np.stack(out)

    v, iters, res = _icg(lambda x: hvp(x) * mask, b * mask, tol, maxit)
    for k, dks in enumerate(_dKf(fit)):
        for u, dKf in enumerate(dks):
            if dKf is not None:
                G[k][u] -= rdot(v, mixed(k, dKf) * mask)
    return G, iters, res
