"""CPU oracle of BLMLQuick's real rank-1 solver on occupied bins (TEST INFRASTRUCTURE ONLY: the product path never
calls this): the block coordinate descent of rahuljhu/band-limited-ml blml_trivial.py:2860-3035 (cd_root :84-89,
cd_line_search :92-104) in float64 NumPy on the dense Gram of the bins (the oracle's unit formulas at lattice
differences), with the block size the GPU solver uses, min(1024, max(32, B / 64)). Pinned by tests/golden/points.npz
(the reference's own point fits)."""
import numpy as np

from blml_oracle import parse_modes, units_of, unit_value


def gram(Z, h, modes):
    """The Gram of the bins Z (centres) on the lattice h under the first mode's product kernel."""
    sp = parse_modes(modes, Z.shape[1])[0]
    Zi = np.round(Z / h)
    G = np.ones((len(Z), len(Z)))
    for kind, dims in units_of(sp['kinds']):
        G *= unit_value(kind, sp['fc'][dims], [sp['periods'][j] for j in dims],
                        [(Zi[:, None, j] - Zi[None, :, j]) * h[j] for j in dims])
    return G


def cd_root(b, cc, sbb):
    disc = np.sqrt(b * b + 4.0 * sbb * cc)
    return np.where(b >= 0, 2.0 * cc / np.maximum(b + disc, 1e-300), (-b + disc) / (2.0 * sbb))


def line_search(e, d, lin, quad, cc, steps):
    pos = e > 0
    if not pos.any():
        return 1.0
    r = np.where(pos, d / np.where(pos, e, 1.0), 0.0)
    with np.errstate(invalid='ignore', divide='ignore'):
        logs = np.log1p(steps[:, None] * r[None, :]) @ np.where(pos, cc, 0.0)
    ok = (steps * lin + 0.5 * steps ** 2 * quad - logs <= 0) & np.all(1 + steps[:, None] * r[None, :] > 0, axis=1)
    return float(steps[np.argmax(ok)]) if ok.any() else 0.0


def block_cd(G, w, tol=1e-8, seed=0, max_sweeps=None):
    """(e, sweeps, converged, max|rho|) of (S e)_b e_b = n w_b by block CD from e = sqrt(n w / S_bb)."""
    B = len(w)
    n = float(w.sum())
    c = n * w
    sbb = float(G[0, 0])
    Bs = min(1024, max(32, B // 64), B)
    rng = np.random.default_rng(seed)
    steps = 0.5 ** np.arange(31)
    e = np.sqrt(c / sbb)
    Se = G @ e
    phi = lambda e, Se: (0.5 * e @ Se - c @ np.log(np.maximum(e, 1e-300))) / n
    resid = lambda e, Se: float(np.max(np.abs(Se * e / c - 1.0)))

    def sweep(e, Se, safeguard):
        perm = rng.permutation(B)
        for s0 in range(0, B, Bs):
            I = perm[s0:s0 + Bs]
            d = cd_root(Se[I] - sbb * e[I], c[I], sbb) - e[I]
            v = G[:, I] @ d
            t = line_search(e[I], d, d @ Se[I], d @ v[I], c[I], steps) if safeguard else 1.0
            e[I] += t * d
            Se += t * v

    safeguard, prev, hist, it, conv = False, phi(e, Se), [], 0, False
    while max_sweeps is None or it < max_sweeps:
        it += 1
        es, Ss = e.copy(), Se.copy()
        sweep(e, Se, safeguard)
        now = phi(e, Se)
        if not safeguard and now > prev + 1e-10 * abs(prev):
            e, Se = es, Ss
            safeguard = True
            sweep(e, Se, True)
            now = phi(e, Se)
        prev = now
        r = resid(e, Se)
        if r < tol:
            Se = G @ e
            r = resid(e, Se)
        hist.append(r)
        if r < tol:
            conv = True
            break
        if len(hist) > 50 and hist[-1] > 0.99 * min(hist[:-50]):
            break
    return e, it, conv, hist[-1]
