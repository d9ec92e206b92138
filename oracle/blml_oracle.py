"""CPU oracle for the BLML binned fitting path -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may import this module, and only as the
checker (or the timed CPU baseline). The product (band-limited-ml_b200/blml_b200) never imports it.

A float64 NumPy/SciPy restatement of the reference's algorithm (rahuljhu/band-limited-ml, blml_binned.py and the
kernel classes of blml_trivial.py), written from its documented behaviour:

  * kernels        sinc / slits / dirichlet / pball / ball unit values       blml_trivial.py:335-720
  * mode spec      make_modes / parse_modes (the subset the binned path uses) blml_trivial.py:1247-1323, 1467-1505
  * operator       padded-lattice table, rFFT, S_k e = irfft(rfft(e) Kf)     blml_binned.py:49-101, 119-168
  * updates        Jacobi coordinate update, cd_root, secular root          blml_binned.py:184-206, 1549-1573
  * merit          merit / rescale / residual                                blml_binned.py:171-220
  * CD solver      Jacobi + Anderson + merit safeguard + damping/gradient    blml_binned.py:223-276, 357-380, 1463-1478
  * L-BFGS         two-loop recursion, Armijo, canonical form               blml_binned.py:278-355
  * start/finish   real rank-1 start, phases, density_/loglik_              blml_binned.py:383-445
  * certificate    lambda_max(D^1/2 S_0 D^1/2)/n via ARPACK                  blml_binned.py:501-518
  * certified fit  rank growth until the certificate is <= 1 + tol           no reference function: the fit with K
                                                                            shared modes and init=, :383-413

Parity pin: tests/golden/*.npz were produced by the reference itself (tests/golden/make_golden.py imports it
read-only) and tests/test_oracle_golden.py checks this module against them.
"""
import numpy as np

# ---------------------------------------------------------------------------------------------------- kernels


def dirichlet_N(fc, P):
    """Harmonics kept on a P-periodic column: floor(fc P / 2) (blml_trivial.py:80-82)."""
    return max(0, int(np.floor(fc * P / 2.0 + 1e-9)))


def dirichlet_inner_M(fc, P, fill):
    """2 Ni + 1 removed harmonics of a periodic two-slit band (blml_trivial.py:107-116)."""
    if fill is None or fill >= 1.0:
        return 0
    Ni = int(np.ceil((1.0 - fill) * fc * P / 2.0 - 1e-9)) - 1
    return max(2 * Ni + 1, 0)


def pball_harmonics(fc, periods):
    """Integer vectors k with sum (k_i / P_i)^2 <= (fc/2)^2, and the scale 1 / prod P (blml_trivial.py:632-639)."""
    P = np.atleast_1d(np.asarray(periods, float))
    R = float(fc) / 2.0
    N = [max(0, int(np.floor(R * p + 1e-9))) for p in P]
    grids = np.meshgrid(*[np.arange(-n, n + 1) for n in N], indexing='ij')
    Kv = np.stack([g.ravel() for g in grids], 1)
    inside = ((Kv / P) ** 2).sum(1) <= R * R * (1 + 1e-9) + 1e-12
    return Kv[inside], 1.0 / float(np.prod(P))


def ball_profile(s, dg):
    """FT of the ball |nu| <= 1/2 in dg dims at radius s (blml_trivial.py:145-154)."""
    from scipy.special import jv, gamma
    s = np.asarray(s, float)
    out = np.full(s.shape, np.pi ** (dg / 2) * 0.5 ** dg / gamma(dg / 2 + 1))
    nz = s > 0
    out[nz] = 0.5 ** (dg / 2) * jv(dg / 2, np.pi * s[nz]) / s[nz] ** (dg / 2)
    return out


def split_kind(kind):
    name, _, tag = str(kind).partition(':')
    return name, tag


def unit_value(kind, fc, periods, diffs):
    """K of one kernel unit at coordinate differences (one array per column of the unit).
    fc / periods: the unit's per-column values."""
    name, tag = split_kind(kind)
    if name == 'sinc':                                                        # blml_trivial.py:368-370
        f = float(fc[0])
        return f * np.sinc(f * diffs[0])
    if name == 'slits':                                                       # blml_trivial.py:442-444
        f = float(fc[0]); fi = (1.0 - float(tag)) * f
        return f * np.sinc(f * diffs[0]) - fi * np.sinc(fi * diffs[0])
    if name == 'dirichlet':                                                   # blml_trivial.py:528-535
        P, f = float(periods[0]), float(fc[0])
        fill = float(tag) if tag else None
        M = 2 * dirichlet_N(f, P) + 1
        Mi = dirichlet_inner_M(f, P, fill)
        t = np.mod(np.abs(diffs[0]), P); t = np.minimum(t, P - t)
        with np.errstate(divide='ignore', invalid='ignore'):
            v = (np.sin(np.pi * M * t / P) - np.sin(np.pi * Mi * t / P)) / np.sin(np.pi * t / P)
        return np.where(t < 1e-10, M - Mi, v) / P
    if name == 'pball':                                                       # blml_trivial.py:656-665
        P = np.asarray(periods, float)
        Kv, sc = pball_harmonics(float(fc[0]), P)
        ph = sum(np.multiply.outer(2 * np.pi * Kv[:, i] / P[i], np.asarray(diffs[i], float)) for i in range(len(P)))
        return sc * np.cos(ph).sum(0)
    if name == 'ball':                                                        # blml_trivial.py:690-694
        f = np.asarray(fc, float)
        s = np.sqrt(sum((fi * dk) ** 2 for fi, dk in zip(f, diffs)))
        return float(np.prod(f)) * ball_profile(s, len(f))
    raise ValueError(f"unknown kernel kind {kind!r}")


def is_group_kind(kind):
    return split_kind(kind)[0] in ('ball', 'pball')


def units_of(kinds):
    """[(kind, dims)]: one unit per one-column kind, then one per multi-column group in order of first appearance
    (blml_trivial.py:330-335, 238-250)."""
    units = [(k, [j]) for j, k in enumerate(kinds) if not is_group_kind(k)]
    groups = {}
    for j, k in enumerate(kinds):
        if is_group_kind(k):
            groups.setdefault(split_kind(k)[1], (split_kind(k)[0], []))[1].append(j)
    return units + [(nm, dims) for nm, dims in groups.values()]


# ---------------------------------------------------------------------------------------------------- mode spec

def make_modes(fc, kinds=None, periods=None, rank=1, d=None):
    """A modes list from per-dim settings (blml_trivial.py:1467-1505): fc scalar, (d,) or (K, d)."""
    F = np.asarray(fc, float)
    if d is None:
        d = len(kinds) if kinds is not None else F.shape[-1]
    F = F if F.ndim == 2 else np.broadcast_to(F, (d,))[None]
    F = np.broadcast_to(F, (int(rank) if len(F) == 1 else len(F), d))
    kinds = list(kinds) if kinds is not None else ['sinc'] * d
    groups = {}
    for j, k in enumerate(kinds):
        if is_group_kind(k):
            groups.setdefault(split_kind(k)[1], []).append(j)
    unit_of = {j: tuple(g) for g in groups.values() for j in g}
    modes = []
    for k in range(len(F)):
        m = {}
        for j in range(d):
            name, tag = split_kind(kinds[j])
            c = dict(kind=name)
            if name in ('slits', 'dirichlet') and tag:
                c['fill'] = float(tag)
            if np.isfinite(F[k, j]):
                c['fc'] = float(F[k, j])
            if name == 'dirichlet':
                c['period'] = periods[j]
            if j in unit_of:
                key = unit_of[j]
                if name == 'pball':
                    c['period'] = [periods[i] for i in key]
                if j == key[0]:
                    m[key] = c
            else:
                m[j] = c
        modes.append(m)
    return modes


def parse_modes(modes, d):
    """Per mode dict(fc (d,), kinds (d,), periods (d,)) in the internal form: group kinds carry the tag of their
    columns ('pball:0-1'), slits / dirichlet carry their fill (blml_trivial.py:1247-1323)."""
    if isinstance(modes, dict) or not isinstance(modes, (list, tuple)) or not modes:
        raise TypeError("modes: a non-empty list of mode dicts")
    specs = []
    for m in modes:
        fc = [np.nan] * d; kinds = [None] * d; periods = [None] * d
        for key, c in m.items():
            kind = c.get('kind', 'sinc')
            fcv = c.get('fc'); fcv = fcv['value'] if isinstance(fcv, dict) else fcv
            per = c.get('period'); per = per['value'] if isinstance(per, dict) else per
            if isinstance(key, tuple):
                tag = '-'.join(map(str, key))
                for i, j in enumerate(key):
                    kinds[j] = f'{kind}:{tag}'
                    fc[j] = float(fcv)
                    periods[j] = None if per is None else float(per[i])
            else:
                fill = c.get('fill')
                kinds[key] = f'{kind}:{float(fill)!r}' if kind in ('slits', 'dirichlet') and fill is not None else kind
                fc[key] = float(fcv)
                periods[key] = None if per is None else float(per)
        if any(k is None for k in kinds):
            raise ValueError("every column 0..d-1 needs an entry")
        specs.append(dict(fc=np.array(fc), kinds=kinds, periods=periods))
    return specs


# ---------------------------------------------------------------------------------------------------- operator

def next_fast_len(n):
    """Smallest 2^a 3^b 5^c >= n (blml_binned.py:1533-1546; scipy's real next_fast_len agrees)."""
    best = 1 << int(np.ceil(np.log2(n)))
    a = 1
    while a <= best:
        b = a
        while b <= best:
            c = b
            while c < n:
                c *= 5
            best = min(best, c)
            b *= 3
        a *= 2
    return best


def pad_rule(shape, h, specs):
    """Per dim: the lattice length when every mode is periodic there with period m h (circular), else the
    fast FFT length >= 2m - 1 (blml_binned.py:130-136)."""
    pad = []
    for j, m in enumerate(shape):
        circ = all(split_kind(sp['kinds'][j])[0] in ('dirichlet', 'pball') and sp['periods'][j] is not None and
                   abs(m * h[j] - sp['periods'][j]) <= 1e-9 * sp['periods'][j] for sp in specs)
        pad.append(m if circ else next_fast_len(2 * m - 1))
    return tuple(pad)


def mode_table(spec, shape, h, pad):
    """One mode's kernel on the padded lattice (offsets folded to [-(L-1)/2, L/2], zero beyond |j| > m-1 on
    linear dims) (blml_binned.py:63-84)."""
    d = len(shape)
    diffs, masks = [], []
    for j, (m, L) in enumerate(zip(shape, pad)):
        idx = np.arange(L)
        off = np.where(idx < (L + 1) // 2, idx, idx - L).astype(float)
        mk = np.ones(L) if L == m else (np.abs(off) <= m - 1).astype(float)
        sh = [1] * d; sh[j] = L
        diffs.append((off * h[j]).reshape(sh)); masks.append(mk.reshape(sh))
    T = 1.0
    for kind, dims in units_of(spec['kinds']):
        T = T * unit_value(kind, spec['fc'][dims], [spec['periods'][j] for j in dims], [diffs[j] for j in dims])
    for mk in masks:
        T = T * mk
    return np.broadcast_to(T, pad).astype(np.float64)


class Operator:
    """S_k for every mode: rFFT of each mode's table (modes with one kernel share it)."""

    def __init__(self, specs, shape, h, workers=None):
        import scipy.fft as sfft
        self.fft = sfft
        self.kw = {} if workers is None else dict(workers=workers)
        self.shape = tuple(shape); self.h = np.asarray(h, float)
        self.pad = pad_rule(self.shape, self.h, specs)
        key = lambda sp: (tuple(sp['fc']), tuple(sp['kinds']), tuple(sp['periods']))
        cache, self.Kf, s = {}, [], []
        for sp in specs:
            k = key(sp)
            if k not in cache:
                T = mode_table(sp, self.shape, self.h, self.pad)
                cache[k] = (sfft.rfftn(T, s=self.pad), float(T[(0,) * len(shape)]))
            self.Kf.append(cache[k][0]); s.append(cache[k][1])
        self.shared = len(cache) == 1
        self.s = np.array(s)

    def S(self, k, e):
        sl = tuple(slice(0, m) for m in self.shape)
        f, kw = self.fft, self.kw
        if np.iscomplexobj(e):
            re = f.irfftn(f.rfftn(e.real, s=self.pad, **kw) * self.Kf[k], s=self.pad, **kw)[sl]
            im = f.irfftn(f.rfftn(e.imag, s=self.pad, **kw) * self.Kf[k], s=self.pad, **kw)[sl]
            return re + 1j * im
        return f.irfftn(f.rfftn(e, s=self.pad, **kw) * self.Kf[k], s=self.pad, **kw)[sl]

    def Sall(self, E):
        return np.stack([self.S(k, E[k]) for k in range(len(self.Kf))])


def dense_gram(spec, shape, h):
    """The exact Gram S_ab = K(z_a - z_b) over every lattice point (small lattices only)."""
    g = np.meshgrid(*[np.arange(m) * hh for m, hh in zip(shape, h)], indexing='ij')
    Z = np.stack([x.ravel() for x in g], 1)
    D = Z[:, None, :] - Z[None, :, :]
    G = 1.0
    for kind, dims in units_of(spec['kinds']):
        G = G * unit_value(kind, spec['fc'][dims], [spec['periods'][j] for j in dims], [D[..., j] for j in dims])
    return G


# ---------------------------------------------------------------------------------------------------- updates

def cd_root(b, c, s):
    """Positive root of s t^2 + b t - c = 0, cancellation-free (blml_trivial.py:84-89)."""
    disc = np.sqrt(b * b + 4.0 * s * c)
    return np.where(b >= 0, 2.0 * c / np.maximum(b + disc, 1e-300), (-b + disc) / (2.0 * s))


def secular(R2, s, c, iters=16):
    """Root lam > max s of lam sum_k R2_k / (lam - s_k)^2 = c: safeguarded Newton on phi^-1/2 in mu = lam - max s
    (blml_binned.py:1556-1573)."""
    smax = float(np.max(s)); tot = R2.sum(0); dd = s - smax
    cp = np.maximum(c, 1e-30)
    hi = (tot + np.sqrt(tot * tot + 4 * cp * smax * tot)) / (2 * cp)
    lo = np.zeros_like(hi); mu = hi
    for _ in range(iters):
        with np.errstate(divide='ignore', over='ignore', invalid='ignore'):
            q = 1.0 / (mu[None] - dd); W = R2 * q * q; A = W.sum(0); B = (W * q).sum(0)
            lam = smax + mu; phi = lam * A
            big = phi > c
            lo = np.where(big, mu, lo); hi = np.where(big, hi, mu)
            nt = mu + 2 * phi * (1 - np.sqrt(phi / cp)) / (A - 2 * lam * B)
        mu = np.where((nt >= lo) & (nt <= hi), nt, 0.5 * (lo + hi))
    return smax + mu


def rdot(a, b):
    return float(np.real(np.sum(np.conj(a) * b)))


class BinnedFit:
    """The reference's BLMLBinned fit, restated in float64 NumPy (see the module docstring for the map)."""

    def __init__(self, tol=1e-5, max_sweeps=None, anderson=5, phase_noise=0.1, seed=0, stall=1000, ll_tol=None,
                 ll_window=100, solver='cd', lbfgs_m=20):
        if solver not in ('cd', 'lbfgs'):
            raise ValueError("solver: 'cd' or 'lbfgs'")
        self.tol, self.max_sweeps, self.anderson = tol, max_sweeps, anderson
        self.phase_noise, self.seed, self.stall = phase_noise, seed, stall
        self.ll_tol, self.ll_window, self.solver, self.lbfgs_m = ll_tol, ll_window, solver, int(lbfgs_m)

    # ---------------------------------------------------------------- pieces
    def Sall(self, E):
        return self.op.Sall(E)

    def merit(self, E, U):
        c, occ, n = self.c, self.occ, self.n
        if self.psd:
            F = (np.abs(U) ** 2).sum(0); Q = rdot(E, U)
            if not Q > 0:
                return -np.inf
            return float((c * np.log(np.maximum(F, 1e-30))).sum()) / n - n * np.log(Q)
        e, u = E[0], U[0]
        if np.any(occ & (self.sg * e <= 0)):
            return -np.inf
        return -(0.5 * float(np.sum(e * u)) - float((c * np.log(np.where(occ, np.abs(e), 1.0))).sum())) / n

    def update(self, E, U):
        c = self.c
        s = self.s.reshape((-1,) + (1,) * self.d)
        R = U - s * E
        if not self.psd:
            t = np.where(self.occ, cd_root(self.sg * R[0], c, float(self.s[0])), 0.0)
            return (self.sg * t)[None].astype(E.dtype)
        a2 = (np.abs(R) ** 2).sum(0); a = np.sqrt(a2)
        if np.allclose(self.s, self.s[0]):
            s0 = float(self.s[0]); t = 2 * c / (a + np.sqrt(a2 + 4 * s0 * c))
            out = R * (t / np.where(a > 0, a, 1.0))[None]
            lone = (a == 0) & (c > 0)
            if lone.any():
                out[0] = np.where(lone, np.sqrt(c / s0), out[0])
            return out.astype(E.dtype)
        lone = (a2 == 0) & (c > 0)
        lam = secular(np.abs(R) ** 2, s, c)
        out = np.where((c > 0)[None] & ~lone[None], R / (lam[None] - s), 0)
        if lone.any():
            out[0] = np.where(lone, np.sqrt(c / float(self.s[0])), out[0])
        return out.astype(E.dtype)

    def rescale(self, E, U):
        Q = rdot(E, U)
        sc = float(self.n / np.sqrt(Q)) if Q > 0 else 1.0
        return E * sc, U * sc

    def resid(self, E, U):
        c, occ = self.c, self.occ
        nrm2 = (np.abs(E) ** 2).sum(0)
        r = np.sqrt((np.abs(U * (nrm2 / np.where(occ, c, 1.0))[None] - E) ** 2).sum(0)) / np.sqrt(np.maximum(nrm2, 1e-300))
        return float(np.max(np.where(occ, r, 0.0)))

    # ---------------------------------------------------------------- CD
    def solve_cd(self, E, cap):
        U = self.Sall(E); E, U = self.rescale(E, U)
        cur = self.merit(E, U); hX, hF = [], []; mA = self.anderson
        n_and = n_damp = n_grad = 0; it = 0; res = self.resid(E, U); hist = [res]
        cap = np.inf if cap is None else cap
        best_res, best_it, best_m = res, 0, cur
        mhist = [cur]; self.stop_reason = 'tol'
        while res >= self.tol and it < cap:
            if it - best_it >= self.stall:
                self.stop_reason = 'stall'; break
            if self.ll_tol is not None and len(mhist) > self.ll_window and \
                    (mhist[-1] - mhist[-1 - self.ll_window]) / self.n < self.ll_tol:
                self.stop_reason = 'll_tol'; break
            it += 1
            EJ = self.update(E, U); UJ = self.Sall(EJ); mJ = self.merit(EJ, UJ)
            if mA:
                f = (EJ - E).ravel()
                hX.append(E.ravel()); hF.append(f); hX, hF = hX[-(mA + 1):], hF[-(mA + 1):]
                if len(hX) >= 3:
                    try:
                        EA = E + f.reshape(E.shape) - anderson_mix(hX, hF, f).reshape(E.shape)
                        UA = self.Sall(EA); mAc = self.merit(EA, UA)
                        if mAc > mJ:
                            EJ, UJ, mJ = EA, UA, mAc; n_and += 1
                    except Exception:
                        hX, hF = [], []
            if mJ < cur - 1e-12 * abs(cur):
                hX, hF = [], []; n_damp += 1
                EP = self.update(E, U); UP = self.Sall(EP); a = 0.5
                while a > 1e-8:
                    EJ, UJ = E + a * (EP - E), U + a * (UP - U); mJ = self.merit(EJ, UJ)
                    if mJ >= cur:
                        break
                    a *= 0.5
                else:
                    EJ, UJ, mJ = E, U, cur
                    if self.psd:
                        EJ, UJ, mJ = self.grad_steps(E, U, cur); n_grad += 1
            E, U = self.rescale(EJ, UJ); cur = mJ if self.psd else self.merit(E, U); mhist.append(cur)
            res = self.resid(E, U); hist.append(res)
            if res < 0.9 * best_res or cur > best_m + 1e-13 * abs(best_m):
                best_res, best_it, best_m = min(res, best_res), it, max(cur, best_m)
        if res >= self.tol and self.stop_reason == 'tol':
            self.stop_reason = 'max_sweeps'
        self.n_sweeps, self.residual, self.converged = it, res, res < self.tol
        self.merit_history, self.rho_history = mhist, hist
        self.n_anderson, self.n_damped, self.n_gradient = n_and, n_damp, n_grad
        return E, U

    def grad_steps(self, E, U, cur, steps=5):
        for _ in range(steps):
            F = (np.abs(U) ** 2).sum(0); Q = rdot(E, U)
            V = np.where(self.occ, self.w / np.where(self.occ, F, 1.0), 0.0)[None] * U
            G = np.where(self.occ[None], self.Sall(V) - (self.n / Q) * U, 0)
            SG = self.Sall(G); g2 = rdot(G, G)
            if not g2 > 0:
                break
            a = getattr(self, '_gstep', None) or 1e-3 * np.sqrt(float(np.sum(np.abs(E) ** 2)) / g2)
            ok = False
            for _ in range(40):
                En, Un = E + a * G, U + a * SG; mn = self.merit(En, Un)
                if mn > cur:
                    ok = True; break
                a *= 0.5
            if not ok:
                break
            E, U, cur = En, Un, mn; self._gstep = 2 * a
        return E, U, cur

    # ---------------------------------------------------------------- L-BFGS
    def lgrad(self, E, U):
        F = (np.abs(U) ** 2).sum(0); Q = rdot(E, U)
        if not Q > 0:
            return -np.inf, None
        L = float((self.w * np.log(np.where(self.occ, F, 1.0))).sum()) - self.n * np.log(Q)
        V = np.where(self.occ, self.w / np.where(self.occ, F, 1.0), 0.0)[None] * U
        G = self.Sall(V) - (self.n / Q) * U
        return L, 2 * np.where(self.occ[None], G, 0)

    def solve_lbfgs(self, E, cap):
        n = self.n; m_ = self.lbfgs_m
        U = self.Sall(E); E, U = self.rescale(E, U)
        L, g = self.lgrad(E, U)
        S_, Y_, R_ = [], [], []; it = 0; res = self.resid(*self.rescale(E, U)); hist = [res]; mhist = [L / n]
        cap = np.inf if cap is None else cap; self.stop_reason = 'tol'; reset = False
        ftol, fwin = (self.ll_tol if self.ll_tol is not None else 1e-11), 10
        while res >= self.tol and it < cap:
            if len(mhist) > fwin and mhist[-1] - mhist[-1 - fwin] < ftol:
                self.stop_reason = 'll_tol'; break
            it += 1
            q = g.copy(); al = []
            for s_, y_, r_ in zip(reversed(S_), reversed(Y_), reversed(R_)):
                a = r_ * rdot(s_, q); al.append(a); q = q - a * y_
            if S_:
                q = q * (rdot(S_[-1], Y_[-1]) / rdot(Y_[-1], Y_[-1]))
            else:
                q = q * (1e-3 * np.sqrt(rdot(E, E) / max(rdot(g, g), 1e-300)))
            for (s_, y_, r_), a in zip(zip(S_, Y_, R_), reversed(al)):
                b = r_ * rdot(y_, q); q = q + (a - b) * s_
            slope = rdot(g, q)
            if not slope > 0:
                S_, Y_, R_ = [], [], []
                q = g * (1e-3 * np.sqrt(rdot(E, E) / max(rdot(g, g), 1e-300))); slope = rdot(g, q)
            t = 1.0; ok = False
            for _ in range(40):
                En = E + t * q; Un = self.Sall(En); Ln, gn = self.lgrad(En, Un)
                if Ln >= L + 1e-4 * t * slope:
                    ok = True; break
                t *= 0.5
            if not ok:
                if reset or not S_:
                    self.stop_reason = 'stall'; break
                S_, Y_, R_ = [], [], []; reset = True; continue
            reset = False
            s_, y_ = En - E, g - gn
            sy = rdot(s_, y_)
            if sy > 1e-12 * np.sqrt(rdot(s_, s_) * rdot(y_, y_)):
                S_.append(s_); Y_.append(y_); R_.append(1.0 / sy)
                if len(S_) > m_:
                    S_.pop(0); Y_.pop(0); R_.pop(0)
            E, U, L, g = En, Un, Ln, gn
            res = self.resid(*self.rescale(E, U)); hist.append(res); mhist.append(L / n)
        if res >= self.tol and self.stop_reason == 'tol':
            self.stop_reason = 'max_sweeps'
        F = (np.abs(U) ** 2).sum(0); Q = rdot(E, U)
        Ec = np.where(self.occ, (Q / n) * self.w / np.where(self.occ, F, 1.0), 0.0)[None] * U
        Uc = self.Sall(Ec); Lc, _ = self.lgrad(Ec, Uc)
        if Lc >= L - 1e-9 * n:
            E, U = Ec, Uc
        E, U = self.rescale(E, U); res = self.resid(E, U)
        self.n_sweeps, self.residual = it, res
        self.converged = res < self.tol or self.stop_reason == 'll_tol'
        self.merit_history, self.rho_history = mhist, hist
        self.n_anderson = self.n_damped = self.n_gradient = 0
        return E, U

    def solve(self, E, cap):
        if self.solver == 'lbfgs' and self.psd:
            lc = getattr(self, 'lbfgs_cap', None)           # a cap on the L-BFGS alone (the start keeps max_sweeps)
            return self.solve_lbfgs(E, cap if lc is None else lc)
        return self.solve_cd(E, cap)

    # ---------------------------------------------------------------- fit
    def fit(self, counts, modes, h=1.0, complex_g=False, signs=None, init=None):
        counts = np.asarray(counts)
        if counts.ndim < 1 or np.any(counts < 0) or not np.all(np.isfinite(counts)):
            raise ValueError("counts: a non-negative finite array on the lattice")
        self.d = counts.ndim; self.shape = counts.shape
        self.specs = parse_modes(modes, self.d)
        self.h = np.broadcast_to(np.asarray(h, float), (self.d,)).copy()
        self.op = Operator(self.specs, self.shape, self.h, getattr(self, 'workers', None))
        self.s = self.op.s.copy(); self.K = len(self.specs); self.shared = self.op.shared
        w = np.asarray(counts, float)
        self.w = w; self.n = float(w.sum())
        if not self.n > 0:
            raise ValueError("counts: no observations")
        self.c = self.n * w; self.occ = w > 0
        self.complex_g = bool(complex_g); self.psd = self.complex_g or self.K > 1
        if signs is not None and self.psd:
            raise ValueError("signs: real rank 1 only")
        sg = np.ones(self.shape) if signs is None else np.sign(np.asarray(signs, float))
        if np.any(sg[self.occ] == 0):
            raise ValueError("signs: nonzero on every occupied bin")
        self.sg = sg
        dt = np.complex128 if self.complex_g else np.float64
        if init is not None and getattr(init, 'e_hat', None) is not None and init.shape == self.shape:
            E0 = np.asarray(init.e_hat)
            E = np.zeros((self.K,) + self.shape, dtype=dt)
            kk = min(self.K, E0.shape[0]); E[:kk] = E0[:kk] if self.complex_g else np.real(E0[:kk])
            E[:, ~self.occ] = 0
            E = self.fill_modes(E, kk, phases=False)
        else:
            E = self.start(dt)
        E, U = self.solve(E, self.max_sweeps)
        self.finish(E, U)
        return self

    def start(self, dt):
        c, s0 = self.c, float(self.s[0])
        e0 = np.where(self.occ, np.sqrt(c / s0), 0.0) * self.sg
        if not self.psd:
            return e0[None]
        save = (self.psd, self.K, self.op.Kf, self.s)
        self.psd, self.K, self.op.Kf, self.s = False, 1, self.op.Kf[:1], self.s[:1]
        er, _ = self.solve(e0[None], self.max_sweeps)
        self.psd, self.K, self.op.Kf, self.s = save
        E = np.zeros((self.K,) + self.shape, dtype=dt); E[0] = er[0]
        return self.fill_modes(E, 1)

    def fill_modes(self, E, kk, phases=True):
        rng = np.random.default_rng(self.seed); pn = self.phase_noise; sh = self.shape
        if self.complex_g and phases:
            E[0] = E[0] * np.exp(1j * pn * rng.standard_normal(sh))
        for k in range(kk, self.K):
            z = rng.standard_normal(sh) + (1j * rng.standard_normal(sh) if self.complex_g else 0)
            E[k] = pn * np.abs(E[0]) * (z / (np.sqrt(2) if self.complex_g else 1))
        return E

    def finish(self, E, U):
        self.e_hat, self.Se = E, U
        F = (np.abs(U) ** 2).sum(0)
        self.density = F / self.n ** 2
        occ = self.occ
        self.loglik = float((self.w[occ] * np.log(self.density[occ])).sum()) / self.n

    def certificate(self, k=1, tol=1e-6):
        """lambda_max(D^1/2 S_0 D^1/2) / n, D = ||e_b||^2 / w_b on occupied bins (blml_binned.py:501-518)."""
        if not self.shared:
            raise ValueError("certificate: shared kernel only")
        from scipy.sparse.linalg import LinearOperator, eigsh
        D = np.where(self.occ, (np.abs(self.e_hat) ** 2).sum(0) / np.where(self.occ, self.w, 1.0), 0.0)
        dh = np.sqrt(D); B = int(np.prod(self.shape))
        op = lambda x: (dh * self.op.S(0, dh * x.reshape(self.shape))).ravel()
        lam = eigsh(LinearOperator((B, B), matvec=op, dtype=np.float64), k=k, which='LA', tol=tol,
                    return_eigenvectors=False)
        return float(np.max(lam)) / self.n

    def certificate_vector(self, tol=1e-8):
        """(lambda_max / n, d): the certificate and its top eigenvector v mapped back to coefficients, d = D^1/2 v
        (the direction a new shared mode takes when the fit grows its rank; shared kernel only)."""
        from scipy.sparse.linalg import LinearOperator, eigsh
        D = np.where(self.occ, (np.abs(self.e_hat) ** 2).sum(0) / np.where(self.occ, self.w, 1.0), 0.0)
        dh = np.sqrt(D); B = int(np.prod(self.shape))
        op = lambda x: (dh * self.op.S(0, dh * x.reshape(self.shape))).ravel()
        lam, v = eigsh(LinearOperator((B, B), matvec=op, dtype=np.float64), k=1, which='LA', tol=tol)
        return float(lam[0]) / self.n, dh * v[:, 0].reshape(self.shape)

    def certificate_dense(self):
        """The same lambda_max from the dense exact Gram (small lattices): the reference's own check
        (results/binned_checks.py:50-53)."""
        G = dense_gram(self.specs[0], self.shape, self.h)
        D = np.where(self.occ, (np.abs(self.e_hat) ** 2).sum(0) / np.where(self.occ, self.w, 1.0), 0.0).ravel()
        dh = np.sqrt(D)
        return float(np.linalg.eigvalsh(dh[:, None] * G * dh[None, :]).max()) / self.n


class _Start:
    """An init= object: e_hat and shape (what BLMLBinned.fit reads from a previous fit, blml_binned.py:403-408)."""

    def __init__(self, e_hat, shape):
        self.e_hat, self.shape = e_hat, shape


def certified_fit(counts, spec, tol=1e-6, cert_tol=1e-3, max_rank=8, grow_iters=300, step=0.1, grow_margin=1.0,
                  ll_tol=None):
    """A certified fit of one shared kernel: the complex L-BFGS fit at rank K = 1, 2, ... until the certificate
    lambda_max(D^1/2 S D^1/2) / n <= 1 + cert_tol (blml_binned.py:501-518), each rank started from the previous fit's
    modes plus a new mode step * (rms mode norm) along d = D^1/2 v, v the certificate's top eigenvector (an ascent
    direction of the convex lift while the certificate exceeds 1). Ranks below max_rank run at most grow_iters
    L-BFGS iterations (at too low a rank the solver crawls); a capped fit within grow_margin cert_tol of the bar, and
    the fit at max_rank, run on to tol at their rank before anything else. The lift is convex, so the certified loglik is that of its unique optimum, whatever the
    path. ll_tol: the L-BFGS stop on L / n gained over 10 iterations (None: 1e-11). Returns (fit, [(K, loglik,
    certificate, iterations, capped), ...])."""
    def run(K, cap, init=None):
        f = BinnedFit(tol=tol, solver='lbfgs', ll_tol=ll_tol)
        f.lbfgs_cap = cap
        return f.fit(counts, [spec] * K, complex_g=True, init=init)

    K, cap = 1, (grow_iters if max_rank > 1 else None)
    fit = run(1, cap)
    path = []
    while True:
        cert, d = fit.certificate_vector()
        capped = cap is not None and fit.stop_reason == 'max_sweeps'
        path.append((K, float(fit.loglik), cert, int(fit.n_sweeps), capped))
        ok = cert <= 1.0 + cert_tol
        if capped and (cert <= 1.0 + grow_margin * cert_tol or K >= max_rank):
            cap = None
            fit = run(K, None, _Start(fit.e_hat.copy(), fit.shape))
            continue
        if ok or K >= max_rank:
            return fit, path
        scale = step * np.sqrt((np.abs(fit.e_hat) ** 2).sum() / K) / max(np.linalg.norm(d), 1e-300)
        init = _Start(np.concatenate([fit.e_hat, (scale * d)[None].astype(complex)], 0), fit.shape)
        K += 1
        cap = grow_iters if K < max_rank else None
        fit = run(K, cap, init)


def anderson_mix(hX, hF, f):
    """(dX + dF) gamma of Anderson type II from float64 normal equations (blml_binned.py:1463-1478)."""
    dX = [hX[i + 1] - hX[i] for i in range(len(hX) - 1)]; dF = [hF[i + 1] - hF[i] for i in range(len(hF) - 1)]
    m = len(dF); G = np.empty((m, m)); rhs = np.array([rdot(a, f) for a in dF])
    for i in range(m):
        for j in range(i, m):
            G[i, j] = G[j, i] = rdot(dF[i], dF[j])
    g = np.linalg.solve(G + 1e-12 * np.trace(G) * np.eye(m), rhs)
    if not np.all(np.isfinite(g)):
        raise np.linalg.LinAlgError
    out = float(g[0]) * (dX[0] + dF[0])
    for i in range(1, m):
        out += float(g[i]) * (dX[i] + dF[i])
    return out
