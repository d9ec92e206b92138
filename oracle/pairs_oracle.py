"""CPU oracle for the lattice-bin pair accumulation -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may use it, as the checker. A float64 NumPy
restatement of the reference's fixed-lattice pair path (rahuljhu/band-limited-ml):

  * binning     Zi = round(X / h) (round half to even), the fixed-lattice entry  blml_trivial.py:3516-3598, 402-403
  * tables      per-column value rows over lattice offsets (code 0), circular distance (1), radial r grid (2),
                rank tables (3), torus tables of a periodic ball (4)              blml_kernels.py:133-200
  * rows        s_r = sum_j w_j prod_u T_u[idx_u(z_r, z_j)], d/dtheta rows        blml_local.py:145-191
  * cols        the explicit block S(ZA_r, ZB_j)                                  blml_local.py:117-141
  * gram        the exact product kernel at lattice differences (BinnedGram)      blml_kernels.py:220-254
  * weighted CD the convex fixed-lattice fit (S e)_b e_b = n w_b                  blml_trivial.py:2860-3035
"""
import numpy as np
from blml_oracle import unit_value, units_of, split_kind, is_group_kind, pball_harmonics

RADIAL_Q = 4          # radial rows: RADIAL_Q grid points per lattice step (blml_trivial.py:199)


def bin_points(X, h):
    """Integer lattice coordinates of points: np.round (half to even) of X / h in float64."""
    return np.round(np.asarray(X, np.float64) / np.asarray(h, np.float64)).astype(np.int64)


def unique_bins(Zi):
    """Occupied bins in lexicographic order of their integer coordinates, and their counts."""
    u, cnt = np.unique(Zi, axis=0, return_counts=True)
    return u, cnt.astype(np.float64)


def gram(ZA, ZB, kinds, fc, periods, h):
    """Exact product kernel K(h (ZA_r - ZB_j)) from the unit formulas."""
    G = np.ones((len(ZA), len(ZB)))
    for kind, dims in units_of(kinds):
        diffs = [(ZA[:, k, None] - ZB[None, :, k]) * h[k] for k in dims]
        G = G * unit_value(kind, np.asarray(fc)[dims], [periods[k] for k in dims], diffs)
    return G


def build_tables(kinds, fc, periods, h, Z, rank=True):
    """Value tables of the product kernel for the bins Z (int64, (B, d)), padded 25% beyond their span as the
    reference pads (blml_kernels.py:102-128): a dict of per-column codes and rows plus group rows."""
    d = len(kinds); fc = np.asarray(fc, float); h = np.asarray(h, float)
    span = np.maximum(np.ceil(np.maximum(Z.max(0) - Z.min(0), 1) * 1.25).astype(np.int64), 1)
    cols = []
    for k in range(d):
        name, tag = split_kind(kinds[k])
        if is_group_kind(kinds[k]):
            cols.append(None); continue
        J = int(span[k])
        if name in ('sinc', 'slits') and rank:
            vals = np.unique(Z[:, k])
            if len(vals) ** 2 < 2 * J + 1:                      # rank table over the occupied values
                dv = (vals[:, None] - vals[None, :]).ravel() * h[k]
                cols.append(dict(code=3, row=unit_value(kinds[k], fc[[k]], [periods[k]], [dv]), vals=vals, m=len(vals)))
                continue
        if name == 'dirichlet':                                  # folded: circular distance 0..nb-1
            P = float(periods[k]); nb = int(round(P / h[k]))
            row = unit_value(kinds[k], fc[[k]], [P], [np.arange(nb) * h[k]])
            cols.append(dict(code=1, row=row, nb=nb)); continue
        off = np.arange(-J, J + 1) * h[k]
        cols.append(dict(code=0, row=unit_value(kinds[k], fc[[k]], [periods[k]], [off]), J=J))
    groups = []
    for kind, dims in units_of(kinds):
        if not is_group_kind(kind):
            continue
        name = split_kind(kind)[0]
        if name == 'pball':                                      # torus table over the group's circular offsets
            P = np.array([periods[j] for j in dims], float)
            ms = np.round(P / h[dims]).astype(np.int64)
            grids = np.meshgrid(*[np.arange(m) * h[j] for m, j in zip(ms, dims)], indexing='ij')
            row = unit_value(kind, fc[dims], list(P), [g.ravel() for g in grids])
            groups.append(dict(code=4, dims=list(dims), row=row, nbins=ms))
        else:                                                    # radial r grid, linear interpolation
            c = float(fc[dims[0]] * h[dims[0]])
            r2max = int((span[dims] ** 2).sum())
            L = int(np.floor(np.sqrt(r2max) * RADIAL_Q)) + 2
            s = c * np.arange(L) / RADIAL_Q
            from blml_oracle import ball_profile
            row = float(np.prod(fc[dims])) * ball_profile(s, len(dims))
            groups.append(dict(code=2, dims=list(dims), row=row))
    return dict(cols=cols, groups=groups, kinds=list(kinds))


def rank_of(vals, z):
    r = np.searchsorted(vals, z)
    if not np.array_equal(vals[np.minimum(r, len(vals) - 1)], z):
        raise RuntimeError("a bin value is not in the rank table")
    return r


def pair_values(tab, ZA, ZB):
    """The (len ZA, len ZB) block of table values (cols)."""
    V = np.ones((len(ZA), len(ZB)))
    for k, c in enumerate(tab['cols']):
        if c is None:
            continue
        za, zb = ZA[:, k, None], ZB[None, :, k]
        if c['code'] == 0:
            V = V * c['row'][za - zb + c['J']]
        elif c['code'] == 3:
            ra, rb = rank_of(c['vals'], ZA[:, k])[:, None], rank_of(c['vals'], ZB[:, k])[None, :]
            V = V * c['row'][ra * c['m'] + rb]
        else:
            nb = c['nb']; m = np.mod(za - zb, nb); m = np.minimum(m, nb - m)
            V = V * c['row'][m]
    for g in tab['groups']:
        if g['code'] == 4:
            idx = 0
            for j, nb in zip(g['dims'], g['nbins']):
                idx = idx * nb + np.mod(ZA[:, j, None] - ZB[None, :, j], nb)
            V = V * g['row'][idx]
        else:
            r2 = sum((ZA[:, j, None] - ZB[None, :, j]) ** 2 for j in g['dims'])
            t = np.sqrt(r2 * 1.0) * RADIAL_Q; i0 = t.astype(np.int64); f = t - i0
            V = V * (g['row'][i0] * (1 - f) + g['row'][i0 + 1] * f)
    return V


def rows(tab, ZA, ZB, w, chunk=2048):
    """s_r = sum_j w_j S(ZA_r, ZB_j) from the tables, float64."""
    s = np.zeros(len(ZA))
    for a in range(0, len(ZA), chunk):
        s[a:a + chunk] = pair_values(tab, ZA[a:a + chunk], ZB) @ np.asarray(w, float)
    return s


def weighted_cd(S, w, tol=1e-7, max_sweeps=100000):
    """Convex fixed-lattice BLML on occupied bins with the explicit Gram S: sequential coordinate descent to
    max_b |e_b (S e)_b / (n w_b) - 1| < tol (the reference's dense exact reference solve,
    results/binned_parity.py:78-85). Returns e, S e."""
    n = float(np.sum(w)); s0 = float(S[0, 0]); e = np.sqrt(n * w / s0); u = S @ e
    for _ in range(max_sweeps):
        for b in range(len(e)):
            bt = u[b] - s0 * e[b]; cc = n * w[b]
            disc = np.sqrt(bt * bt + 4.0 * s0 * cc)
            t = 2.0 * cc / max(bt + disc, 1e-300) if bt >= 0 else (-bt + disc) / (2.0 * s0)
            u += S[:, b] * (t - e[b]); e[b] = t
        if np.max(np.abs(e * u / (n * w) - 1)) < tol:
            break
    return e, u
