"""Pair accumulation over occupied lattice bins on the GPU, with the reference's module surface
(rahuljhu/band-limited-ml, blml_local_gpu.py:423-455 and blml_kernels.py:30-217):

    ProductKernel(kinds, periods, fold).tables(fc, periods, h, Zi, want)   value tables (the reference's dict layout)
    rank_coords(Z, tab)                                                     coordinates as the row kernels read them
    rows(ZA, ZB, w, tab, grad=False, f32=False) -> (s, ds)                  s_r = sum_j S(ZA_r, ZB_j) w_j (+ d/dtheta)
    cols(ZA_dev, ZB_dev, tab, out, f32=False)                               the explicit block S(ZA, ZB) on the device

Tables are assembled on the host in float64 (their size is the lattice span, not the number of pairs) and copied
to the device once per table dict; rows and cols run in libblml_b200 (csrc/pairs.cu)."""
import ctypes as C

import numpy as np
import torch

from . import _lib
from ._lib import call
from .spec import units_of, split_kind, unit_value, is_group, pball_harmonics, ball_profile, dirichlet_N, \
    dirichlet_inner_M

KIND_CODES = dict(offset=0, circular=1, radial=2, rank=3, torus=4)
RADIAL_Q = 4


def _rankable(kind):
    return split_kind(kind)[0] in ('sinc', 'slits')


def _sinc_dshift(f, t):
    pt = np.pi * f * t
    small = np.abs(pt) < 1e-4
    ts = np.where(small, 1.0, t)
    with np.errstate(divide='ignore', invalid='ignore'):
        full = (pt * np.cos(pt) - np.sin(pt)) / (np.pi * ts * ts)
    return np.where(small, -f * (np.pi * f) ** 2 * t / 3.0, full)


def _unit_deriv(kind, fc, periods, p, diffs):
    """dK/dlog fc (p = 'fc') or dK/dt_i (p = 'shift' / ('shift', i)) of one unit at coordinate differences."""
    name, tag = split_kind(kind)
    shift = 0 if p == 'shift' else (int(p[1]) if isinstance(p, tuple) and p[0] == 'shift' else None)
    if name == 'sinc':
        f = float(fc[0])
        return _sinc_dshift(f, diffs[0]) if shift is not None else f * np.cos(np.pi * f * diffs[0])
    if name == 'slits' and shift is None:
        f = float(fc[0]); fi = (1.0 - float(tag)) * f
        return f * np.cos(np.pi * f * diffs[0]) - fi * np.cos(np.pi * fi * diffs[0])
    if name == 'pball' and shift is not None:
        P = np.asarray(periods, float); Kv, sc = pball_harmonics(float(fc[0]), P)
        out = 0.0 * sum(np.asarray(x, float) for x in diffs)
        for k in Kv:
            if not k[shift]:
                continue
            ph = sum((2 * np.pi * k[j] / P[j]) * np.asarray(diffs[j], float) for j in range(len(P)) if k[j])
            out = out - (2 * np.pi * k[shift] / P[shift]) * np.sin(ph)
        return sc * out
    raise NotImplementedError(f"derivative {p!r} of kind {kind!r} is not available in the pair tables")


class ProductKernel:
    """The product kernel's value tables for the pair kernels (blml_kernels.ProductKernel.tables / _assemble)."""

    def __init__(self, kinds, periods=None, fold=None, engine='gpu', f32=False):
        self.kinds = list(kinds); self.d = len(self.kinds)
        self.periods = list(periods) if periods is not None else [None] * self.d
        self.fold = [True] * self.d if fold is None else list(fold)
        self.units = units_of(self.kinds)
        self.groups = [(k, dims) for k, dims in self.units if is_group(k)]
        self.f32 = f32

    def k0(self, fc, periods=None):
        periods = self.periods if periods is None else periods
        diag = np.ones(self.d); sbb = 1.0
        for kind, dims in self.units:
            v = float(np.ravel(unit_value(kind, np.asarray(fc, float)[dims], [periods[j] for j in dims],
                                          [np.zeros(1) for _ in dims]))[0])
            if not is_group(kind):
                diag[dims[0]] = v
            sbb *= v
        return diag, sbb

    def tables(self, fc, periods, h, Zi, want=()):
        periods = self.periods if periods is None else list(periods)
        Zi = np.asarray(Zi, np.int64)
        span = Zi.max(0) - Zi.min(0)
        alloc = np.ceil(np.maximum(span, 1) * 1.25).astype(np.int64)
        occ = [np.unique(Zi[:, k]) if _rankable(kd) else None for k, kd in enumerate(self.kinds)]
        return self._assemble(np.asarray(fc, float), periods, np.asarray(h, float), alloc, list(want), occ)

    def _assemble(self, fc, periods, h, span, want, vals):
        d = self.d; U = len(self.units); G = len(self.groups)
        kinds_arr = np.zeros(d, np.int64); nbins = np.zeros(d, np.int64); grp = np.full(d, -1, np.int64)
        dim_unit = np.full(d, -1, np.int64); grp_unit = np.zeros(max(G, 1), np.int64)
        Jk = np.zeros(d, np.int64); mk = np.zeros(d, np.int64); rvals = [None] * d
        rows, rrows = {}, {}
        for ui, (kind, dims) in enumerate(self.units):
            name, tag = split_kind(kind)
            fcu = fc[dims]; peru = [periods[j] for j in dims]
            if is_group(kind):
                g = [gd for _, gd in self.groups].index(dims)
                grp[dims] = g; grp_unit[g] = ui
                if name == 'pball':
                    if not all(self.fold[k] for k in dims):
                        raise ValueError(f"pball over columns {dims}: needs a folded lattice (fixed periods)")
                    P = np.asarray(peru, float); ms = np.round(P / h[dims]).astype(np.int64)
                    if np.any(np.abs(ms * h[dims] - P) > 1e-9 * P):
                        raise ValueError(f"pball: the lattice steps {h[dims]} must tile the periods {P} with whole bins")
                    grids = np.meshgrid(*[np.arange(m) * h[j] for m, j in zip(ms, dims)], indexing='ij')
                    rrows[g] = np.ravel(unit_value(kind, fcu, peru, [x for x in grids]))
                    kinds_arr[dims] = KIND_CODES['torus']; nbins[dims] = ms
                else:
                    c = fcu * h[dims]
                    if not np.allclose(c, c[0], rtol=1e-9, atol=0):
                        raise ValueError(f"radial group dims {dims}: fc*h must be equal across the group, got {c}")
                    r2max = int((np.asarray(span)[dims] ** 2).sum())
                    L = int(np.floor(np.sqrt(r2max) * RADIAL_Q)) + 2
                    s = float(c[0]) * np.arange(L) / RADIAL_Q
                    rrows[g] = float(np.prod(fcu)) * ball_profile(s, len(dims))
                    kinds_arr[dims] = KIND_CODES['radial']
                continue
            k = dims[0]; dim_unit[k] = ui; J = int(span[k]); Jk[k] = J
            if name == 'dirichlet' and self.fold[k]:
                P = float(peru[0]); nb = int(round(P / h[k]))
                rows[k] = unit_value(kind, fcu, peru, [np.arange(nb) * (P / nb)])
                kinds_arr[k] = KIND_CODES['circular']; nbins[k] = nb
            elif _rankable(kind) and vals[k] is not None and len(vals[k]) ** 2 < 2 * J + 1:
                v = np.asarray(vals[k], np.int64)
                rows[k] = unit_value(kind, fcu, peru, [(v[:, None] - v[None, :]).ravel() * h[k]])
                kinds_arr[k] = KIND_CODES['rank']; mk[k] = len(v); rvals[k] = v
            else:
                rows[k] = unit_value(kind, fcu, peru, [np.arange(-J, J + 1) * h[k]])
                kinds_arr[k] = KIND_CODES['offset']
        nW = len(want)
        wunit = np.zeros(max(nW, 1), np.int64); wcol = np.full(max(nW, 1), -1, np.int64)
        wgrp = np.full(max(nW, 1), -1, np.int64)
        drows, drr = {}, {}
        for q, (ui, p) in enumerate(want):
            kind, dims = self.units[ui]; wunit[q] = ui
            fcu = fc[dims]; peru = [periods[j] for j in dims]
            if is_group(kind):
                g = int(grp[dims[0]]); wgrp[q] = g
                if split_kind(kind)[0] != 'pball':
                    raise NotImplementedError("radial-group derivative rows are not available")
                ms = nbins[dims]
                grids = np.meshgrid(*[np.arange(m) * h[j] for m, j in zip(ms, dims)], indexing='ij')
                drr[q] = np.ravel(_unit_deriv(kind, fcu, peru, p, [x for x in grids]))
            else:
                k = dims[0]; wcol[q] = k
                if kinds_arr[k] == KIND_CODES['rank']:
                    v = rvals[k]
                    drows[q] = _unit_deriv(kind, fcu, peru, p, [(v[:, None] - v[None, :]).ravel() * h[k]])
                else:
                    drows[q] = _unit_deriv(kind, fcu, peru, p, [np.arange(-Jk[k], Jk[k] + 1) * h[k]])

        def flat(rw, n):
            base = np.zeros(max(n, 1), np.int64); parts = []; at = 0
            for k in range(n):
                if k in rw:
                    base[k] = at; parts.append(np.asarray(rw[k], float)); at += len(rw[k])
            return (np.concatenate(parts) if parts else np.zeros(1)), base
        T, base = flat(rows, d); dT, dbase = flat(drows, nW)
        LR = max([len(v) for v in list(rrows.values()) + list(drr.values())] or [2])
        R = np.zeros((max(G, 1), LR)); dR = np.zeros((max(nW, 1), LR))
        for g, v in rrows.items():
            R[g, :len(v)] = v
        for q, v in drr.items():
            dR[q, :len(v)] = v
        return dict(T=T, base=base, Jk=Jk, mk=mk, vals=rvals, kinds=kinds_arr, nbins=nbins, grp=grp, R=R,
                    dim_unit=dim_unit, grp_unit=grp_unit, U=U, dT=dT, dbase=dbase, dR=dR, wunit=wunit, wcol=wcol,
                    wgrp=wgrp, nW=nW)


def rank_coords(Z, tab):
    """Lattice coordinates as the row kernels read them: rank columns replaced by the rank among the table's values;
    a value the table lacks is an error (stale tables), never a wrong value."""
    rc = [k for k, v in enumerate(tab['vals']) if v is not None]
    Z = np.asarray(Z, np.int64)
    if not rc:
        return np.ascontiguousarray(Z)
    Z = Z.copy()
    for k in rc:
        v = tab['vals'][k]; r = np.minimum(np.searchsorted(v, Z[:, k]), len(v) - 1)
        if len(Z) and not np.array_equal(v[r], Z[:, k]):
            raise RuntimeError(f"rank column {k}: a bin value is not in the kernel table (stale tables)")
        Z[:, k] = r
    return np.ascontiguousarray(Z)


def dev_tab(tab, device=None):
    """Device copies of a table dict (made once, kept in it) and the blml_tables struct that points at them."""
    device = torch.device(device or 'cuda')
    key = ('_dev', str(device))
    if key not in tab:
        f64 = lambda a: torch.as_tensor(np.ascontiguousarray(a, np.float64)).to(device)
        i64 = lambda a: torch.as_tensor(np.ascontiguousarray(a, np.int64)).to(device)
        G = int(tab['R'].shape[0]) if (np.asarray(tab['grp']) >= 0).any() else 0
        t = dict(T=f64(tab['T']), R=f64(tab['R']), dT=f64(tab['dT']), dR=f64(tab['dR']))
        for k in ('T', 'R', 'dT', 'dR'):
            t[k + '32'] = t[k].to(torch.float32)
        for k in ('base', 'Jk', 'mk', 'kinds', 'nbins', 'grp', 'dim_unit', 'grp_unit', 'dbase', 'wunit', 'wcol', 'wgrp'):
            t[k] = i64(tab[k])
        t['G'] = G; t['LR'] = int(tab['R'].shape[1])
        tab[key] = t
    return tab[key]


def _struct(tab, t, grad, f32):
    p = lambda k: t[k].data_ptr()
    return _lib.Tables(d=len(tab['kinds']), U=int(tab['U']), G=t['G'], nW=int(tab['nW']) if grad else 0,
                       LR=t['LR'], f32=int(bool(f32)), nT=int(t['T'].numel()), ndT=int(t['dT'].numel()),
                       T=p('T'), base=p('base'), Jk=p('Jk'), mk=p('mk'), kinds=p('kinds'), nbins=p('nbins'),
                       grp=p('grp'), RT=p('R'), dim_unit=p('dim_unit'), grp_unit=p('grp_unit'), dT=p('dT'),
                       dbase=p('dbase'), dR=p('dR'), wunit=p('wunit'), wcol=p('wcol'), wgrp=p('wgrp'),
                       T32=p('T32'), RT32=p('R32'), dT32=p('dT32'), dR32=p('dR32'))


def _coords_dev(Z, tab, device):
    if isinstance(Z, torch.Tensor):
        return Z.to(device=device, dtype=torch.int64).contiguous()
    return torch.as_tensor(rank_coords(Z, tab)).to(device)


def rows_dev(ZA, ZB, w, tab, grad=False, f32=False):
    """rows on device tensors: ZA (R, d), ZB (M, d) int64 rank coordinates, w (M,) float64 -> s (R,), ds (R, nW)."""
    device = w.device
    t = dev_tab(tab, device)
    R = ZA.shape[0]; M = ZB.shape[0]; nW = int(tab['nW'])
    s = torch.empty(R, dtype=torch.float64, device=device)
    ds = torch.zeros((R, max(nW, 1)), dtype=torch.float64, device=device)
    st = _struct(tab, t, grad, f32)
    call('blml_rows', st, ZA.data_ptr(), R, ZB.data_ptr(), M, w.data_ptr(), int(bool(grad)), s.data_ptr(),
         ds.data_ptr(), torch.cuda.current_stream(device).cuda_stream)
    return s, ds


def rows(ZA, ZB, w, tab, grad=False, f32=False, device=None):
    """s_r = sum_j S(ZA_r, ZB_j) w_j and, with grad, ds (R, nW) for the tables' `want` entries (NumPy results, as
    the reference's GPU module returns)."""
    device = torch.device(device or 'cuda')
    A = _coords_dev(ZA, tab, device); Bz = _coords_dev(ZB, tab, device)
    wt = torch.as_tensor(np.ascontiguousarray(w, np.float64)).to(device) if not isinstance(w, torch.Tensor) else \
        w.to(device=device, dtype=torch.float64).contiguous()
    s, ds = rows_dev(A, Bz, wt, tab, grad, f32)
    return s.cpu().numpy(), ds.cpu().numpy()


def rows_multi(ZA, ZB, Wt, tab, umask, grad=False, f32=False, device=None):
    """Fused rows of several densities (blml_local.py:282-286, FusedFit's joint and marginals): s (R, M) with
    s[r, m] = sum_j S_m(ZA_r, ZB_j) Wt[j, m], S_m the product over the units with umask[m, u] = 1, the unit factors
    computed once per pair; ds zeros (R, M, 1) -- values only (grad=True raises). NumPy results."""
    if grad:
        raise NotImplementedError("rows_multi: derivative rows are not available")
    device = torch.device(device or 'cuda')
    um = np.asarray(umask, np.int64)
    Wn = np.ascontiguousarray(Wt, np.float64)
    if Wn.ndim != 2 or um.ndim != 2 or um.shape[0] != Wn.shape[1]:
        raise ValueError("rows_multi: Wt (M bins, densities) and umask (densities, units)")
    bits = np.array([int(sum(1 << u for u in range(um.shape[1]) if um[m, u])) for m in range(um.shape[0])], np.uint32)
    A = _coords_dev(ZA, tab, device); Bz = _coords_dev(ZB, tab, device)
    R, Mm = A.shape[0], Wn.shape[1]
    if Wn.shape[0] != Bz.shape[0]:
        raise ValueError("rows_multi: one weight row per ZB bin")
    t = dev_tab(tab, device)
    st = _struct(tab, t, False, f32)
    W = torch.as_tensor(Wn).to(device)
    s = torch.empty((R, Mm), dtype=torch.float64, device=device)
    call('blml_rows_multi', st, A.data_ptr(), R, Bz.data_ptr(), Bz.shape[0], W.data_ptr(), Mm,
         bits.ctypes.data_as(C.c_void_p), s.data_ptr(), torch.cuda.current_stream(device).cuda_stream)
    return s.cpu().numpy(), np.zeros((R, Mm, 1))


def point_rows_multi(A, Bp, Wt, kinds, fc, periods, umask, want=(), grad=False, device=None):
    """Point sums of several densities (blml_local.py:555-560, FusedFit's joint and marginals at points): s (m, M)
    with s[i, q] = sum_j K_q(A_i - Bp_j) Wt[j, q], K_q the continuous product kernel over the units with
    umask[q, u] = 1 (units in kernel-unit order: one-column units first, then groups); sinc, slits, dirichlet and
    ball units. ds zeros (m, M, 1) -- values only (want / grad raise). NumPy results."""
    if grad or len(want):
        raise NotImplementedError("point_rows_multi: derivatives are not available")
    from .binned import point_cols
    device = torch.device(device or 'cuda')
    A = np.ascontiguousarray(np.atleast_2d(A), np.float64); Bp = np.ascontiguousarray(np.atleast_2d(Bp), np.float64)
    d = A.shape[1]
    Wn = np.ascontiguousarray(Wt, np.float64)
    um = np.asarray(umask, np.int64)
    units = units_of(list(kinds))
    if Wn.ndim != 2 or Wn.shape[0] != Bp.shape[0] or um.shape != (Wn.shape[1], len(units)) or Bp.shape[1] != d:
        raise ValueError("point_rows_multi: Wt (bins, densities), umask (densities, units), A and Bp with d columns")
    sp = {'kinds': list(kinds), 'fc': np.asarray(fc, float),
          'periods': [None if p is None else float(p) for p in (periods if periods is not None else [None] * d)]}
    cols = point_cols(sp, d)
    unit_of = np.zeros(d, np.int32)
    for u, (_, dims) in enumerate(units):
        for c in dims:
            unit_of[c] = u
    masks = np.array([int(sum(1 << u for u in range(len(units)) if um[q, u])) for q in range(um.shape[0])], np.uint32)
    Mm = Wn.shape[1]
    X, Z, W = (torch.as_tensor(v).to(device) for v in (A, Bp, Wn))
    g = torch.empty((A.shape[0], Mm), dtype=torch.float64, device=device)
    call('blml_point_rows_multi', A.shape[0], d, X.data_ptr(), Bp.shape[0], Z.data_ptr(), W.data_ptr(), Mm,
         C.cast(cols, C.c_void_p), unit_of.ctypes.data_as(C.c_void_p), len(units), masks.ctypes.data_as(C.c_void_p),
         g.data_ptr(), torch.cuda.current_stream(device).cuda_stream)
    return g.cpu().numpy(), np.zeros((A.shape[0], Mm, 1))


def cols(ZA_dev, ZB_dev, tab, out, out_m=None, depmask=0, f32=False):
    """The explicit block S(ZA_r, ZB_j) into out (R, M) on the device; ZA_dev, ZB_dev are rank coordinates (torch
    int64 on the device). out float64 or float32. With depmask (a bit per column), out_m receives the marginal: the
    product over the units none of whose columns is in depmask (blml_local_gpu.py:320-361)."""
    if depmask and out_m is None:
        raise ValueError("cols: depmask needs out_m")
    device = out.device
    t = dev_tab(tab, device)
    A = _coords_dev(ZA_dev, tab, device); Bz = _coords_dev(ZB_dev, tab, device)
    R, M = A.shape[0], Bz.shape[0]
    if tuple(out.shape) != (R, M) or not out.is_contiguous():
        raise ValueError(f"cols: out must be a contiguous ({R}, {M}) array")
    st = _struct(tab, t, False, f32)
    if out_m is not None:
        if tuple(out_m.shape) != (R, M) or not out_m.is_contiguous() or out_m.dtype != out.dtype:
            raise ValueError(f"cols: out_m must be a contiguous ({R}, {M}) array of out's dtype")
        call('blml_cols_dep', st, A.data_ptr(), R, Bz.data_ptr(), M, int(depmask), out.data_ptr(), out_m.data_ptr(),
             int(out.dtype == torch.float32), torch.cuda.current_stream(device).cuda_stream)
        return out
    call('blml_cols', st, A.data_ptr(), R, Bz.data_ptr(), M, out.data_ptr(), int(out.dtype == torch.float32),
         torch.cuda.current_stream(device).cuda_stream)
    return out
