"""Restricted transforms of each mode's Gram operator, and the device plans that apply them.

The reference applies S_k e as a zero-padded FFT convolution with the mode's kernel table (blml_binned.py:49-101,
119-168): linear on dims padded to next_fast_len(2m - 1), circular on dims where every mode is periodic with period
m h. Every supported kernel is a weighted sum of plane waves, so the same operator is
    S e = sum_q W_q v_q v_q^H e,   v_q(j) = exp(2 pi i sum_a nu_{a, q_a} j_a),
over a product grid of per-axis frequencies nu (cycles per lattice index):

  dirichlet column      its harmonics k / P (minus the inner band of a fill), weight 1 / P: exact
  pball group           the box of harmonics |k_i| <= N_i per axis, weight 1 / prod P inside the ellipse, 0 outside:
                        exact (on a circular lattice this is the DFT mask of the kernel)
  sinc / slits column   Gauss-Legendre nodes on the band's interval(s), weights (f / 2) w_GL: the node count grows
                        until the quadrature reproduces K at every lattice offset to 1e-15 of K(0)
  ball group (or any    the padded lattice's own DFT: nu = q / L over the pad, weight = FFT of the padded table / L
  unit on demand)       (the reference's operator exactly)

Units multiply, so W is the outer product of the units' weight tensors. Only the mode's plane-wave structure is
built here on the host (float64); the contraction itself runs on the GPU (csrc/matvec.cu)."""
import numpy as np

from . import _lib
from .spec import units_of, split_kind, unit_value, unit_value_dlog, pball_harmonics, dirichlet_N, dirichlet_inner_M


def next_fast_len(n):
    """Smallest 2^a 3^b 5^c >= n."""
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
    """The reference's padded lengths (blml_binned.py:130-136): m where every mode is periodic with period m h."""
    pad = []
    for j, m in enumerate(shape):
        circ = all(split_kind(sp['kinds'][j])[0] in ('dirichlet', 'pball') and sp['periods'][j] is not None and
                   abs(m * h[j] - sp['periods'][j]) <= 1e-9 * sp['periods'][j] for sp in specs)
        pad.append(m if circ else next_fast_len(2 * m - 1))
    return tuple(pad)


def _gl_interval(lo, hi, Q):
    x, w = np.polynomial.legendre.leggauss(Q)
    half = 0.5 * (hi - lo)
    return lo + half * (x + 1.0), half * w


def _quad_unit(kind, fc, h, m, L, tol=1e-14):
    """GL nodes (cycles per index) and weights of a sinc / slits column so that sum_q w_q cos(2 pi nu_q j) equals the
    unit at every offset j h, |j| < m, to tol * K(0); None when that takes L nodes or more (the padded lattice's DFT
    represents the unit exactly with L). A float64 sum of Q such terms carries a rounding error of a few 1e-15 of
    K(0), so tol sits just above that floor: the node count converges about 15% past the band's oscillation count
    pi * width * (m - 1) h / 2 instead of growing to the cap."""
    name, tag = split_kind(kind)
    f = float(fc)
    if name == 'sinc':
        ivals = [(-f / 2, f / 2)]
    else:
        fi = (1.0 - float(tag)) * f
        ivals = [(-f / 2, -fi / 2), (fi / 2, f / 2)] if fi > 0 else [(-f / 2, f / 2)]
    j = np.arange(m, dtype=float)
    exact = unit_value(kind, [f], [None], [j * h])
    k0 = float(unit_value(kind, [f], [None], [np.zeros(1)])[0])
    width = max(hi - lo for lo, hi in ivals)
    Q = max(8, int(np.ceil(np.pi * width * (m - 1) * h / 2)) + 12)
    while len(ivals) * Q < L:
        nus, ws = [], []
        for lo, hi in ivals:
            nu, w = _gl_interval(lo, hi, Q)
            nus.append(nu); ws.append(w)
        nu = np.concatenate(nus); w = np.concatenate(ws)
        approx = np.cos(2 * np.pi * np.outer(j * h, nu)) @ w
        if np.max(np.abs(approx - exact)) <= tol * abs(k0):
            return nu * h, w
        Q = int(Q * 1.15) + 4
    return None


def _pad_unit(kind, fc, periods, dims, shape, h, pad, values=unit_value):
    """The padded-lattice DFT representation of one unit over its dims: frequencies q / L, weights FFT(T) / L, T the
    unit's values (or another table of the same shape, e.g. its dK/dlog fc) at the padded offsets."""
    d = len(dims)
    diffs, masks = [], []
    for i, a in enumerate(dims):
        L, m = pad[a], shape[a]
        idx = np.arange(L)
        off = np.where(idx < (L + 1) // 2, idx, idx - L).astype(float)
        mk = np.ones(L) if L == m else (np.abs(off) <= m - 1).astype(float)
        sh = [1] * d; sh[i] = L
        diffs.append((off * h[a]).reshape(sh)); masks.append(mk.reshape(sh))
    T = values(kind, fc, periods, diffs)
    for mk in masks:
        T = T * mk
    T = np.broadcast_to(T, tuple(pad[a] for a in dims)).astype(np.float64)
    Wt = np.real(np.fft.fftn(T)) / float(np.prod([pad[a] for a in dims]))
    freqs = [np.arange(pad[a]) / float(pad[a]) for a in dims]
    return freqs, Wt


def unit_transform(kind, fc, periods, dims, shape, h, pad):
    """(per-dim frequency arrays in cycles per index, weight tensor over them) for one unit."""
    name, tag = split_kind(kind)
    if name == 'dirichlet':
        a = dims[0]; P = float(periods[0]); f = float(fc[0])
        N = dirichlet_N(f, P); Mi = dirichlet_inner_M(f, P, float(tag) if tag else None)
        k = np.arange(-N, N + 1); k = k[np.abs(k) > (Mi - 1) // 2] if Mi else k
        return [k * h[a] / P], np.full(len(k), 1.0 / P)
    if name == 'pball':
        P = np.asarray(periods, float); f = float(fc[0])
        R = f / 2.0
        N = [max(0, int(np.floor(R * p + 1e-9))) for p in P]
        axes = [np.arange(-n, n + 1) for n in N]
        g = np.meshgrid(*axes, indexing='ij')
        inside = sum((gi / p) ** 2 for gi, p in zip(g, P)) <= R * R * (1 + 1e-9) + 1e-12
        sc = 1.0 / float(np.prod(P))
        return [ax * h[a] / p for ax, a, p in zip(axes, dims, P)], np.where(inside, sc, 0.0)
    if name in ('sinc', 'slits'):
        a = dims[0]
        q = _quad_unit(kind, fc[0], h[a], shape[a], pad[a])
        if q is not None:
            return [q[0]], q[1]
    return _pad_unit(kind, fc, periods, dims, shape, h, pad)


def unit_transform_dlog(kind, fc, periods, dims, shape, h, pad):
    """The plane-wave form of dK/dlog fc of one unit, or None where fc moves in whole harmonics (dirichlet, pball).
    sinc: f cos(pi f t) is the band's two edges, nu = +-f / 2 with weight f / 2 each; slits adds the inner edges
    +-fi / 2 with weight -fi / 2; ball: the padded lattice's DFT of its dlog table (blml_binned.py:92-101)."""
    name, tag = split_kind(kind)
    if name in ('dirichlet', 'pball'):
        return None
    if name in ('sinc', 'slits'):
        a = dims[0]; f = float(fc[0])
        nu, w = [-f / 2, f / 2], [f / 2, f / 2]
        if name == 'slits':
            fi = (1.0 - float(tag)) * f
            if fi > 0:
                nu += [-fi / 2, fi / 2]; w += [-fi / 2, -fi / 2]
        return [np.array(nu) * h[a]], np.array(w)
    return _pad_unit(kind, fc, periods, dims, shape, h, pad, values=unit_value_dlog)


def mode_transform_dlog(spec, shape, h, pad, u):
    """mode_transform of dK/dlog fc_u (unit u of units_of(spec['kinds']) differentiated, the others as they are), or
    None for an integer unit."""
    units = units_of(spec['kinds'])
    kind, dims = units[u]
    per = lambda ds: [spec['periods'][j] for j in ds]
    du = unit_transform_dlog(kind, spec['fc'][dims], per(dims), dims, shape, h, pad)
    if du is None:
        return None
    d = len(shape)
    freqs = [None] * d
    W = np.ones([1] * d)
    for v, (kv, dv) in enumerate(units):
        fq, Wu = du if v == u else unit_transform(kv, spec['fc'][dv], per(dv), dv, shape, h, pad)
        for a, f in zip(dv, fq):
            freqs[a] = np.asarray(f, float)
        sh = [1] * d
        for i, a in enumerate(dv):
            sh[a] = Wu.shape[i]
        W = W * Wu.reshape(sh)
    W = np.broadcast_to(W, tuple(len(f) for f in freqs)).astype(np.float64)
    return freqs, np.ascontiguousarray(W)


def mode_transform(spec, shape, h, pad):
    """Per-axis frequencies (list of d arrays) and the full weight tensor of one mode."""
    d = len(shape)
    freqs = [None] * d
    W = np.ones([1] * d)
    for kind, dims in units_of(spec['kinds']):
        fq, Wu = unit_transform(kind, spec['fc'][dims], [spec['periods'][j] for j in dims], dims, shape, h, pad)
        for a, f in zip(dims, fq):
            freqs[a] = np.asarray(f, float)
        sh = [1] * d
        for i, a in enumerate(dims):
            sh[a] = Wu.shape[i]
        W = W * Wu.reshape(sh)
    W = np.broadcast_to(W, tuple(len(f) for f in freqs)).astype(np.float64)
    return freqs, np.ascontiguousarray(W)


def kernel_at_zero(spec, d):
    """s = K(0) of a mode from the unit formulas."""
    s = 1.0
    for kind, dims in units_of(spec['kinds']):
        s *= float(np.ravel(unit_value(kind, spec['fc'][dims], [spec['periods'][j] for j in dims],
                                       [np.zeros(1) for _ in dims]))[0])
    return s


class Plan:
    """A device plan of one mode kernel: y = S x over batches of lattices (float64 or float32)."""

    def __init__(self, freqs, W, shape, dtype, engine=_lib.ENGINE_SIMT):
        self.shape = tuple(int(m) for m in shape); self.d = len(self.shape)
        self.nfreq = tuple(len(f) for f in freqs)
        self.dtype = dtype; self.engine = engine
        shp = _lib.i64(self.shape)
        nf = np.ascontiguousarray(self.nfreq, np.int32)
        fq = np.ascontiguousarray(np.concatenate(freqs), np.float64)
        Wc = np.ascontiguousarray(W, np.float64)
        import ctypes as C
        h = C.c_void_p()
        _lib.call('blml_plan_create', self.d, _lib.host_ptr(shp), _lib.host_ptr(nf), _lib.host_ptr(fq),
                  _lib.host_ptr(Wc), dtype, engine, C.byref(h))
        self._h = h
        self._ws = {}

    def __del__(self):
        h = getattr(self, '_h', None)
        if h is not None and h.value and _lib._lib is not None:
            _lib.lib().blml_plan_destroy(h)
            self._h = None

    @property
    def route(self):
        """_lib.ROUTE_FFT when blml_matvec runs the row / column FFTs of a DFT-mask kernel, else ROUTE_CONTRACT."""
        return int(_lib.lib().blml_plan_route(self._h))

    @route.setter
    def route(self, r):
        _lib.call('blml_plan_set_route', self._h, int(r))

    def workspace(self, nb, device):
        import torch
        need = int(_lib.lib().blml_matvec_workspace(self._h, nb))
        ws = self._ws.get(nb)
        if ws is None or ws.numel() < need:
            ws = torch.empty(max(need, 1), dtype=torch.uint8, device=device)
            self._ws[nb] = ws
        return ws, need

    def apply(self, x, y, nb, is_complex, stream):
        """y[:nb] = S x[:nb] (torch tensors on the device, contiguous lattices)."""
        ws, need = self.workspace(nb, x.device)
        _lib.call('blml_matvec', self._h, x.data_ptr(), y.data_ptr(), nb, int(is_complex), ws.data_ptr(), need, stream)

    @property
    def flops_per_lattice(self):
        """Useful complex multiply-adds x 8 of one complex lattice through the 2d stages."""
        shape, nf = self.shape, self.nfreq
        d = self.d
        tot = 0
        dims = list(shape)
        for s in range(d):
            a = d - 1 - s
            tot += int(np.prod(dims)) * nf[a]
            dims = [nf[a]] + dims[:-1]
        for s in range(d):
            a = d - 1 - s
            tot += int(np.prod(dims)) * shape[a]
            dims = [shape[a]] + dims[:-1]
        return 8 * tot
