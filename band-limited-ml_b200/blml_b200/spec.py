"""The model spec of the binned path: modes lists (the reference's format), kernel units and their exact values.

Mirrors the reference's spec API (rahuljhu/band-limited-ml, blml_trivial.py): make_modes (:1467-1505),
parse_modes (:1247-1323), with_lattice (:1377-1389), the kernel units (kernel_units :330-335, radial_groups
:238-250) and the unit formulas (SincKernel :368-370, SlitsKernel :442-444, DirichletKernel :528-535, RadialKernel
'ball' :690-694, PeriodicBallKernel :656-665, pball_harmonics :632-639). Host-side set-up only: these values build
the restricted transforms and the pair tables; no fit arithmetic runs here."""
import numpy as np

KINDS = ('sinc', 'dirichlet', 'ball', 'slits', 'pball')
GROUP_KINDS = ('ball', 'pball')                  # multi-column units (tuple keys)
_PARAMS = {'sinc': ('fc',), 'slits': ('fc', 'fill'), 'dirichlet': ('fc', 'period', 'fill'), 'ball': ('fc',),
           'pball': ('fc', 'period')}
_STRUCT = {'kind', 'dep', 'h', '_unit'}


def split_kind(kind):
    name, _, tag = str(kind).partition(':')
    return name, tag


def is_group(kind):
    return split_kind(kind)[0] in GROUP_KINDS


def param_value(v):
    if isinstance(v, dict):
        if set(v) - {'value', 'trainable'}:
            raise ValueError(f"parameter {v}: keys must be 'value' and/or 'trainable'")
        return v.get('value'), v.get('trainable')
    return v, None


def dirichlet_N(fc, P):
    return max(0, int(np.floor(fc * P / 2.0 + 1e-9)))


def dirichlet_inner_M(fc, P, fill):
    if fill is None or fill >= 1.0:
        return 0
    Ni = int(np.ceil((1.0 - fill) * fc * P / 2.0 - 1e-9)) - 1
    return max(2 * Ni + 1, 0)


def pball_harmonics(fc, periods):
    """(H, D) integer harmonic vectors with sum (k_i / P_i)^2 <= (fc / 2)^2, and the scale 1 / prod P."""
    P = np.atleast_1d(np.asarray(periods, float)); R = float(fc) / 2.0
    N = [max(0, int(np.floor(R * p + 1e-9))) for p in P]
    g = np.meshgrid(*[np.arange(-n, n + 1) for n in N], indexing='ij')
    Kv = np.stack([x.ravel() for x in g], 1)
    keep = ((Kv / P) ** 2).sum(1) <= R * R * (1 + 1e-9) + 1e-12
    return Kv[keep], 1.0 / float(np.prod(P))


def ball_profile(s, dg):
    """FT of the ball |nu| <= 1/2 in dg dims at radius s."""
    from scipy.special import jv, gamma
    s = np.asarray(s, float)
    out = np.full(s.shape, np.pi ** (dg / 2) * 0.5 ** dg / gamma(dg / 2 + 1))
    nz = s > 0
    out[nz] = 0.5 ** (dg / 2) * jv(dg / 2, np.pi * s[nz]) / s[nz] ** (dg / 2)
    return out


def unit_value(kind, fc, periods, diffs):
    """K of one unit at coordinate differences (one array per column of the unit); fc / periods per column."""
    name, tag = split_kind(kind)
    if name == 'sinc':
        f = float(fc[0]); return f * np.sinc(f * np.asarray(diffs[0], float))
    if name == 'slits':
        f = float(fc[0]); fi = (1.0 - float(tag)) * f; t = np.asarray(diffs[0], float)
        return f * np.sinc(f * t) - fi * np.sinc(fi * t)
    if name == 'dirichlet':
        P, f = float(periods[0]), float(fc[0])
        M = 2 * dirichlet_N(f, P) + 1; Mi = dirichlet_inner_M(f, P, float(tag) if tag else None)
        t = np.mod(np.abs(np.asarray(diffs[0], float)), P); t = np.minimum(t, P - t)
        with np.errstate(divide='ignore', invalid='ignore'):
            v = (np.sin(np.pi * M * t / P) - np.sin(np.pi * Mi * t / P)) / np.sin(np.pi * t / P)
        return np.where(t < 1e-10, M - Mi, v) / P
    if name == 'pball':
        P = np.asarray(periods, float); Kv, sc = pball_harmonics(float(fc[0]), P)
        out = 0.0
        for k in Kv:
            ph = 0.0
            for i in range(len(P)):
                if k[i]:
                    ph = ph + (2 * np.pi * k[i] / P[i]) * np.asarray(diffs[i], float)
            out = out + np.cos(ph)
        return sc * (out + 0.0 * sum(np.asarray(x, float) for x in diffs))
    if name == 'ball':
        f = np.asarray(fc, float); s = np.sqrt(sum((fi * np.asarray(dk, float)) ** 2 for fi, dk in zip(f, diffs)))
        return float(np.prod(f)) * ball_profile(s, len(f))
    raise ValueError(f"unknown kernel kind {kind!r}")


def ball_profile_dlog(s, dg):
    """s p'(s) of the ball profile: -pi (1/2)^(dg/2) s^(1 - dg/2) J_{dg/2 + 1}(pi s), 0 at s = 0."""
    from scipy.special import jv
    s = np.asarray(s, float)
    out = np.zeros(s.shape)
    nz = s > 0
    out[nz] = -np.pi * 0.5 ** (dg / 2) * s[nz] ** (1 - dg / 2) * jv(dg / 2 + 1, np.pi * s[nz])
    return out


def unit_value_dlog(kind, fc, periods, diffs):
    """dK/dlog fc of one unit with its fc columns scaled together (blml_trivial.py:372-377 sinc, :446-453 slits,
    :593-600 ball with s p'(s) of :146-154), or None where fc moves in whole harmonics (dirichlet, pball)."""
    name, tag = split_kind(kind)
    if name == 'sinc':
        f = float(fc[0]); return f * np.cos(np.pi * f * np.asarray(diffs[0], float))
    if name == 'slits':
        f = float(fc[0]); fi = (1.0 - float(tag)) * f; t = np.asarray(diffs[0], float)
        return f * np.cos(np.pi * f * t) - fi * np.cos(np.pi * fi * t)
    if name == 'ball':
        f = np.asarray(fc, float); D = len(f)
        s = np.sqrt(sum((fi * np.asarray(dk, float)) ** 2 for fi, dk in zip(f, diffs)))
        return float(np.prod(f)) * (D * ball_profile(s, D) + ball_profile_dlog(s, D))
    if name in ('dirichlet', 'pball'):
        return None
    raise ValueError(f"unknown kernel kind {kind!r}")


def units_of(kinds):
    """[(kind, dims)]: one-column units first, then one per group in order of first appearance."""
    units = [(k, [j]) for j, k in enumerate(kinds) if not is_group(k)]
    groups = {}
    for j, k in enumerate(kinds):
        if is_group(k):
            name, tag = split_kind(k)
            g = groups.setdefault(tag, (name, []))
            if g[0] != name:
                raise ValueError(f"group {tag!r} mixes kinds {g[0]!r} and {name!r}")
            g[1].append(j)
    return units + [(f'{nm}:{tag}', dims) for tag, (nm, dims) in groups.items()]


def make_modes(fc, kinds=None, periods=None, rank=1, dep=None, d=None):
    """A modes list from per-dim settings: fc scalar, (d,) or (K, d); kinds per dim ('sinc', 'dirichlet',
    'dirichlet:<fill>', 'slits:<fill>', 'ball', 'ball:<tag>', 'pball', ...); periods per dim; rank K."""
    F = np.asarray(fc, dtype=float)
    if d is None:
        d = len(kinds) if kinds is not None else (F.shape[-1] if F.ndim else None)
    if d is None:
        raise ValueError("make_modes: give kinds or d with a scalar fc")
    F = F if F.ndim == 2 else np.broadcast_to(F, (d,))[None]
    F = np.broadcast_to(F, (int(rank) if len(F) == 1 else len(F), d))
    kinds = list(kinds) if kinds is not None else ['sinc'] * d
    deps = set() if dep is None else {int(j) for j in np.atleast_1d(dep)}
    groups = {}
    for j, k in enumerate(kinds):
        if is_group(k):
            groups.setdefault(split_kind(k)[1], []).append(j)
    unit_of = {j: tuple(g) for g in groups.values() for j in g}
    out = []
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
            if j in deps:
                c['dep'] = True
            key = unit_of.get(j, j)
            if name == 'pball':
                c['period'] = [periods[i] for i in key]
            if key == j or j == key[0]:
                m[key] = c
        out.append(m)
    return out


def with_lattice(modes, h):
    """modes on the fixed lattice h (scalar or per column): counts on bin centres h * integers."""
    out = []
    for m in modes:
        mm = {}
        for key, c in m.items():
            cols = key if isinstance(key, tuple) else (key,)
            hv = np.broadcast_to(np.asarray(h, float), (max(max(cols) + 1, np.size(h)),))
            if isinstance(key, tuple) and len({float(hv[j]) for j in cols}) > 1:
                raise ValueError(f"columns {key}: one unit, one lattice step")
            mm[key] = dict(c, h=float(hv[cols[0]]))
        out.append(mm)
    return out


def modes_lattice(modes, d):
    """The fixed lattice steps (d,) the modes declare (column key 'h'), or None."""
    hs = []
    for k, m in enumerate(modes):
        per = {}
        for key, c in m.items():
            for j in (key if isinstance(key, tuple) else (key,)):
                per[j] = c.get('h')
        hk = [per.get(j) for j in range(d)]
        if any(v is None for v in hk) and any(v is not None for v in hk):
            raise ValueError(f"mode {k}: h (a fixed lattice) must be given for every column or none")
        hs.append(None if hk[0] is None else np.array(hk, float))
    if any((a is None) != (hs[0] is None) or (a is not None and not np.allclose(a, hs[0])) for a in hs):
        raise ValueError("h (the lattice) must be the same in every mode")
    return hs[0]


def parse_modes(modes, d, need_fc=True):
    """(specs, dep): per mode dict(fc (d,), kinds (d,), periods (d,), fc_trainable (d,)) with group kinds tagged by
    their columns ('pball:0-1') and fills carried in the kind ('slits:0.4'); dep, the dependent columns or None.
    fc is a bare value or {'value': v, 'trainable': bool} (trainable by default); need_fc=False lets a trainable fc be
    left out (NaN: a selector template, blml_trivial.py:1247-1323)."""
    if isinstance(modes, dict) or not isinstance(modes, (list, tuple)) or not modes:
        raise TypeError("modes: a non-empty list of mode dicts {column: {...}}; wrap one mode as [mode]")
    specs, deps = [], []
    for k, m in enumerate(modes):
        fc = [None] * d; kinds = [None] * d; periods = [None] * d; dep = [False] * d; tr = [True] * d
        for key, c in m.items():
            kind = c.get('kind', 'sinc')
            if kind not in KINDS:
                raise ValueError(f"mode {k}: kind {kind!r}, expected one of {KINDS}")
            bad = set(c) - _STRUCT - set(_PARAMS[kind])
            if bad:
                raise ValueError(f"mode {k} columns {key}: unknown keys {sorted(bad)}")
            fcv, fct = param_value(c.get('fc'))
            fct = True if fct is None else bool(fct)
            if fcv is None:
                if not fct:
                    raise ValueError(f"mode {k} columns {key}: a fixed (trainable=False) fc needs a value")
                if need_fc:
                    raise ValueError(f"mode {k} columns {key}: fc missing")
                fcv = np.nan
            elif not float(fcv) > 0:
                raise ValueError(f"mode {k} columns {key}: fc must be positive, got {fcv}")
            per = param_value(c.get('period'))[0]
            fill = param_value(c.get('fill'))[0]
            if kind in ('dirichlet', 'pball') and per is None:
                raise ValueError(f"mode {k} columns {key}: period missing (kind {kind!r} needs it)")
            if kind == 'slits' and fill is None:
                raise ValueError(f"mode {k} columns {key}: fill missing (kind 'slits' needs it)")
            if fill is not None and not 0 < float(fill) <= 1:
                raise ValueError(f"mode {k} columns {key}: fill must be in (0, 1], got {fill}")
            if isinstance(key, tuple):
                if kind not in GROUP_KINDS:
                    raise ValueError(f"columns {key}: a tuple key is a multi-column unit ('ball' or 'pball')")
                tag = '-'.join(map(str, key))
                pv = None if per is None else np.broadcast_to(np.asarray(per, float), (len(key),))
                for i, j in enumerate(key):
                    if not 0 <= j < d:
                        raise ValueError(f"mode {k}: column {j} outside 0..{d - 1}")
                    kinds[j] = f'{kind}:{tag}'; fc[j] = float(fcv); tr[j] = fct
                    periods[j] = None if pv is None else float(pv[i]); dep[j] = bool(c.get('dep', False))
            else:
                if kind in GROUP_KINDS:
                    raise ValueError(f"column {key}: kind {kind!r} spans columns: give its unit as a tuple key")
                if not 0 <= key < d:
                    raise ValueError(f"mode {k}: column {key} outside 0..{d - 1}")
                kinds[key] = f'{kind}:{float(fill)!r}' if kind in ('slits', 'dirichlet') and fill is not None else kind
                fc[key] = float(fcv); tr[key] = fct; periods[key] = None if per is None else float(per)
                dep[key] = bool(c.get('dep', False))
        if any(x is None for x in kinds):
            raise ValueError(f"mode {k}: columns {[j for j in range(d) if kinds[j] is None]} missing; "
                             f"expected every column 0..{d - 1}")
        specs.append(dict(fc=np.array(fc, float), kinds=kinds, periods=periods, fc_trainable=np.array(tr, bool)))
        deps.append(dep)
    if any(dp != deps[0] for dp in deps):
        raise ValueError("dep must mark the same columns in every mode")
    dep = [j for j in range(d) if deps[0][j]]
    return specs, (dep or None)


def _columns(m):
    """{column: its entry} of one mode, tuple keys spread over their columns."""
    out = {}
    for key, c in m.items():
        for j in (key if isinstance(key, tuple) else (key,)):
            out[j] = c
    return out


def modes_fc(modes):
    """(K, d) cut-offs of a modes list, NaN where fc is left out (blml_trivial.py:1525-1530)."""
    rows = [_columns(m) for m in modes]
    d = max(max(r) for r in rows) + 1
    val = lambda c: param_value(c.get('fc'))[0]
    return np.array([[np.nan if val(r[j]) is None else float(val(r[j])) for j in range(d)] for r in rows], float)


def modes_trainable(modes):
    """(K, d) whether each column's fc is trainable (default True; blml_trivial.py:1533-1540)."""
    rows = [_columns(m) for m in modes]
    d = max(max(r) for r in rows) + 1
    tr = lambda c: True if param_value(c.get('fc'))[1] is None else bool(param_value(c.get('fc'))[1])
    return np.array([[tr(r[j]) for j in range(d)] for r in rows], bool)


def with_fc(modes, fc):
    """modes with fc replaced (scalar, (d,) for every mode, or (K, d)); a unit takes its first column's value;
    trainability kept (blml_trivial.py:1576-1582)."""
    F = np.broadcast_to(np.asarray(fc, float), modes_fc(modes).shape)
    out = []
    for k, m in enumerate(modes):
        mm = {}
        for key, c in m.items():
            j = key[0] if isinstance(key, tuple) else key
            t = param_value(c.get('fc'))[1]
            mm[key] = dict(c, fc=float(F[k, j]) if t is None else dict(value=float(F[k, j]), trainable=t))
        out.append(mm)
    return out


def spec_key(sp):
    return (tuple(np.round(sp['fc'], 15)), tuple(sp['kinds']), tuple(sp['periods']))
