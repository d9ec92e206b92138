"""Deterministic objectives and search settings for the cut-off search fixtures (tests/golden/selector_search.json)
and the host tests of the batched search driver. Each objective is a function of fc alone, so the reference's search,
the oracle and the product's walk must request the same candidates in the same order."""
import numpy as np

R2 = float(np.sqrt(2.0))
F3 = (R2, 2.0 ** 0.25, 2.0 ** 0.125)


def bowl(centre, weight=None, cap=None, ripple=0.0, freq=9.0):
    """-sum w (log fc - log c)^2 (+ a ripple with local optima); -inf where any fc > cap."""
    c = np.log(np.asarray(centre, float))
    w = np.ones_like(c) if weight is None else np.asarray(weight, float)

    def obj(fc):
        fc = np.asarray(fc, float)
        if cap is not None and np.any(fc > cap):
            return -np.inf
        z = np.log(fc)
        return float(-np.sum(w * (z - c) ** 2) + ripple * np.sum(np.sin(freq * z)))
    return obj


def hashed(seed, scale=1.0):
    """A rough landscape: a bowl plus a deterministic pseudo-random term keyed on the rounded log fc."""

    def obj(fc):
        fc = np.asarray(fc, float)
        key = np.round(np.log(fc), 6)
        h = np.random.default_rng([seed] + [int(abs(v) * 1e6) % (2 ** 31) for v in key]).standard_normal()
        return float(-np.sum((np.log(fc) - np.log(0.1)) ** 2) + scale * h)
    return obj


CASES = {
    'sinc2_fine': dict(d=2, kinds=['sinc', 'sinc'], periods_scaled=[None, None],
                       kw=dict(fc0=0.008, factors=F3), obj=bowl([0.11, 0.07])),
    'sinc3_rugged_cap': dict(d=3, kinds=['sinc'] * 3, periods_scaled=[None] * 3,
                             kw=dict(fc0=0.2, factors=(R2,)), obj=bowl([0.3, 0.45, 0.12], cap=0.5, ripple=0.03)),
    'pball_group_dirichlet': dict(d=3, kinds=['pball', 'pball', 'dirichlet'], periods_scaled=[None, None, 23.0],
                                  kw=dict(fc0=0.05, factors=(R2, 2.0 ** 0.25)),
                                  obj=bowl([0.2, 0.2, 0.31], weight=[1.0, 1.0, 3.0])),
    'start_free': dict(d=3, kinds=['sinc'] * 3, periods_scaled=[None] * 3,
                       kw=dict(fc0=0.02, factors=(R2, 2.0 ** 0.25), start=[np.nan, 0.09, 0.05],
                               free=[True, False, True]), obj=bowl([0.15, 0.2, 0.03])),
    'ball_tags': dict(d=5, kinds=['ball:a', 'ball:a', 'sinc', 'ball:b', 'ball:b'], periods_scaled=[None] * 5,
                      kw=dict(fc0=0.1, factors=(R2,), patience=1, max_sweeps=4),
                      obj=bowl([0.4, 0.4, 0.05, 0.2, 0.2], ripple=0.02)),
    'dirichlet_down': dict(d=2, kinds=['dirichlet', 'dirichlet'], periods_scaled=[16.0, 31.0],
                           kw=dict(fc0=0.3, factors=(R2,)), obj=bowl([0.01, 0.02])),
    'flat_noise': dict(d=1, kinds=['sinc'], periods_scaled=[None],
                       kw=dict(fc0=0.05, patience=3, max_sweeps=4, factors=(R2, 2.0 ** 0.25)),
                       obj=hashed(7, 0.5)),
}


def first_mode_fc(modes, d):
    """fc per column of the first mode (a tuple key gives its value to each of its columns)."""
    fc = np.full(d, np.nan)
    for key, c in modes[0].items():
        v = c.get('fc')
        v = v['value'] if isinstance(v, dict) else v
        for j in (key if isinstance(key, tuple) else (key,)):
            fc[j] = float(v)
    return fc


class StubQuick:
    """A deterministic stand-in for BLMLQuick in the selector tests: fit keeps the points, their weights and the first
    mode's fc per column (recorded in StubQuick.calls); predict is the weighted product-Gaussian kernel density with
    bandwidth 0.2 / fc per column. Smooth in fc, with an interior optimum of the validation log-likelihood."""
    calls = []

    def __init__(self, *a, **k):
        pass

    def fit(self, X, modes, signs=None, complex_g=False, sample_weight=None, init=None):
        X = np.atleast_2d(np.asarray(X, float))
        self.X = X
        self.sw = np.ones(len(X)) if sample_weight is None else np.asarray(sample_weight, float)
        self.fc = first_mode_fc(modes, X.shape[1])
        self.bw = 0.2 / self.fc
        StubQuick.calls.append(self.fc.copy())
        return self

    def predict(self, Xq):
        Xq = np.atleast_2d(np.asarray(Xq, float))
        z = (Xq[:, None, :] - self.X[None, :, :]) / self.bw
        k = np.exp(-0.5 * (z * z).sum(2)) / np.prod(self.bw * np.sqrt(2 * np.pi))
        return (k @ self.sw) / self.sw.sum()


SINC2 = [{0: dict(kind='sinc'), 1: dict(kind='sinc')}]
# name: (lattice shape, seed, modes template, select_counts keywords)
COUNTS_CASES = {
    'counts_default': ((24, 24), 11, SINC2, dict()),
    'counts_capped': ((20, 28), 12, SINC2, dict(fc0=2.0, fc_max=9.0, factors=(2 ** 0.5, 2 ** 0.25))),
}


def counts_lattice(shape, seed):
    """Training / validation counts on a full lattice of bin centres (h = 1 / side per column)."""
    rng = np.random.default_rng(seed)
    h = np.array([1.0 / m for m in shape])
    g = np.meshgrid(*[(np.arange(m) + 0.5) * hh for m, hh in zip(shape, h)], indexing='ij')
    Z = np.stack([x.ravel() for x in g], 1)
    p = np.exp(-0.5 * (((Z - 0.4) / 0.12) ** 2).sum(1)) + 0.5 * np.exp(-0.5 * (((Z - 0.7) / 0.06) ** 2).sum(1))
    p = p / p.sum()
    w_tr = rng.multinomial(3000, p).astype(float); w_va = rng.multinomial(800, p).astype(float)
    return Z, w_tr, w_va, h
