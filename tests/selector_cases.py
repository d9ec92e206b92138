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
