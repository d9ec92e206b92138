"""Certified fits on the batched engine: the certificate of every fit at once (float64 Lanczos in lockstep) against the
oracle's ARPACK certificate at the same coefficients (blml_binned.py:501-518); fits of K shared modes from a given
start against the oracle's fit from the same start; rank growth until the certificate holds, whose loglik is the
convex lift's unique optimum and so must equal the oracle's certified loglik (oracle.certified_fit)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = [((48, 48), 0.3, 2e4, 1), ((32, 64), 0.2, 1e4, 2), ((64, 48), 0.12, 3e4, 3), ((40, 40), 0.4, 5e3, 4)]


def _fits():
    from blml_b200 import workloads
    return [(workloads.two_disk_field(shape, fc=fc, N=N, seed=seed), workloads.pball_modes(shape, fc))
            for shape, fc, N, seed in CASES]


def test_batched_certificate_matches_oracle(cuda_device):
    import blml_oracle as bo
    from blml_b200.sweep import BLMLBinnedBatch
    fits = _fits()
    b = BLMLBinnedBatch(tol=1e-6, device='cuda')
    b.fit([c for c, _ in fits], [m for _, m in fits])
    cert = b.certificate()
    for f, (counts, modes) in enumerate(fits):
        o = bo.BinnedFit(tol=1e-6, solver='lbfgs', max_sweeps=0).fit(counts, modes, complex_g=True)
        o.e_hat = b.e_hat(f).cpu().numpy()
        ref = o.certificate(tol=1e-10)
        assert abs(cert[f] - ref) <= 1e-5 * ref, (f, cert[f], ref)


def test_rank_two_polish_of_oracle_optimum(cuda_device):
    """K = 2 shared modes: the oracle's rank-2 fit (from its rank-1 fit plus a small mode along the certificate's top
    eigenvector) is a stationary point; the batched engine started there stays (loglik to 1e-7, never lower). Rank-2
    fits are non-convex, so two solvers started at the same non-stationary point may end at different optima -- the
    polish test is the reference's own parity test for them (results/pball_parity.py:108-118)."""
    import blml_oracle as bo
    from blml_b200.sweep import BLMLBinnedBatch
    fits = _fits()[:2]
    starts, mods, refs = [], [], []
    for counts, modes in fits:
        o = bo.BinnedFit(tol=1e-6, solver='lbfgs').fit(counts, modes, complex_g=True)
        _, d = o.certificate_vector()
        sc = 0.1 * np.sqrt((np.abs(o.e_hat) ** 2).sum()) / np.linalg.norm(d)
        e0 = np.concatenate([o.e_hat, (sc * d)[None].astype(complex)], 0)
        o2 = bo.BinnedFit(tol=1e-6, solver='lbfgs').fit(counts, [modes[0]] * 2, complex_g=True,
                                                        init=bo._Start(e0, counts.shape))
        starts.append(o2.e_hat); mods.append([modes[0]] * 2); refs.append(o2.loglik)
    b = BLMLBinnedBatch(tol=1e-6, device='cuda')
    res = b.fit([c for c, _ in fits], mods, init=starts)
    for f in range(len(fits)):
        assert abs(res[f].loglik_ - refs[f]) <= 1e-7 * abs(refs[f]) or res[f].loglik_ > refs[f], (f, res[f].loglik_, refs[f])


def test_certified_fits_reach_the_oracle_optimum(cuda_device):
    import blml_oracle as bo
    from blml_b200.sweep import BLMLBinnedBatch
    fits = _fits()
    b = BLMLBinnedBatch(tol=1e-6, device='cuda')
    res = b.fit_certified([c for c, _ in fits], [m for _, m in fits], cert_tol=1e-4)
    for f, (counts, modes) in enumerate(fits):
        r = res[f]
        assert r.certificate_ <= 1 + 1e-4, (f, r.rank_path_)
        _, path = bo.certified_fit(counts, modes[0], cert_tol=1e-4)
        ll = path[-1][1]
        assert abs(r.loglik_ - ll) <= 1e-6 * abs(ll), (f, r.rank_path_, path)
        assert r.density_.shape == counts.shape


def test_float32_history_reaches_the_same_certified_optimum(cuda_device):
    """The L-BFGS history in complex64 storage (fit_certified's default) changes the solver's path, not the certified
    optimum: the same fits certified with a float64 history agree to 1e-6."""
    from blml_b200.sweep import BLMLBinnedBatch
    fits = _fits()
    counts, modes = [c for c, _ in fits], [m for _, m in fits]
    r32 = BLMLBinnedBatch(tol=1e-6, device='cuda').fit_certified(counts, modes, cert_tol=1e-4, history_f32=True)
    r64 = BLMLBinnedBatch(tol=1e-6, device='cuda').fit_certified(counts, modes, cert_tol=1e-4, history_f32=False)
    for f in range(len(fits)):
        assert r32[f].certificate_ <= 1 + 1e-4 and r64[f].certificate_ <= 1 + 1e-4
        assert abs(r32[f].loglik_ - r64[f].loglik_) <= 1e-6 * abs(r64[f].loglik_), (f, r32[f].rank_path_,
                                                                                      r64[f].rank_path_)


def test_two_mode_growth_reaches_the_oracle_optimum(cuda_device):
    """Growing two modes at once (the top two Ritz vectors) changes the path, not the certified optimum."""
    import blml_oracle as bo
    from blml_b200.sweep import BLMLBinnedBatch
    fits = _fits()
    b = BLMLBinnedBatch(tol=1e-6, device='cuda')
    res = b.fit_certified([c for c, _ in fits], [m for _, m in fits], cert_tol=1e-4, grow_two_above=1.0)
    assert b.certify_stats_.get('two_mode_growths', 0) > 0
    for f, (counts, modes) in enumerate(fits):
        r = res[f]
        assert r.certificate_ <= 1 + 1e-4, (f, r.rank_path_)
        _, path = bo.certified_fit(counts, modes[0], cert_tol=1e-4)
        assert abs(r.loglik_ - path[-1][1]) <= 1e-6 * abs(path[-1][1]), (f, r.rank_path_, path)
