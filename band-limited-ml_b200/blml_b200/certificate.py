"""lambda_max of D^1/2 S_0 D^1/2 by float64 Lanczos on the GPU (the certificate of BLMLBinned, blml_binned.py:501-518,
where the reference calls ARPACK's eigsh(k=1, which='LA', tol)). Full reorthogonalisation against the stored
basis (float64 multi-dot and linear-combination kernels), the tridiagonal eigenproblem on the host, restarts from the
Ritz vector. Converged when the Ritz residual |beta_j y_j| <= tol |theta|."""
import time

import numpy as np
import torch

from . import _lib
from ._lib import call, ptrs, dbl


def lanczos_max(plan, dh, red, stream, tol=1e-6, seed=0, max_basis=96, max_restarts=20):
    B = dh.numel()
    dev = dh.device
    code = _lib.F64

    def dots(pairs):
        call('blml_dots', code, B, len(pairs), ptrs([p[0] for p in pairs]), ptrs([p[1] for p in pairs]),
             red.part.data_ptr(), red.out.data_ptr(), stream)
        return red.read(len(pairs))

    def lin(terms, out):
        call('blml_lincomb', code, B, out.data_ptr(), len(terms), dbl([t[0] for t in terms]),
             ptrs([t[1] for t in terms]), stream)
        return out

    tmp = torch.empty(B, dtype=torch.float64, device=dev)

    def op(x, out):
        call('blml_mul_bins', code, 1, B, 0, x.data_ptr(), dh.data_ptr(), tmp.data_ptr(), stream)
        plan.apply(tmp, out, 1, False, stream)
        call('blml_mul_bins', code, 1, B, 0, out.data_ptr(), dh.data_ptr(), out.data_ptr(), stream)
        return out

    nb = min(max_basis, B)
    V = torch.empty((nb + 1, B), dtype=torch.float64, device=dev)
    v0 = np.random.default_rng(seed).standard_normal(B)
    V[0].copy_(torch.as_tensor(v0 / np.linalg.norm(v0)))
    theta = 0.0
    for _ in range(max_restarts + 1):
        alphas, betas = [], []
        w = torch.empty(B, dtype=torch.float64, device=dev)
        j = 0; done = False; y = None
        while j < nb:
            op(V[j], w)
            # full reorthogonalisation (twice is enough) against V[0..j]
            for _pass in range(2):
                for c0 in range(0, j + 1, 63):
                    idx = list(range(c0, min(j + 1, c0 + 63)))
                    cs = dots([(V[i], w) for i in idx])
                    if _pass == 0 and c0 <= j < c0 + 63:
                        alpha = cs[j - c0]
                    lin([(1.0, w)] + [(-cs[t], V[i]) for t, i in enumerate(idx)], w)
            alphas.append(alpha)
            beta = float(np.sqrt(max(dots([(w, w)])[0], 0.0)))
            T = np.diag(alphas) + np.diag(betas, 1) + np.diag(betas, -1)
            ev, evec = np.linalg.eigh(T)
            theta = float(ev[-1]); y = evec[:, -1]
            if abs(beta * y[-1]) <= tol * max(abs(theta), 1e-300) or beta <= 1e-14 * max(abs(theta), 1e-300):
                done = True; j += 1; break
            betas.append(beta)
            lin([(1.0 / beta, w)], V[j + 1])
            j += 1
        if done:
            return theta
        # restart from the Ritz vector of the largest Ritz value
        lin([(float(y[i]), V[i]) for i in range(len(y))], w)
        nrm = float(np.sqrt(dots([(w, w)])[0]))
        lin([(1.0 / nrm, w)], V[0])
    return theta


def lanczos_max_batched(batch, tol=1e-6, seed=0, max_basis=64, max_restarts=12, vectors=False, above=None,
                        second=False):
    """The certificate of every fit of a fitted BLMLBinnedBatch at once: lambda_max(D^1/2 S D^1/2) per fit
    (blml_binned.py:501-518), D = sum_k |e_k|^2 / w on occupied bins, by float64 Lanczos with full
    reorthogonalisation, all fits in lockstep: one grouped mat-vec, segmented inner products and linear combinations
    per step with their coefficients formed on the device (no host round trip inside a step), each fit's tridiagonal
    problem on the host (every third step, when alpha and beta are read back), restarts from the Ritz vector until
    every fit's Ritz residual |beta_j y_j| <= tol |theta|, or its Ritz value moved by less than 1e-8 relative between
    two checks (at a certified optimum the top eigenvalue is K-fold, so the residual of its Ritz vector converges far
    more slowly than the value; 1e-8 is far below any certification bar). above: per-fit thresholds; a Ritz value is
    a lower bound of lambda_max, so a fit whose Ritz value exceeds its threshold is decided there (its Ritz vector
    then has a Rayleigh quotient above the threshold: the direction a new mode takes). The steps run over the fits
    still open only: when they fall to 3/4 of the fits the steps cover, the segment list and the grouped mat-vec are
    rebuilt over them (a fit's arithmetic does not depend on which other fits share the launch). Returns (theta (F,),
    dh, v): dh the per-bin scaling and v the top Ritz vectors (float64 per bin over all fits, None unless vectors)
    -- d = dh v is the direction of a new mode. second (with vectors): v is a pair (top, next) -- the Ritz vector of
    each fit's second Ritz value from the same Krylov basis, a second ascent direction while that value is above n."""
    from .sweep import _Group, _Seg
    clock = {'wait_s': 0.0, 'host_s': 0.0}
    F, dev, st, B = batch.F, batch.device, batch.st, batch.Btot
    code = _lib.F64
    dh = torch.empty(B, dtype=torch.float64, device=dev)
    call('blml_seg_cert_weights', batch.code, F, batch.segs_t.data_ptr(), batch.E_t.data_ptr(), batch.w.data_ptr(),
         dh.data_ptr(), st)
    tmp = torch.empty(B, dtype=torch.float64, device=dev)
    sv = torch.empty(B, dtype=torch.float64, device=dev)

    class Subset:
        """The fits a launch covers: their segment list (offsets into the full vectors) and grouped mat-vec."""

        def __init__(self, idx):
            self.idx = np.asarray(idx, np.int64)
            segs = (_Seg * len(self.idx))(*[_Seg(int(batch.boff[f]), int(batch.boff[f]), int(batch.B[f]), 1, 0)
                                            for f in self.idx])
            self.segs_t = torch.frombuffer(bytearray(segs), dtype=torch.uint8).to(dev)
            off = np.asarray(batch.boff[:-1])[self.idx]
            self.grp = _Group([batch.p64[f] for f in self.idx], tmp, off, sv, off, False)

    def dots(S, pairs):
        n = len(S.idx)
        call('blml_seg_dots', code, n, S.segs_t.data_ptr(), 0, len(pairs), ptrs([p[0] for p in pairs]),
             ptrs([p[1] for p in pairs]), batch.part.data_ptr(), batch.out.data_ptr(), st)
        batch.host[:len(pairs) * n].copy_(batch.out[:len(pairs) * n], non_blocking=True)
        t0 = time.perf_counter()
        torch.cuda.current_stream(dev).synchronize()
        clock['wait_s'] += time.perf_counter() - t0
        out = np.zeros((F, len(pairs)))
        out[S.idx] = batch.host[:len(pairs) * n].numpy().reshape(n, len(pairs))
        return out

    # coefficient uploads through a ring of pinned host slots, so a linear combination does not wait for the stream
    # (a pageable copy would): a slot is reused only after the event recorded behind its copy has completed
    nring, width = 32, F * 48 + 64
    ring_h = torch.empty((nring, width), dtype=torch.float64, pin_memory=True)
    ring_d = torch.empty((nring, width), dtype=torch.float64, device=dev)
    ring_ev = [None] * nring
    slot = [0]

    def lin(S, out, coef, vecs):                     # coef (F, nterms): the rows of S's fits are used
        c = np.ascontiguousarray(np.asarray(coef, np.float64)[S.idx]).ravel()
        k = slot[0]; slot[0] = (k + 1) % nring
        if ring_ev[k] is not None:
            ring_ev[k].synchronize()
        ring_h[k, :c.size].numpy()[:] = c
        ring_d[k, :c.size].copy_(ring_h[k, :c.size], non_blocking=True)
        ev = torch.cuda.Event(); ev.record(torch.cuda.current_stream(dev)); ring_ev[k] = ev
        call('blml_seg_lincomb', code, len(S.idx), S.segs_t.data_ptr(), 0, out.data_ptr(), len(vecs),
             ring_d[k].data_ptr(), ptrs(vecs), st)

    def op(S, x, out):                               # out = dh * S (dh * x) on S's fits
        call('blml_mul_bins', code, 1, B, 0, x.data_ptr(), dh.data_ptr(), tmp.data_ptr(), st)
        S.grp(st)
        call('blml_mul_bins', code, 1, B, 0, sv.data_ptr(), dh.data_ptr(), out.data_ptr(), st)

    every = Subset(np.arange(F))
    nb = max_basis
    V = torch.empty((nb + 1, B), dtype=torch.float64, device=dev)
    V[0].copy_(torch.as_tensor(np.random.default_rng(seed).standard_normal(B)))
    nrm = dots(every, [(V[0], V[0])])[:, 0]
    lin(every, V[0], (1.0 / np.sqrt(np.maximum(nrm, 1e-300)))[:, None], [V[0]])
    theta = np.zeros(F); done = np.zeros(F, bool); prev = np.full(F, np.nan); theta2 = np.full(F, np.nan)
    above = np.full(F, np.inf) if above is None else np.asarray(above, float)
    wv = torch.empty(B, dtype=torch.float64, device=dev)
    vec = torch.zeros(B, dtype=torch.float64, device=dev) if vectors else None
    vec2 = torch.zeros(B, dtype=torch.float64, device=dev) if (vectors and second) else None
    R2 = torch.empty(B, dtype=torch.float64, device=dev) if vec2 is not None else None
    R = torch.empty(B, dtype=torch.float64, device=dev)
    # the steps themselves make no host round trip: the reorthogonalisation's coefficients and alpha / beta come from
    # the inner products on the device (blml_lanczos_coef / _beta); the host reads alpha and beta at the checks
    coef_d = torch.empty(F * 48 + 64, dtype=torch.float64, device=dev)
    bcoef_d = torch.empty(F + 64, dtype=torch.float64, device=dev)
    alpha_d = torch.zeros((nb, F), dtype=torch.float64, device=dev)
    beta_d = torch.zeros((nb, F), dtype=torch.float64, device=dev)

    def dots_dev(S, pairs):                          # inner products into batch.out (rows of S), no read
        call('blml_seg_dots', code, len(S.idx), S.segs_t.data_ptr(), 0, len(pairs), ptrs([p[0] for p in pairs]),
             ptrs([p[1] for p in pairs]), batch.part.data_ptr(), batch.out.data_ptr(), st)

    def lin_dev(S, out, cptr, vecs):
        call('blml_seg_lincomb', code, len(S.idx), S.segs_t.data_ptr(), 0, out.data_ptr(), len(vecs), cptr,
             ptrs(vecs), st)

    steps = 0
    for rnd in range(max_restarts + 1):
        alphas = np.zeros((F, nb)); betas = np.zeros((F, nb))
        conv = np.zeros(F, bool); yr = [None] * F; yr2 = [None] * F
        S = every if not done.any() else Subset(np.where(~done)[0])
        j_end = nb
        fetched = 0                                   # steps whose alpha / beta the host holds
        for j in range(nb):
            op(S, V[j], wv)
            steps += 1
            n = len(S.idx)
            for ps in range(2):                       # full reorthogonalisation against the basis, twice
                for c0 in range(0, j + 1, 47):
                    idx = list(range(c0, min(j + 1, c0 + 47)))
                    dots_dev(S, [(V[i], wv) for i in idx])
                    acol = j - c0 if (ps == 0 and c0 <= j < c0 + 47) else -1
                    call('blml_lanczos_coef', n, len(idx), batch.out.data_ptr(), coef_d.data_ptr(),
                         alpha_d[j].data_ptr() if acol >= 0 else None, acol, st)
                    lin_dev(S, wv, coef_d.data_ptr(), [wv] + [V[i] for i in idx])
            dots_dev(S, [(wv, wv)])
            call('blml_lanczos_beta', n, batch.out.data_ptr(), beta_d[j].data_ptr(), bcoef_d.data_ptr(), st)
            open_ = np.zeros(F, bool); open_[S.idx] = True
            open_ &= ~(done | conv)
            check = j == nb - 1 or (j >= 5 and j % 3 == 2)
            if check:
                t0 = time.perf_counter()
                a_h = alpha_d[fetched:j + 1, :n].cpu().numpy()
                b_h = beta_d[fetched:j + 1, :n].cpu().numpy()
                clock['wait_s'] += time.perf_counter() - t0
                alphas[S.idx, fetched:j + 1] = a_h.T
                betas[S.idx, fetched:j + 1] = b_h.T
                fetched = j + 1
                beta = betas[:, j]
                t0 = time.perf_counter()
                of = np.where(open_)[0]
                # every open fit's tridiagonal problem at once: the largest eigenpair of T_f (j + 1 square)
                T = np.zeros((len(of), j + 1, j + 1))
                ii = np.arange(j + 1)
                T[:, ii, ii] = alphas[of, :j + 1]
                T[:, ii[:-1], ii[1:]] = betas[of, :j]
                T[:, ii[1:], ii[:-1]] = betas[of, :j]
                ev_all, evec_all = np.linalg.eigh(T)
                for t_, f in enumerate(of):
                    th = float(ev_all[t_, -1]); y = evec_all[t_, :, -1].copy()
                    theta[f] = th; yr[f] = y
                    if j > 0:
                        yr2[f] = evec_all[t_, :, -2].copy(); theta2[f] = float(ev_all[t_, -2])
                    if (abs(beta[f] * y[-1]) <= tol * max(abs(th), 1e-300) or beta[f] <= 1e-14 * max(abs(th), 1e-300)
                            or th > above[f] or abs(th - prev[f]) <= 1e-8 * abs(th)):
                        conv[f] = True
                    prev[f] = th
                clock['host_s'] += time.perf_counter() - t0
                if np.all(done | conv):
                    j_end = j + 1
                    break
            lin_dev(S, V[j + 1], bcoef_d.data_ptr(), [wv])
            still = np.where(~(done | conv))[0]
            if check and j + 1 < nb and len(still) <= 0.75 * len(S.idx):
                # the steps go on over the open fits only; the converged ones keep V[0..j], all their Ritz vectors use
                S = Subset(still)
        # the Ritz vector of every fit still open at the start of this round: R = sum_i y_i V[i]
        act = ~done
        SA = Subset(np.where(act)[0])
        R.zero_()
        for c0 in range(0, j_end, 47):
            idx = list(range(c0, min(j_end, c0 + 47)))
            cf = np.zeros((F, 1 + len(idx))); cf[:, 0] = 1.0
            for f in np.where(act)[0]:
                y = yr[f]
                if y is None:
                    continue
                for t, i in enumerate(idx):
                    if i < len(y):
                        cf[f, 1 + t] = y[i]
            lin(SA, R, cf, [R] + [V[i] for i in idx])
        if vec2 is not None:                                      # the second Ritz vectors the same way
            R2.zero_()
            for c0 in range(0, j_end, 47):
                idx = list(range(c0, min(j_end, c0 + 47)))
                cf = np.zeros((F, 1 + len(idx))); cf[:, 0] = 1.0
                for f in np.where(act)[0]:
                    y = yr2[f]
                    if y is None:
                        continue
                    for t, i in enumerate(idx):
                        if i < len(y):
                            cf[f, 1 + t] = y[i]
                lin(SA, R2, cf, [R2] + [V[i] for i in idx])
        if vectors:                                               # keep the vectors of the fits converging now
            keep = (act & conv).astype(float)
            lin(SA, vec, np.stack([keep, 1.0 - keep], 1), [R, vec])
            if vec2 is not None:
                lin(SA, vec2, np.stack([keep, 1.0 - keep], 1), [R2, vec2])
        done |= conv
        if np.all(done):
            break
        SO = Subset(np.where(~done)[0])
        rn = dots(SO, [(R, R)])[:, 0]
        lin(SO, V[0], (1.0 / np.sqrt(np.maximum(rn, 1e-300)))[:, None], [R])
    if vectors:
        nv = dots(every, [(vec, vec)])[:, 0]
        lin(every, vec, (1.0 / np.sqrt(np.maximum(nv, 1e-300)))[:, None], [vec])
        if vec2 is not None:
            nv2 = dots(every, [(vec2, vec2)])[:, 0]
            lin(every, vec2, np.where(nv2 > 0, 1.0 / np.sqrt(np.maximum(nv2, 1e-300)), 0.0)[:, None], [vec2])
            vec = (vec, vec2)
    batch.theta2_ = theta2                                        # the second Ritz values (NaN: none)
    batch.lanczos_stats_ = dict(steps=steps, restarts=rnd, converged=int(done.sum()), wait_s=round(clock['wait_s'], 4),
                                host_s=round(clock['host_s'], 4))
    return theta, dh, vec
