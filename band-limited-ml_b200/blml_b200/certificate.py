"""lambda_max of D^1/2 S_0 D^1/2 by float64 Lanczos on the GPU (the certificate of BLMLBinned, blml_binned.py:501-518,
where the reference calls ARPACK's eigsh(k=1, which='LA', tol)). Full reorthogonalisation against the stored
basis (float64 multi-dot and linear-combination kernels), the tridiagonal eigenproblem on the host, restarts from the
Ritz vector. Converged when the Ritz residual |beta_j y_j| <= tol |theta|."""
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
