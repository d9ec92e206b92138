// The bin-wise solver kernels of the binned fit: coordinate update, merit / residual / likelihood reductions,
// inner products and linear combinations, start and finish. All are bandwidth-bound single passes over the
// (K, B) mode arrays with grid-stride loops; per-bin arithmetic is done in float64 whatever the storage type and
// every sum is a deterministic float64 block reduction (block partials + a fixed-order finish).
#include "common.cuh"

namespace blml {

struct SArr { double v[16]; };         // K(0) of each mode, passed by value

template <typename T, bool CPLX>
struct Acc {
  // element (k, b) of a (K, B) mode array as complex doubles
  static __device__ __forceinline__ void get(const void* p, int64_t i, double& re, double& im) {
    if (CPLX) { const cpx<T> v = reinterpret_cast<const cpx<T>*>(p)[i]; re = (double)v.re; im = (double)v.im; }
    else { re = (double)reinterpret_cast<const T*>(p)[i]; im = 0.0; }
  }
  static __device__ __forceinline__ void put(void* p, int64_t i, double re, double im) {
    if (CPLX) reinterpret_cast<cpx<T>*>(p)[i] = cpx<T>{(T)re, (T)im};
    else reinterpret_cast<T*>(p)[i] = (T)re;
  }
};

__device__ __forceinline__ double cd_root_d(double b, double c, double s) {
  const double disc = sqrt(b * b + 4.0 * s * c);
  return b >= 0 ? 2.0 * c / fmax(b + disc, 1e-300) : (-b + disc) / (2.0 * s);
}

#define GRID_STRIDE(b, B) for (int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; b < (B); \
                               b += (int64_t)gridDim.x * blockDim.x)

static inline int grid_for(int64_t n) {
  int64_t g = (n + 255) / 256;
  return (int)std::min<int64_t>(std::max<int64_t>(g, 1), 148 * 16);
}

// ---------------------------------------------------------------------------------------------- update
template <typename T>
__global__ void k_update_real1(int64_t B, const T* E, const T* U, const T* c, const T* sg, double s0, T* out) {
  GRID_STRIDE(b, B) {
    const double cb = (double)c[b], sgb = (double)sg[b];
    double t = 0.0;
    if (cb > 0) t = cd_root_d(sgb * ((double)U[b] - s0 * (double)E[b]), cb, s0);
    out[b] = (T)(sgb * t);
  }
}

// psd update, every s_k equal: e_b = R_b t / |R_b|, t = 2 c / (|R| + sqrt(|R|^2 + 4 s c)); a bin with c > 0 and
// R = 0 puts mode 0 at sqrt(c / s) (blml_binned.py:196-203)
template <typename T, bool CPLX>
__global__ void k_update_psd_eq(int K, int64_t B, const void* E, const void* U, const T* c, double s0, void* out) {
  GRID_STRIDE(b, B) {
    const double cb = (double)c[b];
    double a2 = 0.0;
    for (int k = 0; k < K; k++) {
      double er, ei, ur, ui;
      Acc<T, CPLX>::get(E, k * B + b, er, ei); Acc<T, CPLX>::get(U, k * B + b, ur, ui);
      const double rr = ur - s0 * er, ri = ui - s0 * ei;
      a2 += rr * rr + ri * ri;
    }
    const double a = sqrt(a2);
    const double t = 2.0 * cb / (a + sqrt(a2 + 4.0 * s0 * cb));
    const double f = t / (a > 0 ? a : 1.0);
    const bool lone = (a == 0.0) && (cb > 0);
    for (int k = 0; k < K; k++) {
      double er, ei, ur, ui;
      Acc<T, CPLX>::get(E, k * B + b, er, ei); Acc<T, CPLX>::get(U, k * B + b, ur, ui);
      double vr = (ur - s0 * er) * f, vi = (ui - s0 * ei) * f;
      if (lone && k == 0) { vr = sqrt(cb / s0); vi = 0.0; }
      Acc<T, CPLX>::put(out, k * B + b, vr, vi);
    }
  }
}

// psd update, unequal s_k: e_bk = R_bk / (lam_b - s_k), lam_b > max s the root of lam sum |R_k|^2/(lam - s_k)^2 = c,
// 16 safeguarded Newton steps on phi^(-1/2) in mu = lam - max s (blml_binned.py:1556-1573)
template <typename T, bool CPLX>
__global__ void k_update_psd_sec(int K, int64_t B, const void* E, const void* U, const T* c, SArr s, void* out) {
  GRID_STRIDE(b, B) {
    const double cb = (double)c[b];
    double R2[16], smax = s.v[0];
    for (int k = 1; k < K; k++) smax = fmax(smax, s.v[k]);
    double tot = 0.0;
    for (int k = 0; k < K; k++) {
      double er, ei, ur, ui;
      Acc<T, CPLX>::get(E, k * B + b, er, ei); Acc<T, CPLX>::get(U, k * B + b, ur, ui);
      const double rr = ur - s.v[k] * er, ri = ui - s.v[k] * ei;
      R2[k] = rr * rr + ri * ri; tot += R2[k];
    }
    const double cp = fmax(cb, 1e-30);
    double hi = (tot + sqrt(tot * tot + 4 * cp * smax * tot)) / (2 * cp), lo = 0.0, mu = hi;
    for (int it = 0; it < 16; it++) {
      double A = 0.0, Bq = 0.0;
      for (int k = 0; k < K; k++) {
        const double q = 1.0 / (mu - (s.v[k] - smax));
        const double w = R2[k] * q * q; A += w; Bq += w * q;
      }
      const double lam = smax + mu, phi = lam * A;
      const bool big = phi > cb;
      if (big) lo = mu; else hi = mu;
      const double nt = mu + 2 * phi * (1 - sqrt(phi / cp)) / (A - 2 * lam * Bq);
      mu = (nt >= lo && nt <= hi) ? nt : 0.5 * (lo + hi);     // NaN steps fail the test and bisect
    }
    const double lam = smax + mu;
    const bool lone = (tot == 0.0) && (cb > 0);
    for (int k = 0; k < K; k++) {
      double er, ei, ur, ui;
      Acc<T, CPLX>::get(E, k * B + b, er, ei); Acc<T, CPLX>::get(U, k * B + b, ur, ui);
      double vr = 0.0, vi = 0.0;
      if (cb > 0 && !lone) { const double f = 1.0 / (lam - s.v[k]); vr = (ur - s.v[k] * er) * f; vi = (ui - s.v[k] * ei) * f; }
      if (lone && k == 0) { vr = sqrt(cb / s.v[0]); vi = 0.0; }
      Acc<T, CPLX>::put(out, k * B + b, vr, vi);
    }
  }
}

// ---------------------------------------------------------------------------------------------- reductions
template <typename T, bool CPLX>
__global__ void k_merit_psd(int K, int64_t B, const void* E, const void* U, const T* c, double* part) {
  double v[3] = {0.0, 0.0, 0.0};
  GRID_STRIDE(b, B) {
    double F = 0.0, Q = 0.0;
    for (int k = 0; k < K; k++) {
      double er, ei, ur, ui;
      Acc<T, CPLX>::get(E, k * B + b, er, ei); Acc<T, CPLX>::get(U, k * B + b, ur, ui);
      F += ur * ur + ui * ui; Q += er * ur + ei * ui;
    }
    const double cb = (double)c[b];
    if (cb != 0.0) v[0] += cb * log(fmax(F, 1e-30));
    v[1] += Q;
  }
  block_partials<3>(v, part);
}

template <typename T>
__global__ void k_merit_real(int64_t B, const T* E, const T* U, const T* c, const T* sg, double* part) {
  double v[3] = {0.0, 0.0, 0.0};
  GRID_STRIDE(b, B) {
    const double e = (double)E[b], cb = (double)c[b];
    v[0] += e * (double)U[b];
    if (cb > 0) {
      v[1] += cb * log(fabs(e));
      if ((double)sg[b] * e <= 0) v[2] += 1.0;
    }
  }
  block_partials<3>(v, part);
}

template <typename T, bool CPLX>
__global__ void k_resid(int K, int64_t B, const void* E, const void* U, const T* c, double sc, double* part) {
  double v[2] = {0.0, 0.0};
  GRID_STRIDE(b, B) {
    const double cb = (double)c[b];
    if (!(cb > 0)) continue;
    double nrm2 = 0.0;
    for (int k = 0; k < K; k++) {
      double er, ei; Acc<T, CPLX>::get(E, k * B + b, er, ei);
      er *= sc; ei *= sc; nrm2 += er * er + ei * ei;
    }
    const double f = nrm2 / cb;
    double r2 = 0.0;
    for (int k = 0; k < K; k++) {
      double er, ei, ur, ui;
      Acc<T, CPLX>::get(E, k * B + b, er, ei); Acc<T, CPLX>::get(U, k * B + b, ur, ui);
      const double dr = ur * sc * f - er * sc, di = ui * sc * f - ei * sc;
      r2 += dr * dr + di * di;
    }
    const double r = sqrt(r2) / sqrt(fmax(nrm2, 1e-300));
    if (r != r) v[1] += 1.0;         // NaN residuals are counted (fmax would drop them)
    else v[0] = fmax(v[0], r);
  }
  block_partials<2>(v, part, 1u);
}

// L-BFGS trial point: En = E + t q, Un = U + t Sq (S is linear, so the trial costs no mat-vec), written out, with
// out[0] = sum_occ w log F(Un) and out[1] = Re <En, Un>
template <typename T, bool CPLX>
__global__ void k_lbfgs_trial(int K, int64_t B, const void* E, const void* q, const void* U, const void* Sq,
                              const T* w, double t, void* En, void* Un, double* part) {
  double v[2] = {0.0, 0.0};
  GRID_STRIDE(b, B) {
    double F = 0.0, Q = 0.0;
    for (int k = 0; k < K; k++) {
      double er, ei, qr, qi, ur, ui, sr, si;
      const int64_t i = k * B + b;
      Acc<T, CPLX>::get(E, i, er, ei); Acc<T, CPLX>::get(q, i, qr, qi);
      Acc<T, CPLX>::get(U, i, ur, ui); Acc<T, CPLX>::get(Sq, i, sr, si);
      double nr = er + t * qr, ni = ei + t * qi, mr = ur + t * sr, mi = ui + t * si;
      Acc<T, CPLX>::put(En, i, nr, ni); Acc<T, CPLX>::put(Un, i, mr, mi);
      Acc<T, CPLX>::get(En, i, nr, ni); Acc<T, CPLX>::get(Un, i, mr, mi);   // the stored (rounded) values
      F += mr * mr + mi * mi; Q += nr * mr + ni * mi;
    }
    const double wb = (double)w[b];
    if (wb > 0) v[0] += wb * log(F);
    v[1] += Q;
  }
  block_partials<2>(v, part);
}

// held-out / prequential score: out[0] = sum_{m > 0} m log max(F inv_z + eps, 1e-300), out[1] = sum m
template <typename T, bool CPLX>
__global__ void k_log_score(int K, int64_t B, const void* U, const T* m, double inv_z, double eps, double* part) {
  double v[2] = {0.0, 0.0};
  GRID_STRIDE(b, B) {
    const double mb = (double)m[b];
    if (!(mb > 0)) continue;
    double F = 0.0;
    for (int k = 0; k < K; k++) { double ur, ui; Acc<T, CPLX>::get(U, k * B + b, ur, ui); F += ur * ur + ui * ui; }
    v[0] += mb * log(fmax(F * inv_z + eps, 1e-300));
    v[1] += mb;
  }
  block_partials<2>(v, part);
}

struct PtrPairs { const void* a[32]; const void* b[32]; };

template <typename T, int NP>
__global__ void k_dots(int64_t n, int np, PtrPairs pp, double* part) {
  double v[NP];
#pragma unroll
  for (int q = 0; q < NP; q++) v[q] = 0.0;
  GRID_STRIDE(i, n) {
#pragma unroll
    for (int q = 0; q < NP; q++)
      if (q < np) v[q] += (double)reinterpret_cast<const T*>(pp.a[q])[i] * (double)reinterpret_cast<const T*>(pp.b[q])[i];
  }
  block_partials<NP>(v, part);
}

struct Terms { double c[64]; const void* v[64]; };

template <typename T>
__global__ void k_lincomb(int64_t n, T* out, int nt, Terms t) {
  GRID_STRIDE(i, n) {
    double acc = 0.0;
    for (int q = 0; q < nt; q++) acc += t.c[q] * (double)reinterpret_cast<const T*>(t.v[q])[i];
    out[i] = (T)acc;
  }
}

template <typename T, bool CPLX>
__global__ void k_mul_bins(int K, int64_t B, const void* x, const T* r, void* out) {
  GRID_STRIDE(b, B) {
    const double rb = (double)r[b];
    for (int k = 0; k < K; k++) {
      double xr, xi; Acc<T, CPLX>::get(x, k * B + b, xr, xi);
      Acc<T, CPLX>::put(out, k * B + b, xr * rb, xi * rb);
    }
  }
}

template <typename T, bool CPLX>
__global__ void k_lgrad_weights(int K, int64_t B, const void* U, const T* w, double vs, void* V, double* part) {
  double v[1] = {0.0};
  GRID_STRIDE(b, B) {
    double F = 0.0;
    for (int k = 0; k < K; k++) { double ur, ui; Acc<T, CPLX>::get(U, k * B + b, ur, ui); F += ur * ur + ui * ui; }
    const double wb = (double)w[b];
    const bool occ = wb > 0;
    if (occ) v[0] += wb * log(F);
    const double f = occ ? vs * wb / F : 0.0;
    for (int k = 0; k < K; k++) {
      double ur, ui; Acc<T, CPLX>::get(U, k * B + b, ur, ui);
      Acc<T, CPLX>::put(V, k * B + b, occ ? ur * f : 0.0, occ ? ui * f : 0.0);
    }
  }
  block_partials<1>(v, part);
}

// ---------------------------------------------------------------------------------------------- fc gradients
// blml_binned.py:543-628: the weights of the score sum m log(F / Z + eps) / sum m, the Hessian's bin-wise inner term
// and the mixed (d grad / dlog fc) terms, on occupied bins only (w > 0), float64 arithmetic per bin.
template <typename T, bool CPLX>
__global__ void k_pgrad_weights(int K, int64_t B, const void* U, const T* m, double add, void* V, double* part) {
  double v[2] = {0.0, 0.0};
  GRID_STRIDE(b, B) {
    double F = 0.0;
    for (int k = 0; k < K; k++) { double ur, ui; Acc<T, CPLX>::get(U, k * B + b, ur, ui); F += ur * ur + ui * ui; }
    const double mb = (double)m[b];
    const double wn = mb > 0 ? mb / fmax(F + add, 1e-300) : 0.0;
    v[0] += wn * F; v[1] += mb;
    for (int k = 0; k < K; k++) {
      double ur, ui; Acc<T, CPLX>::get(U, k * B + b, ur, ui);
      Acc<T, CPLX>::put(V, k * B + b, wn * ur, wn * ui);
    }
  }
  block_partials<2>(v, part);
}

// out_j = (w / F) dU_j - (w dF / F^2) U_j, dF = 2 Re sum_j conj(U_j) dU_j (0 off the occupied bins)
template <typename T, bool CPLX>
__global__ void k_hvp_inner(int K, int64_t B, const void* U, const void* dU, const T* w, void* out) {
  GRID_STRIDE(b, B) {
    const double wb = (double)w[b];
    double F = 0.0, dF = 0.0;
    for (int k = 0; k < K; k++) {
      double ur, ui, dr, di;
      Acc<T, CPLX>::get(U, k * B + b, ur, ui); Acc<T, CPLX>::get(dU, k * B + b, dr, di);
      F += ur * ur + ui * ui; dF += 2.0 * (ur * dr + ui * di);
    }
    const bool occ = wb > 0;
    const double a = occ ? wb / F : 0.0, c = occ ? wb * dF / (F * F) : 0.0;
    for (int k = 0; k < K; k++) {
      double ur, ui, dr, di;
      Acc<T, CPLX>::get(U, k * B + b, ur, ui); Acc<T, CPLX>::get(dU, k * B + b, dr, di);
      Acc<T, CPLX>::put(out, k * B + b, a * dr - c * ur, a * di - c * ui);
    }
  }
}

// for mode kk moved by dUk = dS E_kk: T_j = -(w dF / F^2) U_j (+ (w / F) dUk for j = kk) and Wk = (w / F) U_kk,
// dF = 2 Re conj(U_kk) dUk (0 off the occupied bins)
template <typename T, bool CPLX>
__global__ void k_mixed_terms(int K, int64_t B, const void* U, int kk, const void* dUk, const T* w, void* Tout,
                              void* Wk) {
  GRID_STRIDE(b, B) {
    const double wb = (double)w[b];
    double F = 0.0;
    for (int k = 0; k < K; k++) { double ur, ui; Acc<T, CPLX>::get(U, k * B + b, ur, ui); F += ur * ur + ui * ui; }
    double kr, ki, dr, di;
    Acc<T, CPLX>::get(U, kk * B + b, kr, ki); Acc<T, CPLX>::get(dUk, b, dr, di);
    const bool occ = wb > 0;
    const double ws = occ ? wb / F : 0.0, wd = occ ? wb * 2.0 * (kr * dr + ki * di) / (F * F) : 0.0;
    for (int k = 0; k < K; k++) {
      double ur, ui; Acc<T, CPLX>::get(U, k * B + b, ur, ui);
      double tr = -wd * ur, ti = -wd * ui;
      if (k == kk) { tr += ws * dr; ti += ws * di; }
      Acc<T, CPLX>::put(Tout, k * B + b, tr, ti);
    }
    Acc<T, CPLX>::put(Wk, b, ws * kr, ws * ki);
  }
}

// the real rank-1 objective's Hessian times D: dU + (c / e^2) D on occupied bins (c = n w > 0)
template <typename T>
__global__ void k_hvp_real1(int64_t B, const T* D, const T* E, const T* c, const T* dU, T* out) {
  GRID_STRIDE(b, B) {
    const double cb = (double)c[b], e = (double)E[b];
    out[b] = (T)((double)dU[b] + (cb > 0 ? cb / (e * e) : 0.0) * (double)D[b]);
  }
}

// ---------------------------------------------------------------------------------------------- streaming
// blml_binned.py:1040-1112 (BLMLBinnedStreaming): count updates, leave-batch-out shares, the start of newly occupied
// bins and the paired log-density gains of a hill-climb candidate (blml_binned.py:752-770).
template <typename T>
__global__ void k_counts_axpy(int64_t B, double a, const T* w, double b, const T* m, int clamp, T* out) {
  GRID_STRIDE(i, B) {
    double v = a * (double)w[i] + b * (double)m[i];
    out[i] = (T)(clamp && !(v > 0) ? 0.0 : v);
  }
}

template <typename T>
__global__ void k_bin_ratio(int64_t B, const T* num, const T* den, T* out) {
  GRID_STRIDE(i, B) {
    const double d = (double)den[i];
    out[i] = (T)(d > 0 ? (double)num[i] / d : 0.0);
  }
}

// out_k = Eu_k on occupied bins whose coefficients are all zero (newly occupied), E_k elsewhere
template <typename T, bool CPLX>
__global__ void k_new_bins(int K, int64_t B, const void* E, const void* Eu, const T* w, void* out) {
  GRID_STRIDE(b, B) {
    double a = 0.0;
    for (int k = 0; k < K; k++) { double er, ei; Acc<T, CPLX>::get(E, k * B + b, er, ei); a += fabs(er) + fabs(ei); }
    const bool fresh = (double)w[b] > 0 && a == 0.0;
    for (int k = 0; k < K; k++) {
      double er, ei; Acc<T, CPLX>::get(fresh ? Eu : E, k * B + b, er, ei);
      Acc<T, CPLX>::put(out, k * B + b, er, ei);
    }
  }
}

// on bins with m > 0: dl = log(da sa + eps) - log(db sb + eps); sums m dl, m dl^2, m
template <typename T>
__global__ void k_gain_sums(int64_t B, const T* da, double sa, const T* db, double sb, const T* m, double eps,
                            double* part) {
  double v[3] = {0.0, 0.0, 0.0};
  GRID_STRIDE(i, B) {
    const double mi = (double)m[i];
    if (mi > 0) {
      const double dl = log((double)da[i] * sa + eps) - log((double)db[i] * sb + eps);
      v[0] += mi * dl; v[1] += mi * dl * dl; v[2] += mi;
    }
  }
  block_partials<3>(v, part);
}

// ---------------------------------------------------------------------------------------------- block CD
// The block coordinate descent of the point / lattice fits (blml_trivial.py:2860-3035): a block I of bins takes its
// coordinates' exact roots together, S e follows by one rows pass of every bin against the block, and a safeguarded
// step searches t in 2^-k (cd_line_search, blml_trivial.py:92-104). State e, S e and c = n w in float64; the block's
// bin indices are checked against B (an index outside is skipped).
constexpr int kLsSteps = 31;

__global__ void k_block_root(int m, const int64_t* I, int64_t B, const double* e, const double* Se, const double* c,
                             double sbb, double* d) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < m; j += gridDim.x * blockDim.x) {
    const int64_t b = I[j];
    if (b < 0 || b >= B) { d[j] = 0.0; continue; }
    const double eb = e[b];
    d[j] = cd_root_d(Se[b] - sbb * eb, c[b], sbb) - eb;
  }
}

// one block: out[0] = d . Se[I], out[1] = d . v[I], out[2] = bins with e > 0, out[3 + k] = sum_{e > 0} c log1p(t_k r),
// out[3 + 31 + k] = bins with 1 + t_k r <= 0, r = d / e, t_k = 2^-k
__global__ void __launch_bounds__(256) k_block_search(int m, const int64_t* I, int64_t B, const double* e,
                                                     const double* d, const double* Se, const double* v,
                                                     const double* c, double* out) {
  constexpr int NQ = 3 + 2 * kLsSteps;
  double q[NQ];
#pragma unroll
  for (int k = 0; k < NQ; k++) q[k] = 0.0;
  for (int j = threadIdx.x; j < m; j += blockDim.x) {
    const int64_t b = I[j];
    if (b < 0 || b >= B) continue;
    const double dj = d[j], eb = e[b];
    q[0] += dj * Se[b]; q[1] += dj * v[b];
    if (eb > 0) {
      q[2] += 1.0;
      const double r = dj / eb, cc = c[b];
      double t = 1.0;
#pragma unroll
      for (int k = 0; k < kLsSteps; k++) {
        if (1.0 + t * r > 0) q[3 + k] += cc * log1p(t * r);
        else q[3 + kLsSteps + k] += 1.0;
        t *= 0.5;
      }
    }
  }
  __shared__ double sh[8][NQ];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < NQ; k++) {
    const double x = warp_sum(q[k]);
    if (lane == 0) sh[wid][k] = x;
  }
  __syncthreads();
  const int nw = blockDim.x >> 5;
  for (int k = threadIdx.x; k < NQ; k += blockDim.x) {
    double s = 0.0;
    for (int w = 0; w < nw; w++) s += sh[w][k];
    out[k] = s;
  }
}

__global__ void k_block_apply(int m, const int64_t* I, int64_t B, const double* d, double t, double* e) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < m; j += gridDim.x * blockDim.x) {
    const int64_t b = I[j];
    if (b >= 0 && b < B) e[b] += t * d[j];
  }
}

__global__ void k_gather_rows_i64(int m, int d, const int64_t* src, const int64_t* I, int64_t B, int64_t* out) {
  for (int64_t x = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; x < (int64_t)m * d;
       x += (int64_t)gridDim.x * blockDim.x) {
    const int64_t j = x / d, k = x % d, b = I[j];
    out[x] = (b >= 0 && b < B) ? src[b * d + k] : 0;
  }
}

template <typename T, bool CPLX>
__global__ void k_lgrad_finish(int K, int64_t B, const void* SV, const void* U, const T* w, double nq, void* g) {
  GRID_STRIDE(b, B) {
    const bool occ = (double)w[b] > 0;
    for (int k = 0; k < K; k++) {
      double sr, si, ur, ui;
      Acc<T, CPLX>::get(SV, k * B + b, sr, si); Acc<T, CPLX>::get(U, k * B + b, ur, ui);
      Acc<T, CPLX>::put(g, k * B + b, occ ? 2.0 * (sr - nq * ur) : 0.0, occ ? 2.0 * (si - nq * ui) : 0.0);
    }
  }
}

template <typename T, bool CPLX>
__global__ void k_finish(int K, int64_t B, const void* U, const T* w, double inv_n2, T* dens, double* part) {
  double v[1] = {0.0};
  GRID_STRIDE(b, B) {
    double F = 0.0;
    for (int k = 0; k < K; k++) { double ur, ui; Acc<T, CPLX>::get(U, k * B + b, ur, ui); F += ur * ur + ui * ui; }
    const T dv = (T)(F * inv_n2);
    dens[b] = dv;
    const double wb = (double)w[b];
    if (wb > 0) v[0] += wb * log((double)dv);
  }
  block_partials<1>(v, part);
}

template <typename T>
__global__ void k_start_root(int64_t B, const T* c, const T* sg, double s0, T* e0) {
  GRID_STRIDE(b, B) {
    const double cb = (double)c[b];
    e0[b] = (T)(cb > 0 ? sqrt(cb / s0) * (double)sg[b] : 0.0);
  }
}

template <typename T, bool CPLX>
__global__ void k_fill_modes(int K, int64_t B, int kk, int phases, double pn, const double* z, void* E) {
  GRID_STRIDE(b, B) {
    double e0r, e0i; Acc<T, CPLX>::get(E, b, e0r, e0i);
    int64_t zo = 0;
    if (CPLX && phases) {
      double sn, cs; sincos(pn * z[b], &sn, &cs);
      const double nr = e0r * cs - e0i * sn, ni = e0r * sn + e0i * cs;
      e0r = nr; e0i = ni;
      Acc<T, CPLX>::put(E, b, e0r, e0i);
      zo = B;
    }
    // |E[0]| after the phases (the reference reads E[0] after multiplying it)
    double er0, ei0; Acc<T, CPLX>::get(E, b, er0, ei0);
    const double mag = sqrt(er0 * er0 + ei0 * ei0);
    for (int k = kk; k < K; k++) {
      const int64_t base = zo + (int64_t)(k - kk) * (CPLX ? 2 : 1) * B;
      if (CPLX) {
        const double s2 = 1.0 / sqrt(2.0);
        Acc<T, CPLX>::put(E, k * B + b, pn * mag * z[base + b] * s2, pn * mag * z[base + B + b] * s2);
      } else {
        Acc<T, CPLX>::put(E, k * B + b, pn * mag * z[base + b], 0.0);
      }
    }
  }
}

template <typename T, bool CPLX>
__global__ void k_cert_weights(int K, int64_t B, const void* E, const T* w, double* dh) {
  GRID_STRIDE(b, B) {
    const double wb = (double)w[b];
    double s = 0.0;
    for (int k = 0; k < K; k++) { double er, ei; Acc<T, CPLX>::get(E, k * B + b, er, ei); s += er * er + ei * ei; }
    dh[b] = wb > 0 ? sqrt(s / wb) : 0.0;
  }
}

template <typename T>
static void launch_dots(int64_t n, int np, const PtrPairs& pp, double* part, cudaStream_t st) {
  if (np <= 1) k_dots<T, 1><<<kRedBlocks, kRedThreads, 0, st>>>(n, np, pp, part);
  else if (np <= 2) k_dots<T, 2><<<kRedBlocks, kRedThreads, 0, st>>>(n, np, pp, part);
  else if (np <= 4) k_dots<T, 4><<<kRedBlocks, kRedThreads, 0, st>>>(n, np, pp, part);
  else if (np <= 8) k_dots<T, 8><<<kRedBlocks, kRedThreads, 0, st>>>(n, np, pp, part);
  else if (np <= 16) k_dots<T, 16><<<kRedBlocks, kRedThreads, 0, st>>>(n, np, pp, part);
  else k_dots<T, 32><<<kRedBlocks, kRedThreads, 0, st>>>(n, np, pp, part);
}

}  // namespace blml

using namespace blml;

#define ST reinterpret_cast<cudaStream_t>(stream)
#define DISPATCH_TC(dtype, cplx, F, ...)                                   \
  do {                                                                     \
    if (dtype == BLML_F64) { if (cplx) F<double, true>__VA_ARGS__; else F<double, false>__VA_ARGS__; } \
    else { if (cplx) F<float, true>__VA_ARGS__; else F<float, false>__VA_ARGS__; }                   \
  } while (0)

static int check_dtype(int dtype, const char* who) {
  if (dtype != BLML_F64 && dtype != BLML_F32) { set_error("%s: dtype", who); return BLML_ERR_ARG; }
  return BLML_OK;
}

extern "C" {

int blml_jacobi_update(int dtype, int K, int64_t B, int cplx, int psd, const double* s, const void* E, const void* U,
                       const void* c, const void* sg, void* out, void* stream) {
  if (check_dtype(dtype, "blml_jacobi_update")) return BLML_ERR_ARG;
  if (K < 1 || K > 16 || B < 0 || !s) { set_error("blml_jacobi_update: K in 1..16"); return BLML_ERR_ARG; }
  if (B == 0) return BLML_OK;
  const int g = grid_for(B);
  if (!psd) {
    if (K != 1 || cplx) { set_error("blml_jacobi_update: real rank 1 takes K = 1 real"); return BLML_ERR_ARG; }
    if (dtype == BLML_F64) k_update_real1<double><<<g, 256, 0, ST>>>(B, (const double*)E, (const double*)U,
                                                                     (const double*)c, (const double*)sg, s[0], (double*)out);
    else k_update_real1<float><<<g, 256, 0, ST>>>(B, (const float*)E, (const float*)U, (const float*)c,
                                                  (const float*)sg, s[0], (float*)out);
  } else {
    bool equal = true;
    for (int k = 1; k < K; k++) equal = equal && fabs(s[k] - s[0]) <= 1e-8 * fabs(s[0]) + 1e-8;   // np.allclose
    if (equal) {
      if (dtype == BLML_F64) {
        if (cplx) k_update_psd_eq<double, true><<<g, 256, 0, ST>>>(K, B, E, U, (const double*)c, s[0], out);
        else k_update_psd_eq<double, false><<<g, 256, 0, ST>>>(K, B, E, U, (const double*)c, s[0], out);
      } else {
        if (cplx) k_update_psd_eq<float, true><<<g, 256, 0, ST>>>(K, B, E, U, (const float*)c, s[0], out);
        else k_update_psd_eq<float, false><<<g, 256, 0, ST>>>(K, B, E, U, (const float*)c, s[0], out);
      }
    } else {
      SArr sa; for (int k = 0; k < 16; k++) sa.v[k] = k < K ? s[k] : 0.0;
      if (dtype == BLML_F64) {
        if (cplx) k_update_psd_sec<double, true><<<g, 256, 0, ST>>>(K, B, E, U, (const double*)c, sa, out);
        else k_update_psd_sec<double, false><<<g, 256, 0, ST>>>(K, B, E, U, (const double*)c, sa, out);
      } else {
        if (cplx) k_update_psd_sec<float, true><<<g, 256, 0, ST>>>(K, B, E, U, (const float*)c, sa, out);
        else k_update_psd_sec<float, false><<<g, 256, 0, ST>>>(K, B, E, U, (const float*)c, sa, out);
      }
    }
  }
  BLML_CHECK_LAUNCH("blml_jacobi_update");
  return BLML_OK;
}

int blml_merit_terms(int dtype, int K, int64_t B, int cplx, int psd, const void* E, const void* U, const void* c,
                     const void* sg, double* part, double* out, void* stream) {
  if (check_dtype(dtype, "blml_merit_terms")) return BLML_ERR_ARG;
  if (psd) {
    if (dtype == BLML_F64) {
      if (cplx) k_merit_psd<double, true><<<kRedBlocks, kRedThreads, 0, ST>>>(K, B, E, U, (const double*)c, part);
      else k_merit_psd<double, false><<<kRedBlocks, kRedThreads, 0, ST>>>(K, B, E, U, (const double*)c, part);
    } else {
      if (cplx) k_merit_psd<float, true><<<kRedBlocks, kRedThreads, 0, ST>>>(K, B, E, U, (const float*)c, part);
      else k_merit_psd<float, false><<<kRedBlocks, kRedThreads, 0, ST>>>(K, B, E, U, (const float*)c, part);
    }
  } else {
    if (dtype == BLML_F64)
      k_merit_real<double><<<kRedBlocks, kRedThreads, 0, ST>>>(B, (const double*)E, (const double*)U, (const double*)c,
                                                               (const double*)sg, part);
    else
      k_merit_real<float><<<kRedBlocks, kRedThreads, 0, ST>>>(B, (const float*)E, (const float*)U, (const float*)c,
                                                              (const float*)sg, part);
  }
  BLML_CHECK_LAUNCH("blml_merit_terms");
  return finish_partials(part, 3, kRedBlocks, 0u, out, ST);
}

int blml_resid(int dtype, int K, int64_t B, int cplx, const void* E, const void* U, const void* c, double scale,
               double* part, double* out, void* stream) {
  if (check_dtype(dtype, "blml_resid")) return BLML_ERR_ARG;
  if (dtype == BLML_F64) {
    if (cplx) k_resid<double, true><<<kRedBlocks, kRedThreads, 0, ST>>>(K, B, E, U, (const double*)c, scale, part);
    else k_resid<double, false><<<kRedBlocks, kRedThreads, 0, ST>>>(K, B, E, U, (const double*)c, scale, part);
  } else {
    if (cplx) k_resid<float, true><<<kRedBlocks, kRedThreads, 0, ST>>>(K, B, E, U, (const float*)c, scale, part);
    else k_resid<float, false><<<kRedBlocks, kRedThreads, 0, ST>>>(K, B, E, U, (const float*)c, scale, part);
  }
  BLML_CHECK_LAUNCH("blml_resid");
  return finish_partials(part, 2, kRedBlocks, 1u, out, ST);
}

int blml_dots(int dtype, int64_t n, int npairs, const void* const* a, const void* const* b, double* part,
              double* out, void* stream) {
  if (check_dtype(dtype, "blml_dots")) return BLML_ERR_ARG;
  if (npairs < 1 || npairs > 64 || !a || !b) { set_error("blml_dots: 1..64 pairs"); return BLML_ERR_ARG; }
  for (int q0 = 0; q0 < npairs; q0 += 32) {          // 32 accumulators per pass
    const int np = std::min(32, npairs - q0);
    PtrPairs pp;
    for (int q = 0; q < 32; q++) { pp.a[q] = q < np ? a[q0 + q] : nullptr; pp.b[q] = q < np ? b[q0 + q] : nullptr; }
    double* pt = part + (int64_t)q0 * kRedBlocks;
    if (dtype == BLML_F64) launch_dots<double>(n, np, pp, pt, ST);
    else launch_dots<float>(n, np, pp, pt, ST);
    BLML_CHECK_LAUNCH("blml_dots");
    int e = finish_partials(pt, np, kRedBlocks, 0u, out + q0, ST);
    if (e) return e;
  }
  return BLML_OK;
}

int blml_lincomb(int dtype, int64_t n, void* out, int nterms, const double* coef, const void* const* v, void* stream) {
  if (check_dtype(dtype, "blml_lincomb")) return BLML_ERR_ARG;
  if (nterms < 0 || nterms > 64) { set_error("blml_lincomb: 0..64 terms"); return BLML_ERR_ARG; }
  if (n == 0) return BLML_OK;
  Terms t;
  for (int q = 0; q < 64; q++) { t.c[q] = q < nterms ? coef[q] : 0.0; t.v[q] = q < nterms ? v[q] : nullptr; }
  if (dtype == BLML_F64) k_lincomb<double><<<grid_for(n), 256, 0, ST>>>(n, (double*)out, nterms, t);
  else k_lincomb<float><<<grid_for(n), 256, 0, ST>>>(n, (float*)out, nterms, t);
  BLML_CHECK_LAUNCH("blml_lincomb");
  return BLML_OK;
}

int blml_mul_bins(int dtype, int K, int64_t B, int cplx, const void* x, const void* r, void* out, void* stream) {
  if (check_dtype(dtype, "blml_mul_bins")) return BLML_ERR_ARG;
  if (B == 0) return BLML_OK;
  if (dtype == BLML_F64) {
    if (cplx) k_mul_bins<double, true><<<grid_for(B), 256, 0, ST>>>(K, B, x, (const double*)r, out);
    else k_mul_bins<double, false><<<grid_for(B), 256, 0, ST>>>(K, B, x, (const double*)r, out);
  } else {
    if (cplx) k_mul_bins<float, true><<<grid_for(B), 256, 0, ST>>>(K, B, x, (const float*)r, out);
    else k_mul_bins<float, false><<<grid_for(B), 256, 0, ST>>>(K, B, x, (const float*)r, out);
  }
  BLML_CHECK_LAUNCH("blml_mul_bins");
  return BLML_OK;
}

int blml_lgrad_weights(int dtype, int K, int64_t B, int cplx, const void* U, const void* w, double vscale, void* V,
                       double* part, double* out, void* stream) {
  if (check_dtype(dtype, "blml_lgrad_weights")) return BLML_ERR_ARG;
  if (dtype == BLML_F64) {
    if (cplx) k_lgrad_weights<double, true><<<kRedBlocks, kRedThreads, 0, ST>>>(K, B, U, (const double*)w, vscale, V, part);
    else k_lgrad_weights<double, false><<<kRedBlocks, kRedThreads, 0, ST>>>(K, B, U, (const double*)w, vscale, V, part);
  } else {
    if (cplx) k_lgrad_weights<float, true><<<kRedBlocks, kRedThreads, 0, ST>>>(K, B, U, (const float*)w, vscale, V, part);
    else k_lgrad_weights<float, false><<<kRedBlocks, kRedThreads, 0, ST>>>(K, B, U, (const float*)w, vscale, V, part);
  }
  BLML_CHECK_LAUNCH("blml_lgrad_weights");
  return finish_partials(part, 1, kRedBlocks, 0u, out, ST);
}

int blml_pgrad_weights(int dtype, int K, int64_t B, int cplx, const void* U, const void* m, double add, void* V,
                       double* part, double* out, void* stream) {
  if (check_dtype(dtype, "blml_pgrad_weights")) return BLML_ERR_ARG;
  if (K < 1 || B < 1 || !U || !m || !V || !part || !out) { set_error("blml_pgrad_weights: arguments"); return BLML_ERR_ARG; }
  if (dtype == BLML_F64) {
    if (cplx) k_pgrad_weights<double, true><<<kRedBlocks, kRedThreads, 0, ST>>>(K, B, U, (const double*)m, add, V, part);
    else k_pgrad_weights<double, false><<<kRedBlocks, kRedThreads, 0, ST>>>(K, B, U, (const double*)m, add, V, part);
  } else {
    if (cplx) k_pgrad_weights<float, true><<<kRedBlocks, kRedThreads, 0, ST>>>(K, B, U, (const float*)m, add, V, part);
    else k_pgrad_weights<float, false><<<kRedBlocks, kRedThreads, 0, ST>>>(K, B, U, (const float*)m, add, V, part);
  }
  BLML_CHECK_LAUNCH("blml_pgrad_weights");
  return finish_partials(part, 2, kRedBlocks, 0u, out, ST);
}

int blml_hvp_inner(int dtype, int K, int64_t B, int cplx, const void* U, const void* dU, const void* w, void* out,
                   void* stream) {
  if (check_dtype(dtype, "blml_hvp_inner")) return BLML_ERR_ARG;
  if (K < 1 || B < 1 || !U || !dU || !w || !out) { set_error("blml_hvp_inner: arguments"); return BLML_ERR_ARG; }
  if (dtype == BLML_F64) {
    if (cplx) k_hvp_inner<double, true><<<grid_for(B), 256, 0, ST>>>(K, B, U, dU, (const double*)w, out);
    else k_hvp_inner<double, false><<<grid_for(B), 256, 0, ST>>>(K, B, U, dU, (const double*)w, out);
  } else {
    if (cplx) k_hvp_inner<float, true><<<grid_for(B), 256, 0, ST>>>(K, B, U, dU, (const float*)w, out);
    else k_hvp_inner<float, false><<<grid_for(B), 256, 0, ST>>>(K, B, U, dU, (const float*)w, out);
  }
  BLML_CHECK_LAUNCH("blml_hvp_inner");
  return BLML_OK;
}

int blml_mixed_terms(int dtype, int K, int64_t B, int cplx, const void* U, int k, const void* dUk, const void* w,
                     void* T, void* Wk, void* stream) {
  if (check_dtype(dtype, "blml_mixed_terms")) return BLML_ERR_ARG;
  if (K < 1 || B < 1 || k < 0 || k >= K || !U || !dUk || !w || !T || !Wk) {
    set_error("blml_mixed_terms: arguments"); return BLML_ERR_ARG;
  }
  if (dtype == BLML_F64) {
    if (cplx) k_mixed_terms<double, true><<<grid_for(B), 256, 0, ST>>>(K, B, U, k, dUk, (const double*)w, T, Wk);
    else k_mixed_terms<double, false><<<grid_for(B), 256, 0, ST>>>(K, B, U, k, dUk, (const double*)w, T, Wk);
  } else {
    if (cplx) k_mixed_terms<float, true><<<grid_for(B), 256, 0, ST>>>(K, B, U, k, dUk, (const float*)w, T, Wk);
    else k_mixed_terms<float, false><<<grid_for(B), 256, 0, ST>>>(K, B, U, k, dUk, (const float*)w, T, Wk);
  }
  BLML_CHECK_LAUNCH("blml_mixed_terms");
  return BLML_OK;
}

int blml_hvp_real1(int dtype, int64_t B, const void* D, const void* E, const void* c, const void* dU, void* out,
                   void* stream) {
  if (check_dtype(dtype, "blml_hvp_real1")) return BLML_ERR_ARG;
  if (B < 1 || !D || !E || !c || !dU || !out) { set_error("blml_hvp_real1: arguments"); return BLML_ERR_ARG; }
  if (dtype == BLML_F64)
    k_hvp_real1<double><<<grid_for(B), 256, 0, ST>>>(B, (const double*)D, (const double*)E, (const double*)c,
                                                      (const double*)dU, (double*)out);
  else
    k_hvp_real1<float><<<grid_for(B), 256, 0, ST>>>(B, (const float*)D, (const float*)E, (const float*)c,
                                                     (const float*)dU, (float*)out);
  BLML_CHECK_LAUNCH("blml_hvp_real1");
  return BLML_OK;
}

int blml_counts_axpy(int dtype, int64_t B, double a, const void* w, double b, const void* m, int clamp, void* out,
                     void* stream) {
  if (check_dtype(dtype, "blml_counts_axpy")) return BLML_ERR_ARG;
  if (B < 1 || !w || !m || !out) { set_error("blml_counts_axpy: arguments"); return BLML_ERR_ARG; }
  if (dtype == BLML_F64)
    k_counts_axpy<double><<<grid_for(B), 256, 0, ST>>>(B, a, (const double*)w, b, (const double*)m, clamp, (double*)out);
  else
    k_counts_axpy<float><<<grid_for(B), 256, 0, ST>>>(B, a, (const float*)w, b, (const float*)m, clamp, (float*)out);
  BLML_CHECK_LAUNCH("blml_counts_axpy");
  return BLML_OK;
}

int blml_bin_ratio(int dtype, int64_t B, const void* num, const void* den, void* out, void* stream) {
  if (check_dtype(dtype, "blml_bin_ratio")) return BLML_ERR_ARG;
  if (B < 1 || !num || !den || !out) { set_error("blml_bin_ratio: arguments"); return BLML_ERR_ARG; }
  if (dtype == BLML_F64)
    k_bin_ratio<double><<<grid_for(B), 256, 0, ST>>>(B, (const double*)num, (const double*)den, (double*)out);
  else k_bin_ratio<float><<<grid_for(B), 256, 0, ST>>>(B, (const float*)num, (const float*)den, (float*)out);
  BLML_CHECK_LAUNCH("blml_bin_ratio");
  return BLML_OK;
}

int blml_new_bins(int dtype, int K, int64_t B, int cplx, const void* E, const void* Eu, const void* w, void* out,
                  void* stream) {
  if (check_dtype(dtype, "blml_new_bins")) return BLML_ERR_ARG;
  if (K < 1 || B < 1 || !E || !Eu || !w || !out) { set_error("blml_new_bins: arguments"); return BLML_ERR_ARG; }
  if (dtype == BLML_F64) {
    if (cplx) k_new_bins<double, true><<<grid_for(B), 256, 0, ST>>>(K, B, E, Eu, (const double*)w, out);
    else k_new_bins<double, false><<<grid_for(B), 256, 0, ST>>>(K, B, E, Eu, (const double*)w, out);
  } else {
    if (cplx) k_new_bins<float, true><<<grid_for(B), 256, 0, ST>>>(K, B, E, Eu, (const float*)w, out);
    else k_new_bins<float, false><<<grid_for(B), 256, 0, ST>>>(K, B, E, Eu, (const float*)w, out);
  }
  BLML_CHECK_LAUNCH("blml_new_bins");
  return BLML_OK;
}

int blml_gain_sums(int dtype, int64_t B, const void* da, double sa, const void* db, double sb, const void* m, double eps,
                   double* part, double* out, void* stream) {
  if (check_dtype(dtype, "blml_gain_sums")) return BLML_ERR_ARG;
  if (B < 1 || !da || !db || !m || !part || !out) { set_error("blml_gain_sums: arguments"); return BLML_ERR_ARG; }
  if (dtype == BLML_F64)
    k_gain_sums<double><<<kRedBlocks, kRedThreads, 0, ST>>>(B, (const double*)da, sa, (const double*)db, sb,
                                                            (const double*)m, eps, part);
  else
    k_gain_sums<float><<<kRedBlocks, kRedThreads, 0, ST>>>(B, (const float*)da, sa, (const float*)db, sb,
                                                           (const float*)m, eps, part);
  BLML_CHECK_LAUNCH("blml_gain_sums");
  return finish_partials(part, 3, kRedBlocks, 0u, out, ST);
}

int blml_block_root(int m, const int64_t* I, int64_t B, const double* e, const double* Se, const double* c, double sbb,
                    double* d, void* stream) {
  if (m < 0 || B < 1 || (m > 0 && (!I || !e || !Se || !c || !d))) { set_error("blml_block_root: arguments"); return BLML_ERR_ARG; }
  if (m == 0) return BLML_OK;
  k_block_root<<<grid_for(m), 256, 0, ST>>>(m, I, B, e, Se, c, sbb, d);
  BLML_CHECK_LAUNCH("blml_block_root");
  return BLML_OK;
}

int blml_block_search(int m, const int64_t* I, int64_t B, const double* e, const double* d, const double* Se,
                      const double* v, const double* c, double* out, void* stream) {
  if (m < 0 || B < 1 || !out || (m > 0 && (!I || !e || !d || !Se || !v || !c))) {
    set_error("blml_block_search: arguments"); return BLML_ERR_ARG;
  }
  k_block_search<<<1, 256, 0, ST>>>(m, I, B, e, d, Se, v, c, out);
  BLML_CHECK_LAUNCH("blml_block_search");
  return BLML_OK;
}

int blml_block_apply(int m, const int64_t* I, int64_t B, const double* d, double t, double* e, void* stream) {
  if (m < 0 || B < 1 || (m > 0 && (!I || !d || !e))) { set_error("blml_block_apply: arguments"); return BLML_ERR_ARG; }
  if (m == 0) return BLML_OK;
  k_block_apply<<<grid_for(m), 256, 0, ST>>>(m, I, B, d, t, e);
  BLML_CHECK_LAUNCH("blml_block_apply");
  return BLML_OK;
}

int blml_gather_rows_i64(int m, int d, const int64_t* src, const int64_t* I, int64_t B, int64_t* out, void* stream) {
  if (m < 0 || d < 1 || B < 1 || (m > 0 && (!src || !I || !out))) { set_error("blml_gather_rows_i64: arguments"); return BLML_ERR_ARG; }
  if (m == 0) return BLML_OK;
  k_gather_rows_i64<<<grid_for((int64_t)m * d), 256, 0, ST>>>(m, d, src, I, B, out);
  BLML_CHECK_LAUNCH("blml_gather_rows_i64");
  return BLML_OK;
}

int blml_lgrad_finish(int dtype, int K, int64_t B, int cplx, const void* SV, const void* U, const void* w, double nq,
                      void* g, void* stream) {
  if (check_dtype(dtype, "blml_lgrad_finish")) return BLML_ERR_ARG;
  if (B == 0) return BLML_OK;
  if (dtype == BLML_F64) {
    if (cplx) k_lgrad_finish<double, true><<<grid_for(B), 256, 0, ST>>>(K, B, SV, U, (const double*)w, nq, g);
    else k_lgrad_finish<double, false><<<grid_for(B), 256, 0, ST>>>(K, B, SV, U, (const double*)w, nq, g);
  } else {
    if (cplx) k_lgrad_finish<float, true><<<grid_for(B), 256, 0, ST>>>(K, B, SV, U, (const float*)w, nq, g);
    else k_lgrad_finish<float, false><<<grid_for(B), 256, 0, ST>>>(K, B, SV, U, (const float*)w, nq, g);
  }
  BLML_CHECK_LAUNCH("blml_lgrad_finish");
  return BLML_OK;
}

int blml_finish(int dtype, int K, int64_t B, int cplx, const void* U, const void* w, double inv_n2, void* density,
                double* part, double* out, void* stream) {
  if (check_dtype(dtype, "blml_finish")) return BLML_ERR_ARG;
  if (dtype == BLML_F64) {
    if (cplx) k_finish<double, true><<<kRedBlocks, kRedThreads, 0, ST>>>(K, B, U, (const double*)w, inv_n2, (double*)density, part);
    else k_finish<double, false><<<kRedBlocks, kRedThreads, 0, ST>>>(K, B, U, (const double*)w, inv_n2, (double*)density, part);
  } else {
    if (cplx) k_finish<float, true><<<kRedBlocks, kRedThreads, 0, ST>>>(K, B, U, (const float*)w, inv_n2, (float*)density, part);
    else k_finish<float, false><<<kRedBlocks, kRedThreads, 0, ST>>>(K, B, U, (const float*)w, inv_n2, (float*)density, part);
  }
  BLML_CHECK_LAUNCH("blml_finish");
  return finish_partials(part, 1, kRedBlocks, 0u, out, ST);
}

int blml_start_root(int dtype, int64_t B, const void* c, const void* sg, double s0, void* e0, void* stream) {
  if (check_dtype(dtype, "blml_start_root")) return BLML_ERR_ARG;
  if (B == 0) return BLML_OK;
  if (dtype == BLML_F64) k_start_root<double><<<grid_for(B), 256, 0, ST>>>(B, (const double*)c, (const double*)sg, s0, (double*)e0);
  else k_start_root<float><<<grid_for(B), 256, 0, ST>>>(B, (const float*)c, (const float*)sg, s0, (float*)e0);
  BLML_CHECK_LAUNCH("blml_start_root");
  return BLML_OK;
}

int blml_fill_modes(int dtype, int K, int64_t B, int cplx, int kk, int phases, double pn, const double* z, void* E,
                    void* stream) {
  if (check_dtype(dtype, "blml_fill_modes")) return BLML_ERR_ARG;
  if (B == 0) return BLML_OK;
  if (dtype == BLML_F64) {
    if (cplx) k_fill_modes<double, true><<<grid_for(B), 256, 0, ST>>>(K, B, kk, phases, pn, z, E);
    else k_fill_modes<double, false><<<grid_for(B), 256, 0, ST>>>(K, B, kk, phases, pn, z, E);
  } else {
    if (cplx) k_fill_modes<float, true><<<grid_for(B), 256, 0, ST>>>(K, B, kk, phases, pn, z, E);
    else k_fill_modes<float, false><<<grid_for(B), 256, 0, ST>>>(K, B, kk, phases, pn, z, E);
  }
  BLML_CHECK_LAUNCH("blml_fill_modes");
  return BLML_OK;
}

int blml_cert_weights(int dtype, int K, int64_t B, int cplx, const void* E, const void* w, double* dh, void* stream) {
  if (check_dtype(dtype, "blml_cert_weights")) return BLML_ERR_ARG;
  if (B == 0) return BLML_OK;
  if (dtype == BLML_F64) {
    if (cplx) k_cert_weights<double, true><<<grid_for(B), 256, 0, ST>>>(K, B, E, (const double*)w, dh);
    else k_cert_weights<double, false><<<grid_for(B), 256, 0, ST>>>(K, B, E, (const double*)w, dh);
  } else {
    if (cplx) k_cert_weights<float, true><<<grid_for(B), 256, 0, ST>>>(K, B, E, (const float*)w, dh);
    else k_cert_weights<float, false><<<grid_for(B), 256, 0, ST>>>(K, B, E, (const float*)w, dh);
  }
  BLML_CHECK_LAUNCH("blml_cert_weights");
  return BLML_OK;
}

int blml_lbfgs_trial(int dtype, int K, int64_t B, int cplx, const void* E, const void* q, const void* U,
                     const void* Sq, const void* w, double t, void* En, void* Un, double* part, double* out,
                     void* stream) {
  if (check_dtype(dtype, "blml_lbfgs_trial")) return BLML_ERR_ARG;
  if (dtype == BLML_F64) {
    if (cplx) k_lbfgs_trial<double, true><<<kRedBlocks, kRedThreads, 0, ST>>>(K, B, E, q, U, Sq, (const double*)w, t, En, Un, part);
    else k_lbfgs_trial<double, false><<<kRedBlocks, kRedThreads, 0, ST>>>(K, B, E, q, U, Sq, (const double*)w, t, En, Un, part);
  } else {
    if (cplx) k_lbfgs_trial<float, true><<<kRedBlocks, kRedThreads, 0, ST>>>(K, B, E, q, U, Sq, (const float*)w, t, En, Un, part);
    else k_lbfgs_trial<float, false><<<kRedBlocks, kRedThreads, 0, ST>>>(K, B, E, q, U, Sq, (const float*)w, t, En, Un, part);
  }
  BLML_CHECK_LAUNCH("blml_lbfgs_trial");
  return finish_partials(part, 2, kRedBlocks, 0u, out, ST);
}

}

extern "C" int blml_log_score(int dtype, int K, int64_t B, int cplx, const void* U, const void* m, double inv_z,
                              double eps, double* part, double* out, void* stream) {
  if (check_dtype(dtype, "blml_log_score")) return BLML_ERR_ARG;
  if (dtype == BLML_F64) {
    if (cplx) k_log_score<double, true><<<kRedBlocks, kRedThreads, 0, ST>>>(K, B, U, (const double*)m, inv_z, eps, part);
    else k_log_score<double, false><<<kRedBlocks, kRedThreads, 0, ST>>>(K, B, U, (const double*)m, inv_z, eps, part);
  } else {
    if (cplx) k_log_score<float, true><<<kRedBlocks, kRedThreads, 0, ST>>>(K, B, U, (const float*)m, inv_z, eps, part);
    else k_log_score<float, false><<<kRedBlocks, kRedThreads, 0, ST>>>(K, B, U, (const float*)m, inv_z, eps, part);
  }
  BLML_CHECK_LAUNCH("blml_log_score");
  return finish_partials(part, 2, kRedBlocks, 0u, out, ST);
}
