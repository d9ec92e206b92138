// The fitted amplitude at arbitrary points (BLMLQuick.sqrt_density / predict, rahuljhu/band-limited-ml
// blml_trivial.py:3288-3320 with the continuous product kernel of :2573): g(x_i) = sum_b e_b prod_c K_c(x_ic - z_bc)
// over the fit's B bin centres z_b, the kernel evaluated exactly (not from a lattice table: the query points are off
// the lattice). One thread per query point; the bins are staged through shared memory in tiles shared by the block,
// so each bin centre and coefficient is read from HBM once per block. Per pair: d kernel values (sinpi) and d + 1
// multiplies in float64, summed in a fixed order. A ball unit over a group of D columns (blml_trivial.py:580-591,
// 135-143) is one radial value per pair: prod fc p(s), s = ||fc (x - z)|| over the group, p(s) = (1/2)^(D/2)
// J_(D/2)(pi s) / s^(D/2) -- CUDA's jn for whole orders; for half orders the power series below nu + 12 and, above,
// upward recurrence from the closed forms of J_1/2 and J_3/2 (the standard methods).
#include "common.cuh"

namespace blml {

constexpr int kPtThreads = 256;
constexpr int kPtTile = 256;
constexpr int kPtMaxD = 8;

__device__ __forceinline__ double sinc_unit(double f, double t) {
  // f sinc(f t) = sin(pi f t) / (pi t), f at t = 0
  return t == 0.0 ? f : sinpi(f * t) / (M_PI * t);
}

__device__ __forceinline__ double point_unit(const blml_point_col& c, double t) {
  if (c.kind == BLML_PT_SINC) return sinc_unit(c.f, t);
  if (c.kind == BLML_PT_SLITS) return sinc_unit(c.f, t) - (c.fi > 0 ? sinc_unit(c.fi, t) : 0.0);
  // dirichlet: (sin(pi M u / P) - sin(pi Mi u / P)) / sin(pi u / P) / P, u = |t| folded into [0, P / 2]
  const double P = c.P;
  double u = fmod(fabs(t), P);
  u = fmin(u, P - u);
  if (u < 1e-10) return (c.M - c.Mi) / P;
  return (sinpi(c.M * u / P) - sinpi(c.Mi * u / P)) / sinpi(u / P) / P;
}

// J_(twice_nu / 2)(x), x >= 0, twice_nu odd: the power series sum_k (-1)^k (x/2)^(2k+nu) / (k! Gamma(k+nu+1)) below
// x = nu + 12 (upward recurrence loses accuracy below the order), above it J_{m+1} = (2m / x) J_m - J_{m-1} from
// J_1/2 = c sin x and J_3/2 = c (sin x / x - cos x), c = sqrt(2 / (pi x))
__device__ __noinline__ double bessel_half_order(int twice_nu, double x) {
  const double nu = 0.5 * twice_nu;
  if (x < nu + 12.0) {
    const double xs = 0.5 * x;
    double term = pow(xs, nu) / tgamma(nu + 1.0), acc = term;
    for (int k = 1; k < 80; k++) {
      term = -term * xs * xs / (k * (k + nu));
      acc += term;
    }
    return acc;
  }
  const double c = sqrt(2.0 / (M_PI * x));
  double jm = c * sin(x), jc = c * (sin(x) / x - cos(x)), m = 0.5;
  if (twice_nu == 1) return jm;
  while (m + 1.0 < nu - 1e-9) {
    const double jn1 = (2.0 * (m + 1.0) / x) * jc - jm;
    jm = jc; jc = jn1; m += 1.0;
  }
  return jc;
}

// the ball profile p(s) in D dims; p0 = p(0) = pi^(D/2) (1/2)^D / Gamma(D/2 + 1), the ball's volume
__device__ __noinline__ double ball_profile(double s, int D, double p0) {
  if (s == 0.0) return p0;
  const double x = M_PI * s;
  const double J = (D % 2 == 0) ? jn(D / 2, x) : bessel_half_order(D, x);
  return pow(0.5, 0.5 * D) * J / pow(s, 0.5 * D);
}

__global__ void __launch_bounds__(kPtThreads) k_point_rows(int64_t m, int d, const double* __restrict__ X,
                                                          int64_t B, const double* __restrict__ Z,
                                                          const double* __restrict__ e, blml_point_cols cols,
                                                          double* __restrict__ g) {
  __shared__ double zs[kPtTile * kPtMaxD];
  __shared__ double es[kPtTile];
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  double x[kPtMaxD];
  for (int c = 0; c < d; c++) x[c] = i < m ? X[i * d + c] : 0.0;
  double acc = 0.0;
  for (int64_t b0 = 0; b0 < B; b0 += kPtTile) {
    const int nt = (int)(B - b0 < kPtTile ? B - b0 : kPtTile);
    __syncthreads();
    for (int j = threadIdx.x; j < nt * d; j += blockDim.x) zs[j] = Z[b0 * d + j];
    for (int j = threadIdx.x; j < nt; j += blockDim.x) es[j] = e[b0 + j];
    __syncthreads();
    if (i < m) {
      for (int j = 0; j < nt; j++) {
        double p = es[j];
        for (int c = 0; c < d; c++) {
          const blml_point_col& cc = cols.c[c];
          if (cc.kind == BLML_PT_BALL) {
            if (cc.fi == 0.0) continue;                   // a ball group's value sits on its first column
            double s2 = 0.0;
            for (int c2 = 0; c2 < d; c2++)
              if ((cc.M >> c2) & 1) {
                const double t = cols.c[c2].f * (x[c2] - zs[j * d + c2]);
                s2 += t * t;
              }
            p *= cc.fi * ball_profile(sqrt(s2), cc.Mi, cc.P);
          } else {
            p *= point_unit(cc, x[c] - zs[j * d + c]);
          }
        }
        acc += p;
      }
    }
  }
  if (i < m) g[i] = acc;
}

// Point sums of several densities (blml_local.py:555-560, point_rows_multi: FusedFit's joint and marginals at
// points): g[i][m] = sum_b W[b][m] prod_u (bit u of masks[m] ? K_u(x_i - z_b) : 1), every unit's value computed once
// per (point, bin) pair; unit_of[c] is the unit of column c (a ball group's value sits on its first column).
constexpr int kPtMaxM = 8;
struct PtMulti { int unit_of[kPtMaxD]; unsigned masks[kPtMaxM]; };

__global__ void __launch_bounds__(kPtThreads) k_point_rows_multi(int64_t m, int d, int U, const double* __restrict__ X,
                                                                int64_t B, const double* __restrict__ Z,
                                                                const double* __restrict__ W, int Mm,
                                                                blml_point_cols cols, PtMulti pm,
                                                                double* __restrict__ g) {
  __shared__ double zs[kPtTile * kPtMaxD];
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  double x[kPtMaxD];
  for (int c = 0; c < d; c++) x[c] = i < m ? X[i * d + c] : 0.0;
  double acc[kPtMaxM];
  for (int q = 0; q < kPtMaxM; q++) acc[q] = 0.0;
  for (int64_t b0 = 0; b0 < B; b0 += kPtTile) {
    const int nt = (int)(B - b0 < kPtTile ? B - b0 : kPtTile);
    __syncthreads();
    for (int j = threadIdx.x; j < nt * d; j += blockDim.x) zs[j] = Z[b0 * d + j];
    __syncthreads();
    if (i < m) {
      for (int j = 0; j < nt; j++) {
        double fac[kPtMaxD];
        for (int u = 0; u < U; u++) fac[u] = 1.0;
        for (int c = 0; c < d; c++) {
          const blml_point_col& cc = cols.c[c];
          if (cc.kind == BLML_PT_BALL) {
            if (cc.fi == 0.0) continue;
            double s2 = 0.0;
            for (int c2 = 0; c2 < d; c2++)
              if ((cc.M >> c2) & 1) {
                const double t = cols.c[c2].f * (x[c2] - zs[j * d + c2]);
                s2 += t * t;
              }
            fac[pm.unit_of[c]] = cc.fi * ball_profile(sqrt(s2), cc.Mi, cc.P);
          } else {
            fac[pm.unit_of[c]] = point_unit(cc, x[c] - zs[j * d + c]);
          }
        }
        const int64_t b = b0 + j;
        for (int q = 0; q < Mm; q++) {
          double p = W[b * Mm + q];
          for (int u = 0; u < U; u++)
            if ((pm.masks[q] >> u) & 1u) p *= fac[u];
          acc[q] += p;
        }
      }
    }
  }
  if (i < m)
    for (int q = 0; q < Mm; q++) g[i * Mm + q] = acc[q];
}

}  // namespace blml

using namespace blml;

// the columns' kinds and ball groups checked, copied into cc; nonzero (with the error set) when they are not valid
static int check_point_cols(int d, const blml_point_col* cols, blml_point_cols& cc, const char* who) {
  for (int c = 0; c < d; c++) {
    cc.c[c] = cols[c];
    const int k = cols[c].kind;
    if (k != BLML_PT_SINC && k != BLML_PT_SLITS && k != BLML_PT_DIRICHLET && k != BLML_PT_BALL) {
      set_error("%s: column %d: kind %d (sinc, slits, dirichlet or ball)", who, c, k);
      return 1;
    }
    if (k == BLML_PT_DIRICHLET && !(cols[c].P > 0)) {
      set_error("%s: column %d: dirichlet period must be positive", who, c);
      return 1;
    }
    if (k == BLML_PT_BALL) {
      // the group mask holds this column and only ball columns; the first column of the group carries prod fc (fi),
      // the group size (Mi) and p(0) (P), the others fi = 0
      const int mask = cols[c].M;
      int lead = -1, size = 0;
      for (int c2 = 0; c2 < d; c2++)
        if ((mask >> c2) & 1) { size++; if (lead < 0) lead = c2; }
      bool ok = mask > 0 && mask < (1 << d) && ((mask >> c) & 1) && cols[c].f > 0;
      for (int c2 = 0; c2 < d && ok; c2++)
        if ((mask >> c2) & 1) ok = cols[c2].kind == BLML_PT_BALL && cols[c2].M == mask;
      if (ok && c == lead) ok = cols[c].Mi == size && cols[c].fi > 0 && cols[c].P > 0;
      if (ok && c != lead) ok = cols[c].fi == 0.0;
      if (!ok) {
        set_error("%s: column %d: inconsistent ball group (mask %d)", who, c, mask);
        return 1;
      }
    }
  }
  return 0;
}

extern "C" {

int blml_point_rows(int64_t m, int d, const double* X, int64_t B, const double* Z, const double* e,
                    const blml_point_col* cols, double* g, void* stream) {
  if (m < 0 || B < 0 || d < 1 || d > kPtMaxD || !cols) {
    set_error("blml_point_rows: 1 <= d <= %d columns, m, B >= 0", kPtMaxD);
    return BLML_ERR_ARG;
  }
  if (m == 0) return BLML_OK;
  if (!X || !g || (B > 0 && (!Z || !e))) { set_error("blml_point_rows: null pointer"); return BLML_ERR_ARG; }
  blml_point_cols cc;
  if (check_point_cols(d, cols, cc, "blml_point_rows")) return BLML_ERR_ARG;
  const int64_t blocks = (m + kPtThreads - 1) / kPtThreads;
  k_point_rows<<<(unsigned)blocks, kPtThreads, 0, reinterpret_cast<cudaStream_t>(stream)>>>(m, d, X, B, Z, e, cc, g);
  BLML_CHECK_LAUNCH("blml_point_rows");
  return BLML_OK;
}

int blml_point_rows_multi(int64_t m, int d, const double* X, int64_t B, const double* Z, const double* W, int Mm,
                          const blml_point_col* cols, const int* unit_of, int U, const unsigned* masks, double* g,
                          void* stream) {
  if (m < 0 || B < 0 || d < 1 || d > kPtMaxD || !cols || !unit_of || !masks || Mm < 1 || Mm > kPtMaxM || U < 1 ||
      U > d) {
    set_error("blml_point_rows_multi: 1 <= d <= %d columns, 1 <= U <= d units, 1 <= Mm <= %d densities", kPtMaxD,
              kPtMaxM);
    return BLML_ERR_ARG;
  }
  if (m == 0) return BLML_OK;
  if (!X || !g || (B > 0 && (!Z || !W))) { set_error("blml_point_rows_multi: null pointer"); return BLML_ERR_ARG; }
  blml_point_cols cc;
  if (check_point_cols(d, cols, cc, "blml_point_rows_multi")) return BLML_ERR_ARG;
  PtMulti pm;
  for (int c = 0; c < kPtMaxD; c++) pm.unit_of[c] = 0;
  for (int c = 0; c < d; c++) {
    if (unit_of[c] < 0 || unit_of[c] >= U) { set_error("blml_point_rows_multi: column %d: unit %d of %d", c, unit_of[c], U); return BLML_ERR_ARG; }
    pm.unit_of[c] = unit_of[c];
  }
  for (int q = 0; q < kPtMaxM; q++) pm.masks[q] = q < Mm ? masks[q] : 0u;
  for (int q = 0; q < Mm; q++)
    if (pm.masks[q] >> U) { set_error("blml_point_rows_multi: density %d masks a unit beyond %d", q, U); return BLML_ERR_ARG; }
  const int64_t blocks = (m + kPtThreads - 1) / kPtThreads;
  k_point_rows_multi<<<(unsigned)blocks, kPtThreads, 0, reinterpret_cast<cudaStream_t>(stream)>>>(m, d, U, X, B, Z, W,
                                                                                                 Mm, cc, pm, g);
  BLML_CHECK_LAUNCH("blml_point_rows_multi");
  return BLML_OK;
}

}  // extern "C"
