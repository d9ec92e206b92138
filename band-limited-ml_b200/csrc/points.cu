// The fitted amplitude at arbitrary points (BLMLQuick.sqrt_density / predict, rahuljhu/band-limited-ml
// blml_trivial.py:3288-3320 with the continuous product kernel of :2573): g(x_i) = sum_b e_b prod_c K_c(x_ic - z_bc)
// over the fit's B bin centres z_b, the kernel evaluated exactly (not from a lattice table: the query points are off
// the lattice). One thread per query point; the bins are staged through shared memory in tiles shared by the block,
// so each bin centre and coefficient is read from HBM once per block. Per pair: d kernel values (sinpi) and d + 1
// multiplies in float64, summed in a fixed order.
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
        for (int c = 0; c < d; c++) p *= point_unit(cols.c[c], x[c] - zs[j * d + c]);
        acc += p;
      }
    }
  }
  if (i < m) g[i] = acc;
}

}  // namespace blml

using namespace blml;

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
  for (int c = 0; c < d; c++) {
    cc.c[c] = cols[c];
    const int k = cols[c].kind;
    if (k != BLML_PT_SINC && k != BLML_PT_SLITS && k != BLML_PT_DIRICHLET) {
      set_error("blml_point_rows: column %d: kind %d (sinc, slits or dirichlet)", c, k);
      return BLML_ERR_ARG;
    }
    if (k == BLML_PT_DIRICHLET && !(cols[c].P > 0)) {
      set_error("blml_point_rows: column %d: dirichlet period must be positive", c);
      return BLML_ERR_ARG;
    }
  }
  const int64_t blocks = (m + kPtThreads - 1) / kPtThreads;
  k_point_rows<<<(unsigned)blocks, kPtThreads, 0, reinterpret_cast<cudaStream_t>(stream)>>>(m, d, X, B, Z, e, cc, g);
  BLML_CHECK_LAUNCH("blml_point_rows");
  return BLML_OK;
}

}  // extern "C"
