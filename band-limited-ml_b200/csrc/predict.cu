// The fitted amplitude at arbitrary points for kernels made of harmonics (pball groups, dirichlet columns), the
// binned fit's sqrt_density / predict / predict_grid (rahuljhu/band-limited-ml blml_binned.py:451-500). Such a kernel
// is exactly a weighted sum of plane waves, so
//     g(x) = sum_b e_b K(x - z_b) = sum_q C_q exp(2 pi i nu_q . u),   C = W (v^H e),  u = (x - origin) / h,
// with the spectrum C from the mat-vec plan's forward stages (blml_spectrum). One warp per query point: the lanes
// split the axis-1 frequencies (their phases computed once per chunk of 256), every axis-0 frequency multiplies its
// row's partial sum, and a fixed-order warp reduction ends the point. Phases are reduced to [-1/2, 1/2] cycles before
// sincospi, so the large products nu u of wide lattices keep their accuracy.
#include "common.cuh"

namespace blml {

constexpr int kPwWarps = 8;              // query points per CTA
constexpr int kPwChunk = 8;              // axis-1 frequencies per lane and chunk

__device__ __forceinline__ cpx<double> phase(double nu, double u) {
  double c = nu * u;
  c -= rint(c);
  double sn, cs;
  sincospi(2.0 * c, &sn, &cs);
  return {cs, sn};
}

// spec (H1 x H2 complex, row-major), f1 (H1), f2 (H2) cycles per lattice index, U (m x 2) lattice coordinates
__global__ void __launch_bounds__(32 * kPwWarps) k_planewave_points(int H1, int H2, const double* __restrict__ f1,
                                                                     const double* __restrict__ f2,
                                                                     const cpx<double>* __restrict__ spec, int64_t m,
                                                                     const double* __restrict__ U,
                                                                     cpx<double>* __restrict__ g) {
  const int lane = threadIdx.x & 31;
  const int64_t i = (int64_t)blockIdx.x * kPwWarps + (threadIdx.x >> 5);
  if (i >= m) return;                                   // whole warps leave together
  const double u1 = U[2 * i], u2 = U[2 * i + 1];
  cpx<double> acc = {0.0, 0.0};
  for (int c0 = 0; c0 < H2; c0 += 32 * kPwChunk) {
    cpx<double> ph2[kPwChunk];
#pragma unroll
    for (int c = 0; c < kPwChunk; c++) {
      const int q2 = c0 + lane + 32 * c;
      ph2[c] = q2 < H2 ? phase(f2[q2], u2) : cpx<double>{0.0, 0.0};
    }
    for (int q1 = 0; q1 < H1; q1++) {
      const cpx<double>* row = spec + (int64_t)q1 * H2;
      cpx<double> part = {0.0, 0.0};
#pragma unroll
      for (int c = 0; c < kPwChunk; c++) {
        const int q2 = c0 + lane + 32 * c;
        if (q2 < H2) part = cfma(row[q2], ph2[c], part);
      }
      acc = cfma(part, phase(f1[q1], u1), acc);
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    acc.re += __shfl_down_sync(0xffffffffu, acc.re, o);
    acc.im += __shfl_down_sync(0xffffffffu, acc.im, o);
  }
  if (lane == 0) g[i] = acc;
}

}  // namespace blml

using namespace blml;

extern "C" {

int blml_planewave_points(int H1, int H2, const double* f1, const double* f2, const double* spec, int64_t m,
                          const double* U, double* g, void* stream) {
  if (H1 < 1 || H2 < 1 || m < 0) { set_error("blml_planewave_points: H1, H2 >= 1, m >= 0"); return BLML_ERR_ARG; }
  if (m == 0) return BLML_OK;
  if (!f1 || !f2 || !spec || !U || !g) { set_error("blml_planewave_points: null pointer"); return BLML_ERR_ARG; }
  const unsigned blocks = (unsigned)((m + kPwWarps - 1) / kPwWarps);
  k_planewave_points<<<blocks, 32 * kPwWarps, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      H1, H2, f1, f2, reinterpret_cast<const cpx<double>*>(spec), m, U, reinterpret_cast<cpx<double>*>(g));
  BLML_CHECK_LAUNCH("blml_planewave_points");
  return BLML_OK;
}

}  // extern "C"
