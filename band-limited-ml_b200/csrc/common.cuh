// Shared helpers of libblml_b200: status reporting, complex arithmetic over float / double, and the deterministic
// block reductions every fused kernel uses (FP64 partial sums per block, summed in a fixed order by one block).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <math.h>
#include <string>
#include <algorithm>
#include "blml_b200.h"

namespace blml {

void set_error(const char* fmt, ...);
int cuda_status(cudaError_t e, const char* where);
// cumulative number of kernels this library has launched (blml_launch_count)
void count_launches(int n);

// after each kernel launch: count it and turn a launch error into a status
#define BLML_CHECK_LAUNCH(where)                                   \
  do {                                                             \
    ::blml::count_launches(1);                                     \
    cudaError_t _e = cudaGetLastError();                           \
    if (_e != cudaSuccess) return ::blml::cuda_status(_e, where);  \
  } while (0)

// Number of blocks of every grid-stride reduction kernel: two per SM of a B200 (148 SMs). The partial-sum
// workspace of a reduction with nq quantities is nq * kRedBlocks doubles.
constexpr int kRedBlocks = 296;
constexpr int kRedThreads = 256;

template <typename T> struct cpx { T re, im; };

template <typename T> __device__ __forceinline__ cpx<T> cmul(cpx<T> a, cpx<T> b) {
  return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
template <typename T> __device__ __forceinline__ cpx<T> cfma(cpx<T> a, cpx<T> b, cpx<T> c) {
  // c + a * b
  c.re = fma(a.re, b.re, c.re); c.re = fma(-a.im, b.im, c.re);
  c.im = fma(a.re, b.im, c.im); c.im = fma(a.im, b.re, c.im);
  return c;
}

// Block-wide sum of a double (all threads receive nothing; thread 0 gets the block total).
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
  return v;
}

// Reduce NQ per-thread doubles to per-block partials: part[q * gridDim.x + blockIdx.x]. Sums for q with
// (maxmask >> q) & 1 == 0, maxima otherwise.
template <int NQ>
__device__ __forceinline__ void block_partials(double (&v)[NQ], double* part, unsigned maxmask = 0u) {
  __shared__ double sh[NQ][32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int q = 0; q < NQ; q++) {
    double x = ((maxmask >> q) & 1u) ? warp_max(v[q]) : warp_sum(v[q]);
    if (lane == 0) sh[q][wid] = x;
  }
  __syncthreads();
  if (wid == 0) {
#pragma unroll
    for (int q = 0; q < NQ; q++) {
      const bool mx = (maxmask >> q) & 1u;
      double x = lane < nw ? sh[q][lane] : (mx ? -INFINITY : 0.0);
      x = mx ? warp_max(x) : warp_sum(x);
      if (lane == 0) part[q * gridDim.x + blockIdx.x] = x;
    }
  }
}

// out[q] = the fixed-order reduction of part[q * nblk + 0 .. nblk - 1] (one block, launched after the producer).
int finish_partials(const double* part, int nq, int nblk, unsigned maxmask, double* out, cudaStream_t st);

}  // namespace blml
