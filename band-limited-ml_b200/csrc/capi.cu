// Status reporting and the fixed-order finish of block partial sums shared by every reduction.
#include <stdarg.h>
#include <stdio.h>
#include <atomic>
#include "common.cuh"

namespace blml {

static thread_local char g_err[512] = "";
static std::atomic<long long> g_launches{0};

void count_launches(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

int cuda_status(cudaError_t e, const char* where) {
  if (e == cudaSuccess) return BLML_OK;
  set_error("%s: %s", where, cudaGetErrorString(e));
  return BLML_ERR_CUDA;
}

__global__ void k_finish_partials(const double* part, int nq, int nblk, unsigned maxmask, double* out) {
  // one block; each quantity summed by the whole block in a fixed order, then tree-reduced in a fixed shape
  for (int q = 0; q < nq; q++) {
    const bool mx = (maxmask >> q) & 1u;
    double acc = mx ? -INFINITY : 0.0;
    for (int i = threadIdx.x; i < nblk; i += blockDim.x) {
      double v = part[q * nblk + i];
      acc = mx ? fmax(acc, v) : acc + v;
    }
    double v[1] = {acc};
    __shared__ double sh[32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    double x = mx ? warp_max(v[0]) : warp_sum(v[0]);
    if (lane == 0) sh[wid] = x;
    __syncthreads();
    if (wid == 0) {
      x = lane < nw ? sh[lane] : (mx ? -INFINITY : 0.0);
      x = mx ? warp_max(x) : warp_sum(x);
      if (lane == 0) out[q] = x;
    }
    __syncthreads();
  }
}

int finish_partials(const double* part, int nq, int nblk, unsigned maxmask, double* out, cudaStream_t st) {
  k_finish_partials<<<1, 256, 0, st>>>(part, nq, nblk, maxmask, out);
  BLML_CHECK_LAUNCH("finish_partials");
  return BLML_OK;
}

}  // namespace blml

extern "C" {

const char* blml_last_error(void) { return blml::g_err; }
int blml_abi_version(void) { return 1; }
int blml_reduce_blocks(void) { return blml::kRedBlocks; }
int64_t blml_launch_count(void) { return blml::g_launches.load(std::memory_order_relaxed); }

}
