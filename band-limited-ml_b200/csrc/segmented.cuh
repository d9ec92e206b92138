// Segmented-kernel helpers shared by the batched solver kernels (batched.cu) and the device-side control of the
// batched engine (batch_runner.cu): fit f owns the slice [off_f, off_f + K_f B_f) of every flat mode array and
// [boff_f, boff_f + B_f) of every flat bin array; blockIdx.y is the fit, blockIdx.x strides over its bins.
#pragma once
#include "common.cuh"

namespace blml {

// blocks per fit (gridDim.x) of a segmented launch over F fits: ~16384 blocks in all, 16 to 256 per fit. Fits differ
// in size by up to ~300x (lattice and mode count), and every fit gets the same blocks, so the block count is sized
// for the largest: their blocks then still spread over every SM while the small fits' blocks find little or no work
// and leave at once. The partials of a reduction over F fits take nq * F * seg_blocks_for(F) <= nq * SEG_PART_WIDTH(F)
// doubles.
constexpr int SEG_BLOCKS_MIN = 16, SEG_BLOCKS_MAX = 256, SEG_BLOCKS_TOTAL = 16384;
__host__ __device__ constexpr int64_t SEG_PART_WIDTH(int F) {
  return (int64_t)(SEG_BLOCKS_TOTAL > 16 * F ? SEG_BLOCKS_TOTAL : 16 * F);
}
__host__ __device__ inline int seg_blocks_for(int F) {
  int x = SEG_BLOCKS_TOTAL / (F > 0 ? F : 1);
  return x < SEG_BLOCKS_MIN ? SEG_BLOCKS_MIN : (x > SEG_BLOCKS_MAX ? SEG_BLOCKS_MAX : x);
}

// A block split: SEG_SPLIT_BLOCKS blocks in all, shared out among the fits in proportion to their element counts
// K B (at least one block per fit with work, none per fit without, and no more blocks than SEG_SPLIT_MIN_ELEMS-element
// chunks), so that big and small fits finish together and every block has several tiles to stream. The split is
// computed on the device from the segment table itself (k_seg_split), so it follows fits whose table entry the device
// changes (a converged fit's B set to 0). Its ints: bstart[F + 1] (fit f owns split blocks
// [bstart[f], bstart[f + 1])), then fit_of[G + F] (the fit of each block of a launch of G + F blocks, -1 for blocks
// past the last fit's). Partials of a split reduction: quantity q of block b at part[q * (G + F) + b].
constexpr int SEG_SPLIT_BLOCKS = BLML_SEG_SPLIT_BLOCKS, SEG_SPLIT_MIN_ELEMS = 1024;
__host__ __device__ inline int64_t seg_split_ints(int F) { return 2 * (int64_t)F + 1 + SEG_SPLIT_BLOCKS; }
int seg_split(int F, const blml_seg* segs, int* split, cudaStream_t st);

// the L-BFGS runner's float32 history (batched.cu); split: seg_split's output for these segments
int seg_dots2_h32(int F, const blml_seg* segs, const int* split, int np, const void* const* a, const void* b0,
                  const void* b1, const void* x, double* part, double* out, cudaStream_t st);
int seg_lincomb_mixed(int F, const blml_seg* segs, const int* split, void* out, int out_f32, int nterms,
                      const double* coef, const void* const* v, unsigned long long f32mask, cudaStream_t st);

template <typename T, bool CPLX>
struct SAcc {
  static __device__ __forceinline__ void get(const void* p, int64_t i, double& re, double& im) {
    if (CPLX) { const cpx<T> v = reinterpret_cast<const cpx<T>*>(p)[i]; re = (double)v.re; im = (double)v.im; }
    else { re = (double)reinterpret_cast<const T*>(p)[i]; im = 0.0; }
  }
  static __device__ __forceinline__ void put(void* p, int64_t i, double re, double im) {
    if (CPLX) reinterpret_cast<cpx<T>*>(p)[i] = cpx<T>{(T)re, (T)im};
    else reinterpret_cast<T*>(p)[i] = (T)re;
  }
};

#define SEG_LOOP(b, sg) for (int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; b < (sg).B; \
                             b += (int64_t)gridDim.x * blockDim.x)

// partials layout, quantity-major so it does not depend on how many accumulators a kernel carries:
// part[((q * F) + f) * gridDim.x + blockIdx.x], F = gridDim.y fits
template <int NQ>
__device__ __forceinline__ void seg_partials(double (&v)[NQ], double* part, unsigned maxmask = 0u) {
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
      if (lane == 0) part[((int64_t)q * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x] = x;
    }
  }
}

}  // namespace blml
