// The per-mode Gram mat-vec S e as restricted transforms.
//
// A mode's kernel is a weighted sum of plane waves over a product grid of per-axis frequencies:
//     S e = sum_q W_q v_q v_q^H e,   v_q(j) = exp(2 pi i sum_a nu_{a, q_a} j_a).
// Exact for periodic bands (the harmonics of dirichlet / pball), Gauss-Legendre quadrature for interval bands (sinc,
// slits), and the padded lattice's own DFT for any other kernel. The transform runs as 2d "stages": each contracts
// the LAST axis of the current (nb, R, M) tensor against an (M x N) matrix and writes the result as (nb, N, R),
// i.e. the new axis moves to the front. After d forward stages the spectrum sits in natural order (q_1 .. q_d),
// where the weight W is applied in the last forward stage's epilogue; d inverse stages bring the lattice back in
// natural order. Every stage is one batched GEMM-shaped launch.
#include <vector>
#include <algorithm>
#include "plan.cuh"

namespace blml {

constexpr int TR = 64, TN = 64, TK = 16;

// Y[b, n, r] = (sum_m X[b, r, m] T[m, n]) * (W[n R + r] if WEIGHT); X real or complex, Y complex or (YREAL) its real
// part. grid (ceil(R / TR), ceil(N / TN), nb), 256 threads, 4 x 4 outputs per thread.
template <typename T, bool XREAL, bool WEIGHT, bool YREAL>
__global__ void __launch_bounds__(256) k_contract(const void* __restrict__ X_, const cpx<T>* __restrict__ Tw,
                                                  const T* __restrict__ W, void* __restrict__ Y_, int64_t R, int M,
                                                  int N) {
  __shared__ cpx<T> Xs[TK][TR + 1];
  __shared__ cpx<T> Ts[TK][TN + 1];
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  const int64_t r0 = (int64_t)blockIdx.x * TR;
  const int n0 = blockIdx.y * TN;
  const int64_t b = blockIdx.z;
  const int64_t xoff = b * R * (int64_t)M;
  cpx<T> acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) acc[i][j] = {T(0), T(0)};
  for (int m0 = 0; m0 < M; m0 += TK) {
    // X tile: TR rows (r) x TK (m); thread loads m = tid % 16, r = tid / 16 + 16 i
#pragma unroll
    for (int i = 0; i < 4; i++) {
      const int rr = (tid >> 4) + 16 * i, mm = tid & 15;
      const int64_t r = r0 + rr; const int m = m0 + mm;
      cpx<T> v = {T(0), T(0)};
      if (r < R && m < M) {
        if (XREAL) v.re = reinterpret_cast<const T*>(X_)[xoff + r * M + m];
        else v = reinterpret_cast<const cpx<T>*>(X_)[xoff + r * M + m];
      }
      Xs[mm][rr] = v;
    }
    // T tile: TK (m) x TN (n); thread loads n = tid % 64, m = tid / 64 + 4 i
#pragma unroll
    for (int i = 0; i < 4; i++) {
      const int nn = tid & 63, mm = (tid >> 6) + 4 * i;
      const int n = n0 + nn, m = m0 + mm;
      Ts[mm][nn] = (n < N && m < M) ? Tw[(int64_t)m * N + n] : cpx<T>{T(0), T(0)};
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < TK; kk++) {
      cpx<T> a[4], bb[4];
#pragma unroll
      for (int i = 0; i < 4; i++) a[i] = Xs[kk][tx + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; j++) bb[j] = Ts[kk][ty + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = cfma(a[i], bb[j], acc[i][j]);
    }
    __syncthreads();
  }
  const int64_t yoff = b * (int64_t)N * R;
#pragma unroll
  for (int j = 0; j < 4; j++) {
    const int n = n0 + ty + 16 * j;
    if (n >= N) continue;
#pragma unroll
    for (int i = 0; i < 4; i++) {
      const int64_t r = r0 + tx + 16 * i;
      if (r >= R) continue;
      cpx<T> v = acc[i][j];
      if (WEIGHT) { const T wv = W[(int64_t)n * R + r]; v.re *= wv; v.im *= wv; }
      if (YREAL) reinterpret_cast<T*>(Y_)[yoff + (int64_t)n * R + r] = v.re;
      else reinterpret_cast<cpx<T>*>(Y_)[yoff + (int64_t)n * R + r] = v;
    }
  }
}

// The same stage for small problems (one lattice of a few hundred bins per axis), where 64 x 64 tiles leave most
// SMs idle: 16 x 16 output tiles, one output per thread, K staged 32 deep. grid (ceil(R / 16), ceil(N / 16), nb).
constexpr int SR = 16, SN = 16, SK = 32;
template <typename T, bool XREAL, bool WEIGHT, bool YREAL>
__global__ void __launch_bounds__(256) k_contract_small(const void* __restrict__ X_, const cpx<T>* __restrict__ Tw,
                                                        const T* __restrict__ W, void* __restrict__ Y_, int64_t R,
                                                        int M, int N) {
  __shared__ cpx<T> Xs[SK][SR + 1];
  __shared__ cpx<T> Ts[SK][SN + 1];
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  const int64_t r0 = (int64_t)blockIdx.x * SR;
  const int n0 = blockIdx.y * SN;
  const int64_t b = blockIdx.z;
  const int64_t xoff = b * R * (int64_t)M;
  cpx<T> acc = {T(0), T(0)};
  for (int m0 = 0; m0 < M; m0 += SK) {
#pragma unroll
    for (int i = 0; i < 2; i++) {              // X tile: SR rows x SK (m), thread loads m = tid % 32, r = tid / 32 + 8 i
      const int mm = tid & 31, rr = (tid >> 5) + 8 * i;
      const int64_t r = r0 + rr; const int m = m0 + mm;
      cpx<T> v = {T(0), T(0)};
      if (r < R && m < M) {
        if (XREAL) v.re = reinterpret_cast<const T*>(X_)[xoff + r * M + m];
        else v = reinterpret_cast<const cpx<T>*>(X_)[xoff + r * M + m];
      }
      Xs[mm][rr] = v;
    }
#pragma unroll
    for (int i = 0; i < 2; i++) {              // T tile: SK (m) x SN (n), thread loads n = tid % 16, m = tid / 16 + 16 i
      const int nn = tid & 15, mm = (tid >> 4) + 16 * i;
      const int n = n0 + nn, m = m0 + mm;
      Ts[mm][nn] = (n < N && m < M) ? Tw[(int64_t)m * N + n] : cpx<T>{T(0), T(0)};
    }
    __syncthreads();
#pragma unroll 8
    for (int kk = 0; kk < SK; kk++) acc = cfma(Xs[kk][tx], Ts[kk][ty], acc);
    __syncthreads();
  }
  const int n = n0 + ty;
  const int64_t r = r0 + tx;
  if (n < N && r < R) {
    const int64_t o = b * (int64_t)N * R + (int64_t)n * R + r;
    if (WEIGHT) { const T wv = W[(int64_t)n * R + r]; acc.re *= wv; acc.im *= wv; }
    if (YREAL) reinterpret_cast<T*>(Y_)[o] = acc.re;
    else reinterpret_cast<cpx<T>*>(Y_)[o] = acc;
  }
}

template <typename T>
static int launch_stage(const void* X, bool xreal, const void* Tw, const void* W, void* Y, bool yreal, int64_t R,
                        int M, int N, int nb, cudaStream_t st) {
  dim3 grid((unsigned)((R + TR - 1) / TR), (unsigned)((N + TN - 1) / TN), (unsigned)nb);
  const cpx<T>* t = reinterpret_cast<const cpx<T>*>(Tw);
  const T* w = reinterpret_cast<const T*>(W);
  if ((int64_t)grid.x * grid.y * grid.z < 2 * 148) {     // too few big tiles to fill the GPU: small tiles
    dim3 gs((unsigned)((R + SR - 1) / SR), (unsigned)((N + SN - 1) / SN), (unsigned)nb);
    if (xreal && W) k_contract_small<T, true, true, false><<<gs, 256, 0, st>>>(X, t, w, Y, R, M, N);
    else if (xreal) k_contract_small<T, true, false, false><<<gs, 256, 0, st>>>(X, t, w, Y, R, M, N);
    else if (W) k_contract_small<T, false, true, false><<<gs, 256, 0, st>>>(X, t, w, Y, R, M, N);
    else if (yreal) k_contract_small<T, false, false, true><<<gs, 256, 0, st>>>(X, t, w, Y, R, M, N);
    else k_contract_small<T, false, false, false><<<gs, 256, 0, st>>>(X, t, w, Y, R, M, N);
    BLML_CHECK_LAUNCH("matvec stage");
    return BLML_OK;
  }
  // the combinations the stage schedule uses: first stage (real or complex input), last forward (weights),
  // last inverse (real output when the input was real), and plain complex stages
  if (xreal && W) k_contract<T, true, true, false><<<grid, 256, 0, st>>>(X, t, w, Y, R, M, N);
  else if (xreal) k_contract<T, true, false, false><<<grid, 256, 0, st>>>(X, t, w, Y, R, M, N);
  else if (W) k_contract<T, false, true, false><<<grid, 256, 0, st>>>(X, t, w, Y, R, M, N);
  else if (yreal) k_contract<T, false, false, true><<<grid, 256, 0, st>>>(X, t, w, Y, R, M, N);
  else k_contract<T, false, false, false><<<grid, 256, 0, st>>>(X, t, w, Y, R, M, N);
  BLML_CHECK_LAUNCH("matvec stage");
  return BLML_OK;
}

// the d forward stages alone, the weight in the last one's epilogue: spec = W (v^H x), (nb, H_1 ... H_d) natural order
template <typename T>
static int simt_forward(blml_plan_s* p, const void* x, void* spec, int nb, int xc, void* ws, cudaStream_t st) {
  const int d = p->d;
  std::vector<int64_t> dims(p->shape, p->shape + d);
  const size_t esz = sizeof(cpx<T>);
  char* buf[2] = {reinterpret_cast<char*>(ws), reinterpret_cast<char*>(ws) + (size_t)nb * p->max_elems * esz};
  const void* cur = x; bool cur_real = !xc; int which = 0;
  for (int s = 0; s < d; s++) {
    const int a = d - 1 - s;
    const int64_t M = dims.back();
    int64_t tot = 1; for (auto v : dims) tot *= v;
    const int64_t R = tot / M, N = p->nfreq[a];
    void* out = s == d - 1 ? spec : buf[which];
    int rc = launch_stage<T>(cur, cur_real, p->tf[a], s == d - 1 ? p->W : nullptr, out, false, R, (int)M, (int)N, nb,
                             st);
    if (rc) return rc;
    dims.pop_back(); dims.insert(dims.begin(), N);
    cur = out; cur_real = false; which ^= 1;
  }
  return BLML_OK;
}

template <typename T>
static int simt_matvec(blml_plan_s* p, const void* x, void* y, int nb, int xc, void* ws, cudaStream_t st) {
  const int d = p->d;
  std::vector<int64_t> dims(p->shape, p->shape + d);   // current axis order, natural at the start
  const size_t esz = sizeof(cpx<T>);
  char* buf[2] = {reinterpret_cast<char*>(ws), reinterpret_cast<char*>(ws) + (size_t)nb * p->max_elems * esz};
  const void* cur = x; bool cur_real = !xc; int which = 0;
  for (int s = 0; s < 2 * d; s++) {
    const bool fwd = s < d;
    const int a = d - 1 - (s % d);
    const int64_t M = dims.back();
    int64_t tot = 1; for (auto v : dims) tot *= v;
    const int64_t R = tot / M;
    const int64_t N = fwd ? p->nfreq[a] : p->shape[a];
    const bool last = s == 2 * d - 1;
    void* out = last ? y : buf[which];
    const void* Tw = fwd ? p->tf[a] : p->ti[a];
    const void* W = (s == d - 1) ? p->W : nullptr;
    int rc = launch_stage<T>(cur, cur_real, Tw, W, out, last && !xc, R, (int)M, (int)N, nb, st);
    if (rc) return rc;
    dims.pop_back(); dims.insert(dims.begin(), N);
    cur = out; cur_real = false; which ^= 1;
  }
  return BLML_OK;
}

// ---------------------------------------------------------------------------------------------- grouped stages
// One stage of many mat-vecs (different plans, lattice sizes and buffers) in one launch: problem g = blockIdx.z reads
// its descriptor; rows rho = b R + r of its nb lattices; 32 x 32 output tiles, 2 x 2 outputs per thread.
struct StageDesc {
  const void* X; const void* T; const void* W; void* Y;
  int64_t R; int M, N, nb, flags;      // flags: 1 real input, 2 weight epilogue, 4 real output
};
constexpr int GR = 32, GN = 32, GK = 16;

template <typename T>
__global__ void __launch_bounds__(256) k_contract_grouped(const StageDesc* __restrict__ descs,
                                                          const int* __restrict__ subset,
                                                          const int* __restrict__ live) {
  __shared__ cpx<T> Xs[GK][GR + 1];
  __shared__ cpx<T> Ts[GK][GN + 1];
  const int gi = subset ? subset[blockIdx.z] : blockIdx.z;
  if (live && !live[gi]) return;                       // uniform per CTA: a problem that has stopped
  const StageDesc D = descs[gi];
  const int64_t rows = D.R * D.nb;
  const int64_t r0 = (int64_t)blockIdx.x * GR;
  const int n0 = blockIdx.y * GN;
  if (r0 >= rows || n0 >= D.N) return;                 // uniform per CTA: past this problem's tiles
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  const bool xreal = D.flags & 1;
  const cpx<T>* Tw = reinterpret_cast<const cpx<T>*>(D.T);
  const int M = D.M, N = D.N;
  cpx<T> acc[2][2] = {{{T(0), T(0)}, {T(0), T(0)}}, {{T(0), T(0)}, {T(0), T(0)}}};
  for (int m0 = 0; m0 < M; m0 += GK) {
#pragma unroll
    for (int i = 0; i < 2; i++) {              // X tile GR x GK: m = tid % 16, row = tid / 16 + 16 i
      const int mm = tid & 15, rr = (tid >> 4) + 16 * i;
      const int64_t rho = r0 + rr; const int m = m0 + mm;
      cpx<T> v = {T(0), T(0)};
      if (rho < rows && m < M) {               // rows of all nb lattices are contiguous, M apart
        if (xreal) v.re = reinterpret_cast<const T*>(D.X)[rho * M + m];
        else v = reinterpret_cast<const cpx<T>*>(D.X)[rho * M + m];
      }
      Xs[mm][rr] = v;
    }
#pragma unroll
    for (int i = 0; i < 2; i++) {              // T tile GK x GN: n = tid % 32, m = tid / 32 + 8 i
      const int nn = tid & 31, mm = (tid >> 5) + 8 * i;
      const int n = n0 + nn, m = m0 + mm;
      Ts[mm][nn] = (n < N && m < M) ? Tw[(int64_t)m * N + n] : cpx<T>{T(0), T(0)};
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < GK; kk++) {
      const cpx<T> a0 = Xs[kk][tx], a1 = Xs[kk][tx + 16], b0 = Ts[kk][ty], b1 = Ts[kk][ty + 16];
      acc[0][0] = cfma(a0, b0, acc[0][0]); acc[0][1] = cfma(a0, b1, acc[0][1]);
      acc[1][0] = cfma(a1, b0, acc[1][0]); acc[1][1] = cfma(a1, b1, acc[1][1]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 2; i++)
#pragma unroll
    for (int j = 0; j < 2; j++) {
      const int64_t rho = r0 + tx + 16 * i; const int n = n0 + ty + 16 * j;
      if (rho >= rows || n >= N) continue;
      const int64_t b = rho / D.R, r = rho - b * D.R;
      const int64_t o = b * (int64_t)N * D.R + (int64_t)n * D.R + r;
      cpx<T> v = acc[i][j];
      if (D.flags & 2) { const T wv = reinterpret_cast<const T*>(D.W)[(int64_t)n * D.R + r]; v.re *= wv; v.im *= wv; }
      if (D.flags & 4) reinterpret_cast<T*>(D.Y)[o] = v.re;
      else reinterpret_cast<cpx<T>*>(D.Y)[o] = v;
    }
}

// The same stage with 64 x 64 output tiles (4 x 4 outputs per thread) and the operand tiles staged by cp.async into
// a double buffer, the next K slice loading while the current one is multiplied; for launches with enough tiles to
// fill the GPU. Dynamic shared memory: 2 buffers x (X tile + T tile), BK x (64 + 1) complex each.
__device__ __forceinline__ void cp_async(void* smem, const void* gmem, int bytes, bool pred) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  const int sz = pred ? bytes : 0;                 // 0: nothing read, the destination is zero-filled
  if (bytes == 16) asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(sz));
  else if (bytes == 8) asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(sz));
  else asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(s), "l"(gmem), "r"(sz));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N> __device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

constexpr int BR = 64, BN = 64, BK = 16, BLD = 65;
template <typename T>
constexpr size_t big_smem() { return 2 * 2 * (size_t)BK * BLD * sizeof(cpx<T>); }

template <typename T>
__global__ void __launch_bounds__(256, 2) k_contract_grouped_big(const StageDesc* __restrict__ descs,
                                                                 const int* __restrict__ subset,
                                                                 const int* __restrict__ live) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cpx<T>* Xs = reinterpret_cast<cpx<T>*>(smem_raw);             // [2][BK][BLD]
  cpx<T>* Ts = Xs + 2 * BK * BLD;                                // [2][BK][BLD]
  const int gi = subset ? subset[blockIdx.z] : blockIdx.z;
  if (live && !live[gi]) return;
  const StageDesc D = descs[gi];
  const int64_t rows = D.R * D.nb;
  const int64_t r0 = (int64_t)blockIdx.x * BR;
  const int n0 = blockIdx.y * BN;
  if (r0 >= rows || n0 >= D.N) return;
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  const bool xreal = D.flags & 1;
  const int M = D.M, N = D.N;
  const cpx<T>* Tw = reinterpret_cast<const cpx<T>*>(D.T);
  if (xreal) {                                   // real input: cp.async fills .re only, .im stays zero
    for (int i = tid; i < 2 * BK * BLD; i += 256) Xs[i] = cpx<T>{T(0), T(0)};
    __syncthreads();
  }
  auto load = [&](int buf, int m0) {
#pragma unroll
    for (int i = 0; i < 4; i++) {              // X tile: BR rows x BK (m); m = tid % 16, row = tid / 16 + 16 i
      const int mm = tid & 15, rr = (tid >> 4) + 16 * i;
      const int64_t rho = r0 + rr; const int m = m0 + mm;
      const bool ok = rho < rows && m < M;
      cpx<T>* dst = Xs + ((size_t)buf * BK + mm) * BLD + rr;
      if (xreal) {
        const T* src = reinterpret_cast<const T*>(D.X) + (ok ? rho * M + m : 0);
        cp_async(&dst->re, src, (int)sizeof(T), ok);
      } else {
        const cpx<T>* src = reinterpret_cast<const cpx<T>*>(D.X) + (ok ? rho * M + m : 0);
        cp_async(dst, src, (int)sizeof(cpx<T>), ok);
      }
    }
#pragma unroll
    for (int i = 0; i < 4; i++) {              // T tile: BK (m) x BN; n = tid % 64, m = tid / 64 + 4 i
      const int nn = tid & 63, mm = (tid >> 6) + 4 * i;
      const int n = n0 + nn, m = m0 + mm;
      const bool ok = n < N && m < M;
      cp_async(Ts + ((size_t)buf * BK + mm) * BLD + nn, Tw + (ok ? (int64_t)m * N + n : 0), (int)sizeof(cpx<T>), ok);
    }
    cp_async_commit();
  };
  cpx<T> acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) acc[i][j] = {T(0), T(0)};
  const int nk = (M + BK - 1) / BK;
  load(0, 0);
  for (int kt = 0; kt < nk; kt++) {
    const int buf = kt & 1;
    if (kt + 1 < nk) { load(buf ^ 1, (kt + 1) * BK); cp_async_wait<1>(); }
    else cp_async_wait<0>();
    __syncthreads();
    const cpx<T>* xs = Xs + (size_t)buf * BK * BLD;
    const cpx<T>* ts = Ts + (size_t)buf * BK * BLD;
#pragma unroll
    for (int kk = 0; kk < BK; kk++) {
      cpx<T> a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; i++) a[i] = xs[kk * BLD + tx + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; j++) b[j] = ts[kk * BLD + ty + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = cfma(a[i], b[j], acc[i][j]);
    }
    __syncthreads();                             // the buffer is refilled by the next iteration's load
  }
#pragma unroll
  for (int j = 0; j < 4; j++) {
    const int n = n0 + ty + 16 * j;
    if (n >= N) continue;
#pragma unroll
    for (int i = 0; i < 4; i++) {
      const int64_t rho = r0 + tx + 16 * i;
      if (rho >= rows) continue;
      const int64_t b = rho / D.R, r = rho - b * D.R;
      const int64_t o = b * (int64_t)N * D.R + (int64_t)n * D.R + r;
      cpx<T> v = acc[i][j];
      if (D.flags & 2) { const T wv = reinterpret_cast<const T*>(D.W)[(int64_t)n * D.R + r]; v.re *= wv; v.im *= wv; }
      if (D.flags & 4) reinterpret_cast<T*>(D.Y)[o] = v.re;
      else reinterpret_cast<cpx<T>*>(D.Y)[o] = v;
    }
  }
}

}  // namespace blml

// a set of mat-vecs applied together: per stage a device array of descriptors and the grid that covers them
struct blml_group_s {
  int G, d_max, dtype, nstages;
  std::vector<blml::StageDesc*> dev;    // one descriptor array per stage index
  std::vector<dim3> grids, grids_big;   // 32 x 32 and 64 x 64 tile grids per stage
  std::vector<double> tiles_big;        // 64 x 64 tiles of a stage over all problems
  void* ws;                             // the group's own intermediate buffers
  void* fft;                            // the FFT route's descriptors (every plan a DFT mask), or null
  int route;                            // BLML_ROUTE_CONTRACT or BLML_ROUTE_FFT
};

using namespace blml;

extern "C" {

int blml_plan_create(int d, const int64_t* shape, const int32_t* nfreq, const double* freqs, const double* weights,
                     int dtype, int engine, blml_plan* plan) {
  if (!plan || d < 1 || d > 8 || !shape || !nfreq || !freqs || !weights) {
    set_error("blml_plan_create: bad arguments"); return BLML_ERR_ARG;
  }
  if (dtype != BLML_F64 && dtype != BLML_F32) { set_error("blml_plan_create: dtype"); return BLML_ERR_ARG; }
  if (engine == BLML_ENGINE_TC && (dtype != BLML_F32 || d != 2)) {
    set_error("blml_plan_create: the tensor-core engine takes 2-D lattices in float32"); return BLML_ERR_UNSUPPORTED;
  }
  blml_plan_s* p = new blml_plan_s();
  p->d = d; p->dtype = dtype; p->engine = engine;
  int64_t nf_tot = 1, m_tot = 1;
  for (int a = 0; a < d; a++) {
    if (shape[a] < 1 || nfreq[a] < 1) { delete p; set_error("blml_plan_create: empty axis"); return BLML_ERR_ARG; }
    p->shape[a] = shape[a]; p->nfreq[a] = nfreq[a]; nf_tot *= nfreq[a]; m_tot *= shape[a];
  }
  // largest intermediate: after s forward stages the tensor holds the frequencies of axes >= d - s and the lattice
  // of the others; after s inverse stages the lattice of axes >= d - s and the frequencies of the others
  int64_t mx = 0;
  for (int s = 0; s <= d; s++) {
    int64_t ef = 1, ei = 1;
    for (int a = 0; a < d; a++) {
      ef *= (a >= d - s) ? nfreq[a] : shape[a];
      ei *= (a >= d - s) ? shape[a] : nfreq[a];
    }
    mx = std::max(mx, std::max(ef, ei));
  }
  p->max_elems = mx;
  const bool f64 = dtype == BLML_F64;
  const size_t esz = f64 ? 16 : 8;
  const double* fq = freqs;
  int rc = BLML_OK;
  std::vector<std::vector<double>> fwd_all(d), inv_all(d);
  for (int a = 0; a < d && rc == BLML_OK; a++) {
    const int64_t M = shape[a]; const int H = nfreq[a];
    std::vector<double>& fr = fwd_all[a];
    std::vector<double>& iv = inv_all[a];
    fr.resize(2 * M * H); iv.resize(2 * M * H);
    for (int64_t j = 0; j < M; j++)
      for (int q = 0; q < H; q++) {
        // phase in cycles, reduced before scaling by 2 pi
        double ph = fq[q] * (double)j; ph -= floor(ph);
        const double cs = cos(2.0 * M_PI * ph), sn = sin(2.0 * M_PI * ph);
        fr[2 * (j * H + q)] = cs; fr[2 * (j * H + q) + 1] = -sn;     // conj(v): forward (M x H)
        iv[2 * (q * M + j)] = cs; iv[2 * (q * M + j) + 1] = sn;      // v^T: inverse (H x M)
      }
    fq += H;
    for (int w = 0; w < 2; w++) {
      std::vector<double>& src = w ? iv : fr;
      void* dst = nullptr;
      if (cudaMalloc(&dst, M * H * esz) != cudaSuccess) { rc = BLML_ERR_CUDA; break; }
      if (f64) {
        rc = cuda_status(cudaMemcpy(dst, src.data(), M * H * esz, cudaMemcpyHostToDevice), "plan twiddles");
      } else {
        std::vector<float> s32(src.begin(), src.end());
        rc = cuda_status(cudaMemcpy(dst, s32.data(), M * H * esz, cudaMemcpyHostToDevice), "plan twiddles");
      }
      (w ? p->ti[a] : p->tf[a]) = dst;
    }
  }
  if (rc == BLML_OK) {
    if (cudaMalloc(&p->W, nf_tot * (f64 ? 8 : 4)) != cudaSuccess) rc = BLML_ERR_CUDA;
    else if (f64) rc = cuda_status(cudaMemcpy(p->W, weights, nf_tot * 8, cudaMemcpyHostToDevice), "plan weights");
    else {
      std::vector<float> w32(weights, weights + nf_tot);
      rc = cuda_status(cudaMemcpy(p->W, w32.data(), nf_tot * 4, cudaMemcpyHostToDevice), "plan weights");
    }
  }
  if (rc == BLML_OK && engine == BLML_ENGINE_TC) rc = tc_plan_init(p, fwd_all, inv_all);
  if (rc == BLML_OK && engine == BLML_ENGINE_SIMT) rc = fft_plan_init(p, freqs);
  p->route = p->fft ? BLML_ROUTE_FFT : BLML_ROUTE_CONTRACT;
  if (rc != BLML_OK) {
    if (rc == BLML_ERR_CUDA && blml_last_error()[0] == 0) set_error("blml_plan_create: device allocation failed");
    blml_plan_destroy(p);
    return rc;
  }
  *plan = p;
  return BLML_OK;
}

int blml_plan_destroy(blml_plan p) {
  if (!p) return BLML_OK;
  for (int a = 0; a < p->d; a++) { cudaFree(p->tf[a]); cudaFree(p->ti[a]); }
  cudaFree(p->W);
  if (p->tc) tc_plan_free(p);
  if (p->fft) fft_plan_free(p);
  delete p;
  return BLML_OK;
}

int blml_group_create(int G, const blml_plan* plans, const int* nbatch, int x_complex, const void* x_base,
                      const int64_t* x_off, void* y_base, const int64_t* y_off, blml_group* out) {
  if (G < 1 || G > 65535 || !plans || !nbatch || !x_off || !y_off || !out) {
    set_error("blml_group_create: bad arguments"); return BLML_ERR_ARG;
  }
  const int d = plans[0]->d, dtype = plans[0]->dtype;
  for (int g = 0; g < G; g++)
    if (!plans[g] || plans[g]->d != d || plans[g]->dtype != dtype || nbatch[g] < 1) {
      set_error("blml_group_create: every plan of a group has one dimension count and dtype"); return BLML_ERR_ARG;
    }
  // the 64 x 64 stage kernel's dynamic shared memory (set here, outside any stream capture)
  int e0 = cuda_status(cudaFuncSetAttribute(k_contract_grouped_big<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)big_smem<double>()), "blml_group_create");
  if (!e0) e0 = cuda_status(cudaFuncSetAttribute(k_contract_grouped_big<float>,
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)big_smem<float>()),
                            "blml_group_create");
  if (e0) return e0;
  const size_t esz = dtype == BLML_F64 ? 16 : 8, rsz = dtype == BLML_F64 ? 8 : 4;
  const size_t xsz = x_complex ? esz : rsz, ysz = x_complex ? esz : rsz;
  std::vector<size_t> wso(G + 1, 0);
  for (int g = 0; g < G; g++) wso[g + 1] = wso[g] + 2 * (size_t)nbatch[g] * plans[g]->max_elems * esz;
  blml_group_s* grp = new blml_group_s();
  grp->G = G; grp->d_max = d; grp->dtype = dtype; grp->nstages = 2 * d; grp->ws = nullptr;
  grp->fft = nullptr; grp->route = BLML_ROUTE_CONTRACT;
  if (cudaMalloc(&grp->ws, std::max<size_t>(wso[G], 16)) != cudaSuccess) {
    delete grp; set_error("blml_group_create: workspace allocation"); return BLML_ERR_CUDA;
  }
  std::vector<std::vector<StageDesc>> host(2 * d, std::vector<StageDesc>(G));
  std::vector<int64_t> maxr(2 * d, 0), maxn(2 * d, 0);
  grp->tiles_big.assign(2 * d, 0.0);
  for (int g = 0; g < G; g++) {
    const blml_plan_s* p = plans[g];
    std::vector<int64_t> dims(p->shape, p->shape + d);
    char* buf[2] = {reinterpret_cast<char*>(grp->ws) + wso[g],
                    reinterpret_cast<char*>(grp->ws) + wso[g] + (size_t)nbatch[g] * p->max_elems * esz};
    const void* cur = reinterpret_cast<const char*>(x_base) + x_off[g] * xsz;
    for (int s = 0; s < 2 * d; s++) {
      const bool fwd = s < d, last = s == 2 * d - 1;
      const int a = d - 1 - (s % d);
      const int64_t M = dims.back();
      int64_t tot = 1; for (auto v : dims) tot *= v;
      const int64_t R = tot / M, N = fwd ? p->nfreq[a] : p->shape[a];
      void* outp = last ? reinterpret_cast<char*>(y_base) + y_off[g] * ysz : buf[s & 1];
      StageDesc& D = host[s][g];
      D.X = cur; D.T = fwd ? p->tf[a] : p->ti[a]; D.W = (s == d - 1) ? p->W : nullptr; D.Y = outp;
      D.R = R; D.M = (int)M; D.N = (int)N; D.nb = nbatch[g];
      D.flags = ((s == 0 && !x_complex) ? 1 : 0) | ((s == d - 1) ? 2 : 0) | ((last && !x_complex) ? 4 : 0);
      maxr[s] = std::max(maxr[s], R * nbatch[g]); maxn[s] = std::max<int64_t>(maxn[s], N);
      grp->tiles_big[s] += (double)((R * nbatch[g] + BR - 1) / BR) * (double)((N + BN - 1) / BN);
      dims.pop_back(); dims.insert(dims.begin(), N);
      cur = outp;
    }
  }
  int e = BLML_OK;
  grp->dev.assign(2 * d, nullptr);
  for (int s = 0; s < 2 * d && !e; s++) {
    if (cudaMalloc(&grp->dev[s], G * sizeof(StageDesc)) != cudaSuccess) { set_error("blml_group_create: allocation"); e = BLML_ERR_CUDA; break; }
    e = cuda_status(cudaMemcpy(grp->dev[s], host[s].data(), G * sizeof(StageDesc), cudaMemcpyHostToDevice), "blml_group_create");
    grp->grids.push_back(dim3((unsigned)((maxr[s] + GR - 1) / GR), (unsigned)((maxn[s] + GN - 1) / GN), (unsigned)G));
    grp->grids_big.push_back(dim3((unsigned)((maxr[s] + BR - 1) / BR), (unsigned)((maxn[s] + BN - 1) / BN), (unsigned)G));
  }
  if (!e) {      // the FFT route: problem g keeps its spectrum in the first of its two intermediate buffers
    std::vector<const void*> xs(G); std::vector<void*> ys(G), zs(G);
    for (int g = 0; g < G; g++) {
      xs[g] = reinterpret_cast<const char*>(x_base) + x_off[g] * xsz;
      ys[g] = reinterpret_cast<char*>(y_base) + y_off[g] * ysz;
      zs[g] = reinterpret_cast<char*>(grp->ws) + wso[g];
    }
    e = fft_group_init(&grp->fft, G, plans, nbatch, x_complex, xs.data(), ys.data(), zs.data());
    if (!e && grp->fft) grp->route = BLML_ROUTE_FFT;
  }
  if (e) { blml_group_destroy(grp); return e; }
  *out = grp;
  return BLML_OK;
}

int blml_group_matvec(blml_group grp, void* stream) {
  return blml_group_matvec_masked(grp, nullptr, grp ? grp->G : 0, nullptr, stream);
}

int blml_group_matvec_masked(blml_group grp, const int* subset, int n, const int* live, void* stream) {
  if (!grp) { set_error("blml_group_matvec: null group"); return BLML_ERR_ARG; }
  if (n < 0 || n > grp->G) { set_error("blml_group_matvec_masked: 0 <= n <= G"); return BLML_ERR_ARG; }
  if (n == 0) return BLML_OK;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  if (grp->route == BLML_ROUTE_FFT) return fft_group_launch(grp->fft, grp->dtype, subset, n, live, st);
  for (int s = 0; s < grp->nstages; s++) {
    // 64 x 64 tiles when the launch has enough of them to fill the GPU twice over (the problems of a subset are
    // taken as average ones), else 32 x 32
    const bool big = grp->tiles_big[s] * n / grp->G >= 2.0 * 148;
    dim3 g = big ? grp->grids_big[s] : grp->grids[s]; g.z = (unsigned)n;
    if (big) {
      if (grp->dtype == BLML_F64)
        k_contract_grouped_big<double><<<g, 256, big_smem<double>(), st>>>(grp->dev[s], subset, live);
      else k_contract_grouped_big<float><<<g, 256, big_smem<float>(), st>>>(grp->dev[s], subset, live);
    } else {
      if (grp->dtype == BLML_F64) k_contract_grouped<double><<<g, 256, 0, st>>>(grp->dev[s], subset, live);
      else k_contract_grouped<float><<<g, 256, 0, st>>>(grp->dev[s], subset, live);
    }
    BLML_CHECK_LAUNCH("blml_group_matvec");
  }
  return BLML_OK;
}

int blml_group_destroy(blml_group grp) {
  if (!grp) return BLML_OK;
  for (auto p : grp->dev) cudaFree(p);
  cudaFree(grp->ws);
  fft_group_free(grp->fft);
  delete grp;
  return BLML_OK;
}

int blml_plan_status(blml_plan p) {
  if (!p) { set_error("blml_plan_status: null plan"); return BLML_ERR_ARG; }
  int e = cuda_status(cudaDeviceSynchronize(), "blml_plan_status");
  if (e) return e;
  if (p->tc && tc_error(p)) { set_error("tensor-core mat-vec: a bounded wait timed out"); return BLML_ERR_TIMEOUT; }
  return BLML_OK;
}

int64_t blml_matvec_workspace(blml_plan p, int nb) {
  if (!p || nb < 1) return -1;
  if (p->engine == BLML_ENGINE_TC) return tc_workspace(p, nb);
  if (p->route == BLML_ROUTE_FFT) return fft_workspace(p, nb);
  return 2 * (int64_t)nb * p->max_elems * (p->dtype == BLML_F64 ? 16 : 8);
}

int blml_matvec(blml_plan p, const void* x, void* y, int nb, int xc, void* ws, int64_t wsb, void* stream) {
  if (!p || !x || !y || nb < 1) { set_error("blml_matvec: bad arguments"); return BLML_ERR_ARG; }
  const int64_t need = blml_matvec_workspace(p, nb);
  if (wsb < need || (need > 0 && !ws)) {
    set_error("blml_matvec: workspace of %lld bytes, need %lld", (long long)wsb, (long long)need);
    return BLML_ERR_WORKSPACE;
  }
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  if (p->engine == BLML_ENGINE_TC) return tc_matvec(p, x, y, nb, xc, ws, wsb, st);
  if (p->route == BLML_ROUTE_FFT) return fft_matvec(p, x, y, nb, xc, ws, st);
  return p->dtype == BLML_F64 ? simt_matvec<double>(p, x, y, nb, xc, ws, st)
                              : simt_matvec<float>(p, x, y, nb, xc, ws, st);
}

int blml_plan_set_route(blml_plan p, int route) {
  if (!p) { set_error("blml_plan_set_route: null plan"); return BLML_ERR_ARG; }
  if (route == BLML_ROUTE_AUTO) route = p->fft ? BLML_ROUTE_FFT : BLML_ROUTE_CONTRACT;
  if (route == BLML_ROUTE_FFT && !p->fft) {
    set_error("blml_plan_set_route: this kernel has no FFT route (not a 2-D DFT mask on sides 2^a 3^b)");
    return BLML_ERR_UNSUPPORTED;
  }
  if (route != BLML_ROUTE_FFT && route != BLML_ROUTE_CONTRACT) { set_error("blml_plan_set_route: route"); return BLML_ERR_ARG; }
  p->route = route;
  return BLML_OK;
}

int blml_plan_route(blml_plan p) { return p ? p->route : BLML_ERR_ARG; }

int blml_group_set_route(blml_group grp, int route) {
  if (!grp) { set_error("blml_group_set_route: null group"); return BLML_ERR_ARG; }
  if (route == BLML_ROUTE_AUTO) route = grp->fft ? BLML_ROUTE_FFT : BLML_ROUTE_CONTRACT;
  if (route == BLML_ROUTE_FFT && !grp->fft) {
    set_error("blml_group_set_route: a plan of this group has no FFT route"); return BLML_ERR_UNSUPPORTED;
  }
  if (route != BLML_ROUTE_FFT && route != BLML_ROUTE_CONTRACT) { set_error("blml_group_set_route: route"); return BLML_ERR_ARG; }
  grp->route = route;
  return BLML_OK;
}

int blml_group_route(blml_group grp) { return grp ? grp->route : BLML_ERR_ARG; }

int blml_spectrum(blml_plan p, const void* x, void* spec, int nb, int xc, void* ws, int64_t wsb, void* stream) {
  if (!p || !x || !spec || nb < 1) { set_error("blml_spectrum: bad arguments"); return BLML_ERR_ARG; }
  if (p->engine != BLML_ENGINE_SIMT) { set_error("blml_spectrum: SIMT plans only"); return BLML_ERR_UNSUPPORTED; }
  const int64_t need = 2 * (int64_t)nb * p->max_elems * (p->dtype == BLML_F64 ? 16 : 8);
  if (wsb < need || !ws) {
    set_error("blml_spectrum: workspace of %lld bytes, need %lld", (long long)wsb, (long long)need);
    return BLML_ERR_WORKSPACE;
  }
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  return p->dtype == BLML_F64 ? simt_forward<double>(p, x, spec, nb, xc, ws, st)
                              : simt_forward<float>(p, x, spec, nb, xc, ws, st);
}

int64_t blml_spectrum_workspace(blml_plan p, int nb) {
  if (!p || nb < 1) return -1;
  return 2 * (int64_t)nb * p->max_elems * (p->dtype == BLML_F64 ? 16 : 8);
}

}
