// Segmented kernels of the batched engine: many independent fits of uneven lattice size advance in lockstep, each
// phase one launch over all fits. Fit f owns the slice [off_f, off_f + K_f B_f) of every flat mode array (K_f modes of
// B_f bins, the (K, B) layout of one fit) and [boff_f, boff_f + B_f) of every flat bin array (counts, signs);
// blockIdx.y is the fit, blockIdx.x strides over its bins. Per-fit scalars (step sizes, scales, linear-combination
// coefficients) come from device arrays, so a whole phase needs no host round trip. Reductions are per-fit float64
// block partials summed in a fixed order by blml_seg_finish.
#include "common.cuh"
#include "plan.cuh"
#include "segmented.cuh"

namespace blml {

// one block per fit: out[f * nq + q] = fixed-order reduction of its partials (F = gridDim.x fits)
__global__ void k_seg_finish(const double* part, int nq, int nblk, unsigned maxmask, double* out) {
  const int f = blockIdx.x;
  for (int q = 0; q < nq; q++) {
    const bool mx = (maxmask >> q) & 1u;
    double acc = mx ? -INFINITY : 0.0;
    for (int i = threadIdx.x; i < nblk; i += blockDim.x) {
      const double v = part[((int64_t)q * gridDim.x + f) * nblk + i];
      acc = mx ? fmax(acc, v) : acc + v;
    }
    __shared__ double sh[32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    double x = mx ? warp_max(acc) : warp_sum(acc);
    if (lane == 0) sh[wid] = x;
    __syncthreads();
    if (wid == 0) {
      x = lane < nw ? sh[lane] : (mx ? -INFINITY : 0.0);
      x = mx ? warp_max(x) : warp_sum(x);
      if (lane == 0) out[(int64_t)f * nq + q] = x;
    }
    __syncthreads();
  }
}

// the same with the results of fit f at out[f * stride + q] (several passes fill one fit-major table)
__global__ void k_seg_finish_strided(const double* part, int nq, int nblk, double* out, int stride) {
  const int f = blockIdx.x;
  for (int q = 0; q < nq; q++) {
    double acc = 0.0;
    for (int i = threadIdx.x; i < nblk; i += blockDim.x) acc += part[((int64_t)q * gridDim.x + f) * nblk + i];
    __shared__ double sh[32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    double x = warp_sum(acc);
    if (lane == 0) sh[wid] = x;
    __syncthreads();
    if (wid == 0) {
      x = lane < nw ? sh[lane] : 0.0;
      x = warp_sum(x);
      if (lane == 0) out[(int64_t)f * stride + q] = x;
    }
    __syncthreads();
  }
}

template <typename T>
__global__ void k_seg_start_root(const blml_seg* segs, const T* c, const T* sg, const double* s0, T* e0) {
  const blml_seg S = segs[blockIdx.y];
  SEG_LOOP(b, S) {
    const double cb = (double)c[S.boff + b];
    e0[S.off + b] = (T)(cb > 0 ? sqrt(cb / s0[blockIdx.y]) * (double)sg[S.boff + b] : 0.0);
  }
}

__device__ __forceinline__ double cd_root_s(double b, double c, double s) {
  const double disc = sqrt(b * b + 4.0 * s * c);
  return b >= 0 ? 2.0 * c / fmax(b + disc, 1e-300) : (-b + disc) / (2.0 * s);
}

template <typename T>
__global__ void k_seg_update_real1(const blml_seg* segs, const T* E, const T* U, const T* c, const T* sg,
                                   const double* s0, T* out) {
  const blml_seg S = segs[blockIdx.y];
  const double s = s0[blockIdx.y];
  SEG_LOOP(b, S) {
    const double cb = (double)c[S.boff + b], sgb = (double)sg[S.boff + b];
    double t = 0.0;
    if (cb > 0) t = cd_root_s(sgb * ((double)U[S.off + b] - s * (double)E[S.off + b]), cb, s);
    out[S.off + b] = (T)(sgb * t);
  }
}

// merit terms per fit: psd [sum c log max(F, 1e-30), Q, 0]; real rank 1 [sum e u, sum_occ c log|e|, #(sg e <= 0)]
template <typename T, bool CPLX>
__global__ void k_seg_merit(const blml_seg* segs, int psd, const void* E, const void* U, const T* c, const T* sg,
                            double* part) {
  const blml_seg S = segs[blockIdx.y];
  double v[3] = {0.0, 0.0, 0.0};
  SEG_LOOP(b, S) {
    const double cb = (double)c[S.boff + b];
    if (psd) {
      double F = 0.0, Q = 0.0;
      for (int k = 0; k < S.K; k++) {
        double er, ei, ur, ui;
        const int64_t i = S.off + (int64_t)k * S.B + b;
        SAcc<T, CPLX>::get(E, i, er, ei); SAcc<T, CPLX>::get(U, i, ur, ui);
        F += ur * ur + ui * ui; Q += er * ur + ei * ui;
      }
      if (cb != 0.0) v[0] += cb * log(fmax(F, 1e-30));
      v[1] += Q;
    } else {
      double e, im, u;
      SAcc<T, CPLX>::get(E, S.off + b, e, im); SAcc<T, CPLX>::get(U, S.off + b, u, im);
      v[0] += e * u;
      if (cb > 0) { v[1] += cb * log(fabs(e)); if ((double)sg[S.boff + b] * e <= 0) v[2] += 1.0; }
    }
  }
  seg_partials<3>(v, part);
}

template <typename T, bool CPLX>
__global__ void k_seg_resid(const blml_seg* segs, const void* E, const void* U, const T* c, const double* scale,
                            double* part) {
  const blml_seg S = segs[blockIdx.y];
  const double sc = scale[blockIdx.y];
  double v[2] = {0.0, 0.0};
  SEG_LOOP(b, S) {
    const double cb = (double)c[S.boff + b];
    if (!(cb > 0)) continue;
    double nrm2 = 0.0;
    for (int k = 0; k < S.K; k++) {
      double er, ei; SAcc<T, CPLX>::get(E, S.off + (int64_t)k * S.B + b, er, ei);
      er *= sc; ei *= sc; nrm2 += er * er + ei * ei;
    }
    const double f = nrm2 / cb;
    double r2 = 0.0;
    for (int k = 0; k < S.K; k++) {
      double er, ei, ur, ui;
      const int64_t i = S.off + (int64_t)k * S.B + b;
      SAcc<T, CPLX>::get(E, i, er, ei); SAcc<T, CPLX>::get(U, i, ur, ui);
      const double dr = ur * sc * f - er * sc, di = ui * sc * f - ei * sc;
      r2 += dr * dr + di * di;
    }
    const double r = sqrt(r2) / sqrt(fmax(nrm2, 1e-300));
    if (r != r) v[1] += 1.0; else v[0] = fmax(v[0], r);
  }
  seg_partials<2>(v, part, 1u);
}

struct SegPairs { const void* a[48]; const void* b[48]; };

// per-fit real inner products over the fit's K B elements (complex: 2 K B reals)
template <typename T, int NP>
__global__ void k_seg_dots(const blml_seg* segs, int cplx, int np, SegPairs pp, double* part) {
  const blml_seg S = segs[blockIdx.y];
  const int64_t w = cplx ? 2 : 1;
  const int64_t o = S.off * w, n = (int64_t)S.K * S.B * w;
  double v[NP];
#pragma unroll
  for (int q = 0; q < NP; q++) v[q] = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
#pragma unroll
    for (int q = 0; q < NP; q++)
      if (q < np) v[q] += (double)reinterpret_cast<const T*>(pp.a[q])[o + i] *
                          (double)reinterpret_cast<const T*>(pp.b[q])[o + i];
  }
  seg_partials<NP>(v, part);
}

struct SegList { const void* a[20]; };

// the history scan of the batched L-BFGS: per fit, for the np <= 20 vectors a_q, out = [a_q . b0 (np), a_q . b1 (np),
// b0 . b0, b1 . b1, x . x] (x may be null: 0); b0, b1, x read once per element whatever np is
template <typename T>
__global__ void __launch_bounds__(256) k_seg_dots2(const blml_seg* segs, int cplx, int np, SegList al, const void* b0,
                                                   const void* b1, const void* x, double* part) {
  const blml_seg S = segs[blockIdx.y];
  const int64_t w = cplx ? 2 : 1;
  const int64_t o = S.off * w, n = (int64_t)S.K * S.B * w;
  double v[43];
#pragma unroll
  for (int q = 0; q < 43; q++) v[q] = 0.0;
  const T* B0 = reinterpret_cast<const T*>(b0) + o;
  const T* B1 = reinterpret_cast<const T*>(b1) + o;
  const T* X = x ? reinterpret_cast<const T*>(x) + o : nullptr;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double y0 = (double)B0[i], y1 = (double)B1[i];
#pragma unroll
    for (int q = 0; q < 20; q++)
      if (q < np) {
        const double a = (double)reinterpret_cast<const T*>(al.a[q])[o + i];
        v[q] += a * y0; v[20 + q] += a * y1;
      }
    v[40] += y0 * y0; v[41] += y1 * y1;
    if (X) { const double z = (double)X[i]; v[42] += z * z; }
  }
  seg_partials<43>(v, part);
}

// the same scan for float64 complex vectors, one (re, im) load per element and vector -- the stored vectors (TA)
// and the first shared one (TB0) complex128 (the plain fits' history; the float32 history has its own scan,
// k_seg_dots2_h32, with twice the elements per thread and a block split by fit size). The block's 8 warps
// split the stored vectors (warp w takes q = w, w + 8, w + 16) and walk the same 64-element tiles, so each thread
// holds at most 6 accumulators (full occupancy, many loads in flight) and the two shared vectors are read from HBM
// once per tile and from L1 by the other warps; the last warp also sums the three squared norms. Each quantity's
// block partial comes from one warp (warp_sum, fixed order), in seg_partials' layout.
// one complex128 element as (re, im)
__device__ __forceinline__ double2 ld_c2(const double2* p) { return __ldg(p); }

template <typename TA, typename TB0>
__global__ void __launch_bounds__(256, 3) k_seg_dots2_c128(const blml_seg* segs, int np, SegList al, const void* b0,
                                                           const void* b1, const void* x, double* part) {
  const blml_seg S = segs[blockIdx.y];
  const int64_t o = S.off, n = (int64_t)S.K * S.B;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const TB0* B0 = reinterpret_cast<const TB0*>(b0) + o;
  const double2* B1 = reinterpret_cast<const double2*>(b1) + o;
  const double2* X = x ? reinterpret_cast<const double2*>(x) + o : nullptr;
  const TA* A[3];
  int na = 0;
#pragma unroll
  for (int j = 0; j < 3; j++) {
    const int q = warp + nw * j;
    A[j] = q < np ? reinterpret_cast<const TA*>(al.a[q]) + o : nullptr;
    na += q < np;
  }
  const bool norms = warp == nw - 1;
  double a0[3] = {0.0, 0.0, 0.0}, a1[3] = {0.0, 0.0, 0.0}, n0 = 0.0, n1 = 0.0, nx = 0.0;
  const double2 zero = make_double2(0.0, 0.0);
  for (int64_t t = (int64_t)blockIdx.x * 64; t < n; t += (int64_t)gridDim.x * 64) {
    // both elements' loads issued together: out-of-range lanes read element 0 and zero its shared values, so their
    // products and norms add nothing
    const int64_t i0 = t + lane, i1 = t + 32 + lane;
    const bool v0 = i0 < n, v1 = i1 < n;
    const int64_t j0 = v0 ? i0 : 0, j1 = v1 ? i1 : 0;
    double2 y00 = ld_c2(B0 + j0), y01 = ld_c2(B0 + j1), y10 = __ldg(B1 + j0), y11 = __ldg(B1 + j1);
    double2 a[3][2];
#pragma unroll
    for (int j = 0; j < 3; j++)
      if (j < na) { a[j][0] = ld_c2(A[j] + j0); a[j][1] = ld_c2(A[j] + j1); }
    double2 z0 = zero, z1 = zero;
    if (norms && X) { z0 = __ldg(X + j0); z1 = __ldg(X + j1); }
    if (!v0) { y00 = zero; y10 = zero; z0 = zero; }
    if (!v1) { y01 = zero; y11 = zero; z1 = zero; }
#pragma unroll
    for (int j = 0; j < 3; j++)
      if (j < na) {
        a0[j] += a[j][0].x * y00.x + a[j][0].y * y00.y; a1[j] += a[j][0].x * y10.x + a[j][0].y * y10.y;
        a0[j] += a[j][1].x * y01.x + a[j][1].y * y01.y; a1[j] += a[j][1].x * y11.x + a[j][1].y * y11.y;
      }
    if (norms) {
      n0 += y00.x * y00.x + y00.y * y00.y; n1 += y10.x * y10.x + y10.y * y10.y; nx += z0.x * z0.x + z0.y * z0.y;
      n0 += y01.x * y01.x + y01.y * y01.y; n1 += y11.x * y11.x + y11.y * y11.y; nx += z1.x * z1.x + z1.y * z1.y;
    }
  }
  const int64_t slot = (int64_t)blockIdx.y * gridDim.x + blockIdx.x, qs = (int64_t)gridDim.y * gridDim.x;
#pragma unroll
  for (int j = 0; j < 3; j++) {
    const double s0 = warp_sum(a0[j]), s1 = warp_sum(a1[j]);
    if (j < na && lane == 0) {
      const int q = warp + nw * j;
      part[q * qs + slot] = s0; part[(20 + q) * qs + slot] = s1;
    }
  }
  if (norms) {
    n0 = warp_sum(n0); n1 = warp_sum(n1); nx = warp_sum(nx);
    if (lane == 0) { part[40 * qs + slot] = n0; part[41 * qs + slot] = n1; part[42 * qs + slot] = nx; }
  }
}

// out[f * (2 np + 3) + q] from the 43-quantity partials (quantities 20.. shifted down when np < 20)
__global__ void k_seg_finish_dots2(const double* part, int np, int nblk, double* out) {
  const int f = blockIdx.x, F = gridDim.x, nq = 2 * np + 3;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int q = wid; q < nq; q += nw) {
    const int src = q < np ? q : (q < 2 * np ? 20 + (q - np) : 40 + (q - 2 * np));
    double acc = 0.0;
    for (int i = lane; i < nblk; i += 32) acc += part[((int64_t)src * F + f) * nblk + i];
    acc = warp_sum(acc);
    if (lane == 0) out[(int64_t)f * nq + q] = acc;
  }
}

// The block split of segmented.cuh (one block of 1024 threads): N = sum_f K_f B_f, fit f with n_f elements gets
// nb_f = min(ceil(G n_f / N), ceil(n_f / SEG_SPLIT_MIN_ELEMS)) blocks (0 when n_f = 0), so sum_f nb_f <= G + F; then
// bstart by an exclusive scan and fit_of by a binary search per block.
__global__ void __launch_bounds__(1024) k_seg_split(int F, const blml_seg* segs, int G, int* split) {
  __shared__ long long sh[1024];
  __shared__ long long total;
  const int tid = threadIdx.x, chunk = (F + 1023) / 1024, f0 = tid * chunk, f1 = min(F, f0 + chunk);
  long long nsum = 0;
  for (int f = f0; f < f1; f++) nsum += (long long)segs[f].K * segs[f].B;
  sh[tid] = nsum;
  __syncthreads();
  for (int s = 512; s > 0; s >>= 1) {
    if (tid < s) sh[tid] += sh[tid + s];
    __syncthreads();
  }
  if (tid == 0) total = sh[0];
  __syncthreads();
  const long long N = total;
  long long mine = 0;
  for (int f = f0; f < f1; f++) {
    const long long n = (long long)segs[f].K * segs[f].B;
    if (n > 0) {
      const long long a = (G * n + N - 1) / N, b = (n + SEG_SPLIT_MIN_ELEMS - 1) / SEG_SPLIT_MIN_ELEMS;
      mine += a < b ? a : b;
    }
  }
  __syncthreads();
  sh[tid] = mine;
  __syncthreads();
  for (int s = 1; s < 1024; s <<= 1) {            // inclusive scan of the per-thread block counts
    const long long v = tid >= s ? sh[tid - s] : 0;
    __syncthreads();
    sh[tid] += v;
    __syncthreads();
  }
  long long at = sh[tid] - mine;
  for (int f = f0; f < f1; f++) {
    split[f] = (int)at;
    const long long n = (long long)segs[f].K * segs[f].B;
    if (n > 0) {
      const long long a = (G * n + N - 1) / N, b = (n + SEG_SPLIT_MIN_ELEMS - 1) / SEG_SPLIT_MIN_ELEMS;
      at += a < b ? a : b;
    }
  }
  if (tid == 1023) split[F] = (int)sh[1023];
  __syncthreads();
  const int used = (int)sh[1023];
  int* fit_of = split + F + 1;
  for (int b = tid; b < G + F; b += 1024) {
    int f = -1;
    if (b < used) {                                 // the last f with bstart[f] <= b (empty fits share a start)
      int lo = 0, hi = F - 1;
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (split[mid] <= b) lo = mid; else hi = mid - 1;
      }
      f = lo;
    }
    fit_of[b] = f;
  }
}

// The complex64-history scan over a block split: the stored vectors a_q and b0 complex64, b1 and x complex128, the
// quantities of k_seg_dots2_c128 (same warp roles: warp w takes q = w, w + 8, w + 16, the last warp the norms). Each
// thread loads 4 elements per tile (128-element tiles), twice the complex128 kernel's 2 at half the bytes each, so as
// many bytes are in flight per thread; full tiles take unchecked loads at fixed offsets from one base, the fit's last
// tile the checked ones. Two blocks per SM leave the registers for that without spills.
template <bool CHECK>
__device__ __forceinline__ void h32_tile(int64_t t, int64_t n, int lane, const float2* const* A, int na,
                                         const float2* B0, const double2* B1, const double2* X, bool norms,
                                         double* a0, double* a1, double& n0, double& n1, double& nx) {
  constexpr int EL = 4;
  const double2 zero = make_double2(0.0, 0.0);
  float2 ra[3][EL], r0[EL];
  double2 y1[EL], z[EL];
  bool v[EL];
  if (CHECK) {
    int64_t j[EL];
#pragma unroll
    for (int e = 0; e < EL; e++) { const int64_t i = t + 32 * e + lane; v[e] = i < n; j[e] = v[e] ? i : 0; }
#pragma unroll
    for (int e = 0; e < EL; e++) { r0[e] = __ldg(B0 + j[e]); y1[e] = __ldg(B1 + j[e]); z[e] = zero; }
#pragma unroll
    for (int q = 0; q < 3; q++)
      if (q < na) {
#pragma unroll
        for (int e = 0; e < EL; e++) ra[q][e] = __ldg(A[q] + j[e]);
      }
    if (norms && X) {
#pragma unroll
      for (int e = 0; e < EL; e++) z[e] = __ldg(X + j[e]);
    }
  } else {
    const int64_t base = t + lane;
#pragma unroll
    for (int e = 0; e < EL; e++) {
      v[e] = true; r0[e] = __ldg(B0 + base + 32 * e); y1[e] = __ldg(B1 + base + 32 * e); z[e] = zero;
    }
#pragma unroll
    for (int q = 0; q < 3; q++)
      if (q < na) {
        const float2* p = A[q] + base;
#pragma unroll
        for (int e = 0; e < EL; e++) ra[q][e] = __ldg(p + 32 * e);
      }
    if (norms && X) {
#pragma unroll
      for (int e = 0; e < EL; e++) z[e] = __ldg(X + base + 32 * e);
    }
  }
  double2 y0[EL];
#pragma unroll
  for (int e = 0; e < EL; e++) {
    y0[e] = make_double2((double)r0[e].x, (double)r0[e].y);
    if (CHECK && !v[e]) { y0[e] = zero; y1[e] = zero; z[e] = zero; }
  }
#pragma unroll
  for (int q = 0; q < 3; q++)
    if (q < na) {
#pragma unroll
      for (int e = 0; e < EL; e++) {
        const double ax = (double)ra[q][e].x, ay = (double)ra[q][e].y;
        a0[q] += ax * y0[e].x + ay * y0[e].y;
        a1[q] += ax * y1[e].x + ay * y1[e].y;
      }
    }
  if (norms) {
#pragma unroll
    for (int e = 0; e < EL; e++) {
      n0 += y0[e].x * y0[e].x + y0[e].y * y0[e].y; n1 += y1[e].x * y1[e].x + y1[e].y * y1[e].y;
      nx += z[e].x * z[e].x + z[e].y * z[e].y;
    }
  }
}

__global__ void __launch_bounds__(256, 2) k_seg_dots2_h32(const blml_seg* segs, const int* split, int F, int np,
                                                          SegList al, const float2* b0, const double2* b1,
                                                          const double2* x, double* part) {
  const int b = blockIdx.x, W = gridDim.x, f = split[F + 1 + b];
  if (f < 0) return;
  const int lb = b - split[f], nb = split[f + 1] - split[f];
  const blml_seg S = segs[f];
  const int64_t o = S.off, n = (int64_t)S.K * S.B;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const float2* B0 = b0 + o;
  const double2* B1 = b1 + o;
  const double2* X = x ? x + o : nullptr;
  const float2* A[3];
  int na = 0;
#pragma unroll
  for (int j = 0; j < 3; j++) {
    const int q = warp + nw * j;
    A[j] = q < np ? reinterpret_cast<const float2*>(al.a[q]) + o : nullptr;
    na += q < np;
  }
  const bool norms = warp == nw - 1;
  double a0[3] = {0.0, 0.0, 0.0}, a1[3] = {0.0, 0.0, 0.0}, n0 = 0.0, n1 = 0.0, nx = 0.0;
  constexpr int64_t T = 128;
  const int64_t stride = (int64_t)nb * T;
  int64_t t = (int64_t)lb * T;
  for (; t + T <= n; t += stride) h32_tile<false>(t, n, lane, A, na, B0, B1, X, norms, a0, a1, n0, n1, nx);
  for (; t < n; t += stride) h32_tile<true>(t, n, lane, A, na, B0, B1, X, norms, a0, a1, n0, n1, nx);
#pragma unroll
  for (int j = 0; j < 3; j++) {
    const double s0 = warp_sum(a0[j]), s1 = warp_sum(a1[j]);
    if (j < na && lane == 0) {
      const int q = warp + nw * j;
      part[(int64_t)q * W + b] = s0; part[(int64_t)(20 + q) * W + b] = s1;
    }
  }
  if (norms) {
    n0 = warp_sum(n0); n1 = warp_sum(n1); nx = warp_sum(nx);
    if (lane == 0) { part[40LL * W + b] = n0; part[41LL * W + b] = n1; part[42LL * W + b] = nx; }
  }
}

// out[f * (2 np + 3) + q] from a split scan's partials: fit f's blocks [bstart[f], bstart[f + 1]), fixed order
__global__ void k_seg_finish_dots2_split(const double* part, int W, const int* split, int np, double* out) {
  const int f = blockIdx.x, nq = 2 * np + 3;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int b0 = split[f], b1 = split[f + 1];
  for (int q = wid; q < nq; q += nw) {
    const int src = q < np ? q : (q < 2 * np ? 20 + (q - np) : 40 + (q - 2 * np));
    double acc = 0.0;
    for (int i = b0 + lane; i < b1; i += 32) acc += part[(int64_t)src * W + i];
    acc = warp_sum(acc);
    if (lane == 0) out[(int64_t)f * nq + q] = acc;
  }
}

struct SegTerms { const void* v[48]; };

// out = sum_i coef[f * nt + i] v_i over each fit's slice. The block lists the fit's nonzero terms (pointer, coefficient)
// in shared memory once; each thread then takes two elements at a time and issues the loads of four terms together,
// summing in term order (the sum of the terms in order, zero terms skipped, as a plain loop would). V is the element
// type (double2 / float2: one (re, im) load per complex element). out may be one of the terms: every element is read
// before the same thread writes it.
template <typename T, typename V>
__global__ void __launch_bounds__(256) k_seg_lincomb(const blml_seg* segs, int cplx, T* out, int nt,
                                                     const double* coef, SegTerms t) {
  __shared__ const V* sp[48];
  __shared__ double sc[48];
  __shared__ int snz;
  const blml_seg S = segs[blockIdx.y];
  const double* cf = coef + (int64_t)blockIdx.y * nt;
  if (threadIdx.x == 0) {
    int c = 0;
    for (int q = 0; q < nt; q++) {
      const double v = cf[q];
      if (v != 0.0) { sp[c] = reinterpret_cast<const V*>(t.v[q]); sc[c] = v; c++; }
    }
    snz = c;
  }
  __syncthreads();
  constexpr int W = sizeof(V) / sizeof(T);                  // reals per element: 2 for (re, im) pairs
  const int64_t o = S.off * (cplx ? 2 : 1) / W, n = (int64_t)S.K * S.B * (cplx ? 2 : 1) / W;
  const int nz = snz;
  V* Y = reinterpret_cast<V*>(out);
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += 2 * stride) {
    const int64_t i2 = i + stride;
    const bool two = i2 < n;
    double r0[W], r1[W];
#pragma unroll
    for (int w = 0; w < W; w++) { r0[w] = 0.0; r1[w] = 0.0; }
    int k = 0;
    for (; k + 4 <= nz; k += 4) {
      V v0[4], v1[4];
#pragma unroll
      for (int j = 0; j < 4; j++) { v0[j] = sp[k + j][o + i]; if (two) v1[j] = sp[k + j][o + i2]; }
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const double c = sc[k + j];
        const T* a = reinterpret_cast<const T*>(&v0[j]);
        const T* b = reinterpret_cast<const T*>(&v1[j]);
#pragma unroll
        for (int w = 0; w < W; w++) { r0[w] += c * (double)a[w]; if (two) r1[w] += c * (double)b[w]; }
      }
    }
    for (; k < nz; k++) {
      const double c = sc[k];
      const V v0 = sp[k][o + i];
      const T* a = reinterpret_cast<const T*>(&v0);
#pragma unroll
      for (int w = 0; w < W; w++) r0[w] += c * (double)a[w];
      if (two) {
        const V v1 = sp[k][o + i2];
        const T* b = reinterpret_cast<const T*>(&v1);
#pragma unroll
        for (int w = 0; w < W; w++) r1[w] += c * (double)b[w];
      }
    }
    V y0, y1;
    T* p0 = reinterpret_cast<T*>(&y0);
    T* p1 = reinterpret_cast<T*>(&y1);
#pragma unroll
    for (int w = 0; w < W; w++) { p0[w] = (T)r0[w]; p1[w] = (T)r1[w]; }
    Y[o + i] = y0;
    if (two) Y[o + i2] = y1;
  }
}

// out = sum_i coef[f * nt + i] v_i for complex float64 arithmetic over terms of two storage types: bit i of f32mask
// marks term i as complex64 (a float32 history vector), the others complex128; out is complex64 (VO = float2) or
// complex128. The block lists the fit's nonzero terms by storage type (the complex128 ones, then the complex64 ones,
// each in term order) and sums them in that order, so that no load waits behind a branch on its term's type: four
// terms' loads of four elements per thread are issued together. Blocks follow a block split (segmented.cuh) with
// 1024-element tiles (256 threads x 4 elements). out may be one of the terms: each thread reads its elements of
// every term before it writes them.
template <typename VO>
__global__ void __launch_bounds__(256) k_seg_lincomb_mixed(const blml_seg* segs, const int* split, int F, VO* out,
                                                           int nt, const double* coef, SegTerms t,
                                                           unsigned long long f32mask) {
  constexpr int EL = 4, TB = 4;
  __shared__ const void* sp[48];
  __shared__ double sc[48];
  __shared__ int sn[2];
  const int f = split[F + 1 + blockIdx.x];
  if (f < 0) return;
  const int lb = blockIdx.x - split[f], nb = split[f + 1] - split[f];
  const blml_seg S = segs[f];
  const double* cf = coef + (int64_t)f * nt;
  if (threadIdx.x == 0) {
    int c = 0;
    for (int pass = 0; pass < 2; pass++) {
      for (int q = 0; q < nt; q++) {
        const double v = cf[q];
        if (v != 0.0 && (int)((f32mask >> q) & 1ull) == pass) { sp[c] = t.v[q]; sc[c] = v; c++; }
      }
      sn[pass] = c;
    }
  }
  __syncthreads();
  const int64_t o = S.off, n = (int64_t)S.K * S.B;
  const int n64 = sn[0], nz = sn[1];
  constexpr int64_t T = 256 * EL;
  const int64_t stride = (int64_t)nb * T;
  for (int64_t t0 = (int64_t)lb * T; t0 < n; t0 += stride) {
    int64_t j[EL];
    bool ok[EL];
#pragma unroll
    for (int e = 0; e < EL; e++) {
      const int64_t i = t0 + 256 * e + threadIdx.x;
      ok[e] = i < n; j[e] = o + (ok[e] ? i : 0);
    }
    double rx[EL], ry[EL];
#pragma unroll
    for (int e = 0; e < EL; e++) { rx[e] = 0.0; ry[e] = 0.0; }
    int k = 0;
    for (; k < n64; k++) {
      const double2* p = reinterpret_cast<const double2*>(sp[k]);
      const double c = sc[k];
      double2 v[EL];
#pragma unroll
      for (int e = 0; e < EL; e++) v[e] = __ldg(p + j[e]);
#pragma unroll
      for (int e = 0; e < EL; e++) { rx[e] += c * v[e].x; ry[e] += c * v[e].y; }
    }
    for (; k + TB <= nz; k += TB) {
      float2 v[TB][EL];
#pragma unroll
      for (int q = 0; q < TB; q++) {
        const float2* p = reinterpret_cast<const float2*>(sp[k + q]);
#pragma unroll
        for (int e = 0; e < EL; e++) v[q][e] = __ldg(p + j[e]);
      }
#pragma unroll
      for (int q = 0; q < TB; q++) {
        const double c = sc[k + q];
#pragma unroll
        for (int e = 0; e < EL; e++) { rx[e] += c * (double)v[q][e].x; ry[e] += c * (double)v[q][e].y; }
      }
    }
    for (; k < nz; k++) {
      const float2* p = reinterpret_cast<const float2*>(sp[k]);
      const double c = sc[k];
      float2 v[EL];
#pragma unroll
      for (int e = 0; e < EL; e++) v[e] = __ldg(p + j[e]);
#pragma unroll
      for (int e = 0; e < EL; e++) { rx[e] += c * (double)v[e].x; ry[e] += c * (double)v[e].y; }
    }
#pragma unroll
    for (int e = 0; e < EL; e++)
      if (ok[e]) {
        VO y;
        y.x = rx[e]; y.y = ry[e];
        out[j[e]] = y;
      }
  }
}

template <typename T, bool CPLX>
__global__ void k_seg_lgrad_weights(const blml_seg* segs, const void* U, const T* w, const double* vs, void* V,
                                    double* part) {
  const blml_seg S = segs[blockIdx.y];
  const double vsc = vs[blockIdx.y];
  double v[1] = {0.0};
  SEG_LOOP(b, S) {
    double F = 0.0;
    for (int k = 0; k < S.K; k++) {
      double ur, ui; SAcc<T, CPLX>::get(U, S.off + (int64_t)k * S.B + b, ur, ui); F += ur * ur + ui * ui;
    }
    const double wb = (double)w[S.boff + b];
    const bool occ = wb > 0;
    if (occ) v[0] += wb * log(F);
    const double f = occ ? vsc * wb / F : 0.0;
    for (int k = 0; k < S.K; k++) {
      const int64_t i = S.off + (int64_t)k * S.B + b;
      double ur, ui; SAcc<T, CPLX>::get(U, i, ur, ui);
      SAcc<T, CPLX>::put(V, i, occ ? ur * f : 0.0, occ ? ui * f : 0.0);
    }
  }
  seg_partials<1>(v, part);
}

template <typename T, bool CPLX>
__global__ void k_seg_lgrad_finish(const blml_seg* segs, const void* SV, const void* U, const T* w, const double* nq,
                                   void* g) {
  const blml_seg S = segs[blockIdx.y];
  const double q = nq[blockIdx.y];
  SEG_LOOP(b, S) {
    const bool occ = (double)w[S.boff + b] > 0;
    for (int k = 0; k < S.K; k++) {
      const int64_t i = S.off + (int64_t)k * S.B + b;
      double sr, si, ur, ui;
      SAcc<T, CPLX>::get(SV, i, sr, si); SAcc<T, CPLX>::get(U, i, ur, ui);
      SAcc<T, CPLX>::put(g, i, occ ? 2.0 * (sr - q * ur) : 0.0, occ ? 2.0 * (si - q * ui) : 0.0);
    }
  }
}

// the Armijo search of every fit in one pass: for t_j = 2^-j, j < NT, sum_occ w log F(U + t_j S q); and the three
// inner products <q, U>, <E, S q>, <q, S q> from which Q(t) = Q + t (<q, U> + <E, S q>) + t^2 <q, S q>
constexpr int NT = 40;
template <typename T, bool CPLX>
__global__ void __launch_bounds__(256) k_seg_trials(const blml_seg* segs, const void* E, const void* q, const void* U,
                                                    const void* Sq, const T* w, double* part) {
  const blml_seg S = segs[blockIdx.y];
  double v[NT + 3];
#pragma unroll
  for (int j = 0; j < NT + 3; j++) v[j] = 0.0;
  SEG_LOOP(b, S) {
    const double wb = (double)w[S.boff + b];
    double a = 0.0, bb = 0.0, cc = 0.0;        // F(t) = a + 2 t b + t^2 c
    for (int k = 0; k < S.K; k++) {
      const int64_t i = S.off + (int64_t)k * S.B + b;
      double er, ei, qr, qi, ur, ui, sr, si;
      SAcc<T, CPLX>::get(E, i, er, ei); SAcc<T, CPLX>::get(q, i, qr, qi);
      SAcc<T, CPLX>::get(U, i, ur, ui); SAcc<T, CPLX>::get(Sq, i, sr, si);
      a += ur * ur + ui * ui; bb += ur * sr + ui * si; cc += sr * sr + si * si;
      v[NT] += qr * ur + qi * ui; v[NT + 1] += er * sr + ei * si; v[NT + 2] += qr * sr + qi * si;
    }
    if (wb > 0) {
      double t = 1.0;
#pragma unroll
      for (int j = 0; j < NT; j++) { v[j] += wb * log(a + t * (2.0 * bb + t * cc)); t *= 0.5; }
    }
  }
  seg_partials<NT + 3>(v, part);
}

// the accepted step of every fit: E += t_f q, U += t_f S q (t_f = 0 leaves a fit unchanged)
template <typename T, bool CPLX>
__global__ void k_seg_axpy2(const blml_seg* segs, void* E, const void* q, void* U, const void* Sq, const double* t) {
  const blml_seg S = segs[blockIdx.y];
  const double tf = t[blockIdx.y];
  if (tf == 0.0) return;
  SEG_LOOP(b, S) {
    for (int k = 0; k < S.K; k++) {
      const int64_t i = S.off + (int64_t)k * S.B + b;
      double er, ei, qr, qi, ur, ui, sr, si;
      SAcc<T, CPLX>::get(E, i, er, ei); SAcc<T, CPLX>::get(q, i, qr, qi);
      SAcc<T, CPLX>::get(U, i, ur, ui); SAcc<T, CPLX>::get(Sq, i, sr, si);
      SAcc<T, CPLX>::put(E, i, er + tf * qr, ei + tf * qi); SAcc<T, CPLX>::put(U, i, ur + tf * sr, ui + tf * si);
    }
  }
}

template <typename T, bool CPLX>
__global__ void k_seg_finish_fit(const blml_seg* segs, const void* U, const T* w, const double* inv_n2, T* dens,
                                 double* part) {
  const blml_seg S = segs[blockIdx.y];
  const double s = inv_n2[blockIdx.y];
  double v[1] = {0.0};
  SEG_LOOP(b, S) {
    double F = 0.0;
    for (int k = 0; k < S.K; k++) {
      double ur, ui; SAcc<T, CPLX>::get(U, S.off + (int64_t)k * S.B + b, ur, ui); F += ur * ur + ui * ui;
    }
    const T dv = (T)(F * s);
    dens[S.boff + b] = dv;
    const double wb = (double)w[S.boff + b];
    if (wb > 0) v[0] += wb * log((double)dv);
  }
  seg_partials<1>(v, part);
}

// held-out score per fit: [sum_{m > 0} m log max(F inv_z + eps, 1e-300), sum m]
template <typename T, bool CPLX>
__global__ void k_seg_log_score(const blml_seg* segs, const void* U, const T* m, const double* inv_z, double eps,
                                double* part) {
  const blml_seg S = segs[blockIdx.y];
  const double iz = inv_z[blockIdx.y];
  double v[2] = {0.0, 0.0};
  SEG_LOOP(b, S) {
    const double mb = (double)m[S.boff + b];
    if (!(mb > 0)) continue;
    double F = 0.0;
    for (int k = 0; k < S.K; k++) {
      double ur, ui; SAcc<T, CPLX>::get(U, S.off + (int64_t)k * S.B + b, ur, ui); F += ur * ur + ui * ui;
    }
    v[0] += mb * log(fmax(F * iz + eps, 1e-300)); v[1] += mb;
  }
  seg_partials<2>(v, part);
}

// the cut-off search's validation score per fit (selector.py:712-716): with f the fitted density on every bin of the
// lattice and p = max(f, 1e-300), the three sums sum_b p, sum_b va log p and sum_b va; the score is
// (sum va log p - sum va log sum p) / sum va, the mean log-probability of the validation counts
template <typename T>
__global__ void k_seg_val_score(const blml_seg* segs, const T* dens, const T* va, double* part) {
  const blml_seg S = segs[blockIdx.y];
  double v[3] = {0.0, 0.0, 0.0};
  SEG_LOOP(b, S) {
    const double p = fmax((double)dens[S.boff + b], 1e-300);
    const double a = (double)va[S.boff + b];
    v[0] += p;
    if (a > 0) { v[1] += a * log(p); v[2] += a; }
  }
  seg_partials<3>(v, part);
}

// start noise of every fit (the phases of mode 0; complex fits of one mode): E[0] *= exp(i pn z), z per fit at boff
template <typename T>
__global__ void k_seg_phases(const blml_seg* segs, double pn, const double* z, void* E) {
  const blml_seg S = segs[blockIdx.y];
  SEG_LOOP(b, S) {
    double er, ei; SAcc<T, true>::get(E, S.off + b, er, ei);
    double sn, cs; sincos(pn * z[S.boff + b], &sn, &cs);
    SAcc<T, true>::put(E, S.off + b, er * cs - ei * sn, er * sn + ei * cs);
  }
}

template <typename T>
__global__ void k_seg_real_to_complex(const blml_seg* real_segs, const blml_seg* cplx_segs, const T* er, void* E) {
  const blml_seg S = real_segs[blockIdx.y], C = cplx_segs[blockIdx.y];
  SEG_LOOP(b, S) SAcc<T, true>::put(E, C.off + b, (double)er[S.off + b], 0.0);
}

// the certificate's diagonal scaling of every fit: dh[boff + b] = sqrt(sum_k |E_kb|^2 / w_b) on occupied bins, 0 elsewhere
template <typename T>
__global__ void k_seg_cert_weights(const blml_seg* segs, const void* E, const T* w, double* dh) {
  const blml_seg S = segs[blockIdx.y];
  SEG_LOOP(b, S) {
    const double wb = (double)w[S.boff + b];
    double s = 0.0;
    for (int k = 0; k < S.K; k++) {
      double er, ei; SAcc<T, true>::get(E, S.off + (int64_t)k * S.B + b, er, ei); s += er * er + ei * ei;
    }
    dh[S.boff + b] = wb > 0 ? sqrt(s / wb) : 0.0;
  }
}

// one more mode per fit: the K modes of E (old layout) copied to the first K of the new layout (K + 1 modes), the new
// one set to scale_f dh v (real direction v per bin, the certificate's top Ritz vector in scaled coordinates)
template <typename T>
__global__ void k_seg_append_mode(const blml_seg* old_segs, const blml_seg* new_segs, const void* E, const double* dh,
                                  const double* v, const double* scale, void* En) {
  const blml_seg S = old_segs[blockIdx.y], N = new_segs[blockIdx.y];
  const double sc = scale[blockIdx.y];
  SEG_LOOP(b, S) {
    for (int k = 0; k < S.K; k++) {
      double er, ei; SAcc<T, true>::get(E, S.off + (int64_t)k * S.B + b, er, ei);
      SAcc<T, true>::put(En, N.off + (int64_t)k * N.B + b, er, ei);
    }
    SAcc<T, true>::put(En, N.off + (int64_t)S.K * N.B + b, sc * dh[S.boff + b] * v[S.boff + b], 0.0);
  }
}

static int seg_finish(const double* part, int F, int nq, unsigned maxmask, double* out, cudaStream_t st) {
  k_seg_finish<<<F, 256, 0, st>>>(part, nq, seg_blocks_for(F), maxmask, out);
  BLML_CHECK_LAUNCH("seg finish");
  return BLML_OK;
}

template <typename T>
static void seg_dots_launch(dim3 g, const blml_seg* s, int cplx, int np, const SegPairs& pp, double* part,
                            cudaStream_t st) {
  if (np <= 1) k_seg_dots<T, 1><<<g, 256, 0, st>>>(s, cplx, np, pp, part);
  else if (np <= 2) k_seg_dots<T, 2><<<g, 256, 0, st>>>(s, cplx, np, pp, part);
  else if (np <= 4) k_seg_dots<T, 4><<<g, 256, 0, st>>>(s, cplx, np, pp, part);
  else if (np <= 8) k_seg_dots<T, 8><<<g, 256, 0, st>>>(s, cplx, np, pp, part);
  else if (np <= 16) k_seg_dots<T, 16><<<g, 256, 0, st>>>(s, cplx, np, pp, part);
  else if (np <= 24) k_seg_dots<T, 24><<<g, 256, 0, st>>>(s, cplx, np, pp, part);
  else k_seg_dots<T, 48><<<g, 256, 0, st>>>(s, cplx, np, pp, part);
}

// Lanczos steps of the batched certificate without a host round trip: the reorthogonalisation w -= V c takes its
// coefficients [1, -c] straight from the inner products on the device (and keeps alpha, the one against the newest
// basis vector); the next basis vector is w / beta with beta = |w|, 0 when w vanishes. d holds n rows of np values.
__global__ void k_lz_coef(int n, int np, const double* __restrict__ d, double* __restrict__ coef,
                          double* __restrict__ alpha, int acol) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    coef[(int64_t)r * (np + 1)] = 1.0;
    for (int q = 0; q < np; q++) coef[(int64_t)r * (np + 1) + 1 + q] = -d[(int64_t)r * np + q];
    if (alpha && acol >= 0) alpha[r] = d[(int64_t)r * np + acol];
  }
}

__global__ void k_lz_beta(int n, const double* __restrict__ d, double* __restrict__ beta, double* __restrict__ coef) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    const double b = sqrt(fmax(d[r], 0.0));
    beta[r] = b;
    coef[r] = b > 0.0 ? 1.0 / b : 0.0;
  }
}

}  // namespace blml

using namespace blml;
#define SST reinterpret_cast<cudaStream_t>(stream)
namespace blml {
// the L-BFGS runner's history with float32 storage (internal to the library): the scan over complex64 stored vectors
// and a complex64 first shared vector, and linear combinations over complex128 / complex64 terms
int seg_split(int F, const blml_seg* segs, int* split, cudaStream_t st) {
  k_seg_split<<<1, 1024, 0, st>>>(F, segs, SEG_SPLIT_BLOCKS, split);
  BLML_CHECK_LAUNCH("segment block split");
  return BLML_OK;
}

int seg_dots2_h32(int F, const blml_seg* segs, const int* split, int np, const void* const* a, const void* b0,
                  const void* b1, const void* x, double* part, double* out, cudaStream_t st) {
  if (np < 1 || np > 20 || !a || !b0 || !b1) { set_error("history scan: 1..20 vectors, b0 and b1"); return BLML_ERR_ARG; }
  SegList al;
  for (int q = 0; q < 20; q++) al.a[q] = q < np ? a[q] : nullptr;
  const int W = SEG_SPLIT_BLOCKS + F;
  k_seg_dots2_h32<<<W, 256, 0, st>>>(segs, split, F, np, al, (const float2*)b0, (const double2*)b1,
                                     (const double2*)x, part);
  BLML_CHECK_LAUNCH("history scan (float32 history)");
  k_seg_finish_dots2_split<<<F, 256, 0, st>>>(part, W, split, np, out);
  BLML_CHECK_LAUNCH("history scan finish");
  return BLML_OK;
}

int seg_lincomb_mixed(int F, const blml_seg* segs, const int* split, void* out, int out_f32, int nterms,
                      const double* coef, const void* const* v, unsigned long long f32mask, cudaStream_t st) {
  if (nterms < 1 || nterms > 48) { set_error("linear combination: 1..48 terms"); return BLML_ERR_ARG; }
  SegTerms t;
  for (int q = 0; q < 48; q++) t.v[q] = q < nterms ? v[q] : nullptr;
  const unsigned W = (unsigned)(SEG_SPLIT_BLOCKS + F);
  if (out_f32) k_seg_lincomb_mixed<float2><<<W, 256, 0, st>>>(segs, split, F, (float2*)out, nterms, coef, t, f32mask);
  else k_seg_lincomb_mixed<double2><<<W, 256, 0, st>>>(segs, split, F, (double2*)out, nterms, coef, t, f32mask);
  BLML_CHECK_LAUNCH("linear combination (mixed storage)");
  return BLML_OK;
}
}  // namespace blml

#define SGRID(F) dim3((unsigned)seg_blocks_for(F), (unsigned)(F))
#define TYPED(dtype, cplx, K, ...)                                          \
  do {                                                                      \
    if (dtype == BLML_F64) { if (cplx) K<double, true>__VA_ARGS__; else K<double, false>__VA_ARGS__; } \
    else { if (cplx) K<float, true>__VA_ARGS__; else K<float, false>__VA_ARGS__; }                   \
  } while (0)

static int seg_args(int dtype, int F, const blml_seg* segs, const char* who) {
  if ((dtype != BLML_F64 && dtype != BLML_F32) || F < 1 || F > 65535 || !segs) {
    set_error("%s: dtype, 1 <= F <= 65535 fits and a segment table", who); return BLML_ERR_ARG;
  }
  return BLML_OK;
}

extern "C" {

int blml_seg_blocks(void) { return SEG_BLOCKS_MAX; }

int blml_seg_start_root(int dtype, int F, const blml_seg* segs, const void* c, const void* sg, const double* s0,
                        void* e0, void* stream) {
  if (seg_args(dtype, F, segs, "blml_seg_start_root")) return BLML_ERR_ARG;
  if (dtype == BLML_F64) k_seg_start_root<double><<<SGRID(F), 256, 0, SST>>>(segs, (const double*)c, (const double*)sg, s0, (double*)e0);
  else k_seg_start_root<float><<<SGRID(F), 256, 0, SST>>>(segs, (const float*)c, (const float*)sg, s0, (float*)e0);
  BLML_CHECK_LAUNCH("blml_seg_start_root");
  return BLML_OK;
}

int blml_seg_update_real1(int dtype, int F, const blml_seg* segs, const void* E, const void* U, const void* c,
                          const void* sg, const double* s0, void* out, void* stream) {
  if (seg_args(dtype, F, segs, "blml_seg_update_real1")) return BLML_ERR_ARG;
  if (dtype == BLML_F64)
    k_seg_update_real1<double><<<SGRID(F), 256, 0, SST>>>(segs, (const double*)E, (const double*)U, (const double*)c,
                                                          (const double*)sg, s0, (double*)out);
  else
    k_seg_update_real1<float><<<SGRID(F), 256, 0, SST>>>(segs, (const float*)E, (const float*)U, (const float*)c,
                                                         (const float*)sg, s0, (float*)out);
  BLML_CHECK_LAUNCH("blml_seg_update_real1");
  return BLML_OK;
}

int blml_seg_merit(int dtype, int F, const blml_seg* segs, int cplx, int psd, const void* E, const void* U,
                   const void* c, const void* sg, double* part, double* out, void* stream) {
  if (seg_args(dtype, F, segs, "blml_seg_merit")) return BLML_ERR_ARG;
  if (dtype == BLML_F64) {
    if (cplx) k_seg_merit<double, true><<<SGRID(F), 256, 0, SST>>>(segs, psd, E, U, (const double*)c, (const double*)sg, part);
    else k_seg_merit<double, false><<<SGRID(F), 256, 0, SST>>>(segs, psd, E, U, (const double*)c, (const double*)sg, part);
  } else {
    if (cplx) k_seg_merit<float, true><<<SGRID(F), 256, 0, SST>>>(segs, psd, E, U, (const float*)c, (const float*)sg, part);
    else k_seg_merit<float, false><<<SGRID(F), 256, 0, SST>>>(segs, psd, E, U, (const float*)c, (const float*)sg, part);
  }
  BLML_CHECK_LAUNCH("blml_seg_merit");
  return seg_finish(part, F, 3, 0u, out, SST);
}

int blml_seg_resid(int dtype, int F, const blml_seg* segs, int cplx, const void* E, const void* U, const void* c,
                   const double* scale, double* part, double* out, void* stream) {
  if (seg_args(dtype, F, segs, "blml_seg_resid")) return BLML_ERR_ARG;
  if (dtype == BLML_F64) {
    if (cplx) k_seg_resid<double, true><<<SGRID(F), 256, 0, SST>>>(segs, E, U, (const double*)c, scale, part);
    else k_seg_resid<double, false><<<SGRID(F), 256, 0, SST>>>(segs, E, U, (const double*)c, scale, part);
  } else {
    if (cplx) k_seg_resid<float, true><<<SGRID(F), 256, 0, SST>>>(segs, E, U, (const float*)c, scale, part);
    else k_seg_resid<float, false><<<SGRID(F), 256, 0, SST>>>(segs, E, U, (const float*)c, scale, part);
  }
  BLML_CHECK_LAUNCH("blml_seg_resid");
  return seg_finish(part, F, 2, 1u, out, SST);
}

int blml_seg_dots(int dtype, int F, const blml_seg* segs, int cplx, int npairs, const void* const* a,
                  const void* const* b, double* part, double* out, void* stream) {
  if (seg_args(dtype, F, segs, "blml_seg_dots")) return BLML_ERR_ARG;
  if (npairs < 1 || npairs > 48) { set_error("blml_seg_dots: 1..48 pairs"); return BLML_ERR_ARG; }
  // one pass (at most 48 accumulators per thread); out[f * npairs + q]
  SegPairs pp;
  for (int q = 0; q < 48; q++) { pp.a[q] = q < npairs ? a[q] : nullptr; pp.b[q] = q < npairs ? b[q] : nullptr; }
  if (dtype == BLML_F64) seg_dots_launch<double>(SGRID(F), segs, cplx, npairs, pp, part, SST);
  else seg_dots_launch<float>(SGRID(F), segs, cplx, npairs, pp, part, SST);
  BLML_CHECK_LAUNCH("blml_seg_dots");
  k_seg_finish_strided<<<F, 256, 0, SST>>>(part, npairs, seg_blocks_for(F), out, npairs);
  BLML_CHECK_LAUNCH("blml_seg_dots finish");
  return BLML_OK;
}

int blml_seg_dots2(int dtype, int F, const blml_seg* segs, int cplx, int np, const void* const* a, const void* b0,
                   const void* b1, const void* x, double* part, double* out, void* stream) {
  if (seg_args(dtype, F, segs, "blml_seg_dots2")) return BLML_ERR_ARG;
  if (np < 1 || np > 20 || !a || !b0 || !b1) { set_error("blml_seg_dots2: 1..20 vectors, b0 and b1"); return BLML_ERR_ARG; }
  SegList al;
  for (int q = 0; q < 20; q++) al.a[q] = q < np ? a[q] : nullptr;
  if (dtype == BLML_F64 && cplx)
    k_seg_dots2_c128<double2, double2><<<SGRID(F), 256, 0, SST>>>(segs, np, al, b0, b1, x, part);
  else if (dtype == BLML_F64) k_seg_dots2<double><<<SGRID(F), 256, 0, SST>>>(segs, cplx, np, al, b0, b1, x, part);
  else k_seg_dots2<float><<<SGRID(F), 256, 0, SST>>>(segs, cplx, np, al, b0, b1, x, part);
  BLML_CHECK_LAUNCH("blml_seg_dots2");
  k_seg_finish_dots2<<<F, 256, 0, SST>>>(part, np, seg_blocks_for(F), out);
  BLML_CHECK_LAUNCH("blml_seg_dots2 finish");
  return BLML_OK;
}

int blml_seg_lincomb(int dtype, int F, const blml_seg* segs, int cplx, void* out, int nterms, const double* coef,
                     const void* const* v, void* stream) {
  if (seg_args(dtype, F, segs, "blml_seg_lincomb")) return BLML_ERR_ARG;
  if (nterms < 1 || nterms > 48) { set_error("blml_seg_lincomb: 1..48 terms"); return BLML_ERR_ARG; }
  SegTerms t;
  for (int q = 0; q < 48; q++) t.v[q] = q < nterms ? v[q] : nullptr;
  if (dtype == BLML_F64 && cplx)
    k_seg_lincomb<double, double2><<<SGRID(F), 256, 0, SST>>>(segs, cplx, (double*)out, nterms, coef, t);
  else if (dtype == BLML_F64)
    k_seg_lincomb<double, double><<<SGRID(F), 256, 0, SST>>>(segs, cplx, (double*)out, nterms, coef, t);
  else if (cplx)
    k_seg_lincomb<float, float2><<<SGRID(F), 256, 0, SST>>>(segs, cplx, (float*)out, nterms, coef, t);
  else k_seg_lincomb<float, float><<<SGRID(F), 256, 0, SST>>>(segs, cplx, (float*)out, nterms, coef, t);
  BLML_CHECK_LAUNCH("blml_seg_lincomb");
  return BLML_OK;
}

int blml_seg_lgrad_weights(int dtype, int F, const blml_seg* segs, int cplx, const void* U, const void* w,
                           const double* vscale, void* V, double* part, double* out, void* stream) {
  if (seg_args(dtype, F, segs, "blml_seg_lgrad_weights")) return BLML_ERR_ARG;
  if (dtype == BLML_F64) {
    if (cplx) k_seg_lgrad_weights<double, true><<<SGRID(F), 256, 0, SST>>>(segs, U, (const double*)w, vscale, V, part);
    else k_seg_lgrad_weights<double, false><<<SGRID(F), 256, 0, SST>>>(segs, U, (const double*)w, vscale, V, part);
  } else {
    if (cplx) k_seg_lgrad_weights<float, true><<<SGRID(F), 256, 0, SST>>>(segs, U, (const float*)w, vscale, V, part);
    else k_seg_lgrad_weights<float, false><<<SGRID(F), 256, 0, SST>>>(segs, U, (const float*)w, vscale, V, part);
  }
  BLML_CHECK_LAUNCH("blml_seg_lgrad_weights");
  return seg_finish(part, F, 1, 0u, out, SST);
}

int blml_seg_lgrad_finish(int dtype, int F, const blml_seg* segs, int cplx, const void* SV, const void* U,
                          const void* w, const double* nq, void* g, void* stream) {
  if (seg_args(dtype, F, segs, "blml_seg_lgrad_finish")) return BLML_ERR_ARG;
  if (dtype == BLML_F64) {
    if (cplx) k_seg_lgrad_finish<double, true><<<SGRID(F), 256, 0, SST>>>(segs, SV, U, (const double*)w, nq, g);
    else k_seg_lgrad_finish<double, false><<<SGRID(F), 256, 0, SST>>>(segs, SV, U, (const double*)w, nq, g);
  } else {
    if (cplx) k_seg_lgrad_finish<float, true><<<SGRID(F), 256, 0, SST>>>(segs, SV, U, (const float*)w, nq, g);
    else k_seg_lgrad_finish<float, false><<<SGRID(F), 256, 0, SST>>>(segs, SV, U, (const float*)w, nq, g);
  }
  BLML_CHECK_LAUNCH("blml_seg_lgrad_finish");
  return BLML_OK;
}

int blml_seg_trials(int dtype, int F, const blml_seg* segs, int cplx, const void* E, const void* q, const void* U,
                    const void* Sq, const void* w, double* part, double* out, void* stream) {
  if (seg_args(dtype, F, segs, "blml_seg_trials")) return BLML_ERR_ARG;
  if (dtype == BLML_F64) {
    if (cplx) k_seg_trials<double, true><<<SGRID(F), 256, 0, SST>>>(segs, E, q, U, Sq, (const double*)w, part);
    else k_seg_trials<double, false><<<SGRID(F), 256, 0, SST>>>(segs, E, q, U, Sq, (const double*)w, part);
  } else {
    if (cplx) k_seg_trials<float, true><<<SGRID(F), 256, 0, SST>>>(segs, E, q, U, Sq, (const float*)w, part);
    else k_seg_trials<float, false><<<SGRID(F), 256, 0, SST>>>(segs, E, q, U, Sq, (const float*)w, part);
  }
  BLML_CHECK_LAUNCH("blml_seg_trials");
  return seg_finish(part, F, NT + 3, 0u, out, SST);
}

int blml_seg_axpy2(int dtype, int F, const blml_seg* segs, int cplx, void* E, const void* q, void* U, const void* Sq,
                   const double* t, void* stream) {
  if (seg_args(dtype, F, segs, "blml_seg_axpy2")) return BLML_ERR_ARG;
  TYPED(dtype, cplx, k_seg_axpy2, <<<SGRID(F), 256, 0, SST>>>(segs, E, q, U, Sq, t));
  BLML_CHECK_LAUNCH("blml_seg_axpy2");
  return BLML_OK;
}

int blml_seg_finish(int dtype, int F, const blml_seg* segs, int cplx, const void* U, const void* w,
                    const double* inv_n2, void* density, double* part, double* out, void* stream) {
  if (seg_args(dtype, F, segs, "blml_seg_finish")) return BLML_ERR_ARG;
  if (dtype == BLML_F64) {
    if (cplx) k_seg_finish_fit<double, true><<<SGRID(F), 256, 0, SST>>>(segs, U, (const double*)w, inv_n2, (double*)density, part);
    else k_seg_finish_fit<double, false><<<SGRID(F), 256, 0, SST>>>(segs, U, (const double*)w, inv_n2, (double*)density, part);
  } else {
    if (cplx) k_seg_finish_fit<float, true><<<SGRID(F), 256, 0, SST>>>(segs, U, (const float*)w, inv_n2, (float*)density, part);
    else k_seg_finish_fit<float, false><<<SGRID(F), 256, 0, SST>>>(segs, U, (const float*)w, inv_n2, (float*)density, part);
  }
  BLML_CHECK_LAUNCH("blml_seg_finish");
  return seg_finish(part, F, 1, 0u, out, SST);
}

int blml_seg_log_score(int dtype, int F, const blml_seg* segs, int cplx, const void* U, const void* m,
                       const double* inv_z, double eps, double* part, double* out, void* stream) {
  if (seg_args(dtype, F, segs, "blml_seg_log_score")) return BLML_ERR_ARG;
  if (dtype == BLML_F64) {
    if (cplx) k_seg_log_score<double, true><<<SGRID(F), 256, 0, SST>>>(segs, U, (const double*)m, inv_z, eps, part);
    else k_seg_log_score<double, false><<<SGRID(F), 256, 0, SST>>>(segs, U, (const double*)m, inv_z, eps, part);
  } else {
    if (cplx) k_seg_log_score<float, true><<<SGRID(F), 256, 0, SST>>>(segs, U, (const float*)m, inv_z, eps, part);
    else k_seg_log_score<float, false><<<SGRID(F), 256, 0, SST>>>(segs, U, (const float*)m, inv_z, eps, part);
  }
  BLML_CHECK_LAUNCH("blml_seg_log_score");
  return seg_finish(part, F, 2, 0u, out, SST);
}

int blml_seg_val_score(int dtype, int F, const blml_seg* segs, const void* dens, const void* va, double* part,
                       double* out, void* stream) {
  if (seg_args(dtype, F, segs, "blml_seg_val_score") || !dens || !va || !part || !out) return BLML_ERR_ARG;
  if (dtype == BLML_F64)
    k_seg_val_score<double><<<SGRID(F), 256, 0, SST>>>(segs, (const double*)dens, (const double*)va, part);
  else k_seg_val_score<float><<<SGRID(F), 256, 0, SST>>>(segs, (const float*)dens, (const float*)va, part);
  BLML_CHECK_LAUNCH("blml_seg_val_score");
  return seg_finish(part, F, 3, 0u, out, SST);
}

int blml_seg_phases(int dtype, int F, const blml_seg* segs, double pn, const double* z, void* E, void* stream) {
  if (seg_args(dtype, F, segs, "blml_seg_phases")) return BLML_ERR_ARG;
  if (dtype == BLML_F64) k_seg_phases<double><<<SGRID(F), 256, 0, SST>>>(segs, pn, z, E);
  else k_seg_phases<float><<<SGRID(F), 256, 0, SST>>>(segs, pn, z, E);
  BLML_CHECK_LAUNCH("blml_seg_phases");
  return BLML_OK;
}

int blml_seg_real_to_complex(int dtype, int F, const blml_seg* real_segs, const blml_seg* cplx_segs, const void* er,
                             void* E, void* stream) {
  if (seg_args(dtype, F, real_segs, "blml_seg_real_to_complex") || !cplx_segs) return BLML_ERR_ARG;
  if (dtype == BLML_F64) k_seg_real_to_complex<double><<<SGRID(F), 256, 0, SST>>>(real_segs, cplx_segs, (const double*)er, E);
  else k_seg_real_to_complex<float><<<SGRID(F), 256, 0, SST>>>(real_segs, cplx_segs, (const float*)er, E);
  BLML_CHECK_LAUNCH("blml_seg_real_to_complex");
  return BLML_OK;
}

int blml_seg_cert_weights(int dtype, int F, const blml_seg* segs, const void* E, const void* w, double* dh,
                          void* stream) {
  if (seg_args(dtype, F, segs, "blml_seg_cert_weights") || !E || !w || !dh) return BLML_ERR_ARG;
  if (dtype == BLML_F64) k_seg_cert_weights<double><<<SGRID(F), 256, 0, SST>>>(segs, E, (const double*)w, dh);
  else k_seg_cert_weights<float><<<SGRID(F), 256, 0, SST>>>(segs, E, (const float*)w, dh);
  BLML_CHECK_LAUNCH("blml_seg_cert_weights");
  return BLML_OK;
}

int blml_seg_append_mode(int dtype, int F, const blml_seg* old_segs, const blml_seg* new_segs, const void* E,
                         const double* dh, const double* v, const double* scale, void* E_new, void* stream) {
  if (seg_args(dtype, F, old_segs, "blml_seg_append_mode") || !new_segs || !E || !dh || !v || !scale || !E_new)
    return BLML_ERR_ARG;
  if (dtype == BLML_F64) k_seg_append_mode<double><<<SGRID(F), 256, 0, SST>>>(old_segs, new_segs, E, dh, v, scale, E_new);
  else k_seg_append_mode<float><<<SGRID(F), 256, 0, SST>>>(old_segs, new_segs, E, dh, v, scale, E_new);
  BLML_CHECK_LAUNCH("blml_seg_append_mode");
  return BLML_OK;
}

int blml_lanczos_coef(int n, int np, const double* dots, double* coef, double* alpha, int alpha_col, void* stream) {
  if (n < 1 || np < 1 || np > 47 || !dots || !coef || alpha_col >= np) {
    set_error("blml_lanczos_coef: n >= 1 rows of 1..47 inner products"); return BLML_ERR_ARG;
  }
  k_lz_coef<<<(n + 127) / 128, 128, 0, SST>>>(n, np, dots, coef, alpha, alpha_col);
  BLML_CHECK_LAUNCH("blml_lanczos_coef");
  return BLML_OK;
}

int blml_lanczos_beta(int n, const double* dots, double* beta, double* coef, void* stream) {
  if (n < 1 || !dots || !beta || !coef) { set_error("blml_lanczos_beta: bad arguments"); return BLML_ERR_ARG; }
  k_lz_beta<<<(n + 127) / 128, 128, 0, SST>>>(n, dots, beta, coef);
  BLML_CHECK_LAUNCH("blml_lanczos_beta");
  return BLML_OK;
}

int blml_seg_dots2_h32(int F, const blml_seg* segs, int* split, int np, const void* const* a, const void* b0,
                       const void* b1, const void* x, double* part, double* out, void* stream) {
  if (F < 1 || F > 65535 || !segs || !split || !a || !part) {
    set_error("blml_seg_dots2_h32: bad arguments"); return BLML_ERR_ARG;
  }
  if (seg_split(F, segs, split, SST)) return BLML_ERR_CUDA;
  return seg_dots2_h32(F, segs, split, np, a, b0, b1, x, part, out, SST);
}

int64_t blml_seg_split_ints(int F) { return F < 1 ? 0 : seg_split_ints(F); }

int blml_seg_lincomb_h32(int F, const blml_seg* segs, int* split, void* out, int out_f32, int nterms,
                         const double* coef, const void* const* v, unsigned long long f32mask, void* stream) {
  if (F < 1 || F > 65535 || !segs || !split || !out || !coef || !v) {
    set_error("blml_seg_lincomb_h32: bad arguments"); return BLML_ERR_ARG;
  }
  if (seg_split(F, segs, split, SST)) return BLML_ERR_CUDA;
  return seg_lincomb_mixed(F, segs, split, out, out_f32, nterms, coef, v, f32mask, SST);
}

}  // extern "C"
