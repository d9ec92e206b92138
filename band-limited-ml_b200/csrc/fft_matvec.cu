// The FFT route of the mat-vec for kernels that are exact DFT masks on a circular 2-D lattice.
//
// A pball group, or dirichlet columns, on a lattice whose every axis is one period (the reference's circular pad,
// blml_binned.py:130-136) has plane waves at integer harmonics: nu = k / M on an M-point axis. Then
//     S e = sum_q W_q v_q v_q^H e
// is the unnormalised inverse 2-D DFT of W times the forward DFT of e, restricted to the band's harmonics: the
// reference's rfftn -> x Kf -> irfftn (blml_binned.py:156-168) with Kf zero outside the band. Three grouped stages
// run it over every fit of a batch, each a batch of 1-D FFTs in shared memory:
//   A  rows:    FFT of every lattice row (length M2), keep the H2 harmonics of axis 1 -> Z (nb, H2, M1)
//   B  columns: FFT of every Z column (length M1), times W over the band (zero elsewhere), inverse FFT -> Z
//   C  rows:    scatter each row's H2 harmonics into a zero spectrum, inverse FFT (length M2) -> the lattice row
// The FFTs are mixed-radix (2, 3, 4, 6, 8) Stockham passes: sides 2^a 3^b (the benchmark sweep's {64, ..., 384}).
// Each CTA holds two buffers of up to kCtaBytes / 2 (several rows or columns, one padded row per transform;
// a single transform when the side is longer) and the length's twiddle table; passes run out of place between them.
// Versus the restricted transforms (matvec.cu) this costs O(M log M) per row instead of O(M H), and in float64 it
// rounds like an FFT (~1e-16 log M relative), so the route changes no result beyond rounding.
#include <vector>
#include <algorithm>
#include <functional>
#include <cmath>
#include "plan.cuh"

namespace blml {

constexpr int kFT = 256;                 // threads per CTA
constexpr int kCtaBytesMax = 72 * 1024;  // the largest shared-memory budget a CTA may aim for (3 CTAs per SM)

// launch shape of the route, chosen by blml_fft_set_shape (the project's autotuner writes a table the package applies)
// and read when a plan's descriptor is made: the shared memory a CTA aims for (several transforms per CTA; one when
// longer) and the most columns a CTA of the column stage takes
static int g_cta_bytes = kCtaBytesMax;
static int g_max_cols = 2;
constexpr int kMaxSide = 4096;           // longest side of the route
constexpr int kMaxRad = 12;

// Shared-memory index of point i of a transform: one pad slot after every 8 points, so the first pass's stores at
// stride R (and the row gathers) spread over the banks; a transform occupies ld(N) slots, an odd count, so that
// transforms side by side start on different banks.
__host__ __device__ __forceinline__ int pidx(int i) { return i + (i >> 3); }

// one complex value global -> shared without a register round trip (cp.async: the loads of a stage's data are all
// in flight at once; cp.async.wait_all and a barrier before the first pass)
template <typename V>
__device__ __forceinline__ void cp_async_el(V* dst, const V* src) {
  static_assert(sizeof(V) == 16 || sizeof(V) == 8, "complex float64 or float32");
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
  if (sizeof(V) == 16) asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" :: "r"(d), "l"(src) : "memory");
  else asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" :: "r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }
__host__ __device__ __forceinline__ int pld(int N) { return N + (N >> 3) + 1; }

// x / d for 0 <= x < 2^16 and 1 <= d < 2^16 by a multiply and a shift: m = floor((2^32 - 1) / d) + 1 (0 for d = 1)
__host__ __device__ __forceinline__ unsigned magic_of(unsigned d) { return d <= 1 ? 0u : 0xFFFFFFFFu / d + 1u; }
__device__ __forceinline__ int div_m(int x, unsigned m) { return m ? (int)__umulhi((unsigned)x, m) : x; }

static int fft_smem_once();

// per-plan data of the route (host struct holding device pointers)
// The passes of one axis's transform: radix, sub-transform length Ns before the pass, the magic numbers of the
// divisions by N / R and by Ns, and where the pass's twiddles start in the axis's table. The table holds, pass after
// pass (Ns > 1), w^(r k N / (Ns R)) for k < Ns, 1 <= r < R at [k (R - 1) + r - 1], w = exp(-2 pi i / N): N - R_0
// values in all, read with consecutive k by consecutive threads.
struct FftAxis {
  int N, npass, ntw;
  int8_t rad[kMaxRad];
  int ns[kMaxRad], twoff[kMaxRad];
  unsigned mnbt[kMaxRad], mns[kMaxRad];
};

// per-plan data of the route (host struct holding device pointers)
struct FftPlan {
  int M1, M2, H1, H2;
  FftAxis ax1, ax2;                      // axis 0 (columns, length M1) and axis 1 (rows, length M2)
  void* tw1; void* tw2;                  // the axes' pass twiddle tables, complex of the plan's dtype
  int* k2;                               // the H2 harmonics of axis 1 as DFT indices (k mod M2)
  int* map1;                             // per DFT index of axis 0: its position in the band's axis-0 list, or -1
};

struct FftDesc {
  const void* X; void* Y; void* Z; const void* W;
  const void* tw1; const void* tw2; const int* k2; const int* map1;
  int M1, M2, H1, H2, nb, flags;         // flags: 1 real input, 4 real output
  int rows, cols;                        // transforms per CTA: rows (stages A, C), columns (stage B)
  int ctasA, ctasB;                      // CTAs of this problem in stages A / C and B
  FftAxis ax1, ax2;
};

// ------------------------------------------------------------------------------------------------- butterflies
// y_s = sum_r a_r exp(sign 2 pi i r s / R), sign = +1 for the inverse transform, -1 forward.
template <typename T, bool INV> __device__ __forceinline__ cpx<T> mul_i(cpx<T> a) {   // a * (sign i)
  return INV ? cpx<T>{-a.im, a.re} : cpx<T>{a.im, -a.re};
}
template <typename T> __device__ __forceinline__ cpx<T> cadd(cpx<T> a, cpx<T> b) { return {a.re + b.re, a.im + b.im}; }
template <typename T> __device__ __forceinline__ cpx<T> csub(cpx<T> a, cpx<T> b) { return {a.re - b.re, a.im - b.im}; }

template <typename T, bool INV> __device__ __forceinline__ void dft2(cpx<T>& a0, cpx<T>& a1) {
  const cpx<T> t = a0; a0 = cadd(t, a1); a1 = csub(t, a1);
}
template <typename T, bool INV> __device__ __forceinline__ void dft4(cpx<T>& a0, cpx<T>& a1, cpx<T>& a2, cpx<T>& a3) {
  const cpx<T> t0 = cadd(a0, a2), t1 = csub(a0, a2), t2 = cadd(a1, a3), t3 = mul_i<T, INV>(csub(a1, a3));
  a0 = cadd(t0, t2); a2 = csub(t0, t2); a1 = cadd(t1, t3); a3 = csub(t1, t3);
}
template <typename T, bool INV> __device__ __forceinline__ void dft3(cpx<T>& a0, cpx<T>& a1, cpx<T>& a2) {
  const T h = T(0.8660254037844386);      // sin(pi / 3)
  const cpx<T> t = cadd(a1, a2), u = csub(a1, a2);
  const cpx<T> m = {a0.re - T(0.5) * t.re, a0.im - T(0.5) * t.im};
  const cpx<T> v = mul_i<T, INV>(cpx<T>{h * u.re, h * u.im});
  a0 = cadd(a0, t); a1 = cadd(m, v); a2 = csub(m, v);
}
template <typename T, int R, bool INV> __device__ __forceinline__ void butterfly(cpx<T> (&a)[R]) {
  if constexpr (R == 2) {
    dft2<T, INV>(a[0], a[1]);
  } else if constexpr (R == 3) {
    dft3<T, INV>(a[0], a[1], a[2]);
  } else if constexpr (R == 4) {
    dft4<T, INV>(a[0], a[1], a[2], a[3]);
  } else if constexpr (R == 6) {            // evens and odds by DFT3, joined with exp(sign 2 pi i s / 6)
    cpx<T> e0 = a[0], e1 = a[2], e2 = a[4], o0 = a[1], o1 = a[3], o2 = a[5];
    dft3<T, INV>(e0, e1, e2); dft3<T, INV>(o0, o1, o2);
    const T h = T(0.8660254037844386);
    const cpx<T> w1 = {T(0.5), INV ? h : -h}, w2 = {T(-0.5), INV ? h : -h};
    const cpx<T> p1 = cmul(o1, w1), p2 = cmul(o2, w2);
    a[0] = cadd(e0, o0); a[3] = csub(e0, o0);
    a[1] = cadd(e1, p1); a[4] = csub(e1, p1);
    a[2] = cadd(e2, p2); a[5] = csub(e2, p2);
  } else {                                  // R == 8: evens and odds by DFT4, joined with exp(sign 2 pi i s / 8)
    cpx<T> e0 = a[0], e1 = a[2], e2 = a[4], e3 = a[6], o0 = a[1], o1 = a[3], o2 = a[5], o3 = a[7];
    dft4<T, INV>(e0, e1, e2, e3); dft4<T, INV>(o0, o1, o2, o3);
    const T c = T(0.7071067811865476);       // cos(pi / 4)
    const cpx<T> p1 = INV ? cpx<T>{c * (o1.re - o1.im), c * (o1.im + o1.re)}
                          : cpx<T>{c * (o1.re + o1.im), c * (o1.im - o1.re)};
    const cpx<T> p2 = mul_i<T, INV>(o2);
    const cpx<T> p3 = INV ? cpx<T>{c * (-o3.re - o3.im), c * (o3.re - o3.im)}
                          : cpx<T>{c * (-o3.re + o3.im), c * (-o3.re - o3.im)};
    a[0] = cadd(e0, o0); a[4] = csub(e0, o0);
    a[1] = cadd(e1, p1); a[5] = csub(e1, p1);
    a[2] = cadd(e2, p2); a[6] = csub(e2, p2);
    a[3] = cadd(e3, p3); a[7] = csub(e3, p3);
  }
}

// One Stockham pass of radix R over ntr transforms of length N, from src to dst in shared memory (transform t at
// + t * ld, point i at pidx(i), in both), after Ns points of each sub-transform are done: butterfly j (of N / R)
// reads src[j + r N / R] times w^(r (j mod Ns) N / (Ns R)) and writes its R outputs to dst[(j - j mod Ns) R +
// j mod Ns + s Ns]. A thread holds one butterfly's R values at a time; one barrier per pass.
template <typename T, int R, bool INV>
__device__ __forceinline__ void fft_pass(const cpx<T>* src, cpx<T>* dst, const cpx<T>* tw, int N, int ld, int ntr,
                                         int Ns, unsigned mnbt, unsigned mns) {
  const int nbt = N / R, total = nbt * ntr;
  for (int b = threadIdx.x; b < total; b += kFT) {
    const int t = div_m(b, mnbt), j = b - t * nbt;
    const int k = j - div_m(j, mns) * Ns;
    const cpx<T>* s = src + t * ld;
    cpx<T> v[R];
#pragma unroll
    for (int r = 0; r < R; r++) v[r] = s[pidx(j + r * nbt)];
    if (Ns > 1) {
      const cpx<T>* w = tw + k * (R - 1);
#pragma unroll
      for (int r = 1; r < R; r++) {
        cpx<T> ww = w[r - 1];
        if (INV) ww.im = -ww.im;
        v[r] = cmul(v[r], ww);
      }
    }
    butterfly<T, R, INV>(v);
    cpx<T>* d = dst + t * ld;
    const int o = (j - k) * R + k;
#pragma unroll
    for (int r = 0; r < R; r++) d[pidx(o + r * Ns)] = v[r];
  }
  __syncthreads();
}

// All passes of the transform, alternating between the two buffers; returns the one holding the result.
template <typename T, bool INV>
__device__ cpx<T>* smem_fft(cpx<T>* a, cpx<T>* b, const cpx<T>* tw, int ld, int ntr, const FftAxis& ax) {
  for (int p = 0; p < ax.npass; p++) {
    const cpx<T>* twp = tw + ax.twoff[p];
    const int N = ax.N, Ns = ax.ns[p];
    const unsigned m1 = ax.mnbt[p], m2 = ax.mns[p];
    switch (ax.rad[p]) {
      case 8: fft_pass<T, 8, INV>(a, b, twp, N, ld, ntr, Ns, m1, m2); break;
      case 6: fft_pass<T, 6, INV>(a, b, twp, N, ld, ntr, Ns, m1, m2); break;
      case 4: fft_pass<T, 4, INV>(a, b, twp, N, ld, ntr, Ns, m1, m2); break;
      case 3: fft_pass<T, 3, INV>(a, b, twp, N, ld, ntr, Ns, m1, m2); break;
      default: fft_pass<T, 2, INV>(a, b, twp, N, ld, ntr, Ns, m1, m2); break;
    }
    cpx<T>* t = a; a = b; b = t;
  }
  return a;
}

// ------------------------------------------------------------------------------------------------- stages
// Each stage is a device body over one problem's descriptor and one CTA index, behind two entry points: grouped
// (grid (max CTAs of a problem, 1, n); problem gi = subset[blockIdx.z] or blockIdx.z; problems with live[gi] == 0 and
// CTAs past the problem's own count return at once, uniformly per CTA) and single-plan (the descriptor by value).
// Dynamic shared memory: (2 x transforms x (length + 1) + length) complex values.
template <typename T>
__device__ __forceinline__ void rows_fwd_body(const FftDesc& D, int cta, unsigned char* smem) {
  const int tid = threadIdx.x;
  const int N = D.M2, ld = pld(N), rows_tot = D.nb * D.M1;
  const int r0 = cta * D.rows, nr = min(D.rows, rows_tot - r0);
  cpx<T>* buf = reinterpret_cast<cpx<T>*>(smem);
  cpx<T>* alt = buf + D.rows * ld;
  cpx<T>* tw = alt + D.rows * ld;
  for (int i = tid; i < D.ax2.ntw; i += kFT) cp_async_el(&tw[i], reinterpret_cast<const cpx<T>*>(D.tw2) + i);
  const int64_t base = (int64_t)r0 * N;
  if (D.flags & 1) {
    const T* X = reinterpret_cast<const T*>(D.X) + base;
    for (int i = tid; i < nr * N; i += kFT) { const int t = i / N; buf[t * ld + pidx(i - t * N)] = cpx<T>{X[i], T(0)}; }
  } else {
    const cpx<T>* X = reinterpret_cast<const cpx<T>*>(D.X) + base;
    for (int i = tid; i < nr * N; i += kFT) { const int t = i / N; cp_async_el(&buf[t * ld + pidx(i - t * N)], X + i); }
  }
  cp_async_wait_all();
  __syncthreads();
  buf = smem_fft<T, false>(buf, alt, tw, ld, nr, D.ax2);
  cpx<T>* Z = reinterpret_cast<cpx<T>*>(D.Z);
  for (int i = tid; i < nr * D.H2; i += kFT) {
    const int q2 = i / nr, t = i - q2 * nr;
    const int row = r0 + t, b = row / D.M1, r = row - b * D.M1;
    Z[((int64_t)b * D.H2 + q2) * D.M1 + r] = buf[t * ld + pidx(__ldg(D.k2 + q2))];
  }
}

template <typename T>
__device__ __forceinline__ void cols_body(const FftDesc& D, int cta, unsigned char* smem) {
  const int tid = threadIdx.x;
  const int N = D.M1, ld = pld(N), cols_tot = D.nb * D.H2;
  const int c0 = cta * D.cols, nc = min(D.cols, cols_tot - c0);
  cpx<T>* base = reinterpret_cast<cpx<T>*>(smem);
  cpx<T>* buf = base;
  cpx<T>* alt = base + D.cols * ld;
  cpx<T>* tw = alt + D.cols * ld;
  for (int i = tid; i < D.ax1.ntw; i += kFT) cp_async_el(&tw[i], reinterpret_cast<const cpx<T>*>(D.tw1) + i);
  cpx<T>* Z = reinterpret_cast<cpx<T>*>(D.Z) + (int64_t)c0 * N;
  for (int i = tid; i < nc * N; i += kFT) { const int t = i / N; cp_async_el(&buf[t * ld + pidx(i - t * N)], Z + i); }
  cp_async_wait_all();
  __syncthreads();
  buf = smem_fft<T, false>(buf, alt, tw, ld, nc, D.ax1);
  alt = buf == base ? base + D.cols * ld : base;
  const T* W = reinterpret_cast<const T*>(D.W);
  for (int i = tid; i < nc * N; i += kFT) {
    const int t = i / N, k1 = i - t * N;
    const int q1 = __ldg(D.map1 + k1), q2 = (c0 + t) % D.H2;
    const T w = q1 >= 0 ? W[(int64_t)q1 * D.H2 + q2] : T(0);
    cpx<T>& v = buf[t * ld + pidx(k1)];
    v.re *= w; v.im *= w;
  }
  __syncthreads();
  buf = smem_fft<T, true>(buf, alt, tw, ld, nc, D.ax1);
  for (int i = tid; i < nc * N; i += kFT) { const int t = i / N; Z[i] = buf[t * ld + pidx(i - t * N)]; }
}

template <typename T>
__device__ __forceinline__ void rows_inv_body(const FftDesc& D, int cta, unsigned char* smem) {
  const int tid = threadIdx.x;
  const int N = D.M2, ld = pld(N), rows_tot = D.nb * D.M1;
  const int r0 = cta * D.rows, nr = min(D.rows, rows_tot - r0);
  cpx<T>* buf = reinterpret_cast<cpx<T>*>(smem);
  cpx<T>* alt = buf + D.rows * ld;
  cpx<T>* tw = alt + D.rows * ld;
  for (int i = tid; i < D.ax2.ntw; i += kFT) cp_async_el(&tw[i], reinterpret_cast<const cpx<T>*>(D.tw2) + i);
  for (int i = tid; i < nr * ld; i += kFT) buf[i] = cpx<T>{T(0), T(0)};
  __syncthreads();
  const cpx<T>* Z = reinterpret_cast<const cpx<T>*>(D.Z);
  for (int i = tid; i < nr * D.H2; i += kFT) {
    const int q2 = i / nr, t = i - q2 * nr;
    const int row = r0 + t, b = row / D.M1, r = row - b * D.M1;
    cp_async_el(&buf[t * ld + pidx(__ldg(D.k2 + q2))], Z + ((int64_t)b * D.H2 + q2) * D.M1 + r);
  }
  cp_async_wait_all();
  __syncthreads();
  buf = smem_fft<T, true>(buf, alt, tw, ld, nr, D.ax2);
  const int64_t base = (int64_t)r0 * N;
  if (D.flags & 4) {
    T* Y = reinterpret_cast<T*>(D.Y) + base;
    for (int i = tid; i < nr * N; i += kFT) { const int t = i / N; Y[i] = buf[t * ld + pidx(i - t * N)].re; }
  } else {
    cpx<T>* Y = reinterpret_cast<cpx<T>*>(D.Y) + base;
    for (int i = tid; i < nr * N; i += kFT) { const int t = i / N; Y[i] = buf[t * ld + pidx(i - t * N)]; }
  }
}

// The grouped launches cover only the work of the problems taking part: k_fft_schedule (one block) lists the
// problems of the launch (subset[i], or i), drops those with live == 0, and writes the exclusive prefix sums of
// their CTA counts for stages A / C and B; CTA x of a stage finds its problem by binary search over those sums
// and returns at once when x is past the total. The grid is the host's bound: the sum of the n largest counts.
constexpr int kSchedMax = 2048;          // problems a schedule takes (a launch over more runs in chunks of 2048)

struct FftSched {
  int n;                                 // problems in the schedule
  int prob[kSchedMax];                   // their indices
  int offA[kSchedMax + 1], offB[kSchedMax + 1];
};

__global__ void k_fft_schedule(const FftDesc* __restrict__ descs, const int* __restrict__ subset, int n0, int n,
                               const int* __restrict__ live, FftSched* sch) {
  __shared__ int cA[kSchedMax], cB[kSchedMax], pr[kSchedMax];
  __shared__ int wsA[32], wsB[32];
  const int tid = threadIdx.x;
  for (int i = tid; i < n; i += blockDim.x) {
    const int g = subset ? subset[n0 + i] : n0 + i;
    const bool on = !live || live[g];
    pr[i] = g; cA[i] = on ? descs[g].ctasA : 0; cB[i] = on ? descs[g].ctasB : 0;
  }
  __syncthreads();
  if (tid < 32) {                        // one warp: a serial scan per lane chunk, then a warp scan of the chunk sums
    const int per = (n + 31) / 32, lo = tid * per, hi = min(n, lo + per);
    int sa = 0, sb = 0;
    for (int i = lo; i < hi; i++) { sa += cA[i]; sb += cB[i]; }
    int xa = sa, xb = sb;
    for (int o = 1; o < 32; o <<= 1) {
      const int ya = __shfl_up_sync(0xffffffffu, xa, o), yb = __shfl_up_sync(0xffffffffu, xb, o);
      if (tid >= o) { xa += ya; xb += yb; }
    }
    wsA[tid] = xa - sa; wsB[tid] = xb - sb;
    int ra = wsA[tid], rb = wsB[tid];
    for (int i = lo; i < hi; i++) {
      sch->offA[i] = ra; sch->offB[i] = rb; sch->prob[i] = pr[i];
      ra += cA[i]; rb += cB[i];
    }
    if (tid == 31) { sch->offA[n] = xa; sch->offB[n] = xb; sch->n = n; }
  }
}

// the problem and local CTA index of CTA x in a schedule (offsets off[0 .. n]), or -1 past the total
__device__ __forceinline__ int sched_find(const int* off, int n, int x, int& local) {
  if (x >= off[n]) return -1;
  int lo = 0, hi = n - 1;                // the last i with off[i] <= x
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (off[mid] <= x) lo = mid; else hi = mid - 1;
  }
  local = x - off[lo];
  return lo;
}

#define FFT_STAGE(NAME, BODY, OFF)                                                                                \
  template <typename T>                                                                                          \
  __global__ void __launch_bounds__(kFT, 3) NAME##_grp(const FftDesc* __restrict__ descs,                           \
                                                    const FftSched* __restrict__ sch) {                          \
    extern __shared__ __align__(16) unsigned char fft_smem[];                                                    \
    __shared__ __align__(16) FftDesc Ds;                                                                         \
    int local = 0;                                                                                               \
    const int i = sched_find(sch->OFF, sch->n, (int)blockIdx.x, local);                                          \
    if (i < 0) return;                                                                                           \
    {                                   /* the problem's descriptor, staged once per CTA */                     \
      const int* src = reinterpret_cast<const int*>(descs + sch->prob[i]);                                       \
      int* dst = reinterpret_cast<int*>(&Ds);                                                                    \
      for (int q = threadIdx.x; q < (int)(sizeof(FftDesc) / 4); q += kFT) dst[q] = src[q];                       \
    }                                                                                                            \
    __syncthreads();                                                                                             \
    BODY<T>(Ds, local, fft_smem);                                                                                \
  }                                                                                                              \
  template <typename T>                                                                                          \
  __global__ void __launch_bounds__(kFT, 3) NAME##_one(const FftDesc D) {                                           \
    extern __shared__ __align__(16) unsigned char fft_smem[];                                                    \
    BODY<T>(D, blockIdx.x, fft_smem);                                                                            \
  }

FFT_STAGE(k_fft_rows_fwd, rows_fwd_body, offA)
FFT_STAGE(k_fft_cols, cols_body, offB)
FFT_STAGE(k_fft_rows_inv, rows_inv_body, offA)

// ------------------------------------------------------------------------------------------------- host side
// radices of an N = 2^a 3^b point FFT: 8s, then a 4 or 2, then 3s, a 2 and a 3 merged into a 6 (fewest passes); 0
// when N has another prime factor or needs more than kMaxRad passes
static int radix_plan(int N, int8_t* rad) {
  int a = 0, b = 0, m = N;
  while (m % 2 == 0) { m /= 2; a++; }
  while (m % 3 == 0) { m /= 3; b++; }
  if (m != 1 || N < 2) return 0;
  std::vector<int> r;
  for (; a >= 3; a -= 3) r.push_back(8);
  int two = 0;
  if (a == 2) r.push_back(4);
  else if (a == 1) two = 1;
  for (int i = 0; i < b; i++) {
    if (two) { r.push_back(6); two = 0; }
    else r.push_back(3);
  }
  if (two) r.push_back(2);
  if ((int)r.size() > kMaxRad) return 0;
  for (size_t i = 0; i < r.size(); i++) rad[i] = (int8_t)r[i];
  return (int)r.size();
}

// an axis's passes and its twiddle table (float64 host values, interleaved complex); false when N has no plan
static bool axis_plan(int N, FftAxis& ax, std::vector<double>& tw) {
  ax = FftAxis{};
  ax.N = N;
  ax.npass = radix_plan(N, ax.rad);
  if (!ax.npass) return false;
  tw.clear();
  int Ns = 1;
  for (int p = 0; p < ax.npass; p++) {
    const int R = ax.rad[p];
    ax.ns[p] = Ns; ax.mnbt[p] = magic_of((unsigned)(N / R)); ax.mns[p] = magic_of((unsigned)Ns);
    ax.twoff[p] = (int)(tw.size() / 2);
    if (Ns > 1) {
      const int stride = N / (Ns * R);
      for (int k = 0; k < Ns; k++)
        for (int r = 1; r < R; r++) {
          const long long e = (long long)r * k * stride % N;
          const double ph = 2.0 * M_PI * (double)e / (double)N;
          tw.push_back(std::cos(ph)); tw.push_back(-std::sin(ph));
        }
    }
    Ns *= R;
  }
  ax.ntw = std::max(1, (int)(tw.size() / 2));
  if (tw.empty()) { tw.push_back(1.0); tw.push_back(0.0); }
  return true;
}

// transforms of length N per CTA: as many as two padded buffers and the twiddles hold within kCtaBytes, at least one
static int transforms_per_cta(int N, size_t esz) {
  const long long room = (long long)(g_cta_bytes / esz) - N;
  return (int)std::max<long long>(1, room / (2LL * pld(N)));
}

// two buffers of ntr padded transforms, then the twiddle table (N values at most)
static size_t stage_smem(int ntr, int N, size_t esz) { return (2 * (size_t)ntr * pld(N) + N) * esz; }

int fft_plan_init(blml_plan_s* p, const double* freqs) {
  p->fft = nullptr;
  if (p->d != 2 || p->engine != BLML_ENGINE_SIMT) return BLML_OK;
  const int M1 = (int)p->shape[0], M2 = (int)p->shape[1], H1 = p->nfreq[0], H2 = p->nfreq[1];
  if (M1 > kMaxSide || M2 > kMaxSide || H1 > M1 || H2 > M2) return BLML_OK;
  FftPlan fp{};
  fp.M1 = M1; fp.M2 = M2; fp.H1 = H1; fp.H2 = H2;
  std::vector<double> tws1, tws2;
  if (!axis_plan(M1, fp.ax1, tws1) || !axis_plan(M2, fp.ax2, tws2)) return BLML_OK;
  // integer harmonics, distinct modulo the side: then S is exactly the DFT mask
  std::vector<int> k2(H2), map1(M1, -1), seen2(M2, 0);
  for (int q = 0; q < H1 + H2; q++) {
    const int M = q < H1 ? M1 : M2;
    const double x = freqs[q] * M, r = std::nearbyint(x);
    if (std::fabs(x - r) > 1e-9 * std::max(1.0, std::fabs(r))) return BLML_OK;
    const int k = (int)(((long long)r % M + M) % M);
    if (q < H1) {
      if (map1[k] >= 0) return BLML_OK;
      map1[k] = q;
    } else {
      if (seen2[k]) return BLML_OK;
      seen2[k] = 1; k2[q - H1] = k;
    }
  }
  const bool f64 = p->dtype == BLML_F64;
  const size_t esz = f64 ? 16 : 8;
  auto table = [&](const std::vector<double>& t, void** dst) -> int {
    const size_t n = t.size() / 2;
    if (cudaMalloc(dst, n * esz) != cudaSuccess) { set_error("FFT plan: device allocation"); return BLML_ERR_CUDA; }
    if (f64) return cuda_status(cudaMemcpy(*dst, t.data(), n * esz, cudaMemcpyHostToDevice), "FFT plan twiddles");
    std::vector<float> t32(t.begin(), t.end());
    return cuda_status(cudaMemcpy(*dst, t32.data(), n * esz, cudaMemcpyHostToDevice), "FFT plan twiddles");
  };
  int rc = table(tws1, &fp.tw1);
  if (!rc) rc = table(tws2, &fp.tw2);
  if (!rc && cudaMalloc(&fp.k2, H2 * sizeof(int)) != cudaSuccess) { set_error("FFT plan: device allocation"); rc = BLML_ERR_CUDA; }
  if (!rc) rc = cuda_status(cudaMemcpy(fp.k2, k2.data(), H2 * sizeof(int), cudaMemcpyHostToDevice), "FFT plan");
  if (!rc && cudaMalloc(&fp.map1, M1 * sizeof(int)) != cudaSuccess) { set_error("FFT plan: device allocation"); rc = BLML_ERR_CUDA; }
  if (!rc) rc = cuda_status(cudaMemcpy(fp.map1, map1.data(), M1 * sizeof(int), cudaMemcpyHostToDevice), "FFT plan");
  if (rc) {
    cudaFree(fp.tw1); cudaFree(fp.tw2); cudaFree(fp.k2); cudaFree(fp.map1);
    return rc;
  }
  p->fft = new FftPlan(fp);
  return fft_smem_once();
}

void fft_plan_free(blml_plan_s* p) {
  FftPlan* fp = reinterpret_cast<FftPlan*>(p->fft);
  if (!fp) return;
  cudaFree(fp->tw1); cudaFree(fp->tw2); cudaFree(fp->k2); cudaFree(fp->map1);
  delete fp;
  p->fft = nullptr;
}

static FftDesc make_desc(const blml_plan_s* p, const void* x, void* y, void* z, int nb, int xc) {
  const FftPlan* fp = reinterpret_cast<const FftPlan*>(p->fft);
  FftDesc D{};
  D.X = x; D.Y = y; D.Z = z; D.W = p->W;
  D.tw1 = fp->tw1; D.tw2 = fp->tw2; D.k2 = fp->k2; D.map1 = fp->map1;
  D.M1 = fp->M1; D.M2 = fp->M2; D.H1 = fp->H1; D.H2 = fp->H2; D.nb = nb;
  D.flags = xc ? 0 : (1 | 4);
  const size_t esz = p->dtype == BLML_F64 ? 16 : 8;
  // the column stage has few transforms (H2 per lattice): at most 2 per CTA, so its launch still fills the GPU
  D.rows = transforms_per_cta(fp->M2, esz); D.cols = std::min(g_max_cols, transforms_per_cta(fp->M1, esz));
  D.ctasA = (nb * fp->M1 + D.rows - 1) / D.rows;
  D.ctasB = (nb * fp->H2 + D.cols - 1) / D.cols;
  D.ax1 = fp->ax1; D.ax2 = fp->ax2;
  return D;
}

struct FftGroup {
  FftDesc* dev;                  // G descriptors
  FftSched* sch;                 // the schedule of the current launch (written by k_fft_schedule)
  std::vector<int> boundA, boundB;   // [n]: the sum of the n largest CTA counts (grid bounds), n <= kSchedMax
  size_t smemA, smemB;           // largest dynamic shared memory of a problem's stage
};

// the largest dynamic shared memory any stage asks for: two padded buffers of one kMaxSide-point transform and its
// twiddles, in float64 (shorter transforms stay within the CTA budget)
constexpr size_t kMaxSmem = (size_t)(2 * (kMaxSide + kMaxSide / 8 + 1) + kMaxSide) * 16;

// the six kernels' dynamic shared-memory limit, set once per device (outside any stream capture: at plan creation)
template <typename T>
static int set_fft_smem() {
  const int v = (int)kMaxSmem;
  int e = BLML_OK;
  auto set = [&](const void* f) {
    if (!e) e = cuda_status(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, v), "FFT route");
  };
  set((const void*)k_fft_rows_fwd_grp<T>); set((const void*)k_fft_cols_grp<T>); set((const void*)k_fft_rows_inv_grp<T>);
  set((const void*)k_fft_rows_fwd_one<T>); set((const void*)k_fft_cols_one<T>); set((const void*)k_fft_rows_inv_one<T>);
  return e;
}

static int fft_smem_once() {
  static bool done[64] = {};
  int dev = 0;
  int e = cuda_status(cudaGetDevice(&dev), "FFT route");
  if (e || (dev < 64 && done[dev])) return e;
  e = set_fft_smem<double>();
  if (!e) e = set_fft_smem<float>();
  if (!e && dev < 64) done[dev] = true;
  return e;
}

template <typename T>
static int launch_fft_grp(const FftGroup* fg, const int* subset, int n0, int n, const int* live, cudaStream_t st) {
  k_fft_schedule<<<1, 256, 0, st>>>(fg->dev, subset, n0, n, live, fg->sch);
  BLML_CHECK_LAUNCH("FFT route: schedule");
  const int gA = fg->boundA[n], gB = fg->boundB[n];
  if (gA > 0) {
    k_fft_rows_fwd_grp<T><<<gA, kFT, fg->smemA, st>>>(fg->dev, fg->sch);
    BLML_CHECK_LAUNCH("FFT route: rows");
  }
  if (gB > 0) {
    k_fft_cols_grp<T><<<gB, kFT, fg->smemB, st>>>(fg->dev, fg->sch);
    BLML_CHECK_LAUNCH("FFT route: columns");
  }
  if (gA > 0) {
    k_fft_rows_inv_grp<T><<<gA, kFT, fg->smemA, st>>>(fg->dev, fg->sch);
    BLML_CHECK_LAUNCH("FFT route: inverse rows");
  }
  return BLML_OK;
}

template <typename T>
static int launch_fft_one(const FftDesc& D, size_t smA, size_t smB, cudaStream_t st) {
  k_fft_rows_fwd_one<T><<<D.ctasA, kFT, smA, st>>>(D);
  BLML_CHECK_LAUNCH("FFT route: rows");
  k_fft_cols_one<T><<<D.ctasB, kFT, smB, st>>>(D);
  BLML_CHECK_LAUNCH("FFT route: columns");
  k_fft_rows_inv_one<T><<<D.ctasA, kFT, smA, st>>>(D);
  BLML_CHECK_LAUNCH("FFT route: inverse rows");
  return BLML_OK;
}

int fft_group_init(void** out, int G, const blml_plan* plans, const int* nbatch, int xc, const void* const* x,
                   void* const* y, void* const* z) {
  *out = nullptr;
  for (int g = 0; g < G; g++)
    if (!plans[g]->fft) return BLML_OK;
  const size_t esz = plans[0]->dtype == BLML_F64 ? 16 : 8;
  std::vector<FftDesc> h(G);
  FftGroup* fg = new FftGroup();
  fg->dev = nullptr; fg->sch = nullptr; fg->smemA = fg->smemB = 0;
  std::vector<int> cA(G), cB(G);
  for (int g = 0; g < G; g++) {
    h[g] = make_desc(plans[g], x[g], y[g], z[g], nbatch[g], xc);
    cA[g] = h[g].ctasA; cB[g] = h[g].ctasB;
    fg->smemA = std::max(fg->smemA, stage_smem(h[g].rows, h[g].M2, esz));
    fg->smemB = std::max(fg->smemB, stage_smem(h[g].cols, h[g].M1, esz));
  }
  std::sort(cA.begin(), cA.end(), std::greater<int>()); std::sort(cB.begin(), cB.end(), std::greater<int>());
  const int nmax = std::min(G, kSchedMax);
  fg->boundA.assign(nmax + 1, 0); fg->boundB.assign(nmax + 1, 0);
  for (int i = 0; i < nmax; i++) { fg->boundA[i + 1] = fg->boundA[i] + cA[i]; fg->boundB[i + 1] = fg->boundB[i] + cB[i]; }
  int e = fft_smem_once();
  if (!e && cudaMalloc(&fg->dev, G * sizeof(FftDesc)) != cudaSuccess) { set_error("FFT route: allocation"); e = BLML_ERR_CUDA; }
  if (!e && cudaMalloc(&fg->sch, sizeof(FftSched)) != cudaSuccess) { set_error("FFT route: allocation"); e = BLML_ERR_CUDA; }
  if (!e) e = cuda_status(cudaMemcpy(fg->dev, h.data(), G * sizeof(FftDesc), cudaMemcpyHostToDevice), "FFT route");
  if (e) { fft_group_free(fg); return e; }
  *out = fg;
  return BLML_OK;
}

void fft_group_free(void* fgv) {
  FftGroup* fg = reinterpret_cast<FftGroup*>(fgv);
  if (!fg) return;
  cudaFree(fg->dev); cudaFree(fg->sch);
  delete fg;
}

// problems of the launch in chunks of kSchedMax (one schedule buffer: the chunks run one after another on st)
int fft_group_launch(void* fgv, int dtype, const int* subset, int n, const int* live, cudaStream_t st) {
  const FftGroup* fg = reinterpret_cast<const FftGroup*>(fgv);
  for (int n0 = 0; n0 < n; n0 += kSchedMax) {
    const int nc = std::min(kSchedMax, n - n0);
    const int e = dtype == BLML_F64 ? launch_fft_grp<double>(fg, subset, n0, nc, live, st)
                                    : launch_fft_grp<float>(fg, subset, n0, nc, live, st);
    if (e) return e;
  }
  return BLML_OK;
}

// one plan over nb lattices: Z (nb, H2, M1) in the caller's workspace, the descriptor passed by value
int64_t fft_workspace(const blml_plan_s* p, int nb) {
  const FftPlan* fp = reinterpret_cast<const FftPlan*>(p->fft);
  const size_t esz = p->dtype == BLML_F64 ? 16 : 8;
  return (int64_t)((size_t)nb * fp->H2 * fp->M1 * esz);
}

int fft_matvec(blml_plan_s* p, const void* x, void* y, int nb, int xc, void* ws, cudaStream_t st) {
  const size_t esz = p->dtype == BLML_F64 ? 16 : 8;
  const FftDesc D = make_desc(p, x, y, ws, nb, xc);
  const size_t smA = stage_smem(D.rows, D.M2, esz), smB = stage_smem(D.cols, D.M1, esz);
  return p->dtype == BLML_F64 ? launch_fft_one<double>(D, smA, smB, st) : launch_fft_one<float>(D, smA, smB, st);
}

}  // namespace blml

extern "C" {

int blml_fft_set_shape(int cta_bytes, int max_cols) {
  if (cta_bytes < 8 * 1024 || cta_bytes > blml::kCtaBytesMax || max_cols < 1 || max_cols > 64) {
    blml::set_error("blml_fft_set_shape: 8 KiB <= cta_bytes <= %d, 1 <= max_cols <= 64", blml::kCtaBytesMax);
    return BLML_ERR_ARG;
  }
  blml::g_cta_bytes = cta_bytes; blml::g_max_cols = max_cols;
  return BLML_OK;
}

int blml_fft_get_shape(int* cta_bytes, int* max_cols) {
  if (!cta_bytes || !max_cols) { blml::set_error("blml_fft_get_shape: null argument"); return BLML_ERR_ARG; }
  *cta_bytes = blml::g_cta_bytes; *max_cols = blml::g_max_cols;
  return BLML_OK;
}

}
