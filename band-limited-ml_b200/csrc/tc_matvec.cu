// Tensor-core (tcgen05) engine of the restricted-transform mat-vec: float32 storage, split-TF32 operands.
//
// Each stage of the transform (csrc/matvec.cu: contract the last axis, move the new axis to the front) is a real GEMM
// once complex numbers are embedded as 2 x 2 real blocks: the interleaved (re, im) storage of a complex (R x M)
// matrix IS a real (R x 2M) matrix, and the twiddle matrix T (M x N) becomes the real (2M x 2N) block matrix
// [[Tr, Ti], [-Ti, Tr]] (rows / columns interleaved the same way), so C = A B comes out interleaved as complex
// (R x N). Operands are TF32-split (x = hi + lo, hi the TF32 rounding of x): A_hi B_hi + A_hi B_lo + A_lo B_hi,
// three tcgen05.mma.kind::tf32 products accumulated in FP32 in tensor memory, which keeps float32 accuracy.
//
// Per CTA: a 128-row x NT-column output tile (NT <= 256). Per K block of 32: one thread issues TMA loads of the A
// tile (128 x 32 fp32, 128-byte swizzle) and the B hi / lo tiles (NT x 32, the twiddles precomputed K-major); the
// CTA splits A into hi / lo in shared memory; one thread issues 4 K-steps x 3 MMAs (M 128, N NT, K 8) and commits to
// an mbarrier. The epilogue reads the accumulators with tcgen05.ld (warp w owns TMEM lanes 32w..32w+31) and writes
// the stage's transposed layout Y[b][n][r] (optionally weighted, or real part only). Every wait is bounded: on
// timeout the kernel records an error code, frees its tensor memory and returns.
#include <cuda.h>
#include <string.h>
#include <vector>
#include "plan.cuh"

namespace blml {

constexpr int TC_BM = 128, TC_BK = 32;
constexpr int TC_THREADS = 128;

// one GEMM operand B (the real-embedded twiddles of one stage), K-major: rows n (2N or, for a real-input first stage,
// 2N with K = M), columns k, hi and lo parts
struct TcB {
  int K, Nr, ldk;            // logical K, output real columns, padded row length (floats)
  float* hi; float* lo;
  CUtensorMap mh, ml;        // their tensor maps, encoded once when the plan is built
};
struct TcPlan {
  TcB fwd[8], fwd_real[8], inv[8];
  int* err;                  // device error word (0 = fine)
};

// ----------------------------------------------------------------------------------------------- device helpers
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// bounded wait for the phase with the given parity; false on timeout
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  for (long it = 0; it < (1L << 22); it++) {
    uint32_t done;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
                 : "=r"(done) : "r"(smem_u32(bar)), "r"(parity) : "memory");
    if (done) return true;
  }
  return false;
}
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int c0, int c1, uint64_t* bar) {
  asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
               :: "r"(smem_u32(dst)), "l"(map), "r"(c0), "r"(c1), "r"(smem_u32(bar)) : "memory");
}

// shared-memory matrix descriptor of a K-major, 128-byte-swizzled tile: 8-row core groups 1024 bytes apart
__device__ __forceinline__ uint64_t umma_desc(const void* p) {
  const uint64_t addr = smem_u32(p);
  uint64_t d = 0;
  d |= (addr >> 4) & 0x3FFFull;                 // start address
  d |= (uint64_t)(16 >> 4) << 16;               // leading byte offset (unused for swizzled K-major)
  d |= (uint64_t)(1024 >> 4) << 32;             // stride byte offset
  d |= (uint64_t)1 << 46;                       // descriptor version (sm_100)
  d |= (uint64_t)2 << 61;                       // 128-byte swizzle
  return d;
}
// instruction descriptor: kind::tf32, D f32, A / B tf32, both K-major, M = 128, N = n
__host__ __device__ constexpr uint32_t idesc_tf32(int n) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(TC_BM >> 4) << 24);
}

__device__ __forceinline__ float tf32_hi(float x) {
  return __uint_as_float((__float_as_uint(x) + 0x1000u) & 0xFFFFE000u);
}

template <bool WEIGHT, bool YREAL>
__global__ void __launch_bounds__(TC_THREADS) k_tc_stage(const __grid_constant__ CUtensorMap mA,
                                                         const __grid_constant__ CUtensorMap mBh,
                                                         const __grid_constant__ CUtensorMap mBl, int K, int Nr,
                                                         int NT, int tcols, int64_t rows, int64_t Rs, int64_t ldout,
                                                         const float* __restrict__ W, void* __restrict__ Y, int* err) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  float* sA = reinterpret_cast<float*>(base);
  float* sAl = sA + TC_BM * TC_BK;
  float* sBh = sAl + TC_BM * TC_BK;
  float* sBl = sBh + NT * TC_BK;
  uint64_t* bars = reinterpret_cast<uint64_t*>(sBl + NT * TC_BK);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + 2);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int64_t m0 = (int64_t)blockIdx.x * TC_BM;
  const int n0 = blockIdx.y * NT;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" :: "r"(smem_u32(tslot)), "r"(tcols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    mbar_init(&bars[0], 1); mbar_init(&bars[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t taddr = *tslot;
  const int nk = (K + TC_BK - 1) / TC_BK;
  const uint32_t tx = (uint32_t)(TC_BM * TC_BK * 4 + 2 * NT * TC_BK * 4);
  const uint32_t idesc = idesc_tf32(NT);
  bool ok = true;
  uint32_t par_last = 0;
  for (int kb = 0; kb < nk && ok; kb++) {
    const uint32_t par = kb & 1;
    par_last = par;
    if (tid == 0) {
      mbar_expect_tx(&bars[0], tx);
      tma_load_2d(sA, &mA, kb * TC_BK, (int)m0, &bars[0]);
      tma_load_2d(sBh, &mBh, kb * TC_BK, n0, &bars[0]);
      tma_load_2d(sBl, &mBl, kb * TC_BK, n0, &bars[0]);
    }
    ok = mbar_wait(&bars[0], par);
    if (!ok) break;
    for (int i = tid; i < TC_BM * TC_BK; i += TC_THREADS) {    // split A into TF32 hi / lo in place
      const float x = sA[i], hi = tf32_hi(x);
      sA[i] = hi; sAl[i] = x - hi;
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
      for (int j = 0; j < TC_BK / 8; j++) {
        const uint64_t ah = umma_desc(sA + j * 8), al = umma_desc(sAl + j * 8);
        const uint64_t bh = umma_desc(sBh + j * 8), bl = umma_desc(sBl + j * 8);
        const uint32_t acc0 = (kb > 0 || j > 0) ? 1u : 0u;
        asm volatile("{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                     " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n"
                     :: "r"(taddr), "l"(ah), "l"(bh), "r"(idesc), "r"(acc0));
        asm volatile("tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, 1;"
                     :: "r"(taddr), "l"(ah), "l"(bl), "r"(idesc));
        asm volatile("tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, 1;"
                     :: "r"(taddr), "l"(al), "l"(bh), "r"(idesc));
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                   :: "r"(smem_u32(&bars[1])) : "memory");
    }
    ok = mbar_wait(&bars[1], par);
  }
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (!ok) {
    // a bounded wait gave up: record it, then give copies / MMAs in flight one more bounded wait before the tensor
    // memory is released
    if (tid == 0) atomicExch(err, 1);
    mbar_wait(&bars[0], par_last);
    mbar_wait(&bars[1], par_last);
  } else {
    const int64_t row = m0 + 32 * warp + lane;
    const int64_t b = row / Rs, r = row - (row / Rs) * Rs;
    for (int c0 = 0; c0 < NT; c0 += 16) {
      uint32_t v[16];
      asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
                   "%13, %14, %15}, [%16];"
                   : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                     "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
                     "=r"(v[15])
                   : "r"(taddr + ((uint32_t)(32 * warp) << 16) + (uint32_t)c0));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (row < rows) {
#pragma unroll
        for (int p = 0; p < 8; p++) {
          const int col = n0 + c0 + 2 * p;
          if (col >= Nr) break;
          const int n = col >> 1;
          float re = __uint_as_float(v[2 * p]), im = __uint_as_float(v[2 * p + 1]);
          const int64_t o = b * (int64_t)(Nr >> 1) * ldout + (int64_t)n * ldout + r;
          if (WEIGHT) { const float wv = W[(int64_t)n * Rs + r]; re *= wv; im *= wv; }
          if (YREAL) reinterpret_cast<float*>(Y)[o] = re;
          else reinterpret_cast<float2*>(Y)[o] = make_float2(re, im);
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(taddr), "r"(tcols));
}

// ----------------------------------------------------------------------------------------------- host side
typedef CUresult (*EncodeFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                             const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                             CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeFn encode_fn() {
  static EncodeFn fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeFn>(p);
  }
  return fn;
}

// a 2-D fp32 tensor map (inner extent `inner` floats, `outer` rows of `ld` floats), box {32, box_rows}, 128B swizzle
static int make_map(CUtensorMap* m, const void* ptr, int64_t inner, int64_t outer, int64_t ld, int box_rows) {
  EncodeFn fn = encode_fn();
  if (!fn) { set_error("tensor-core engine: cuTensorMapEncodeTiled unavailable"); return BLML_ERR_CUDA; }
  if ((reinterpret_cast<uintptr_t>(ptr) & 15) || (ld * 4) % 16) {
    set_error("tensor-core engine: operand not 16-byte aligned"); return BLML_ERR_ARG;
  }
  cuuint64_t dims[2] = {(cuuint64_t)inner, (cuuint64_t)outer};
  cuuint64_t strides[1] = {(cuuint64_t)(ld * 4)};
  cuuint32_t box[2] = {(cuuint32_t)TC_BK, (cuuint32_t)box_rows};
  cuuint32_t es[2] = {1, 1};
  CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<void*>(ptr), dims, strides, box, es,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) { set_error("tensor-core engine: tensor map encoding failed (%d)", (int)r); return BLML_ERR_CUDA; }
  return BLML_OK;
}

static inline int64_t even(int64_t x) { return (x + 1) & ~(int64_t)1; }
static inline int out_tile(int Nr) { return Nr <= 256 ? (int)((Nr + 15) / 16 * 16) : 256; }
static inline int tmem_cols(int nt) { int c = 32; while (c < nt) c <<= 1; return c; }
static inline size_t tc_smem(int nt) { return 1024 + (size_t)(2 * TC_BM * TC_BK + 2 * nt * TC_BK) * 4 + 64; }

// upload one real-embedded twiddle operand: B^T (Nr x K) from the complex matrix T (Mc x Nc, row-major, interleaved)
// complex input: K = 2 Mc, Nr = 2 Nc; real input: K = Mc, Nr = 2 Nc
static int upload_B(TcB& b, const std::vector<double>& T, int Mc, int Nc, bool real_input) {
  b.K = real_input ? Mc : 2 * Mc; b.Nr = 2 * Nc; b.ldk = (int)((b.K + 3) & ~3);
  std::vector<float> hi((size_t)b.Nr * b.ldk, 0.f), lo((size_t)b.Nr * b.ldk, 0.f);
  for (int m = 0; m < Mc; m++)
    for (int n = 0; n < Nc; n++) {
      const double tr = T[2 * ((size_t)m * Nc + n)], ti = T[2 * ((size_t)m * Nc + n) + 1];
      // C[:, 2n] (re) and C[:, 2n + 1] (im) from A[:, 2m] (re) and A[:, 2m + 1] (im)
      double e[2][2] = {{tr, ti}, {-ti, tr}};
      for (int ka = 0; ka < (real_input ? 1 : 2); ka++)
        for (int c = 0; c < 2; c++) {
          const int k = real_input ? m : 2 * m + ka, nr = 2 * n + c;
          const double v = e[ka][c];
          const float h = (float)v;
          uint32_t u; memcpy(&u, &h, 4); u = (u + 0x1000u) & 0xFFFFE000u;
          float hh; memcpy(&hh, &u, 4);
          hi[(size_t)nr * b.ldk + k] = hh; lo[(size_t)nr * b.ldk + k] = (float)(v - (double)hh);
        }
    }
  const size_t bytes = hi.size() * 4;
  if (cudaMalloc(&b.hi, bytes) != cudaSuccess || cudaMalloc(&b.lo, bytes) != cudaSuccess) {
    set_error("tensor-core engine: device allocation failed"); return BLML_ERR_CUDA;
  }
  int e = cuda_status(cudaMemcpy(b.hi, hi.data(), bytes, cudaMemcpyHostToDevice), "tc twiddles");
  if (!e) e = cuda_status(cudaMemcpy(b.lo, lo.data(), bytes, cudaMemcpyHostToDevice), "tc twiddles");
  const int nt = out_tile(b.Nr);
  if (!e) e = make_map(&b.mh, b.hi, b.K, b.Nr, b.ldk, nt);
  if (!e) e = make_map(&b.ml, b.lo, b.K, b.Nr, b.ldk, nt);
  return e;
}

static void free_B(TcB& b) { cudaFree(b.hi); cudaFree(b.lo); b.hi = b.lo = nullptr; }

int tc_plan_init(blml_plan_s* p, const std::vector<std::vector<double>>& fwd,
                 const std::vector<std::vector<double>>& inv) {
  if (p->d != 2) { set_error("tensor-core engine: 2-D lattices only"); return BLML_ERR_UNSUPPORTED; }
  if (!encode_fn()) { set_error("tensor-core engine: cuTensorMapEncodeTiled unavailable"); return BLML_ERR_CUDA; }
  TcPlan* tp = new TcPlan();
  memset(tp, 0, sizeof(TcPlan));
  p->tc = tp;
  int e = BLML_OK;
  for (int a = 0; a < p->d && !e; a++) {
    const int M = (int)p->shape[a], H = p->nfreq[a];
    e = upload_B(tp->fwd[a], fwd[a], M, H, false);
    if (!e) e = upload_B(tp->fwd_real[a], fwd[a], M, H, true);
    if (!e) e = upload_B(tp->inv[a], inv[a], H, M, false);
  }
  if (!e && cudaMalloc(&tp->err, sizeof(int)) != cudaSuccess) { set_error("tc plan: allocation"); e = BLML_ERR_CUDA; }
  if (!e) e = cuda_status(cudaMemset(tp->err, 0, sizeof(int)), "tc plan");
  if (e) tc_plan_free(p);
  return e;
}

void tc_plan_free(blml_plan_s* p) {
  TcPlan* tp = reinterpret_cast<TcPlan*>(p->tc);
  if (!tp) return;
  for (int a = 0; a < 8; a++) { free_B(tp->fwd[a]); free_B(tp->fwd_real[a]); free_B(tp->inv[a]); }
  cudaFree(tp->err);
  delete tp;
  p->tc = nullptr;
}

// the stage schedule with even leading dimensions (16-byte rows for TMA): returns the workspace elements per lattice
static int64_t tc_elems(const blml_plan_s* p) {
  const int d = p->d;
  std::vector<int64_t> dims(p->shape, p->shape + d);
  int64_t mx = 0;
  for (int s = 0; s < 2 * d - 1; s++) {
    const int a = d - 1 - (s % d);
    const int64_t N = s < d ? p->nfreq[a] : p->shape[a];
    dims.pop_back(); dims.insert(dims.begin(), N);
    int64_t R = 1; for (size_t i = 1; i < dims.size(); i++) R *= dims[i];
    mx = std::max(mx, N * even(R));
  }
  return mx;
}

int64_t tc_workspace(const blml_plan_s* p, int nb) { return 2 * (int64_t)nb * tc_elems(p) * 8; }

template <bool W_, bool YR>
static int launch_tc(const CUtensorMap& mA, const TcB& B, int64_t rows, int64_t Rs, int64_t ldout, const float* W,
                     void* Y, int* err, cudaStream_t st) {
  const int nt = out_tile(B.Nr);
  const size_t sm = tc_smem(nt);
  static int attr_dev = -1;                     // the largest tile's shared memory, set once per device
  int dev = 0;
  cudaGetDevice(&dev);
  if (attr_dev != dev) {
    int e = cuda_status(cudaFuncSetAttribute(k_tc_stage<W_, YR>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)tc_smem(256)), "tc stage");
    if (e) return e;
    attr_dev = dev;
  }
  dim3 grid((unsigned)((rows + TC_BM - 1) / TC_BM), (unsigned)((B.Nr + nt - 1) / nt));
  k_tc_stage<W_, YR><<<grid, TC_THREADS, sm, st>>>(mA, B.mh, B.ml, B.K, B.Nr, nt, tmem_cols(nt), rows, Rs, ldout, W,
                                                  Y, err);
  BLML_CHECK_LAUNCH("tc stage");
  return BLML_OK;
}

int tc_matvec(blml_plan_s* p, const void* x, void* y, int nb, int xc, void* ws, int64_t wsb, cudaStream_t st) {
  TcPlan* tp = reinterpret_cast<TcPlan*>(p->tc);
  if (!tp) { set_error("blml_matvec: tensor-core plan not initialised"); return BLML_ERR_UNSUPPORTED; }
  if (p->shape[p->d - 1] % 4) {
    set_error("blml_matvec: the tensor-core engine needs the last lattice axis a multiple of 4");
    return BLML_ERR_UNSUPPORTED;
  }
  const int d = p->d;
  const int64_t per = tc_elems(p);
  char* buf[2] = {reinterpret_cast<char*>(ws), reinterpret_cast<char*>(ws) + (size_t)nb * per * 8};
  (void)wsb;
  std::vector<int64_t> dims(p->shape, p->shape + d);
  const void* cur = x; bool cur_real = !xc; int64_t cur_ld = p->shape[d - 1];
  int which = 0;
  for (int s = 0; s < 2 * d; s++) {
    const bool fwd = s < d;
    const int a = d - 1 - (s % d);
    const int64_t M = dims.back();
    int64_t tot = 1; for (auto v : dims) tot *= v;
    const int64_t Rs = tot / M;                  // rows per lattice
    const bool last = s == 2 * d - 1;
    const TcB& B = fwd ? (cur_real ? tp->fwd_real[a] : tp->fwd[a]) : tp->inv[a];
    const int64_t N = B.Nr / 2;
    const int64_t ldout = last ? Rs : even(Rs);
    void* out = last ? y : buf[which];
    CUtensorMap mA;
    const int64_t inner = cur_real ? M : 2 * M, ldA = cur_real ? cur_ld : 2 * cur_ld;
    int e = make_map(&mA, cur, inner, nb * Rs, ldA, TC_BM);
    if (e) return e;
    const float* W = (s == d - 1) ? reinterpret_cast<const float*>(p->W) : nullptr;
    const int64_t rows = nb * Rs;
    if (W) e = launch_tc<true, false>(mA, B, rows, Rs, ldout, W, out, tp->err, st);
    else if (last && !xc) e = launch_tc<false, true>(mA, B, rows, Rs, ldout, nullptr, out, tp->err, st);
    else e = launch_tc<false, false>(mA, B, rows, Rs, ldout, nullptr, out, tp->err, st);
    if (e) return e;
    dims.pop_back(); dims.insert(dims.begin(), N);
    cur = out; cur_real = false; cur_ld = ldout; which ^= 1;
  }
  return BLML_OK;
}

int tc_error(blml_plan_s* p) {
  TcPlan* tp = reinterpret_cast<TcPlan*>(p->tc);
  if (!tp) return 0;
  int h = 0;
  cudaMemcpy(&h, tp->err, sizeof(int), cudaMemcpyDeviceToHost);
  return h;
}

}  // namespace blml
