// Kernels of the learned warm start: a small convolutional U-Net that maps (log counts, cut-off, kernel kind) on a
// lattice to the field u = S e / n of the fit, trained on fits the engine produces. No counterpart in the reference
// (its start is the real rank-1 solve, blml_binned.py:415-436); the net replaces that start for the fits it covers.
//
// Activations are NHWC (channels innermost) in BF16, read from / written to channel slices of wider buffers so the
// decoder's skip concatenation needs no copy; gradients are FP32 in the same layout. A 3 x 3 convolution (pad 1) is
// an implicit GEMM over an explicit im2col matrix Col[p][(ky 3 + kx) C + c]:
//   forward        Y[P x Cout]   = Col[P x 9C] . W[Cout x 9C]^T
//   data grad      dCol[P x 9C]  = dPre[P x Cout] . Wt[9C x Cout]^T      (then col2im gathers the 9 taps)
//   weight grad    dW[Cout x 9C] = dPreT[Cout x P] . ColT[9C x P]^T      (split over P, partials summed in order)
// Every GEMM is C = A B^T with A (M x K) and B (N x K) K-major BF16 and FP32 output, on tcgen05: TMA loads of
// 128-byte-swizzled 64-deep K slices into a ring of up to 8 stages, one elected thread issuing kind::f16 MMAs (M 128,
// N <= 256, K 16) into one of two TMEM accumulators, tcgen05.ld epilogue overlapping the next tile's MMAs. Waits are bounded: on timeout the kernel sets the caller's error word, gives
// copies and MMAs in flight one more bounded wait, frees its tensor memory and returns.
#include <cuda.h>
#include <cuda_bf16.h>
#include <string.h>
#include <vector>
#include "common.cuh"

namespace blml {

constexpr int NN_BM = 128, NN_BK = 64;

__device__ __forceinline__ uint32_t nn_smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void nn_mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(nn_smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void nn_mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(nn_smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool nn_mbar_wait(uint64_t* bar, uint32_t parity) {
  for (long it = 0; it < (1L << 20); it++) {
    uint32_t done;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
                 : "=r"(done) : "r"(nn_smem_u32(bar)), "r"(parity) : "memory");
    if (done) return true;
  }
  return false;
}
__device__ __forceinline__ void nn_tma_2d(void* dst, const CUtensorMap* map, int c0, int c1, uint64_t* bar) {
  asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
               :: "r"(nn_smem_u32(dst)), "l"(map), "r"(c0), "r"(c1), "r"(nn_smem_u32(bar)) : "memory");
}
// K-major, 128-byte-swizzled operand tile: 8-row core groups 1024 bytes apart
__device__ __forceinline__ uint64_t nn_desc(const void* p) {
  const uint64_t addr = nn_smem_u32(p);
  uint64_t d = 0;
  d |= (addr >> 4) & 0x3FFFull;
  d |= (uint64_t)(16 >> 4) << 16;
  d |= (uint64_t)(1024 >> 4) << 32;
  d |= (uint64_t)1 << 46;
  d |= (uint64_t)2 << 61;
  return d;
}
// kind::f16 instruction descriptor: D f32, A and B bf16, both K-major, M = 128, N = n
__host__ __device__ constexpr uint32_t idesc_bf16(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(NN_BM >> 4) << 24);
}

// C[z][m][n] = sum_{k in split z} A[m][k] B[n][k]. Persistent, one CTA per SM (its shared memory keeps a second
// one out), warp-specialised over a ring of `stages` shared-memory K slices and two TMEM accumulators:
//   warp 4 lane 0   TMA producer: waits for a free slice (empty[s]), loads A and B of the next K slice (full[s])
//   warp 5 lane 0   MMA issuer: waits for a loaded slice, issues its four K = 16 MMAs into the tile's accumulator and
//                   commits to empty[s] (the slice is reusable once those MMAs have read it); after a tile's last
//                   slice it commits to tfull[a]
//   warps 0-3       epilogue: wait for tfull[a], tcgen05.ld their 32 TMEM lanes, store, arrive on tempty[a]
// so the loads run `stages` slices ahead of the MMAs and a tile's epilogue overlaps the next tile's MMAs. Tiles are
// walked t = blockIdx.x, blockIdx.x + gridDim.x, ... with the n tile fastest, so the CTAs that share an A tile run
// at the same time and the second read of it comes from L2. Tiles whose split has an empty K range are written as
// zeros by the epilogue and skipped by the other roles.
constexpr int NN_PIPE_THREADS = 192, NN_MAX_STAGES = 8;

struct NNPipeShared {
  uint64_t full[NN_MAX_STAGES], empty[NN_MAX_STAGES], tfull[2], tempty[2];
  uint32_t tslot;
  int abort;
  long long issued, consumed;           // K slices loaded by the producer / taken by the MMA issuer
};

__device__ __forceinline__ bool nn_wait_or_abort(uint64_t* bar, uint32_t parity, volatile int* abort) {
  for (long it = 0; it < (1L << 20); it++) {
    uint32_t done;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
                 : "=r"(done) : "r"(nn_smem_u32(bar)), "r"(parity) : "memory");
    if (done) return true;
    if ((it & 63) == 63 && abort && *abort) return false;
  }
  return false;
}

__device__ __forceinline__ void nn_fail(volatile int* abort, int* err) {
  *abort = 1;
  atomicExch(err, 1);
}

__global__ void __launch_bounds__(NN_PIPE_THREADS, 1) k_gemm_bf16(const __grid_constant__ CUtensorMap mA,
                                                                  const __grid_constant__ CUtensorMap mB, int M, int N,
                                                                  int NT, int tcols, int nkb, int kb_per_split,
                                                                  int splits, int stages, float* C, int* err) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  const uint32_t a_bytes = NN_BM * NN_BK * 2, stage_bytes = a_bytes + (uint32_t)NT * NN_BK * 2;
  NNPipeShared* sh = reinterpret_cast<NNPipeShared*>(base + (size_t)stages * stage_bytes);
  volatile int* abort = &sh->abort;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int Mt = (M + NN_BM - 1) / NN_BM, Nt = (N + NT - 1) / NT;
  const long long tiles = (long long)Mt * Nt * splits;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :: "r"(nn_smem_u32(&sh->tslot)), "r"(2 * tcols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 32) {
    for (int s = 0; s < stages; s++) { nn_mbar_init(&sh->full[s], 1); nn_mbar_init(&sh->empty[s], 1); }
    for (int a = 0; a < 2; a++) { nn_mbar_init(&sh->tfull[a], 1); nn_mbar_init(&sh->tempty[a], 4); }
    sh->abort = 0; sh->issued = 0; sh->consumed = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t taddr = sh->tslot;

  if (warp == 4 && lane == 0) {                                   // ---- TMA producer
    const uint32_t tx = stage_bytes;
    long long g = 0;
    for (long long t = blockIdx.x; t < tiles && !*abort; t += gridDim.x) {
      const int z = (int)(t / ((long long)Mt * Nt));
      const long long rem = t - (long long)z * Mt * Nt;
      const int mt_i = (int)(rem / Nt), nt_i = (int)(rem - (long long)mt_i * Nt);
      const int kb0 = z * kb_per_split, kb1 = min(nkb, kb0 + kb_per_split);
      for (int kb = kb0; kb < kb1; kb++, g++) {
        const int s = (int)(g % stages);
        const long long r = g / stages;
        if (r > 0 && !nn_wait_or_abort(&sh->empty[s], (uint32_t)((r - 1) & 1), abort)) { nn_fail(abort, err); break; }
        uint8_t* sa = base + (size_t)s * stage_bytes;
        nn_mbar_expect_tx(&sh->full[s], tx);
        nn_tma_2d(sa, &mA, kb * NN_BK, mt_i * NN_BM, &sh->full[s]);
        nn_tma_2d(sa + a_bytes, &mB, kb * NN_BK, nt_i * NT, &sh->full[s]);
        *(volatile long long*)&sh->issued = g + 1;
      }
    }
  } else if (warp == 5 && lane == 0) {                            // ---- MMA issuer
    const uint32_t idesc = idesc_bf16(NT);
    long long g = 0, it = 0;
    for (long long t = blockIdx.x; t < tiles && !*abort; t += gridDim.x) {
      const int z = (int)(t / ((long long)Mt * Nt));
      const int kb0 = z * kb_per_split, kb1 = min(nkb, kb0 + kb_per_split);
      if (kb0 >= kb1) continue;
      const int a = (int)(it & 1);
      const long long u = it >> 1;
      if (u > 0 && !nn_wait_or_abort(&sh->tempty[a], (uint32_t)((u - 1) & 1), abort)) { nn_fail(abort, err); break; }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t acc_addr = taddr + (uint32_t)(a * tcols);
      bool ok = true;
      for (int kb = kb0; kb < kb1; kb++, g++) {
        const int s = (int)(g % stages);
        if (!nn_wait_or_abort(&sh->full[s], (uint32_t)((g / stages) & 1), abort)) { ok = false; break; }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const __nv_bfloat16* sa = reinterpret_cast<const __nv_bfloat16*>(base + (size_t)s * stage_bytes);
        const __nv_bfloat16* sb = reinterpret_cast<const __nv_bfloat16*>(base + (size_t)s * stage_bytes + a_bytes);
#pragma unroll
        for (int j = 0; j < NN_BK / 16; j++) {
          const uint64_t ad = nn_desc(sa + j * 16), bd = nn_desc(sb + j * 16);
          const uint32_t acc = (kb > kb0 || j > 0) ? 1u : 0u;
          asm volatile("{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                       " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n"
                       :: "r"(acc_addr), "l"(ad), "l"(bd), "r"(idesc), "r"(acc));
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                     :: "r"(nn_smem_u32(&sh->empty[s])) : "memory");
        *(volatile long long*)&sh->consumed = g + 1;
      }
      if (!ok) { nn_fail(abort, err); break; }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                   :: "r"(nn_smem_u32(&sh->tfull[a])) : "memory");
      it++;
    }
  } else if (warp < 4) {                                          // ---- epilogue
    const bool vec = (N % 4 == 0) && ((reinterpret_cast<uintptr_t>(C) & 15) == 0);
    long long it = 0;
    for (long long t = blockIdx.x; t < tiles; t += gridDim.x) {
      if (__any_sync(0xffffffffu, *abort != 0)) break;            // warp-uniform: the tcgen05.ld below are .aligned
      const int z = (int)(t / ((long long)Mt * Nt));
      const long long rem = t - (long long)z * Mt * Nt;
      const int mt_i = (int)(rem / Nt), nt_i = (int)(rem - (long long)mt_i * Nt);
      const int m0 = mt_i * NN_BM, n0 = nt_i * NT;
      const int kb0 = z * kb_per_split, kb1 = min(nkb, kb0 + kb_per_split);
      float* Cz = C + (size_t)z * M * N;
      const int row = m0 + 32 * warp + lane;
      if (kb0 >= kb1) {                                           // an empty K range: the partial is zero
        if (row < M)
          for (int col = n0; col < min(N, n0 + NT); col++) Cz[(size_t)row * N + col] = 0.f;
        continue;
      }
      const int a = (int)(it & 1);
      const long long u = it >> 1;
      const bool got = nn_wait_or_abort(&sh->tfull[a], (uint32_t)(u & 1), abort);
      if (!__all_sync(0xffffffffu, got)) { if (lane == 0) nn_fail(abort, err); break; }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      for (int c0 = 0; c0 < NT; c0 += 16) {
        uint32_t v[16];
        asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
                     "%13, %14, %15}, [%16];"
                     : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                       "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
                       "=r"(v[15])
                     : "r"(taddr + ((uint32_t)(32 * warp) << 16) + (uint32_t)(a * tcols + c0)));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (row < M) {
          float* out = Cz + (size_t)row * N + n0 + c0;
          const int nv = min(16, N - (n0 + c0));
          if (vec && nv == 16) {
#pragma unroll
            for (int i = 0; i < 16; i += 4)
              *reinterpret_cast<float4*>(out + i) = make_float4(__uint_as_float(v[i]), __uint_as_float(v[i + 1]),
                                                                __uint_as_float(v[i + 2]), __uint_as_float(v[i + 3]));
          } else {
#pragma unroll
            for (int i = 0; i < 16; i++)
              if (i < nv) out[i] = __uint_as_float(v[i]);
          }
        }
      }
      // this warp's accumulator reads are done: the MMA issuer may overwrite the accumulator
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncwarp();
      if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" :: "r"(nn_smem_u32(&sh->tempty[a])) : "memory");
      it++;
    }
  }
  __syncthreads();
  if (*abort && tid == 0) {
    // a bounded wait gave up: the slices still loading and the MMAs last committed get one more bounded wait each
    // before the shared and tensor memory are released
    const long long iss = *(volatile long long*)&sh->issued, con = *(volatile long long*)&sh->consumed;
    for (long long g = con; g < iss; g++)
      nn_wait_or_abort(&sh->full[g % stages], (uint32_t)((g / stages) & 1), nullptr);
    if (con > 0) nn_wait_or_abort(&sh->empty[(con - 1) % stages], (uint32_t)(((con - 1) / stages) & 1), nullptr);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(taddr), "r"(2 * tcols));
}

// ---------------------------------------------------------------------------------------------- layout kernels
// Col[p][(ky 3 + kx) C + c] = X[n, y + ky - 1, x + kx - 1, c0 + c] (0 outside), or its transpose ColT[k][p]
__global__ void k_im2col(const __nv_bfloat16* __restrict__ X, int Nb, int H, int W, int Cs, int c0, int C,
                         __nv_bfloat16* __restrict__ col, int transposed) {
  const int64_t P = (int64_t)Nb * H * W, K9 = 9 * (int64_t)C;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P * K9) return;
  int64_t p, k;
  if (transposed) { k = i / P; p = i - k * P; } else { p = i / K9; k = i - p * K9; }
  const int tap = (int)(k / C), c = (int)(k - (int64_t)tap * C);
  const int ky = tap / 3, kx = tap - 3 * ky;
  const int x = (int)(p % W), y = (int)((p / W) % H); const int64_t n = p / ((int64_t)W * H);
  const int yy = y + ky - 1, xx = x + kx - 1;
  __nv_bfloat16 v = __float2bfloat16(0.0f);
  if (yy >= 0 && yy < H && xx >= 0 && xx < W) v = X[((n * H + yy) * W + xx) * Cs + c0 + c];
  col[i] = v;
}

// dX[n, y, x, c0 + c] = sum over the 9 taps of dCol[p'][(ky 3 + kx) C + c], p' = (n, y - ky + 1, x - kx + 1)
__global__ void k_col2im(const float* __restrict__ dcol, int Nb, int H, int W, int C, float* __restrict__ dX, int Cs,
                         int c0) {
  const int64_t P = (int64_t)Nb * H * W;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P * C) return;
  const int64_t p = i / C; const int c = (int)(i - p * C);
  const int x = (int)(p % W), y = (int)((p / W) % H); const int64_t n = p / ((int64_t)W * H);
  float acc = 0.0f;
#pragma unroll
  for (int ky = 0; ky < 3; ky++)
#pragma unroll
    for (int kx = 0; kx < 3; kx++) {
      const int yy = y - ky + 1, xx = x - kx + 1;
      if (yy < 0 || yy >= H || xx < 0 || xx >= W) continue;
      acc += dcol[((n * H + yy) * W + xx) * 9 * (int64_t)C + (ky * 3 + kx) * C + c];
    }
  dX[p * Cs + c0 + c] = acc;
}

// Y[p, c0 + n] = act(sum_z C[z][p][n] + bias[n]) in BF16 (split partials summed in order)
__global__ void k_bias_act(const float* __restrict__ Cm, int splits, int64_t P, int N, const float* __restrict__ bias,
                           int relu, __nv_bfloat16* __restrict__ Y, int Cs, int c0) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P * N) return;
  const int64_t p = i / N; const int n = (int)(i - p * N);
  float v = bias ? bias[n] : 0.0f;
  for (int z = 0; z < splits; z++) v += Cm[(size_t)z * P * N + i];
  if (relu) v = fmaxf(v, 0.0f);
  Y[p * Cs + c0 + n] = __float2bfloat16(v);
}

// through the ReLU: dPre = dY (Y > 0), BF16 in both [P x C] and [C x P] layouts
__global__ void k_relu_bwd(const float* __restrict__ dY, int Csd, int c0d, const __nv_bfloat16* __restrict__ Y, int Csy,
                           int c0y, int64_t P, int C, __nv_bfloat16* __restrict__ dpre, __nv_bfloat16* __restrict__ dpreT) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P * C) return;
  const int64_t p = i / C; const int c = (int)(i - p * C);
  const float y = __bfloat162float(Y[p * Csy + c0y + c]);
  const float d = y > 0.0f ? dY[p * Csd + c0d + c] : 0.0f;
  const __nv_bfloat16 b = __float2bfloat16(d);
  dpre[i] = b;
  dpreT[(int64_t)c * P + p] = b;
}

// bias gradient partials: part[chunk][c] = sum over the chunk's rows of dY (Y > 0); block = chunk, thread = channel
__global__ void k_bias_grad(const float* __restrict__ dY, int Csd, int c0d, const __nv_bfloat16* __restrict__ Y,
                            int Csy, int c0y, int64_t P, int C, int relu, float* __restrict__ part) {
  const int c = threadIdx.x;
  if (c >= C) return;
  const int64_t rows = (P + gridDim.x - 1) / gridDim.x;
  const int64_t p0 = (int64_t)blockIdx.x * rows, p1 = min(P, p0 + rows);
  float acc = 0.0f;
  for (int64_t p = p0; p < p1; p++) {
    const float d = dY[p * Csd + c0d + c];
    if (!relu || __bfloat162float(Y[p * Csy + c0y + c]) > 0.0f) acc += d;
  }
  part[(size_t)blockIdx.x * C + c] = acc;
}

// out[i] = sum_z in[z][i] (fixed order)
__global__ void k_sum_splits(const float* __restrict__ in, int splits, int64_t n, float* __restrict__ out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float v = 0.0f;
  for (int z = 0; z < splits; z++) v += in[(size_t)z * n + i];
  out[i] = v;
}

// 2 x 2 average pooling, NHWC slices: Y[n, y, x, c] = mean of X[n, 2y + a, 2x + b, c]
__global__ void k_pool_fwd(const __nv_bfloat16* __restrict__ X, int Nb, int H, int W, int Csx, int c0x, int C,
                           __nv_bfloat16* __restrict__ Y, int Csy, int c0y) {
  const int h = H / 2, w = W / 2;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (int64_t)Nb * h * w * C) return;
  const int c = (int)(i % C); const int64_t q = i / C;
  const int x = (int)(q % w), y = (int)((q / w) % h); const int64_t n = q / ((int64_t)w * h);
  float s = 0.0f;
  for (int a = 0; a < 2; a++)
    for (int b = 0; b < 2; b++) s += __bfloat162float(X[((n * H + 2 * y + a) * W + 2 * x + b) * Csx + c0x + c]);
  Y[q * Csy + c0y + c] = __float2bfloat16(0.25f * s);
}

// its gradient, added into dX (the encoder output's gradient also receives the skip path's)
__global__ void k_pool_bwd_add(const float* __restrict__ dY, int Nb, int H, int W, int C, float* __restrict__ dX,
                               int Csx, int c0x) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (int64_t)Nb * H * W * C) return;
  const int c = (int)(i % C); const int64_t q = i / C;
  const int x = (int)(q % W), y = (int)((q / W) % H); const int64_t n = q / ((int64_t)W * H);
  const int h = H / 2, w = W / 2;
  dX[q * Csx + c0x + c] += 0.25f * dY[((n * h + y / 2) * w + x / 2) * C + c];
}

// nearest-neighbour x2 upsampling into a channel slice, and its gradient (sum of the 4 copies)
__global__ void k_up_fwd(const __nv_bfloat16* __restrict__ X, int Nb, int h, int w, int C,
                         __nv_bfloat16* __restrict__ Y, int Csy, int c0y) {
  const int H = 2 * h, W = 2 * w;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (int64_t)Nb * H * W * C) return;
  const int c = (int)(i % C); const int64_t q = i / C;
  const int x = (int)(q % W), y = (int)((q / W) % H); const int64_t n = q / ((int64_t)W * H);
  Y[q * Csy + c0y + c] = X[((n * h + y / 2) * w + x / 2) * C + c];
}

__global__ void k_up_bwd(const float* __restrict__ dY, int Nb, int h, int w, int Csy, int c0y, int C,
                         float* __restrict__ dX) {
  const int H = 2 * h, W = 2 * w;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (int64_t)Nb * h * w * C) return;
  const int c = (int)(i % C); const int64_t q = i / C;
  const int x = (int)(q % w), y = (int)((q / w) % h); const int64_t n = q / ((int64_t)w * h);
  float s = 0.0f;
  for (int a = 0; a < 2; a++)
    for (int b = 0; b < 2; b++) s += dY[((n * H + 2 * y + a) * W + 2 * x + b) * Csy + c0y + c];
  dX[q * C + c] = s;
}

// the output head: a 1 x 1 convolution to Cout (<= 4) channels in FP32, forward and gradients
__global__ void k_head_fwd(const __nv_bfloat16* __restrict__ X, int64_t P, int Cin, const float* __restrict__ Wt,
                           const float* __restrict__ b, int Cout, float* __restrict__ Y) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P) return;
  for (int o = 0; o < Cout; o++) {
    float acc = b[o];
    for (int c = 0; c < Cin; c++) acc += Wt[o * Cin + c] * __bfloat162float(X[p * Cin + c]);
    Y[p * Cout + o] = acc;
  }
}

__global__ void k_head_bwd_data(const float* __restrict__ dY, int64_t P, int Cout, const float* __restrict__ Wt,
                                int Cin, float* __restrict__ dX) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P * Cin) return;
  const int64_t p = i / Cin; const int c = (int)(i - p * Cin);
  float acc = 0.0f;
  for (int o = 0; o < Cout; o++) acc += dY[p * Cout + o] * Wt[o * Cin + c];
  dX[i] = acc;
}

// head weight / bias gradient partials: part[chunk][o (Cin + 1) + c] (c = Cin: the bias); block = chunk
__global__ void k_head_bwd_weight(const float* __restrict__ dY, const __nv_bfloat16* __restrict__ X, int64_t P,
                                  int Cin, int Cout, float* __restrict__ part) {
  const int nq = Cout * (Cin + 1);
  const int64_t rows = (P + gridDim.x - 1) / gridDim.x;
  const int64_t p0 = (int64_t)blockIdx.x * rows, p1 = min(P, p0 + rows);
  for (int q = threadIdx.x; q < nq; q += blockDim.x) {
    const int o = q / (Cin + 1), c = q - o * (Cin + 1);
    float acc = 0.0f;
    for (int64_t p = p0; p < p1; p++)
      acc += dY[p * Cout + o] * (c < Cin ? __bfloat162float(X[p * Cin + c]) : 1.0f);
    part[(size_t)blockIdx.x * nq + q] = acc;
  }
}

// the phase- and conjugation-invariant loss per sample s (HW complex values u, target t):
//   l_s = min over (t, conj t) and a global phase of |u - e^{i th} t|^2 / |t|^2
//       = (|u|^2 + |t|^2 - 2 max(|<t, u>|, |<conj t, u>|)) / |t|^2
// stats[s] = [|u|^2, |t|^2, Re a, Im a, Re b, Im b] with a = sum conj(t) u, b = sum t u (one block per sample)
__global__ void k_loss_stats(const float* __restrict__ u, const float* __restrict__ t, int64_t HW,
                             double* __restrict__ stats) {
  const int s = blockIdx.x;
  const float* us = u + (size_t)s * HW * 2;
  const float* ts = t + (size_t)s * HW * 2;
  double v[6] = {0, 0, 0, 0, 0, 0};
  for (int64_t i = threadIdx.x; i < HW; i += blockDim.x) {
    const double ur = us[2 * i], ui = us[2 * i + 1], tr = ts[2 * i], ti = ts[2 * i + 1];
    v[0] += ur * ur + ui * ui; v[1] += tr * tr + ti * ti;
    v[2] += tr * ur + ti * ui; v[3] += tr * ui - ti * ur;       // conj(t) u
    v[4] += tr * ur - ti * ui; v[5] += tr * ui + ti * ur;       // t u
  }
  __shared__ double sh[6][32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int q = 0; q < 6; q++) {
    double x = warp_sum(v[q]);
    if (lane == 0) sh[q][wid] = x;
  }
  __syncthreads();
  if (wid == 0)
    for (int q = 0; q < 6; q++) {
      double x = lane < nw ? sh[q][lane] : 0.0;
      x = warp_sum(x);
      if (lane == 0) stats[s * 6 + q] = x;
    }
}

// loss[s] and du = dl_s / du / S (the batch mean), from the stats
__global__ void k_loss_grad(const float* __restrict__ u, const float* __restrict__ t, int64_t HW, int S,
                            const double* __restrict__ stats, float* __restrict__ du, double* __restrict__ loss) {
  const int s = blockIdx.y;
  const double* st = stats + s * 6;
  const double tt = fmax(st[1], 1e-300), am = hypot(st[2], st[3]), bm = hypot(st[4], st[5]);
  const bool cj = bm > am;
  const double m = cj ? bm : am;
  const double pr = m > 0 ? (cj ? st[4] : st[2]) / m : 1.0, pi = m > 0 ? (cj ? st[5] : st[3]) / m : 0.0;
  if (blockIdx.x == 0 && threadIdx.x == 0) loss[s] = (st[0] + st[1] - 2.0 * m) / tt;
  const double sc = 2.0 / (tt * S);
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < HW; i += (int64_t)gridDim.x * blockDim.x) {
    const size_t o = ((size_t)s * HW + i) * 2;
    const double ur = u[o], ui = u[o + 1], tr = t[o], ti = cj ? -t[o + 1] : t[o + 1];
    // the aligned target: conj branch uses conj(t); gradient of -2|<t', u>| is -2 t' (phase)
    const double gr = tr * pr - ti * pi, gi = tr * pi + ti * pr;
    du[o] = (float)(sc * (ur - gr));
    du[o + 1] = (float)(sc * (ui - gi));
  }
}

// Adam (bias-corrected) on FP32 master weights, with a BF16 copy and, for conv weights [Cout x K9], its BF16
// transpose [K9 x Cout]
__global__ void k_adam(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                       int64_t n, float lr, float b1, float b2, float eps, float c1, float c2,
                       __nv_bfloat16* __restrict__ wb, __nv_bfloat16* __restrict__ wbt, int rows, int cols) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.0f - b1) * gi, vi = b2 * v[i] + (1.0f - b2) * gi * gi;
  m[i] = mi; v[i] = vi;
  const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  w[i] = wi;
  if (wb) wb[i] = __float2bfloat16(wi);
  if (wbt) { const int64_t r = i / cols, c = i - r * cols; wbt[c * rows + r] = __float2bfloat16(wi); }
}

__global__ void k_to_bf16(const float* __restrict__ x, int64_t n, __nv_bfloat16* __restrict__ y,
                          __nv_bfloat16* __restrict__ yt, int rows, int cols) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const __nv_bfloat16 b = __float2bfloat16(x[i]);
  if (y) y[i] = b;
  if (yt) { const int64_t r = i / cols, c = i - r * cols; yt[c * rows + r] = b; }
}

// ----------------------------------------------------------------------------------------------------- host side
typedef CUresult (*NNEncodeFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                               const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                               CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static NNEncodeFn nn_encode() {
  static NNEncodeFn fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<NNEncodeFn>(p);
  }
  return fn;
}

// a BF16 [rows x K] K-major operand, box {64, box_rows}, 128-byte swizzle, zero fill outside
static int nn_map(CUtensorMap* m, const void* ptr, int64_t K, int64_t rows, int box_rows) {
  NNEncodeFn fn = nn_encode();
  if (!fn) { set_error("bf16 gemm: cuTensorMapEncodeTiled unavailable"); return BLML_ERR_CUDA; }
  if ((reinterpret_cast<uintptr_t>(ptr) & 15) || (K * 2) % 16) {
    set_error("bf16 gemm: operands need 16-byte aligned rows (K a multiple of 8)"); return BLML_ERR_ARG;
  }
  cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)(K * 2)};
  cuuint32_t box[2] = {(cuuint32_t)NN_BK, (cuuint32_t)box_rows};
  cuuint32_t es[2] = {1, 1};
  CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(ptr), dims, strides, box, es,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) { set_error("bf16 gemm: tensor map encoding failed (%d)", (int)r); return BLML_ERR_CUDA; }
  return BLML_OK;
}

static inline unsigned g1(int64_t n, int t = 256) { return (unsigned)((n + t - 1) / t); }

}  // namespace blml

using namespace blml;
#define NST reinterpret_cast<cudaStream_t>(stream)

extern "C" {

int blml_nn_gemm_bf16(const void* A, const void* B, float* C, int M, int N, int K, int splits, int* err,
                      void* stream) {
  if (!A || !B || !C || !err || M < 1 || N < 1 || K < 8 || splits < 1 || splits > 4096) {
    set_error("blml_nn_gemm_bf16: bad arguments"); return BLML_ERR_ARG;
  }
  // n tiles of equal width (a multiple of 16, at most 256: the MMA's N), so N = 288 is two tiles of 144, not 256 + 32
  const int ntiles = (N + 255) / 256;
  const int NT = ((N + ntiles - 1) / ntiles + 15) / 16 * 16;
  int tcols = 32; while (tcols < NT) tcols <<= 1;                 // two accumulators: 2 tcols <= 512 TMEM columns
  CUtensorMap mA, mB;
  int e = nn_map(&mA, A, K, M, NN_BM);
  if (!e) e = nn_map(&mB, B, K, N, NT);
  if (e) return e;
  const int nkb = (K + NN_BK - 1) / NN_BK;
  const int per = (nkb + splits - 1) / splits;
  // as many K slices in flight as the shared memory holds (at most 8); more than half of it, so one CTA per SM
  constexpr size_t kSmemMax = 227 * 1024;
  const size_t stage_bytes = (size_t)(NN_BM + NT) * NN_BK * 2;
  const size_t fixed = 1024 + sizeof(NNPipeShared);
  const int stages = (int)std::min<size_t>(NN_MAX_STAGES, (kSmemMax - fixed) / stage_bytes);
  const size_t smem = std::max<size_t>(fixed + (size_t)stages * stage_bytes, 120 * 1024);
  static bool attr = false;
  if (!attr) {
    e = cuda_status(cudaFuncSetAttribute(k_gemm_bf16, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemMax),
                    "blml_nn_gemm_bf16");
    if (e) return e;
    attr = true;
  }
  const long long tiles = (long long)((M + NN_BM - 1) / NN_BM) * ((N + NT - 1) / NT) * splits;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const unsigned grid = (unsigned)std::min<long long>(tiles, sms);
  k_gemm_bf16<<<grid, NN_PIPE_THREADS, smem, NST>>>(mA, mB, M, N, NT, tcols, nkb, per, splits, stages, C, err);
  BLML_CHECK_LAUNCH("blml_nn_gemm_bf16");
  return BLML_OK;
}

int blml_nn_im2col(const void* X, int Nb, int H, int W, int Cs, int c0, int C, void* col, int transposed,
                   void* stream) {
  if (!X || !col || Nb < 1 || H < 1 || W < 1 || C < 1 || c0 < 0 || c0 + C > Cs) {
    set_error("blml_nn_im2col: bad arguments"); return BLML_ERR_ARG;
  }
  const int64_t n = (int64_t)Nb * H * W * 9 * C;
  k_im2col<<<g1(n), 256, 0, NST>>>((const __nv_bfloat16*)X, Nb, H, W, Cs, c0, C, (__nv_bfloat16*)col, transposed);
  BLML_CHECK_LAUNCH("blml_nn_im2col");
  return BLML_OK;
}

int blml_nn_col2im(const float* dcol, int Nb, int H, int W, int C, float* dX, int Cs, int c0, void* stream) {
  if (!dcol || !dX || Nb < 1 || H < 1 || W < 1 || C < 1 || c0 < 0 || c0 + C > Cs) {
    set_error("blml_nn_col2im: bad arguments"); return BLML_ERR_ARG;
  }
  k_col2im<<<g1((int64_t)Nb * H * W * C), 256, 0, NST>>>(dcol, Nb, H, W, C, dX, Cs, c0);
  BLML_CHECK_LAUNCH("blml_nn_col2im");
  return BLML_OK;
}

int blml_nn_bias_act(const float* Cm, int splits, int64_t P, int N, const float* bias, int relu, void* Y, int Cs,
                     int c0, void* stream) {
  if (!Cm || !Y || P < 1 || N < 1 || splits < 1 || c0 < 0 || c0 + N > Cs) {
    set_error("blml_nn_bias_act: bad arguments"); return BLML_ERR_ARG;
  }
  k_bias_act<<<g1(P * N), 256, 0, NST>>>(Cm, splits, P, N, bias, relu, (__nv_bfloat16*)Y, Cs, c0);
  BLML_CHECK_LAUNCH("blml_nn_bias_act");
  return BLML_OK;
}

int blml_nn_relu_bwd(const float* dY, int Csd, int c0d, const void* Y, int Csy, int c0y, int64_t P, int C,
                     void* dpre, void* dpreT, void* stream) {
  if (!dY || !Y || !dpre || !dpreT || P < 1 || C < 1) { set_error("blml_nn_relu_bwd: bad arguments"); return BLML_ERR_ARG; }
  k_relu_bwd<<<g1(P * C), 256, 0, NST>>>(dY, Csd, c0d, (const __nv_bfloat16*)Y, Csy, c0y, P, C,
                                         (__nv_bfloat16*)dpre, (__nv_bfloat16*)dpreT);
  BLML_CHECK_LAUNCH("blml_nn_relu_bwd");
  return BLML_OK;
}

// db[c] = sum_p dY[p, c] (Y > 0 when relu); part: chunks x C floats
int blml_nn_bias_grad(const float* dY, int Csd, int c0d, const void* Y, int Csy, int c0y, int64_t P, int C, int relu,
                      int chunks, float* part, float* db, void* stream) {
  if (!dY || !part || !db || P < 1 || C < 1 || C > 1024 || chunks < 1 || (relu && !Y)) {
    set_error("blml_nn_bias_grad: bad arguments"); return BLML_ERR_ARG;
  }
  k_bias_grad<<<chunks, ((C + 31) / 32) * 32, 0, NST>>>(dY, Csd, c0d, (const __nv_bfloat16*)Y, Csy, c0y, P, C, relu,
                                                        part);
  BLML_CHECK_LAUNCH("blml_nn_bias_grad");
  k_sum_splits<<<g1(C), 256, 0, NST>>>(part, chunks, C, db);
  BLML_CHECK_LAUNCH("blml_nn_bias_grad finish");
  return BLML_OK;
}

int blml_nn_sum_splits(const float* in, int splits, int64_t n, float* out, void* stream) {
  if (!in || !out || splits < 1 || n < 1) { set_error("blml_nn_sum_splits: bad arguments"); return BLML_ERR_ARG; }
  k_sum_splits<<<g1(n), 256, 0, NST>>>(in, splits, n, out);
  BLML_CHECK_LAUNCH("blml_nn_sum_splits");
  return BLML_OK;
}

int blml_nn_pool_fwd(const void* X, int Nb, int H, int W, int Csx, int c0x, int C, void* Y, int Csy, int c0y,
                     void* stream) {
  if (!X || !Y || (H & 1) || (W & 1) || C < 1) { set_error("blml_nn_pool_fwd: bad arguments"); return BLML_ERR_ARG; }
  k_pool_fwd<<<g1((int64_t)Nb * (H / 2) * (W / 2) * C), 256, 0, NST>>>((const __nv_bfloat16*)X, Nb, H, W, Csx, c0x, C,
                                                                        (__nv_bfloat16*)Y, Csy, c0y);
  BLML_CHECK_LAUNCH("blml_nn_pool_fwd");
  return BLML_OK;
}

int blml_nn_pool_bwd_add(const float* dY, int Nb, int H, int W, int C, float* dX, int Csx, int c0x, void* stream) {
  if (!dY || !dX || (H & 1) || (W & 1) || C < 1) { set_error("blml_nn_pool_bwd_add: bad arguments"); return BLML_ERR_ARG; }
  k_pool_bwd_add<<<g1((int64_t)Nb * H * W * C), 256, 0, NST>>>(dY, Nb, H, W, C, dX, Csx, c0x);
  BLML_CHECK_LAUNCH("blml_nn_pool_bwd_add");
  return BLML_OK;
}

int blml_nn_up_fwd(const void* X, int Nb, int h, int w, int C, void* Y, int Csy, int c0y, void* stream) {
  if (!X || !Y || C < 1) { set_error("blml_nn_up_fwd: bad arguments"); return BLML_ERR_ARG; }
  k_up_fwd<<<g1((int64_t)Nb * 4 * h * w * C), 256, 0, NST>>>((const __nv_bfloat16*)X, Nb, h, w, C,
                                                              (__nv_bfloat16*)Y, Csy, c0y);
  BLML_CHECK_LAUNCH("blml_nn_up_fwd");
  return BLML_OK;
}

int blml_nn_up_bwd(const float* dY, int Nb, int h, int w, int Csy, int c0y, int C, float* dX, void* stream) {
  if (!dY || !dX || C < 1) { set_error("blml_nn_up_bwd: bad arguments"); return BLML_ERR_ARG; }
  k_up_bwd<<<g1((int64_t)Nb * h * w * C), 256, 0, NST>>>(dY, Nb, h, w, Csy, c0y, C, dX);
  BLML_CHECK_LAUNCH("blml_nn_up_bwd");
  return BLML_OK;
}

int blml_nn_head_fwd(const void* X, int64_t P, int Cin, const float* Wt, const float* b, int Cout, float* Y,
                     void* stream) {
  if (!X || !Wt || !b || !Y || Cout < 1 || Cout > 4) { set_error("blml_nn_head_fwd: bad arguments"); return BLML_ERR_ARG; }
  k_head_fwd<<<g1(P), 256, 0, NST>>>((const __nv_bfloat16*)X, P, Cin, Wt, b, Cout, Y);
  BLML_CHECK_LAUNCH("blml_nn_head_fwd");
  return BLML_OK;
}

// dX = dY W; dW, db from chunked partials (part: chunks x Cout (Cin + 1) floats) into gw [Cout (Cin + 1)]
int blml_nn_head_bwd(const float* dY, const void* X, int64_t P, int Cin, int Cout, const float* Wt, float* dX,
                     int chunks, float* part, float* gw, void* stream) {
  if (!dY || !X || !Wt || !part || !gw || Cout < 1 || Cout > 4 || chunks < 1) {
    set_error("blml_nn_head_bwd: bad arguments"); return BLML_ERR_ARG;
  }
  if (dX) {
    k_head_bwd_data<<<g1(P * Cin), 256, 0, NST>>>(dY, P, Cout, Wt, Cin, dX);
    BLML_CHECK_LAUNCH("blml_nn_head_bwd");
  }
  k_head_bwd_weight<<<chunks, 256, 0, NST>>>(dY, (const __nv_bfloat16*)X, P, Cin, Cout, part);
  BLML_CHECK_LAUNCH("blml_nn_head_bwd");
  k_sum_splits<<<g1((int64_t)Cout * (Cin + 1)), 256, 0, NST>>>(part, chunks, (int64_t)Cout * (Cin + 1), gw);
  BLML_CHECK_LAUNCH("blml_nn_head_bwd");
  return BLML_OK;
}

// loss[s] and du for S samples of HW complex values (interleaved FP32); stats: 6 S doubles
int blml_nn_phase_loss(const float* u, const float* t, int64_t HW, int S, double* stats, float* du, double* loss,
                       void* stream) {
  if (!u || !t || !stats || !du || !loss || HW < 1 || S < 1 || S > 65535) {
    set_error("blml_nn_phase_loss: bad arguments"); return BLML_ERR_ARG;
  }
  k_loss_stats<<<S, 256, 0, NST>>>(u, t, HW, stats);
  BLML_CHECK_LAUNCH("blml_nn_phase_loss");
  k_loss_grad<<<dim3(g1(HW), (unsigned)S), 256, 0, NST>>>(u, t, HW, S, stats, du, loss);
  BLML_CHECK_LAUNCH("blml_nn_phase_loss");
  return BLML_OK;
}

int blml_nn_adam(float* w, const float* g, float* m, float* v, int64_t n, float lr, float b1, float b2, float eps,
                 int step, void* wb, void* wbt, int rows, int cols, void* stream) {
  if (!w || !g || !m || !v || n < 1 || step < 1 || (wbt && (int64_t)rows * cols != n)) {
    set_error("blml_nn_adam: bad arguments"); return BLML_ERR_ARG;
  }
  const float c1 = 1.0f - powf(b1, (float)step), c2 = 1.0f - powf(b2, (float)step);
  k_adam<<<g1(n), 256, 0, NST>>>(w, g, m, v, n, lr, b1, b2, eps, c1, c2, (__nv_bfloat16*)wb, (__nv_bfloat16*)wbt,
                                 rows, cols);
  BLML_CHECK_LAUNCH("blml_nn_adam");
  return BLML_OK;
}

int blml_nn_to_bf16(const float* x, int64_t n, void* y, void* yt, int rows, int cols, void* stream) {
  if (!x || n < 1 || (yt && (int64_t)rows * cols != n)) { set_error("blml_nn_to_bf16: bad arguments"); return BLML_ERR_ARG; }
  k_to_bf16<<<g1(n), 256, 0, NST>>>(x, n, (__nv_bfloat16*)y, (__nv_bfloat16*)yt, rows, cols);
  BLML_CHECK_LAUNCH("blml_nn_to_bf16");
  return BLML_OK;
}

}
