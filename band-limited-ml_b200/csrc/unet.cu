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
// 128-byte-swizzled 64-deep K slices, one elected thread issuing kind::f16 MMAs (M 128, N <= 256, K 16) into a TMEM
// accumulator, tcgen05.ld epilogue. Waits are bounded: on timeout the kernel sets the caller's error word, gives
// copies and MMAs in flight one more bounded wait, frees its tensor memory and returns.
#include <cuda.h>
#include <cuda_bf16.h>
#include <string.h>
#include <vector>
#include "common.cuh"

namespace blml {

constexpr int NN_BM = 128, NN_BK = 64, NN_THREADS = 128;

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

// C[z][m][n] = sum_{k in split z} A[m][k] B[n][k]. Persistent: at most 2 CTAs per SM (their TMEM accumulators fit
// the SM's 512 columns together), each allocating its accumulator once and walking the tiles (m tile, n tile, split)
// t = blockIdx.x, blockIdx.x + gridDim.x, ...; between tiles the epilogue's reads finish before the next tile's
// first MMA overwrites the accumulator.
__global__ void __launch_bounds__(NN_THREADS) k_gemm_bf16(const __grid_constant__ CUtensorMap mA,
                                                          const __grid_constant__ CUtensorMap mB, int M, int N,
                                                          int NT, int tcols, int nkb, int kb_per_split, int splits,
                                                          float* C, int* err) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  __nv_bfloat16* sA = reinterpret_cast<__nv_bfloat16*>(base);
  __nv_bfloat16* sB = sA + NN_BM * NN_BK;
  uint64_t* bars = reinterpret_cast<uint64_t*>(sB + (size_t)NT * NN_BK);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + 2);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int Mt = (M + NN_BM - 1) / NN_BM, Nt = (N + NT - 1) / NT;
  const long long tiles = (long long)Mt * Nt * splits;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" :: "r"(nn_smem_u32(tslot)), "r"(tcols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    nn_mbar_init(&bars[0], 1); nn_mbar_init(&bars[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t taddr = *tslot;
  const uint32_t tx = (uint32_t)((NN_BM + NT) * NN_BK * 2);
  const uint32_t idesc = idesc_bf16(NT);
  bool ok = true;
  uint32_t par_last = 0;
  long long phase = 0;                         // mbarrier phases used so far (both barriers advance together)
  for (long long t = blockIdx.x; t < tiles && ok; t += gridDim.x) {
    const int z = (int)(t / ((long long)Mt * Nt));
    const long long rem = t - (long long)z * Mt * Nt;
    const int nt_i = (int)(rem / Mt), mt_i = (int)(rem - (long long)nt_i * Mt);
    const int m0 = mt_i * NN_BM, n0 = nt_i * NT;
    const int kb0 = z * kb_per_split, kb1 = min(nkb, kb0 + kb_per_split);
    int done = 0;
    for (int kb = kb0; kb < kb1 && ok; kb++, done++, phase++) {
      const uint32_t par = (uint32_t)(phase & 1);
      par_last = par;
      if (tid == 0) {
        nn_mbar_expect_tx(&bars[0], tx);
        nn_tma_2d(sA, &mA, kb * NN_BK, m0, &bars[0]);
        nn_tma_2d(sB, &mB, kb * NN_BK, n0, &bars[0]);
      }
      ok = nn_mbar_wait(&bars[0], par);
      if (!ok) break;
      if (tid == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
        for (int j = 0; j < NN_BK / 16; j++) {
          const uint64_t ad = nn_desc(sA + j * 16), bd = nn_desc(sB + j * 16);
          const uint32_t acc = (done > 0 || j > 0) ? 1u : 0u;
          asm volatile("{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                       " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n"
                       :: "r"(taddr), "l"(ad), "l"(bd), "r"(idesc), "r"(acc));
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                     :: "r"(nn_smem_u32(&bars[1])) : "memory");
      }
      ok = nn_mbar_wait(&bars[1], par);
    }
    if (!ok) break;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    float* Cz = C + (size_t)z * M * N;
    const int row = m0 + 32 * warp + lane;
    for (int c0 = 0; c0 < NT; c0 += 16) {
      uint32_t v[16];
      if (done > 0) {
        asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
                     "%13, %14, %15}, [%16];"
                     : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                       "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
                       "=r"(v[15])
                     : "r"(taddr + ((uint32_t)(32 * warp) << 16) + (uint32_t)c0));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      } else {
#pragma unroll
        for (int i = 0; i < 16; i++) v[i] = 0u;            // an empty K range: the partial is zero
      }
      if (row < M) {
#pragma unroll
        for (int i = 0; i < 16; i++) {
          const int col = n0 + c0 + i;
          if (col < N) Cz[(size_t)row * N + col] = __uint_as_float(v[i]);
        }
      }
    }
    // every warp's accumulator reads are done before thread 0 issues the next tile's first MMA
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  }
  if (!ok) {
    // a bounded wait gave up: record it, then give the copy and the MMAs in flight one more bounded wait before the
    // tensor memory is released
    if (tid == 0) atomicExch(err, 1);
    nn_mbar_wait(&bars[0], par_last);
    nn_mbar_wait(&bars[1], par_last);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(taddr), "r"(tcols));
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
  const int NT = N <= 256 ? (N + 15) / 16 * 16 : 256;
  int tcols = 32; while (tcols < NT) tcols <<= 1;
  CUtensorMap mA, mB;
  int e = nn_map(&mA, A, K, M, NN_BM);
  if (!e) e = nn_map(&mB, B, K, N, NT);
  if (e) return e;
  const int nkb = (K + NN_BK - 1) / NN_BK;
  const int per = (nkb + splits - 1) / splits;
  // shared memory sized so at most 2 CTAs share an SM (their TMEM accumulators then always fit its 512 columns)
  const size_t smem = std::max<size_t>(1024 + (size_t)(NN_BM + NT) * NN_BK * 2 + 64, 80 * 1024);
  static bool attr = false;
  if (!attr) {
    e = cuda_status(cudaFuncSetAttribute(k_gemm_bf16, cudaFuncAttributeMaxDynamicSharedMemorySize, 80 * 1024),
                    "blml_nn_gemm_bf16");
    if (e) return e;
    attr = true;
  }
  const long long tiles = (long long)((M + NN_BM - 1) / NN_BM) * ((N + NT - 1) / NT) * splits;
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0);
  const unsigned grid = (unsigned)std::min<long long>(tiles, 2LL * sms);    // 2 CTAs per SM: TMEM 2 x 256 columns
  k_gemm_bf16<<<grid, NN_THREADS, smem, NST>>>(mA, mB, M, N, NT, tcols, nkb, per, splits, C, err);
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
