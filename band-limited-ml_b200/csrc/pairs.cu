// Pair accumulation over occupied lattice bins from the product kernel's value tables:
//     rows:  s_r = sum_j w_j prod_u T_u[idx_u(ZA_r, ZB_j)]   (+ d/dtheta rows with grad)
//     cols:  out[r, j] = prod_u T_u[idx_u(ZA_r, ZB_j)]
// Every CTA keeps the value tables in shared memory and streams the columns j in chunks (coordinates and weights
// staged in shared memory, read as warp broadcasts). Each thread owns rows; products are in REAL (float or
// double, the reference's f32 flag), sums in float64. Column slices of one row block are reduced in a fixed order
// by a second kernel, so results are deterministic (the reference combines slices with float64 atomics).
// Before any launch the coordinates are checked against the tables' extents on the device, so a stale table is an
// error, never an out-of-range read.
#include <mutex>
#include <cuda.h>
#include "common.cuh"

namespace blml {

constexpr int RQ = 4;               // radial rows: grid points per lattice step (linear interpolation)
constexpr int PR_THREADS = 128;     // rows per CTA (one per thread)
constexpr int PR_CHUNK = 256;       // columns staged per shared-memory chunk
constexpr int MAXD = 8, MAXU = 8, MAXG = 4, MAXW = 8;

struct ColMeta {
  int d, U, G, nW, LR;
  int code[MAXD], grp[MAXD], dim_unit[MAXD];
  int64_t base[MAXD], J[MAXD], mk[MAXD], nb[MAXD];
  int grp_unit[MAXG];
  int wunit[MAXW], wcol[MAXW], wgrp[MAXW];
  int64_t dbase[MAXW];
  int64_t Tn, dTn;
};

template <typename REAL>
__device__ __forceinline__ REAL col_value(const ColMeta& cm, const REAL* T, int k, int64_t za, int64_t zb) {
  const int code = cm.code[k];
  int64_t idx;
  if (code == 0) idx = cm.base[k] + za - zb + cm.J[k];
  else if (code == 3) idx = cm.base[k] + za * cm.mk[k] + zb;
  else {                                     // circular distance, |za - zb| < nb
    const int64_t nb = cm.nb[k];
    int64_t m = za - zb;
    if (m < 0) m += nb; else if (m >= nb) m -= nb;
    if (m > nb - m) m = nb - m;
    idx = cm.base[k] + m;
  }
  return T[idx];
}

// One pair's unit factors (fac[u]) and the group indices (r2 / torus index per group).
template <typename REAL>
__device__ __forceinline__ void pair_factors(const ColMeta& cm, const REAL* T, const REAL* RT, const int64_t* za,
                                             const int64_t* zb, REAL* fac, int64_t* r2, bool* tor) {
  for (int g = 0; g < cm.G; g++) { r2[g] = 0; tor[g] = false; }
  for (int k = 0; k < cm.d; k++) {
    const int code = cm.code[k];
    const int64_t off = za[k] - zb[k];
    if (code == 2) { r2[cm.grp[k]] += off * off; continue; }
    if (code == 4) {
      const int g = cm.grp[k]; const int64_t nb = cm.nb[k];
      const int64_t m = off < 0 ? off + nb : off;
      r2[g] = r2[g] * nb + m; tor[g] = true; continue;
    }
    fac[cm.dim_unit[k]] = col_value(cm, T, k, za[k], zb[k]);
  }
  for (int g = 0; g < cm.G; g++) {
    const REAL* row = RT + (int64_t)g * cm.LR;
    if (tor[g]) { fac[cm.grp_unit[g]] = row[r2[g]]; continue; }
    const double t = sqrt((double)r2[g]) * RQ; const int i0 = (int)t; const REAL f = (REAL)(t - i0);
    fac[cm.grp_unit[g]] = row[i0] * (REAL(1) - f) + row[i0 + 1] * f;
  }
}

// derivative entry q of a pair (the reference's dval): a column's derivative row (raw offsets, rank tables), a
// group's torus row, or a radial row on the r grid times the offset of column wcol[q] for a shift entry
template <typename REAL>
__device__ __forceinline__ REAL dval(const ColMeta& cm, const REAL* dT, const REAL* dR, int q, const int64_t* za,
                                     const int64_t* zb, const int64_t* r2, const bool* tor) {
  const int g = cm.wgrp[q], k = cm.wcol[q];
  if (g >= 0 && tor[g]) return dR[(int64_t)q * cm.LR + r2[g]];
  if (g < 0) {
    const int64_t idx = cm.code[k] == 3 ? za[k] * cm.mk[k] + zb[k] : za[k] - zb[k] + cm.J[k];
    return dT[cm.dbase[q] + idx];
  }
  const double t = sqrt((double)r2[g]) * RQ; const int i0 = (int)t; const REAL f = (REAL)(t - i0);
  REAL v = dR[(int64_t)q * cm.LR + i0] * (REAL(1) - f) + dR[(int64_t)q * cm.LR + i0 + 1] * f;
  if (k >= 0) v *= (REAL)(za[k] - zb[k]);
  return v;
}

// General rows kernel: any column codes, groups and derivative entries. grid (row blocks, column slices).
// part[slice][r] (and dpart[slice][r][q]) are the slice sums.
template <typename REAL, bool GRAD>
__global__ void __launch_bounds__(PR_THREADS) k_rows_general(ColMeta cm, const REAL* Tg, const REAL* RTg,
                                                             const REAL* dTg, const REAL* dRg, const int64_t* ZA,
                                                             int64_t R, const int64_t* ZB, const double* w,
                                                             int64_t j0s, int64_t slice, int64_t M, double* part,
                                                             double* dpart) {
  extern __shared__ unsigned char smem_raw[];
  REAL* Ts = reinterpret_cast<REAL*>(smem_raw);
  REAL* RTs = Ts + cm.Tn;
  const int64_t nRT = (int64_t)cm.G * cm.LR;
  for (int64_t i = threadIdx.x; i < cm.Tn; i += blockDim.x) Ts[i] = Tg[i];
  for (int64_t i = threadIdx.x; i < nRT; i += blockDim.x) RTs[i] = RTg[i];
  __syncthreads();
  const int64_t r = (int64_t)blockIdx.x * PR_THREADS + threadIdx.x;
  const int64_t j0 = j0s + (int64_t)blockIdx.y * slice, j1 = min(M, j0 + slice);
  int64_t za[MAXD];
  const bool live = r < R;
  for (int k = 0; k < cm.d; k++) za[k] = live ? ZA[r * cm.d + k] : 0;
  double acc = 0.0, dacc[MAXW];
  for (int q = 0; q < MAXW; q++) dacc[q] = 0.0;
  REAL fac[MAXU + 1];
  for (int u = 0; u < MAXU; u++) fac[u] = REAL(1);
  int64_t r2[MAXG]; bool tor[MAXG];
  for (int64_t j = j0; j < j1 && live; j++) {
    const double wj = w[j];
    if (wj == 0.0) continue;
    int64_t zb[MAXD];
    for (int k = 0; k < cm.d; k++) zb[k] = ZB[j * cm.d + k];
    pair_factors<REAL>(cm, Ts, RTs, za, zb, fac, r2, tor);
    REAL pre[MAXU + 1];
    pre[0] = REAL(1);
    for (int u = 0; u < cm.U; u++) pre[u + 1] = pre[u] * fac[u];
    acc += (double)pre[cm.U] * wj;
    if (GRAD) {
      REAL suf[MAXU + 1];
      suf[cm.U] = REAL(1);
      for (int u = cm.U - 1; u >= 0; u--) suf[u] = suf[u + 1] * fac[u];
      for (int q = 0; q < cm.nW; q++) {
        const int u = cm.wunit[q];
        const REAL dv = dval<REAL>(cm, dTg, dRg, q, za, zb, r2, tor);
        dacc[q] += (double)(dv * pre[u] * suf[u + 1]) * wj;
      }
    }
  }
  if (!live) return;
  part[(int64_t)blockIdx.y * R + r] = acc;
  if (GRAD)
    for (int q = 0; q < cm.nW; q++) dpart[((int64_t)blockIdx.y * R + r) * cm.nW + q] = dacc[q];
}

// Fused rows of several densities over the same pairs (blml_local.py:213-286, rows_multi): s[r][m] = sum_j W[j][m]
// prod_u (bit u of umask[m] ? fac_u : 1), the unit factors computed once per pair and each density multiplying the
// units its mask keeps, in unit order (the joint: every unit; a marginal: the units of its columns). part[slice][r][m].
constexpr int MAXM = 8;
struct DensMasks { unsigned bits[MAXM]; };

template <typename REAL>
__global__ void __launch_bounds__(PR_THREADS) k_rows_multi(ColMeta cm, const REAL* Tg, const REAL* RTg,
                                                           const int64_t* ZA, int64_t R, const int64_t* ZB,
                                                           const double* W, int Mm, DensMasks dm, int64_t slice,
                                                           int64_t M, double* part) {
  extern __shared__ unsigned char smem_raw[];
  REAL* Ts = reinterpret_cast<REAL*>(smem_raw);
  REAL* RTs = Ts + cm.Tn;
  const int64_t nRT = (int64_t)cm.G * cm.LR;
  for (int64_t i = threadIdx.x; i < cm.Tn; i += blockDim.x) Ts[i] = Tg[i];
  for (int64_t i = threadIdx.x; i < nRT; i += blockDim.x) RTs[i] = RTg[i];
  __syncthreads();
  const int64_t r = (int64_t)blockIdx.x * PR_THREADS + threadIdx.x;
  const int64_t j0 = (int64_t)blockIdx.y * slice, j1 = min(M, j0 + slice);
  int64_t za[MAXD];
  const bool live = r < R;
  for (int k = 0; k < cm.d; k++) za[k] = live ? ZA[r * cm.d + k] : 0;
  double acc[MAXM];
  for (int m = 0; m < MAXM; m++) acc[m] = 0.0;
  REAL fac[MAXU + 1];
  for (int u = 0; u < MAXU; u++) fac[u] = REAL(1);
  int64_t r2[MAXG]; bool tor[MAXG];
  for (int64_t j = j0; j < j1 && live; j++) {
    int64_t zb[MAXD];
    for (int k = 0; k < cm.d; k++) zb[k] = ZB[j * cm.d + k];
    pair_factors<REAL>(cm, Ts, RTs, za, zb, fac, r2, tor);
    for (int m = 0; m < Mm; m++) {
      const double wj = W[j * Mm + m];
      if (wj == 0.0) continue;
      REAL p = REAL(1);
      for (int u = 0; u < cm.U; u++) p = p * (((dm.bits[m] >> u) & 1u) ? fac[u] : REAL(1));
      acc[m] += (double)p * wj;
    }
  }
  if (!live) return;
  for (int m = 0; m < Mm; m++) part[((int64_t)blockIdx.y * R + r) * Mm + m] = acc[m];
}

// shared-memory layout of k_rows_offset (the host sizes the launch with the same functions): the table, then the
// chunk's column coordinates (int32, D per column), then its weights, each part 16-byte aligned
__host__ __device__ constexpr size_t align16(size_t b) { return (b + 15) & ~(size_t)15; }
template <typename REAL> __host__ __device__ constexpr size_t offset_smem_zb(int64_t Tn) {
  return align16((size_t)Tn * sizeof(REAL));
}
template <typename REAL> __host__ __device__ constexpr size_t offset_smem_w(int64_t Tn, int D) {
  return offset_smem_zb<REAL>(Tn) + align16((size_t)PR_CHUNK * D * sizeof(int));
}
template <typename REAL> __host__ __device__ constexpr size_t offset_smem_bytes(int64_t Tn, int D) {
  return offset_smem_w<REAL>(Tn, D) + (size_t)PR_CHUNK * sizeof(double);
}

// Fast rows kernel for product kernels whose columns are all offset rows (sinc / slits / raw dirichlet): each
// thread keeps one pointer per column into the shared-memory table (T_k + base_k + J_k + za_k), so a pair costs
// D shared-memory gathers, D - 1 multiplies and one float64 FMA; column coordinates (int32) and weights are staged
// per chunk and read as broadcasts.
template <typename REAL, int D>
__global__ void __launch_bounds__(PR_THREADS) k_rows_offset(ColMeta cm, const REAL* Tg, const int64_t* ZA, int64_t R,
                                                            const int64_t* ZB, const double* w, int64_t slice,
                                                            int64_t M, double* part) {
  extern __shared__ unsigned char smem_raw[];
  REAL* Ts = reinterpret_cast<REAL*>(smem_raw);
  int* zbs = reinterpret_cast<int*>(smem_raw + offset_smem_zb<REAL>(cm.Tn));
  double* ws = reinterpret_cast<double*>(smem_raw + offset_smem_w<REAL>(cm.Tn, D));
  for (int64_t i = threadIdx.x; i < cm.Tn; i += blockDim.x) Ts[i] = Tg[i];
  const int64_t r = (int64_t)blockIdx.x * PR_THREADS + threadIdx.x;
  const bool live = r < R;
  const REAL* ptr[D];
#pragma unroll
  for (int k = 0; k < D; k++) ptr[k] = Ts + cm.base[k] + cm.J[k] + (live ? ZA[r * D + k] : 0);
  const int64_t j0 = (int64_t)blockIdx.y * slice, j1 = min(M, j0 + slice);
  double acc = 0.0;
  for (int64_t c0 = j0; c0 < j1; c0 += PR_CHUNK) {
    const int n = (int)(j1 - c0 < PR_CHUNK ? j1 - c0 : PR_CHUNK);
    __syncthreads();
    for (int i = threadIdx.x; i < n * D; i += blockDim.x) zbs[i] = (int)ZB[c0 * D + i];
    for (int i = threadIdx.x; i < n; i += blockDim.x) ws[i] = w[c0 + i];
    __syncthreads();
    if (live) {
#pragma unroll 4
      for (int jj = 0; jj < n; jj++) {
        REAL p = ptr[0][-zbs[jj * D]];
#pragma unroll
        for (int k = 1; k < D; k++) p *= ptr[k][-zbs[jj * D + k]];
        acc = fma((double)p, ws[jj], acc);
      }
    }
  }
  if (live) part[(int64_t)blockIdx.y * R + r] = acc;
}

__global__ void k_sum_slices(const double* part, int nsl, int64_t n, double* out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int y = 0; y < nsl; y++) s += part[(int64_t)y * n + i];
    out[i] = s;
  }
}

// out[r, j] = S(ZA_r, ZB_j); with out_m, also the product over the units whose bit in dep_units is clear (the
// marginal of the columns outside the dep mask, from the same lookups)
template <typename REAL, typename OUT>
__global__ void k_cols(ColMeta cm, const REAL* T, const REAL* RT, const int64_t* ZA, int64_t R, const int64_t* ZB,
                       int64_t M, OUT* out, OUT* out_m, unsigned dep_units) {
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < R * M;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = idx / M, j = idx % M;
    int64_t za[MAXD], zb[MAXD], r2[MAXG]; bool tor[MAXG];
    REAL fac[MAXU];
    for (int u = 0; u < MAXU; u++) fac[u] = REAL(1);
    for (int k = 0; k < cm.d; k++) { za[k] = ZA[r * cm.d + k]; zb[k] = ZB[j * cm.d + k]; }
    pair_factors<REAL>(cm, T, RT, za, zb, fac, r2, tor);
    REAL v = REAL(1), vdep = REAL(1);
    for (int u = 0; u < cm.U; u++) {
      if ((dep_units >> u) & 1u) vdep *= fac[u];
      else v *= fac[u];
    }
    out[idx] = (OUT)(v * vdep);
    if (out_m) out_m[idx] = (OUT)v;
  }
}

// lattice coordinates of bin centres: round(Z / h) in float64, ties to even (np.round's rule, so bit-exact with it)
__global__ void k_lattice_coords(const double* Z, int64_t n, int d, const double* h, int64_t* out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n * d; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = (int64_t)rint(Z[i] / h[i % d]);
}

// per column: min and max of ZA and ZB (for the extent check); out[4 * k + {0,1,2,3}] = minA, maxA, minB, maxB
__global__ void k_coord_range(const int64_t* ZA, int64_t R, const int64_t* ZB, int64_t M, int d, long long* out) {
  const int k = blockIdx.x;
  long long mnA = LLONG_MAX, mxA = LLONG_MIN, mnB = LLONG_MAX, mxB = LLONG_MIN;
  for (int64_t i = threadIdx.x; i < R; i += blockDim.x) { long long v = ZA[i * d + k]; mnA = min(mnA, v); mxA = max(mxA, v); }
  for (int64_t i = threadIdx.x; i < M; i += blockDim.x) { long long v = ZB[i * d + k]; mnB = min(mnB, v); mxB = max(mxB, v); }
  __shared__ long long sh[4][256];
  sh[0][threadIdx.x] = mnA; sh[1][threadIdx.x] = mxA; sh[2][threadIdx.x] = mnB; sh[3][threadIdx.x] = mxB;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) {
      sh[0][threadIdx.x] = min(sh[0][threadIdx.x], sh[0][threadIdx.x + s]);
      sh[1][threadIdx.x] = max(sh[1][threadIdx.x], sh[1][threadIdx.x + s]);
      sh[2][threadIdx.x] = min(sh[2][threadIdx.x], sh[2][threadIdx.x + s]);
      sh[3][threadIdx.x] = max(sh[3][threadIdx.x], sh[3][threadIdx.x + s]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) for (int q = 0; q < 4; q++) out[4 * k + q] = sh[q][0];
}

}  // namespace blml

using namespace blml;

static int read_meta(const blml_tables* tb, ColMeta& cm, cudaStream_t st) {
  if (!tb || tb->d < 1 || tb->d > MAXD || tb->U < 1 || tb->U > MAXU || tb->G < 0 || tb->G > MAXG || tb->nW < 0 ||
      tb->nW > MAXW) {
    set_error("pair tables: d <= %d, units <= %d, groups <= %d, derivative entries <= %d", MAXD, MAXU, MAXG, MAXW);
    return BLML_ERR_ARG;
  }
  const int d = tb->d;
  cm.d = d; cm.U = tb->U; cm.G = tb->G; cm.nW = tb->nW; cm.LR = tb->LR;
  cm.Tn = tb->nT; cm.dTn = tb->ndT;
  auto fetch = [&](const int64_t* src, int n, int64_t* dst) -> int {
    if (n == 0) return BLML_OK;
    return cuda_status(cudaMemcpyAsync(dst, src, n * sizeof(int64_t), cudaMemcpyDeviceToHost, st), "pair tables");
  };
  int64_t base[MAXD], J[MAXD], mk[MAXD], nb[MAXD], grp[MAXD], du[MAXD], gu[MAXG], wu[MAXW], wc[MAXW], wg[MAXW], db[MAXW];
  int64_t codes[MAXD];
  struct { const int64_t* s; int n; int64_t* d; } req[] = {
      {tb->kinds, d, codes}, {tb->base, d, base}, {tb->Jk, d, J}, {tb->mk, d, mk}, {tb->nbins, d, nb},
      {tb->grp, d, grp}, {tb->dim_unit, d, du}, {tb->grp_unit, tb->G, gu}, {tb->wunit, tb->nW, wu},
      {tb->wcol, tb->nW, wc}, {tb->wgrp, tb->nW, wg}, {tb->dbase, tb->nW, db}};
  for (auto& q : req) {
    if (q.n && !q.s) { set_error("pair tables: a metadata array is missing"); return BLML_ERR_ARG; }
    int e = fetch(q.s, q.n, q.d);
    if (e) return e;
  }
  int e = cuda_status(cudaStreamSynchronize(st), "pair tables");
  if (e) return e;
  for (int k = 0; k < d; k++) {
    cm.code[k] = (int)codes[k]; cm.base[k] = base[k]; cm.J[k] = J[k]; cm.mk[k] = mk[k]; cm.nb[k] = nb[k];
    cm.grp[k] = (int)grp[k]; cm.dim_unit[k] = (int)du[k];
    if (codes[k] < 0 || codes[k] > 4) { set_error("pair tables: column %d has kind code %lld", k, (long long)codes[k]); return BLML_ERR_ARG; }
    if ((codes[k] == 2 || codes[k] == 4) && (grp[k] < 0 || grp[k] >= tb->G)) { set_error("pair tables: column %d group", k); return BLML_ERR_ARG; }
    if (!(codes[k] == 2 || codes[k] == 4) && (du[k] < 0 || du[k] >= tb->U)) { set_error("pair tables: column %d unit", k); return BLML_ERR_ARG; }
  }
  for (int k = 0; k < d; k++) {              // every column block lies inside the flat value array
    int64_t len = 0;
    if (cm.code[k] == 0) len = 2 * cm.J[k] + 1;
    else if (cm.code[k] == 3) len = cm.mk[k] * cm.mk[k];
    else if (cm.code[k] == 1) len = cm.nb[k] / 2 + 1;
    if (cm.base[k] < 0 || cm.base[k] + len > cm.Tn || cm.J[k] < 0 || cm.mk[k] < 0 || cm.nb[k] < 0) {
      set_error("pair tables: column %d block outside the value array of %lld", k, (long long)cm.Tn);
      return BLML_ERR_ARG;
    }
  }
  for (int g = 0; g < tb->G; g++) {
    cm.grp_unit[g] = (int)gu[g];
    if (gu[g] < 0 || gu[g] >= tb->U) { set_error("pair tables: group %d unit", g); return BLML_ERR_ARG; }
  }
  for (int q = 0; q < tb->nW; q++) {
    cm.wunit[q] = (int)wu[q]; cm.wcol[q] = (int)wc[q]; cm.wgrp[q] = (int)wg[q]; cm.dbase[q] = db[q];
    bool ok = wu[q] >= 0 && wu[q] < tb->U && wg[q] < tb->G && wc[q] < d;
    if (ok && wg[q] < 0) {                   // a column's derivative row: inside dT, with the column's block length
      const int k = (int)wc[q];
      ok = k >= 0 && (cm.code[k] == 0 || cm.code[k] == 3) && db[q] >= 0 &&
           db[q] + (cm.code[k] == 3 ? cm.mk[k] * cm.mk[k] : 2 * cm.J[k] + 1) <= cm.dTn;
    }
    if (!ok) { set_error("pair tables: derivative entry %d outside its tables", q); return BLML_ERR_ARG; }
  }
  return BLML_OK;
}

// the per-column coordinate ranges hr[4 k + (0..3)] = min / max of ZA, min / max of ZB against the tables' extents:
// offsets within +-J (offset rows), ranks within the rank table, folded coordinates within the period (circular /
// torus), radii within the radial row
static int extents_ok(const ColMeta& cm, const long long* hr) {
  double rad[MAXG] = {0, 0, 0, 0};
  for (int k = 0; k < cm.d; k++) {
    const long long mnA = hr[4 * k], mxA = hr[4 * k + 1], mnB = hr[4 * k + 2], mxB = hr[4 * k + 3];
    const long long span = std::max(mxA - mnB, mxB - mnA);
    bool ok = true;
    switch (cm.code[k]) {
      case 0: ok = span <= cm.J[k]; break;
      case 3: ok = mnA >= 0 && mnB >= 0 && mxA < cm.mk[k] && mxB < cm.mk[k]; break;
      case 1: case 4: ok = mnA >= 0 && mnB >= 0 && mxA < cm.nb[k] && mxB < cm.nb[k]; break;
      case 2: rad[cm.grp[k]] += (double)span * (double)span; break;
    }
    if (!ok) {
      set_error("pair tables: column %d coordinates outside the tables' span (stale tables)", k);
      return BLML_ERR_ARG;
    }
  }
  for (int k = 0; k < cm.d; k++)
    if (cm.code[k] == 2 && sqrt(rad[cm.grp[k]]) * RQ + 1 >= cm.LR) {
      set_error("pair tables: radial group %d radius outside its row (stale tables)", cm.grp[k]);
      return BLML_ERR_ARG;
    }
  return BLML_OK;
}

// the coordinates must lie in the tables' extents: offsets within +-J (offset rows), ranks within the rank table,
// folded coordinates within the period (circular / torus), radii within the radial row
static int check_extents(const ColMeta& cm, const int64_t* ZA, int64_t R, const int64_t* ZB, int64_t M,
                         cudaStream_t st) {
  if (R == 0 || M == 0) return BLML_OK;
  long long* dr = nullptr;
  long long hr[4 * MAXD];
  int e = cuda_status(cudaMallocAsync((void**)&dr, 4 * cm.d * sizeof(long long), st), "pair extents");
  if (e) return e;
  k_coord_range<<<cm.d, 256, 0, st>>>(ZA, R, ZB, M, cm.d, dr);
  count_launches(1);
  e = cuda_status(cudaMemcpyAsync(hr, dr, 4 * cm.d * sizeof(long long), cudaMemcpyDeviceToHost, st), "pair extents");
  cudaFreeAsync(dr, st);
  if (!e) e = cuda_status(cudaStreamSynchronize(st), "pair extents");
  if (e) return e;
  return extents_ok(cm, hr);
}

// column slices of a rows launch: so that the grid covers the GPU about four times
static void rows_slices(int64_t R, int64_t M, int64_t& nsl, int64_t& slice) {
  const int64_t rblocks = (R + PR_THREADS - 1) / PR_THREADS;
  nsl = std::max<int64_t>(1, std::min<int64_t>((4 * 148 + rblocks - 1) / rblocks, (M + 1023) / 1024));
  nsl = std::min<int64_t>(nsl, 65535);
  slice = (M + nsl - 1) / nsl;
  nsl = (M + slice - 1) / slice;
}

// ws: the slice partials (nsl R (1 + nW) doubles) when the caller provides them, else a stream-ordered allocation
template <typename REAL>
static int rows_impl(const blml_tables* tb, const ColMeta& cm, const REAL* T, const REAL* RT, const REAL* dT,
                     const REAL* dR, const int64_t* ZA, int64_t R, const int64_t* ZB, int64_t M, const double* w,
                     int grad, double* s, double* ds, cudaStream_t st, double* ws = nullptr) {
  const int64_t rblocks = (R + PR_THREADS - 1) / PR_THREADS;
  int64_t nsl, slice;
  rows_slices(R, M, nsl, slice);
  const int nW = grad ? cm.nW : 0;
  double* part = ws;
  const size_t pbytes = (size_t)nsl * R * (1 + nW) * sizeof(double);
  int e = BLML_OK;
  if (!part) {
    e = cuda_status(cudaMallocAsync((void**)&part, std::max<size_t>(pbytes, 8), st), "blml_rows workspace");
    if (e) return e;
  }
  double* dpart = part + (size_t)nsl * R;
  bool offset_only = cm.G == 0 && !grad;
  for (int k = 0; k < cm.d; k++) offset_only = offset_only && cm.code[k] == 0;
  const size_t tsz = (size_t)cm.Tn * sizeof(REAL);
  dim3 grid((unsigned)rblocks, (unsigned)nsl);
  if (offset_only) {
    const size_t sm = offset_smem_bytes<REAL>(cm.Tn, cm.d);
    if (sm > 200 * 1024) { if (!ws) cudaFreeAsync(part, st); set_error("blml_rows: tables too large for shared memory"); return BLML_ERR_UNSUPPORTED; }
#define ROWS_OFF(DD) case DD: \
      cudaFuncSetAttribute(k_rows_offset<REAL, DD>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm); \
      k_rows_offset<REAL, DD><<<grid, PR_THREADS, sm, st>>>(cm, T, ZA, R, ZB, w, slice, M, part); break;
    switch (cm.d) { ROWS_OFF(1) ROWS_OFF(2) ROWS_OFF(3) ROWS_OFF(4) ROWS_OFF(5) ROWS_OFF(6) ROWS_OFF(7) ROWS_OFF(8) }
#undef ROWS_OFF
  } else {
    const size_t sm = tsz + (size_t)cm.G * cm.LR * sizeof(REAL);
    if (sm > 200 * 1024) { if (!ws) cudaFreeAsync(part, st); set_error("blml_rows: tables too large for shared memory"); return BLML_ERR_UNSUPPORTED; }
    if (grad) {
      cudaFuncSetAttribute(k_rows_general<REAL, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
      k_rows_general<REAL, true><<<grid, PR_THREADS, sm, st>>>(cm, T, RT, dT, dR, ZA, R, ZB, w, 0, slice, M, part, dpart);
    } else {
      cudaFuncSetAttribute(k_rows_general<REAL, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
      k_rows_general<REAL, false><<<grid, PR_THREADS, sm, st>>>(cm, T, RT, dT, dR, ZA, R, ZB, w, 0, slice, M, part, dpart);
    }
  }
  e = cuda_status(cudaGetLastError(), "blml_rows");
  if (!e) {
    count_launches(2);                       // the rows kernel and the slice sum
    k_sum_slices<<<std::min<int64_t>((R + 255) / 256, 4096), 256, 0, st>>>(part, (int)nsl, R, s);
    if (grad && nW) {
      k_sum_slices<<<std::min<int64_t>((R * nW + 255) / 256, 4096), 256, 0, st>>>(dpart, (int)nsl, R * nW, ds);
      count_launches(1);
    }
    e = cuda_status(cudaGetLastError(), "blml_rows finish");
  }
  if (!ws) cudaFreeAsync(part, st);
  return e;
}

extern "C" {

// a rows plan: the tables' metadata read and the coordinates' extents checked once, for many value-row passes over
// rows of the same coordinate set (the block coordinate descent's passes of every bin against a block)
struct blml_rows_plan_s {
  blml_tables tb;
  ColMeta cm;
};

int blml_rows_plan_create(const blml_tables* tb, const int64_t* Z, int64_t n, void* stream, blml_rows_plan* out) {
  if (!tb || !out || n < 0 || (n > 0 && !Z)) { set_error("blml_rows_plan_create: bad arguments"); return BLML_ERR_ARG; }
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  blml_rows_plan_s* p = new blml_rows_plan_s();
  p->tb = *tb;
  int e = read_meta(tb, p->cm, st);
  if (!e && n > 0) e = check_extents(p->cm, Z, n, Z, n, st);          // every pair within Z: min / max per column
  if (!e && (tb->f32 ? (!tb->T32 || (p->cm.G && !tb->RT32)) : (!tb->T || (p->cm.G && !tb->RT)))) {
    set_error("blml_rows_plan_create: value tables missing"); e = BLML_ERR_ARG;
  }
  if (e) { delete p; return e; }
  *out = p;
  return BLML_OK;
}

int64_t blml_rows_plan_workspace(blml_rows_plan p, int64_t R, int64_t M) {
  if (!p || R < 0 || M < 1) return -1;
  int64_t nsl, slice;
  rows_slices(R, M, nsl, slice);
  return nsl * R * (int64_t)sizeof(double);
}

int blml_rows_plan_run(blml_rows_plan p, const int64_t* ZA, int64_t R, const int64_t* ZB, int64_t M, const double* w,
                       double* s, void* ws, int64_t ws_bytes, void* stream) {
  if (!p || R < 0 || M < 0) { set_error("blml_rows_plan_run: bad arguments"); return BLML_ERR_ARG; }
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  if (R == 0) return BLML_OK;
  if (M == 0) return cuda_status(cudaMemsetAsync(s, 0, R * sizeof(double), st), "blml_rows_plan_run");
  const int64_t need = blml_rows_plan_workspace(p, R, M);
  if (!ws || ws_bytes < need) {
    set_error("blml_rows_plan_run: workspace of %lld bytes, need %lld", (long long)ws_bytes, (long long)need);
    return BLML_ERR_WORKSPACE;
  }
  const blml_tables* tb = &p->tb;
  if (tb->f32)
    return rows_impl<float>(tb, p->cm, tb->T32, tb->RT32, nullptr, nullptr, ZA, R, ZB, M, w, 0, s, nullptr, st,
                            reinterpret_cast<double*>(ws));
  return rows_impl<double>(tb, p->cm, tb->T, tb->RT, nullptr, nullptr, ZA, R, ZB, M, w, 0, s, nullptr, st,
                           reinterpret_cast<double*>(ws));
}

int blml_rows_plan_destroy(blml_rows_plan p) {
  delete p;
  return BLML_OK;
}

int blml_rows(const blml_tables* tb, const int64_t* ZA, int64_t R, const int64_t* ZB, int64_t M, const double* w,
              int grad, double* s, double* ds, void* stream) {
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  ColMeta cm;
  int e = read_meta(tb, cm, st);
  if (e) return e;
  if (grad && cm.nW == 0) grad = 0;
  if (R == 0) return BLML_OK;
  if (M == 0) return cuda_status(cudaMemsetAsync(s, 0, R * sizeof(double), st), "blml_rows");
  e = check_extents(cm, ZA, R, ZB, M, st);
  if (e) return e;
  if (tb->f32) {
    if (!tb->T32 || (cm.G && !tb->RT32) || (grad && (!tb->dT32 || !tb->dR32))) { set_error("blml_rows: float32 tables missing"); return BLML_ERR_ARG; }
    return rows_impl<float>(tb, cm, tb->T32, tb->RT32, tb->dT32, tb->dR32, ZA, R, ZB, M, w, grad, s, ds, st);
  }
  if (!tb->T || (cm.G && !tb->RT) || (grad && (!tb->dT || !tb->dR))) { set_error("blml_rows: tables missing"); return BLML_ERR_ARG; }
  return rows_impl<double>(tb, cm, tb->T, tb->RT, tb->dT, tb->dR, ZA, R, ZB, M, w, grad, s, ds, st);
}

}  // extern "C"

template <typename REAL>
static int rows_multi_impl(const ColMeta& cm, const REAL* T, const REAL* RT, const int64_t* ZA, int64_t R,
                           const int64_t* ZB, int64_t M, const double* W, int Mm, const DensMasks& dm, double* s,
                           cudaStream_t st) {
  const int64_t rblocks = (R + PR_THREADS - 1) / PR_THREADS;
  int64_t nsl, slice;
  rows_slices(R, M, nsl, slice);
  double* part = nullptr;
  int e = cuda_status(cudaMallocAsync((void**)&part, std::max<size_t>((size_t)nsl * R * Mm * sizeof(double), 8), st),
                      "blml_rows_multi workspace");
  if (e) return e;
  const size_t sm = (size_t)cm.Tn * sizeof(REAL) + (size_t)cm.G * cm.LR * sizeof(REAL);
  if (sm > 200 * 1024) { cudaFreeAsync(part, st); set_error("blml_rows_multi: tables too large for shared memory"); return BLML_ERR_UNSUPPORTED; }
  cudaFuncSetAttribute(k_rows_multi<REAL>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  k_rows_multi<REAL><<<dim3((unsigned)rblocks, (unsigned)nsl), PR_THREADS, sm, st>>>(cm, T, RT, ZA, R, ZB, W, Mm, dm,
                                                                                   slice, M, part);
  e = cuda_status(cudaGetLastError(), "blml_rows_multi");
  if (!e) {
    count_launches(2);
    k_sum_slices<<<std::min<int64_t>((R * Mm + 255) / 256, 4096), 256, 0, st>>>(part, (int)nsl, R * Mm, s);
    e = cuda_status(cudaGetLastError(), "blml_rows_multi finish");
  }
  cudaFreeAsync(part, st);
  return e;
}

extern "C" {

int blml_rows_multi(const blml_tables* tb, const int64_t* ZA, int64_t R, const int64_t* ZB, int64_t M,
                    const double* W, int Mm, const unsigned* umask, double* s, void* stream) {
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  if (Mm < 1 || Mm > MAXM || !umask) { set_error("blml_rows_multi: 1 to %d densities with a unit mask each", MAXM); return BLML_ERR_ARG; }
  ColMeta cm;
  int e = read_meta(tb, cm, st);
  if (e) return e;
  DensMasks dm;
  for (int m = 0; m < MAXM; m++) dm.bits[m] = m < Mm ? umask[m] : 0u;
  for (int m = 0; m < Mm; m++)
    if (dm.bits[m] >> cm.U) { set_error("blml_rows_multi: density %d masks a unit beyond the tables' %d", m, cm.U); return BLML_ERR_ARG; }
  if (R == 0) return BLML_OK;
  if (M == 0) return cuda_status(cudaMemsetAsync(s, 0, R * Mm * sizeof(double), st), "blml_rows_multi");
  if (!ZA || !ZB || !W || !s) { set_error("blml_rows_multi: null pointer"); return BLML_ERR_ARG; }
  e = check_extents(cm, ZA, R, ZB, M, st);
  if (e) return e;
  if (tb->f32) {
    if (!tb->T32 || (cm.G && !tb->RT32)) { set_error("blml_rows_multi: float32 tables missing"); return BLML_ERR_ARG; }
    return rows_multi_impl<float>(cm, tb->T32, tb->RT32, ZA, R, ZB, M, W, Mm, dm, s, st);
  }
  if (!tb->T || (cm.G && !tb->RT)) { set_error("blml_rows_multi: tables missing"); return BLML_ERR_ARG; }
  return rows_multi_impl<double>(cm, tb->T, tb->RT, ZA, R, ZB, M, W, Mm, dm, s, st);
}

}  // extern "C"

// ---- blml_rows_noalloc: the value rows with a fixed scratch array instead of any device allocation ----
// Its scratch (the per-column coordinate ranges of the extent check, then the column-slice partial sums) lives in
// this file-scope device array: 4 MiB on every GPU that loads the library, held until the process exits. Host code
// must not pass the symbol itself to a kernel (on the host it names a stand-in, not device memory): the device
// address comes from cudaGetSymbolAddress, taken once per device with that device current, on the first call (and
// again if the device's context has changed since).
constexpr int64_t kRowsScratchDoubles = (int64_t)1 << 19;       // 4 MiB
constexpr int64_t kRowsScratchRangeSlots = 64;                   // 4 * d <= 32 range words, padded to 512 bytes
constexpr int64_t kRowsNoAllocMaxR = kRowsScratchDoubles - kRowsScratchRangeSlots;
static __device__ __align__(256) double g_rows_scratch[kRowsScratchDoubles];

static int rows_scratch(double** out) {
  int dev = 0;
  int e = cuda_status(cudaGetDevice(&dev), "blml_rows_noalloc");
  if (e) return e;
  if (dev < 0 || dev >= 64) { set_error("blml_rows_noalloc: device ordinal %d above 63", dev); return BLML_ERR_ARG; }
  // the address belongs to the device's current context: taken again when that context is not the one it was
  // taken in (after a cudaDeviceReset, or under another context)
  // cuCtxGetCurrent through the runtime's driver entry point, so that the library needs no link to libcuda and
  // loads on a host without a driver
  using CtxGetFn = CUresult (*)(CUcontext*);
  static CtxGetFn ctx_get = []() -> CtxGetFn {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      return reinterpret_cast<CtxGetFn>(p);
    return nullptr;
  }();
  CUcontext ctx = nullptr;
  if (!ctx_get || ctx_get(&ctx) != CUDA_SUCCESS) {
    set_error("blml_rows_noalloc: no current context"); return BLML_ERR_CUDA;
  }
  static std::mutex mu;
  static double* ptrs[64] = {nullptr};
  static CUcontext ctxs[64] = {nullptr};
  std::lock_guard<std::mutex> lock(mu);
  if (!ptrs[dev] || ctxs[dev] != ctx) {
    void* p = nullptr;
    e = cuda_status(cudaGetSymbolAddress(&p, g_rows_scratch), "blml_rows_noalloc scratch address");
    if (e) return e;
    ptrs[dev] = reinterpret_cast<double*>(p); ctxs[dev] = ctx;
  }
  *out = ptrs[dev];
  return BLML_OK;
}

template <typename REAL>
static int rows_noalloc_launch(const ColMeta& cm, const REAL* T, const REAL* RT, const int64_t* ZA, int64_t R,
                               const int64_t* ZB, int64_t M, const double* w, double* part, double* s,
                               cudaStream_t st) {
  const int64_t rblocks = (R + PR_THREADS - 1) / PR_THREADS;
  int64_t nsl = std::max<int64_t>(1, std::min<int64_t>((4 * 148 + rblocks - 1) / rblocks, (M + 1023) / 1024));
  nsl = std::min<int64_t>(std::min<int64_t>(nsl, 65535), std::max<int64_t>(1, kRowsNoAllocMaxR / R));
  const int64_t slice = (M + nsl - 1) / nsl;
  nsl = (M + slice - 1) / slice;
  bool offset_only = cm.G == 0;
  for (int k = 0; k < cm.d; k++) offset_only = offset_only && cm.code[k] == 0;
  dim3 grid((unsigned)rblocks, (unsigned)nsl);
  if (offset_only) {
    const size_t sm = offset_smem_bytes<REAL>(cm.Tn, cm.d);
    if (sm > 200 * 1024) { set_error("blml_rows_noalloc: tables too large for shared memory"); return BLML_ERR_UNSUPPORTED; }
#define ROWS_OFF_NA(DD) case DD: \
      cudaFuncSetAttribute(k_rows_offset<REAL, DD>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm); \
      k_rows_offset<REAL, DD><<<grid, PR_THREADS, sm, st>>>(cm, T, ZA, R, ZB, w, slice, M, part); break;
    switch (cm.d) { ROWS_OFF_NA(1) ROWS_OFF_NA(2) ROWS_OFF_NA(3) ROWS_OFF_NA(4) ROWS_OFF_NA(5) ROWS_OFF_NA(6) ROWS_OFF_NA(7) ROWS_OFF_NA(8) }
#undef ROWS_OFF_NA
  } else {
    const size_t sm = (size_t)cm.Tn * sizeof(REAL) + (size_t)cm.G * cm.LR * sizeof(REAL);
    if (sm > 200 * 1024) { set_error("blml_rows_noalloc: tables too large for shared memory"); return BLML_ERR_UNSUPPORTED; }
    cudaFuncSetAttribute(k_rows_general<REAL, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k_rows_general<REAL, false><<<grid, PR_THREADS, sm, st>>>(cm, T, RT, nullptr, nullptr, ZA, R, ZB, w, 0, slice, M,
                                                              part, nullptr);
  }
  int e = cuda_status(cudaGetLastError(), "blml_rows_noalloc");
  if (e) return e;
  k_sum_slices<<<std::min<int64_t>((R + 255) / 256, 4096), 256, 0, st>>>(part, (int)nsl, R, s);
  count_launches(2);
  return cuda_status(cudaGetLastError(), "blml_rows_noalloc finish");
}

extern "C" {

int blml_rows_noalloc(const blml_tables* tb, const int64_t* ZA, int64_t R, const int64_t* ZB, int64_t M,
                      const double* w, double* s, void* stream) {
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  ColMeta cm;
  int e = read_meta(tb, cm, st);
  if (e) return e;
  if (R < 0 || M < 0) { set_error("blml_rows_noalloc: negative sizes"); return BLML_ERR_ARG; }
  if (R > kRowsNoAllocMaxR) {
    set_error("blml_rows_noalloc: %lld rows exceed the fixed scratch (at most %lld rows)", (long long)R,
              (long long)kRowsNoAllocMaxR);
    return BLML_ERR_ARG;
  }
  if (R == 0) return BLML_OK;
  if (M == 0) return cuda_status(cudaMemsetAsync(s, 0, R * sizeof(double), st), "blml_rows_noalloc");
  double* scratch = nullptr;
  e = rows_scratch(&scratch);
  if (e) return e;
  // extent check: per-column coordinate ranges into the scratch head, read back, compared with the tables
  long long* ranges = reinterpret_cast<long long*>(scratch);
  k_coord_range<<<cm.d, 256, 0, st>>>(ZA, R, ZB, M, cm.d, ranges);
  count_launches(1);
  long long hr[4 * MAXD];
  e = cuda_status(cudaMemcpyAsync(hr, ranges, 4 * cm.d * sizeof(long long), cudaMemcpyDeviceToHost, st),
                  "blml_rows_noalloc extents");
  if (!e) e = cuda_status(cudaStreamSynchronize(st), "blml_rows_noalloc extents");
  if (e) return e;
  e = extents_ok(cm, hr);
  if (e) return e;
  double* part = scratch + kRowsScratchRangeSlots;
  if (tb->f32) {
    if (!tb->T32 || (cm.G && !tb->RT32)) { set_error("blml_rows_noalloc: float32 tables missing"); return BLML_ERR_ARG; }
    return rows_noalloc_launch<float>(cm, tb->T32, tb->RT32, ZA, R, ZB, M, w, part, s, st);
  }
  if (!tb->T || (cm.G && !tb->RT)) { set_error("blml_rows_noalloc: tables missing"); return BLML_ERR_ARG; }
  return rows_noalloc_launch<double>(cm, tb->T, tb->RT, ZA, R, ZB, M, w, part, s, st);
}

int blml_lattice_coords(const double* Z, int64_t n, int d, const double* h, int64_t* out, void* stream) {
  if (n < 0 || d < 1) { set_error("blml_lattice_coords: bad sizes"); return BLML_ERR_ARG; }
  if (n == 0) return BLML_OK;
  const int g = (int)std::min<int64_t>((n * d + 255) / 256, 148 * 32);
  k_lattice_coords<<<g, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(Z, n, d, h, out);
  count_launches(1);
  return cuda_status(cudaGetLastError(), "blml_lattice_coords");
}

static int cols_launch(const blml_tables* tb, const int64_t* ZA, int64_t R, const int64_t* ZB, int64_t M, void* out,
                       void* out_m, int64_t depmask, int out_f32, void* stream, const char* who) {
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  ColMeta cm;
  int e = read_meta(tb, cm, st);
  if (e) return e;
  if (depmask < 0 || (cm.d < 63 && (depmask >> cm.d) != 0)) { set_error("%s: depmask has bits past column d", who); return BLML_ERR_ARG; }
  if (R == 0 || M == 0) return BLML_OK;
  e = check_extents(cm, ZA, R, ZB, M, st);
  if (e) return e;
  unsigned dep_units = 0;                        // a unit (column or radial group) is dep when one of its columns is
  for (int k = 0; k < cm.d; k++)              // a group column's unit is its group's
    if ((depmask >> k) & 1) dep_units |= 1u << ((cm.code[k] == 2 || cm.code[k] == 4) ? cm.grp_unit[cm.grp[k]] : cm.dim_unit[k]);
  const int64_t n = R * M;
  const int g = (int)std::min<int64_t>((n + 255) / 256, 148 * 32);
  if (tb->f32) {
    if (out_f32) k_cols<float, float><<<g, 256, 0, st>>>(cm, tb->T32, tb->RT32, ZA, R, ZB, M, (float*)out, (float*)out_m, dep_units);
    else k_cols<float, double><<<g, 256, 0, st>>>(cm, tb->T32, tb->RT32, ZA, R, ZB, M, (double*)out, (double*)out_m, dep_units);
  } else {
    if (out_f32) k_cols<double, float><<<g, 256, 0, st>>>(cm, tb->T, tb->RT, ZA, R, ZB, M, (float*)out, (float*)out_m, dep_units);
    else k_cols<double, double><<<g, 256, 0, st>>>(cm, tb->T, tb->RT, ZA, R, ZB, M, (double*)out, (double*)out_m, dep_units);
  }
  count_launches(1);
  return cuda_status(cudaGetLastError(), who);
}

int blml_cols(const blml_tables* tb, const int64_t* ZA, int64_t R, const int64_t* ZB, int64_t M, void* out,
              int out_f32, void* stream) {
  return cols_launch(tb, ZA, R, ZB, M, out, nullptr, 0, out_f32, stream, "blml_cols");
}

int blml_cols_dep(const blml_tables* tb, const int64_t* ZA, int64_t R, const int64_t* ZB, int64_t M, int64_t depmask,
                  void* out, void* out_m, int out_f32, void* stream) {
  if (!out_m) { set_error("blml_cols_dep: out_m"); return BLML_ERR_ARG; }
  return cols_launch(tb, ZA, R, ZB, M, out, out_m, depmask, out_f32, stream, "blml_cols_dep");
}

}
