// Device-side control of the batched engine. The per-fit scalar logic of the two solver phases -- the real rank-1
// start (Jacobi updates, Anderson mixing, the merit safeguard; blml_binned.py:223-276) and L-BFGS (compact
// direction, Armijo choice, pair update, stop rules; blml_trivial.py:2590-2645 as blml_binned.py runs it) -- runs as
// small kernels over the fits, so one iteration is a fixed sequence of launches with no host decision in it. A ring
// of iterations (one per memory slot) is captured once as a CUDA graph and replayed until every fit has stopped;
// the host reads one active mask per replay, and when the active set has shrunk it captures the graph again over
// the fits still iterating (compact index j -> fit f = fid[j]; per-fit state is indexed by f, per-launch scalar
// tables by j). A fit that stops inside a replay gets an empty segment (B = 0) and a cleared live flag, which every
// later launch of the replay reads, so it does no more work.
#include <vector>
#include <algorithm>
#include <limits.h>
#include "common.cuh"
#include "plan.cuh"
#include "segmented.cuh"

namespace blml {

constexpr int LB_MMAX = 20, LB_FWIN = 10, LB_NT = 40, AA_MMAX = 8, DAMP_NT = 26;
enum { STOP_TOL = 0, STOP_LLTOL = 1, STOP_STALL = 2 };

__device__ __forceinline__ double warp_allsum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// the start's merit from its three terms [sum e u, sum_occ c log|e|, #(sg e <= 0)] (blml_binned.py:208-220)
__device__ __forceinline__ double merit_value(const double* r, double n) {
  const double m = -(0.5 * r[0] - r[1]) / n;
  return r[2] > 0 ? -INFINITY : m;
}

__device__ __forceinline__ void set_live(int j, int f, int on, int* live, const blml_seg* segs_c, blml_seg* segs_eff) {
  live[f] = on;
  blml_seg s = segs_c[j];
  if (!on) s.B = 0;
  segs_eff[j] = s;
}

__global__ void k_fill_int(int* a, int n, int v) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) a[i] = v;
}

__global__ void k_fill_double(double* a, int64_t n, double v) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) a[i] = v;
}

// one warp per quantity: out[j * nq + q] = the fixed-order sum of the fit's nblk partials, for the fits whose flag
// is set
__global__ void k_finish_flagged(const double* part, int nq, int nblk, const int* flag, double* out) {
  const int j = blockIdx.x, Fa = gridDim.x;
  if (flag && !flag[j]) return;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int q = wid; q < nq; q += nw) {
    double x = 0.0;
    for (int i = lane; i < nblk; i += 32) x += part[((int64_t)q * Fa + j) * nblk + i];
    x = warp_sum(x);
    if (lane == 0) out[(int64_t)j * nq + q] = x;
  }
}

// ------------------------------------------------------------------------------------------------ L-BFGS control
struct LbState {
  double *L, *Q, *Qn, *n, *res, *slope, *qq, *mh, *SY, *YY;
  int *active, *it, *stop, *reset, *nh, *ok, *stamp, *step;
  const long long* caps;                 // per-fit iteration caps (null: the runner's one cap for every fit)
};

// the compact L-BFGS direction of fit f (one warp): q = gam g + S p - gam Y t over the fit's pairs in the order they
// entered (R = triu(S^T Y), R t = S^T g, R^T p = (D + gam Y^T Y) t - gam Y^T g); the scaled gradient when there are
// no pairs or the direction is not an ascent one (which also clears the memory). Block 0 advances the step counter.
__global__ void k_lb_dir(int m, const int* fid, const int* live, const double* H1, const double* H2, LbState s,
                         double* cq_all) {
  const int j = blockIdx.x, lane = threadIdx.x, f = fid[j];
  if (j == 0 && lane == 0) (*s.step)++;
  const int nc = 1 + 2 * m;
  double* cq = cq_all + (int64_t)j * nc;
  for (int i = lane; i < nc; i += 32) cq[i] = 0.0;
  if (!live[f]) return;
  __syncwarp();
  // the history scan of the previous iteration: H1 = [S_q . y_p, S_q . g, y_p . y_p, g . g, E . E],
  // H2 = [Y_q . y_p, Y_q . g, ...] (stride 2 m + 3)
  const double* h1 = H1 + (int64_t)j * (2 * m + 3);
  const double* h2 = H2 + (int64_t)j * (2 * m + 3);
  const double gg = h1[2 * m + 1], ee = h1[2 * m + 2];
  const double first = 1e-3 * sqrt(fmax(ee, 0.0) / fmax(gg, 1e-300));
  int* stamp = s.stamp + (int64_t)f * m;
  __shared__ int ord[LB_MMAX];
  __shared__ int kk;
  __shared__ double R[LB_MMAX][LB_MMAX + 1], Yy[LB_MMAX][LB_MMAX + 1], ts[LB_MMAX];
  if (lane == 0) {
    int k = 0;
    for (int q = 0; q < m; q++)
      if (stamp[q] >= 0) ord[k++] = q;
    for (int i = 1; i < k; i++) {                     // chronological order of the stored pairs
      const int x = ord[i];
      int jj = i - 1;
      while (jj >= 0 && stamp[ord[jj]] > stamp[x]) { ord[jj + 1] = ord[jj]; jj--; }
      ord[jj + 1] = x;
    }
    kk = k;
  }
  __syncwarp();
  const int k = kk;
  bool first_only = true;
  double slope = 0.0, gam = 0.0, t_l = 0.0, p_l = 0.0;
  if (k > 0) {
    const double* SY = s.SY + (int64_t)f * m * m;
    const double* YY = s.YY + (int64_t)f * m * m;
    for (int idx = lane; idx < k * k; idx += 32) {
      const int i = idx / k, c = idx - (idx / k) * k;
      R[i][c] = c >= i ? SY[ord[i] * m + ord[c]] : 0.0;
      Yy[i][c] = YY[ord[i] * m + ord[c]];
    }
    __syncwarp();
    const int last = ord[k - 1];
    gam = SY[last * m + last] / YY[last * m + last];
    const double ao = lane < k ? h1[m + ord[lane]] : 0.0, bo = lane < k ? h2[m + ord[lane]] : 0.0;
    double r = ao;                                    // back substitution, R t = ao
    for (int i = k - 1; i >= 0; i--) {
      const double ti = __shfl_sync(0xffffffffu, r, i) / R[i][i];
      if (lane == i) t_l = ti;
      if (lane < i) r -= R[lane][i] * ti;
    }
    if (lane < k) ts[lane] = t_l;
    __syncwarp();
    r = 0.0;
    if (lane < k) {
      double acc = 0.0;
      for (int c = 0; c < k; c++) acc += ((c == lane ? R[lane][lane] : 0.0) + gam * Yy[lane][c]) * ts[c];
      r = acc - gam * bo;
    }
    for (int i = 0; i < k; i++) {                     // forward substitution, R^T p = rhs
      const double pi = __shfl_sync(0xffffffffu, r, i) / R[i][i];
      if (lane == i) p_l = pi;
      if (lane > i && lane < k) r -= R[i][lane] * pi;
    }
    const double s1 = warp_allsum(lane < k ? ao * p_l : 0.0), s2 = warp_allsum(lane < k ? bo * t_l : 0.0);
    slope = gam * gg + s1 - gam * s2;
    first_only = !(slope > 0);
  }
  __syncwarp();
  if (first_only) {
    if (lane == 0) { cq[0] = first; s.slope[f] = first * gg; }
    if (k > 0)
      for (int q = lane; q < m; q += 32) stamp[q] = -1;
  } else {
    if (lane == 0) { cq[0] = gam; s.slope[f] = slope; }
    if (lane < k) { cq[1 + ord[lane]] = p_l; cq[1 + m + ord[lane]] = -gam * t_l; }
  }
}

// the Armijo trials t_j = 2^-j, j0 <= j < j0 + NTG, of the fits whose flag is set (all when null): sum_occ w log F(U +
// t_j S q); the first group also <q, U>, <E, S q>, <q, S q> (Q(t) = Q + t (<q, U> + <E, S q>) + t^2 <q, S q>) and <q, q>
template <typename T, int NTG, bool FIRST>
__global__ void __launch_bounds__(256) k_lb_trials(const blml_seg* segs, const int* flag, int j0, const void* E,
                                                   const void* q, const void* U, const void* Sq, const T* w,
                                                   double* part) {
  if (flag && !flag[blockIdx.y]) return;
  const blml_seg S = segs[blockIdx.y];
  constexpr int NQ = NTG + (FIRST ? 4 : 0);
  double v[NQ];
#pragma unroll
  for (int j = 0; j < NQ; j++) v[j] = 0.0;
  const double t0 = ldexp(1.0, -j0);
  SEG_LOOP(b, S) {
    const double wb = (double)w[S.boff + b];
    double a = 0.0, bb = 0.0, cc = 0.0;        // F(t) = a + 2 t b + t^2 c
    for (int k = 0; k < S.K; k++) {
      const int64_t i = S.off + (int64_t)k * S.B + b;
      double er, ei, qr, qi, ur, ui, sr, si;
      SAcc<T, true>::get(E, i, er, ei); SAcc<T, true>::get(q, i, qr, qi);
      SAcc<T, true>::get(U, i, ur, ui); SAcc<T, true>::get(Sq, i, sr, si);
      a += ur * ur + ui * ui; bb += ur * sr + ui * si; cc += sr * sr + si * si;
      if (FIRST) {
        v[NTG] += qr * ur + qi * ui; v[NTG + 1] += er * sr + ei * si; v[NTG + 2] += qr * sr + qi * si;
        v[NTG + 3] += qr * qr + qi * qi;
      }
    }
    if (wb > 0) {
      double t = t0;
#pragma unroll
      for (int j = 0; j < NTG; j++) { v[j] += wb * log(a + t * (2.0 * bb + t * cc)); t *= 0.5; }
    }
  }
  seg_partials<NQ>(v, part);
}

constexpr int LB_T1 = 8, LB_T2 = LB_NT - LB_T1;

__device__ __forceinline__ bool armijo_scan(const double* tr, int nt, double t, double Qa, double A, double Cc,
                                            double La, double na, double slope, double& tok) {
  for (int jj = 0; jj < nt; jj++) {
    const double Qt = Qa + t * A + t * t * Cc;
    const double Lt = Qt > 0 ? tr[jj] - na * log(Qt) : -INFINITY;
    if (Lt >= La + 1e-4 * t * slope) { tok = t; return true; }
    t *= 0.5;
  }
  return false;
}

// the Armijo choice over the first 8 trials; need2[j] marks the fits that try the other 32
__global__ void k_lb_select1(int Fa, const int* fid, const int* live, const double* T1, LbState s, double* tA,
                             int* need2) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= Fa) return;
  const int f = fid[j];
  need2[j] = 0; tA[j] = 0.0;
  if (!live[f]) { s.ok[f] = 0; return; }
  const double* tr = T1 + (int64_t)j * (LB_T1 + 4);
  const double A = tr[LB_T1] + tr[LB_T1 + 1], Cc = tr[LB_T1 + 2];
  s.qq[f] = tr[LB_T1 + 3];
  double t = 0.0;
  const bool ok = armijo_scan(tr, LB_T1, 1.0, s.Q[f], A, Cc, s.L[f], s.n[f], s.slope[f], t);
  s.ok[f] = ok; tA[j] = ok ? t : 0.0;
  need2[j] = !ok;
}

// the remaining trials of the fits that need them, then every fit's outcome: a failed search clears the memory once
// and stops the fit ('stall') when it fails again or had no pairs; the coefficient rows of the pair and g updates
__global__ void k_lb_select2(int Fa, int m, const int* fid, const int* live, const double* T1, const double* T2,
                             const int* need2, LbState s, double* tA, double* cS, double* cY, double* cG) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= Fa) return;
  const int f = fid[j];
  int ok = 0;
  double t = 0.0;
  if (live[f]) {
    ok = s.ok[f]; t = tA[j];
    if (need2[j]) {
      const double* tr1 = T1 + (int64_t)j * (LB_T1 + 4);
      const double A = tr1[LB_T1] + tr1[LB_T1 + 1], Cc = tr1[LB_T1 + 2];
      ok = armijo_scan(T2 + (int64_t)j * LB_T2, LB_T2, ldexp(1.0, -LB_T1), s.Q[f], A, Cc, s.L[f], s.n[f],
                       s.slope[f], t);
      if (!ok) t = 0.0;
    }
    int* stamp = s.stamp + (int64_t)f * m;
    if (!ok) {
      bool nopairs = true;
      for (int q = 0; q < m; q++) nopairs &= stamp[q] < 0;
      if (s.reset[f] || nopairs) { s.stop[f] = STOP_STALL; s.active[f] = 0; }
      else { for (int q = 0; q < m; q++) stamp[q] = -1; s.reset[f] = 1; }
    } else {
      s.reset[f] = 0;
    }
  }
  s.ok[f] = ok;
  const double o = ok ? 1.0 : 0.0;
  tA[j] = t;
  cS[2 * j] = t; cS[2 * j + 1] = 1.0 - o;
  cY[3 * j] = o; cY[3 * j + 1] = -o; cY[3 * j + 2] = 1.0 - o;
  cG[2 * j] = o; cG[2 * j + 1] = 1.0 - o;
}

// the gradient weights at the new point fused with Q: F = sum_k |U_k|^2, V = (w / F) U on occupied bins,
// [sum_occ w log F, Re <E, U>] per fit
template <typename T>
__global__ void __launch_bounds__(256) k_lb_weights(const blml_seg* segs, const void* E, const void* U, const T* w,
                                                    void* V, double* part) {
  const blml_seg S = segs[blockIdx.y];
  double v[2] = {0.0, 0.0};
  SEG_LOOP(b, S) {
    double F = 0.0;
    for (int k = 0; k < S.K; k++) {
      const int64_t i = S.off + (int64_t)k * S.B + b;
      double er, ei, ur, ui;
      SAcc<T, true>::get(E, i, er, ei); SAcc<T, true>::get(U, i, ur, ui);
      F += ur * ur + ui * ui; v[1] += er * ur + ei * ui;
    }
    const double wb = (double)w[S.boff + b];
    const bool occ = wb > 0;
    if (occ) v[0] += wb * log(F);
    const double fw = occ ? wb / F : 0.0;
    for (int k = 0; k < S.K; k++) {
      const int64_t i = S.off + (int64_t)k * S.B + b;
      double ur, ui; SAcc<T, true>::get(U, i, ur, ui);
      SAcc<T, true>::put(V, i, occ ? ur * fw : 0.0, occ ? ui * fw : 0.0);
    }
  }
  seg_partials<2>(v, part);
}

// Q at the new point, and the scales of the gradient finish (n / Q) and of the residual (n / sqrt Q)
__global__ void k_lb_qeff(int Fa, const int* fid, const int* live, const double* outD, LbState s, double* nqA,
                          double* scrA) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= Fa) return;
  const int f = fid[j];
  if (!live[f]) { nqA[j] = 0.0; scrA[j] = 1.0; return; }
  const double Qn = outD[2 * j + 1];
  s.Qn[f] = Qn;
  const double Qe = s.ok[f] ? Qn : s.Q[f];
  nqA[j] = s.n[f] / Qe;
  scrA[j] = Qe > 0 ? s.n[f] / sqrt(fmax(Qe, 1e-300)) : 1.0;
}

// the end of an iteration: the new pair (s, y) into slot p when its curvature is positive, the accepted state, the
// likelihood window, then the stop rules the next iteration starts with (tol, ll_tol, the iteration cap)
__global__ void k_lb_post(int Fa, int m, int p, double tol, double ftol, long long cap, const int* fid, int* live,
                          const blml_seg* segs_c, blml_seg* segs_eff, const double* H1, const double* H2,
                          const double* outD, const double* outE, const double* tA, LbState s) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= Fa) return;
  const int f = fid[j];
  if (!live[f]) { set_live(j, f, 0, live, segs_c, segs_eff); return; }
  const int ok = s.ok[f];
  const double nf = s.n[f], Qn = s.Qn[f];
  const double Ln = Qn > 0 ? outD[2 * j] - nf * log(Qn) : -INFINITY;
  const double r = outE[2 * j + 1] > 0 ? NAN : outE[2 * j];
  const double* h1 = H1 + (int64_t)j * (2 * m + 3);
  const double* h2 = H2 + (int64_t)j * (2 * m + 3);
  const double sy = h1[p], yy = h1[2 * m], ss = tA[j] * tA[j] * s.qq[f];     // s_p = t q
  const bool enter = ok && (sy > 1e-12 * sqrt(fmax(ss * yy, 0.0)));
  int* stamp = s.stamp + (int64_t)f * m;
  if (ok) stamp[p] = -1;
  if (enter) {
    stamp[p] = *s.step;
    double* SY = s.SY + (int64_t)f * m * m;
    double* YY = s.YY + (int64_t)f * m * m;
    for (int q = 0; q < m; q++) SY[q * m + p] = h1[q];
    SY[p * m + p] = sy;
    for (int q = 0; q < m; q++) { YY[q * m + p] = h2[q]; YY[p * m + q] = h2[q]; }
    YY[p * m + p] = yy;
  }
  double* h = s.mh + (int64_t)f * (LB_FWIN + 1);
  if (ok) {
    s.L[f] = Ln; s.Q[f] = Qn; s.res[f] = r;
    for (int i = 0; i < LB_FWIN; i++) h[i] = h[i + 1];
    h[LB_FWIN] = Ln / nf;
    s.nh[f]++;
    if (r < tol) s.active[f] = 0;
  }
  int a = s.active[f];
  if (a && s.nh[f] > LB_FWIN && h[LB_FWIN] - h[0] < ftol) { s.stop[f] = STOP_LLTOL; a = 0; }
  if (a && s.it[f] >= (s.caps ? s.caps[f] : cap)) a = 0;
  if (a) s.it[f]++;
  s.active[f] = a;
  set_live(j, f, a, live, segs_c, segs_eff);
}

// set-up: the scale n / sqrt(Q) that normalises E and U, and Q after it
__global__ void k_lbi_scale(int Fa, const int* fid, const double* outC, LbState s, double* sc, double* nqA,
                            double* scrA) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= Fa) return;
  const int f = fid[j];
  const double Qv = outC[j], nf = s.n[f];
  const double c = Qv > 0 ? nf / sqrt(fmax(Qv, 1e-300)) : 1.0;
  sc[j] = c;
  const double Q = Qv * c * c;
  s.Q[f] = Q;
  nqA[j] = nf / Q;
  scrA[j] = Q > 0 ? nf / sqrt(fmax(Q, 1e-300)) : 1.0;
}

__global__ void k_lbi_state(int Fa, int m, double tol, long long cap, const int* fid, int* live,
                            const blml_seg* segs_c, blml_seg* segs_eff, const double* outD, const double* outE,
                            LbState s) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= Fa) return;
  const int f = fid[j];
  const double nf = s.n[f];
  s.L[f] = outD[2 * j] - nf * log(s.Q[f]);
  const double r = outE[2 * j + 1] > 0 ? NAN : outE[2 * j];
  s.res[f] = r;
  for (int q = 0; q < m; q++) s.stamp[(int64_t)f * m + q] = -1;
  for (int q = 0; q < m * m; q++) { s.SY[(int64_t)f * m * m + q] = 0.0; s.YY[(int64_t)f * m * m + q] = 0.0; }
  double* h = s.mh + (int64_t)f * (LB_FWIN + 1);
  for (int i = 0; i < LB_FWIN; i++) h[i] = NAN;
  h[LB_FWIN] = s.L[f] / nf;
  s.nh[f] = 1; s.reset[f] = 0; s.stop[f] = STOP_TOL; s.ok[f] = 0; s.it[f] = 0;
  int a = r >= tol;
  if (a && 0 >= (s.caps ? s.caps[f] : cap)) a = 0;
  if (a) s.it[f] = 1;
  s.active[f] = a;
  set_live(j, f, a, live, segs_c, segs_eff);
  if (j == 0) *s.step = -1;
}

// --------------------------------------------------------------------------------------------------- start control
struct StState {
  double *n, *s0, *cur, *res, *best_res, *best_m, *mJ, *G;
  int *valid, *has_prev, *best_it, *it, *active;
};

// per fit: the Anderson normal equations on the valid history slots, (G + 1e-12 tr(G) I) gamma = rhs, by LU with
// partial pivoting (blml_binned.py:1470-1474); false when singular or not finite
__device__ bool anderson_solve(int mA, const double* G, const int* valid, const double* rhs, double* gam) {
  double A[AA_MMAX][AA_MMAX + 1];
  double tr = 0.0;
  for (int i = 0; i < mA; i++) tr += valid[i] ? G[i * mA + i] : 0.0;
  for (int i = 0; i < mA; i++) {
    for (int c = 0; c < mA; c++) A[i][c] = (valid[i] && valid[c]) ? G[i * mA + c] : 0.0;
    A[i][i] += valid[i] ? 1e-12 * tr : 1.0;
    A[i][mA] = valid[i] ? rhs[i] : 0.0;
  }
  for (int c = 0; c < mA; c++) {
    int piv = c;
    for (int i = c + 1; i < mA; i++)
      if (fabs(A[i][c]) > fabs(A[piv][c])) piv = i;
    if (A[piv][c] == 0.0) return false;
    if (piv != c)
      for (int k = 0; k <= mA; k++) { const double t = A[c][k]; A[c][k] = A[piv][k]; A[piv][k] = t; }
    for (int i = c + 1; i < mA; i++) {
      const double l = A[i][c] / A[c][c];
      for (int k = c; k <= mA; k++) A[i][k] -= l * A[c][k];
    }
  }
  for (int i = mA - 1; i >= 0; i--) {
    double x = A[i][mA];
    for (int k = i + 1; k < mA; k++) x -= A[i][k] * gam[k];
    gam[i] = x / A[i][i];
  }
  for (int i = 0; i < mA; i++)
    if (!isfinite(gam[i])) return false;
  for (int i = 0; i < mA; i++)
    if (!valid[i]) gam[i] = 0.0;
  return true;
}

// Anderson step of every fit: slot p of the difference history, the mixing weights, the coefficients of
// E_A = E + f - DX gamma - DF gamma over [E, f, DX_0.., DF_0..]
__global__ void k_st_anderson(int Fa, int mA, int p, const int* fid, const int* live, const double* outM1,
                              const double* outA, StState s, double* cA, int* useA) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= Fa) return;
  const int f = fid[j];
  const int nc = 2 + 2 * mA;
  double* row = cA + (int64_t)j * nc;
  for (int i = 0; i < nc; i++) row[i] = 0.0;
  row[0] = 1.0;
  useA[j] = 0;
  if (!live[f]) return;
  s.mJ[f] = merit_value(outM1 + 3 * j, s.n[f]);
  int* valid = s.valid + (int64_t)f * mA;
  double* G = s.G + (int64_t)f * mA * mA;
  const double* vals = outA + (int64_t)j * 2 * mA;
  valid[p] = s.has_prev[f];
  for (int q = 0; q < mA; q++) { G[p * mA + q] = vals[q]; G[q * mA + p] = vals[q]; }
  s.has_prev[f] = 1;
  int nv = 0;
  for (int q = 0; q < mA; q++) nv += valid[q] ? 1 : 0;
  if (nv < 2) return;
  double gam[AA_MMAX];
  if (!anderson_solve(mA, G, valid, vals + mA, gam)) {
    for (int q = 0; q < mA; q++) valid[q] = 0;
    s.has_prev[f] = 0;
    return;
  }
  row[1] = 1.0;
  for (int q = 0; q < mA; q++) { row[2 + q] = -gam[q]; row[2 + mA + q] = -gam[q]; }
  useA[j] = 1;
}

// the better of the Jacobi and Anderson points, and whether the step needs damping (no ascent of the merit)
__global__ void k_st_take(int Fa, int mA, const int* fid, const int* live, const double* outM1, const double* outM2,
                          const int* useA, StState s, double* cT, int* damp) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= Fa) return;
  const int f = fid[j];
  cT[2 * j] = 0.0; cT[2 * j + 1] = 1.0; damp[j] = 0;
  if (!live[f]) return;
  double mJ = mA ? s.mJ[f] : merit_value(outM1 + 3 * j, s.n[f]);
  if (mA && useA[j]) {
    const double mAc = merit_value(outM2 + 3 * j, s.n[f]);
    if (mAc > mJ) { mJ = mAc; cT[2 * j] = 1.0; cT[2 * j + 1] = 0.0; }
  }
  s.mJ[f] = mJ;
  const double cur = s.cur[f];
  if (mJ < cur - 1e-12 * fabs(cur)) {
    damp[j] = 1;
    for (int q = 0; q < mA; q++) s.valid[(int64_t)f * mA + q] = 0;
    s.has_prev[f] = 0;
  }
}

// the damped Jacobi steps of the fits whose flag is set, the trials a = 2^-(j0 + 1) .. 2^-(j0 + NTG) in one pass: the
// merit terms of E + a (E_J - E), U + a (U_J - U), formed as the linear-combination kernel forms them
constexpr int DAMP_T1 = 4, DAMP_T2 = DAMP_NT - DAMP_T1;
template <int NTG>
__global__ void __launch_bounds__(256) k_st_damp_trials(const blml_seg* segs, const int* flag, int j0, const double* E,
                                                        const double* EJ, const double* U, const double* UJ,
                                                        const double* c, const double* sg, double* part) {
  if (!flag[blockIdx.y]) return;
  const blml_seg S = segs[blockIdx.y];
  double v[3 * NTG];
#pragma unroll
  for (int q = 0; q < 3 * NTG; q++) v[q] = 0.0;
  const double a0 = ldexp(1.0, -(j0 + 1));
  SEG_LOOP(b, S) {
    const double e0 = E[S.off + b], e1 = EJ[S.off + b], u0 = U[S.off + b], u1 = UJ[S.off + b];
    const double cb = c[S.boff + b], sgb = sg[S.boff + b];
    double a = a0;
#pragma unroll
    for (int k = 0; k < NTG; k++) {
      const double e = fma(a, e1, (1.0 - a) * e0), u = fma(a, u1, (1.0 - a) * u0);
      v[3 * k] += e * u;
      if (cb > 0) { v[3 * k + 1] += cb * log(fabs(e)); if (sgb * e <= 0) v[3 * k + 2] += 1.0; }
      a *= 0.5;
    }
  }
  seg_partials<3 * NTG>(v, part);
}

// the first damped trial (of the first 4) whose merit does not fall below the current one; the coefficients of the
// new iterate over [E, E_J, E_T]; need2 marks the damping fits that try the other 22
__global__ void k_st_damp_pick1(int Fa, const int* fid, const int* live, const int* damp, const double* T1, StState s,
                                double* cE, int* need2) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= Fa) return;
  const int f = fid[j];
  double* ce = cE + 3 * (int64_t)j;
  ce[0] = 0.0; ce[1] = 0.0; ce[2] = 1.0;
  need2[j] = 0;
  if (!live[f] || !damp[j]) return;
  ce[0] = 1.0; ce[2] = 0.0;                       // no step found: the iterate stays
  const double cur = s.cur[f];
  double a = 0.5;
  for (int k = 0; k < DAMP_T1; k++) {
    const double mt = merit_value(T1 + (int64_t)j * 3 * DAMP_T1 + 3 * k, s.n[f]);
    if (mt >= cur) { ce[0] = 1.0 - a; ce[1] = a; s.mJ[f] = mt; return; }
    a *= 0.5;
  }
  need2[j] = 1;
}

__global__ void k_st_damp_pick2(int Fa, const int* fid, const int* need2, const double* T2, StState s, double* cE) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= Fa || !need2[j]) return;
  const int f = fid[j];
  double* ce = cE + 3 * (int64_t)j;
  const double cur = s.cur[f];
  double a = ldexp(1.0, -(DAMP_T1 + 1));
  for (int k = 0; k < DAMP_T2; k++) {
    const double mt = merit_value(T2 + (int64_t)j * 3 * DAMP_T2 + 3 * k, s.n[f]);
    if (mt >= cur) { ce[0] = 1.0 - a; ce[1] = a; s.mJ[f] = mt; return; }
    a *= 0.5;
  }
}

// the Anderson history update fused with its inner products (the real start, one mode): f = E_J - E,
// DX_p = E - pX, DF_p = f - pF, pX = E, pF = f (each formed as the linear-combination kernel forms it), and per fit
// [DF_p . DF_q, DF_q . f] for q < mA (quantities q and AA_MMAX + q)
struct StHist { double* DX[AA_MMAX]; double* DF[AA_MMAX]; };
__global__ void __launch_bounds__(256) k_st_hist(const blml_seg* segs, int mA, int p, const double* EJ, const double* E,
                                                 double* fv, double* pX, double* pF, StHist h, double* part) {
  const blml_seg S = segs[blockIdx.y];
  double v[2 * AA_MMAX];
#pragma unroll
  for (int q = 0; q < 2 * AA_MMAX; q++) v[q] = 0.0;
  SEG_LOOP(b, S) {
    const int64_t i = S.off + b;
    const double ej = EJ[i], e = E[i], px = pX[i], pf = pF[i];
    const double f = fma(-1.0, e, ej), dx = fma(-1.0, px, e), df = fma(-1.0, pf, f);
    fv[i] = f; h.DX[p][i] = dx; h.DF[p][i] = df; pX[i] = e; pF[i] = f;
#pragma unroll
    for (int q = 0; q < AA_MMAX; q++)
      if (q < mA) {
        const double dq = q == p ? df : h.DF[q][i];
        v[q] += df * dq; v[AA_MMAX + q] += dq * f;
      }
  }
  seg_partials<2 * AA_MMAX>(v, part);
}

// out[j * 2 mA + k]: quantity k (k < mA) or AA_MMAX + k - mA of the fit's partials, summed in order (one warp each)
__global__ void k_st_hist_finish(const double* part, int mA, int nblk, double* out) {
  const int j = blockIdx.x, Fa = gridDim.x;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int k = wid; k < 2 * mA; k += nw) {
    const int q = k < mA ? k : AA_MMAX + (k - mA);
    double x = 0.0;
    for (int i = lane; i < nblk; i += 32) x += part[((int64_t)q * Fa + j) * nblk + i];
    x = warp_sum(x);
    if (lane == 0) out[(int64_t)j * 2 * mA + k] = x;
  }
}

// two real linear combinations with the same per-fit coefficients (nt <= 3 terms; zero coefficients skipped, as in
// the linear-combination kernel): oa = sum_i c_i a_i, ob = sum_i c_i b_i (out may alias an input)
struct Terms3 { const double* v[3]; };
__global__ void k_st_lin2(const blml_seg* segs, int nt, const double* coef, Terms3 a, double* oa, Terms3 b,
                          double* ob) {
  const blml_seg S = segs[blockIdx.y];
  const double* cf = coef + (int64_t)blockIdx.y * nt;
  SEG_LOOP(i, S) {
    const int64_t o = S.off + i;
    double xa = 0.0, xb = 0.0;
    for (int q = 0; q < nt; q++) {
      const double c = cf[q];
      if (c != 0.0) { xa += c * a.v[q][o]; xb += c * b.v[q][o]; }
    }
    oa[o] = xa; ob[o] = xb;
  }
}

// merit terms and residual of the real iterate (E, U) in one pass: [sum e u, sum_occ c log|e|, #(sg e <= 0),
// max rho, #NaN rho] (the merit and residual kernels' formulas at scale 1)
__global__ void __launch_bounds__(256) k_st_merit_resid(const blml_seg* segs, const double* E, const double* U,
                                                        const double* c, const double* sg, double* part) {
  const blml_seg S = segs[blockIdx.y];
  double v[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  SEG_LOOP(b, S) {
    const double e = E[S.off + b], u = U[S.off + b], cb = c[S.boff + b];
    v[0] += e * u;
    if (cb > 0) {
      v[1] += cb * log(fabs(e));
      if (sg[S.boff + b] * e <= 0) v[2] += 1.0;
      const double nrm2 = e * e, f = nrm2 / cb, dr = u * f - e;
      const double r = sqrt(dr * dr) / sqrt(fmax(nrm2, 1e-300));
      if (r != r) v[4] += 1.0; else v[3] = fmax(v[3], r);
    }
  }
  seg_partials<5>(v, part, 1u << 3);
}

// out[j * 5 + q] from the fused merit / residual partials (q = 3 a maximum), one warp per quantity
__global__ void k_finish_mr(const double* part, int nblk, double* out) {
  const int j = blockIdx.x, Fa = gridDim.x;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (wid >= 5) return;
  const bool mx = wid == 3;
  double x = mx ? -INFINITY : 0.0;
  for (int i = lane; i < nblk; i += 32) {
    const double y = part[((int64_t)wid * Fa + j) * nblk + i];
    x = mx ? fmax(x, y) : x + y;
  }
  x = mx ? warp_max(x) : warp_sum(x);
  if (lane == 0) out[(int64_t)j * 5 + wid] = x;
}

__global__ void k_st_scale(int Fa, const int* fid, const double* outQ, const double* n, double* sc) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= Fa) return;
  const double Qv = outQ[j], nf = n[fid[j]];
  sc[j] = Qv > 0 ? nf / sqrt(fmax(Qv, 1e-300)) : 1.0;
}

// NaN-propagating min / max (np.minimum / np.maximum)
__device__ __forceinline__ double nmin(double a, double b) { return (a != a || b != b) ? NAN : fmin(a, b); }
__device__ __forceinline__ double nmax(double a, double b) { return (a != a || b != b) ? NAN : fmax(a, b); }

// the end of a start sweep (or the set-up when init): merit and residual of the new iterate, the progress record,
// then the stop rules the next sweep starts with (tol, stall, the sweep cap)
__global__ void k_st_post(int Fa, int init, double tol, long long cap, long long stall, const int* fid, int* live,
                          const blml_seg* segs_c, blml_seg* segs_eff, const double* outMR, StState s) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= Fa) return;
  const int f = fid[j];
  if (!init && !live[f]) { set_live(j, f, 0, live, segs_c, segs_eff); return; }
  const double* mr = outMR + 5 * (int64_t)j;                 // [merit terms (3), max rho, #NaN]
  const double cur = merit_value(mr, s.n[f]);
  const double r = mr[4] > 0 ? NAN : mr[3];
  s.cur[f] = cur; s.res[f] = r;
  int a;
  if (init) {
    s.it[f] = 0; s.best_res[f] = r; s.best_it[f] = 0; s.best_m[f] = cur; s.has_prev[f] = 0;
    a = r >= tol;
  } else {
    const double bm = s.best_m[f];
    if ((r < 0.9 * s.best_res[f]) || (cur > bm + 1e-13 * fabs(bm))) {
      s.best_res[f] = nmin(r, s.best_res[f]); s.best_it[f] = s.it[f]; s.best_m[f] = nmax(cur, bm);
    }
    a = s.active[f] && r >= tol;
  }
  if (a && (long long)(s.it[f] - s.best_it[f]) >= stall) a = 0;
  if (a && s.it[f] >= cap) a = 0;
  if (a) s.it[f]++;
  s.active[f] = a;
  set_live(j, f, a, live, segs_c, segs_eff);
}

// ------------------------------------------------------------------------------------------------ the runner base
#define RC(x) do { int _r = (x); if (_r) return _r; } while (0)
#define KCHECK(where) BLML_CHECK_LAUNCH(where)

struct Runner {
  static constexpr long long kMaxSteps = 4000000;   // a host-side bound on the iterations of one run
  int F = 0, Fa = 0;
  std::vector<blml_seg> segs_all;
  std::vector<int> ids;                 // current compact set (fit ids)
  blml_seg *d_segs_c = nullptr, *d_segs_eff = nullptr;
  int *d_fid = nullptr, *d_live = nullptr, *h_live = nullptr;
  cudaStream_t st = nullptr;
  cudaEvent_t ev = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  long long nodes = 0, steps = 0, replays = 0, rebuilds = 0;
  std::vector<void*> allocs;

  void* dalloc(size_t bytes) {
    void* p = nullptr;
    if (cudaMalloc(&p, std::max<size_t>(bytes, 16)) != cudaSuccess) return nullptr;
    allocs.push_back(p);
    return p;
  }
  int base_init(int F_, const blml_seg* segs) {
    F = F_;
    segs_all.assign(segs, segs + F);
    d_segs_c = (blml_seg*)dalloc(F * sizeof(blml_seg));
    d_segs_eff = (blml_seg*)dalloc(F * sizeof(blml_seg));
    d_fid = (int*)dalloc(F * sizeof(int));
    d_live = (int*)dalloc(F * sizeof(int));
    if (!d_segs_c || !d_segs_eff || !d_fid || !d_live) { set_error("batch runner: device allocation"); return BLML_ERR_CUDA; }
    if (cudaMallocHost(&h_live, F * sizeof(int)) != cudaSuccess) { set_error("batch runner: pinned allocation"); return BLML_ERR_CUDA; }
    RC(cuda_status(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "batch runner stream"));
    RC(cuda_status(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "batch runner event"));
    return BLML_OK;
  }
  void drop_graph() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    exec = nullptr; graph = nullptr;
  }
  void base_free() {
    drop_graph();
    if (st) cudaStreamSynchronize(st);
    for (void* p : allocs) cudaFree(p);
    allocs.clear();
    if (h_live) cudaFreeHost(h_live);
    if (ev) cudaEventDestroy(ev);
    if (st) cudaStreamDestroy(st);
    h_live = nullptr; ev = nullptr; st = nullptr;
  }
  // the compact set: fits `sel`, all live, largest first (launches over fits dispatch their blocks in compact order,
  // so the longest-running fits start first and the small ones fill in behind them)
  int set_compact(const std::vector<int>& sel_in) {
    std::vector<int> sel = sel_in;
    std::stable_sort(sel.begin(), sel.end(), [this](int a, int b) { return segs_all[a].B > segs_all[b].B; });
    ids = sel; Fa = (int)sel.size();
    std::vector<blml_seg> sc(Fa);
    for (int j = 0; j < Fa; j++) sc[j] = segs_all[sel[j]];
    RC(cuda_status(cudaMemcpyAsync(d_segs_c, sc.data(), Fa * sizeof(blml_seg), cudaMemcpyHostToDevice, st), "compact"));
    RC(cuda_status(cudaMemcpyAsync(d_segs_eff, sc.data(), Fa * sizeof(blml_seg), cudaMemcpyHostToDevice, st), "compact"));
    RC(cuda_status(cudaMemcpyAsync(d_fid, sel.data(), Fa * sizeof(int), cudaMemcpyHostToDevice, st), "compact"));
    return cuda_status(cudaStreamSynchronize(st), "compact");
  }
  // the live mask of every fit -> the fits still iterating
  int read_live(std::vector<int>& on) {
    RC(cuda_status(cudaMemcpyAsync(h_live, d_live, F * sizeof(int), cudaMemcpyDeviceToHost, st), "live mask"));
    RC(cuda_status(cudaStreamSynchronize(st), "live mask"));
    on.clear();
    for (int f = 0; f < F; f++)
      if (h_live[f]) on.push_back(f);
    return BLML_OK;
  }
  // capture `ring` iterations enqueued by iter(i) into a graph (launches counted at replay, not at capture)
  template <typename Iter>
  int capture(int ring, Iter iter) {
    drop_graph();
    const long long l0 = blml_launch_count();
    RC(cuda_status(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "graph capture"));
    int rc = BLML_OK;
    for (int i = 0; i < ring && rc == BLML_OK; i++) rc = iter(i);
    cudaGraph_t g = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(st, &g);
    nodes = blml_launch_count() - l0;
    count_launches((int)-nodes);
    if (rc != BLML_OK) { if (g) cudaGraphDestroy(g); return rc; }
    RC(cuda_status(ce, "graph capture end"));
    graph = g;
    RC(cuda_status(cudaGraphInstantiate(&exec, graph, 0), "graph instantiate"));
    rebuilds++;
    return BLML_OK;
  }
  int replay() {
    RC(cuda_status(cudaGraphLaunch(exec, st), "graph launch"));
    count_launches((int)nodes);
    replays++;
    return BLML_OK;
  }
  // run until no fit is live: replay the ring, re-capture over the fits still iterating when they fall to 3/4;
  // before each capture, prep() uploads what the compact set needs
  template <typename Iter, typename Prep>
  int run_rings(int ring, Iter iter, Prep prep) {
    std::vector<int> on;
    for (;;) {
      RC(read_live(on));
      if (on.empty()) return BLML_OK;
      if (!exec || (int)on.size() * 4 <= Fa * 3) {
        RC(set_compact(on));
        RC(prep());
        RC(capture(ring, iter));
      }
      RC(replay());
      steps += ring;
      if (steps > kMaxSteps) { set_error("batch runner: more than %lld iterations", kMaxSteps); return BLML_ERR_ARG; }
    }
  }
  int begin(void* caller) {
    cudaStream_t cs = reinterpret_cast<cudaStream_t>(caller);
    RC(cuda_status(cudaEventRecord(ev, cs), "runner begin"));
    return cuda_status(cudaStreamWaitEvent(st, ev, 0), "runner begin");
  }
  int end(void* caller) {
    cudaStream_t cs = reinterpret_cast<cudaStream_t>(caller);
    RC(cuda_status(cudaEventRecord(ev, st), "runner end"));
    return cuda_status(cudaStreamWaitEvent(cs, ev, 0), "runner end");
  }
  int all_live() {
    std::vector<int> all(F);
    for (int f = 0; f < F; f++) all[f] = f;
    RC(set_compact(all));
    k_fill_int<<<(F + 255) / 256, 256, 0, st>>>(d_live, F, 1);
    KCHECK("runner live");
    return BLML_OK;
  }
};

static inline unsigned nblk(int n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace blml

using namespace blml;

// ------------------------------------------------------------------------------------------------ L-BFGS runner
struct blml_lbfgs_batch_s : Runner {
  int m = 20, dtype = BLML_F64;
  double tol = 1e-5, ftol = 1e-11;
  long long cap = LLONG_MAX;
  blml_group gEU = nullptr, gq = nullptr, gV = nullptr;
  void *E = nullptr, *U = nullptr;
  const void *w = nullptr, *c = nullptr;
  void *g = nullptr, *gn = nullptr, *q = nullptr, *Sq = nullptr, *V = nullptr, *SV = nullptr;
  void *Sh[LB_MMAX] = {}, *Yh[LB_MMAX] = {};
  int h32 = 0;                           // the history (Sh, Yh) in complex64 storage (float64 state only)
  int64_t tot = 0;                       // elements of every mode array (the fits' K B summed)
  void* hvec = nullptr;                  // the history's allocation
  double *part = nullptr, *H1 = nullptr, *H2 = nullptr, *T1 = nullptr, *T2 = nullptr, *outC = nullptr,
         *outD = nullptr, *outE = nullptr;
  double *cq = nullptr, *tA = nullptr, *cS = nullptr, *cY = nullptr, *cG = nullptr, *nqA = nullptr, *scrA = nullptr,
         *ones = nullptr, *sc = nullptr;
  int* need2 = nullptr;
  int* split = nullptr;                  // the block split of the float32 history's kernels (seg_split)
  LbState s{};
  long long* d_caps = nullptr;

  // the history scan: H1 = [S_q . y_p, S_q . g, y_p . y_p, g . g, E . E], H2 = [Y_q . y_p, Y_q . g, ...]
  int hist(int Fa_, const blml_seg* S, int p) {
    const void* a[LB_MMAX];
    for (int i = 0; i < m; i++) a[i] = Sh[i];
    if (h32) RC(seg_dots2_h32(Fa_, S, split, m, a, Yh[p], g, E, part, H1, st));
    else RC(blml_seg_dots2(dtype, Fa_, S, 1, m, a, Yh[p], g, E, part, H1, st));
    for (int i = 0; i < m; i++) a[i] = Yh[i];
    if (h32) return seg_dots2_h32(Fa_, S, split, m, a, Yh[p], g, nullptr, part, H2, st);
    return blml_seg_dots2(dtype, Fa_, S, 1, m, a, Yh[p], g, nullptr, part, H2, st);
  }

  template <typename T>
  int trials(int Fa_, const blml_seg* S) {
    const dim3 grid((unsigned)seg_blocks_for(Fa_), (unsigned)Fa_);
    const int nb = seg_blocks_for(Fa_);
    k_lb_trials<T, LB_T1, true><<<grid, 256, 0, st>>>(S, nullptr, 0, E, q, U, Sq, (const T*)w, part);
    KCHECK("lbfgs trials");
    k_finish_flagged<<<Fa_, 256, 0, st>>>(part, LB_T1 + 4, nb, nullptr, T1);
    KCHECK("lbfgs trials finish");
    k_lb_select1<<<nblk(Fa_, 128), 128, 0, st>>>(Fa_, d_fid, d_live, T1, s, tA, need2);
    KCHECK("lbfgs select");
    k_lb_trials<T, LB_T2, false><<<grid, 256, 0, st>>>(S, need2, LB_T1, E, q, U, Sq, (const T*)w, part);
    KCHECK("lbfgs trials");
    k_finish_flagged<<<Fa_, 256, 0, st>>>(part, LB_T2, nb, need2, T2);
    KCHECK("lbfgs trials finish");
    k_lb_select2<<<nblk(Fa_, 128), 128, 0, st>>>(Fa_, m, d_fid, d_live, T1, T2, need2, s, tA, cS, cY, cG);
    KCHECK("lbfgs select");
    return BLML_OK;
  }

  template <typename T>
  int weights(int Fa_, const blml_seg* S) {
    k_lb_weights<T><<<dim3((unsigned)seg_blocks_for(Fa_), (unsigned)Fa_), 256, 0, st>>>(S, E, U, (const T*)w, V,
                                                                                        part);
    KCHECK("lbfgs weights");
    k_finish_flagged<<<Fa_, 256, 0, st>>>(part, 2, seg_blocks_for(Fa_), nullptr, outD);
    KCHECK("lbfgs weights finish");
    return BLML_OK;
  }

  int iter(int p) {
    const int dt = dtype, Fa_ = Fa;
    const blml_seg* S = d_segs_eff;
    void* sv = st;
    // the block split of this iteration's compact set, for the float32 history's kernels (a fit that converges at the
    // iteration's end keeps its blocks, idle)
    if (h32) RC(seg_split(Fa_, S, split, st));
    // direction from the previous iteration's history scan
    k_lb_dir<<<Fa_, 32, 0, st>>>(m, d_fid, d_live, H1, H2, s, cq);
    KCHECK("lbfgs direction");
    const void* terms[48];
    terms[0] = g;
    for (int i = 0; i < m; i++) { terms[1 + i] = Sh[i]; terms[1 + m + i] = Yh[i]; }
    if (h32) RC(seg_lincomb_mixed(Fa_, S, split, q, 0, 1 + 2 * m, cq, terms, ((1ull << (2 * m)) - 1ull) << 1, st));
    else RC(blml_seg_lincomb(dt, Fa_, S, 1, q, 1 + 2 * m, cq, terms, sv));
    RC(blml_group_matvec_masked(gq, d_fid, Fa_, d_live, sv));
    // every fit's Armijo search (8 trials, then 32 more for the fits that need them), the accepted steps, U = S E
    RC(dt == BLML_F64 ? trials<double>(Fa_, S) : trials<float>(Fa_, S));
    RC(blml_seg_axpy2(dt, Fa_, S, 1, E, q, U, Sq, tA, sv));
    // U + t S q is S(E + t q) up to rounding: float32 state recomputes U = S E exactly at every step (its rounding
    // would otherwise accumulate into the null space of S); float64 once per ring of m steps
    if (dt == BLML_F32 || p == m - 1) RC(blml_group_matvec_masked(gEU, d_fid, Fa_, d_live, sv));
    // gradient at the new point (with Q), the new pair into slot p, g, the residual, the history scan
    RC(dt == BLML_F64 ? weights<double>(Fa_, S) : weights<float>(Fa_, S));
    k_lb_qeff<<<nblk(Fa_, 128), 128, 0, st>>>(Fa_, d_fid, d_live, outD, s, nqA, scrA);
    KCHECK("lbfgs qeff");
    RC(blml_group_matvec_masked(gV, d_fid, Fa_, d_live, sv));
    RC(blml_seg_lgrad_finish(dt, Fa_, S, 1, SV, U, w, nqA, gn, sv));
    terms[0] = q; terms[1] = Sh[p];
    if (h32) RC(seg_lincomb_mixed(Fa_, S, split, Sh[p], 1, 2, cS, terms, 2ull, st));
    else RC(blml_seg_lincomb(dt, Fa_, S, 1, Sh[p], 2, cS, terms, sv));
    terms[0] = g; terms[1] = gn; terms[2] = Yh[p];
    if (h32) RC(seg_lincomb_mixed(Fa_, S, split, Yh[p], 1, 3, cY, terms, 4ull, st));
    else RC(blml_seg_lincomb(dt, Fa_, S, 1, Yh[p], 3, cY, terms, sv));
    terms[0] = gn; terms[1] = g;
    RC(blml_seg_lincomb(dt, Fa_, S, 1, g, 2, cG, terms, sv));
    RC(blml_seg_resid(dt, Fa_, S, 1, E, U, c, scrA, part, outE, sv));
    RC(hist(Fa_, S, p));
    k_lb_post<<<nblk(Fa_, 128), 128, 0, st>>>(Fa_, m, p, tol, ftol, cap, d_fid, d_live, d_segs_c, d_segs_eff, H1,
                                              H2, outD, outE, tA, s);
    KCHECK("lbfgs post");
    return BLML_OK;
  }

  int setup() {
    RC(all_live());
    const int dt = dtype;
    const blml_seg* S = d_segs_eff;
    void* sv = st;
    RC(blml_group_matvec_masked(gEU, d_fid, F, d_live, sv));
    const void* a[1] = {E}; const void* b[1] = {U};
    RC(blml_seg_dots(dt, F, S, 1, 1, a, b, part, outC, sv));
    k_lbi_scale<<<nblk(F, 128), 128, 0, st>>>(F, d_fid, outC, s, sc, nqA, scrA);
    KCHECK("lbfgs set-up");
    const void* t1[1] = {E};
    RC(blml_seg_lincomb(dt, F, S, 1, E, 1, sc, t1, sv));
    t1[0] = U;
    RC(blml_seg_lincomb(dt, F, S, 1, U, 1, sc, t1, sv));
    RC(dt == BLML_F64 ? weights<double>(F, S) : weights<float>(F, S));
    RC(blml_group_matvec_masked(gV, d_fid, F, d_live, sv));
    RC(blml_seg_lgrad_finish(dt, F, S, 1, SV, U, w, nqA, gn, sv));
    t1[0] = gn;
    RC(blml_seg_lincomb(dt, F, S, 1, g, 1, ones, t1, sv));
    RC(blml_seg_resid(dt, F, S, 1, E, U, c, scrA, part, outE, sv));
    if (h32) RC(seg_split(F, S, split, st));
    RC(hist(F, S, 0));                                  // empty history: g . g and E . E for the first direction
    k_lbi_state<<<nblk(F, 128), 128, 0, st>>>(F, m, tol, cap, d_fid, d_live, d_segs_c, d_segs_eff, outD, outE, s);
    KCHECK("lbfgs set-up");
    return BLML_OK;
  }

  void release() {
    if (gEU) blml_group_destroy(gEU);
    if (gq) blml_group_destroy(gq);
    if (gV) blml_group_destroy(gV);
    base_free();
  }
};

// ------------------------------------------------------------------------------------------------- start runner
struct blml_start_batch_s : Runner {
  int mA = 5;
  double tol = 1e-5;
  long long cap = LLONG_MAX, stall = 1000;
  blml_group gEU = nullptr, gJ = nullptr, gA = nullptr;
  double* E = nullptr;
  const double *c = nullptr, *sg = nullptr;
  double *U, *EJ, *UJ, *EA, *UA, *ET, *UT, *fv, *pX, *pF;
  double *DX[AA_MMAX] = {}, *DF[AA_MMAX] = {};
  double *part = nullptr, *outM1, *outM2, *outA, *outQ, *outR, *outDT, *outDT2;
  double *cA, *cT, *cE, *scA, *s0c;
  int *useA, *damp, *need2d;
  std::vector<double> s0_host;
  StState s{};

  int rescale_post(int init) {
    const blml_seg* S = d_segs_eff;
    void* sv = st;
    const int Fa_ = Fa;
    const void* a[1] = {E}; const void* b[1] = {U};
    RC(blml_seg_dots(BLML_F64, Fa_, S, 0, 1, a, b, part, outQ, sv));
    k_st_scale<<<nblk(Fa_, 128), 128, 0, st>>>(Fa_, d_fid, outQ, s.n, scA);
    KCHECK("start scale");
    const dim3 grid((unsigned)seg_blocks_for(Fa_), (unsigned)Fa_);
    k_st_lin2<<<grid, 256, 0, st>>>(S, 1, scA, Terms3{{E, nullptr, nullptr}}, E, Terms3{{U, nullptr, nullptr}}, U);
    KCHECK("start rescale");
    k_st_merit_resid<<<grid, 256, 0, st>>>(S, E, U, c, sg, part);
    KCHECK("start merit / residual");
    RC(seg_finish_mr(Fa_));
    k_st_post<<<nblk(Fa_, 128), 128, 0, st>>>(Fa_, init, tol, cap, stall, d_fid, d_live, d_segs_c, d_segs_eff, outR,
                                              s);
    KCHECK("start post");
    return BLML_OK;
  }

  // the fused merit / residual partials -> outR [Fa x 5] (sums, the residual as a maximum)
  int seg_finish_mr(int Fa_) {
    k_finish_mr<<<Fa_, 256, 0, st>>>(part, seg_blocks_for(Fa_), outR);
    KCHECK("start merit / residual finish");
    return BLML_OK;
  }

  int iter(int p) {
    const blml_seg* S = d_segs_eff;
    void* sv = st;
    const int Fa_ = Fa;
    RC(blml_seg_update_real1(BLML_F64, Fa_, S, E, U, c, sg, s0c, EJ, sv));
    RC(blml_group_matvec_masked(gJ, d_fid, Fa_, d_live, sv));
    RC(blml_seg_merit(BLML_F64, Fa_, S, 0, 0, EJ, UJ, c, sg, part, outM1, sv));
    const void* t[2 + 2 * AA_MMAX];
    const dim3 grid((unsigned)seg_blocks_for(Fa_), (unsigned)Fa_);
    if (mA) {
      StHist h{};
      for (int q = 0; q < mA; q++) { h.DX[q] = DX[q]; h.DF[q] = DF[q]; }
      k_st_hist<<<grid, 256, 0, st>>>(S, mA, p, EJ, E, fv, pX, pF, h, part);
      KCHECK("start history");
      k_st_hist_finish<<<Fa_, 256, 0, st>>>(part, mA, seg_blocks_for(Fa_), outA);
      KCHECK("start history finish");
      k_st_anderson<<<nblk(Fa_, 128), 128, 0, st>>>(Fa_, mA, p, d_fid, d_live, outM1, outA, s, cA, useA);
      KCHECK("start anderson");
      t[0] = E; t[1] = fv;
      for (int q = 0; q < mA; q++) { t[2 + q] = DX[q]; t[2 + mA + q] = DF[q]; }
      RC(blml_seg_lincomb(BLML_F64, Fa_, S, 0, EA, 2 + 2 * mA, cA, t, sv));
      RC(blml_group_matvec_masked(gA, d_fid, Fa_, d_live, sv));
      RC(blml_seg_merit(BLML_F64, Fa_, S, 0, 0, EA, UA, c, sg, part, outM2, sv));
    }
    k_st_take<<<nblk(Fa_, 128), 128, 0, st>>>(Fa_, mA, d_fid, d_live, outM1, outM2, useA, s, cT, damp);
    KCHECK("start take");
    k_st_lin2<<<grid, 256, 0, st>>>(S, 2, cT, Terms3{{EA, EJ, nullptr}}, ET, Terms3{{UA, UJ, nullptr}}, UT);
    KCHECK("start candidate");
    // damped steps: 4 trials, then 22 more for the fits none of the 4 served
    k_st_damp_trials<DAMP_T1><<<grid, 256, 0, st>>>(S, damp, 0, E, EJ, U, UJ, c, sg, part);
    KCHECK("start damping trials");
    k_finish_flagged<<<Fa_, 256, 0, st>>>(part, 3 * DAMP_T1, seg_blocks_for(Fa_), damp, outDT);
    KCHECK("start damping finish");
    k_st_damp_pick1<<<nblk(Fa_, 128), 128, 0, st>>>(Fa_, d_fid, d_live, damp, outDT, s, cE, need2d);
    KCHECK("start damping pick");
    k_st_damp_trials<DAMP_T2><<<grid, 256, 0, st>>>(S, need2d, DAMP_T1, E, EJ, U, UJ, c, sg, part);
    KCHECK("start damping trials");
    k_finish_flagged<<<Fa_, 256, 0, st>>>(part, 3 * DAMP_T2, seg_blocks_for(Fa_), need2d, outDT2);
    KCHECK("start damping finish");
    k_st_damp_pick2<<<nblk(Fa_, 128), 128, 0, st>>>(Fa_, d_fid, need2d, outDT2, s, cE);
    KCHECK("start damping pick");
    k_st_lin2<<<grid, 256, 0, st>>>(S, 3, cE, Terms3{{E, EJ, ET}}, E, Terms3{{U, UJ, UT}}, U);
    KCHECK("start step");
    return rescale_post(0);
  }

  // the kernel values K(0) of the compact set's fits, in compact order
  int upload_s0() {
    std::vector<double> v(Fa);
    for (int j = 0; j < Fa; j++) v[j] = s0_host[ids[j]];
    RC(cuda_status(cudaMemcpyAsync(s0c, v.data(), Fa * sizeof(double), cudaMemcpyHostToDevice, st), "start s0"));
    return cuda_status(cudaStreamSynchronize(st), "start s0");
  }

  int setup() {
    RC(all_live());
    RC(upload_s0());
    RC(blml_seg_start_root(BLML_F64, F, d_segs_eff, c, sg, s0c, E, st));
    RC(blml_group_matvec_masked(gEU, d_fid, F, d_live, st));
    return rescale_post(1);
  }

  void release() {
    if (gEU) blml_group_destroy(gEU);
    if (gJ) blml_group_destroy(gJ);
    if (gA) blml_group_destroy(gA);
    base_free();
  }
};

// one grouped mat-vec over every fit's K modes (the K lattices of fit f from off[f], one plan per fit)
static int make_group(int F, const blml_plan* plans, const blml_seg* segs, int xc, const void* x, void* y,
                      const std::vector<int64_t>& off, blml_group* out) {
  std::vector<int> nb(F);
  for (int f = 0; f < F; f++) nb[f] = segs[f].K;
  return blml_group_create(F, plans, nb.data(), xc, x, off.data(), y, off.data(), out);
}

extern "C" {

int blml_lbfgs_batch_create(int dtype, int F, const blml_seg* segs, const blml_plan* plans, int m, double tol,
                            double ll_tol, int64_t max_iters, const double* n, const void* w, const void* c, void* E,
                            void* U, blml_lbfgs_batch* out) {
  if ((dtype != BLML_F64 && dtype != BLML_F32) || F < 1 || F > 65535 || !segs || !plans || !n || !w || !c || !E ||
      !U || !out || m < 1 || m > LB_MMAX) {
    set_error("blml_lbfgs_batch_create: dtype, 1 <= F <= 65535 fits, 1 <= m <= 20 and every pointer");
    return BLML_ERR_ARG;
  }
  int64_t tot = 0;
  std::vector<int64_t> off(F);
  for (int f = 0; f < F; f++) {
    if (segs[f].K < 1 || segs[f].K > 64 || segs[f].B < 1) {
      set_error("blml_lbfgs_batch_create: 1 to 64 modes (one shared kernel) per fit"); return BLML_ERR_ARG;
    }
    if (!plans[f] || plans[f]->dtype != dtype) { set_error("blml_lbfgs_batch_create: plan dtype"); return BLML_ERR_ARG; }
    off[f] = segs[f].off;
    tot = std::max<int64_t>(tot, segs[f].off + (int64_t)segs[f].K * segs[f].B);
  }
  blml_lbfgs_batch_s* r = new blml_lbfgs_batch_s();
  r->m = m; r->dtype = dtype; r->tol = tol; r->ftol = ll_tol; r->cap = max_iters < 0 ? LLONG_MAX : max_iters;
  r->E = E; r->U = U; r->w = w; r->c = c;
  int rc = r->base_init(F, segs);
  const size_t esz = dtype == BLML_F64 ? 16 : 8;
  char* vec = rc ? nullptr : (char*)r->dalloc(6 * tot * esz);
  char* hv = rc ? nullptr : (char*)r->dalloc(2 * (size_t)m * tot * esz);
  if (!rc && (!vec || !hv)) { set_error("blml_lbfgs_batch_create: vector allocation"); rc = BLML_ERR_CUDA; }
  if (!rc) {
    r->tot = tot; r->hvec = hv;
    void** v6[6] = {&r->g, &r->gn, &r->q, &r->Sq, &r->V, &r->SV};
    for (int i = 0; i < 6; i++) *v6[i] = vec + (size_t)i * tot * esz;
    for (int i = 0; i < m; i++) {
      r->Sh[i] = hv + (size_t)i * tot * esz;
      r->Yh[i] = hv + ((size_t)m + i) * tot * esz;
    }
    cudaMemsetAsync(vec, 0, 6 * tot * esz, r->st);
    cudaMemsetAsync(hv, 0, 2 * (size_t)m * tot * esz, r->st);
    // >= Fa * seg_blocks_for(Fa) for every Fa <= F, and 48 pw >= 43 (SEG_SPLIT_BLOCKS + Fa) for the split scan
    const size_t pw = (size_t)SEG_PART_WIDTH(F);
    const int nq = 48;                    // the widest reduction: blml_seg_dots' 48 accumulators
    const int hs = 2 * m + 3;
    double* scr = (double*)r->dalloc(sizeof(double) * (nq * pw + (size_t)F * (2 * hs + (LB_T1 + 4) + LB_T2 + 1 + 2 + 2 +
                                                                             (1 + 2 * m) + 1 + 2 + 3 + 2 + 1 + 1 + 1 +
                                                                             1)));
    double* stt = (double*)r->dalloc(sizeof(double) * (size_t)F * (7 + (LB_FWIN + 1) + 2 * (size_t)m * m));
    int* ist = (int*)r->dalloc(sizeof(int) * ((size_t)F * (8 + m) + 1));
    r->split = (int*)r->dalloc(sizeof(int) * (size_t)seg_split_ints(F));   // >= seg_split_ints(Fa) for Fa <= F
    if (!scr || !stt || !ist || !r->split) { set_error("blml_lbfgs_batch_create: allocation"); rc = BLML_ERR_CUDA; }
    else {
      r->part = scr;
      double* x = scr + nq * pw;
      auto take = [&](size_t k) { double* p = x; x += k * F; return p; };
      r->H1 = take(hs); r->H2 = take(hs); r->T1 = take(LB_T1 + 4); r->T2 = take(LB_T2); r->outC = take(1);
      r->outD = take(2); r->outE = take(2); r->cq = take(1 + 2 * m); r->tA = take(1); r->cS = take(2);
      r->cY = take(3); r->cG = take(2); r->nqA = take(1); r->scrA = take(1); r->ones = take(1); r->sc = take(1);
      double* y = stt;
      auto tk = [&](size_t k) { double* p = y; y += k * F; return p; };
      r->s.L = tk(1); r->s.Q = tk(1); r->s.Qn = tk(1); r->s.n = tk(1); r->s.res = tk(1); r->s.slope = tk(1);
      r->s.qq = tk(1);
      r->s.mh = tk(LB_FWIN + 1); r->s.SY = tk((size_t)m * m); r->s.YY = tk((size_t)m * m);
      int* z = ist;
      auto ti = [&](size_t k) { int* p = z; z += k * F; return p; };
      r->s.active = ti(1); r->s.it = ti(1); r->s.stop = ti(1); r->s.reset = ti(1); r->s.nh = ti(1); r->s.ok = ti(1);
      r->need2 = ti(1); ti(1);
      r->s.stamp = ti(m); r->s.step = z;
      k_fill_double<<<nblk(F, 256), 256, 0, r->st>>>(r->ones, F, 1.0);
      rc = cuda_status(cudaMemcpyAsync(r->s.n, n, F * sizeof(double), cudaMemcpyHostToDevice, r->st), "lbfgs n");
      if (!rc) rc = cuda_status(cudaStreamSynchronize(r->st), "lbfgs create");
    }
  }
  if (!rc) rc = make_group(F, plans, segs, 1, E, U, off, &r->gEU);
  if (!rc) rc = make_group(F, plans, segs, 1, r->q, r->Sq, off, &r->gq);
  if (!rc) rc = make_group(F, plans, segs, 1, r->V, r->SV, off, &r->gV);
  if (rc) { r->release(); delete r; return rc; }
  *out = r;
  return BLML_OK;
}

int blml_lbfgs_batch_set_history(blml_lbfgs_batch r, int f32) {
  if (!r) { set_error("blml_lbfgs_batch_set_history: null runner"); return BLML_ERR_ARG; }
  if (!f32 || r->h32) return BLML_OK;
  if (r->dtype != BLML_F64) return BLML_OK;          // float32 state: the history is float32 already
  // a complex64 history in place of the complex128 one (half its size); the old allocation is released
  const size_t bytes = 2 * (size_t)r->m * r->tot * 8;
  void* hv = nullptr;
  if (cudaMalloc(&hv, bytes) != cudaSuccess) { set_error("blml_lbfgs_batch_set_history: allocation"); return BLML_ERR_CUDA; }
  int rc = cuda_status(cudaStreamSynchronize(r->st), "blml_lbfgs_batch_set_history");
  if (!rc) rc = cuda_status(cudaMemsetAsync(hv, 0, bytes, r->st), "blml_lbfgs_batch_set_history");
  if (rc) { cudaFree(hv); return rc; }
  for (auto& p : r->allocs)
    if (p == r->hvec) { cudaFree(p); p = hv; break; }
  r->hvec = hv;
  for (int i = 0; i < r->m; i++) {
    r->Sh[i] = (char*)hv + (size_t)i * r->tot * 8;
    r->Yh[i] = (char*)hv + ((size_t)r->m + i) * r->tot * 8;
  }
  r->h32 = 1;
  return BLML_OK;
}

int blml_lbfgs_batch_set_caps(blml_lbfgs_batch r, const int64_t* caps) {
  if (!r || !caps) { set_error("blml_lbfgs_batch_set_caps: null argument"); return BLML_ERR_ARG; }
  if (!r->d_caps) {
    r->d_caps = (long long*)r->dalloc(sizeof(long long) * (size_t)r->F);
    if (!r->d_caps) { set_error("blml_lbfgs_batch_set_caps: allocation"); return BLML_ERR_CUDA; }
  }
  std::vector<long long> c(r->F);
  for (int f = 0; f < r->F; f++) c[f] = caps[f] < 0 ? LLONG_MAX : (long long)caps[f];
  int rc = cuda_status(cudaMemcpyAsync(r->d_caps, c.data(), sizeof(long long) * r->F, cudaMemcpyHostToDevice, r->st),
                       "blml_lbfgs_batch_set_caps");
  if (!rc) rc = cuda_status(cudaStreamSynchronize(r->st), "blml_lbfgs_batch_set_caps");
  if (!rc) r->s.caps = r->d_caps;
  return rc;
}

int blml_lbfgs_batch_run(blml_lbfgs_batch r, void* stream) {
  if (!r) { set_error("blml_lbfgs_batch_run: null runner"); return BLML_ERR_ARG; }
  RC(r->begin(stream));
  RC(r->setup());
  RC(r->run_rings(r->m, [r](int i) { return r->iter(i); }, [] { return (int)BLML_OK; }));
  return r->end(stream);
}

int blml_lbfgs_batch_result(blml_lbfgs_batch r, int64_t* iters, int32_t* stop, double* L, double* Q, double* res) {
  if (!r) { set_error("blml_lbfgs_batch_result: null runner"); return BLML_ERR_ARG; }
  const int F = r->F;
  std::vector<int> it(F), sp(F);
  RC(cuda_status(cudaStreamSynchronize(r->st), "lbfgs result"));
  RC(cuda_status(cudaMemcpy(it.data(), r->s.it, F * sizeof(int), cudaMemcpyDeviceToHost), "lbfgs result"));
  RC(cuda_status(cudaMemcpy(sp.data(), r->s.stop, F * sizeof(int), cudaMemcpyDeviceToHost), "lbfgs result"));
  if (L) RC(cuda_status(cudaMemcpy(L, r->s.L, F * sizeof(double), cudaMemcpyDeviceToHost), "lbfgs result"));
  if (Q) RC(cuda_status(cudaMemcpy(Q, r->s.Q, F * sizeof(double), cudaMemcpyDeviceToHost), "lbfgs result"));
  if (res) RC(cuda_status(cudaMemcpy(res, r->s.res, F * sizeof(double), cudaMemcpyDeviceToHost), "lbfgs result"));
  for (int f = 0; f < F; f++) {
    if (iters) iters[f] = it[f];
    if (stop) stop[f] = sp[f];
  }
  return BLML_OK;
}

int blml_lbfgs_batch_stats(blml_lbfgs_batch r, int64_t* out4) {
  if (!r || !out4) { set_error("blml_lbfgs_batch_stats: bad arguments"); return BLML_ERR_ARG; }
  out4[0] = r->steps; out4[1] = r->replays; out4[2] = r->rebuilds; out4[3] = r->nodes;
  return BLML_OK;
}

int blml_lbfgs_batch_destroy(blml_lbfgs_batch r) {
  if (!r) return BLML_OK;
  r->release();
  delete r;
  return BLML_OK;
}

int blml_start_batch_create(int F, const blml_seg* segs, const blml_plan* plans, int mA, double tol,
                            int64_t max_sweeps, int64_t stall, const double* n, const double* s0, const double* c,
                            const double* sg, double* E, blml_start_batch* out) {
  if (F < 1 || F > 65535 || !segs || !plans || !n || !s0 || !c || !sg || !E || !out || mA < 0 || mA > AA_MMAX) {
    set_error("blml_start_batch_create: 1 <= F <= 65535 fits, 0 <= anderson <= 8 and every pointer");
    return BLML_ERR_ARG;
  }
  int64_t tot = 0;
  std::vector<int64_t> off(F);
  for (int f = 0; f < F; f++) {
    if (segs[f].K != 1 || segs[f].B < 1) { set_error("blml_start_batch_create: one mode per fit"); return BLML_ERR_ARG; }
    if (!plans[f] || plans[f]->dtype != BLML_F64) { set_error("blml_start_batch_create: float64 plans"); return BLML_ERR_ARG; }
    off[f] = segs[f].off;
    tot = std::max<int64_t>(tot, segs[f].off + segs[f].B);
  }
  blml_start_batch_s* r = new blml_start_batch_s();
  r->mA = mA; r->tol = tol; r->cap = max_sweeps < 0 ? LLONG_MAX : max_sweeps; r->stall = stall;
  r->E = E; r->c = c; r->sg = sg;
  r->s0_host.assign(s0, s0 + F);
  int rc = r->base_init(F, segs);
  double* vec = rc ? nullptr : (double*)r->dalloc((10 + 2 * (size_t)mA) * tot * sizeof(double));
  if (!rc && !vec) { set_error("blml_start_batch_create: vector allocation"); rc = BLML_ERR_CUDA; }
  if (!rc) {
    double** v10[10] = {&r->U, &r->EJ, &r->UJ, &r->EA, &r->UA, &r->ET, &r->UT, &r->fv, &r->pX, &r->pF};
    for (int i = 0; i < 10; i++) *v10[i] = vec + (size_t)i * tot;
    for (int i = 0; i < mA; i++) { r->DX[i] = vec + (10 + (size_t)i) * tot; r->DF[i] = vec + (10 + (size_t)mA + i) * tot; }
    cudaMemsetAsync(vec, 0, (10 + 2 * (size_t)mA) * tot * sizeof(double), r->st);
    const int nq = 3 * DAMP_NT;           // the widest reduction: the damping trials' 78 quantities
    const size_t pw = (size_t)SEG_PART_WIDTH(F);   // >= Fa * seg_blocks_for(Fa) for every Fa <= F
    double* scr = (double*)r->dalloc(sizeof(double) * (nq * pw + (size_t)F *
                                     (3 + 3 + 2 * AA_MMAX + 1 + 5 + nq + nq + (2 + 2 * AA_MMAX) + 2 + 3 + 1 + 1)));
    double* stt = (double*)r->dalloc(sizeof(double) * (size_t)F * (8 + (size_t)AA_MMAX * AA_MMAX));
    int* ist = (int*)r->dalloc(sizeof(int) * (size_t)F * (6 + AA_MMAX + 3));
    if (!scr || !stt || !ist) { set_error("blml_start_batch_create: allocation"); rc = BLML_ERR_CUDA; }
    else {
      r->part = scr;
      double* x = scr + nq * pw;
      auto take = [&](size_t k) { double* p = x; x += k * F; return p; };
      r->outM1 = take(3); r->outM2 = take(3); r->outA = take(2 * AA_MMAX);
      r->outQ = take(1); r->outR = take(5); r->outDT = take(nq); r->outDT2 = take(nq);
      r->cA = take(2 + 2 * AA_MMAX); r->cT = take(2); r->cE = take(3); r->scA = take(1); r->s0c = take(1);
      double* y = stt;
      auto tk = [&](size_t k) { double* p = y; y += k * F; return p; };
      r->s.n = tk(1); r->s.s0 = tk(1); r->s.cur = tk(1); r->s.res = tk(1); r->s.best_res = tk(1); r->s.best_m = tk(1);
      r->s.mJ = tk(1); tk(1); r->s.G = tk((size_t)AA_MMAX * AA_MMAX);
      int* z = ist;
      auto ti = [&](size_t k) { int* p = z; z += k * F; return p; };
      r->s.valid = ti(AA_MMAX); r->s.has_prev = ti(1); r->s.best_it = ti(1); r->s.it = ti(1); r->s.active = ti(1);
      r->useA = ti(1); r->damp = ti(1); r->need2d = ti(1);
      cudaMemsetAsync(r->s.G, 0, sizeof(double) * (size_t)F * AA_MMAX * AA_MMAX, r->st);
      cudaMemsetAsync(r->s.valid, 0, sizeof(int) * (size_t)F * AA_MMAX, r->st);
      cudaMemsetAsync(r->outM2, 0, sizeof(double) * 3 * (size_t)F, r->st);
      cudaMemsetAsync(r->useA, 0, sizeof(int) * (size_t)F, r->st);
      rc = cuda_status(cudaMemcpyAsync(r->s.n, n, F * sizeof(double), cudaMemcpyHostToDevice, r->st), "start n");
      if (!rc) rc = cuda_status(cudaStreamSynchronize(r->st), "start create");
    }
  }
  if (!rc) rc = make_group(F, plans, segs, 0, E, r->U, off, &r->gEU);
  if (!rc) rc = make_group(F, plans, segs, 0, r->EJ, r->UJ, off, &r->gJ);
  if (!rc) rc = make_group(F, plans, segs, 0, r->EA, r->UA, off, &r->gA);
  if (rc) { r->release(); delete r; return rc; }
  *out = r;
  return BLML_OK;
}

int blml_start_batch_run(blml_start_batch r, void* stream) {
  if (!r) { set_error("blml_start_batch_run: null runner"); return BLML_ERR_ARG; }
  RC(r->begin(stream));
  RC(r->setup());
  const int ring = r->mA > 0 ? r->mA : 1;
  RC(r->run_rings(ring, [r](int i) { return r->iter(i); }, [r] { return r->upload_s0(); }));
  return r->end(stream);
}

int blml_start_batch_result(blml_start_batch r, int64_t* sweeps, double* res) {
  if (!r) { set_error("blml_start_batch_result: null runner"); return BLML_ERR_ARG; }
  const int F = r->F;
  std::vector<int> it(F);
  RC(cuda_status(cudaStreamSynchronize(r->st), "start result"));
  RC(cuda_status(cudaMemcpy(it.data(), r->s.it, F * sizeof(int), cudaMemcpyDeviceToHost), "start result"));
  if (res) RC(cuda_status(cudaMemcpy(res, r->s.res, F * sizeof(double), cudaMemcpyDeviceToHost), "start result"));
  if (sweeps)
    for (int f = 0; f < F; f++) sweeps[f] = it[f];
  return BLML_OK;
}

int blml_start_batch_stats(blml_start_batch r, int64_t* out4) {
  if (!r || !out4) { set_error("blml_start_batch_stats: bad arguments"); return BLML_ERR_ARG; }
  out4[0] = r->steps; out4[1] = r->replays; out4[2] = r->rebuilds; out4[3] = r->nodes;
  return BLML_OK;
}

int blml_start_batch_destroy(blml_start_batch r) {
  if (!r) return BLML_OK;
  r->release();
  delete r;
  return BLML_OK;
}

}
