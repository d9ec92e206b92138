/* libblml_b200 -- the C ABI of the B200 engine for BLML's binned fitting path.
 *
 * Every entry point takes plain device pointers (e.g. torch tensors' data_ptr()), sizes and a CUDA stream
 * (cudaStream_t passed as void*), and returns 0 on success or a negative BLML_ERR_* code (blml_last_error() gives
 * the message). Arrays of modes are (K, B) row-major, B = the number of lattice bins; complex arrays are
 * interleaved (re, im) pairs (torch complex64 / complex128). `dtype` selects float64 (BLML_F64) or float32
 * (BLML_F32) storage; every reduction accumulates in float64 and is deterministic (fixed-order block partials:
 * `part` holds nq * blml_reduce_blocks() doubles, `out` receives nq doubles, both on the device).
 *
 * The reference (rahuljhu/band-limited-ml) is Python over NumPy/CuPy; each entry point below names the method
 * whose arithmetic it replaces (file:line in the reference).
 */
#ifndef BLML_B200_H
#define BLML_B200_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { BLML_OK = 0, BLML_ERR_ARG = -1, BLML_ERR_CUDA = -2, BLML_ERR_WORKSPACE = -3, BLML_ERR_UNSUPPORTED = -4,
       BLML_ERR_TIMEOUT = -5 };
enum { BLML_F64 = 0, BLML_F32 = 1 };
/* mat-vec engines: SIMT contraction (float64 or float32), or tcgen05 tensor cores with split-TF32 operands
   (float32 storage, three products per term, FP32 accumulation in TMEM) */
enum { BLML_ENGINE_SIMT = 0, BLML_ENGINE_TC = 1 };
/* routes of the SIMT engine: restricted-transform contractions, or FFTs of the lattice rows and columns when the
   kernel is a DFT mask (2-D, every axis one period, integer harmonics; sides 2^a 3^b up to 4,096) */
enum { BLML_ROUTE_AUTO = 0, BLML_ROUTE_CONTRACT = 1, BLML_ROUTE_FFT = 2 };

typedef struct blml_plan_s* blml_plan;

const char* blml_last_error(void);
int blml_abi_version(void);
/* blocks of every reduction grid: `part` buffers hold nq * blml_reduce_blocks() doubles */
int blml_reduce_blocks(void);
/* cumulative number of kernels the library has launched in this process (for launch accounting) */
int64_t blml_launch_count(void);

/* ---- the per-mode Gram mat-vec S_k e (replaces _ModeKernel + BLMLBinned._S, blml_binned.py:49-101, 156-168) ----
 * The mode's kernel on a d-dim lattice of `shape`, given as restricted transforms: per axis a nfreq[a] frequencies
 * (cycles per lattice index, concatenated over axes in `freqs`) and a weight tensor over the product frequency grid
 * (prod nfreq doubles, row-major): S e = sum_q W_q v_q v_q^H e, v_q(j) = exp(2 pi i sum_a nu_{a,q_a} j_a). */
int blml_plan_create(int d, const int64_t* shape, const int32_t* nfreq, const double* freqs, const double* weights,
                     int dtype, int engine, blml_plan* plan);
int blml_plan_destroy(blml_plan plan);
/* bytes of workspace one blml_matvec call over nbatch lattices needs */
int64_t blml_matvec_workspace(blml_plan plan, int nbatch);
/* y[b] = S x[b] for b < nbatch lattices; x real (x_complex = 0: y real) or complex */
int blml_matvec(blml_plan plan, const void* x, void* y, int nbatch, int x_complex, void* ws, int64_t ws_bytes,
                void* stream);
/* synchronises the device and reports whether a tensor-core mat-vec gave up on a bounded wait since the plan was
   made (BLML_ERR_TIMEOUT; the results of that call are invalid) or BLML_OK */
int blml_plan_status(blml_plan plan);
/* choose the route of blml_matvec (BLML_ROUTE_AUTO: the FFT route wherever the plan has one); BLML_ERR_UNSUPPORTED
   when the FFT route is asked of a kernel without one. Both routes apply the same operator; the FFT route is the
   reference's own FFT convolution (blml_binned.py:156-168) restricted to the band's harmonics. */
int blml_plan_set_route(blml_plan plan, int route);
/* the route blml_matvec takes (BLML_ROUTE_CONTRACT or BLML_ROUTE_FFT) */
int blml_plan_route(blml_plan plan);

/* ---- grouped mat-vecs: many plans (fits of uneven lattice size and band) applied in one launch per stage ----
 * Problem g: y_base[y_off[g] ...] = S_g x_base[x_off[g] ...] over nbatch[g] lattices of plan g (SIMT engine); every
 * plan of a group has the same dimension count and dtype; offsets count elements (complex elements when
 * x_complex). The group owns its intermediate buffers and the per-stage descriptor arrays. Replaces the reference's
 * sequential per-fit _Sall calls of a cut-off sweep (selector.py:488-553 calling blml_binned.py:156-168). */
typedef struct blml_group_s* blml_group;
int blml_group_create(int G, const blml_plan* plans, const int* nbatch, int x_complex, const void* x_base,
                      const int64_t* x_off, void* y_base, const int64_t* y_off, blml_group* group);
int blml_group_matvec(blml_group group, void* stream);
/* the same for the n problems g = subset[i] (device int array; null: problems 0 .. n-1), skipping those with
   live[g] == 0 (device int array over all G problems, or null), both read when the kernels run, so a captured CUDA
   graph follows problems that stop between its replays */
int blml_group_matvec_masked(blml_group group, const int* subset, int n, const int* live, void* stream);
int blml_group_destroy(blml_group group);
/* the route of every stage launch of a group: the FFT route (three launches: row FFTs, column FFT x weight x inverse
   FFT, inverse row FFTs) when every plan has one and BLML_ROUTE_AUTO, else the 2 d restricted-transform stages */
int blml_group_set_route(blml_group group, int route);
int blml_group_route(blml_group group);
/* the FFT route's launch shape for descriptors made from now on (plans' single mat-vecs, groups created later): the
   shared memory a CTA aims for (8 KiB .. 72 KiB; several rows per CTA up to it) and the most columns per CTA of the
   column stage. The package sets the shape its autotuner measured fastest (bench.py --tune) at import. */
int blml_fft_set_shape(int cta_bytes, int max_cols);
int blml_fft_get_shape(int* cta_bytes, int* max_cols);

/* ---- coordinate (Jacobi) update of every bin (BLMLBinned._update / _secular / _cd_root,
 *      blml_binned.py:184-206, 1549-1573; cd_root blml_trivial.py:84-89) ----
 * psd = 0: real rank 1, out = sg * cd_root(sg * (U - s0 E), c, s0) on occupied bins (c > 0), 0 elsewhere.
 * psd = 1: complex and/or rank K; the closed form when every s_k is equal, else the safeguarded secular root.
 * s: K host doubles (K(0) of each mode). */
int blml_jacobi_update(int dtype, int K, int64_t B, int cplx, int psd, const double* s, const void* E, const void* U,
                       const void* c, const void* sg, void* out, void* stream);

/* ---- merit terms (BLMLBinned._merit, blml_binned.py:171-182) ----
 * psd: out[0] = sum_b c_b log max(F_b, 1e-30), F_b = sum_k |U_kb|^2; out[1] = Q = Re sum conj(E) U; out[2] = 0.
 * real rank 1: out[0] = sum e u, out[1] = sum_occ c log|e|, out[2] = #occupied bins with sg e <= 0. nq = 3. */
int blml_merit_terms(int dtype, int K, int64_t B, int cplx, int psd, const void* E, const void* U, const void* c,
                     const void* sg, double* part, double* out, void* stream);

/* ---- stationarity residual max_b rho_b of (scale E, scale U) (BLMLBinned._resid, blml_binned.py:216-220);
 *      out[0] = the largest finite rho_b, out[1] = the number of bins whose rho_b is NaN; nq = 2 */
int blml_resid(int dtype, int K, int64_t B, int cplx, const void* E, const void* U, const void* c, double scale,
               double* part, double* out, void* stream);

/* ---- real inner products Re sum conj(a_i) b_i over n scalars (complex arrays: 2n reals) in float64, npairs <= 64
 *      pairs (32 per pass) (_rdot, _anderson_mix, the L-BFGS dots; blml_binned.py:1463-1482, 290-335) ----
 * a, b: host arrays of device pointers. nq = npairs. */
int blml_dots(int dtype, int64_t n, int npairs, const void* const* a, const void* const* b, double* part,
              double* out, void* stream);

/* ---- out = sum_i coef_i v_i over n scalars, nterms <= 64 (out may alias any v_i): Anderson mixing, damping, L-BFGS
 *      directions and steps (blml_binned.py:243-258, 307-321, 1475-1478) ---- */
int blml_lincomb(int dtype, int64_t n, void* out, int nterms, const double* coef, const void* const* v, void* stream);

/* ---- out[k, b] = x[k, b] * r[b] (r real, same dtype as x): masks and diagonal scalings ---- */
int blml_mul_bins(int dtype, int K, int64_t B, int cplx, const void* x, const void* r, void* out, void* stream);

/* ---- likelihood gradient pieces (BLMLBinned._lgrad, blml_binned.py:278-288; canonical form :345-349) ----
 * weights: F = sum_k |U_k|^2; V = vscale * w / F * U on occupied bins (0 elsewhere); out[0] = sum_occ w log F. nq = 1
 * finish:  g = 2 (SV - nq U) on occupied bins, 0 elsewhere. */
int blml_lgrad_weights(int dtype, int K, int64_t B, int cplx, const void* U, const void* w, double vscale, void* V,
                       double* part, double* out, void* stream);
int blml_lgrad_finish(int dtype, int K, int64_t B, int cplx, const void* SV, const void* U, const void* w, double nq,
                      void* g, void* stream);
/* ---- fc gradients of a fit (blml_binned.py:520-628: fc_grad, param_grad, implicit_grad) ----
   the score P = sum_b m_b log(F_b / Z + eps) / sum m: V_k = wn U_k with wn = m / max(F + add, 1e-300) on bins with
   m > 0 (add = eps Z), out[0] = sum wn F, out[1] = sum m (blml_binned.py:551-553) */
int blml_pgrad_weights(int dtype, int K, int64_t B, int cplx, const void* U, const void* m, double add, void* V,
                       double* part, double* out, void* stream);                                   /* nq = 2 */
/* the Hessian of the minimised objective (blml_binned.py:596-606), its bin term:
   out_k = (w / F) dU_k - (w dF / F^2) U_k, dF = 2 Re sum_k conj(U_k) dU_k, on occupied bins (0 elsewhere) */
int blml_hvp_inner(int dtype, int K, int64_t B, int cplx, const void* U, const void* dU, const void* w, void* out,
                   void* stream);
/* d(gradient)/dlog fc of mode k at fixed coefficients (blml_binned.py:610-628), its bin terms for dUk = dS E_k:
   T_j = -(w dF / F^2) U_j (+ (w / F) dUk for j = k), Wk = (w / F) U_k, dF = 2 Re conj(U_k) dUk (occupied bins) */
int blml_mixed_terms(int dtype, int K, int64_t B, int cplx, const void* U, int k, const void* dUk, const void* w,
                     void* T, void* Wk, void* stream);
/* the real rank-1 objective's Hessian times D (blml_binned.py:599-601): out = dU + (c / e^2) D where c > 0 */
int blml_hvp_real1(int dtype, int64_t B, const void* D, const void* E, const void* c, const void* dU, void* out,
                   void* stream);

/* ---- streaming fits (BLMLBinnedStreaming, blml_binned.py:1040-1112) ----
   counts: out = a w + b m, clamped at 0 when clamp (decay w + batch; the held counts less a batch, :1070-1074) */
int blml_counts_axpy(int dtype, int64_t B, double a, const void* w, double b, const void* m, int clamp, void* out,
                     void* stream);
/* out = num / den where den > 0, else 0 (each bin's remaining share after leaving a batch out, :1075) */
int blml_bin_ratio(int dtype, int64_t B, const void* num, const void* den, void* out, void* stream);
/* out_k = Eu_k on occupied bins whose coefficients are all 0 (newly occupied: their own root from S e, :1098-1100),
   E_k elsewhere */
int blml_new_bins(int dtype, int K, int64_t B, int cplx, const void* E, const void* Eu, const void* w, void* out,
                  void* stream);
/* a hill-climb candidate's paired gain on a batch m (blml_binned.py:765-770): over bins with m > 0,
   dl = log(da sa + eps) - log(db sb + eps); out = [sum m dl, sum m dl^2, sum m] */
int blml_gain_sums(int dtype, int64_t B, const void* da, double sa, const void* db, double sb, const void* m, double eps,
                   double* part, double* out, void* stream);                                       /* nq = 3 */

/* ---- block coordinate descent of the point / lattice fits (blml_trivial.py:2860-3035), float64 state ----
   root:   d[j] = cd_root(Se[b] - sbb e[b], c[b], sbb) - e[b], b = I[j] (the block's exact roots, less e)
   search: out[0] = d . Se[I], out[1] = d . v[I] (v = S[:, I] d), out[2] = #{e[I] > 0}, out[3 + k] =
           sum_{e > 0} c log1p(2^-k d / e), out[34 + k] = #{1 + 2^-k d / e <= 0}, k < 31 (cd_line_search, :92-104)
   apply:  e[I[j]] += t d[j];   gather: out[j, :] = src[I[j], :] (int64 rows, d columns)
   indices outside [0, B) are skipped */
int blml_block_root(int m, const int64_t* I, int64_t B, const double* e, const double* Se, const double* c, double sbb,
                    double* d, void* stream);
int blml_block_search(int m, const int64_t* I, int64_t B, const double* e, const double* d, const double* Se,
                      const double* v, const double* c, double* out, void* stream);        /* out: 65 doubles */
int blml_block_apply(int m, const int64_t* I, int64_t B, const double* d, double t, double* e, void* stream);
int blml_gather_rows_i64(int m, int d, const int64_t* src, const int64_t* I, int64_t B, int64_t* out, void* stream);

/* ---- the fitted amplitude at arbitrary points (BLMLQuick.sqrt_density / predict, blml_trivial.py:3288-3320) ----
   g[i] = sum_b e[b] prod_c K_c(X[i, c] - Z[b, c]) with the exact one-column kernels (X: m x d, Z: B x d row-major
   float64, d <= 8): sinc f sinc(f t); slits f sinc(f t) - fi sinc(fi t); dirichlet
   (sin(pi M u / P) - sin(pi Mi u / P)) / (P sin(pi u / P)), u = |t| folded into [0, P / 2], (M - Mi) / P at u = 0;
   ball (a radial unit over a group of columns, blml_trivial.py:580-591): every column of the group has kind ball,
   f its fc and M the group's column bit mask; the group's first column holds fi = prod fc, Mi = D (the group size)
   and P = p(0), the others fi = 0; the unit's value is fi p(||fc t||), p(s) = (1/2)^(D/2) J_(D/2)(pi s) / s^(D/2) */
enum { BLML_PT_SINC = 0, BLML_PT_SLITS = 1, BLML_PT_DIRICHLET = 2, BLML_PT_BALL = 3 };
typedef struct { int kind; int M, Mi; double f, fi, P; } blml_point_col;
typedef struct { blml_point_col c[8]; } blml_point_cols;
int blml_point_rows(int64_t m, int d, const double* X, int64_t B, const double* Z, const double* e,
                    const blml_point_col* cols, double* g, void* stream);
/* ---- point sums of several densities (blml_local.py:555-560 point_rows_multi: FusedFit's joint and marginals at
 *      points, K10 of blml_local_gpu.py): g[i * Mm + q] = sum_b W[b * Mm + q] prod_u (bit u of masks[q] ? K_u : 1),
 *      unit_of[c] the kernel unit of column c (one-column units first, then groups), U units, 1 <= Mm <= 8 ---- */
int blml_point_rows_multi(int64_t m, int d, const double* X, int64_t B, const double* Z, const double* W, int Mm,
                          const blml_point_col* cols, const int* unit_of, int U, const unsigned* masks, double* g,
                          void* stream);

/* ---- the binned fit at arbitrary points for harmonic kernels (BLMLBinned.sqrt_density / predict / predict_grid,
 *      blml_binned.py:451-500) ----
 * spectrum: spec (nbatch x prod nfreq, complex of the plan's dtype, natural order) = W (v^H x), the forward half of
 * blml_matvec (SIMT plans); workspace blml_spectrum_workspace bytes.
 * planewave: g[i] = sum_{q1, q2} spec[q1 H2 + q2] exp(2 pi i (f1[q1] U[i, 0] + f2[q2] U[i, 1])) for m points U (m x 2,
 * lattice coordinates (x - origin) / h), frequencies in cycles per lattice index, spec and g complex128; a 1-D
 * kernel is H1 = 1, f1 = {0}, U[i, 0] = 0. Exact for pball groups and dirichlet columns, whose kernels are sums of
 * harmonics (the reference evaluates the same sums, blml_trivial.py:632-665). */
int64_t blml_spectrum_workspace(blml_plan plan, int nbatch);
int blml_spectrum(blml_plan plan, const void* x, void* spec, int nbatch, int x_complex, void* ws, int64_t ws_bytes,
                  void* stream);
int blml_planewave_points(int H1, int H2, const double* f1, const double* f2, const double* spec, int64_t m,
                          const double* U, double* g, void* stream);

/* ---- one Armijo trial of the L-BFGS line search (BLMLBinned._solve_lbfgs, blml_binned.py:316-321) ----
 * En = E + t q and Un = U + t Sq (S linear: U + t S q = S(E + t q)), both written; out[0] = sum_occ w log F(Un),
 * out[1] = Re <En, Un>, from which L(En) = out[0] - n log out[1]. nq = 2. */
int blml_lbfgs_trial(int dtype, int K, int64_t B, int cplx, const void* E, const void* q, const void* U,
                     const void* Sq, const void* w, double t, void* En, void* Un, double* part, double* out,
                     void* stream);

/* ---- fit outputs (BLMLBinned._finish, blml_binned.py:438-445): density = F / n^2; out[0] = sum_occ w log density */
int blml_finish(int dtype, int K, int64_t B, int cplx, const void* U, const void* w, double inv_n2, void* density,
                double* part, double* out, void* stream);

/* ---- lattice score (BLMLBinned.log_density / _val_score, blml_binned.py:630-645): out[0] = sum over m_b > 0 of
 *      m_b log max(F_b inv_z + eps, 1e-300), out[1] = sum m_b; m (B) in the fit dtype. nq = 2 ---- */
int blml_log_score(int dtype, int K, int64_t B, int cplx, const void* U, const void* m, double inv_z, double eps,
                   double* part, double* out, void* stream);

/* ---- start (BLMLBinned._start / _fill_modes, blml_binned.py:415-436) ----
 * start_root: e0 = sg sqrt(c / s0) on occupied bins, 0 elsewhere (real, dtype).
 * fill_modes: with phases, E[0] *= exp(i pn z); modes k >= kk: E[k] = pn |E[0]| z_k (complex: (zr + i zi) / sqrt 2).
 * z: float64 normals on the device in the order the reference draws them (phases first, then per mode re, im). */
int blml_start_root(int dtype, int64_t B, const void* c, const void* sg, double s0, void* e0, void* stream);
int blml_fill_modes(int dtype, int K, int64_t B, int cplx, int kk, int phases, double pn, const double* z, void* E,
                    void* stream);

/* ---- certificate weights (BLMLBinned.certificate, blml_binned.py:506-507): dh = sqrt(sum_k |E_k|^2 / w) on
 *      occupied bins, 0 elsewhere, float64 output whatever the fit dtype ---- */
int blml_cert_weights(int dtype, int K, int64_t B, int cplx, const void* E, const void* w, double* dh, void* stream);

/* ---- segmented (batched) solver kernels: F independent fits in lockstep, one launch per phase ----
 * Fit f owns elements [off, off + K B) of every flat mode array (its (K, B) block) and [boff, boff + B) of every flat
 * bin array (counts, signs); `segs` is a device array of F entries. Per-fit scalars are device arrays of F doubles
 * (coefficient tables: F x nterms). Reductions give out[f * nq + q] (part: F * nq * blml_seg_blocks() doubles, an
 * upper bound: a launch over F fits uses min(256, max(16, 16384 / F)) blocks per fit; blml_seg_dots takes nq = 48,
 * blml_seg_dots2 nq = 43).
 * These are the reference's single-fit operations (blml_binned.py:171-220, 278-355, 415-445, 630-645) applied to a
 * sweep of fits at once, as selector._search / the cut-off sweeps run them one after another. */
typedef struct { int64_t off; int64_t boff; int64_t B; int32_t K; int32_t pad; } blml_seg;
int blml_seg_blocks(void);
int blml_seg_start_root(int dtype, int F, const blml_seg* segs, const void* c, const void* sg, const double* s0,
                        void* e0, void* stream);
int blml_seg_update_real1(int dtype, int F, const blml_seg* segs, const void* E, const void* U, const void* c,
                          const void* sg, const double* s0, void* out, void* stream);
int blml_seg_merit(int dtype, int F, const blml_seg* segs, int cplx, int psd, const void* E, const void* U,
                   const void* c, const void* sg, double* part, double* out, void* stream);        /* nq = 3 */
int blml_seg_resid(int dtype, int F, const blml_seg* segs, int cplx, const void* E, const void* U, const void* c,
                   const double* scale, double* part, double* out, void* stream);                   /* nq = 2 */
int blml_seg_dots(int dtype, int F, const blml_seg* segs, int cplx, int npairs, const void* const* a,
                  const void* const* b, double* part, double* out, void* stream);                   /* npairs <= 48 */
/* the L-BFGS history scan (blml_binned.py:297-313 reads the same products pair by pair): for np <= 20 vectors a_q,
   out[f * (2 np + 3) + .] = [a_q . b0 (np), a_q . b1 (np), b0 . b0, b1 . b1, x . x] (x may be null: 0) */
int blml_seg_dots2(int dtype, int F, const blml_seg* segs, int cplx, int np, const void* const* a, const void* b0,
                   const void* b1, const void* x, double* part, double* out, void* stream);
int blml_seg_lincomb(int dtype, int F, const blml_seg* segs, int cplx, void* out, int nterms, const double* coef,
                     const void* const* v, void* stream);                                           /* nterms <= 48 */
int blml_seg_lgrad_weights(int dtype, int F, const blml_seg* segs, int cplx, const void* U, const void* w,
                           const double* vscale, void* V, double* part, double* out, void* stream);  /* nq = 1 */
int blml_seg_lgrad_finish(int dtype, int F, const blml_seg* segs, int cplx, const void* SV, const void* U,
                          const void* w, const double* nq, void* g, void* stream);
/* every fit's Armijo search in one pass: out[f * 43 + j] = sum_occ w log F(U + 2^-j S q) for j < 40, then
   <q, U>, <E, S q>, <q, S q> (blml_binned.py:316-321 evaluates the same trials one at a time) */
int blml_seg_trials(int dtype, int F, const blml_seg* segs, int cplx, const void* E, const void* q, const void* U,
                    const void* Sq, const void* w, double* part, double* out, void* stream);
int blml_seg_axpy2(int dtype, int F, const blml_seg* segs, int cplx, void* E, const void* q, void* U, const void* Sq,
                   const double* t, void* stream);
int blml_seg_finish(int dtype, int F, const blml_seg* segs, int cplx, const void* U, const void* w,
                    const double* inv_n2, void* density, double* part, double* out, void* stream);  /* nq = 1 */
int blml_seg_log_score(int dtype, int F, const blml_seg* segs, int cplx, const void* U, const void* m,
                       const double* inv_z, double eps, double* part, double* out, void* stream);   /* nq = 2 */
/* the cut-off search's validation score (replaces the objective of select_counts, selector.py:712-716, and of
   dslit_job.py:165-168, one fit at a time): per fit, with p = max(density, 1e-300) over every bin of its lattice,
   out[3 f + 0..2] = sum_b p, sum_b va log p, sum_b va; score = (sum va log p - sum va log sum p) / sum va.
   density and va are real arrays of the fit dtype laid out like the bins (boff) */
int blml_seg_val_score(int dtype, int F, const blml_seg* segs, const void* density, const void* va, double* part,
                       double* out, void* stream);                                                  /* nq = 3 */
int blml_seg_phases(int dtype, int F, const blml_seg* segs, double pn, const double* z, void* E, void* stream);
int blml_seg_real_to_complex(int dtype, int F, const blml_seg* real_segs, const blml_seg* cplx_segs, const void* er,
                             void* E, void* stream);
/* the certificate of every fit (BLMLBinned.certificate, blml_binned.py:501-518): the diagonal scaling
 * dh = sqrt(sum_k |e_kb|^2 / w_b) of D^1/2 S D^1/2 on occupied bins, float64 per bin in the boff layout (E complex) */
int blml_seg_cert_weights(int dtype, int F, const blml_seg* segs, const void* E, const void* w, double* dh,
                          void* stream);
/* rank growth towards a certified fit: the certificate lambda_max(D^1/2 S D^1/2) / n <= 1 (blml_binned.py:501-518)
 * holds at the optimum of the convex lift, which a fit with enough shared modes reaches; the next fit starts from the
 * current modes plus the top eigenvector's direction (the reference's fit with K shared modes and init=,
 * blml_binned.py:403-408). E_new (K_f + 1 modes, new_segs layout) = E's K_f modes, then scale_f dh v as the new mode
 * (v: float64 per bin, boff layout; scale: F device doubles). No single reference function does this step. */
int blml_seg_append_mode(int dtype, int F, const blml_seg* old_segs, const blml_seg* new_segs, const void* E,
                         const double* dh, const double* v, const double* scale, void* E_new, void* stream);
/* Lanczos steps of the batched certificate (blml_binned.py:501-518, ARPACK there) with no host round trip: from n
   rows of np <= 47 inner products (the layout blml_seg_dots writes), coef rows [1, -c] for w -= V c, and alpha[r]
   = c[r][alpha_col] when alpha is given (alpha_col < 0: none); and beta[r] = sqrt(max(d[r], 0)) with coef[r] =
   1 / beta (0 when beta is 0) for the next basis vector. */
int blml_lanczos_coef(int n, int np, const double* dots, double* coef, double* alpha, int alpha_col, void* stream);
int blml_lanczos_beta(int n, const double* dots, double* beta, double* coef, void* stream);

/* ---- batched solver phases with device-side control: the per-fit decisions of every
 *      iteration run as kernels, a ring of iterations is one CUDA graph replayed until every fit has stopped, the
 *      host reading one active mask per replay; the graph is captured again over the fits still iterating when
 *      they fall to three quarters of those it covers. Stop codes: 0 tol, 1 ll_tol, 2 stall. ----
 * L-BFGS ascent of L = sum w log F - n log Q from E (complex of dtype, the segs layout; U: S E is written there),
 * memory m <= 20, Armijo over t = 2^-j, j < 40, U = S E recomputed at accepted steps, stop at max|rho| < tol, at a
 * likelihood gain below ll_tol over 10 iterations, or after max_iters (< 0: none) -- blml_trivial.py:2590-2645
 * (lbfgs_psd) as BLMLBinned.fit runs it (blml_binned.py:278-355, 429-445) for each fit of a cut-off sweep
 * (selector.py:488-553). w, c: float of dtype per bin (counts / n and counts); n: F host doubles. Fit f has
 * segs[f].K modes (1 to 64) of one shared kernel (plans[f]); its modes are K lattices from segs[f].off. The start
 * runner below takes one mode per fit. */
typedef struct blml_lbfgs_batch_s* blml_lbfgs_batch;
int blml_lbfgs_batch_create(int dtype, int F, const blml_seg* segs, const blml_plan* plans, int m, double tol,
                            double ll_tol, int64_t max_iters, const double* n, const void* w, const void* c, void* E,
                            void* U, blml_lbfgs_batch* runner);
/* per-fit iteration caps (F host values, < 0: none) in place of max_iters, before blml_lbfgs_batch_run: rounds of a
   certified fit cap the fits still growing their rank and let the final ones run to tol */
int blml_lbfgs_batch_set_caps(blml_lbfgs_batch runner, const int64_t* caps);
/* The runner's L-BFGS history (its 2 m stored step and gradient-difference vectors) kept in complex64 storage when
   f32 != 0 and the state is float64: the direction and the history scan read half the bytes, the iterate, gradient
   and line search stay float64. No counterpart in the reference (its history is float64); for runs whose answer does
   not depend on the path, e.g. certified fits. Call before the first run. */
int blml_lbfgs_batch_set_history(blml_lbfgs_batch runner, int f32);
/* The history kernels of such a runner share their blocks out among the fits in proportion to the fits' sizes K B:
   BLML_SEG_SPLIT_BLOCKS blocks in all (at most one per 1024 elements of a fit), the split computed on the device from
   segs into `split`, device scratch of blml_seg_split_ints(F) ints. */
#define BLML_SEG_SPLIT_BLOCKS 2048
int64_t blml_seg_split_ints(int F);
/* The history scan (blml_seg_dots2's quantities, complex): the np stored vectors a and the first shared vector b0
   complex64, b1 and x complex128; float64 sums. part: 43 * (BLML_SEG_SPLIT_BLOCKS + F) doubles. */
int blml_seg_dots2_h32(int F, const blml_seg* segs, int* split, int np, const void* const* a, const void* b0,
                       const void* b1, const void* x, double* part, double* out, void* stream);
/* The direction's linear combination (blml_seg_lincomb, complex): out = sum_i coef[f * nterms + i] v_i, bit i of
   f32mask marking v_i complex64, the others complex128; out complex64 (out_f32) or complex128; float64 arithmetic,
   the complex128 terms summed first, then the complex64 ones, each in term order. */
int blml_seg_lincomb_h32(int F, const blml_seg* segs, int* split, void* out, int out_f32, int nterms,
                         const double* coef, const void* const* v, unsigned long long f32mask, void* stream);
int blml_lbfgs_batch_run(blml_lbfgs_batch runner, void* stream);
/* per fit (host arrays of F, any may be null): iterations, stop code, L, Q, max|rho| */
int blml_lbfgs_batch_result(blml_lbfgs_batch runner, int64_t* iters, int32_t* stop, double* L, double* Q,
                            double* res);
/* [iterations enqueued, graph replays, graph captures, kernels per replay] */
int blml_lbfgs_batch_stats(blml_lbfgs_batch runner, int64_t* out4);
int blml_lbfgs_batch_destroy(blml_lbfgs_batch runner);
/* the real rank-1 start of every fit in float64 (BLMLBinned._start with psd False, blml_binned.py:223-276): the
 * seeded root, Jacobi updates with Anderson mixing (history anderson <= 8) and the merit safeguard, the damped
 * step a = 2^-1 .. 2^-26 when no ascent, stop at max|rho| < tol, after `stall` sweeps without progress or after
 * max_sweeps (< 0: none). c = w n, sg: float64 per bin; n, s0 (K(0) of each fit's kernel): F host doubles; E:
 * float64 output in the segs layout. */
typedef struct blml_start_batch_s* blml_start_batch;
int blml_start_batch_create(int F, const blml_seg* segs, const blml_plan* plans, int anderson, double tol,
                            int64_t max_sweeps, int64_t stall, const double* n, const double* s0, const double* c,
                            const double* sg, double* E, blml_start_batch* runner);
int blml_start_batch_run(blml_start_batch runner, void* stream);
int blml_start_batch_result(blml_start_batch runner, int64_t* sweeps, double* res);
int blml_start_batch_stats(blml_start_batch runner, int64_t* out4);
int blml_start_batch_destroy(blml_start_batch runner);

/* ---- the learned warm start: a small convolutional U-Net mapping (log counts, cut-off, kernel kind) on a lattice to
 *      the fit's field u = S e / n (no counterpart in the reference: it replaces the real rank-1 start of
 *      blml_binned.py:415-436 for the fits it covers). Activations NHWC BF16 in channel slices (Cs channels per
 *      pixel, the slice starting at c0); gradients FP32 in the same layout. ----
 * C[z] = A B^T over split z of K (A: M x K, B: N x K, K-major BF16, K a multiple of 8, 16-byte aligned; C: FP32,
 * splits x M x N): tcgen05 kind::f16, TMA-staged 128-byte-swizzled tiles, TMEM accumulators. *err (device int) is
 * set when a bounded wait gave up (the results are then invalid). */
int blml_nn_gemm_bf16(const void* A, const void* B, float* C, int M, int N, int K, int splits, int* err,
                      void* stream);
/* 3 x 3 (pad 1) im2col of a BF16 slice: col[p][(ky 3 + kx) C + c], or its transpose [9 C][p] */
int blml_nn_im2col(const void* X, int Nb, int H, int W, int Cs, int c0, int C, void* col, int transposed,
                   void* stream);
/* the gradient of im2col: dX slice = sum of the 9 taps of dcol ([P][9 C] FP32), overwritten */
int blml_nn_col2im(const float* dcol, int Nb, int H, int W, int C, float* dX, int Cs, int c0, void* stream);
/* Y slice = act(sum of the split partials + bias) in BF16 (relu: max(., 0)) */
int blml_nn_bias_act(const float* Cm, int splits, int64_t P, int N, const float* bias, int relu, void* Y, int Cs,
                     int c0, void* stream);
/* dPre = dY (Y > 0) in BF16, [P x C] and [C x P] */
int blml_nn_relu_bwd(const float* dY, int Csd, int c0d, const void* Y, int Csy, int c0y, int64_t P, int C,
                     void* dpre, void* dpreT, void* stream);
/* db[c] = sum_p dY[p, c] (restricted to Y > 0 when relu), fixed-order chunk partials (part: chunks x C floats) */
int blml_nn_bias_grad(const float* dY, int Csd, int c0d, const void* Y, int Csy, int c0y, int64_t P, int C, int relu,
                      int chunks, float* part, float* db, void* stream);
/* out = sum over splits of in (fixed order) */
int blml_nn_sum_splits(const float* in, int splits, int64_t n, float* out, void* stream);
/* 2 x 2 average pooling (forward into a slice; gradient added into a slice) */
int blml_nn_pool_fwd(const void* X, int Nb, int H, int W, int Csx, int c0x, int C, void* Y, int Csy, int c0y,
                     void* stream);
int blml_nn_pool_bwd_add(const float* dY, int Nb, int H, int W, int C, float* dX, int Csx, int c0x, void* stream);
/* nearest x2 upsampling of an (h, w) tensor into a slice, and its gradient */
int blml_nn_up_fwd(const void* X, int Nb, int h, int w, int C, void* Y, int Csy, int c0y, void* stream);
int blml_nn_up_bwd(const float* dY, int Nb, int h, int w, int Csy, int c0y, int C, float* dX, void* stream);
/* the 1 x 1 output head (Cout <= 4, FP32 weights [Cout x Cin] and bias): forward, data gradient (dX may be null) and
   weight / bias gradient gw [Cout x (Cin + 1)] from chunk partials (part: chunks x Cout (Cin + 1) floats) */
int blml_nn_head_fwd(const void* X, int64_t P, int Cin, const float* W, const float* b, int Cout, float* Y,
                     void* stream);
int blml_nn_head_bwd(const float* dY, const void* X, int64_t P, int Cin, int Cout, const float* W, float* dX,
                     int chunks, float* part, float* gw, void* stream);
/* per sample s (HW complex values, interleaved FP32): loss[s] = min over a global phase and conjugation of
   |u - e^{i th} t|^2 / |t|^2, and du = d(mean loss)/du; stats: 6 S doubles */
int blml_nn_phase_loss(const float* u, const float* t, int64_t HW, int S, double* stats, float* du, double* loss,
                       void* stream);
/* Adam (bias-corrected, step >= 1) on FP32 weights; optional BF16 copy wb and BF16 transpose wbt of a rows x cols
   matrix */
int blml_nn_adam(float* w, const float* g, float* m, float* v, int64_t n, float lr, float b1, float b2, float eps,
                 int step, void* wb, void* wbt, int rows, int cols, void* stream);
int blml_nn_to_bf16(const float* x, int64_t n, void* y, void* yt, int rows, int cols, void* stream);

/* ---- pair accumulation over lattice bins from the row-kernel value tables (blml_local_gpu.rows / cols,
 *      blml_local_gpu.py:42-105, 320-361, 408-455; numba twins blml_local.py:117-191) ----
 * ZA (R, d), ZB (M, d): int64 lattice coordinates as the tables read them (rank columns: ranks). Table arrays are
 * the ProductKernel layout (blml_kernels.py:133-200): T flat values, base / Jk / mk / kinds / nbins / grp per column,
 * RT (G, LR) group rows, dim_unit / grp_unit, and for grad the derivative rows dT / dbase / dR / wunit / wcol /
 * wgrp (nW entries). rows: s (R) float64 = sum_j w_j S(ZA_r, ZB_j); ds (R, nW) with grad.
 * f32 = 1: table values and products in float32 (sums in float64), as the reference's f32 flag. */
typedef struct {
  int d, U, G, nW, LR, f32;
  int64_t nT, ndT;                    /* lengths of the flat value arrays T and dT */
  const double* T; const int64_t* base; const int64_t* Jk; const int64_t* mk; const int64_t* kinds;
  const int64_t* nbins; const int64_t* grp; const double* RT; const int64_t* dim_unit; const int64_t* grp_unit;
  const double* dT; const int64_t* dbase; const double* dR; const int64_t* wunit; const int64_t* wcol;
  const int64_t* wgrp;
  const float* T32; const float* RT32; const float* dT32; const float* dR32;   /* float32 copies when f32 = 1 */
} blml_tables;
int blml_rows(const blml_tables* tab, const int64_t* ZA, int64_t R, const int64_t* ZB, int64_t M, const double* w,
              int grad, double* s, double* ds, void* stream);
/* ---- fused rows of several densities (blml_local.py:213-286 rows_multi, FusedFit's joint and marginals; K9 of
 *      blml_local_gpu.py:107-180): s[r * Mm + m] = sum_j W[j * Mm + m] prod_u (bit u of umask[m] ? T_u : 1), the unit
 *      factors of a pair computed once; 1 <= Mm <= 8 densities, values only (no derivative rows) ---- */
int blml_rows_multi(const blml_tables* tab, const int64_t* ZA, int64_t R, const int64_t* ZB, int64_t M,
                    const double* W, int Mm, const unsigned* umask, double* s, void* stream);
/* ---- value rows over one coordinate set, validated once (the block coordinate descent of BLMLQuick,
 *      blml_trivial.py:2860-3035 / blml_gpu.py:340-373, whose passes run every bin against a block of bins) ----
 * plan_create reads the tables' metadata and checks that every pair of rows of Z (n x d rank coordinates, device)
 * lies in the tables' extents; plan_run then computes s = rows(ZA, ZB, w) (value rows, as blml_rows) for ZA and ZB made
 * of rows of that Z -- the caller's promise, not re-checked -- with no host synchronisation and no allocation:
 * ws holds blml_rows_plan_workspace(plan, R, M) bytes. The plan copies the table struct; the device tables it points
 * to must outlive it. */
typedef struct blml_rows_plan_s* blml_rows_plan;
int blml_rows_plan_create(const blml_tables* tab, const int64_t* Z, int64_t n, void* stream, blml_rows_plan* plan);
int64_t blml_rows_plan_workspace(blml_rows_plan plan, int64_t R, int64_t M);
int blml_rows_plan_run(blml_rows_plan plan, const int64_t* ZA, int64_t R, const int64_t* ZB, int64_t M,
                       const double* w, double* s, void* ws, int64_t ws_bytes, void* stream);
int blml_rows_plan_destroy(blml_rows_plan plan);
/* ---- blml_rows without any allocation: no counterpart in the reference ----
 * For callers that cannot allocate device memory themselves or let the library do it: processes whose device
 * memory is reserved up front by another allocator (a cudaMalloc would fail or fragment that pool), and embedded
 * hosts that forbid allocation after start-up.
 * blml_rows allocates its column-slice partial sums and its extent-check buffer stream-ordered on every call; this
 * entry point keeps them in a fixed 4 MiB device array inside the library instead (every GPU that loads the library
 * holds it until the process exits), so it takes at most 524,224 rows (R), and larger R is rejected with
 * BLML_ERR_ARG. Value rows only (no derivative rows); same tables, inputs, outputs and results as blml_rows.
 * The first call on a device looks up the array's device address (cudaGetSymbolAddress) and must come before any
 * stream capture on that device. Every call shares the one array: calls that overlap on the GPU (other streams,
 * other host threads) race and give wrong sums, so serialise them. Every scratch entry is written before it is
 * read, so nothing needs clearing between calls. */
int blml_rows_noalloc(const blml_tables* tab, const int64_t* ZA, int64_t R, const int64_t* ZB, int64_t M,
                      const double* w, double* s, void* stream);

/* ---- fixed-lattice binning (BLMLQuick._fit_lattice, blml_trivial.py:3572; SincKernel.quantize :402-403) ----
 * out (n, d) int64 = round(Z / h) of bin centres Z (n, d) float64, h (d) float64, ties to even as np.round */
int blml_lattice_coords(const double* Z, int64_t n, int d, const double* h, int64_t* out, void* stream);

/* out (R, M) row-major = S(ZA_r, ZB_j), float64 (out_f32 = 0) or float32 */
int blml_cols(const blml_tables* tab, const int64_t* ZA, int64_t R, const int64_t* ZB, int64_t M, void* out,
              int out_f32, void* stream);
/* the joint and marginal blocks of a conditional fit (cols_kernel with depmask, blml_local_gpu.py:320-361): out as
 * blml_cols, out_m (R, M) = the product over the units (columns, or whole radial groups) none of whose columns has
 * its bit set in depmask -- the marginal kernel of the other columns -- from the same table lookups */
int blml_cols_dep(const blml_tables* tab, const int64_t* ZA, int64_t R, const int64_t* ZB, int64_t M, int64_t depmask,
                  void* out, void* out_m, int out_f32, void* stream);

#ifdef __cplusplus
}
#endif
#endif
