// The mat-vec plan shared by the SIMT (matvec.cu) and tensor-core (tc_matvec.cu) engines.
#pragma once
#include <vector>
#include "common.cuh"

struct blml_plan_s {
  int d, dtype, engine;
  int64_t shape[8];
  int32_t nfreq[8];
  int64_t max_elems;                 // largest intermediate tensor of one lattice (elements), SIMT schedule
  void* tf[8];                       // forward twiddles per axis: (M x H) conj(v), complex of dtype
  void* ti[8];                       // inverse twiddles per axis: (H x M) v^T
  void* W;                           // weights over the frequency grid, real of dtype
  void* tc;                          // tensor-core engine state (split-TF32 operands), or null
  void* fft;                         // FFT route state (fft_matvec.cu) when the kernel is a DFT mask, or null
  int route;                         // BLML_ROUTE_*: which route blml_matvec takes
};

namespace blml {
// fwd[a] / inv[a]: the float64 twiddles of axis a, interleaved complex, (M x H) conj(v) and (H x M) v^T
int tc_plan_init(blml_plan_s* p, const std::vector<std::vector<double>>& fwd,
                 const std::vector<std::vector<double>>& inv);
void tc_plan_free(blml_plan_s* p);
int tc_matvec(blml_plan_s* p, const void* x, void* y, int nb, int xc, void* ws, int64_t wsb, cudaStream_t st);
int64_t tc_workspace(const blml_plan_s* p, int nb);
int tc_error(blml_plan_s* p);

// the FFT route (fft_matvec.cu): set up when the plan is a 2-D DFT mask on sides 2^a 3^b (else p->fft stays null)
int fft_plan_init(blml_plan_s* p, const double* freqs);
void fft_plan_free(blml_plan_s* p);
int64_t fft_workspace(const blml_plan_s* p, int nb);
int fft_matvec(blml_plan_s* p, const void* x, void* y, int nb, int xc, void* ws, cudaStream_t st);
// a group's descriptors: problem g reads x[g], writes y[g] and keeps its spectrum in z[g] (its workspace); *out stays
// null when a plan has no FFT route
int fft_group_init(void** out, int G, const blml_plan* plans, const int* nbatch, int xc, const void* const* x,
                   void* const* y, void* const* z);
void fft_group_free(void* fg);
int fft_group_launch(void* fg, int dtype, const int* subset, int n, const int* live, cudaStream_t st);
}  // namespace blml
