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
};

namespace blml {
// fwd[a] / inv[a]: the float64 twiddles of axis a, interleaved complex, (M x H) conj(v) and (H x M) v^T
int tc_plan_init(blml_plan_s* p, const std::vector<std::vector<double>>& fwd,
                 const std::vector<std::vector<double>>& inv);
void tc_plan_free(blml_plan_s* p);
int tc_matvec(blml_plan_s* p, const void* x, void* y, int nb, int xc, void* ws, int64_t wsb, cudaStream_t st);
int64_t tc_workspace(const blml_plan_s* p, int nb);
int tc_error(blml_plan_s* p);
}  // namespace blml
