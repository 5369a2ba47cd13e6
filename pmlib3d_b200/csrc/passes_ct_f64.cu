// passes_ct_f64.cu -- compile-time-plan y / z line passes for double fields of 3
// components (see passes_ct_f32.cu).
#include "passes.cuh"

namespace pmgpu {

#define PMGPU_CT(N, A, B, C, T)                                                                              \
  if (ct_match<CtPlan<N, A, B, C>>(rp) && TK == T) return k_rlines_ct<double, 3, false, N, A, B, C, T>;

LinesKernel<double> ct_lines_f64(const RegPlan &rp, int TK) {
  PMGPU_CT(528, 12, 11, 4, 8)
  PMGPU_CT(528, 8, 6, 11, 8)
  return nullptr;
}

#undef PMGPU_CT

int upload_cs_ct_f64(const void *t32, const void *t64) { return upload_cs_local(t32, t64); }

}  // namespace pmgpu
