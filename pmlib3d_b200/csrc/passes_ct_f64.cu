// passes_ct_f64.cu -- compile-time-plan line passes for double fields of 3
// components (see passes_ct_f32.cu).
#include "passes.cuh"
#include "xpass_ct.cuh"

namespace pmgpu {

#define PMGPU_CT(N, A, B, C, T)                                                                              \
  if (ct_match<CtPlan<N, A, B, C>>(rp) && TK == T) return k_rlines_ct<double, 3, false, N, A, B, C, T>;

LinesKernel<double> ct_lines_f64(const RegPlan &rp, int TK) {
  PMGPU_CT(528, 12, 11, 4, 8)
  PMGPU_CT(528, 8, 6, 11, 8)
  PMGPU_CT(528, 12, 11, 4, 4)
  PMGPU_CT(528, 8, 6, 11, 4)
  PMGPU_CT(512, 8, 8, 8, 8)
  PMGPU_CT(512, 8, 8, 8, 4)
  PMGPU_CT(512, 16, 8, 4, 8)
  PMGPU_CT(512, 16, 8, 4, 4)
  PMGPU_CT(512, 8, 16, 4, 8)
  PMGPU_CT(512, 8, 16, 4, 4)
  PMGPU_CT(512, 16, 4, 8, 8)
  PMGPU_CT(512, 16, 4, 8, 4)
  PMGPU_CT(512, 8, 4, 16, 8)
  PMGPU_CT(512, 8, 4, 16, 4)
  PMGPU_CT(512, 4, 16, 8, 8)
  PMGPU_CT(512, 4, 16, 8, 4)
  return nullptr;
}

#undef PMGPU_CT

// x passes of the free-axis rows of 256 cells with four ghost layers (264 reals, a
// 264-point packed transform) and of the periodic rows of 512 cells (a 256-point packed
// transform), with the rows per tile the launcher picks
RxfKernel<double> ct_rxfwd_f64(const RegPlan &rp, int RB, int P0, int Hp) {
  if (ct_match<CtPlan<256, 16, 16>>(rp) && RB == 4 && P0 == 512 && Hp == 264)
    return k_rxfwd_ct<double, 3, 256, 16, 16, 1, 4, 512, 264>;
  if (ct_match<CtPlan<264, 12, 11, 2>>(rp) && RB == 5 && P0 == 264 && Hp == 272)
    return k_rxfwd_ct<double, 3, 264, 12, 11, 2, 5, 264, 272>;
  return nullptr;
}
RxiKernel<double> ct_rxinv_f64(const RegPlan &rp, int RB, int P0, int Hp) {
  if (ct_match<CtPlan<256, 16, 16>>(rp) && RB == 4 && P0 == 512 && Hp == 264)
    return k_rxinv_ct<double, 3, 256, 16, 16, 1, 4, 512, 264>;
  if (ct_match<CtPlan<264, 12, 11, 2>>(rp) && RB == 4 && P0 == 264 && Hp == 272)
    return k_rxinv_ct<double, 3, 264, 12, 11, 2, 4, 264, 272>;
  return nullptr;
}

int upload_cs_ct_f64(const void *t32, const void *t64) { return upload_cs_local(t32, t64); }

}  // namespace pmgpu
