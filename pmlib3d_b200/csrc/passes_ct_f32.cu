// passes_ct_f32.cu -- compile-time-plan line passes for float fields of 3
// components: y / z passes for the plans and kx tiles of the 528-point lines (256
// cells with four ghost layers, free) and of the 512-point periodic lines, with the
// radix orders and tiles the schedule tuner chooses between, and x passes for the rows
// of those grids.  Other plans run the run-time engine.
#include "passes.cuh"
#include "xpass_ct.cuh"

namespace pmgpu {

#define PMGPU_CT(N, A, B, C, T)                                                                              \
  if (ct_match<CtPlan<N, A, B, C>>(rp) && TK == T)                                                           \
    return k_rlines_ct<float, 3, (A > 17 || B > 17 || C > 17), N, A, B, C, T>;

LinesKernel<float> ct_lines_f32(const RegPlan &rp, int TK) {
  PMGPU_CT(528, 24, 22, 1, 8)
  PMGPU_CT(528, 22, 24, 1, 8)
  PMGPU_CT(528, 12, 11, 4, 8)
  PMGPU_CT(528, 24, 22, 1, 4)
  PMGPU_CT(528, 22, 24, 1, 4)
  PMGPU_CT(528, 12, 11, 4, 4)
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
RxfKernel<float> ct_rxfwd_f32(const RegPlan &rp, int RB, int P0, int Hp) {
  if (ct_match<CtPlan<256, 16, 16>>(rp) && RB == 5 && P0 == 512 && Hp == 264)
    return k_rxfwd_ct<float, 3, 256, 16, 16, 1, 5, 512, 264>;
  if (ct_match<CtPlan<264, 12, 11, 2>>(rp) && RB == 7 && P0 == 264 && Hp == 272)
    return k_rxfwd_ct<float, 3, 264, 12, 11, 2, 7, 264, 272>;
  return nullptr;
}
RxiKernel<float> ct_rxinv_f32(const RegPlan &rp, int RB, int P0, int Hp) {
  if (ct_match<CtPlan<256, 16, 16>>(rp) && RB == 5 && P0 == 512 && Hp == 264)
    return k_rxinv_ct<float, 3, 256, 16, 16, 1, 5, 512, 264>;
  if (ct_match<CtPlan<264, 12, 11, 2>>(rp) && RB == 5 && P0 == 264 && Hp == 272)
    return k_rxinv_ct<float, 3, 264, 12, 11, 2, 5, 264, 272>;
  return nullptr;
}

int upload_cs_ct_f32(const void *t32, const void *t64) { return upload_cs_local(t32, t64); }

}  // namespace pmgpu
