// passes.cuh -- host launchers of the FFT passes of the solve (x forward + y
// forward, the fused z pass, y inverse + x inverse).  Included by the pass units
// passes_*.cu, each of which instantiates them for one precision and component
// count, so the heavy kernels compile in parallel.
#pragma once

#include <algorithm>

#include "host.h"
#include "solve.cuh"

namespace pmgpu {

template <typename K> static int persistent_grid(K kernel, size_t smem, int ntiles) {
  int per = 1;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, PASS_THREADS, smem) != cudaSuccess || per < 1) per = 1;
  return std::max(1, std::min(ntiles, per * num_sms()));
}


template <typename R, int NC>
static int launch_lines(SolveGeom<R> &g, const typename cplx_t<R>::type *in, typename cplx_t<R>::type *out, int axis,
                        int lmode, int zmode, int reproj, int use_zeta, int rows_in, int rows_out, long long in_os,
                        long long in_rs, long long out_os, long long out_rs, int nouter, cudaStream_t st,
                        const char *caller) {
  typedef typename cplx_t<R>::type C;
  const int n = g.M[axis];
  if (axis == 1 ? g.ry_ok : g.rz_ok) {
    const RegPlan &rp = axis == 1 ? g.ry : g.rz;
    const int mt = rp.n;  // transform length (Bluestein: > n)
    bool wide = false;
    for (int p = 0; p < rp.np; p++) wide = wide || reg_radix_wide(rp.rad[p]);
    if (wide && sizeof(R) != 4) {
      set_error(caller, "wide radices are FP32 only.");
      return -1;
    }
    int TK = axis == 1 ? g.tky : g.tkz;  // a tuned tile, if it fits
    if (TK <= 0 || g.Hp % TK || reg_smem(n, mt, NC, TK, sizeof(C)) > PASS_SMEM_BUDGET)
      TK = pick_tk_reg(n, mt, NC, sizeof(C), g.Hp, wide ? reg_budget_wide() : reg_budget(sizeof(R)));
    if (TK > 0) {
      LineTiles lt;
      lt.n = n;
      lt.rows_in = rows_in;
      lt.rows_out = rows_out;
      lt.in_os = in_os;
      lt.in_rs = in_rs;
      lt.out_os = out_os;
      lt.out_rs = out_rs;
      lt.nouter = nouter;
      lt.nkt = g.Hp / TK;
      lt.TK = TK;
      lt.dLG = make_fastdiv((unsigned)(NC * TK / RVec<R>::G));
      const size_t sm = reg_smem(n, mt, NC, TK, sizeof(C));
      auto launch = [&](auto kern) -> int {
        CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm), caller);
        int per = 1;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, RL_THREADS, sm) != cudaSuccess || per < 1)
          per = 1;
        const int grid = std::max(1, std::min(lt.nouter * lt.nkt, per * num_sms()));
        kern<<<grid, RL_THREADS, sm, st>>>(g, lt, in, out, axis, lmode, zmode, reproj, use_zeta);
        PM_LAUNCHED();
        CKL(caller);
        return 0;
      };
      if constexpr (sizeof(R) == 4) {
        if (wide) return launch(k_rlines<R, NC, true>);
      }
      return launch(k_rlines<R, NC, false>);
    }
  }
  const int ntw = (axis == 1) ? g.fy.ntw : g.fz.ntw;
  const int TK = pick_tk(n, NC, sizeof(C), ntw);
  if (TK == 0) {
    set_error(caller, "FFT length too large for the shared-memory transform.");
    return -1;
  }
  LineTiles lt;
  lt.n = n;
  lt.rows_in = rows_in;
  lt.rows_out = rows_out;
  lt.in_os = in_os;
  lt.in_rs = in_rs;
  lt.out_os = out_os;
  lt.out_rs = out_rs;
  lt.nouter = nouter;
  lt.nkt = g.Hp / TK;
  lt.TK = TK;
  const size_t sm = lines_smem(n, NC, TK, sizeof(C), ntw);
  CK(cudaFuncSetAttribute(k_lines<R, NC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm), caller);
  const int grid = persistent_grid(k_lines<R, NC>, sm, lt.nouter * lt.nkt);
  k_lines<R, NC><<<grid, PASS_THREADS, sm, st>>>(g, lt, in, out, axis, lmode, zmode, reproj, use_zeta);
  PM_LAUNCHED();
  CKL(caller);
  return 0;
}

template <typename R, int NC>
int fwd_xy(SolveGeom<R> &g, const R *in, typename cplx_t<R>::type *X, typename cplx_t<R>::type *Y,
           cudaStream_t st, const char *caller, int cs) {
  typedef typename cplx_t<R>::type C;
  const bool vec16r = cs == NC && ((size_t)g.ext[0] * NC * sizeof(R)) % 16 == 0 &&
                      ((size_t)g.off[0] * NC * sizeof(R)) % 16 == 0 && ((size_t)g.P[0] * NC * sizeof(R)) % 16 == 0;
  if (g.rx_ok) {
    const int RB = pick_rb_reg(g.N2, g.rx.n, g.H, g.P[0], g.Hp, NC, sizeof(C), sizeof(R), false, reg_budget(sizeof(R)));
    if (RB > 0) {
      const size_t sm = rx_smem(g.N2, g.rx.n, g.H, g.P[0], g.Hp, NC, RB, sizeof(C), sizeof(R), false);
      CK(cudaFuncSetAttribute(k_rxfwd<R, NC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm), caller);
      const int rows = g.P[1] * g.P[2];
      const int ntiles = (rows + RB - 1) / RB;
      int per = 1;
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_rxfwd<R, NC>, RL_THREADS, sm) != cudaSuccess || per < 1)
        per = 1;
      const int grid = std::max(1, std::min(ntiles, per * num_sms()));
      { KTimer kt_(KC_XFWD, st);
        k_rxfwd<R, NC><<<grid, RL_THREADS, sm, st>>>(g, in, X, RB, cs, vec16r ? 1 : 0,
                                                     make_fastdiv((unsigned)(NC * RB / RVec<R>::G))); }
      PM_LAUNCHED();
      CKL(caller);
      const long long Hp = g.Hp;
      KTimer kt_(KC_YFWD, st);
      return launch_lines<R, NC>(g, X, Y, 1, L_FWD, 0, 0, 0, g.P[1], g.M[1], (long long)g.P[1] * Hp, Hp,
                                 (long long)g.M[1] * Hp, Hp, g.P[2], st, caller);
    }
  }
  const int ntwx = g.fx.ntw + g.fx.next;
  const int RB = pick_rb(g.N2, g.P[0], g.Hp, NC, sizeof(C), sizeof(R), ntwx, false);
  if (RB == 0) {
    set_error(caller, "FFT length too large for the shared-memory transform.");
    return -1;
  }
  const size_t stage = (((size_t)RB * g.P[0] * NC * sizeof(R) + 15) / 16) * 16;
  const size_t sm = tw_bytes(ntwx, sizeof(C)) + stage + 2 * (size_t)NC * RB * g.N2 * sizeof(C);
  const bool vec16 = cs == NC && ((size_t)g.ext[0] * NC * sizeof(R)) % 16 == 0 &&
                     ((size_t)g.off[0] * NC * sizeof(R)) % 16 == 0 && ((size_t)g.P[0] * NC * sizeof(R)) % 16 == 0;
  CK(cudaFuncSetAttribute(k_xfwd<R, NC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm), caller);
  const int rows = g.P[1] * g.P[2];
  const int ntiles = (rows + RB - 1) / RB;
  { KTimer kt_(KC_XFWD, st);
    k_xfwd<R, NC><<<persistent_grid(k_xfwd<R, NC>, sm, ntiles), PASS_THREADS, sm, st>>>(g, in, X, RB, cs, vec16 ? 1 : 0); }
  PM_LAUNCHED();
  CKL(caller);
  const long long Hp = g.Hp;
  KTimer kt_(KC_YFWD, st);
  return launch_lines<R, NC>(g, X, Y, 1, L_FWD, 0, 0, 0, g.P[1], g.M[1], (long long)g.P[1] * Hp, Hp,
                             (long long)g.M[1] * Hp, Hp, g.P[2], st, caller);
}

// one forward (or inverse) pass along y over the X layout -> Y layout, as in fwd_xy
template <typename R, int NC>
int ypass(SolveGeom<R> &g, const typename cplx_t<R>::type *X, typename cplx_t<R>::type *Y, int inverse,
          cudaStream_t st, const char *caller) {
  const long long Hp = g.Hp;
  if (inverse)
    return launch_lines<R, NC>(g, Y, (typename cplx_t<R>::type *)X, 1, L_INV, 0, 0, 0, g.M[1], g.P[1],
                               (long long)g.M[1] * Hp, Hp, (long long)g.P[1] * Hp, Hp, g.P[2], st, caller);
  return launch_lines<R, NC>(g, X, Y, 1, L_FWD, 0, 0, 0, g.P[1], g.M[1], (long long)g.P[1] * Hp, Hp,
                             (long long)g.M[1] * Hp, Hp, g.P[2], st, caller);
}

template <typename R, int NC>
int zpass(SolveGeom<R> &g, const typename cplx_t<R>::type *in, typename cplx_t<R>::type *out, int mode,
                 int reproj, int use_zeta, int rows_y, cudaStream_t st, const char *caller) {
  const long long Hp = g.Hp;
  // Z_FORWARD: forward transform only, P rows in (the rest zero), M rows out
  const int rows_in = g.P[2], rows_out = (mode == Z_FORWARD) ? g.M[2] : g.P[2];
  KTimer kt_(KC_ZPASS, st);
  return launch_lines<R, NC>(g, in, out, 2, mode == Z_FORWARD ? L_FWD : L_Z, mode, reproj, use_zeta, rows_in,
                             rows_out, Hp, (long long)g.M[1] * Hp, Hp, (long long)g.M[1] * Hp, rows_y, st, caller);
}

template <typename R, int NC>
int inv_yx(SolveGeom<R> &g, const pmgpu_topo *topo, typename cplx_t<R>::type *Y,
           typename cplx_t<R>::type *X, R *out, cudaStream_t st, const char *caller, int cs, bool ghosts) {
  typedef typename cplx_t<R>::type C;
  const long long Hp = g.Hp;
  {
    KTimer kt_(KC_YINV, st);
    if (launch_lines<R, NC>(g, Y, X, 1, L_INV, 0, 0, 0, g.M[1], g.P[1], (long long)g.M[1] * Hp, Hp,
                            (long long)g.P[1] * Hp, Hp, g.P[2], st, caller))
      return -1;
  }
  const int rows = g.P[1] * g.P[2];
  const int RBr = g.rx_ok ? pick_rb_reg(g.N2, g.rx.n, g.H, g.P[0], g.Hp, NC, sizeof(C), sizeof(R), true, reg_budget(sizeof(R))) : 0;
  if (RBr > 0) {
    const size_t sm = rx_smem(g.N2, g.rx.n, g.H, g.P[0], g.Hp, NC, RBr, sizeof(C), sizeof(R), true);
    CK(cudaFuncSetAttribute(k_rxinv<R, NC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm), caller);
    const int ntiles = (rows + RBr - 1) / RBr;
    int per = 1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_rxinv<R, NC>, RL_THREADS, sm) != cudaSuccess || per < 1)
      per = 1;
    const int grid = std::max(1, std::min(ntiles, per * num_sms()));
    { KTimer kt_(KC_XINV, st);
      k_rxinv<R, NC><<<grid, RL_THREADS, sm, st>>>(g, X, out, RBr, cs, make_fastdiv((unsigned)(NC * RBr / RVec<R>::G))); }
    PM_LAUNCHED();
    CKL(caller);
  } else {
    const int ntwx = g.fx.ntw + g.fx.next;
    const int RB = pick_rb(g.N2, g.P[0], g.Hp, NC, sizeof(C), sizeof(R), ntwx, true);
    if (RB == 0) {
      set_error(caller, "FFT length too large for the shared-memory transform.");
      return -1;
    }
    const size_t sm =
        tw_bytes(ntwx, sizeof(C)) + (size_t)RB * g.Hp * NC * sizeof(C) + 2 * (size_t)NC * RB * g.N2 * sizeof(C);
    CK(cudaFuncSetAttribute(k_xinv<R, NC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm), caller);
    const int ntiles = (rows + RB - 1) / RB;
    { KTimer kt_(KC_XINV, st);
      k_xinv<R, NC><<<persistent_grid(k_xinv<R, NC>, sm, ntiles), PASS_THREADS, sm, st>>>(g, X, out, RB, cs); }
    PM_LAUNCHED();
    CKL(caller);
  }
  // periodic ghosts (x, then y, then z)
  for (int d = 0; d < 3 && ghosts; d++) {
    if (topo->bound_cond[2 * d] == 0 || topo->bound_cond[2 * d + 1] == 0) continue;
    const int S = topo->nghost[2 * d] + topo->nghost[2 * d + 1];
    const long long total = (long long)S * g.ext[(d + 1) % 3] * g.ext[(d + 2) % 3];
    const int nblk = (int)std::min<long long>((total + 255) / 256, 148 * 16);
    { KTimer kt_(KC_GFILL, st); k_ghost_fill<R><<<std::max(nblk, 1), 256, 0, st>>>(out, g.ext[0], g.ext[1], g.ext[2], cs, d, topo->ncell[d],
                                                        topo->nghost[2 * d], topo->nghost[2 * d + 1]); }
    PM_LAUNCHED();
    CKL(caller);
  }
  return 0;
}


// copies the DFT constant tables into this unit's constant memory
static int upload_cs_local(const void *t32, const void *t64) {
  if (cudaMemcpyToSymbol(c_cs32, t32, sizeof(c_cs32)) != cudaSuccess) return -1;
  if (cudaMemcpyToSymbol(c_cs64, t64, sizeof(c_cs64)) != cudaSuccess) return -1;
  return 0;
}

}  // namespace pmgpu

#define PMGPU_INSTANTIATE_PASSES(R, NC, NAME)                                                                  \
  namespace pmgpu {                                                                                            \
  template int fwd_xy<R, NC>(SolveGeom<R> &, const R *, cplx_t<R>::type *, cplx_t<R>::type *, cudaStream_t,    \
                             const char *, int);                                                               \
  template int zpass<R, NC>(SolveGeom<R> &, const cplx_t<R>::type *, cplx_t<R>::type *, int, int, int, int,    \
                            cudaStream_t, const char *);                                                       \
  template int inv_yx<R, NC>(SolveGeom<R> &, const pmgpu_topo *, cplx_t<R>::type *, cplx_t<R>::type *, R *,    \
                             cudaStream_t, const char *, int, bool);                                           \
  template int ypass<R, NC>(SolveGeom<R> &, const cplx_t<R>::type *, cplx_t<R>::type *, int, cudaStream_t,      \
                            const char *);                                                                     \
  int upload_cs_##NAME(const void *t32, const void *t64) { return upload_cs_local(t32, t64); }                 \
  }
