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


// kx tile of the register-engine line pass along `axis` within `slack` bytes less
// than the usual shared-memory budget (0: the pass takes the Stockham path); wide:
// the plan has a wide composite radix
template <typename R, int NC>
static int rl_pick_tk(const SolveGeom<R> &g, int axis, size_t slack, bool &wide) {
  typedef typename cplx_t<R>::type C;
  wide = false;
  if (!(axis == 1 ? g.ry_ok : g.rz_ok)) return 0;
  const int n = g.M[axis];
  const RegPlan &rp = axis == 1 ? g.ry : g.rz;
  const int mt = rp.n;  // transform length (Bluestein: > n)
  for (int p = 0; p < rp.np; p++) wide = wide || reg_radix_wide(rp.rad[p]);
  const size_t budget = (wide ? reg_budget_wide() : reg_budget(sizeof(R))) - slack;
  int TK = axis == 1 ? g.tky : g.tkz;  // a tuned tile, if it fits
  if (TK <= 0 || g.Hp % TK || reg_smem(n, mt, NC, TK, sizeof(C)) > PASS_SMEM_BUDGET - slack)
    TK = pick_tk_reg(n, mt, NC, sizeof(C), g.Hp, budget);
  if (TK > 0 && reg_smem(n, mt, NC, TK, sizeof(C)) > PASS_SMEM_BUDGET - slack) TK = 0;
  return TK;
}

// a line-pass kernel (k_rlines and its compile-time-plan instances)
template <typename R>
using LinesKernel = void (*)(SolveGeom<R>, LineTiles, const typename cplx_t<R>::type *, typename cplx_t<R>::type *,
                             int, int, int, int, int);
// the compile-time-plan kernel of 3-component lines for plan rp and kx tile TK
// (nullptr: none compiled); defined in passes_ct_*.cu
LinesKernel<float> ct_lines_f32(const RegPlan &rp, int TK);
LinesKernel<double> ct_lines_f64(const RegPlan &rp, int TK);
// x passes (k_rxfwd / k_rxinv and their compile-time-plan instances)
template <typename R>
using RxfKernel = void (*)(SolveGeom<R>, const R *, typename cplx_t<R>::type *, int, int, int, FastDiv);
template <typename R>
using RxiKernel = void (*)(SolveGeom<R>, const typename cplx_t<R>::type *, R *, int, int, FastDiv);
// the compile-time-plan x passes of 3-component fields for plan rp, rows per tile RB,
// real row length P0 and spectrum pitch Hp (nullptr: none compiled); passes_ct_*.cu
RxfKernel<float> ct_rxfwd_f32(const RegPlan &rp, int RB, int P0, int Hp);
RxiKernel<float> ct_rxinv_f32(const RegPlan &rp, int RB, int P0, int Hp);
RxfKernel<double> ct_rxfwd_f64(const RegPlan &rp, int RB, int P0, int Hp);
RxiKernel<double> ct_rxinv_f64(const RegPlan &rp, int RB, int P0, int Hp);

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
    const int TK = rl_pick_tk<R, NC>(g, axis, 0, wide);
    if (wide && sizeof(R) != 4) {
      set_error(caller, "wide radices are FP32 only.");
      return -1;
    }
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
        if (smem_attr((const void *)kern, sm, caller)) return -1;
        int per = 1;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, RL_THREADS, sm) != cudaSuccess || per < 1)
          per = 1;
        const int grid = std::max(1, std::min(lt.nouter * lt.nkt, per * num_sms()));
        kern<<<grid, RL_THREADS, sm, st>>>(g, lt, in, out, axis, lmode, zmode, reproj, use_zeta);
        PM_LAUNCHED();
        CKL(caller);
        return 0;
      };
      if constexpr (NC == 3) {
        if (g_fft_ct) {
          LinesKernel<R> ck;
          if constexpr (sizeof(R) == 4) ck = ct_lines_f32(rp, TK);
          else ck = ct_lines_f64(rp, TK);
          if (ck) return launch(ck);
        }
      }
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
  if (smem_attr((const void *)k_lines<R, NC>, sm, caller)) return -1;
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
      RxfKernel<R> kern = k_rxfwd<R, NC>;
      if constexpr (NC == 3) {
        if (g_fft_ct && !g.rx.bl) {
          RxfKernel<R> ck;
          if constexpr (sizeof(R) == 4) ck = ct_rxfwd_f32(g.rx, RB, g.P[0], (int)g.Hp);
          else ck = ct_rxfwd_f64(g.rx, RB, g.P[0], (int)g.Hp);
          if (ck) kern = ck;
        }
      }
      if (smem_attr((const void *)kern, sm, caller)) return -1;
      const int rows = g.P[1] * g.P[2];
      const int ntiles = (rows + RB - 1) / RB;
      int per = 1;
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, RL_THREADS, sm) != cudaSuccess || per < 1)
        per = 1;
      const int grid = std::max(1, std::min(ntiles, per * num_sms()));
      { KTimer kt_(KC_XFWD, st);
        kern<<<grid, RL_THREADS, sm, st>>>(g, in, X, RB, cs, vec16r ? 1 : 0,
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
  if (smem_attr((const void *)k_xfwd<R, NC>, sm, caller)) return -1;
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
    RxiKernel<R> kern = k_rxinv<R, NC>;
    if constexpr (NC == 3) {
      if (g_fft_ct && !g.rx.bl) {
        RxiKernel<R> ck;
        if constexpr (sizeof(R) == 4) ck = ct_rxinv_f32(g.rx, RBr, g.P[0], (int)g.Hp);
        else ck = ct_rxinv_f64(g.rx, RBr, g.P[0], (int)g.Hp);
        if (ck) kern = ck;
      }
    }
    if (smem_attr((const void *)kern, sm, caller)) return -1;
    const int ntiles = (rows + RBr - 1) / RBr;
    int per = 1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, RL_THREADS, sm) != cudaSuccess || per < 1)
      per = 1;
    const int grid = std::max(1, std::min(ntiles, per * num_sms()));
    { KTimer kt_(KC_XINV, st);
      kern<<<grid, RL_THREADS, sm, st>>>(g, X, out, RBr, cs, make_fastdiv((unsigned)(NC * RBr / RVec<R>::G))); }
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
    if (smem_attr((const void *)k_xinv<R, NC>, sm, caller)) return -1;
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


// ---------------------------------------------------------------- batches of patches
// shared memory the batched kernels keep for their own bookkeeping (the patch
// descriptor copy and the chunk counter), taken off the per-CTA budgets so that as
// many CTAs fit on an SM as in the passes of a single plan
constexpr size_t BATCH_SMEM_SLACK = 3 * 1024;

template <typename R, int NC>
int batch_layout(int n, const SolveGeom<R> *g, typename cplx_t<R>::type *const *X,
                 typename cplx_t<R>::type *const *Y, const pmgpu_topo *const *topo, std::vector<unsigned char> &desc,
                 BatchLayout &lay, const char *caller) {
  typedef typename cplx_t<R>::type C;
  static_assert(sizeof(PassDesc<R>) + 64 <= BATCH_SMEM_SLACK, "descriptor copy exceeds the reserved shared memory");
  if (n <= 0 || n > BATCH_MAX) return -1;
  lay = BatchLayout();
  lay.npatch = n;
  std::vector<PassDesc<R>> d[5];
  for (int f = 0; f < 5; f++) {
    d[f].resize(n);
    memset(d[f].data(), 0, sizeof(PassDesc<R>) * n);
    lay.pass[f].nitems = 0;
    lay.pass[f].smem = 0;
    lay.pass[f].wide = 0;
  }
  std::vector<GhostDesc> gd[3];
  for (int i = 0; i < n; i++) {
    const SolveGeom<R> &gi = g[i];
    if (!gi.rx_ok || !gi.ry_ok || !gi.rz_ok) return -1;
    const long long Hp = gi.Hp;
    // x forward and x inverse (rows per tile as the single-plan passes, within the slack)
    for (int inv = 0; inv < 2; inv++) {
      const int f = inv ? 4 : 0;
      const int RB = pick_rb_reg(gi.N2, gi.rx.n, gi.H, gi.P[0], gi.Hp, NC, sizeof(C), sizeof(R), inv != 0,
                                 reg_budget(sizeof(R)) - BATCH_SMEM_SLACK);
      if (RB <= 0) return -1;
      const size_t sm = rx_smem(gi.N2, gi.rx.n, gi.H, gi.P[0], gi.Hp, NC, RB, sizeof(C), sizeof(R), inv != 0);
      if (sm > PASS_SMEM_BUDGET - BATCH_SMEM_SLACK) return -1;
      PassDesc<R> &q = d[f][i];
      q.g = gi;
      q.RB = RB;
      q.cs = NC;
      q.vec16 = ((size_t)gi.ext[0] * NC * sizeof(R)) % 16 == 0 && ((size_t)gi.off[0] * NC * sizeof(R)) % 16 == 0 &&
                ((size_t)gi.P[0] * NC * sizeof(R)) % 16 == 0;
      q.dLG = make_fastdiv((unsigned)(NC * RB / RVec<R>::G));
      q.in = inv ? X[i] : nullptr;   // x forward reads the caller's vorticity
      q.out = inv ? nullptr : X[i];  // x inverse writes the caller's velocity
      q.ntiles = (gi.P[1] * gi.P[2] + RB - 1) / RB;
      q.first = lay.pass[f].nitems;
      lay.pass[f].nitems += q.ntiles;
      lay.pass[f].smem = std::max(lay.pass[f].smem, sm);
    }
    // y forward, z pass, y inverse (run_solve's launch_lines arguments)
    for (int f = 1; f <= 3; f++) {
      const int axis = f == 2 ? 2 : 1;
      bool wide = false;
      const int TK = rl_pick_tk<R, NC>(gi, axis, BATCH_SMEM_SLACK, wide);
      if (TK <= 0 || (wide && sizeof(R) != 4)) return -1;
      const RegPlan &rp = axis == 1 ? gi.ry : gi.rz;
      PassDesc<R> &q = d[f][i];
      q.g = gi;
      LineTiles &lt = q.lt;
      lt.n = gi.M[axis];
      lt.TK = TK;
      lt.nkt = gi.Hp / TK;
      lt.dLG = make_fastdiv((unsigned)(NC * TK / RVec<R>::G));
      lt.nouter = f == 2 ? gi.M[1] : gi.P[2];
      if (f == 1) {  // X -> Y
        lt.rows_in = gi.P[1];
        lt.rows_out = gi.M[1];
        lt.in_os = (long long)gi.P[1] * Hp;
        lt.in_rs = Hp;
        lt.out_os = (long long)gi.M[1] * Hp;
        lt.out_rs = Hp;
        q.in = X[i];
        q.out = Y[i];
      } else if (f == 2) {  // Y -> Y, fused multiply
        lt.rows_in = gi.P[2];
        lt.rows_out = gi.P[2];
        lt.in_os = Hp;
        lt.in_rs = (long long)gi.M[1] * Hp;
        lt.out_os = Hp;
        lt.out_rs = (long long)gi.M[1] * Hp;
        q.in = Y[i];
        q.out = Y[i];
      } else {  // Y -> X
        lt.rows_in = gi.M[1];
        lt.rows_out = gi.P[1];
        lt.in_os = (long long)gi.M[1] * Hp;
        lt.in_rs = Hp;
        lt.out_os = (long long)gi.P[1] * Hp;
        lt.out_rs = Hp;
        q.in = Y[i];
        q.out = X[i];
      }
      q.ntiles = lt.nouter * lt.nkt;
      q.first = lay.pass[f].nitems;
      lay.pass[f].nitems += q.ntiles;
      lay.pass[f].smem = std::max(lay.pass[f].smem, reg_smem(lt.n, rp.n, NC, TK, sizeof(C)));
      lay.pass[f].wide |= wide ? 1 : 0;
    }
    // periodic ghosts of the velocity (x, then y, then z)
    for (int a = 0; a < 3; a++) {
      const pmgpu_topo *t = topo[i];
      if (t->bound_cond[2 * a] == 0 || t->bound_cond[2 * a + 1] == 0) continue;
      GhostDesc q;
      memset(&q, 0, sizeof(q));
      q.patch = i;
      for (int e = 0; e < 3; e++) q.ext[e] = gi.ext[e];
      q.nv = NC;
      q.N = t->ncell[a];
      q.ngl = t->nghost[2 * a];
      q.ngh = t->nghost[2 * a + 1];
      q.total = (long long)(q.ngl + q.ngh) * gi.ext[(a + 1) % 3] * gi.ext[(a + 2) % 3];
      q.first = lay.ghost[a].total;
      lay.ghost[a].total += q.total;
      gd[a].push_back(q);
    }
  }
  // chunks of work items: about eight per CTA slot of the GPU
  size_t off = 0;
  for (int f = 0; f < 5; f++) {
    lay.pass[f].desc_off = off;
    off += sizeof(PassDesc<R>) * n;
    off = (off + 255) & ~(size_t)255;
    const int slots = num_sms() * 3;
    lay.pass[f].chunk = std::max(1, std::min(16, lay.pass[f].nitems / (8 * slots)));
  }
  for (int a = 0; a < 3; a++) {
    lay.ghost[a].desc_off = off;
    lay.ghost[a].npatch = (int)gd[a].size();
    off += sizeof(GhostDesc) * gd[a].size();
    off = (off + 255) & ~(size_t)255;
  }
  lay.bytes = off;
  desc.assign(off, 0);
  for (int f = 0; f < 5; f++) memcpy(desc.data() + lay.pass[f].desc_off, d[f].data(), sizeof(PassDesc<R>) * n);
  for (int a = 0; a < 3; a++)
    if (!gd[a].empty()) memcpy(desc.data() + lay.ghost[a].desc_off, gd[a].data(), sizeof(GhostDesc) * gd[a].size());
  return 0;
}

template <typename R, int NC>
int batch_launch(const BatchLayout &lay, const void *d_desc, unsigned *counters, const void *const *vort,
                 void *const *vel, cudaStream_t st, const char *caller) {
  const int n = lay.npatch;
  BatchIo vin, vout;
  memset(&vin, 0, sizeof(vin));
  memset(&vout, 0, sizeof(vout));
  for (int i = 0; i < n; i++) {
    vin.p[i] = vort[i];
    vout.p[i] = vel[i];
  }
  CK(cudaMemsetAsync(counters, 0, 5 * sizeof(unsigned), st), caller);
  const char *base = reinterpret_cast<const char *>(d_desc);
  auto work = [&](int f) {
    BatchWork bw;
    bw.desc = base + lay.pass[f].desc_off;
    bw.npatch = n;
    bw.nitems = lay.pass[f].nitems;
    bw.chunk = lay.pass[f].chunk;
    bw.pad = 0;
    bw.counter = counters + f;
    return bw;
  };
  auto launch = [&](auto kern, int f, auto... args) -> int {
    const size_t sm = lay.pass[f].smem;
    if (smem_attr((const void *)kern, sm, caller)) return -1;
    int per = 1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, RL_THREADS, sm) != cudaSuccess || per < 1) per = 1;
    const int grid = std::max(1, std::min(lay.pass[f].nitems, per * num_sms()));
    kern<<<grid, RL_THREADS, sm, st>>>(work(f), args...);
    PM_LAUNCHED();
    CKL(caller);
    return 0;
  };
  auto lines = [&](int f, int axis, int lmode, int zmode) -> int {
    if constexpr (sizeof(R) == 4) {
      if (lay.pass[f].wide) return launch(k_rlines_batch<R, NC, true>, f, axis, lmode, zmode, 0, 0);
    }
    return launch(k_rlines_batch<R, NC, false>, f, axis, lmode, zmode, 0, 0);
  };
  { KTimer kt_(KC_XFWD, st); if (launch(k_rxfwd_batch<R, NC>, 0, vin)) return -1; }
  { KTimer kt_(KC_YFWD, st); if (lines(1, 1, L_FWD, 0)) return -1; }
  { KTimer kt_(KC_ZPASS, st); if (lines(2, 2, L_Z, Z_VEL)) return -1; }
  { KTimer kt_(KC_YINV, st); if (lines(3, 1, L_INV, 0)) return -1; }
  { KTimer kt_(KC_XINV, st); if (launch(k_rxinv_batch<R, NC>, 4, vout)) return -1; }
  for (int a = 0; a < 3; a++) {
    if (lay.ghost[a].npatch == 0) continue;
    const long long total = lay.ghost[a].total;
    const int nblk = (int)std::min<long long>((total + 255) / 256, 148 * 16);
    const GhostDesc *gd = reinterpret_cast<const GhostDesc *>(base + lay.ghost[a].desc_off);
    { KTimer kt_(KC_GFILL, st);
      k_ghost_fill_batch<R><<<std::max(nblk, 1), 256, 0, st>>>(gd, lay.ghost[a].npatch, total, a, vout); }
    PM_LAUNCHED();
    CKL(caller);
  }
  return 0;
}

// copies the DFT constant tables into this unit's constant memory// copies the DFT constant tables into this unit's constant memory
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

#define PMGPU_INSTANTIATE_BATCH(R, NC)                                                                         \
  namespace pmgpu {                                                                                            \
  template int batch_layout<R, NC>(int, const SolveGeom<R> *, cplx_t<R>::type *const *,                        \
                                   cplx_t<R>::type *const *, const pmgpu_topo *const *,                        \
                                   std::vector<unsigned char> &, BatchLayout &, const char *);                 \
  template int batch_launch<R, NC>(const BatchLayout &, const void *, unsigned *, const void *const *,          \
                                   void *const *, cudaStream_t, const char *);                                 \
  }
