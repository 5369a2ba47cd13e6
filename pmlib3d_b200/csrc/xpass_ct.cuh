// xpass_ct.cuh -- x forward (R2C) and x inverse (C2R) passes compiled for one plan:
// the packed half-length transform's plan P (no Bluestein), the rows per tile RB,
// the padded real row length P0 and the spectrum row pitch HP known to the compiler.
// The packing, the half-length phases and the twist are the run-time passes'
// (rxf_tile / rxi_tile in solve.cuh) with constants for the loop bounds and the
// divisions, so the results are those of the run-time engine.  Included only by the
// compile-time-plan units (passes_ct_*.cu).
#pragma once

#include "solve.cuh"

namespace pmgpu {

// x forward of a staged tile (the caller waited for its copies and synchronised);
// `prefetch` runs once the stage has been read.  Ends with a barrier.
template <typename R, int NC, typename P, int RB, int P0, int HP, typename Prefetch>
__device__ __forceinline__ void rxf_tile_ct(const SolveGeom<R> &g, typename cplx_t<R>::type *__restrict__ X,
                                            const RxSmem<R> &s, int tile, Prefetch prefetch) {
  typedef typename cplx_t<R>::type C;
  constexpr int N = P::n, L = NC * RB, H = N + 1;
  constexpr int NPK = (P0 + 1) / 2;  // packed points that hold data
  static_assert(RVec<R>::G == 1, "one complex point per vector");
  const int nrows = g.P[1] * g.P[2];
  const R *Sr = reinterpret_cast<const R *>(s.stage);
  C *Bc = reinterpret_cast<C *>(s.buf);
  const int row0 = tile * RB;
  for (int t = threadIdx.x; t < RB * NPK; t += REG_THREADS) {
    const int rr = t / NPK, m = t - rr * NPK;
    const R *xr = Sr + (size_t)rr * P0 * NC;
    const int x0 = 2 * m, x1 = 2 * m + 1;
    const bool ok = row0 + rr < nrows;
    if constexpr (NC == 3 && P0 % 2 == 0) {
      // the six reals of points 2m and 2m+1 as three aligned pairs (rows of 3 P0
      // reals start on even offsets): conflict-free within each half-warp
      C v[3];
#pragma unroll
      for (int h = 0; h < 3; h++) v[h] = ok ? reinterpret_cast<const C *>(xr)[3 * m + h] : mk(R(0), R(0));
      Bc[m * L + rr * NC + 0] = mk(v[0].x, v[1].y);
      Bc[m * L + rr * NC + 1] = mk(v[0].y, v[2].x);
      Bc[m * L + rr * NC + 2] = mk(v[1].x, v[2].y);
    } else {
#pragma unroll
      for (int c = 0; c < NC; c++) {
        const R a = ok ? xr[x0 * NC + c] : R(0);
        const R b = (ok && x1 < P0) ? xr[x1 * NC + c] : R(0);
        Bc[m * L + rr * NC + c] = mk(a, b);
      }
    }
  }
  __syncthreads();
  prefetch();
  PhaseGlobal gl;
  gl.in = nullptr;
  gl.out = nullptr;
  gl.rs_in = gl.rs_out = 0;
  gl.rows_in = NPK;  // the first phase treats positions from NPK on as zero
  gl.rows_out = N;
  rfft_fwd_ct<P, R, L, false, false, P::np>(s.buf, s.tw, gl);
  for (int t = threadIdx.x; t < RB * HP; t += REG_THREADS) {
    const int rr = t / HP, k = t - rr * HP;
    const int row = row0 + rr;
    if (row >= nrows) continue;
    C o[NC];
    if (k < H) {
      const int kk = (k == N) ? 0 : k;
      const int km = (k == 0 || k == N) ? 0 : N - k;
      const int pk = s.xpos[kk], pm = s.xpos[km];
      const C w = s.ext[k];
#pragma unroll
      for (int c = 0; c < NC; c++) {
        const C zk = Bc[pk * L + rr * NC + c];
        const C zn = cconj(Bc[pm * L + rr * NC + c]);
        const C a = cadd(zk, zn), bb = csub(zk, zn);
        const C wb = cmul(w, bb);
        o[c] = mk(R(0.5) * (a.x + wb.y), R(0.5) * (a.y - wb.x));  // (a - i W^k b) / 2
      }
    } else {
#pragma unroll
      for (int c = 0; c < NC; c++) o[c] = mk(R(0), R(0));
    }
#pragma unroll
    for (int c = 0; c < NC; c++) X[((size_t)row * HP + k) * NC + c] = o[c];
  }
  __syncthreads();
}

template <typename R, int NC, int N, int R0, int R1, int R2, int RB, int P0, int HP>
__global__ void __launch_bounds__(RL_THREADS, RMinBlocks<R>::v) k_rxfwd_ct(SolveGeom<R> g, const R *__restrict__ in,
                                                                            typename cplx_t<R>::type *__restrict__ X,
                                                                            int RBrt, int cs, int vec16, FastDiv dLG) {
  static_assert(RL_THREADS == REG_THREADS, "the compile-time phases stride by REG_THREADS");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const RxSmem<R> s = rx_setup<R, NC>(g, RB, false, smem_raw);
  const int nrows = g.P[1] * g.P[2];
  const int ntiles = (nrows + RB - 1) / RB;
  int tile = blockIdx.x;
  if (tile < ntiles) rxf_load<R, NC>(g, in, RB, cs, vec16, s, tile);
  for (; tile < ntiles; tile += gridDim.x) {
    cp_async_wait_all();
    __syncthreads();
    const int next = tile + gridDim.x;
    rxf_tile_ct<R, NC, CtPlan<N, R0, R1, R2>, RB, P0, HP>(g, X, s, tile, [&]() {
      if (next < ntiles) rxf_load<R, NC>(g, in, RB, cs, vec16, s, next);
    });
  }
  cp_async_wait_all();
}

// x inverse of a staged tile (the caller waited for its copies and synchronised);
// `prefetch` runs once the stage has been read.  Ends with a barrier.
template <typename R, int NC, typename P, int RB, int P0, int HP, typename Prefetch>
__device__ __forceinline__ void rxi_tile_ct(const SolveGeom<R> &g, R *__restrict__ outp, int cs, const RxSmem<R> &s,
                                            int tile, Prefetch prefetch) {
  typedef typename cplx_t<R>::type C;
  constexpr int N = P::n, L = NC * RB;
  constexpr size_t rowc = (size_t)HP * NC;
  constexpr int nout = (P0 + 1) / 2;
  const int nrows = g.P[1] * g.P[2];
  const C *Sc = reinterpret_cast<const C *>(s.stage);
  C *Bc = reinterpret_cast<C *>(s.buf);
  const int row0 = tile * RB;
  for (int t = threadIdx.x; t < RB * N; t += REG_THREADS) {
    const int rr = t / N, m = t - rr * N;
    const C w = cconj(s.ext[m]);
    const bool ok = row0 + rr < nrows;
    const int pm = s.xpos[m];
#pragma unroll
    for (int c = 0; c < NC; c++) {
      C z = mk(R(0), R(0));
      if (ok) {
        C xm = Sc[rr * rowc + (size_t)m * NC + c];
        C xn = Sc[rr * rowc + (size_t)(N - m) * NC + c];
        if (m == 0) {
          xm.y = R(0);
          xn.y = R(0);
        }  // DC and Nyquist are real
        const C a = cadd(xm, cconj(xn));
        const C b = csub(xm, cconj(xn));
        const C wb = cmul(w, b);
        z = mk(a.x - wb.y, a.y + wb.x);  // a + i W^{-m} b
      }
      Bc[pm * L + rr * NC + c] = z;
    }
  }
  __syncthreads();
  prefetch();
  PhaseGlobal gl;
  gl.in = nullptr;
  gl.out = nullptr;
  gl.rs_in = gl.rs_out = 0;
  gl.rows_in = gl.rows_out = N;
  rfft_inv_ct<P, R, L, false, false, P::np - 1>(s.buf, s.tw, gl);
  for (int t = threadIdx.x; t < RB * nout; t += REG_THREADS) {
    const int rr = t / nout, m = t - rr * nout;
    const int row = row0 + rr;
    if (row >= nrows) continue;
    const int y = row % g.P[1], z = row / g.P[1];
    R *dst = outp + (((size_t)(z + g.off[2]) * g.ext[1] + (y + g.off[1])) * g.ext[0] + g.off[0]) * cs;
    const int x0 = 2 * m, x1 = 2 * m + 1;
#pragma unroll
    for (int c = 0; c < NC; c++) {
      const C v = Bc[m * L + rr * NC + c];
      dst[(size_t)x0 * cs + c] = v.x;
      if (x1 < P0) dst[(size_t)x1 * cs + c] = v.y;
    }
  }
  __syncthreads();
}

template <typename R, int NC, int N, int R0, int R1, int R2, int RB, int P0, int HP>
__global__ void __launch_bounds__(RL_THREADS, RMinBlocks<R>::v) k_rxinv_ct(SolveGeom<R> g,
                                                                            const typename cplx_t<R>::type *__restrict__ X,
                                                                            R *__restrict__ outp, int RBrt, int cs,
                                                                            FastDiv dLG) {
  static_assert(RL_THREADS == REG_THREADS, "the compile-time phases stride by REG_THREADS");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const RxSmem<R> s = rx_setup<R, NC>(g, RB, true, smem_raw);
  const int nrows = g.P[1] * g.P[2];
  const int ntiles = (nrows + RB - 1) / RB;
  int tile = blockIdx.x;
  if (tile < ntiles) rxi_load<R, NC>(g, X, RB, s, tile);
  for (; tile < ntiles; tile += gridDim.x) {
    cp_async_wait_all();
    __syncthreads();
    const int next = tile + gridDim.x;
    rxi_tile_ct<R, NC, CtPlan<N, R0, R1, R2>, RB, P0, HP>(g, outp, cs, s, tile, [&]() {
      if (next < ntiles) rxi_load<R, NC>(g, X, RB, s, next);
    });
  }
  cp_async_wait_all();
}

}  // namespace pmgpu
