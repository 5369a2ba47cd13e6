// solve.cuh -- the unbounded FFT Poisson solve as five HBM passes.
//
// The reference (source/poisson/pmlib_poisson_solve.f) transforms the complex copy
// of the cuboid vorticity along fft_seq(1) and fft_seq(2), runs the third-axis lines
// (zero-pad, FFT, multiply by the Green's function, spectral curl, iFFT, truncate),
// transforms back and keeps REAL().  The 3-D DFT is separable, so the result does
// not depend on the axis order; here the passes always run x, y, z:
//
//   x_fwd : real cuboid -> X[z][y][kx][c], kx < H = Mx/2+1   (R2C, zero-pad fused)
//   y_fwd : X -> Y[z][ky][kx][c], ky < My                      (C2C, zero-pad fused)
//   z_pass: Y -> Y (or another buffer): pad, FFT, multiply+curl, iFFT, truncate
//   y_inv : Y -> X (truncate to the pencil extent)
//   x_inv : X -> real cuboid                                     (C2R, truncate fused)
//
// REAL() of the reference's complex inverse equals the C2R inverse of the Hermitian
// part of the spectrum.  The curl's Nyquist wavenumber (-M/(2L), source
// pmlib_poisson_solve.f:268-306) makes i k x w non-Hermitian on the Nyquist planes;
// its Hermitian part is the curl with the Nyquist components of k set to zero, which
// is what z_pass applies (the filter zeta uses |k|^2 and keeps them).
#pragma once

#include "common.cuh"
#include "fft.cuh"

namespace pmgpu {

template <typename R> struct SolveGeom {
  typedef typename cplx_t<R>::type C;
  int ext[3];      // cuboid extents including ghosts (x, y, z)
  int off[3];      // first pencil point inside the cuboid (0 free, nghost periodic)
  int P[3];        // pencil extents (free: N + 2 nghost, periodic: N)
  int M[3];        // FFT lengths (free: 2 P, periodic: P)
  int H;           // Mx / 2 + 1
  int N2;          // Mx / 2
  FftDesc fx, fy, fz;
  const C *twx, *twy, *twz;
  const R *kxt, *kyt, *kzt;  // wavenumbers (cycles / length), Nyquist index included
  const R *green;            // real octant G(kx, |ky|, |kz|) * dx dy dz / (Mx My Mz)
  int gM1, gM2;              // My / 2 + 1, Mz / 2 + 1
  R scale;                   // 1 / (Mx My Mz)
  R eps2pi;                  // 2 pi epsilon (filter argument scale)
  int order;                 // filter order (poisson order or reg_order)
  int allper;                // all axes periodic: spectral Green's function
};

enum ZMode { Z_VEL = 0, Z_VORT = 1, Z_VECPOT = 2, Z_REGULARISE = 3, Z_FORWARD = 4 };

// zeta(s) = (1 + s^2/2 + s^4/8 + s^6/48 + s^8/384 ...) exp(-s^2/2), truncated by order
// (source/poisson/pmlib_poisson_solve.f:309-334, source/regularise/pmlib_regularise.f:255-282)
template <typename R> __device__ __forceinline__ R zeta_filter(int order, R s) {
  const R s2 = s * s;
  const R e = exp(R(-0.5) * s2);
  R p = R(1);
  if (order >= 4) p += R(0.5) * s2;
  if (order >= 6) p += R(0.125) * s2 * s2;
  if (order >= 8) p += (R(1) / R(48)) * s2 * s2 * s2;
  if (order >= 10) p += (R(1) / R(384)) * s2 * s2 * s2 * s2;
  return order == 0 ? R(1) : p * e;
}

// ---------------------------------------------------------------- x forward (R2C)
template <typename R, int NC>
__global__ void __launch_bounds__(256, 2) k_xfwd(SolveGeom<R> g, const R *__restrict__ in,
                                              typename cplx_t<R>::type *__restrict__ X, int RB, int cs) {
  typedef typename cplx_t<R>::type C;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ FftDesc sd;
  if (threadIdx.x == 0) sd = g.fx;
  const int N = g.N2, L = NC * RB;
  const int ntw = g.fx.ntw + g.fx.next;
  C *tw = reinterpret_cast<C *>(smem_raw);
  C *A = tw + ((ntw + 1) & ~1);
  C *B = A + (size_t)L * N;
  stage_table(tw, g.twx, ntw);
  const int nrows = g.P[1] * g.P[2];
  const int row0 = blockIdx.x * RB;
  for (int t = threadIdx.x; t < RB * N; t += blockDim.x) {
    const int rr = t / N, m = t - rr * N;
    const int row = row0 + rr;
    R a[NC], b[NC];
#pragma unroll
    for (int c = 0; c < NC; c++) { a[c] = R(0); b[c] = R(0); }
    if (row < nrows) {
      const int y = row % g.P[1], z = row / g.P[1];
      const R *src = in + (((size_t)(z + g.off[2]) * g.ext[1] + (y + g.off[1])) * g.ext[0] + g.off[0]) * cs;
      const int x0 = 2 * m, x1 = 2 * m + 1;
      if (x0 < g.P[0]) {
#pragma unroll
        for (int c = 0; c < NC; c++) a[c] = src[(size_t)x0 * cs + c];
      }
      if (x1 < g.P[0]) {
#pragma unroll
        for (int c = 0; c < NC; c++) b[c] = src[(size_t)x1 * cs + c];
      }
    }
#pragma unroll
    for (int c = 0; c < NC; c++) A[m * L + rr * NC + c] = mk(a[c], b[c]);
  }
  __syncthreads();
  C *Z = fft_batch<false>(A, B, L, sd, tw);
  const C *W = tw + g.fx.extoff;  // exp(-2 pi i k / Mx), k < H
  for (int t = threadIdx.x; t < RB * g.H; t += blockDim.x) {
    const int rr = t / g.H, k = t - rr * g.H;
    const int row = row0 + rr;
    if (row >= nrows) continue;
    const int kk = (k == N) ? 0 : k;
    const int km = (k == 0 || k == N) ? 0 : N - k;
    const C w = W[k];
#pragma unroll
    for (int c = 0; c < NC; c++) {
      const C zk = Z[kk * L + rr * NC + c];
      const C zn = cconj(Z[km * L + rr * NC + c]);
      const C a = cadd(zk, zn), bb = csub(zk, zn);
      const C wb = cmul(w, bb);
      // X[k] = (a - i W^k b) / 2
      X[((size_t)row * g.H + k) * NC + c] = mk(R(0.5) * (a.x + wb.y), R(0.5) * (a.y - wb.x));
    }
  }
}

// ---------------------------------------------------------------- y forward / inverse
// lines along y for a tile of TK consecutive kx at one z; IN has `rows_in` rows,
// the transform length is M1, OUT receives `rows_out` rows.
template <typename R, int NC, bool INV>
__global__ void __launch_bounds__(256, 2) k_ypass(SolveGeom<R> g, const typename cplx_t<R>::type *__restrict__ in,
                                               typename cplx_t<R>::type *__restrict__ out, int TK,
                                               int rows_in, int rows_out) {
  typedef typename cplx_t<R>::type C;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ FftDesc sd;
  if (threadIdx.x == 0) sd = g.fy;
  const int N = g.M[1], L = NC * TK;
  const int ntw = g.fy.ntw;
  C *tw = reinterpret_cast<C *>(smem_raw);
  C *A = tw + ((ntw + 1) & ~1);
  C *B = A + (size_t)L * N;
  stage_table(tw, g.twy, ntw);
  const int k0 = blockIdx.x * TK, z = blockIdx.y;
  const int nk = min(TK, g.H - k0), Lv = NC * nk;
  const C zero = mk(R(0), R(0));
  for (int t = threadIdx.x; t < N * L; t += blockDim.x) {
    const int y = t / L, l = t - y * L;
    C v = zero;
    if (y < rows_in && l < Lv) v = in[(((size_t)z * rows_in + y) * g.H + k0) * NC + l];
    A[t] = v;
  }
  __syncthreads();
  C *res = fft_batch<INV>(A, B, L, sd, tw);
  for (int t = threadIdx.x; t < rows_out * L; t += blockDim.x) {
    const int y = t / L, l = t - y * L;
    if (l < Lv) out[(((size_t)z * rows_out + y) * g.H + k0) * NC + l] = res[t];
  }
}

// ---------------------------------------------------------------- z pass (fused)
template <typename R, int NC>
__global__ void __launch_bounds__(256, 2) k_zpass(SolveGeom<R> g, const typename cplx_t<R>::type *in,
                                               typename cplx_t<R>::type *out, int TK,
                                               int mode, int reproj, int use_zeta) {
  typedef typename cplx_t<R>::type C;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ FftDesc sd;
  if (threadIdx.x == 0) sd = g.fz;
  const int N = g.M[2], L = NC * TK;
  const int ntw = g.fz.ntw;
  C *tw = reinterpret_cast<C *>(smem_raw);
  C *A = tw + ((ntw + 1) & ~1);
  C *B = A + (size_t)L * N;
  stage_table(tw, g.twz, ntw);
  const int k0 = blockIdx.x * TK, y = blockIdx.y;
  const int nk = min(TK, g.H - k0), Lv = NC * nk;
  const int M1 = g.M[1];
  const int rows_in = (mode == Z_FORWARD) ? g.M[2] : g.P[2];
  const C zero = mk(R(0), R(0));
  for (int t = threadIdx.x; t < N * L; t += blockDim.x) {
    const int z = t / L, l = t - z * L;
    C v = zero;
    if (z < rows_in && l < Lv) v = in[(((size_t)z * M1 + y) * g.H + k0) * NC + l];
    A[t] = v;
  }
  __syncthreads();
  C *res = fft_batch<false>(A, B, L, sd, tw);
  if (mode == Z_FORWARD) {
    for (int t = threadIdx.x; t < N * L; t += blockDim.x) {
      const int z = t / L, l = t - z * L;
      if (l < Lv) out[(((size_t)z * M1 + y) * g.H + k0) * NC + l] = res[t];
    }
    return;
  }
  C *other = (res == A) ? B : A;
  const R twopi = R(6.283185307179586476925286766559);
  const R ky = g.kyt[y];
  const R kyc = (2 * y == g.M[1]) ? R(0) : ky;  // Nyquist component dropped in the curl
  for (int t = threadIdx.x; t < N * TK; t += blockDim.x) {
    const int z = t / TK, kk = t - z * TK;
    if (kk >= nk) continue;
    const int kx_i = k0 + kk;
    const R kx = g.kxt[kx_i], kz = g.kzt[z];
    const R kxc = (2 * kx_i == g.M[0]) ? R(0) : kx;
    const R kzc = (2 * z == g.M[2]) ? R(0) : kz;
    C *v = res + z * L + kk * NC;
    const R kmag = kx * kx + ky * ky + kz * kz;
    if (mode == Z_REGULARISE) {
      const R zt = zeta_filter<R>(g.order, g.eps2pi * sqrt(kmag)) * g.scale;
#pragma unroll
      for (int c = 0; c < NC; c++) v[c] = cscale(v[c], zt);
      continue;
    }
    if constexpr (NC == 3) {
      R zt = R(1);
      if (use_zeta) zt = zeta_filter<R>(g.order, g.eps2pi * sqrt(kmag));
      R G;
      if (g.allper) {
        G = (kmag > R(0)) ? zt / (twopi * twopi * kmag) * g.scale : R(0);
      } else {
        const int iy = min(y, g.M[1] - y), iz = min(z, g.M[2] - z);
        G = g.green[((size_t)iz * g.gM1 + iy) * g.H + kx_i];
      }
      const C w1 = v[0], w2 = v[1], w3 = v[2];
      if (mode == Z_VEL) {
        // u = G 2 pi i (k x w)
        const C c1 = csub(cscale(w3, kyc), cscale(w2, kzc));
        const C c2 = csub(cscale(w1, kzc), cscale(w3, kxc));
        const C c3 = csub(cscale(w2, kxc), cscale(w1, kyc));
        const R f = G * twopi;
        v[0] = mk(-f * c1.y, f * c1.x);
        v[1] = mk(-f * c2.y, f * c2.x);
        v[2] = mk(-f * c3.y, f * c3.x);
      } else if (mode == Z_VECPOT) {
        v[0] = cscale(w1, G);
        v[1] = cscale(w2, G);
        v[2] = cscale(w3, G);
      } else {  // Z_VORT: zeta w (+ reprojection -4 pi^2 G k (k . w), Hermitian part)
        C o1 = cscale(w1, zt * g.scale), o2 = cscale(w2, zt * g.scale), o3 = cscale(w3, zt * g.scale);
        if (reproj) {
          const R nx = kx - kxc, ny = ky - kyc, nz = kz - kzc;
          const C da = cadd(cadd(cscale(w1, kxc), cscale(w2, kyc)), cscale(w3, kzc));
          const C dn = cadd(cadd(cscale(w1, nx), cscale(w2, ny)), cscale(w3, nz));
          const R f = -twopi * twopi * G;
          o1 = cadd(o1, cscale(cadd(cscale(da, kxc), cscale(dn, nx)), f));
          o2 = cadd(o2, cscale(cadd(cscale(da, kyc), cscale(dn, ny)), f));
          o3 = cadd(o3, cscale(cadd(cscale(da, kzc), cscale(dn, nz)), f));
        }
        v[0] = o1;
        v[1] = o2;
        v[2] = o3;
      }
    }
  }
  // padding lines (kk >= nk) stay zero through the multiply
  __syncthreads();
  C *res2 = fft_batch<true>(res, other, L, sd, tw);
  for (int t = threadIdx.x; t < g.P[2] * L; t += blockDim.x) {
    const int z = t / L, l = t - z * L;
    if (l < Lv) out[(((size_t)z * M1 + y) * g.H + k0) * NC + l] = res2[t];
  }
}

// ---------------------------------------------------------------- x inverse (C2R)
template <typename R, int NC>
__global__ void __launch_bounds__(256, 2) k_xinv(SolveGeom<R> g, const typename cplx_t<R>::type *__restrict__ X,
                                              R *__restrict__ outp, int RB, int cs) {
  typedef typename cplx_t<R>::type C;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ FftDesc sd;
  if (threadIdx.x == 0) sd = g.fx;
  const int N = g.N2, L = NC * RB;
  const int ntw = g.fx.ntw + g.fx.next;
  C *tw = reinterpret_cast<C *>(smem_raw);
  C *A = tw + ((ntw + 1) & ~1);
  C *B = A + (size_t)L * N;
  stage_table(tw, g.twx, ntw);
  __syncthreads();
  const C *W = tw + g.fx.extoff;
  const int nrows = g.P[1] * g.P[2];
  const int row0 = blockIdx.x * RB;
  for (int t = threadIdx.x; t < RB * N; t += blockDim.x) {
    const int rr = t / N, m = t - rr * N;
    const int row = row0 + rr;
    const C w = cconj(W[m]);
#pragma unroll
    for (int c = 0; c < NC; c++) {
      C z = mk(R(0), R(0));
      if (row < nrows) {
        C xm = X[((size_t)row * g.H + m) * NC + c];
        C xn = X[((size_t)row * g.H + (N - m)) * NC + c];
        if (m == 0) { xm.y = R(0); xn.y = R(0); }  // DC and Nyquist are real
        const C a = cadd(xm, cconj(xn));
        const C b = csub(xm, cconj(xn));
        const C wb = cmul(w, b);
        z = mk(a.x - wb.y, a.y + wb.x);  // a + i W^{-m} b
      }
      A[m * L + rr * NC + c] = z;
    }
  }
  __syncthreads();
  C *res = fft_batch<true>(A, B, L, sd, tw);
  for (int t = threadIdx.x; t < RB * N; t += blockDim.x) {
    const int rr = t / N, m = t - rr * N;
    const int row = row0 + rr;
    if (row >= nrows) continue;
    const int y = row % g.P[1], z = row / g.P[1];
    R *dst = outp + (((size_t)(z + g.off[2]) * g.ext[1] + (y + g.off[1])) * g.ext[0] + g.off[0]) * cs;
    const int x0 = 2 * m, x1 = 2 * m + 1;
#pragma unroll
    for (int c = 0; c < NC; c++) {
      const C v = res[m * L + rr * NC + c];
      if (x0 < g.P[0]) dst[(size_t)x0 * cs + c] = v.x;
      if (x1 < g.P[0]) dst[(size_t)x1 * cs + c] = v.y;
    }
  }
}

// ---------------------------------------------------------------- periodic ghosts
// ghost fill after the inverse transform (source/fourier/pmlib_fourier_ifft.f:247-253):
// along a periodic axis the ghosts copy the interior one period away.
template <typename R>
__global__ void k_ghost_fill(R *__restrict__ mesh, int ex, int ey, int ez, int nv, int axis, int N,
                             int ngl, int ngh) {
  const int e[3] = {ex, ey, ez};
  const int ng = ngl + ngh;
  const int o1 = axis == 0 ? 1 : 0, o2 = axis == 2 ? 1 : 2;
  const long long total = (long long)ng * e[o1] * e[o2];
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int s = (int)(t % ng);
    const long long r = t / ng;
    const int a = (int)(r % e[o1]), b = (int)(r / e[o1]);
    int dstc = (s < ngl) ? s : ngl + N + (s - ngl);
    int srcc = (s < ngl) ? dstc + N : dstc - N;
    int id[3], is[3];
    id[o1] = a; id[o2] = b; id[axis] = dstc;
    is[o1] = a; is[o2] = b; is[axis] = srcc;
    const size_t di = (((size_t)id[2] * ey + id[1]) * ex + id[0]) * nv;
    const size_t si = (((size_t)is[2] * ey + is[1]) * ex + is[0]) * nv;
    for (int c = 0; c < nv; c++) mesh[di + c] = mesh[si + c];
  }
}

}  // namespace pmgpu
