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
// (the kx extent of X and Y is padded to Hp, a multiple of 8, for aligned tiles)
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
#include "regfft.cuh"

namespace pmgpu {

template <typename R> struct SolveGeom {
  typedef typename cplx_t<R>::type C;
  int ext[3];      // cuboid extents including ghosts (x, y, z)
  int off[3];      // first pencil point inside the cuboid (0 free, nghost periodic)
  int P[3];        // pencil extents (free: N + 2 nghost, periodic: N)
  int M[3];        // FFT lengths (free: 2 P, periodic: P)
  int H;           // Mx / 2 + 1
  int Hp;          // H padded to a multiple of 8 (16-byte aligned tile rows)
  int N2;          // Mx / 2
  FftDesc fx, fy, fz;
  const C *twx, *twy, *twz;
  const R *kxt, *kyt, *kzt;  // wavenumbers (cycles / length), Nyquist index included
  const R *green;            // real octant G(kx, |ky|, |kz|) * dx dy dz / (Mx My Mz)
  int gM1, gM2;              // My / 2 + 1, Mz / 2 + 1
  int kernel2;               // derivative kernel (3 components); green holds its spectrum
  R scale;                   // 1 / (Mx My Mz)
  R eps2pi;                  // 2 pi epsilon (filter argument scale)
  int order;                 // filter order (poisson order or reg_order)
  int allper;                // all axes periodic: spectral Green's function
  // in-place register FFTs along y and z (when the lengths factor into register radices)
  int rx_ok, ry_ok, rz_ok;
  RegPlan rx, ry, rz;        // rx: the half-length complex transform of the x passes
  const C *rtwx, *rtwy, *rtwz;  // w_n^q, q < n
  const C *rextx;            // exp(-2 pi i k / Mx), k < H
  const int *xpos;           // frequency -> position of the x transform
  int tky, tkz;              // kx tile of the y / z register passes (0: chosen by shared memory)
  const C *rchx, *rchy, *rchz;  // Bluestein plans: chirp exp(-i pi j^2 / n), j < n
  const C *rbx, *rby, *rbz;     // Bluestein plans: FFT of the wrapped chirp, by position
  const int *yk;             // row of the y spectrum -> ky index (nullptr: natural order)
  const int *zk;             // position of the z transform -> kz index
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

// ---------------------------------------------------------------- common tile machinery
// All passes are persistent: a CTA loops over tiles, and while it transforms tile i
// the rows of tile i+1 stream into a staging buffer with cp.async.  Buffers: S
// (staging), A and B (ping-pong); the first pass reads S, later passes alternate A/B.
constexpr int PASS_THREADS = 512;

template <bool INV, typename R>
__device__ __forceinline__ void vpass_any(const typename Vec<R>::V *src, typename Vec<R>::V *dst, int LG,
                                          const FftDesc &d, int p, const typename cplx_t<R>::type *tw,
                                          const LineMap &lm) {
  const typename cplx_t<R>::type *t = tw + d.twoff[p];
  const int ns = d.ns[p], n = d.n;
  switch (d.rad[p]) {
    case 2: vpass<2, INV, R>(src, dst, LG, n, ns, t, lm); break;
    case 3: vpass<3, INV, R>(src, dst, LG, n, ns, t, lm); break;
    case 4: vpass<4, INV, R>(src, dst, LG, n, ns, t, lm); break;
    case 5: vpass<5, INV, R>(src, dst, LG, n, ns, t, lm); break;
    case 7: vpass<7, INV, R>(src, dst, LG, n, ns, t, lm); break;
    case 8: vpass<8, INV, R>(src, dst, LG, n, ns, t, lm); break;
    case 11: vpass<11, INV, R>(src, dst, LG, n, ns, t, lm); break;
    case 13: vpass<13, INV, R>(src, dst, LG, n, ns, t, lm); break;
    case 16: vpass<16, INV, R>(src, dst, LG, n, ns, t, lm); break;
    case 17: vpass<17, INV, R>(src, dst, LG, n, ns, t, lm); break;
    default: vpass_generic<INV, R>(src, dst, LG, n, ns, d.rad[p], t, tw + d.rootoff[p], lm); break;
  }
}

// A transform that reads `first` (S or A) and ping-pongs between A and B; `hook`
// runs once after the first pass has finished reading `first` (the prefetch point).
template <bool INV, typename R, typename Hook>
__device__ __forceinline__ typename Vec<R>::V *vfft_chain(typename Vec<R>::V *first, typename Vec<R>::V *A,
                                                          typename Vec<R>::V *B, int LG, const FftDesc &d,
                                                          const typename cplx_t<R>::type *tw, const LineMap &lm,
                                                          Hook hook) {
  typedef typename Vec<R>::V V;
  V *src = first, *dst = (first == A) ? B : A;
  for (int p = 0; p < d.npass; p++) {
    vpass_any<INV, R>(src, dst, LG, d, p, tw, lm);
    __syncthreads();
    if (p == 0) hook();
    V *nsrc = dst;
    V *ndst = (dst == A) ? B : A;
    src = nsrc;
    dst = ndst;
  }
  if (d.npass == 0) hook();
  return src;
}

struct NoHook {
  __device__ void operator()() const {}
};

// ---------------------------------------------------------------- y and z passes
// Tile t = (outer o, kx-tile kt): L = NC * TK lines of n points.  Row r of the tile
// starts at complex offset ((o * os + kt * TK) + r * rs) * NC and holds L complex.
struct LineTiles {
  int n;          // transform length
  int rows_in;    // rows read (the rest is zero padding)
  int rows_out;   // rows written (truncation)
  long long in_os, in_rs, out_os, out_rs;
  int nouter, nkt, TK;
  FastDiv dLG;    // division by the line vectors per row (register engine)
};

enum LMode { L_FWD = 0, L_INV = 1, L_Z = 2 };

template <typename R>
__device__ __forceinline__ void tile_rows_load(typename cplx_t<R>::type *S, const typename cplx_t<R>::type *in,
                                               long long base, long long rs, int nrows, int L, int NC) {
  // 16-byte chunks; rows are 16-byte aligned (kx padded to a multiple of 8)
  const int cpr = (L * (int)sizeof(typename cplx_t<R>::type)) / 16;
  const int rsub = threadIdx.x / cpr, c = threadIdx.x - rsub * cpr;
  const int RS = blockDim.x / cpr;
  if (rsub >= RS) return;
  const char *src = reinterpret_cast<const char *>(in + base * NC);
  char *dst = reinterpret_cast<char *>(S);
  const size_t rowb = (size_t)L * sizeof(typename cplx_t<R>::type);
  const size_t strideb = (size_t)rs * NC * sizeof(typename cplx_t<R>::type);
  for (int r = rsub; r < nrows; r += RS) cp_async16(dst + r * rowb + c * 16, src + r * strideb + c * 16);
}

template <typename R>
__device__ __forceinline__ void tile_rows_store(typename cplx_t<R>::type *out, const typename cplx_t<R>::type *Rb,
                                                long long base, long long rs, int nrows, int L, int NC) {
  const int cpr = (L * (int)sizeof(typename cplx_t<R>::type)) / 16;
  const int rsub = threadIdx.x / cpr, c = threadIdx.x - rsub * cpr;
  const int RS = blockDim.x / cpr;
  if (rsub >= RS) return;
  char *dst = reinterpret_cast<char *>(out + base * NC);
  const char *src = reinterpret_cast<const char *>(Rb);
  const size_t rowb = (size_t)L * sizeof(typename cplx_t<R>::type);
  const size_t strideb = (size_t)rs * NC * sizeof(typename cplx_t<R>::type);
  for (int r = rsub; r < nrows; r += RS)
    *reinterpret_cast<float4 *>(dst + r * strideb + c * 16) = *reinterpret_cast<const float4 *>(src + r * rowb + c * 16);
}

// the spectral multiply at one point (kx index kx_i, row y of the y spectrum, kz
// index z): the NC values v of the point in place.  kxp: kx wavenumber, Gp: the
// Green's function value (loaded by the caller for the plain velocity solve)
template <typename R, int NC>
__device__ __forceinline__ void z_point(const SolveGeom<R> &g, typename cplx_t<R>::type *v, int kx_i, R kxp, R Gp,
                                        R ky, R kyc, int y, int iy, int z, R kz, int zmode, int reproj,
                                        int use_zeta) {
  typedef typename cplx_t<R>::type C;
  const R twopi = R(6.283185307179586476925286766559);
  if (kx_i >= g.H) {
#pragma unroll
    for (int c = 0; c < NC; c++) v[c] = mk(R(0), R(0));
    return;
  }
  const R kx = kxp;
  const R kxc = (2 * kx_i == g.M[0]) ? R(0) : kx;
  const R kzc = (2 * z == g.M[2]) ? R(0) : kz;
  const R kmag = kx * kx + ky * ky + kz * kz;
  if (zmode == Z_REGULARISE) {
    const R zt = zeta_filter<R>(g.order, g.eps2pi * sqrt(kmag)) * g.scale;
#pragma unroll
    for (int c = 0; c < NC; c++) v[c] = cscale(v[c], zt);
    return;
  }
  if constexpr (NC == 3) {
    R zt = R(1);
    if (use_zeta) zt = zeta_filter<R>(g.order, g.eps2pi * sqrt(kmag));
    if (g.kernel2 && !g.allper) {
      // derivative kernel K (pmlib_poisson_solve.f, kernel 2): component c is
      // i S_c + (-1)^(k_c) E_c, S_c odd along axis c and even along the others
      // (stored for |ky|, |kz| with the sign of the odd axis applied here), E_c the
      // spectrum of the kernel's plane at -M_c/2 dx_c
      const size_t noct = (size_t)g.gM2 * g.gM1 * g.H;
      const int iz = min(z, g.M[2] - z);
      const size_t oc = ((size_t)iz * g.gM1 + iy) * g.H + kx_i;
      const R *E = g.green + 3 * noct;
      R sx = g.green[oc], sy = g.green[noct + oc], sz = g.green[2 * noct + oc];
      if (2 * y > g.M[1]) sy = -sy;
      if (2 * z > g.M[2]) sz = -sz;
      R ex = E[(size_t)iz * g.gM1 + iy];
      R ey = E[(size_t)g.gM2 * g.gM1 + (size_t)iz * g.H + kx_i];
      R ez = E[(size_t)g.gM2 * (g.gM1 + g.H) + (size_t)iy * g.H + kx_i];
      if (kx_i & 1) ex = -ex;
      if (y & 1) ey = -ey;
      if (z & 1) ez = -ez;
      const C Kx = mk(ex, sx), Ky = mk(ey, sy), Kz = mk(ez, sz);
      const C w1 = v[0], w2 = v[1], w3 = v[2];
      if (zmode == Z_VEL) {
        v[0] = csub(cmul(Ky, w3), cmul(Kz, w2));
        v[1] = csub(cmul(Kz, w1), cmul(Kx, w3));
        v[2] = csub(cmul(Kx, w2), cmul(Ky, w1));
      } else {  // Z_VORT: zeta w (+ K 2 pi i (k . w), Nyquist components dropped)
        C o1 = cscale(w1, zt * g.scale), o2 = cscale(w2, zt * g.scale), o3 = cscale(w3, zt * g.scale);
        if (reproj) {
          const C da = cadd(cadd(cscale(w1, kxc), cscale(w2, kyc)), cscale(w3, kzc));
          const C dv = mk(-twopi * da.y, twopi * da.x);
          o1 = cadd(o1, cmul(Kx, dv));
          o2 = cadd(o2, cmul(Ky, dv));
          o3 = cadd(o3, cmul(Kz, dv));
        }
        v[0] = o1;
        v[1] = o2;
        v[2] = o3;
      }
      return;
    }
    R G;
    if (g.allper) {
      G = (kmag > R(0)) ? zt / (twopi * twopi * kmag) * g.scale : R(0);
    } else {
      G = Gp;
    }
    const C w1 = v[0], w2 = v[1], w3 = v[2];
    if (zmode == Z_VEL) {
      const C c1 = csub(cscale(w3, kyc), cscale(w2, kzc));
      const C c2 = csub(cscale(w1, kzc), cscale(w3, kxc));
      const C c3 = csub(cscale(w2, kxc), cscale(w1, kyc));
      const R f = G * twopi;
      v[0] = mk(-f * c1.y, f * c1.x);
      v[1] = mk(-f * c2.y, f * c2.x);
      v[2] = mk(-f * c3.y, f * c3.x);
    } else if (zmode == Z_VECPOT) {
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

// z-pass spectral multiply of one tile held in buffer V (complex view C).
// zpos: position -> kz index (nullptr: natural order); kzs: kz wavenumbers (shared
// copy of g.kzt, or nullptr)
template <typename R, int NC>
__device__ __forceinline__ void z_multiply(const SolveGeom<R> &g, typename cplx_t<R>::type *Cb, int L, int TK, int k0,
                                           int y, int zmode, int reproj, int use_zeta, const int *zpos,
                                           const R *kzs = nullptr) {
  typedef typename cplx_t<R>::type C;
  const R twopi = R(6.283185307179586476925286766559);
  const int N = g.M[2];
  const R ky = g.kyt[y];
  const R kyc = (2 * y == g.M[1]) ? R(0) : ky;  // Nyquist component dropped in the curl
  const int iy = min(y, g.M[1] - y);
  const int tks = __ffs(TK) - 1;  // TK is a power of two
  const R *kzt = kzs ? kzs : g.kzt;
  // a thread's points are taken U at a time: the Green's function values and
  // wavenumbers of all U are loaded before any is used, so that their global-memory
  // latencies overlap
  const bool pre = NC == 3 && zmode != Z_REGULARISE && !g.allper && !g.kernel2;
  auto point = [&](int t, R kxp, R Gp) {
    const int q = t >> tks, kk = t - (q << tks);
    const int z = zpos ? zpos[q] : q;
    const int kx_i = k0 + kk;
    C *v = Cb + q * L + kk * NC;
    z_point<R, NC>(g, v, kx_i, kxp, Gp, ky, kyc, y, iy, z, kzt[z], zmode, reproj, use_zeta);
  };
  constexpr int U = 4;
  const int total = N * TK;
  for (int t0 = threadIdx.x; t0 < total; t0 += U * blockDim.x) {
    R kxv[U], Gv[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int t = t0 + u * (int)blockDim.x;
      kxv[u] = R(0);
      Gv[u] = R(0);
      if (t < total) {
        const int q = t >> tks, kk = t - (q << tks);
        const int kx_i = k0 + kk;
        if (kx_i < g.H) {
          kxv[u] = g.kxt[kx_i];
          if (pre) {
            const int z = zpos ? zpos[q] : q;
            Gv[u] = g.green[((size_t)min(z, g.M[2] - z) * g.gM1 + iy) * g.H + kx_i];
          }
        }
      }
    }
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int t = t0 + u * (int)blockDim.x;
      if (t < total) point(t, kxv[u], Gv[u]);
    }
  }
}

// ---------------------------------------------------------------- fused middle of the z pass
// Largest last radix of a z plan whose last forward phase, spectral multiply and first
// inverse phase run in registers (three component lines of RL points a thread).
__host__ __device__ inline bool z_fusable(const RegPlan &pl, int rsize) {
  if (pl.bl || pl.np < 2) return false;
  const int r = pl.rad[pl.np - 1];
  return r >= 2 && r <= (rsize == 4 ? 8 : 6);
}

// The z pass's last forward phase, spectral multiply and first inverse phase in
// registers: a thread takes one block of RL consecutive (digit-reversed) positions of
// the NC component lines of one kx, runs the RL-point forward DFT of each (the last
// decimation-in-frequency phase has no twiddles), multiplies every point, runs the
// inverse DFTs (the first decimation-in-time phase has none either) and writes the
// block back in place.  The arithmetic is that of the two phases and the multiply
// done apart, so the result is the same; two shared-memory round trips and two
// barriers per tile are saved.  Ends with a barrier.
// NCT, TKC: the transform length and the kx tile when known at compile time (0: read
// from pl and TK)
template <int RL, typename R, int NC, int NCT = 0, int TKC = 0>
__device__ __forceinline__ void z_fused_mid_r(const SolveGeom<R> &g, const RegPlan &pl,
                                              typename cplx_t<R>::type *Cb, int L, int TK, int k0, int y, int zmode,
                                              int reproj, int use_zeta, const int *zpos, const R *kzs) {
  typedef typename cplx_t<R>::type C;
  const int nblk = NCT ? NCT / RL : pl.n / RL;
  const R ky = g.kyt[y];
  const R kyc = (2 * y == g.M[1]) ? R(0) : ky;  // Nyquist component dropped in the curl
  const int iy = min(y, g.M[1] - y);
  const bool pre = NC == 3 && zmode != Z_REGULARISE && !g.allper && !g.kernel2;
  const int tks = TKC ? (TKC == 1 ? 0 : TKC == 2 ? 1 : TKC == 4 ? 2 : TKC == 8 ? 3 : 4) : __ffs(TK) - 1;  // TK: 2^k
  if (TKC) L = NC * TKC;
  const int total = nblk * (TKC ? TKC : TK);
  for (int t = threadIdx.x; t < total; t += blockDim.x) {
    const int beta = t >> tks, kk = t - (beta << tks);
    const int kx_i = k0 + kk;
    C *base = Cb + (size_t)beta * RL * L + kk * NC;
    int zs[RL];
    R Gv[RL];
    const R kxp = kx_i < g.H ? g.kxt[kx_i] : R(0);
#pragma unroll
    for (int k = 0; k < RL; k++) {
      zs[k] = zpos[beta * RL + k];
      Gv[k] = R(0);
      if (pre && kx_i < g.H) Gv[k] = g.green[((size_t)min(zs[k], g.M[2] - zs[k]) * g.gM1 + iy) * g.H + kx_i];
    }
    C a[NC][RL];
    // FP32, compile-time kx tile 8, three components and RL = 4: the four blocks of a
    // warp sit a multiple of 16 complex apart, so the same position of every block
    // falls in the same banks.  Threads of odd blocks walk their positions rotated
    // by one (position j + 1 at step j), which puts the warp's two block parities 8
    // complex apart: two wavefronts per access instead of four.  Only the order of
    // the loads and stores changes.  (FP64 accesses need four wavefronts anyway.)
    constexpr bool ROT = sizeof(R) == 4 && RL == 4 && TKC == 8 && NC == 3;
    const int rot = ROT ? (beta & 1) : 0;
#pragma unroll
    for (int c = 0; c < NC; c++) {
      if constexpr (ROT) {
        C tmp[RL];
#pragma unroll
        for (int j = 0; j < RL; j++) tmp[j] = base[((j + rot) & (RL - 1)) * L + c];
#pragma unroll
        for (int j = 0; j < RL; j++) a[c][j] = rot ? tmp[(j + RL - 1) & (RL - 1)] : tmp[j];
      } else {
#pragma unroll
        for (int j = 0; j < RL; j++) a[c][j] = base[j * L + c];
      }
      dft<RL, false>(a[c]);
    }
#pragma unroll
    for (int k = 0; k < RL; k++) {
      C v[NC];
#pragma unroll
      for (int c = 0; c < NC; c++) v[c] = a[c][k];
      z_point<R, NC>(g, v, kx_i, kxp, Gv[k], ky, kyc, y, iy, zs[k], kzs[zs[k]], zmode, reproj, use_zeta);
#pragma unroll
      for (int c = 0; c < NC; c++) a[c][k] = v[c];
    }
#pragma unroll
    for (int c = 0; c < NC; c++) {
      dft<RL, true>(a[c]);
      if constexpr (ROT) {
#pragma unroll
        for (int j = 0; j < RL; j++) base[((j + rot) & (RL - 1)) * L + c] = rot ? a[c][(j + 1) & (RL - 1)] : a[c][j];
      } else {
#pragma unroll
        for (int j = 0; j < RL; j++) base[j * L + c] = a[c][j];
      }
    }
  }
  __syncthreads();
}

template <typename R, int NC>
__device__ __forceinline__ void z_fused_mid(const SolveGeom<R> &g, const RegPlan &pl, typename cplx_t<R>::type *Cb,
                                            int L, int TK, int k0, int y, int zmode, int reproj, int use_zeta,
                                            const int *zpos, const R *kzs) {
  switch (pl.rad[pl.np - 1]) {
    case 2: z_fused_mid_r<2, R, NC>(g, pl, Cb, L, TK, k0, y, zmode, reproj, use_zeta, zpos, kzs); break;
    case 3: z_fused_mid_r<3, R, NC>(g, pl, Cb, L, TK, k0, y, zmode, reproj, use_zeta, zpos, kzs); break;
    case 4: z_fused_mid_r<4, R, NC>(g, pl, Cb, L, TK, k0, y, zmode, reproj, use_zeta, zpos, kzs); break;
    case 5: z_fused_mid_r<5, R, NC>(g, pl, Cb, L, TK, k0, y, zmode, reproj, use_zeta, zpos, kzs); break;
    case 6: z_fused_mid_r<6, R, NC>(g, pl, Cb, L, TK, k0, y, zmode, reproj, use_zeta, zpos, kzs); break;
    default:
      if constexpr (sizeof(R) == 4) {
        if (pl.rad[pl.np - 1] == 7) z_fused_mid_r<7, R, NC>(g, pl, Cb, L, TK, k0, y, zmode, reproj, use_zeta, zpos, kzs);
        else z_fused_mid_r<8, R, NC>(g, pl, Cb, L, TK, k0, y, zmode, reproj, use_zeta, zpos, kzs);
      }
      break;
  }
}

// lines along y (lmode L_FWD / L_INV) or the fused z pass (L_Z, or L_FWD along z
// for the Green's function transform).  axis: 1 = y, 2 = z.
template <typename R, int NC>
__global__ void __launch_bounds__(PASS_THREADS, 1) k_lines(SolveGeom<R> g, LineTiles lt,
                                                            const typename cplx_t<R>::type *in,
                                                            typename cplx_t<R>::type *out, int axis, int lmode,
                                                            int zmode, int reproj, int use_zeta) {
  typedef typename cplx_t<R>::type C;
  typedef typename Vec<R>::V V;
  constexpr int G = Vec<R>::G;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ FftDesc sd;
  if (threadIdx.x == 0) sd = (axis == 1) ? g.fy : g.fz;
  const FftDesc &dsrc = (axis == 1) ? g.fy : g.fz;
  const int ntw = dsrc.ntw;
  C *tw = reinterpret_cast<C *>(smem_raw);
  const int N = lt.n, TK = lt.TK, L = NC * TK, LG = L / G;
  V *S = reinterpret_cast<V *>(tw + ((ntw + 7) & ~7));
  V *A = S + (size_t)LG * N;
  V *B = A + (size_t)LG * N;
  stage_table(tw, axis == 1 ? g.twy : g.twz, ntw);
  {
    C *Sc = reinterpret_cast<C *>(S);
    for (int i = threadIdx.x; i < L * N; i += blockDim.x) Sc[i] = mk(R(0), R(0));
  }
  __syncthreads();
  const LineMap lm = line_map(LG);
  const int ntiles = lt.nouter * lt.nkt;
  auto load = [&](int tile) {
    const int o = tile / lt.nkt, kt = tile - o * lt.nkt;
    tile_rows_load<R>(reinterpret_cast<C *>(S), in, o * lt.in_os + (long long)kt * TK, lt.in_rs, lt.rows_in, L, NC);
    cp_async_commit();
  };
  int tile = blockIdx.x;
  if (tile < ntiles) load(tile);
  for (; tile < ntiles; tile += gridDim.x) {
    cp_async_wait_all();
    __syncthreads();
    const int next = tile + gridDim.x;
    auto hook = [&]() {
      if (next < ntiles) load(next);
    };
    const int o = tile / lt.nkt, kt = tile - o * lt.nkt;
    V *res;
    if (lmode == L_INV) {
      res = vfft_chain<true, R>(S, A, B, LG, sd, tw, lm, hook);
    } else {
      res = vfft_chain<false, R>(S, A, B, LG, sd, tw, lm, hook);
      if (lmode == L_Z) {
        z_multiply<R, NC>(g, reinterpret_cast<C *>(res), L, TK, kt * TK, g.yk ? g.yk[o] : o, zmode, reproj,
                          use_zeta, nullptr);
        __syncthreads();
        res = vfft_chain<true, R>(res, A, B, LG, sd, tw, lm, NoHook());
      }
    }
    tile_rows_store<R>(out, reinterpret_cast<C *>(res), o * lt.out_os + (long long)kt * TK, lt.out_rs, lt.rows_out,
                       L, NC);
    __syncthreads();
  }
  cp_async_wait_all();
}

// Register-engine version of k_lines (lmode L_FWD along y, L_INV along y, L_Z):
// one tile buffer per CTA, transformed in place; the first phase reads the rows
// from global memory (zero padding not read) and the last phase writes them back
// (truncation not written).  Forward y output rows are stored in digit-reversed
// order (row -> ky through g.yk); the z pass keeps its spectrum digit-reversed in
// shared memory (position -> kz through g.zk).  Several CTAs share an SM so that
// one CTA's loads overlap another's transforms.
constexpr int RL_THREADS = 256;

// shared memory of a line pass: tables of the geometry, then the tile buffer
template <typename R> struct RlSmem {
  typename cplx_t<R>::type *tw, *chirp, *bpos;
  int *zpos;
  R *kzs;
  typename RVec<R>::V *buf;
};

// carves the shared memory of a line pass of geometry g and stages its tables (the
// caller synchronises before the first tile)
template <typename R>
__device__ __forceinline__ RlSmem<R> rl_setup(const SolveGeom<R> &g, const LineTiles &lt, int axis, int lmode,
                                              unsigned char *smem_raw) {
  typedef typename cplx_t<R>::type C;
  typedef typename RVec<R>::V V;
  const RegPlan &pl = (axis == 1) ? g.ry : g.rz;
  const int m = pl.n, nl = lt.n;
  const bool blue = pl.bl != 0;
  RlSmem<R> s;
  unsigned char *sp = smem_raw;
  s.tw = reinterpret_cast<C *>(sp);
  sp += ((size_t)m * sizeof(C) + 15) & ~(size_t)15;
  s.zpos = reinterpret_cast<int *>(sp);
  sp += ((size_t)nl * sizeof(int) + 15) & ~(size_t)15;
  s.kzs = reinterpret_cast<R *>(sp);
  sp += ((size_t)nl * sizeof(R) + 15) & ~(size_t)15;
  s.chirp = reinterpret_cast<C *>(sp);
  s.bpos = s.chirp + nl;
  if (blue) sp += ((size_t)(nl + m) * sizeof(C) + 15) & ~(size_t)15;
  s.buf = reinterpret_cast<V *>(sp);
  const C *twg = (axis == 1) ? g.rtwy : g.rtwz;
  for (int i = threadIdx.x; i < m; i += blockDim.x) s.tw[i] = twg[i];
  if (lmode == L_Z)
    for (int i = threadIdx.x; i < nl; i += blockDim.x) {
      s.zpos[i] = g.zk[i];
      s.kzs[i] = g.kzt[i];
    }
  if (blue) {
    const C *cg = (axis == 1) ? g.rchy : g.rchz, *bg = (axis == 1) ? g.rby : g.rbz;
    for (int i = threadIdx.x; i < nl; i += blockDim.x) s.chirp[i] = cg[i];
    for (int i = threadIdx.x; i < m; i += blockDim.x) s.bpos[i] = bg[i];
  }
  return s;
}

// one tile of a line pass (ends with a barrier)
template <typename R, int NC, bool WIDE>
__device__ __forceinline__ void rl_tile(const SolveGeom<R> &g, const LineTiles &lt, const typename cplx_t<R>::type *in,
                                        typename cplx_t<R>::type *out, int axis, int lmode, int zmode, int reproj,
                                        int use_zeta, const RlSmem<R> &s, int tile) {
  typedef typename cplx_t<R>::type C;
  constexpr int G = RVec<R>::G;
  const RegPlan &pl = (axis == 1) ? g.ry : g.rz;
  const int nl = lt.n, TK = lt.TK, L = NC * TK, LG = L / G;
  const bool blue = pl.bl != 0;
  const int o = tile / lt.nkt, kt = tile - o * lt.nkt;
  PhaseGlobal gl;
  gl.in = in + (o * lt.in_os + (long long)kt * TK) * NC;
  gl.out = out + (o * lt.out_os + (long long)kt * TK) * NC;
  gl.rs_in = lt.in_rs * NC;
  gl.rs_out = lt.out_rs * NC;
  gl.rows_in = lt.rows_in;
  gl.rows_out = lt.rows_out;
  if (lmode == L_FWD) {
    if (blue) bfft<R, false>(pl, s.buf, LG, lt.dLG, s.tw, s.chirp, s.bpos, true, true, gl, lt.rows_in, nl);
    else rfft_fwd<R, WIDE>(pl, s.buf, LG, lt.dLG, s.tw, true, true, gl);
  } else if (lmode == L_INV) {
    if (blue) bfft<R, true>(pl, s.buf, LG, lt.dLG, s.tw, s.chirp, s.bpos, true, true, gl, nl, lt.rows_out);
    else rfft_inv<R, WIDE>(pl, s.buf, LG, lt.dLG, s.tw, true, true, gl);
  } else if (!blue && NC == 3 && z_fusable(pl, (int)sizeof(R))) {
    rfft_fwd<R, WIDE>(pl, s.buf, LG, lt.dLG, s.tw, true, false, gl, -1, pl.np - 1);
    z_fused_mid<R, NC>(g, pl, reinterpret_cast<C *>(s.buf), L, TK, kt * TK, g.yk ? g.yk[o] : o, zmode, reproj,
                       use_zeta, s.zpos, s.kzs);
    rfft_inv<R, WIDE>(pl, s.buf, LG, lt.dLG, s.tw, false, true, gl, pl.np - 2);
  } else {
    if (blue) bfft<R, false>(pl, s.buf, LG, lt.dLG, s.tw, s.chirp, s.bpos, true, false, gl, lt.rows_in, nl);
    else rfft_fwd<R, WIDE>(pl, s.buf, LG, lt.dLG, s.tw, true, false, gl);
    z_multiply<R, NC>(g, reinterpret_cast<C *>(s.buf), L, TK, kt * TK, g.yk ? g.yk[o] : o, zmode, reproj, use_zeta,
                      blue ? nullptr : s.zpos, s.kzs);
    __syncthreads();
    if (blue) bfft<R, true>(pl, s.buf, LG, lt.dLG, s.tw, s.chirp, s.bpos, false, true, gl, nl, lt.rows_out);
    else rfft_inv<R, WIDE>(pl, s.buf, LG, lt.dLG, s.tw, false, true, gl);
  }
}

template <typename R, int NC, bool WIDE = false>
__global__ void __launch_bounds__(RL_THREADS, WIDE ? 2 : RMinBlocks<R>::v) k_rlines(SolveGeom<R> g, LineTiles lt,
                                                          const typename cplx_t<R>::type *in,
                                                          typename cplx_t<R>::type *out, int axis, int lmode,
                                                          int zmode, int reproj, int use_zeta) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const RlSmem<R> s = rl_setup<R>(g, lt, axis, lmode, smem_raw);
  __syncthreads();
  const int ntiles = lt.nouter * lt.nkt;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x)
    rl_tile<R, NC, WIDE>(g, lt, in, out, axis, lmode, zmode, reproj, use_zeta, s, tile);
}

// ---------------------------------------------------------------- compile-time line passes
// rl_tile for a plan P (no Bluestein) and a kx tile TK known at compile time: the
// same phases, multiply and fused middle, so the results equal those of rl_tile bit
// for bit.
template <typename P, typename R> __host__ __device__ constexpr bool ct_z_fusable() {
  return P::np >= 2 && P::rad(P::np - 1) >= 2 && P::rad(P::np - 1) <= (sizeof(R) == 4 ? 8 : 6);
}

template <typename R, int NC, typename P, int TK>
__device__ __forceinline__ void rl_tile_ct(const SolveGeom<R> &g, const LineTiles &lt,
                                           const typename cplx_t<R>::type *in, typename cplx_t<R>::type *out,
                                           int lmode, int zmode, int reproj, int use_zeta, const RlSmem<R> &s,
                                           int tile) {
  typedef typename cplx_t<R>::type C;
  constexpr int L = NC * TK, LG = L / RVec<R>::G;
  const int o = tile / lt.nkt, kt = tile - o * lt.nkt;
  PhaseGlobal gl;
  gl.in = in + (o * lt.in_os + (long long)kt * TK) * NC;
  gl.out = out + (o * lt.out_os + (long long)kt * TK) * NC;
  gl.rs_in = lt.in_rs * NC;
  gl.rs_out = lt.out_rs * NC;
  gl.rows_in = lt.rows_in;
  gl.rows_out = lt.rows_out;
  if (lmode == L_FWD) {
    rfft_fwd_ct<P, R, LG, true, true, P::np>(s.buf, s.tw, gl);
  } else if (lmode == L_INV) {
    rfft_inv_ct<P, R, LG, true, true, P::np - 1>(s.buf, s.tw, gl);
  } else {
    const int y = g.yk ? g.yk[o] : o;
    if constexpr (NC == 3 && ct_z_fusable<P, R>()) {
      rfft_fwd_ct<P, R, LG, true, false, P::np - 1>(s.buf, s.tw, gl);
      z_fused_mid_r<P::rad(P::np - 1), R, NC, P::n, TK>(g, RegPlan(), reinterpret_cast<C *>(s.buf), L, TK, kt * TK,
                                                        y, zmode, reproj, use_zeta, s.zpos, s.kzs);
      rfft_inv_ct<P, R, LG, false, true, P::np - 2>(s.buf, s.tw, gl);
    } else {
      rfft_fwd_ct<P, R, LG, true, false, P::np>(s.buf, s.tw, gl);
      z_multiply<R, NC>(g, reinterpret_cast<C *>(s.buf), L, TK, kt * TK, y, zmode, reproj, use_zeta, s.zpos,
                        s.kzs);
      __syncthreads();
      rfft_inv_ct<P, R, LG, false, true, P::np - 1>(s.buf, s.tw, gl);
    }
  }
}

// k_rlines for the compile-time plan (N; R0, R1, R2) and kx tile TK
template <typename R, int NC, bool WIDE, int N, int R0, int R1, int R2, int TK>
__global__ void __launch_bounds__(RL_THREADS, WIDE ? 2 : RMinBlocks<R>::v) k_rlines_ct(SolveGeom<R> g, LineTiles lt,
                                                          const typename cplx_t<R>::type *in,
                                                          typename cplx_t<R>::type *out, int axis, int lmode,
                                                          int zmode, int reproj, int use_zeta) {
  static_assert(RL_THREADS == REG_THREADS, "the compile-time phases stride by REG_THREADS");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const RlSmem<R> s = rl_setup<R>(g, lt, axis, lmode, smem_raw);
  __syncthreads();
  const int ntiles = lt.nouter * lt.nkt;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x)
    rl_tile_ct<R, NC, CtPlan<N, R0, R1, R2>, TK>(g, lt, in, out, lmode, zmode, reproj, use_zeta, s, tile);
}

// ---------------------------------------------------------------- batches of patches
// A batched pass runs one pass family (x forward, y forward, the fused z pass, y
// inverse or x inverse) of every patch of a batch in one launch.  Every patch has a
// descriptor (its geometry and the pass's tiles and arrays) and a range of work
// items, one per tile.  CTAs take chunks of consecutive items from a counter in
// global memory (zeroed before the launch) and load a patch's descriptor and tables
// into shared memory when the patch changes.  Each tile is transformed by the same
// code as in the pass of a single plan, so a patch's result is bit-identical to
// its solve alone.
template <typename R> struct PassDesc {
  SolveGeom<R> g;
  LineTiles lt;     // line passes: the tiles of this patch's lines
  const void *in;   // pass input (x forward: the patch's vorticity)
  void *out;        // pass output (x inverse: the patch's velocity)
  int RB, cs;       // x passes: rows per tile, component stride of the real field
  int vec16;        // x forward: rows are staged in 16-byte chunks
  int first;        // first work item of the patch
  FastDiv dLG;      // x passes: division by the line vectors of a tile
  int ntiles, pad;
};
struct BatchWork {
  const void *desc;   // PassDesc<R>[npatch]
  int npatch, nitems, chunk, pad;
  unsigned *counter;  // zero at the launch
};
// the caller's arrays of a batched solve, one per patch (x forward: vorticity, x
// inverse and ghost fill: velocity), passed by value with the launch
constexpr int BATCH_MAX = 1024;
struct BatchIo {
  const void *p[BATCH_MAX];
};

// the CTA's next chunk of work items [i0, i1); false when none is left
__device__ __forceinline__ bool batch_next(const BatchWork &bw, int &i0, int &i1) {
  __shared__ int s_next;
  __syncthreads();
  if (threadIdx.x == 0) s_next = (int)atomicAdd(bw.counter, (unsigned)bw.chunk);
  __syncthreads();
  i0 = s_next;
  i1 = min(i0 + bw.chunk, bw.nitems);
  return i0 < bw.nitems;
}

// the patch that holds work item `item`, and a copy of its descriptor in shared
// memory when it is not the current one (all threads; ends with a barrier when it
// loads).  Returns true when the patch changed.
template <typename R>
__device__ __forceinline__ bool batch_patch(const BatchWork &bw, int item, PassDesc<R> &sd, int &cur) {
  const PassDesc<R> *d = reinterpret_cast<const PassDesc<R> *>(bw.desc);
  if (cur >= 0 && item >= sd.first && item < sd.first + sd.ntiles) return false;
  int lo = 0, hi = bw.npatch - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (d[mid].first <= item) lo = mid;
    else hi = mid - 1;
  }
  __syncthreads();  // everyone is done with the previous descriptor
  const unsigned *src = reinterpret_cast<const unsigned *>(d + lo);
  unsigned *dst = reinterpret_cast<unsigned *>(&sd);
  for (int i = threadIdx.x; i < (int)(sizeof(PassDesc<R>) / 4); i += blockDim.x) dst[i] = src[i];
  __syncthreads();
  cur = lo;
  return true;
}

template <typename R, int NC, bool WIDE = false>
__global__ void __launch_bounds__(RL_THREADS, WIDE ? 2 : RMinBlocks<R>::v) k_rlines_batch(BatchWork bw, int axis,
                                                                int lmode, int zmode, int reproj, int use_zeta) {
  typedef typename cplx_t<R>::type C;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ PassDesc<R> sd;
  RlSmem<R> s;
  int cur = -1, i0, i1;
  while (batch_next(bw, i0, i1)) {
    for (int it = i0; it < i1; it++) {
      if (batch_patch<R>(bw, it, sd, cur)) {
        s = rl_setup<R>(sd.g, sd.lt, axis, lmode, smem_raw);
        __syncthreads();
      }
      rl_tile<R, NC, WIDE>(sd.g, sd.lt, reinterpret_cast<const C *>(sd.in), reinterpret_cast<C *>(sd.out), axis,
                           lmode, zmode, reproj, use_zeta, s, it - sd.first);
    }
  }
}

// ---------------------------------------------------------------- x passes, register engine
// As k_xfwd / k_xinv below (R2C / C2R through a half-length complex transform),
// with the transform done in place by the register engine: the packed line has
// its second half zero (not read), and the digit-reversed spectrum is addressed
// through the frequency -> position table.
template <typename R> struct RxSmem {
  typename cplx_t<R>::type *tw, *ext, *chirp, *bpos;
  int *xpos;
  void *stage;  // raw rows (forward: reals, inverse: spectrum rows)
  typename RVec<R>::V *buf;
};

// carves the shared memory of an x pass of geometry g with RB rows per tile and
// stages its tables; inverse: the staged rows are spectrum rows of Hp complex
template <typename R, int NC>
__device__ __forceinline__ RxSmem<R> rx_setup(const SolveGeom<R> &g, int RB, bool inverse, unsigned char *smem_raw) {
  typedef typename cplx_t<R>::type C;
  typedef typename RVec<R>::V V;
  const RegPlan &pl = g.rx;
  const bool blue = pl.bl != 0;
  const int N = blue ? pl.bn : pl.n, m = pl.n, H = g.H;
  RxSmem<R> s;
  unsigned char *sp = smem_raw;
  s.tw = reinterpret_cast<C *>(sp);
  sp += ((size_t)m * sizeof(C) + 15) & ~(size_t)15;
  s.ext = reinterpret_cast<C *>(sp);
  sp += ((size_t)H * sizeof(C) + 15) & ~(size_t)15;
  s.xpos = reinterpret_cast<int *>(sp);
  sp += ((size_t)N * sizeof(int) + 15) & ~(size_t)15;
  s.chirp = reinterpret_cast<C *>(sp);
  s.bpos = s.chirp + N;
  if (blue) sp += ((size_t)(N + m) * sizeof(C) + 15) & ~(size_t)15;
  s.stage = sp;
  if (inverse) sp += (size_t)RB * g.Hp * NC * sizeof(C);
  else sp += ((size_t)RB * g.P[0] * NC * sizeof(R) + 15) & ~(size_t)15;
  s.buf = reinterpret_cast<V *>(sp);
  for (int i = threadIdx.x; i < m; i += blockDim.x) s.tw[i] = g.rtwx[i];
  for (int i = threadIdx.x; i < N; i += blockDim.x) s.xpos[i] = g.xpos[i];
  for (int i = threadIdx.x; i < H; i += blockDim.x) s.ext[i] = g.rextx[i];
  if (blue) {
    for (int i = threadIdx.x; i < N; i += blockDim.x) s.chirp[i] = g.rchx[i];
    for (int i = threadIdx.x; i < m; i += blockDim.x) s.bpos[i] = g.rbx[i];
  }
  return s;
}

// x forward: raw rows of tile `tile` into the stage (cp.async, committed)
template <typename R, int NC>
__device__ __forceinline__ void rxf_load(const SolveGeom<R> &g, const R *__restrict__ in, int RB, int cs, int vec16,
                                         const RxSmem<R> &s, int tile) {
  const int P0 = g.P[0];
  const int nrows = g.P[1] * g.P[2];
  R *Sr = reinterpret_cast<R *>(s.stage);
  const int row0 = tile * RB;
  for (int rr = 0; rr < RB; rr++) {
    const int row = row0 + rr;
    if (row >= nrows) break;
    const int y = row % g.P[1], z = row / g.P[1];
    const R *src = in + (((size_t)(z + g.off[2]) * g.ext[1] + (y + g.off[1])) * g.ext[0] + g.off[0]) * cs;
    R *dst = Sr + (size_t)rr * P0 * NC;
    if (vec16) {
      const int nch = (P0 * NC * (int)sizeof(R)) / 16;
      for (int c = threadIdx.x; c < nch; c += blockDim.x)
        cp_async16(reinterpret_cast<char *>(dst) + 16 * c, reinterpret_cast<const char *>(src) + 16 * c);
    } else {
      for (int e = threadIdx.x; e < P0 * NC; e += blockDim.x) {
        const int x = e / NC, c = e - x * NC;
        if (sizeof(R) == 8) cp_async8(dst + e, src + (size_t)x * cs + c);
        else cp_async4(dst + e, src + (size_t)x * cs + c);
      }
    }
  }
  cp_async_commit();
}

// x forward of a staged tile (the caller waited for its copies and synchronised);
// `prefetch` runs once the stage has been read.  Ends with a barrier.
template <typename R, int NC, typename Prefetch>
__device__ __forceinline__ void rxf_tile(const SolveGeom<R> &g, typename cplx_t<R>::type *__restrict__ X, int RB,
                                         const FastDiv &dLG, const RxSmem<R> &s, int tile, Prefetch prefetch) {
  typedef typename cplx_t<R>::type C;
  constexpr int G = RVec<R>::G;
  const RegPlan &pl = g.rx;
  const bool blue = pl.bl != 0;
  const int N = blue ? pl.bn : pl.n, L = NC * RB, LG = L / G, H = g.H;
  const int P0 = g.P[0];
  const int nrows = g.P[1] * g.P[2];
  const int npk = (P0 + 1) / 2;  // packed points that hold data
  const R *Sr = reinterpret_cast<const R *>(s.stage);
  C *Bc = reinterpret_cast<C *>(s.buf);
  const int row0 = tile * RB;
  for (int t = threadIdx.x; t < RB * npk; t += blockDim.x) {
    const int rr = t / npk, m = t - rr * npk;
    const R *xr = Sr + (size_t)rr * P0 * NC;
    const int x0 = 2 * m, x1 = 2 * m + 1;
    const bool ok = row0 + rr < nrows;
#pragma unroll
    for (int c = 0; c < NC; c++) {
      const R a = ok ? xr[x0 * NC + c] : R(0);
      const R b = (ok && x1 < P0) ? xr[x1 * NC + c] : R(0);
      Bc[m * L + rr * NC + c] = mk(a, b);
    }
  }
  __syncthreads();
  prefetch();
  PhaseGlobal gl;
  gl.in = nullptr;
  gl.out = nullptr;
  gl.rs_in = gl.rs_out = 0;
  gl.rows_in = gl.rows_out = N;
  if (blue) bfft<R, false>(pl, s.buf, LG, dLG, s.tw, s.chirp, s.bpos, false, false, gl, npk, N);
  else rfft_fwd<R>(pl, s.buf, LG, dLG, s.tw, false, false, gl, npk);
  for (int t = threadIdx.x; t < RB * g.Hp; t += blockDim.x) {
    const int rr = t / g.Hp, k = t - rr * g.Hp;
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
    for (int c = 0; c < NC; c++) X[((size_t)row * g.Hp + k) * NC + c] = o[c];
  }
  __syncthreads();
}

template <typename R, int NC>
__global__ void __launch_bounds__(RL_THREADS, RMinBlocks<R>::v) k_rxfwd(SolveGeom<R> g, const R *__restrict__ in,
                                                         typename cplx_t<R>::type *__restrict__ X, int RB, int cs,
                                                         int vec16, FastDiv dLG) {
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
    rxf_tile<R, NC>(g, X, RB, dLG, s, tile, [&]() {
      if (next < ntiles) rxf_load<R, NC>(g, in, RB, cs, vec16, s, next);
    });
  }
  cp_async_wait_all();
}

template <typename R, int NC>
__global__ void __launch_bounds__(RL_THREADS, RMinBlocks<R>::v) k_rxfwd_batch(BatchWork bw, BatchIo io) {
  typedef typename cplx_t<R>::type C;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ PassDesc<R> sd;
  RxSmem<R> s;
  int cur = -1, i0, i1, staged = -1;
  while (batch_next(bw, i0, i1)) {
    for (int it = i0; it < i1; it++) {
      if (cur >= 0 && (it < sd.first || it >= sd.first + sd.ntiles)) {
        cp_async_wait_all();  // no copy into the old layout may still be in flight
        staged = -1;
      }
      if (batch_patch<R>(bw, it, sd, cur)) {
        s = rx_setup<R, NC>(sd.g, sd.RB, false, smem_raw);
        __syncthreads();
      }
      const R *in = reinterpret_cast<const R *>(io.p[cur]);
      if (staged != it) rxf_load<R, NC>(sd.g, in, sd.RB, sd.cs, sd.vec16, s, it - sd.first);
      cp_async_wait_all();
      __syncthreads();
      const int next = it + 1;
      const bool pre = next < i1 && next < sd.first + sd.ntiles;
      rxf_tile<R, NC>(sd.g, reinterpret_cast<C *>(sd.out), sd.RB, sd.dLG, s, it - sd.first, [&]() {
        if (pre) rxf_load<R, NC>(sd.g, in, sd.RB, sd.cs, sd.vec16, s, next - sd.first);
      });
      staged = pre ? next : -1;
    }
  }
  cp_async_wait_all();
}

// x inverse: spectrum rows of tile `tile` into the stage (cp.async, committed)
template <typename R, int NC>
__device__ __forceinline__ void rxi_load(const SolveGeom<R> &g, const typename cplx_t<R>::type *__restrict__ X, int RB,
                                         const RxSmem<R> &s, int tile) {
  typedef typename cplx_t<R>::type C;
  const size_t rowc = (size_t)g.Hp * NC;
  const int nrows = g.P[1] * g.P[2];
  const int row0 = tile * RB;
  const int nr = min(RB, nrows - row0);
  const size_t nch = (size_t)nr * rowc * sizeof(C) / 16;
  const char *src = reinterpret_cast<const char *>(X + (size_t)row0 * rowc);
  for (size_t c = threadIdx.x; c < nch; c += blockDim.x)
    cp_async16(reinterpret_cast<char *>(s.stage) + 16 * c, src + 16 * c);
  cp_async_commit();
}

// x inverse of a staged tile (the caller waited for its copies and synchronised);
// `prefetch` runs once the stage has been read.  Ends with a barrier.
template <typename R, int NC, typename Prefetch>
__device__ __forceinline__ void rxi_tile(const SolveGeom<R> &g, R *__restrict__ outp, int RB, int cs,
                                         const FastDiv &dLG, const RxSmem<R> &s, int tile, Prefetch prefetch) {
  typedef typename cplx_t<R>::type C;
  constexpr int G = RVec<R>::G;
  const RegPlan &pl = g.rx;
  const bool blue = pl.bl != 0;
  const int N = blue ? pl.bn : pl.n, L = NC * RB, LG = L / G;
  const size_t rowc = (size_t)g.Hp * NC;
  const int nrows = g.P[1] * g.P[2];
  const C *Sc = reinterpret_cast<const C *>(s.stage);
  C *Bc = reinterpret_cast<C *>(s.buf);
  const int row0 = tile * RB;
  for (int t = threadIdx.x; t < RB * N; t += blockDim.x) {
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
  const int P0 = g.P[0];
  const int nout = (P0 + 1) / 2;
  if (blue) bfft<R, true>(pl, s.buf, LG, dLG, s.tw, s.chirp, s.bpos, false, false, gl, N, nout);
  else rfft_inv<R>(pl, s.buf, LG, dLG, s.tw, false, false, gl);
  for (int t = threadIdx.x; t < RB * nout; t += blockDim.x) {
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

template <typename R, int NC>
__global__ void __launch_bounds__(RL_THREADS, RMinBlocks<R>::v) k_rxinv(SolveGeom<R> g,
                                                         const typename cplx_t<R>::type *__restrict__ X,
                                                         R *__restrict__ outp, int RB, int cs, FastDiv dLG) {
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
    rxi_tile<R, NC>(g, outp, RB, cs, dLG, s, tile, [&]() {
      if (next < ntiles) rxi_load<R, NC>(g, X, RB, s, next);
    });
  }
  cp_async_wait_all();
}

template <typename R, int NC>
__global__ void __launch_bounds__(RL_THREADS, RMinBlocks<R>::v) k_rxinv_batch(BatchWork bw, BatchIo io) {
  typedef typename cplx_t<R>::type C;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ PassDesc<R> sd;
  RxSmem<R> s;
  int cur = -1, i0, i1, staged = -1;
  while (batch_next(bw, i0, i1)) {
    for (int it = i0; it < i1; it++) {
      if (cur >= 0 && (it < sd.first || it >= sd.first + sd.ntiles)) {
        cp_async_wait_all();
        staged = -1;
      }
      if (batch_patch<R>(bw, it, sd, cur)) {
        s = rx_setup<R, NC>(sd.g, sd.RB, true, smem_raw);
        __syncthreads();
      }
      const C *X = reinterpret_cast<const C *>(sd.in);
      if (staged != it) rxi_load<R, NC>(sd.g, X, sd.RB, s, it - sd.first);
      cp_async_wait_all();
      __syncthreads();
      const int next = it + 1;
      const bool pre = next < i1 && next < sd.first + sd.ntiles;
      rxi_tile<R, NC>(sd.g, (R *)io.p[cur], sd.RB, sd.cs, sd.dLG, s, it - sd.first, [&]() {
        if (pre) rxi_load<R, NC>(sd.g, X, sd.RB, s, next - sd.first);
      });
      staged = pre ? next : -1;
    }
  }
  cp_async_wait_all();
}

// ---------------------------------------------------------------- x forward (R2C)
// RB rows per tile, L = NC RB real lines packed as N = Mx/2 complex points
// (z[m] = x[2m] + i x[2m+1]); the Mx-point spectrum X[k], k < H follows from Z[k]
// and Z[N-k].  Rows of the real cuboid are staged raw in S.
template <typename R, int NC>
__global__ void __launch_bounds__(PASS_THREADS, 1) k_xfwd(SolveGeom<R> g, const R *__restrict__ in,
                                                           typename cplx_t<R>::type *__restrict__ X, int RB, int cs,
                                                           int vec16) {
  typedef typename cplx_t<R>::type C;
  typedef typename Vec<R>::V V;
  constexpr int G = Vec<R>::G;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ FftDesc sd;
  if (threadIdx.x == 0) sd = g.fx;
  const int ntw = g.fx.ntw + g.fx.next;
  C *tw = reinterpret_cast<C *>(smem_raw);
  const int N = g.N2, L = NC * RB, LG = L / G;
  const int P0 = g.P[0];
  const size_t sreal = (size_t)RB * P0 * NC;  // staged reals
  const size_t sS = ((sreal * sizeof(R) + 15) / 16) * 16 / sizeof(V);
  V *S = reinterpret_cast<V *>(tw + ((ntw + 7) & ~7));
  V *A = S + sS;
  V *B = A + (size_t)LG * N;
  stage_table(tw, g.twx, ntw);
  const LineMap lm = line_map(LG);
  const int nrows = g.P[1] * g.P[2];
  const int ntiles = (nrows + RB - 1) / RB;
  R *Sr = reinterpret_cast<R *>(S);
  auto load = [&](int tile) {
    const int row0 = tile * RB;
    for (int rr = 0; rr < RB; rr++) {
      const int row = row0 + rr;
      if (row >= nrows) break;
      const int y = row % g.P[1], z = row / g.P[1];
      const R *src = in + (((size_t)(z + g.off[2]) * g.ext[1] + (y + g.off[1])) * g.ext[0] + g.off[0]) * cs;
      R *dst = Sr + (size_t)rr * P0 * NC;
      if (vec16) {
        const int nch = (P0 * NC * (int)sizeof(R)) / 16;
        for (int c = threadIdx.x; c < nch; c += blockDim.x)
          cp_async16(reinterpret_cast<char *>(dst) + 16 * c, reinterpret_cast<const char *>(src) + 16 * c);
      } else {
        for (int e = threadIdx.x; e < P0 * NC; e += blockDim.x) {
          const int x = e / NC, c = e - x * NC;
          if (sizeof(R) == 8) cp_async8(dst + e, src + (size_t)x * cs + c);
          else cp_async4(dst + e, src + (size_t)x * cs + c);
        }
      }
    }
    cp_async_commit();
  };
  int tile = blockIdx.x;
  if (tile < ntiles) load(tile);
  for (; tile < ntiles; tile += gridDim.x) {
    cp_async_wait_all();
    __syncthreads();
    const int row0 = tile * RB;
    // pack the staged reals into complex lines
    C *Ac = reinterpret_cast<C *>(A);
    for (int t = threadIdx.x; t < RB * N; t += blockDim.x) {
      const int rr = t / N, m = t - rr * N;
      const R *xr = Sr + (size_t)rr * P0 * NC;
      const int x0 = 2 * m, x1 = 2 * m + 1;
#pragma unroll
      for (int c = 0; c < NC; c++) {
        const R a = (x0 < P0 && row0 + rr < nrows) ? xr[x0 * NC + c] : R(0);
        const R b = (x1 < P0 && row0 + rr < nrows) ? xr[x1 * NC + c] : R(0);
        Ac[m * L + rr * NC + c] = mk(a, b);
      }
    }
    __syncthreads();
    const int next = tile + gridDim.x;
    if (next < ntiles) load(next);
    V *res = vfft_chain<false, R>(A, A, B, LG, sd, tw, lm, NoHook());
    const C *Z = reinterpret_cast<const C *>(res);
    const C *W = tw + sd.extoff;  // exp(-2 pi i k / Mx), k < H
    for (int t = threadIdx.x; t < RB * g.Hp; t += blockDim.x) {
      const int rr = t / g.Hp, k = t - rr * g.Hp;
      const int row = row0 + rr;
      if (row >= nrows) continue;
      C o[NC];
      if (k < g.H) {
        const int kk = (k == N) ? 0 : k;
        const int km = (k == 0 || k == N) ? 0 : N - k;
        const C w = W[k];
#pragma unroll
        for (int c = 0; c < NC; c++) {
          const C zk = Z[kk * L + rr * NC + c];
          const C zn = cconj(Z[km * L + rr * NC + c]);
          const C a = cadd(zk, zn), bb = csub(zk, zn);
          const C wb = cmul(w, bb);
          o[c] = mk(R(0.5) * (a.x + wb.y), R(0.5) * (a.y - wb.x));  // (a - i W^k b) / 2
        }
      } else {
#pragma unroll
        for (int c = 0; c < NC; c++) o[c] = mk(R(0), R(0));
      }
#pragma unroll
      for (int c = 0; c < NC; c++) X[((size_t)row * g.Hp + k) * NC + c] = o[c];
    }
    __syncthreads();
  }
  cp_async_wait_all();
}

// ---------------------------------------------------------------- x inverse (C2R)
template <typename R, int NC>
__global__ void __launch_bounds__(PASS_THREADS, 1) k_xinv(SolveGeom<R> g, const typename cplx_t<R>::type *__restrict__ X,
                                                           R *__restrict__ outp, int RB, int cs) {
  typedef typename cplx_t<R>::type C;
  typedef typename Vec<R>::V V;
  constexpr int G = Vec<R>::G;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ FftDesc sd;
  if (threadIdx.x == 0) sd = g.fx;
  const int ntw = g.fx.ntw + g.fx.next;
  C *tw = reinterpret_cast<C *>(smem_raw);
  const int N = g.N2, L = NC * RB, LG = L / G;
  const size_t rowc = (size_t)g.Hp * NC;  // complex per X row
  const size_t sS = (RB * rowc * sizeof(C)) / sizeof(V);
  V *S = reinterpret_cast<V *>(tw + ((ntw + 7) & ~7));
  V *A = S + sS;
  V *B = A + (size_t)LG * N;
  stage_table(tw, g.twx, ntw);
  const LineMap lm = line_map(LG);
  const int nrows = g.P[1] * g.P[2];
  const int ntiles = (nrows + RB - 1) / RB;
  C *Sc = reinterpret_cast<C *>(S);
  auto load = [&](int tile) {
    const int row0 = tile * RB;
    const int nr = min(RB, nrows - row0);
    const size_t nch = (size_t)nr * rowc * sizeof(C) / 16;
    const char *src = reinterpret_cast<const char *>(X + (size_t)row0 * rowc);
    for (size_t c = threadIdx.x; c < nch; c += blockDim.x)
      cp_async16(reinterpret_cast<char *>(Sc) + 16 * c, src + 16 * c);
    cp_async_commit();
  };
  int tile = blockIdx.x;
  if (tile < ntiles) load(tile);
  for (; tile < ntiles; tile += gridDim.x) {
    cp_async_wait_all();
    __syncthreads();
    const int row0 = tile * RB;
    const C *W = tw + sd.extoff;
    C *Ac = reinterpret_cast<C *>(A);
    for (int t = threadIdx.x; t < RB * N; t += blockDim.x) {
      const int rr = t / N, m = t - rr * N;
      const C w = cconj(W[m]);
      const bool ok = row0 + rr < nrows;
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
        Ac[m * L + rr * NC + c] = z;
      }
    }
    __syncthreads();
    const int next = tile + gridDim.x;
    if (next < ntiles) load(next);
    V *res = vfft_chain<true, R>(A, A, B, LG, sd, tw, lm, NoHook());
    const C *Rc = reinterpret_cast<const C *>(res);
    for (int t = threadIdx.x; t < RB * N; t += blockDim.x) {
      const int rr = t / N, m = t - rr * N;
      const int row = row0 + rr;
      if (row >= nrows) continue;
      const int y = row % g.P[1], z = row / g.P[1];
      R *dst = outp + (((size_t)(z + g.off[2]) * g.ext[1] + (y + g.off[1])) * g.ext[0] + g.off[0]) * cs;
      const int x0 = 2 * m, x1 = 2 * m + 1;
#pragma unroll
      for (int c = 0; c < NC; c++) {
        const C v = Rc[m * L + rr * NC + c];
        if (x0 < g.P[0]) dst[(size_t)x0 * cs + c] = v.x;
        if (x1 < g.P[0]) dst[(size_t)x1 * cs + c] = v.y;
      }
    }
    __syncthreads();
  }
  cp_async_wait_all();
}

// ---------------------------------------------------------------- periodic ghosts
// ghost fill after the inverse transform (source/fourier/pmlib_fourier_ifft.f:247-253):
// along a periodic axis the ghosts copy the interior one period away.
// ghost point t of the (ngl + ngh) x e[o1] x e[o2] strips along `axis`
template <typename R>
__device__ __forceinline__ void ghost_fill_point(R *__restrict__ mesh, int ex, int ey, int ez, int nv, int axis, int N,
                                                 int ngl, int ngh, long long t) {
  const int e[3] = {ex, ey, ez};
  const int ng = ngl + ngh;
  const int o1 = axis == 0 ? 1 : 0, o2 = axis == 2 ? 1 : 2;
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

template <typename R>
__global__ void k_ghost_fill(R *__restrict__ mesh, int ex, int ey, int ez, int nv, int axis, int N,
                             int ngl, int ngh) {
  const int e[3] = {ex, ey, ez};
  const int o1 = axis == 0 ? 1 : 0, o2 = axis == 2 ? 1 : 2;
  const long long total = (long long)(ngl + ngh) * e[o1] * e[o2];
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x)
    ghost_fill_point<R>(mesh, ex, ey, ez, nv, axis, N, ngl, ngh, t);
}

// the ghost fill along one axis of every patch of a batch that is periodic there:
// patch i's ghost points are items [first, first + total) of one index space
struct GhostDesc {
  long long first, total;
  int patch, ext[3], nv, N, ngl, ngh;
};
template <typename R>
__global__ void k_ghost_fill_batch(const GhostDesc *__restrict__ d, int npatch, long long total, int axis,
                                   BatchIo io) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    int lo = 0, hi = npatch - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (d[mid].first <= t) lo = mid;
      else hi = mid - 1;
    }
    const GhostDesc &q = d[lo];
    ghost_fill_point<R>((R *)io.p[q.patch], q.ext[0], q.ext[1], q.ext[2], q.nv, axis, q.N, q.ngl, q.ngh,
                        t - q.first);
  }
}

}  // namespace pmgpu
