// regfft.cuh -- in-place, register-blocked line FFTs for the solve passes.
//
// A line of length n = R0 R1 ... (at most three phases, radices up to 17) is
// transformed in place in shared memory:
//
//   forward (decimation in frequency): phase p works on blocks of B_p points with
//   stride s_p = B_p / R_p.  Butterfly (block beta, offset r) reads the R_p points
//   beta B_p + r + s_p j, takes their R_p-point DFT in registers, multiplies output k
//   by w_{B_p}^{r k} (skipped in the last phase, where s = 1) and writes it back to
//   beta B_p + r + s_p k.  The result is in digit-reversed order: position
//   p = k0 B_1 + k1 B_2 + k2 holds frequency k0 + R0 (k1 + R1 k2).
//   inverse (decimation in time): the same phases in reverse order with conjugate
//   twiddles applied before the inverse DFT; digit-reversed input, natural output.
//
// The first forward phase can read its points straight from global memory (points
// beyond the row count are the zero padding and are not read), and the last
// inverse phase can write straight to global memory (rows beyond the row count are
// the truncation and are not written), so padding and truncation cost no traffic.
// Consumers of a digit-reversed spectrum index it through a position -> frequency
// table.  Lines are held as vectors of G lines (FP32: float4 = two complex lines;
// FP64: double2 = one) interleaved by position: vector g of position q sits at
// buf[q * LG + g], so consecutive threads touch consecutive 16-byte vectors.
// Twiddles come from one table of w_n^q, q < n, built in long double on the host.
#pragma once

#include "common.cuh"
#include "fft.cuh"

namespace pmgpu {

// u / d for u < 2^31 by multiply-high (Granlund-Montgomery): l = ceil(log2 d),
// m = floor(2^32 (2^l - d) / d) + 1, q = (umulhi(u, m) + u) >> l
struct FastDiv {
  unsigned d, m, l;
};
static inline FastDiv make_fastdiv(unsigned d) {
  FastDiv f;
  f.d = d;
  unsigned l = 0;
  while ((1ull << l) < d) l++;
  f.l = l;
  f.m = (unsigned)((((1ull << l) - d) << 32) / d + 1);
  return f;
}
__host__ __device__ __forceinline__ unsigned fdiv(unsigned u, const FastDiv &f) {
#ifdef __CUDA_ARCH__
  return (__umulhi(u, f.m) + u) >> f.l;
#else
  return (unsigned)((((unsigned long long)u * f.m) >> 32) + u) >> f.l;
#endif
}

constexpr int RP_MAX = 3;
struct RegPlan {
  int n, np;
  int rad[RP_MAX];  // radix of each phase, outermost first
  int blk[RP_MAX];  // block size B_p = n / (R_0 ... R_{p-1})
  int str[RP_MAX];  // stride s_p = B_p / R_p
  int twm[RP_MAX];  // n / B_p: w_{B_p}^q = w_n^{twm q}
  FastDiv dstr[RP_MAX];
  // Bluestein: a line of length bn (with a prime factor above 17) is transformed as
  // a convolution of length n >= 2 bn - 1 (the phases above describe that length)
  int bl, bn;
};

// radices with a register DFT
__host__ __device__ constexpr bool reg_radix(int r) {
  return r == 2 || r == 3 || r == 4 || r == 5 || r == 6 || r == 7 || r == 8 || r == 9 || r == 10 || r == 11 ||
         r == 12 || r == 13 || r == 16 || r == 17;
}
// composite radices of the wide variant of the y / z passes (FP32 only): a thread
// holds up to 24 points, so lengths such as 528 = 22 x 24 take two phases instead
// of three; the kernels that may run them are compiled for two CTAs per SM
__host__ __device__ constexpr bool reg_radix_wide(int r) { return r == 18 || r == 20 || r == 22 || r == 24; }

// where a phase reads from / writes to
struct PhaseGlobal {
  const void *in;          // tile base (complex), row = position
  void *out;
  long long rs_in, rs_out; // row strides in complex elements
  int rows_in;             // rows present in `in` (the rest is zero)
  int rows_out;            // rows wanted in `out`
};

// One line per thread and butterfly: the vector is one complex point, so a radix-R
// butterfly holds R complex values in registers.
template <typename R> struct RVec {
  typedef typename cplx_t<R>::type V;
  static constexpr int G = 1;
};
// CTAs per SM the register-engine kernels are compiled for (register budget)
template <typename R> struct RMinBlocks;
template <> struct RMinBlocks<float> { static constexpr int v = 3; };
template <> struct RMinBlocks<double> { static constexpr int v = 2; };

template <typename V> __device__ __forceinline__ void rsplit(const V &v, V *a) { a[0] = v; }
template <typename V> __device__ __forceinline__ V rmerge(const V *a) { return a[0]; }

template <typename R> __device__ __forceinline__ typename RVec<R>::V ldg_vec(const typename RVec<R>::V *p);
template <> __device__ __forceinline__ float2 ldg_vec<float>(const float2 *p) { return __ldg(p); }
template <> __device__ __forceinline__ double2 ldg_vec<double>(const double2 *p) { return __ldg(p); }

template <typename R> __device__ __forceinline__ typename RVec<R>::V zero_vec();
template <> __device__ __forceinline__ float2 zero_vec<float>() { return make_float2(0.f, 0.f); }
template <> __device__ __forceinline__ double2 zero_vec<double>() { return make_double2(0.0, 0.0); }

// One phase over a tile of LG line vectors.  gsrc / gdst: read from / write to
// global memory instead of `buf`.  twid: the phase carries twiddles.
// nz: points at positions >= nz are zero and are not read (the zero padding of
// the first forward phase; n otherwise)
template <int RAD, bool INV, typename R>
__device__ __forceinline__ void rphase(const RegPlan &pl, int p, typename RVec<R>::V *buf, int LG, const FastDiv &dLG,
                                       const typename cplx_t<R>::type *__restrict__ tw, bool gsrc, bool gdst,
                                       bool twid, const PhaseGlobal &gl, int nz) {
  typedef typename cplx_t<R>::type C;
  typedef typename RVec<R>::V V;
  constexpr int G = RVec<R>::G;
  const int s = pl.str[p], B = pl.blk[p], tm = pl.twm[p];
  const unsigned total = (unsigned)(pl.n / RAD) * (unsigned)LG;
  const V *gin = reinterpret_cast<const V *>(gl.in);
  V *gout = reinterpret_cast<V *>(gl.out);
  const long long vri = gl.rs_in / G, vro = gl.rs_out / G;  // row strides in vectors
  for (unsigned u = threadIdx.x; u < total; u += blockDim.x) {
    const unsigned b = fdiv(u, dLG);
    const int g = (int)(u - b * (unsigned)LG);
    const unsigned beta = fdiv(b, pl.dstr[p]);
    const int r = (int)(b - beta * (unsigned)s);
    const int pos0 = (int)beta * B + r;
    C a[G][RAD];
    if (gsrc) {
      const V *src = gin + (long long)pos0 * vri + g;
#pragma unroll
      for (int j = 0; j < RAD; j++) {
        V v = zero_vec<R>();
        if (pos0 + s * j < nz) v = ldg_vec<R>(src + (long long)(s * j) * vri);
        C t[G];
        rsplit(v, t);
#pragma unroll
        for (int h = 0; h < G; h++) a[h][j] = t[h];
      }
    } else {
      const V *src = buf + pos0 * LG + g;
      if (nz >= pl.n) {
#pragma unroll
        for (int j = 0; j < RAD; j++) {
          C t[G];
          rsplit(src[s * j * LG], t);
#pragma unroll
          for (int h = 0; h < G; h++) a[h][j] = t[h];
        }
      } else {
#pragma unroll
        for (int j = 0; j < RAD; j++) {
          C t[G];
          rsplit(pos0 + s * j < nz ? src[s * j * LG] : zero_vec<R>(), t);
#pragma unroll
          for (int h = 0; h < G; h++) a[h][j] = t[h];
        }
      }
    }
    if (INV && twid) {
      const int tb = tm * r;
#pragma unroll
      for (int j = 1; j < RAD; j++) {
        const C w = tw[tb * j];
#pragma unroll
        for (int h = 0; h < G; h++) a[h][j] = cmulc(a[h][j], w);
      }
    }
#pragma unroll
    for (int h = 0; h < G; h++) dft<RAD, INV>(a[h]);
    if (!INV && twid) {
      const int tb = tm * r;
#pragma unroll
      for (int k = 1; k < RAD; k++) {
        const C w = tw[tb * k];
#pragma unroll
        for (int h = 0; h < G; h++) a[h][k] = cmul(a[h][k], w);
      }
    }
    if (gdst) {
      V *dst = gout + (long long)pos0 * vro + g;
#pragma unroll
      for (int k = 0; k < RAD; k++) {
        C t[G];
#pragma unroll
        for (int h = 0; h < G; h++) t[h] = a[h][k];
        if (pos0 + s * k < gl.rows_out) dst[(long long)(s * k) * vro] = rmerge(t);
      }
    } else {
      V *dst = buf + pos0 * LG + g;
#pragma unroll
      for (int k = 0; k < RAD; k++) {
        C t[G];
#pragma unroll
        for (int h = 0; h < G; h++) t[h] = a[h][k];
        dst[s * k * LG] = rmerge(t);
      }
    }
  }
}

template <bool INV, typename R, bool WIDE = false>
__device__ __forceinline__ void rphase_any(const RegPlan &pl, int p, typename RVec<R>::V *buf, int LG,
                                           const FastDiv &dLG, const typename cplx_t<R>::type *tw, bool gsrc,
                                           bool gdst, bool twid, const PhaseGlobal &gl, int nz) {
  if constexpr (WIDE) {
    switch (pl.rad[p]) {
      case 18: rphase<18, INV, R>(pl, p, buf, LG, dLG, tw, gsrc, gdst, twid, gl, nz); return;
      case 20: rphase<20, INV, R>(pl, p, buf, LG, dLG, tw, gsrc, gdst, twid, gl, nz); return;
      case 22: rphase<22, INV, R>(pl, p, buf, LG, dLG, tw, gsrc, gdst, twid, gl, nz); return;
      case 24: rphase<24, INV, R>(pl, p, buf, LG, dLG, tw, gsrc, gdst, twid, gl, nz); return;
      default: break;
    }
  }
  switch (pl.rad[p]) {
    case 2: rphase<2, INV, R>(pl, p, buf, LG, dLG, tw, gsrc, gdst, twid, gl, nz); break;
    case 3: rphase<3, INV, R>(pl, p, buf, LG, dLG, tw, gsrc, gdst, twid, gl, nz); break;
    case 4: rphase<4, INV, R>(pl, p, buf, LG, dLG, tw, gsrc, gdst, twid, gl, nz); break;
    case 5: rphase<5, INV, R>(pl, p, buf, LG, dLG, tw, gsrc, gdst, twid, gl, nz); break;
    case 6: rphase<6, INV, R>(pl, p, buf, LG, dLG, tw, gsrc, gdst, twid, gl, nz); break;
    case 7: rphase<7, INV, R>(pl, p, buf, LG, dLG, tw, gsrc, gdst, twid, gl, nz); break;
    case 8: rphase<8, INV, R>(pl, p, buf, LG, dLG, tw, gsrc, gdst, twid, gl, nz); break;
    case 9: rphase<9, INV, R>(pl, p, buf, LG, dLG, tw, gsrc, gdst, twid, gl, nz); break;
    case 10: rphase<10, INV, R>(pl, p, buf, LG, dLG, tw, gsrc, gdst, twid, gl, nz); break;
    case 11: rphase<11, INV, R>(pl, p, buf, LG, dLG, tw, gsrc, gdst, twid, gl, nz); break;
    case 12: rphase<12, INV, R>(pl, p, buf, LG, dLG, tw, gsrc, gdst, twid, gl, nz); break;
    case 13: rphase<13, INV, R>(pl, p, buf, LG, dLG, tw, gsrc, gdst, twid, gl, nz); break;
    case 16: rphase<16, INV, R>(pl, p, buf, LG, dLG, tw, gsrc, gdst, twid, gl, nz); break;
    case 17: rphase<17, INV, R>(pl, p, buf, LG, dLG, tw, gsrc, gdst, twid, gl, nz); break;
    default: break;  // plans only hold register radices
  }
}

// forward transform of a tile: natural-order input (global when gfirst, else buf),
// digit-reversed output in buf, or in global memory when glast.  The caller
// synchronises before; every phase but a final global one ends with a barrier.
// nz0: nonzero leading points of an input in buf (the rest is zero padding)
template <typename R, bool WIDE = false>
__device__ __forceinline__ void rfft_fwd(const RegPlan &pl, typename RVec<R>::V *buf, int LG, const FastDiv &dLG,
                                         const typename cplx_t<R>::type *tw, bool gfirst, bool glast,
                                         const PhaseGlobal &gl, int nz0 = -1, int pend = -1) {
  // pend: phases [0, pend) only (the default: all)
  const int np = pend >= 0 ? pend : pl.np;
  for (int p = 0; p < np; p++) {
    const bool last = p == pl.np - 1;
    const int nz = p > 0 ? pl.n : gfirst ? gl.rows_in : nz0 >= 0 ? nz0 : pl.n;
    rphase_any<false, R, WIDE>(pl, p, buf, LG, dLG, tw, gfirst && p == 0, glast && last, !last, gl, nz);
    __syncthreads();
  }
}

// inverse transform: digit-reversed input (global when gfirst, else buf), natural
// output in buf, or in global memory (rows < rows_out) when glast
template <typename R, bool WIDE = false>
__device__ __forceinline__ void rfft_inv(const RegPlan &pl, typename RVec<R>::V *buf, int LG, const FastDiv &dLG,
                                         const typename cplx_t<R>::type *tw, bool gfirst, bool glast,
                                         const PhaseGlobal &gl, int pstart = -1) {
  // pstart: phases pstart, ..., 0 only (the default: all)
  for (int p = pstart >= 0 ? pstart : pl.np - 1; p >= 0; p--) {
    const bool gs = gfirst && p == pl.np - 1;
    rphase_any<true, R, WIDE>(pl, p, buf, LG, dLG, tw, gs, glast && p == 0, p < pl.np - 1, gl,
                              gs ? gl.rows_in : pl.n);
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Compile-time plans.  The phases of rphase / rfft_fwd / rfft_inv with the length,
// the radices and the line vectors of a tile known to the compiler: the block and
// stride arithmetic becomes multiplication by constants, the shared-memory offsets
// of a butterfly's points become immediates, no plan field is read at run time and
// the phase loop unrolls.  The arithmetic (the DFT codelets, the twiddles and their
// order) is that of the run-time engine, so the results are bit-identical.
constexpr int REG_THREADS = 256;  // threads of the CTAs that run the compile-time phases

template <int N_, int R0_, int R1_, int R2_ = 1> struct CtPlan {
  static constexpr int n = N_;
  static constexpr int np = R2_ > 1 ? 3 : (R1_ > 1 ? 2 : 1);
  __host__ __device__ static constexpr int rad(int p) { return p == 0 ? R0_ : p == 1 ? R1_ : R2_; }
  __host__ __device__ static constexpr int blk(int p) { return p == 0 ? N_ : p == 1 ? N_ / R0_ : N_ / (R0_ * R1_); }
  __host__ __device__ static constexpr int str(int p) { return blk(p) / rad(p); }
  __host__ __device__ static constexpr int twm(int p) { return N_ / blk(p); }
  static_assert(R0_ * R1_ * R2_ == N_, "the radices multiply to the length");
};

// the run-time plan `pl` is the compile-time plan P
template <typename P> __host__ __device__ inline bool ct_match(const RegPlan &pl) {
  if (pl.bl || pl.n != P::n || pl.np != P::np) return false;
  for (int p = 0; p < P::np; p++)
    if (pl.rad[p] != P::rad(p)) return false;
  return true;
}

// phase p of plan P over a tile of LG line vectors (rphase with constants)
template <typename P, int p, bool INV, typename R, int LG, bool GSRC, bool GDST>
__device__ __forceinline__ void rphase_ct(typename RVec<R>::V *buf, const typename cplx_t<R>::type *__restrict__ tw,
                                          const PhaseGlobal &gl, int nz) {
  typedef typename cplx_t<R>::type C;
  typedef typename RVec<R>::V V;
  constexpr int G = RVec<R>::G;
  constexpr int RAD = P::rad(p), s = P::str(p), B = P::blk(p), tm = P::twm(p);
  constexpr bool twid = p < P::np - 1;
  constexpr unsigned total = (unsigned)(P::n / RAD) * (unsigned)LG;
  static_assert(G == 1, "one complex point per vector");
  const V *gin = reinterpret_cast<const V *>(gl.in);
  V *gout = reinterpret_cast<V *>(gl.out);
  const long long vri = gl.rs_in, vro = gl.rs_out;
#pragma unroll 1
  for (unsigned u = threadIdx.x; u < total; u += REG_THREADS) {
    const unsigned b = u / (unsigned)LG;
    const int g = (int)(u - b * (unsigned)LG);
    const unsigned beta = b / (unsigned)s;
    const int r = (int)(b - beta * (unsigned)s);
    const int pos0 = (int)beta * B + r;
    C a[RAD];
    if constexpr (GSRC) {
      const V *src = gin + (long long)pos0 * vri + g;
#pragma unroll
      for (int j = 0; j < RAD; j++) {
        V v = zero_vec<R>();
        if (pos0 + s * j < nz) v = ldg_vec<R>(src + (long long)(s * j) * vri);
        a[j] = v;
      }
    } else {
      const V *src = buf + pos0 * LG + g;
      if (nz >= P::n) {
#pragma unroll
        for (int j = 0; j < RAD; j++) a[j] = src[s * j * LG];
      } else {
#pragma unroll
        for (int j = 0; j < RAD; j++) a[j] = pos0 + s * j < nz ? src[s * j * LG] : zero_vec<R>();
      }
    }
    if constexpr (INV && twid) {
      const int tb = tm * r;
#pragma unroll
      for (int j = 1; j < RAD; j++) a[j] = cmulc(a[j], tw[tb * j]);
    }
    dft<RAD, INV>(a);
    if constexpr (!INV && twid) {
      const int tb = tm * r;
#pragma unroll
      for (int k = 1; k < RAD; k++) a[k] = cmul(a[k], tw[tb * k]);
    }
    if constexpr (GDST) {
      V *dst = gout + (long long)pos0 * vro + g;
#pragma unroll
      for (int k = 0; k < RAD; k++)
        if (pos0 + s * k < gl.rows_out) dst[(long long)(s * k) * vro] = a[k];
    } else {
      V *dst = buf + pos0 * LG + g;
#pragma unroll
      for (int k = 0; k < RAD; k++) dst[s * k * LG] = a[k];
    }
  }
}

// forward phases p .. PEND - 1 of plan P (rfft_fwd); each ends with a barrier
template <typename P, typename R, int LG, bool GFIRST, bool GLAST, int PEND, int p = 0>
__device__ __forceinline__ void rfft_fwd_ct(typename RVec<R>::V *buf, const typename cplx_t<R>::type *tw,
                                            const PhaseGlobal &gl) {
  if constexpr (p < PEND) {
    const int nz = p == 0 ? gl.rows_in : P::n;  // phase 0: positions from rows_in on are zero
    rphase_ct<P, p, false, R, LG, GFIRST && p == 0, GLAST && p == P::np - 1>(buf, tw, gl, nz);
    __syncthreads();
    rfft_fwd_ct<P, R, LG, GFIRST, GLAST, PEND, p + 1>(buf, tw, gl);
  }
}

// inverse phases p = PSTART .. 0 of plan P (rfft_inv); each ends with a barrier
template <typename P, typename R, int LG, bool GFIRST, bool GLAST, int p>
__device__ __forceinline__ void rfft_inv_ct(typename RVec<R>::V *buf, const typename cplx_t<R>::type *tw,
                                            const PhaseGlobal &gl) {
  if constexpr (p >= 0) {
    constexpr bool gs = GFIRST && p == P::np - 1;
    rphase_ct<P, p, true, R, LG, gs, GLAST && p == 0>(buf, tw, gl, gs ? gl.rows_in : P::n);
    __syncthreads();
    rfft_inv_ct<P, R, LG, GFIRST, GLAST, p - 1>(buf, tw, gl);
  }
}

// ---------------------------------------------------------------------------
// Bluestein (chirp-z) transform of lines of length n with a plan of length m >= 2n-1:
//   X[k] = c[k] sum_j (x[j] c[j]) conj(c[k - j]),   c[j] = exp(-i pi j^2 / n),
// a circular convolution of length m: forward transform of the chirped input (zero
// beyond n), product with B = FFT_m(conj c wrapped), inverse transform, chirp.  The
// inverse DFT is conj(forward(conj x)).  `bpos` holds B at the plan's digit-reversed
// positions, so the product needs no reordering; the scale 1/m is folded into the
// output chirp.  Input and output are in natural order (first nin / nout points),
// read from global rows or buf, written to global rows or buf.
template <typename R>
__device__ __forceinline__ void bl_chirp_in(typename RVec<R>::V *buf, int L, const FastDiv &dL,
                                            const typename cplx_t<R>::type *__restrict__ chirp, int nin, bool conj_in,
                                            bool gsrc, const PhaseGlobal &gl) {
  typedef typename cplx_t<R>::type C;
  const C *gin = reinterpret_cast<const C *>(gl.in);
  const unsigned total = (unsigned)nin * (unsigned)L;
  for (unsigned t = threadIdx.x; t < total; t += blockDim.x) {
    const unsigned j = fdiv(t, dL);
    const int l = (int)(t - j * (unsigned)L);
    C v = gsrc ? ldg_vec<R>(gin + (long long)j * gl.rs_in + l) : buf[j * L + l];
    if (conj_in) v.y = -v.y;
    buf[j * L + l] = cmul(v, chirp[j]);
  }
}

template <typename R>
__device__ __forceinline__ void bl_mul(typename RVec<R>::V *buf, int L, const FastDiv &dL,
                                       const typename cplx_t<R>::type *__restrict__ bpos, int m) {
  const unsigned total = (unsigned)m * (unsigned)L;
  for (unsigned t = threadIdx.x; t < total; t += blockDim.x) {
    const unsigned q = fdiv(t, dL);
    buf[t] = cmul(buf[t], bpos[q]);
  }
}

template <typename R>
__device__ __forceinline__ void bl_chirp_out(typename RVec<R>::V *buf, int L, const FastDiv &dL,
                                             const typename cplx_t<R>::type *__restrict__ chirp, R scale, int nout,
                                             bool conj_out, bool gdst, const PhaseGlobal &gl) {
  typedef typename cplx_t<R>::type C;
  C *gout = reinterpret_cast<C *>(gl.out);
  const unsigned total = (unsigned)nout * (unsigned)L;
  for (unsigned t = threadIdx.x; t < total; t += blockDim.x) {
    const unsigned k = fdiv(t, dL);
    const int l = (int)(t - k * (unsigned)L);
    C v = cscale(cmul(buf[k * L + l], chirp[k]), scale);
    if (conj_out) v.y = -v.y;
    if (gdst) gout[(long long)k * gl.rs_out + l] = v;
    else buf[k * L + l] = v;
  }
}

// ends with a barrier
template <typename R, bool INV>
__device__ __forceinline__ void bfft(const RegPlan &pl, typename RVec<R>::V *buf, int L, const FastDiv &dL,
                                     const typename cplx_t<R>::type *tw, const typename cplx_t<R>::type *chirp,
                                     const typename cplx_t<R>::type *bpos, bool gsrc, bool gdst,
                                     const PhaseGlobal &gl, int nin, int nout) {
  bl_chirp_in<R>(buf, L, dL, chirp, nin, INV, gsrc, gl);
  __syncthreads();
  PhaseGlobal none = gl;
  none.rows_in = none.rows_out = pl.n;
  rfft_fwd<R>(pl, buf, L, dL, tw, false, false, none, nin);
  bl_mul<R>(buf, L, dL, bpos, pl.n);
  __syncthreads();
  rfft_inv<R>(pl, buf, L, dL, tw, false, false, none);
  bl_chirp_out<R>(buf, L, dL, chirp, R(1) / R(pl.n), nout, INV, gdst, gl);
  __syncthreads();
}

}  // namespace pmgpu
