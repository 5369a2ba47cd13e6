// fft.cuh -- batched mixed-radix Stockham FFT in shared memory.
//
// A CTA transforms L lines of length n held in shared memory with the lines
// interleaved (element (line l, index m) at buf[m * L + l]), so that a warp's
// threads, which take consecutive lines of the same butterfly, touch consecutive
// addresses in every pass.  Each pass does radix-R butterflies in registers
// (R = 2, 3, 4, 5, 7, 8, 11, 13, 16, 17 unrolled; any other prime through a
// generic O(R) per output path) and writes the self-sorting Stockham order into
// the other half of a ping-pong buffer pair.  Twiddles come from a table built on
// the host in long double and staged in shared memory by the caller.
//
// Forward transforms use exp(-2 pi i k m / n), inverse exp(+...), unnormalised,
// the conventions of source/fourier/pmlib_fourier_fft.f:382-384 and
// pmlib_fourier_ifft.f:401-403 in pmlib3d.
#pragma once

#include "common.cuh"

namespace pmgpu {

constexpr int FFT_MAXPASS = 12;

struct FftDesc {
  int n;                     // transform length
  int npass;
  int rad[FFT_MAXPASS];      // radix of each pass
  int ns[FFT_MAXPASS];       // product of the radices of the earlier passes
  int twoff[FFT_MAXPASS];    // offset of the pass twiddles exp(-2 pi i k r / (ns R))
  int rootoff[FFT_MAXPASS];  // generic passes: offset of exp(-2 pi i q / R), q < R
  int ntw;                   // table entries used by the passes
  int extoff;                // offset of an extra caller table (R2C twiddles), or -1
  int next;                  // entries of the extra table
};

// (cos, sin)(2 pi m / R) for R <= 32 (prime radices and the composite radices'
// internal twiddles), m < R; every translation unit that runs the transforms holds
// its own copy, filled once per device by the host
constexpr int CS_R = 33, CS_M = 32;
static __constant__ float c_cs32[CS_R][CS_M][2];
static __constant__ double c_cs64[CS_R][CS_M][2];

template <typename T> __device__ __forceinline__ T cs_c(int R, int m);
template <typename T> __device__ __forceinline__ T cs_s(int R, int m);
template <> __device__ __forceinline__ float cs_c<float>(int R, int m) { return c_cs32[R][m][0]; }
template <> __device__ __forceinline__ float cs_s<float>(int R, int m) { return c_cs32[R][m][1]; }
template <> __device__ __forceinline__ double cs_c<double>(int R, int m) { return c_cs64[R][m][0]; }
template <> __device__ __forceinline__ double cs_s<double>(int R, int m) { return c_cs64[R][m][1]; }

template <int R, bool INV, typename C> __device__ __forceinline__ void dft(C *v);

template <bool INV, typename C> __device__ __forceinline__ void dft2(C *v) {
  C a = v[0], b = v[1];
  v[0] = cadd(a, b);
  v[1] = csub(a, b);
}

template <bool INV, typename C> __device__ __forceinline__ void dft4(C *v) {
  C t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
  C t2 = cadd(v[1], v[3]), t3 = csub(v[1], v[3]);
  v[0] = cadd(t0, t2);
  v[2] = csub(t0, t2);
  // forward: X1 = t1 - i t3, X3 = t1 + i t3
  C it3 = mk(-t3.y, t3.x);  // i * t3
  if (!INV) {
    v[1] = csub(t1, it3);
    v[3] = cadd(t1, it3);
  } else {
    v[1] = cadd(t1, it3);
    v[3] = csub(t1, it3);
  }
}

// odd prime R: pairs (n, R-n) share cos terms and antisymmetric sin terms; the
// outputs overwrite v once the sums s_n = v_n + v_{R-n}, d_n = v_n - v_{R-n} exist
template <int R, bool INV, typename C> __device__ __forceinline__ void dft_prime(C *v) {
  typedef typename real_of<C>::type T;
  constexpr int h = (R - 1) / 2;
  C s[h + 1], d[h + 1];
  const C x0 = v[0];
  C sum = x0;
#pragma unroll
  for (int n = 1; n <= h; n++) {
    s[n] = cadd(v[n], v[R - n]);
    d[n] = csub(v[n], v[R - n]);
    sum = cadd(sum, s[n]);
  }
  v[0] = sum;
#pragma unroll
  for (int k = 1; k <= h; k++) {
    C a = x0;
    C b = mk(T(0), T(0));
#pragma unroll
    for (int n = 1; n <= h; n++) {
      const int m = (n * k) % R;
      const T c = cs_c<T>(R, m), sn = cs_s<T>(R, m);
      a = cfma_r(s[n], c, a);
      b = cfma_r(d[n], sn, b);
    }
    if (!INV) {
      v[k] = mk(a.x + b.y, a.y - b.x);
      v[R - k] = mk(a.x - b.y, a.y + b.x);
    } else {
      v[k] = mk(a.x - b.y, a.y + b.x);
      v[R - k] = mk(a.x + b.y, a.y - b.x);
    }
  }
}

// N = R1 * R2 in registers: n = R2 n1 + n2, k = k1 + R1 k2
template <int R1, int R2, bool INV, typename C> __device__ __forceinline__ void dft_comp(C *v) {
  typedef typename real_of<C>::type T;
  constexpr int N = R1 * R2;
  C y[N];
#pragma unroll
  for (int n2 = 0; n2 < R2; n2++) {
    C t[R1];
#pragma unroll
    for (int n1 = 0; n1 < R1; n1++) t[n1] = v[R2 * n1 + n2];
    dft<R1, INV>(t);
#pragma unroll
    for (int k1 = 0; k1 < R1; k1++) y[n2 * R1 + k1] = t[k1];
  }
#pragma unroll
  for (int n2 = 1; n2 < R2; n2++)
#pragma unroll
    for (int k1 = 1; k1 < R1; k1++) {
      const int m = (n2 * k1) % N;
      const T c = cs_c<T>(N, m), s = cs_s<T>(N, m);
      C a = y[n2 * R1 + k1];
      y[n2 * R1 + k1] = INV ? mk(a.x * c - a.y * s, a.y * c + a.x * s)
                            : mk(a.x * c + a.y * s, a.y * c - a.x * s);
    }
#pragma unroll
  for (int k1 = 0; k1 < R1; k1++) {
    C t[R2];
#pragma unroll
    for (int n2 = 0; n2 < R2; n2++) t[n2] = y[n2 * R1 + k1];
    dft<R2, INV>(t);
#pragma unroll
    for (int k2 = 0; k2 < R2; k2++) v[k1 + R1 * k2] = t[k2];
  }
}

template <int R, bool INV, typename C> __device__ __forceinline__ void dft(C *v) {
  if constexpr (R == 1) {
  } else if constexpr (R == 2) {
    dft2<INV>(v);
  } else if constexpr (R == 4) {
    dft4<INV>(v);
  } else if constexpr (R == 6) {
    dft_comp<3, 2, INV>(v);
  } else if constexpr (R == 8) {
    dft_comp<4, 2, INV>(v);
  } else if constexpr (R == 9) {
    dft_comp<3, 3, INV>(v);
  } else if constexpr (R == 10) {
    dft_comp<5, 2, INV>(v);
  } else if constexpr (R == 12) {
    dft_comp<4, 3, INV>(v);
  } else if constexpr (R == 16) {
    dft_comp<4, 4, INV>(v);
  } else if constexpr (R == 18) {
    dft_comp<6, 3, INV>(v);
  } else if constexpr (R == 20) {
    dft_comp<5, 4, INV>(v);
  } else if constexpr (R == 22) {
    dft_comp<11, 2, INV>(v);
  } else if constexpr (R == 24) {
    dft_comp<8, 3, INV>(v);
  } else if constexpr (R == 26) {
    dft_comp<13, 2, INV>(v);
  } else if constexpr (R == 32) {
    dft_comp<8, 4, INV>(v);
  } else {
    dft_prime<R, INV>(v);
  }
}

// ---------------------------------------------------------------------------
// Vectorised passes.  Shared-memory buffers hold LG vectors per transform index,
// a vector being G consecutive lines (FP32: float4 = two complex lines, FP64:
// double2 = one).  A thread owns one line group g and the butterflies j = jt,
// jt + JS, ...; the twiddle index k = j mod ns and j - k advance incrementally, so
// the passes contain no integer division.
template <typename R> struct Vec;
template <> struct Vec<float> {
  typedef float4 V;
  static constexpr int G = 2;
};
template <> struct Vec<double> {
  typedef double2 V;
  static constexpr int G = 1;
};

__device__ __forceinline__ void vsplit(const float4 &v, float2 *a) {
  a[0] = make_float2(v.x, v.y);
  a[1] = make_float2(v.z, v.w);
}
__device__ __forceinline__ void vsplit(const double2 &v, double2 *a) { a[0] = v; }
__device__ __forceinline__ float4 vmerge(const float2 *a) { return make_float4(a[0].x, a[0].y, a[1].x, a[1].y); }
__device__ __forceinline__ double2 vmerge(const double2 *a) { return a[0]; }

struct LineMap {
  int jt;  // first butterfly of this thread
  int JS;  // butterfly stride (threads per line group)
  int g;   // line group, -1 for an idle thread
};

__device__ __forceinline__ LineMap line_map(int LG) {
  LineMap m;
  m.JS = blockDim.x / LG;
  m.jt = threadIdx.x / LG;
  m.g = threadIdx.x - m.jt * LG;
  if (m.jt >= m.JS) m.g = -1;
  return m;
}

template <int RAD, bool INV, typename R>
__device__ __forceinline__ void vpass(const typename Vec<R>::V *__restrict__ src, typename Vec<R>::V *__restrict__ dst,
                                      int LG, int n, int ns, const typename cplx_t<R>::type *__restrict__ tw,
                                      const LineMap &lm) {
  typedef typename cplx_t<R>::type C;
  typedef typename Vec<R>::V V;
  constexpr int G = Vec<R>::G;
  if (lm.g < 0) return;
  const int nr = n / RAD;
  int j = lm.jt;
  int k = j % ns;
  int jmk = j - k;
  const int JSm = lm.JS % ns;
  const int JSq = lm.JS - JSm;
  while (j < nr) {
    C a[G][RAD];
#pragma unroll
    for (int r = 0; r < RAD; r++) {
      C t[G];
      vsplit(src[(j + r * nr) * LG + lm.g], t);
#pragma unroll
      for (int h = 0; h < G; h++) a[h][r] = t[h];
    }
    if (k != 0) {
      const C *w = tw + k * (RAD - 1) - 1;
#pragma unroll
      for (int r = 1; r < RAD; r++) {
        const C ww = w[r];
#pragma unroll
        for (int h = 0; h < G; h++) a[h][r] = INV ? cmulc(a[h][r], ww) : cmul(a[h][r], ww);
      }
    }
#pragma unroll
    for (int h = 0; h < G; h++) dft<RAD, INV>(a[h]);
    const int base = jmk * RAD + k;
#pragma unroll
    for (int r = 0; r < RAD; r++) {
      C t[G];
#pragma unroll
      for (int h = 0; h < G; h++) t[h] = a[h][r];
      dst[(base + r * ns) * LG + lm.g] = vmerge(t);
    }
    j += lm.JS;
    k += JSm;
    jmk += JSq;
    if (k >= ns) {
      k -= ns;
      jmk += ns;
    }
  }
}

// generic radix (primes without an unrolled kernel): O(RAD^2) per butterfly
template <bool INV, typename R>
__device__ __forceinline__ void vpass_generic(const typename Vec<R>::V *__restrict__ src,
                                              typename Vec<R>::V *__restrict__ dst, int LG, int n, int ns,
                                              int RAD, const typename cplx_t<R>::type *__restrict__ tw,
                                              const typename cplx_t<R>::type *__restrict__ roots,
                                              const LineMap &lm) {
  typedef typename cplx_t<R>::type C;
  constexpr int G = Vec<R>::G;
  if (lm.g < 0) return;
  const int nr = n / RAD;
  for (int j = lm.jt; j < nr; j += lm.JS) {
    const int k = j % ns;
    const int base = (j - k) * RAD + k;
    for (int m = 0; m < RAD; m++) {
      C acc[G];
#pragma unroll
      for (int h = 0; h < G; h++) acc[h] = mk(R(0), R(0));
      for (int r = 0; r < RAD; r++) {
        C t[G];
        vsplit(src[(j + r * nr) * LG + lm.g], t);
        C w2 = roots[(r * m) % RAD];
        if (k != 0 && r > 0) {
          const C w = tw[k * (RAD - 1) + r - 1];
          w2 = cmul(w2, w);
        }
#pragma unroll
        for (int h = 0; h < G; h++) acc[h] = cadd(acc[h], INV ? cmulc(t[h], w2) : cmul(t[h], w2));
      }
      dst[(base + m * ns) * LG + lm.g] = vmerge(acc);
    }
  }
}

// Transforms the lines in buffer a (partner b); returns the buffer with the result.
// The caller synchronises before (data staged); every pass ends with a barrier.
template <bool INV, typename R>
__device__ __forceinline__ typename Vec<R>::V *vfft(typename Vec<R>::V *a, typename Vec<R>::V *b, int LG,
                                                    const FftDesc &d, const typename cplx_t<R>::type *__restrict__ tw,
                                                    const LineMap &lm) {
  typedef typename Vec<R>::V V;
  const int np = d.npass, n = d.n;
  for (int p = 0; p < np; p++) {
    const typename cplx_t<R>::type *t = tw + d.twoff[p];
    const int ns = d.ns[p];
    switch (d.rad[p]) {
      case 2: vpass<2, INV, R>(a, b, LG, n, ns, t, lm); break;
      case 3: vpass<3, INV, R>(a, b, LG, n, ns, t, lm); break;
      case 4: vpass<4, INV, R>(a, b, LG, n, ns, t, lm); break;
      case 5: vpass<5, INV, R>(a, b, LG, n, ns, t, lm); break;
      case 7: vpass<7, INV, R>(a, b, LG, n, ns, t, lm); break;
      case 8: vpass<8, INV, R>(a, b, LG, n, ns, t, lm); break;
      case 11: vpass<11, INV, R>(a, b, LG, n, ns, t, lm); break;
      case 13: vpass<13, INV, R>(a, b, LG, n, ns, t, lm); break;
      case 16: vpass<16, INV, R>(a, b, LG, n, ns, t, lm); break;
      case 17: vpass<17, INV, R>(a, b, LG, n, ns, t, lm); break;
      default: vpass_generic<INV, R>(a, b, LG, n, ns, d.rad[p], t, tw + d.rootoff[p], lm); break;
    }
    __syncthreads();
    V *s = a;
    a = b;
    b = s;
  }
  return a;
}

// ---------------------------------------------------------------------------
// asynchronous global -> shared copies (sm_80+ cp.async; completion is waited for
// with cp.async.wait_group, no spinning)
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async4(void *smem, const void *gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// copy a table from global to shared memory (caller synchronises)
template <typename C>
__device__ __forceinline__ void stage_table(C *dst, const C *__restrict__ src, int n) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = src[i];
}

}  // namespace pmgpu
