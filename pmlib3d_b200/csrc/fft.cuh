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

// (cos, sin)(2 pi m / R) for R <= 17, m < R; filled once per device by the host
// (the library is a single translation unit, so these are defined here)
__constant__ float c_cs32[18][17][2];
__constant__ double c_cs64[18][17][2];

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
      a = mk(a.x + s[n].x * c, a.y + s[n].y * c);
      b = mk(b.x + d[n].x * sn, b.y + d[n].y * sn);
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
  } else if constexpr (R == 8) {
    dft_comp<4, 2, INV>(v);
  } else if constexpr (R == 16) {
    dft_comp<4, 4, INV>(v);
  } else {
    dft_prime<R, INV>(v);
  }
}

// one Stockham pass of radix R over L interleaved lines
template <int R, bool INV, typename C>
__device__ __noinline__ void stockham_pass(const C *__restrict__ src, C *__restrict__ dst, int L,
                                              int n, int ns, const C *__restrict__ tw) {
  const int nr = n / R;
  const int total = L * nr;
  for (int t = threadIdx.x; t < total; t += blockDim.x) {
    const int j = t / L;
    const int l = t - j * L;
    const int k = j % ns;
    C v[R];
#pragma unroll
    for (int r = 0; r < R; r++) v[r] = src[(j + r * nr) * L + l];
    if (ns > 1) {
      const C *w = tw + k * (R - 1) - 1;
#pragma unroll
      for (int r = 1; r < R; r++) v[r] = INV ? cmulc(v[r], w[r]) : cmul(v[r], w[r]);
    }
    dft<R, INV>(v);
    const int base = (j - k) * R + k;
#pragma unroll
    for (int r = 0; r < R; r++) dst[(base + r * ns) * L + l] = v[r];
  }
}

// generic radix: one output per work item, O(R) terms each
template <bool INV, typename C>
__device__ __noinline__ void stockham_generic(const C *__restrict__ src, C *__restrict__ dst,
                                                 int L, int n, int ns, int R,
                                                 const C *__restrict__ tw,
                                                 const C *__restrict__ roots) {
  const int nr = n / R;
  const int total = L * n;
  for (int t = threadIdx.x; t < total; t += blockDim.x) {
    const int q = t / L;
    const int l = t - q * L;
    const int m = q / nr;       // output within the butterfly
    const int j = q - m * nr;   // butterfly
    const int k = j % ns;
    C acc = mk((typename real_of<C>::type)0, (typename real_of<C>::type)0);
    for (int r = 0; r < R; r++) {
      C v = src[(j + r * nr) * L + l];
      if (ns > 1 && r > 0) {
        C w = tw[k * (R - 1) + r - 1];
        v = INV ? cmulc(v, w) : cmul(v, w);
      }
      C w2 = roots[(r * m) % R];
      acc = cadd(acc, INV ? cmulc(v, w2) : cmul(v, w2));
    }
    dst[((j - k) * R + k + m * ns) * L + l] = acc;
  }
}

// Transforms the L lines in buffer a (ping-pong partner b); returns the buffer
// holding the result.  The radix passes are separate (non-inlined) functions so
// every kernel shares one compiled copy per precision and direction.  Caller
// synchronises before (data staged) and after.
template <bool INV, typename C>
__device__ __noinline__ C *fft_batch(C *a, C *b, int L, const FftDesc &d, const C *__restrict__ tw) {
  const int np = d.npass, n = d.n;
  for (int p = 0; p < np; p++) {
    const C *t = tw + d.twoff[p];
    const int ns = d.ns[p];
    switch (d.rad[p]) {
      case 2: stockham_pass<2, INV>(a, b, L, n, ns, t); break;
      case 3: stockham_pass<3, INV>(a, b, L, n, ns, t); break;
      case 4: stockham_pass<4, INV>(a, b, L, n, ns, t); break;
      case 5: stockham_pass<5, INV>(a, b, L, n, ns, t); break;
      case 7: stockham_pass<7, INV>(a, b, L, n, ns, t); break;
      case 8: stockham_pass<8, INV>(a, b, L, n, ns, t); break;
      case 11: stockham_pass<11, INV>(a, b, L, n, ns, t); break;
      case 13: stockham_pass<13, INV>(a, b, L, n, ns, t); break;
      case 16: stockham_pass<16, INV>(a, b, L, n, ns, t); break;
      case 17: stockham_pass<17, INV>(a, b, L, n, ns, t); break;
      default:
        stockham_generic<INV>(a, b, L, n, ns, d.rad[p], t, tw + d.rootoff[p]);
        break;
    }
    __syncthreads();
    C *s = a;
    a = b;
    b = s;
  }
  return a;
}

// copy a table from global to shared memory (caller synchronises)
template <typename C>
__device__ __forceinline__ void stage_table(C *dst, const C *__restrict__ src, int n) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = src[i];
}

}  // namespace pmgpu
