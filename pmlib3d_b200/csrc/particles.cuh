// particles.cuh -- particle binning, stable sort, deterministic M4'/M6* deposition
// (P2M), mesh-to-particle interpolation (M2P) and remesh.
//
// P2M (source/interpolation/pmlib_interp_particle_mesh.f) scatters every particle
// into its 4^3 (M4') or 6^3 (M6*) stencil with the particle loop in index order.
// Here particles are binned by the reference's base cell NINT((x - xmin) / dx)
// (:153-155, bit-exact index arithmetic), sorted stably by bin (ties keep particle
// order), and every cell then gathers the contributions of the
// bins whose stencil covers it, in a fixed order: no floating-point atomics, and
// the same result on every run.  The stable order comes from a counting sort: slots
// within a bin are taken by integer atomics and then put back in particle order.
#pragma once

#include "common.cuh"
#include "fft.cuh"  // cp.async helpers

namespace pmgpu {

// ------------------------------------------------------------------ geometry
template <typename R> struct PartGeom {
  int ext[3];     // cuboid extents including ghosts
  int lo[3];      // 1-based index of the first cuboid point (1 - nghost_lo)
  int nint[3];    // interior cells
  int nglo[3];    // ghosts on the low face
  int bclo[3], bchi[3];  // face types (0 free, 1 periodic)
  int blo[3];     // base index of bin 0 along each axis
  int nb[3];      // bins per axis
  unsigned nbins; // nb0 nb1 nb2 (the sentinel key of skipped particles)
  R xmin[3], xmax[3], dx[3], c1dx[3];
};

template <int W> struct Stencil;
template <> struct Stencil<4> { static constexpr int off = 1; };  // base-1 .. base+2
template <> struct Stencil<6> { static constexpr int off = 2; };  // base-2 .. base+3

// NINT((x - xmin) * (1/dx)): the product is not contracted and rounding is half
// away from zero, as Fortran NINT.
__device__ __forceinline__ long long base_index(double x, double xmin, double c1dx) {
  const double t = __dmul_rn(__dsub_rn(x, xmin), c1dx);
  if (!(fabs(t) < 1.0e15)) return (long long)-4611686018427387904LL;
  return (long long)round(t);
}
__device__ __forceinline__ long long base_index(float x, float xmin, float c1dx) {
  const float t = __fmul_rn(__fsub_rn(x, xmin), c1dx);
  if (!(fabsf(t) < 1.0e9f)) return (long long)-4611686018427387904LL;
  return (long long)roundf(t);
}

// M4' weights at offsets d+1, d, 1-d, 2-d (interp_particle_mesh.f:201-214)
template <typename R> __device__ __forceinline__ void weights_m4(R d2, R *a) {
  const R d1 = d2 + R(1), d3 = R(1) - d2, d4 = R(2) - d2;
  const R t1 = R(2) - d1, t4 = R(2) - d4;
  a[0] = R(0.5) * (t1 * t1) * (R(1) - d1);
  a[1] = R(1) - R(2.5) * (d2 * d2) + R(1.5) * (d2 * d2 * d2);
  a[2] = R(1) - R(2.5) * (d3 * d3) + R(1.5) * (d3 * d3 * d3);
  a[3] = R(0.5) * (t4 * t4) * (R(1) - d4);
}
// M6* weights (interp_particle_mesh.f:564-602)
template <typename R> __device__ __forceinline__ void weights_m6(R d3, R *a) {
  const R c1 = R(-1) / R(24), c2 = R(1) / R(24), c3 = R(-1) / R(12);
  const R d1 = d3 + R(2), d2 = d3 + R(1), d4 = R(1) - d3, d5 = R(2) - d3, d6 = R(3) - d3;
  R u;
  u = d1 - R(3);
  a[0] = c1 * (d1 - R(2)) * (u * u * u) * (R(5) * d1 - R(8));
  a[1] = c2 * (d2 - R(1)) * (d2 - R(2)) * (R(25) * (d2 * d2 * d2) - R(114) * (d2 * d2) + R(153) * d2 - R(48));
  a[2] = c3 * (d3 - R(1)) * (R(25) * (d3 * d3 * d3 * d3) - R(38) * (d3 * d3 * d3) - R(3) * (d3 * d3) + R(12) * d3 + R(12));
  a[3] = c3 * (d4 - R(1)) * (R(25) * (d4 * d4 * d4 * d4) - R(38) * (d4 * d4 * d4) - R(3) * (d4 * d4) + R(12) * d4 + R(12));
  a[4] = c2 * (d5 - R(1)) * (d5 - R(2)) * (R(25) * (d5 * d5 * d5) - R(114) * (d5 * d5) + R(153) * d5 - R(48));
  u = d6 - R(3);
  a[5] = c1 * (d6 - R(2)) * (u * u * u) * (R(5) * d6 - R(8));
}
template <typename R, int W> __device__ __forceinline__ void weights(R d, R *a) {
  if constexpr (W == 4) weights_m4<R>(d, a); else weights_m6<R>(d, a);
}

// normalised offset of x from its base cell centre
template <typename R>
__device__ __forceinline__ R cell_offset(R x, R xmin, R dx, long long b, R scale) {
  return (x - xmin - dx * ((R)b - R(0.5))) * scale;
}

// ------------------------------------------------------------------ binning
// key = flattened base cell in the bin box; particles whose stencil misses the
// cuboid, or which lie outside [xmin, xmax] across a periodic face (all weights
// zeroed, :229-246), get the sentinel key nbins and are skipped by P2M (they still
// take a slot, so the sorted order is a permutation of all particles).
// rank = the particle's provisional slot within its bin (one atomic per particle; the
// order within a bin is put right by the stable fix-up).
template <typename R, int W>
__global__ void k_bin(PartGeom<R> g, const R *__restrict__ pos, int n, unsigned *__restrict__ key,
                      unsigned *__restrict__ rank, unsigned *__restrict__ counts) {
  constexpr int off = Stencil<W>::off;
  const int stride = gridDim.x * blockDim.x;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += stride) {
    bool ok = true;
    long long bi[3];
#pragma unroll
    for (int e = 0; e < 3; e++) {
      const R x = pos[(size_t)3 * p + e];
      const long long b = base_index(x, g.xmin[e], g.c1dx[e]);
      const long long first = b - off, last = b - off + W - 1;
      const int hi = g.lo[e] + g.ext[e] - 1;
      if (!(last >= g.lo[e] && first <= hi)) ok = false;
      if (g.bclo[e] != 0 && x < g.xmin[e]) ok = false;
      if (g.bchi[e] != 0 && x > g.xmax[e]) ok = false;
      bi[e] = b - g.blo[e];
    }
    unsigned k = g.nbins;
    if (ok) k = (unsigned)(bi[0] + (long long)g.nb[0] * (bi[1] + (long long)g.nb[1] * bi[2]));
    key[p] = k;
    rank[p] = atomicAdd(&counts[k], 1u);
  }
}

// order[start[key] + rank] = p
__global__ void k_place(const unsigned *__restrict__ key, const unsigned *__restrict__ rank, int n,
                        const unsigned *__restrict__ start, int *__restrict__ order) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x)
    order[start[key[p]] + rank[p]] = p;
}

// Slots within a bin were taken in atomic order; restore ascending particle index
// so the sorted order is the stable one.  Bins of up to FIX_SMALL particles are
// sorted in place by one thread; larger bins go to an overflow list (ovf[0] =
// count, ovf[1..] = bins) for k_fixup_big.  The sentinel bin is not needed in order.
constexpr int FIX_SMALL = 32;
// one bin [s, e) of the stable fix-up; bins of up to eight ids are sorted in
// registers (all loads in flight together), larger ones in place
__device__ __forceinline__ void fixup_bin(unsigned b, unsigned s, unsigned e, int *__restrict__ order,
                                          unsigned *__restrict__ ovf) {
  const unsigned k = e - s;
  if (k < 2) return;
  if (k > (unsigned)FIX_SMALL) {
    const unsigned i = atomicAdd(&ovf[0], 1u);
    ovf[1 + i] = b;
    return;
  }
  int *o = order + s;
  if (k <= 8) {
    int v[8];
#pragma unroll
    for (int i = 0; i < 8; i++) v[i] = (unsigned)i < k ? o[i] : 0x7fffffff;
#pragma unroll
    for (int i = 1; i < 8; i++)
#pragma unroll
      for (int j = i; j > 0; j--) {
        const int a = v[j - 1], c = v[j];
        v[j - 1] = min(a, c);
        v[j] = max(a, c);
      }
#pragma unroll
    for (int i = 0; i < 8; i++)
      if ((unsigned)i < k) o[i] = v[i];
    return;
  }
  for (unsigned i = 1; i < k; i++) {
    const int v = o[i];
    unsigned j = i;
    while (j > 0 && o[j - 1] > v) {
      o[j] = o[j - 1];
      j--;
    }
    o[j] = v;
  }
}
// a thread takes four consecutive bins (one 16-byte load of their starts and the
// next bin's start)
__global__ void k_fixup_small(const unsigned *__restrict__ start, unsigned nbins, int *__restrict__ order,
                              unsigned *__restrict__ ovf) {
  const unsigned ngroups = (nbins + 3) / 4;
  for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < ngroups; t += gridDim.x * blockDim.x) {
    const unsigned b0 = 4 * t;
    if (b0 + 4 <= nbins) {
      const uint4 v = *reinterpret_cast<const uint4 *>(start + b0);
      const unsigned e3 = start[b0 + 4];
      fixup_bin(b0, v.x, v.y, order, ovf);
      fixup_bin(b0 + 1, v.y, v.z, order, ovf);
      fixup_bin(b0 + 2, v.z, v.w, order, ovf);
      fixup_bin(b0 + 3, v.w, e3, order, ovf);
    } else {
      for (unsigned b = b0; b < nbins; b++) fixup_bin(b, start[b], start[b + 1], order, ovf);
    }
  }
}

// One CTA sorts one overflow bin at a time: runs of FIX_CHUNK ids by a bitonic sort
// in shared memory, then merge-path merges of doubling runs through `tmp` (same
// offsets as `order`).  Ids in a bin are distinct, so the order is unique.
constexpr int FIX_THREADS = 1024;
constexpr int FIX_CHUNK = 4096;
__global__ void __launch_bounds__(FIX_THREADS) k_fixup_big(const unsigned *__restrict__ start,
                                                           const unsigned *__restrict__ ovf, int *__restrict__ order,
                                                           int *__restrict__ tmp) {
  __shared__ int sh[FIX_CHUNK];
  const unsigned nov = ovf[0];
  for (unsigned ib = blockIdx.x; ib < nov; ib += gridDim.x) {
    const unsigned b = ovf[1 + ib];
    const unsigned s = start[b];
    const int k = (int)(start[b + 1] - s);
    // 1. sort chunks in shared memory
    for (int c0 = 0; c0 < k; c0 += FIX_CHUNK) {
      const int m = min(FIX_CHUNK, k - c0);
      int P = 1;
      while (P < m) P <<= 1;
      for (int i = threadIdx.x; i < P; i += blockDim.x) sh[i] = i < m ? order[s + c0 + i] : 0x7FFFFFFF;
      __syncthreads();
      for (int sz = 2; sz <= P; sz <<= 1)
        for (int st = sz >> 1; st > 0; st >>= 1) {
          for (int i = threadIdx.x; i < P; i += blockDim.x) {
            const int j = i ^ st;
            if (j > i) {
              const bool up = (i & sz) == 0;
              const int a = sh[i], c = sh[j];
              if ((a > c) == up) {
                sh[i] = c;
                sh[j] = a;
              }
            }
          }
          __syncthreads();
        }
      for (int i = threadIdx.x; i < m; i += blockDim.x) order[s + c0 + i] = sh[i];
      __syncthreads();
    }
    // 2. merge runs of width w into 2w, ping-pong between order and tmp
    int *src = order + s, *dst = tmp + s;
    for (int w = FIX_CHUNK; w < k; w <<= 1) {
      for (int a0 = 0; a0 < k; a0 += 2 * w) {
        const int na = min(w, k - a0), nb = max(0, min(w, k - a0 - w));
        const int *A = src + a0, *B = src + a0 + na;
        const int m = na + nb;
        const int per = (m + blockDim.x - 1) / blockDim.x;
        const int d0 = min(m, (int)threadIdx.x * per), d1 = min(m, d0 + per);
        if (d0 < d1) {
          // merge path: i elements from A and d0 - i from B precede diagonal d0
          int lo = max(0, d0 - nb), hi = min(d0, na);
          while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (A[mid] < B[d0 - mid - 1]) lo = mid + 1;
            else hi = mid;
          }
          int i = lo, j = d0 - lo;
          for (int d = d0; d < d1; d++) {
            if (j >= nb || (i < na && A[i] < B[j])) dst[a0 + d] = A[i++];
            else dst[a0 + d] = B[j++];
          }
        }
      }
      __syncthreads();
      int *t = src;
      src = dst;
      dst = t;
    }
    if (src != order + s)
      for (int i = threadIdx.x; i < k; i += blockDim.x) order[s + i] = src[i];
    __syncthreads();
  }
}

// ------------------------------------------------------------------ scans (exclusive, u32)
constexpr int SCAN_THREADS = 1024;
constexpr int SCAN_PER_THREAD = 16;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_PER_THREAD;

__device__ __forceinline__ unsigned block_exclusive_scan(unsigned v, unsigned *warp_sums, unsigned *total) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  unsigned x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    unsigned y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_sums[wid] = x;
  __syncthreads();
  if (wid == 0) {
    const int nw = blockDim.x >> 5;
    unsigned s = lane < nw ? warp_sums[lane] : 0u;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      unsigned y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    if (lane < nw) warp_sums[lane] = s;
    if (lane == nw - 1) *total = s;
  }
  __syncthreads();
  const unsigned before = wid > 0 ? warp_sums[wid - 1] : 0u;
  const unsigned r = before + x - v;
  __syncthreads();
  return r;
}

// a thread's SCAN_PER_THREAD consecutive values (16-byte loads inside the array; the
// arrays scanned here start on 16-byte boundaries)
static_assert(SCAN_PER_THREAD % 4 == 0, "scan loads are 16-byte vectors");
__device__ __forceinline__ void scan_load(const unsigned *__restrict__ in, size_t n, size_t base, unsigned *v) {
  if (base + SCAN_PER_THREAD <= n) {
#pragma unroll
    for (int i = 0; i < SCAN_PER_THREAD; i += 4) {
      const uint4 q = *reinterpret_cast<const uint4 *>(in + base + i);
      v[i] = q.x; v[i + 1] = q.y; v[i + 2] = q.z; v[i + 3] = q.w;
    }
  } else {
#pragma unroll
    for (int i = 0; i < SCAN_PER_THREAD; i++) v[i] = (base + i < n) ? in[base + i] : 0u;
  }
}

__global__ void __launch_bounds__(SCAN_THREADS) k_scan_reduce(const unsigned *__restrict__ in, size_t n,
                                                              unsigned *__restrict__ part) {
  __shared__ unsigned ws[32];
  __shared__ unsigned tot;
  const size_t base = (size_t)blockIdx.x * SCAN_TILE + (size_t)threadIdx.x * SCAN_PER_THREAD;
  unsigned v[SCAN_PER_THREAD];
  scan_load(in, n, base, v);
  unsigned s = 0;
#pragma unroll
  for (int i = 0; i < SCAN_PER_THREAD; i++) s += v[i];
  block_exclusive_scan(s, ws, &tot);
  if (threadIdx.x == 0) part[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(SCAN_THREADS) k_scan_partials(unsigned *__restrict__ part, int np) {
  __shared__ unsigned ws[32];
  __shared__ unsigned tot;
  const int per = (np + blockDim.x - 1) / blockDim.x;
  const int b = threadIdx.x * per;
  unsigned s = 0;
  for (int i = 0; i < per; i++)
    if (b + i < np) s += part[b + i];
  unsigned off = block_exclusive_scan(s, ws, &tot);
  for (int i = 0; i < per; i++)
    if (b + i < np) {
      const unsigned v = part[b + i];
      part[b + i] = off;
      off += v;
    }
}

__global__ void __launch_bounds__(SCAN_THREADS) k_scan_apply(const unsigned *__restrict__ in, size_t n,
                                                             const unsigned *__restrict__ part,
                                                             unsigned *__restrict__ out) {
  __shared__ unsigned ws[32];
  __shared__ unsigned tot;
  const size_t base = (size_t)blockIdx.x * SCAN_TILE + (size_t)threadIdx.x * SCAN_PER_THREAD;
  unsigned v[SCAN_PER_THREAD];
  scan_load(in, n, base, v);
  unsigned s = 0;
#pragma unroll
  for (int i = 0; i < SCAN_PER_THREAD; i++) s += v[i];
  unsigned off = block_exclusive_scan(s, ws, &tot) + part[blockIdx.x];
  unsigned o[SCAN_PER_THREAD];
#pragma unroll
  for (int i = 0; i < SCAN_PER_THREAD; i++) {
    o[i] = off;
    off += v[i];
  }
  if (base + SCAN_PER_THREAD <= n) {
#pragma unroll
    for (int i = 0; i < SCAN_PER_THREAD; i += 4)
      *reinterpret_cast<uint4 *>(out + base + i) = make_uint4(o[i], o[i + 1], o[i + 2], o[i + 3]);
  } else {
#pragma unroll
    for (int i = 0; i < SCAN_PER_THREAD; i++)
      if (base + i < n) out[base + i] = o[i];
  }
}

// ------------------------------------------------------------------ deposition (gather)
// Every cell gathers the particles of the W x W x W bins that reach it, so no
// floating-point atomics are needed and the sum order per cell is fixed (bin layer,
// bin row, bin, particle index): the same result on every run.
//
// Work split.  The cuboid is cut into tiles of TW x TH cell columns of equal size
// (TW <= 32, TH <= CY); all (tile, cell layer) pairs, tile by tile and layer by
// layer, are divided into consecutive shares of equal cost, one per CTA (a persistent grid of one CTA per SM).  A
// CTA's share is one or a few segments: a tile and a range of cell layers.  For a
// segment the CTA marches up the bin layers that reach its cell layers.
//
// Roles.  A CTA has NCW consumer warps and two groups of NPG producer warps.  The
// producers stage one bin layer at a time in shared memory: the bin starts of the
// (32+W-1) x (CY+W-1) bins of the layer that reach the tile, and for each of their
// particles a record (values, bin x), its z weights, x weights and zero-padded y
// weights.  The consumers add the staged particles to a rolling window of W cell
// layers held in registers; each consumer thread owns two cell columns adjacent
// along y.  The two producer groups take alternate bin layers, each into its own
// buffer, handed over by named barriers (FULL_g: group g arrives, consumers wait;
// EMPTY_g: consumers arrive, group g waits): a group's global loads for layer k + 2
// overlap the consumers' sums over layers k and k + 1.  A bin layer with more
// particles than a buffer holds is staged in several chunks, taken by both sides in
// the same order.
//
// Consumer visits.  The W bins of one bin row that reach a cell column are
// consecutive in the sorted order, so a thread walks one contiguous range of
// staged particles per bin row; its W + 1 ranges (bin rows 2 ty .. 2 ty + W) are
// walked as one flattened loop, and every visit adds to both columns of the pair
// (the weight of a row that does not reach one of them is a stored zero).  A cell
// layer is final once the last bin layer that reaches it has been added.
constexpr int DEP_TX = 32;

template <typename R, int W> struct DepCfg;
// ncw consumer warps, two producer groups of npg warps, staging capacity per buffer
template <> struct DepCfg<float, 4> { static constexpr int ncw = 14, npg = 4, cap = 1152, ws = 4; };
template <> struct DepCfg<float, 6> { static constexpr int ncw = 12, npg = 2, cap = 1024, ws = 8; };
template <> struct DepCfg<double, 4> { static constexpr int ncw = 8, npg = 2, cap = 704, ws = 4; };
template <> struct DepCfg<double, 6> { static constexpr int ncw = 6, npg = 2, cap = 512, ws = 8; };

template <typename R, int W> __host__ __device__ constexpr int dep_threads() {
  return 32 * (DepCfg<R, W>::ncw + 2 * DepCfg<R, W>::npg);
}
template <typename R, int W> __host__ __device__ constexpr int dep_cells_y() { return 2 * DepCfg<R, W>::ncw; }

// one staging buffer: records [cap][4], z weights [cap][ws], x weights [W][cap],
// y weights [W + 2][cap] (rows 0 and W + 1 zero), bin starts [BYB][BX + 1], staged
// row offsets [BYB + 2]
template <typename R, int W> __host__ __device__ constexpr size_t dep_buf_vals() {
  return (size_t)DepCfg<R, W>::cap * (4 + DepCfg<R, W>::ws + W + (W + 2));
}
template <typename R, int W> __host__ __device__ constexpr size_t dep_buf_ints() {
  return (size_t)(dep_cells_y<R, W>() + W - 1) * (DEP_TX + W) + (dep_cells_y<R, W>() + W - 1) + 2;
}
template <typename R, int W> __host__ __device__ constexpr size_t dep_buf_bytes() {
  return (dep_buf_vals<R, W>() * sizeof(R) + 15) / 16 * 16;
}
template <typename R, int W> __host__ __device__ constexpr size_t dep_slot_bytes() {
  return (dep_buf_ints<R, W>() * sizeof(int) + 15) / 16 * 16;
}
// two staging buffers, four bin-start tables (two per producer group, alternating), the
// CTA's share
template <typename R, int W> __host__ __device__ constexpr size_t deposit_smem() {
  return 2 * dep_buf_bytes<R, W>() + 4 * dep_slot_bytes<R, W>() + 16 * sizeof(int);
}
static_assert(deposit_smem<float, 4>() <= 227 * 1024 && deposit_smem<float, 6>() <= 227 * 1024 &&
                  deposit_smem<double, 4>() <= 227 * 1024 && deposit_smem<double, 6>() <= 227 * 1024,
              "the deposit's staging must fit one CTA's shared memory");

// an int carried in a value slot (bit pattern)
template <typename R> __device__ __forceinline__ R int_bits(int v);
template <> __device__ __forceinline__ float int_bits<float>(int v) { return __int_as_float(v); }
template <> __device__ __forceinline__ double int_bits<double>(int v) { return __longlong_as_double((long long)v); }
template <typename R> __device__ __forceinline__ int bits_int(R v);
template <> __device__ __forceinline__ int bits_int<float>(float v) { return __float_as_int(v); }
template <> __device__ __forceinline__ int bits_int<double>(double v) { return (int)__double_as_longlong(v); }

template <typename R> __device__ __forceinline__ void lds4(const R *p, R *o);
template <> __device__ __forceinline__ void lds4<float>(const float *p, float *o) {
  const float4 v = *reinterpret_cast<const float4 *>(p);
  o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
}
template <> __device__ __forceinline__ void lds4<double>(const double *p, double *o) {
  const double2 a = *reinterpret_cast<const double2 *>(p), b = *reinterpret_cast<const double2 *>(p + 2);
  o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y;
}
template <typename R> __device__ __forceinline__ void sts4(R *p, R a, R b, R c, R d);
template <> __device__ __forceinline__ void sts4<float>(float *p, float a, float b, float c, float d) {
  *reinterpret_cast<float4 *>(p) = make_float4(a, b, c, d);
}
template <> __device__ __forceinline__ void sts4<double>(double *p, double a, double b, double c, double d) {
  *reinterpret_cast<double2 *>(p) = make_double2(a, b);
  *reinterpret_cast<double2 *>(p + 2) = make_double2(c, d);
}

// accumulators of a column pair: FP32 as packed pairs (one FFMA2 adds to both
// columns), FP64 as two scalars
template <typename R> struct PairAcc;
template <> struct PairAcc<float> {
  float2 a;
  __device__ __forceinline__ void zero() { a = make_float2(0.f, 0.f); }
  __device__ __forceinline__ void fma(float2 w, float v) { a = __ffma2_rn(w, make_float2(v, v), a); }
  __device__ __forceinline__ float lo() const { return a.x; }
  __device__ __forceinline__ float hi() const { return a.y; }
};
template <> struct PairAcc<double> {
  double x, y;
  __device__ __forceinline__ void zero() { x = 0.0; y = 0.0; }
  __device__ __forceinline__ void fma(double2 w, double v) { x = __fma_rn(w.x, v, x); y = __fma_rn(w.y, v, y); }
  __device__ __forceinline__ double lo() const { return x; }
  __device__ __forceinline__ double hi() const { return y; }
};
template <typename R> struct Pair2;
template <> struct Pair2<float> { using T = float2; };
template <> struct Pair2<double> { using T = double2; };
__device__ __forceinline__ float2 pmul(float2 a, float s) { return __fmul2_rn(a, make_float2(s, s)); }
__device__ __forceinline__ double2 pmul(double2 a, double s) { return make_double2(a.x * s, a.y * s); }

// one value copied asynchronously from global to shared memory
template <typename R> __device__ __forceinline__ void cp_async_val(R *sdst, const R *gsrc);
template <> __device__ __forceinline__ void cp_async_val<float>(float *sdst, const float *gsrc) { cp_async4(sdst, gsrc); }
template <> __device__ __forceinline__ void cp_async_val<double>(double *sdst, const double *gsrc) {
  cp_async8(sdst, gsrc);
}

// named CTA barriers: barrier.sync waits until `n` threads (a multiple of 32) have
// arrived, barrier.arrive counts the calling threads without waiting (their
// shared-memory writes before it are visible to the threads that wait)
__device__ __forceinline__ void nb_sync(int id, int n) {
  __syncwarp();
  asm volatile("barrier.sync %0, %1;" ::"r"(id), "r"(n) : "memory");
}
__device__ __forceinline__ void nb_arrive(int id, int n) {
  __syncwarp();
  asm volatile("barrier.arrive %0, %1;" ::"r"(id), "r"(n) : "memory");
}
constexpr int DEP_BAR_FULL = 1, DEP_BAR_EMPTY = 3, DEP_BAR_PROD = 5;  // + group (0, 1)

// The (tile, cell layer) position where share s starts.  A tile layer costs its
// cells plus a fixed part (the staging round trip and hand-over of a bin layer),
// counted as a quarter of a full tile.
struct DepPos { int t, z; };
__device__ __forceinline__ long long dep_layer_cost(int t, int ntx, int ext0, int ext1, int tw, int th) {
  const int tx = t % ntx, ty = t / ntx;
  return (long long)min(tw, ext0 - tx * tw) * min(th, ext1 - ty * th) + (tw * th) / 4;
}
__device__ inline DepPos dep_share_start(long long s, long long nshare, int ntx, int nt, int ext0, int ext1, int ext2,
                                         int tw, int th) {
  long long total = 0;
  for (int t = 0; t < nt; t++) total += dep_layer_cost(t, ntx, ext0, ext1, tw, th) * ext2;
  const long long P = s * total / nshare;
  long long cum = 0;
  for (int t = 0; t < nt; t++) {
    const long long a = dep_layer_cost(t, ntx, ext0, ext1, tw, th);
    const long long w = a * ext2;
    if (P < cum + w) return DepPos{t, (int)((P - cum) / a)};
    cum += w;
  }
  return DepPos{nt, 0};
}

// staging buffer of producer group `grp` and its bin-start table `par`
template <typename R, int W> struct DepBuf {
  R *recs, *wzs, *wxs, *wyp;
  int *sraw, *rowo;
  __device__ __forceinline__ DepBuf(unsigned char *smem, int grp, int par) {
    constexpr int CAP = DepCfg<R, W>::cap, WS = DepCfg<R, W>::ws;
    recs = reinterpret_cast<R *>(smem + grp * dep_buf_bytes<R, W>());
    wzs = recs + (size_t)4 * CAP;
    wxs = wzs + (size_t)WS * CAP;
    wyp = wxs + (size_t)W * CAP;
    sraw = reinterpret_cast<int *>(smem + 2 * dep_buf_bytes<R, W>() + (2 * grp + par) * dep_slot_bytes<R, W>());
    rowo = sraw + (dep_cells_y<R, W>() + W - 1) * (DEP_TX + W);
  }
};

template <typename R, int W, int NV>
__global__ void __launch_bounds__(dep_threads<R, W>(), 1)
    k_deposit(PartGeom<R> g, const R *__restrict__ pos, const R *__restrict__ val, int vstride,
              const unsigned *__restrict__ start, const int *__restrict__ perm, R *__restrict__ mesh, int mstride,
              int clear_mode, int TW, int TH) {
  using P2 = typename Pair2<R>::T;
  constexpr int CAP = DepCfg<R, W>::cap, WS = DepCfg<R, W>::ws;
  constexpr int NCW = DepCfg<R, W>::ncw, NPG = DepCfg<R, W>::npg;
  constexpr int NPT = 32 * NPG;            // threads of one producer group
  constexpr int NBAR = 32 * (NCW + NPG);   // consumers + one group
  constexpr int CY = dep_cells_y<R, W>();
  constexpr int BX = DEP_TX + W - 1, BYB = CY + W - 1;
  constexpr int NSR = BYB * (BX + 1);      // bin starts per layer
  constexpr int KSR = (NSR + NPT - 1) / NPT;
  static_assert(BYB <= 64, "one warp scans the bin rows of a layer");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  int *share = reinterpret_cast<int *>(smem_raw + 2 * dep_buf_bytes<R, W>() + 4 * dep_slot_bytes<R, W>());

  // tiles of TW x TH cells (TW <= 32, TH <= CY, equal sizes chosen by the host)
  const int ntx = (g.ext[0] + TW - 1) / TW, nty = (g.ext[1] + TH - 1) / TH, nt = ntx * nty;
  const int BXr = TW + W - 1, BYr = TH + W - 1;  // bins per row and bin rows that reach a tile
  if (threadIdx.x == 0) {
    const DepPos a = dep_share_start(blockIdx.x, gridDim.x, ntx, nt, g.ext[0], g.ext[1], g.ext[2], TW, TH);
    const DepPos b = dep_share_start(blockIdx.x + 1, gridDim.x, ntx, nt, g.ext[0], g.ext[1], g.ext[2], TW, TH);
    share[0] = a.t; share[1] = a.z; share[2] = b.t; share[3] = b.z;
  }
  __syncthreads();
  const int ta = share[0], za = share[1], tb = share[2], zb = share[3];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if (warp >= NCW) {
    // ======================================================== producers
    const int grp = (warp - NCW) / NPG;            // bin layers L with L % 2 == grp
    const int pt = threadIdx.x - 32 * (NCW + grp * NPG);
    const int pw = pt >> 5;
    int L = 0;  // running bin-layer count of this CTA (both roles count alike)
    int m = 0;  // chunks staged by this group
    for (int t = ta; t <= tb && t < nt; t++) {
      const int z0 = (t == ta) ? za : 0, z1 = (t == tb) ? zb : g.ext[2];
      if (z0 >= z1) continue;
      const int x0 = (t % ntx) * TW, y0 = (t / ntx) * TH;
      for (int bz = z0; bz <= z1 + W - 2; bz++, L++) {
        if ((L & 1) != grp) continue;
        const bool zin = bz < g.nb[2] && x0 < g.nb[0];
        int c0 = 0, total = 0;
        do {
          // this chunk's bin-start table was last read for the group's chunk m - 2,
          // which the consumers have handed back: it is filled before the buffer is free
          DepBuf<R, W> B(smem_raw, grp, m & 1);
          // ---- bin starts of the layer's rows (clamped to the row end), copied
          // asynchronously so that all of a thread's loads are in flight together
#pragma unroll 4
          for (int k = 0; k < KSR; k++) {
            const int i = pt + k * NPT;
            const int row = i / (BX + 1), bx = i - row * (BX + 1);
            const int by = y0 + row;
            if (i < NSR) {
              if (zin && row < BYr && by < g.nb[1]) {
                const unsigned rb = (unsigned)g.nb[0] * ((unsigned)by + (unsigned)g.nb[1] * (unsigned)bz);
                cp_async4(B.sraw + i, start + rb + (unsigned)min(x0 + min(bx, BXr), g.nb[0]));
              } else {
                B.sraw[i] = 0;
              }
            }
          }
          cp_async_commit();
          cp_async_wait_all();
          nb_sync(DEP_BAR_PROD + grp, NPT);
          if (pw == 0) {
            // exclusive prefix of the row lengths, two rows per lane (BYB <= 64)
            int len[2];
#pragma unroll
            for (int h = 0; h < 2; h++) {
              const int row = 2 * lane + h;
              len[h] = row < BYB ? B.sraw[row * (BX + 1) + BX] - B.sraw[row * (BX + 1)] : 0;
            }
            int x = len[0] + len[1];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
              const int y = __shfl_up_sync(0xffffffffu, x, o);
              if (lane >= o) x += y;
            }
            const int ex = x - len[0] - len[1];
            if (2 * lane <= BYB) B.rowo[2 * lane] = ex;
            if (2 * lane + 1 <= BYB) B.rowo[2 * lane + 1] = ex + len[0];
          }
          nb_sync(DEP_BAR_PROD + grp, NPT);
          total = B.rowo[BYB];
          const int c1 = min(total, c0 + CAP);
          // ---- stage particles [c0, c1).  Pass 1: each particle's index (row search
          // and sorted order), then asynchronous copies of its position into its
          // z-weight slots and of its values into its record, eight particles' loads
          // in flight at a time and all copies of the thread outstanding together.
          constexpr int U = 8;
          int pp[U];
          auto indices = [&](int qb) {
#pragma unroll
            for (int u = 0; u < U; u++) {
              const int q = qb + u * NPT;
              pp[u] = -1;
              if (q < c1) {
                int a = 0, bb = BYB - 1;  // last row with rowo[row] <= q
                while (a < bb) {
                  const int mid = (a + bb + 1) >> 1;
                  if (B.rowo[mid] <= q) a = mid;
                  else bb = mid - 1;
                }
                pp[u] = perm[B.sraw[a * (BX + 1)] + (q - B.rowo[a])];
              }
            }
          };
          // the first batch's indices are loaded before the buffer is free
          indices(c0 + pt);
          if (m >= 1) nb_sync(DEP_BAR_EMPTY + grp, NBAR);  // consumers are done with this buffer
          for (int qb = c0 + pt; qb < c1; qb += U * NPT) {
            if (qb != c0 + pt) indices(qb);
#pragma unroll
            for (int u = 0; u < U; u++) {
              if (pp[u] < 0) continue;
              const int i = qb + u * NPT - c0;
#pragma unroll
              for (int e = 0; e < 3; e++) cp_async_val<R>(B.wzs + (size_t)i * WS + e, pos + (size_t)3 * pp[u] + e);
#pragma unroll
              for (int c = 0; c < NV; c++) cp_async_val<R>(B.recs + (size_t)i * 4 + c, val + (size_t)vstride * pp[u] + c);
            }
          }
          cp_async_commit();
          cp_async_wait_all();
          // Pass 2: weights from the staged positions (a thread reads only the copies
          // it issued itself)
#pragma unroll 2
          for (int q = c0 + pt; q < c1; q += NPT) {
            const int i = q - c0;
            R wv[3][WS];
            long long bxi = 0;
#pragma unroll
            for (int e = 0; e < 3; e++) {
              const R x = B.wzs[(size_t)i * WS + e];
              const long long b2 = base_index(x, g.xmin[e], g.c1dx[e]);
              if (e == 0) bxi = b2;
              weights<R, W>(cell_offset<R>(x, g.xmin[e], g.dx[e], b2, g.c1dx[e]), wv[e]);
#pragma unroll
              for (int tt = W; tt < WS; tt++) wv[e][tt] = R(0);
            }
#pragma unroll
            for (int tt = 0; tt < W; tt++) {
              B.wxs[tt * CAP + i] = wv[0][tt];
              B.wyp[(tt + 1) * CAP + i] = wv[1][tt];
            }
            B.wyp[i] = R(0);
            B.wyp[(W + 1) * CAP + i] = R(0);
#pragma unroll
            for (int tt = 0; tt < WS; tt += 4)
              sts4<R>(B.wzs + i * WS + tt, wv[2][tt], wv[2][tt + 1], wv[2][tt + 2], wv[2][tt + 3]);
            const int bx = (int)(bxi - g.blo[0]) - x0;
            B.recs[(size_t)i * 4 + 3] = int_bits<R>(-bx * CAP);
          }
          nb_arrive(DEP_BAR_FULL + grp, NBAR);
          m++;
          c0 += CAP;
        } while (c0 < total);
      }
    }
    // drain: wait for the consumers' last hand-back so that every arrive on the
    // EMPTY barrier has its matching wait
    if (m >= 1) nb_sync(DEP_BAR_EMPTY + grp, NBAR);
    return;
  }

  // ========================================================== consumers
  const int tx = lane, ty = warp;
  int L = 0;
  int mc0 = 0, mc1 = 0;  // chunks taken from each producer group (their bin-start tables alternate)
  for (int t = ta; t <= tb && t < nt; t++) {
    const int z0 = (t == ta) ? za : 0, z1 = (t == tb) ? zb : g.ext[2];
    if (z0 >= z1) continue;
    const int x0 = (t % ntx) * TW, y0 = (t / ntx) * TH;
    const int cx = x0 + tx, cy = y0 + 2 * ty;
    const bool active = tx < TW && cx < g.ext[0] && 2 * ty < TH && cy < g.ext[1];
    // acc[s] is cell layer bz - (W - 1) + s of the columns (cx, cy) and (cx, cy + 1)
    // while bin layer bz is added
    PairAcc<R> acc[W][NV];
#pragma unroll
    for (int s = 0; s < W; s++)
#pragma unroll
      for (int c = 0; c < NV; c++) acc[s][c].zero();
    for (int bz = z0; bz <= z1 + W - 2; bz++, L++) {
      const int b = L & 1;
      int c0 = 0, total = 0;
      do {
        const int mcb = b ? mc1 : mc0;
        DepBuf<R, W> B(smem_raw, b, mcb & 1);
        nb_sync(DEP_BAR_FULL + b, NBAR);
        total = B.rowo[BYB];
        const int c1 = min(total, c0 + CAP);
        if (active && c1 > c0) {
          // this thread's W + 1 particle ranges (staged order), bin rows 2 ty .. 2 ty + W
          // (2 ty + W <= BYB - 1: every row exists), clamped to [c0, c1); one loop per
          // row with the row's y-weight offsets as constants, staged data addressed by
          // byte offsets from the shared-memory base
          const unsigned char *sb = smem_raw + b * dep_buf_bytes<R, W>();
          constexpr unsigned O_WZ = 4u * CAP * sizeof(R), O_WX = O_WZ + (unsigned)WS * CAP * sizeof(R);
          constexpr unsigned O_WY = O_WX + (unsigned)W * CAP * sizeof(R);
#pragma unroll
          for (int r = 0; r <= W; r++) {
            const int *sr = B.sraw + (2 * ty + r) * (BX + 1);
            const int l = B.rowo[2 * ty + r] + sr[tx] - sr[0];
            const int q0 = max(l, c0) - c0, q1 = min(l + sr[tx + W] - sr[tx], c1) - c0;
            // row r: y weights of the pair are wyp[W - r] and wyp[W + 1 - r]
            const unsigned char *prec = sb + (size_t)q0 * 4 * sizeof(R);
            const unsigned char *pwz = sb + O_WZ + (size_t)q0 * WS * sizeof(R);
            const unsigned char *pwy = sb + O_WY + (unsigned)(W - r) * CAP * sizeof(R) + (size_t)q0 * sizeof(R);
            const unsigned char *pwx = sb + O_WX + (unsigned)(W - 1 + tx) * CAP * sizeof(R) + (size_t)q0 * sizeof(R);
            // two particles per iteration (their loads in flight together), then the
            // odd one
            auto visit = [&](const R *v, const R *wz, R wx, R wy0, R wy1) {
              P2 wxy;
              wxy.x = wx * wy0;
              wxy.y = wx * wy1;
#pragma unroll
              for (int sz = 0; sz < W; sz++) {
                const P2 w = pmul(wxy, wz[sz]);
#pragma unroll
                for (int c = 0; c < NV; c++) acc[sz][c].fma(w, v[c]);
              }
            };
            int q = q0;
#pragma unroll 1
            for (; q + 1 < q1; q += 2) {
              R v[2][4], wz[2][WS];
#pragma unroll
              for (int h = 0; h < 2; h++) {
                lds4<R>(reinterpret_cast<const R *>(prec) + 4 * h, v[h]);
                lds4<R>(reinterpret_cast<const R *>(pwz) + WS * h, wz[h]);
                if constexpr (WS == 8) lds4<R>(reinterpret_cast<const R *>(pwz) + WS * h + 4, wz[h] + 4);
              }
              R wx[2], wy0[2], wy1[2];
#pragma unroll
              for (int h = 0; h < 2; h++) {
                wx[h] = *reinterpret_cast<const R *>(pwx + (ptrdiff_t)(bits_int<R>(v[h][3]) + h) * (ptrdiff_t)sizeof(R));
                wy0[h] = *reinterpret_cast<const R *>(pwy + h * sizeof(R));
                wy1[h] = *reinterpret_cast<const R *>(pwy + (CAP + h) * sizeof(R));
              }
              visit(v[0], wz[0], wx[0], wy0[0], wy1[0]);
              visit(v[1], wz[1], wx[1], wy0[1], wy1[1]);
              prec += 8 * sizeof(R);
              pwz += 2 * WS * sizeof(R);
              pwy += 2 * sizeof(R);
              pwx += 2 * sizeof(R);
            }
            if (q < q1) {
              R v[4], wz[WS];
              lds4<R>(reinterpret_cast<const R *>(prec), v);
              lds4<R>(reinterpret_cast<const R *>(pwz), wz);
              if constexpr (WS == 8) lds4<R>(reinterpret_cast<const R *>(pwz) + 4, wz + 4);
              const R wx = *reinterpret_cast<const R *>(pwx + (ptrdiff_t)bits_int<R>(v[3]) * (ptrdiff_t)sizeof(R));
              visit(v, wz, wx, *reinterpret_cast<const R *>(pwy), *reinterpret_cast<const R *>(pwy + CAP * sizeof(R)));
            }
          }
        }
        nb_arrive(DEP_BAR_EMPTY + b, NBAR);
        if (b) mc1++;
        else mc0++;
        c0 += CAP;
      } while (c0 < total);
      // ---- cell layer bz - (W - 1) is complete
      const int cz = bz - (W - 1);
      if (active && cz >= z0 && cz < z1) {
#pragma unroll
        for (int h = 0; h < 2; h++) {
          const int yy = cy + h;
          if (2 * ty + h < TH && yy < g.ext[1]) {
            const size_t m = (((size_t)cz * g.ext[1] + yy) * g.ext[0] + cx) * mstride;
            const int ii = cx + g.lo[0], jj = yy + g.lo[1], kk = cz + g.lo[2];
            const bool ghost = ii < 1 || ii > g.nint[0] || jj < 1 || jj > g.nint[1] || kk < 1 || kk > g.nint[2];
            const bool overwrite = clear_mode == 1 || (clear_mode == 2 && ghost);
#pragma unroll
            for (int c = 0; c < NV; c++) {
              const R a = h ? acc[0][c].hi() : acc[0][c].lo();
              mesh[m + c] = overwrite ? a : mesh[m + c] + a;
            }
          }
        }
      }
#pragma unroll
      for (int s = 0; s < W; s++)
#pragma unroll
        for (int c = 0; c < NV; c++) {
          if (s + 1 < W) acc[s][c] = acc[s + 1][c];
          else acc[s][c].zero();
        }
    }
  }
}

// a constant vector added to every point of a (3, n) field (the client's free-stream
// velocity, vortex_codes/vortex_penalisation/source/main.f:425-437)
template <typename R> __global__ void k_add_vec3(R *__restrict__ f, size_t n, R a, R b, R c) {
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x) {
    f[3 * t] = f[3 * t] + a;
    f[3 * t + 1] = f[3 * t + 1] + b;
    f[3 * t + 2] = f[3 * t + 2] + c;
  }
}

// periodic ghost reverse-add of P2M, one axis (pmlib_mesh_map_ghost.f:119-207 with
// pmlib_comm_unpack.f:269-273): both strips [1-ngl, ngh] and [N-ngl+1, N+ngh]
// receive the sum of the two, from the values before the exchange.
template <typename R>
__global__ void k_ghost_add(R *__restrict__ mesh, int ex, int ey, int ez, int nv, int axis, int N, int ngl,
                            int ngh) {
  const int e[3] = {ex, ey, ez};
  const int S = ngl + ngh;
  const int o1 = axis == 0 ? 1 : 0, o2 = axis == 2 ? 1 : 2;
  const long long total = (long long)S * e[o1] * e[o2];
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int s = (int)(t % S);
    const long long r = t / S;
    const int a = (int)(r % e[o1]), b = (int)(r / e[o1]);
    int iw[3], ie[3];
    iw[o1] = a; iw[o2] = b; iw[axis] = s;
    ie[o1] = a; ie[o2] = b; ie[axis] = N + s;
    const size_t mw = (((size_t)iw[2] * ey + iw[1]) * ex + iw[0]) * nv;
    const size_t me = (((size_t)ie[2] * ey + ie[1]) * ex + ie[0]) * nv;
    for (int c = 0; c < nv; c++) {
      const R w = mesh[mw + c], v = mesh[me + c];
      mesh[me + c] = v + w;
      mesh[mw + c] = w + v;
    }
  }
}

// ------------------------------------------------------------------ M2P
// source/interpolation/pmlib_interp_mesh_particle.f:76-409 (M4'), :412-1266 (M6*):
// stencil indices clamp to the cuboid with zero weight, no particle is skipped, and
// the M4' branch scales the y and z offsets by 1/dx(1) (:115-116).
// Particles order[i] for i in [first ? *first : 0, n).
template <typename R, int W>
__global__ void k_m2p(PartGeom<R> g, const R *__restrict__ pos, const int *__restrict__ order, int n,
                      const unsigned *__restrict__ first, const R *__restrict__ f0, const R *__restrict__ f1,
                      const R *__restrict__ f2, R *__restrict__ o0, R *__restrict__ o1, R *__restrict__ o2) {
  constexpr int off = Stencil<W>::off;
  const int i0 = first ? (int)*first : 0;
  for (int i = i0 + blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int p = order ? order[i] : i;
    R w[3][W];
    int idx[3][W];
#pragma unroll
    for (int e = 0; e < 3; e++) {
      const R x = pos[(size_t)3 * p + e];
      long long b = base_index(x, g.xmin[e], g.c1dx[e]);
      const R scale = (W == 4) ? g.c1dx[0] : g.c1dx[e];
      const long long bc = b < -(1LL << 40) ? 0 : b;
      weights<R, W>(cell_offset<R>(x, g.xmin[e], g.dx[e], bc, scale), w[e]);
      const long long hi = g.lo[e] + g.ext[e] - 1;
#pragma unroll
      for (int s = 0; s < W; s++) {
        long long ii = bc - off + s;
        if (b < -(1LL << 40)) { w[e][s] = R(0); ii = g.lo[e]; }
        if (ii < g.lo[e]) { w[e][s] = R(0); ii = g.lo[e]; }
        if (ii > hi) { w[e][s] = R(0); ii = hi; }
        idx[e][s] = (int)(ii - g.lo[e]);
      }
    }
    const R *fs[3] = {f0, f1, f2};
    R *os[3] = {o0, o1, o2};
#pragma unroll
    for (int f = 0; f < 3; f++) {
      if (!fs[f]) continue;
      const R *m = fs[f];
      R a0 = R(0), a1 = R(0), a2 = R(0);
#pragma unroll
      for (int sk = 0; sk < W; sk++)
#pragma unroll
        for (int sj = 0; sj < W; sj++) {
          const size_t rowb = ((size_t)idx[2][sk] * g.ext[1] + idx[1][sj]) * g.ext[0];
          const R wjk = w[1][sj] * w[2][sk];
#pragma unroll
          for (int si = 0; si < W; si++) {
            const R wt = w[0][si] * wjk;
            const R *q = m + (rowb + idx[0][si]) * 3;
            a0 += wt * __ldg(q);
            a1 += wt * __ldg(q + 1);
            a2 += wt * __ldg(q + 2);
          }
        }
      os[f][(size_t)3 * p + 0] = a0;
      os[f][(size_t)3 * p + 1] = a1;
      os[f][(size_t)3 * p + 2] = a2;
    }
  }
}

// M2P over particles sorted by bin (the order of the preceding deposition): a CTA
// owns TX x TY x TZ bins, stages the cells their stencils reach in shared memory
// (one plane per component, zero outside the cuboid, where the weight is zero as
// well) and interpolates the particles of those bins from there.  A warp's lanes
// take consecutive particles of a bin row, so each per-component load of a stencil
// point reads words of neighbouring cells: one shared-memory wavefront, bank
// conflicts only where the warp spans two bin rows.  The particles of one bin row
// are one contiguous range of the sorted order.  Same index and weight rules as
// k_m2p; particles with the sentinel key (outside every bin) are left to k_m2p.
constexpr int M2P_TX = 32, M2P_TY = 8, M2P_TZ = 8, M2P_THREADS = 256;

template <typename R, int W> __host__ __device__ constexpr size_t m2p_tile_smem() {
  return (size_t)(M2P_TX + W - 1) * (M2P_TY + W - 1) * (M2P_TZ + W - 1) * 3 * sizeof(R);
}

template <typename R, int W>
__global__ void __launch_bounds__(M2P_THREADS) k_m2p_tile(PartGeom<R> g, const R *__restrict__ pos,
                                                          const unsigned *__restrict__ start,
                                                          const int *__restrict__ perm, const R *__restrict__ f,
                                                          R *__restrict__ o, int3 org) {
  constexpr int off = Stencil<W>::off;
  constexpr int CX = M2P_TX + W - 1, CY = M2P_TY + W - 1, CZ = M2P_TZ + W - 1, NR = M2P_TY * M2P_TZ;
  constexpr int PLANE = CZ * CY * CX;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  // components 0 and 1 as pairs [CZ][CY][CX][2], component 2 as a plane [CZ][CY][CX]:
  // one 8-byte (FP64: 16-byte) and one 4-byte (8-byte) load a stencil point
  R *cells = reinterpret_cast<R *>(smem_raw);
  __shared__ int rs[NR + 1], rg[NR];
  // tile origin in bins; org (<= 0) puts the tile edges on the first interior bin, so
  // that one particle per cell fills whole 32-bin rows (warp-aligned, no empty tiles)
  const int x0 = blockIdx.x * M2P_TX + org.x, y0 = blockIdx.y * M2P_TY + org.y, z0 = blockIdx.z * M2P_TZ + org.z;
  const int cx0 = x0 - (W - 1), cy0 = y0 - (W - 1), cz0 = z0 - (W - 1);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  // ---- particle ranges of the bin rows (two rows a lane, NR <= 64)
  static_assert(NR <= 64, "one warp scans the bin rows of a tile");
  if (threadIdx.x < 32) {
    int len[2] = {0, 0};
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int r = 2 * lane + h;
      int gs = 0;
      if (r < NR) {
        const int by = y0 + r % M2P_TY, bz = z0 + r / M2P_TY;
        if (by >= 0 && bz >= 0 && by < g.nb[1] && bz < g.nb[2]) {
          const unsigned rb = (unsigned)g.nb[0] * ((unsigned)by + (unsigned)g.nb[1] * (unsigned)bz);
          gs = (int)start[rb + (unsigned)max(x0, 0)];
          len[h] = (int)start[rb + (unsigned)min(x0 + M2P_TX, g.nb[0])] - gs;
        }
        rg[r] = gs;
      }
    }
    int x = len[0] + len[1];
#pragma unroll
    for (int o2 = 1; o2 < 32; o2 <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, x, o2);
      if (lane >= o2) x += y;
    }
    const int ex = x - len[0] - len[1];
    if (2 * lane < NR) rs[2 * lane] = ex;
    if (2 * lane + 1 < NR) rs[2 * lane + 1] = ex + len[0];
    if (lane == 31) rs[NR] = x;
  }
  __syncthreads();
  if (rs[NR] == 0) return;  // no particle in the tile: nothing to stage
  // ---- stage the cells: one warp per cell row; lane offsets are the same in every row
  {
    constexpr int NE = (CX * 3 + 31) / 32;
    int so[NE], dof[NE];
    bool ok[NE], pair[NE];
#pragma unroll
    for (int k = 0; k < NE; k++) {
      const int e = lane + 32 * k;
      const int xx = e / 3, c = e - 3 * xx;
      const int cx = cx0 + xx;
      ok[k] = e < CX * 3 && cx >= 0 && cx < g.ext[0];
      so[k] = cx * 3 + c;
      pair[k] = c < 2;
      dof[k] = e < CX * 3 ? (c < 2 ? 2 * xx + c : 2 * PLANE + xx) : -1;
    }
    for (int row = wid; row < CZ * CY; row += nw) {
      const int yy = row % CY, zz = row / CY;
      const int cy = cy0 + yy, cz = cz0 + zz;
      R *dst01 = cells + (size_t)2 * row * CX, *dst2 = cells + (size_t)row * CX;
      const bool rowin = cy >= 0 && cy < g.ext[1] && cz >= 0 && cz < g.ext[2];
      const R *src = f + (((size_t)(rowin ? cz : 0) * g.ext[1] + (rowin ? cy : 0)) * g.ext[0]) * 3;
      R v[NE];
#pragma unroll
      for (int k = 0; k < NE; k++) v[k] = (rowin && ok[k]) ? __ldg(src + so[k]) : R(0);
#pragma unroll
      for (int k = 0; k < NE; k++)
        if (dof[k] >= 0) (pair[k] ? dst01 : dst2)[dof[k]] = v[k];
    }
  }
  __syncthreads();
  const int total = rs[NR];
  for (int q = threadIdx.x; q < total; q += blockDim.x) {
    int lo = 0, hi = NR - 1;  // last row with rs[row] <= q
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (rs[mid] <= q) lo = mid;
      else hi = mid - 1;
    }
    const int p = perm[rg[lo] + (q - rs[lo])];
    R w[3][W];
    int tb[3];
#pragma unroll
    for (int e = 0; e < 3; e++) {
      const R x = pos[(size_t)3 * p + e];
      const int b = (int)base_index(x, g.xmin[e], g.c1dx[e]);  // a binned particle has a small index
      const R scale = (W == 4) ? g.c1dx[0] : g.c1dx[e];
      weights<R, W>(cell_offset<R>(x, g.xmin[e], g.dx[e], (long long)b, scale), w[e]);
      const int lo_e = g.lo[e], hi_e = g.lo[e] + g.ext[e] - 1;
#pragma unroll
      for (int s2 = 0; s2 < W; s2++) {
        const int ii = b - off + s2;
        if (ii < lo_e || ii > hi_e) w[e][s2] = R(0);
      }
      // first stencil cell relative to the tile: bin - tile origin
      tb[e] = b - g.blo[e] - (e == 0 ? x0 : e == 1 ? y0 : z0);
    }
    typedef typename Pair2<R>::T P2;
    const int c0i = (tb[2] * CY + tb[1]) * CX + tb[0];
    const P2 *base01 = reinterpret_cast<const P2 *>(cells) + c0i;
    const R *base2 = cells + 2 * PLANE + c0i;
    R a0 = R(0), a1 = R(0), a2 = R(0);
#pragma unroll
    for (int sk = 0; sk < W; sk++)
#pragma unroll
      for (int sj = 0; sj < W; sj++) {
        const R wjk = w[1][sj] * w[2][sk];
        const int ro = (sk * CY + sj) * CX;
#pragma unroll
        for (int si = 0; si < W; si++) {
          const R wt = w[0][si] * wjk;
          const P2 u01 = base01[ro + si];
          a0 += wt * u01.x;
          a1 += wt * u01.y;
          a2 += wt * base2[ro + si];
        }
      }
    o[(size_t)3 * p + 0] = a0;
    o[(size_t)3 * p + 1] = a1;
    o[(size_t)3 * p + 2] = a2;
  }
}

// ------------------------------------------------------------------ diagnostics
// Global particle diagnostics in FP64 whatever the field precision
// (vortex_codes/vortex_structures/source/diagnostics/diagnostics_knot.f:75-158):
//   0-2 impulse 1/2 sum x*w, 3-5 angular impulse 1/3 sum x*(x*w), 6 kinetic energy
//   sum u.(x*w), 7 enstrophy sum |w|^2, 8 helicity sum u.w (all times dx dy dz),
//   9-11 sum |w|^2 x and 12 sum |w|^2 sqrt(y^2 + z^2) (normalised by the enstrophy
//   on the host), 13 max |w|.  Each block sums a fixed slice in a fixed order, so
//   the totals are the same on every run.
constexpr int DIAG_N = 14;
constexpr int DIAG_THREADS = 256;
template <typename R>
__global__ void __launch_bounds__(DIAG_THREADS) k_diag_partial(const R *__restrict__ pos, const R *__restrict__ vel,
                                                               const R *__restrict__ vort, int n, double dv,
                                                               double *__restrict__ part) {
  double acc[DIAG_N];
#pragma unroll
  for (int i = 0; i < DIAG_N; i++) acc[i] = 0.0;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    const double x = pos[3 * (size_t)p], y = pos[3 * (size_t)p + 1], z = pos[3 * (size_t)p + 2];
    const double u = vel[3 * (size_t)p], v = vel[3 * (size_t)p + 1], w = vel[3 * (size_t)p + 2];
    const double a = vort[3 * (size_t)p], b = vort[3 * (size_t)p + 1], c = vort[3 * (size_t)p + 2];
    const double m1x = y * c - z * b, m1y = z * a - x * c, m1z = x * b - y * a;  // x * w
    const double m2x = y * m1z - z * m1y, m2y = z * m1x - x * m1z, m2z = x * m1y - y * m1x;
    const double e = a * a + b * b + c * c;
    acc[0] += 0.5 * m1x * dv;
    acc[1] += 0.5 * m1y * dv;
    acc[2] += 0.5 * m1z * dv;
    acc[3] += (1.0 / 3.0) * m2x * dv;
    acc[4] += (1.0 / 3.0) * m2y * dv;
    acc[5] += (1.0 / 3.0) * m2z * dv;
    acc[6] += (u * m1x + v * m1y + w * m1z) * dv;
    acc[7] += e * dv;
    acc[8] += (u * a + v * b + w * c) * dv;
    acc[9] += e * x * dv;
    acc[10] += e * y * dv;
    acc[11] += e * z * dv;
    acc[12] += e * sqrt(y * y + z * z) * dv;
    acc[13] = fmax(acc[13], sqrt(e));
  }
  __shared__ double sh[DIAG_THREADS];
  for (int i = 0; i < DIAG_N; i++) {
    sh[threadIdx.x] = acc[i];
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
      if ((int)threadIdx.x < s) sh[threadIdx.x] = i == 13 ? fmax(sh[threadIdx.x], sh[threadIdx.x + s])
                                                          : sh[threadIdx.x] + sh[threadIdx.x + s];
      __syncthreads();
    }
    if (threadIdx.x == 0) part[(size_t)blockIdx.x * DIAG_N + i] = sh[0];
    __syncthreads();
  }
}

// one thread per quantity sums the block partials in block order
__global__ void k_diag_final(const double *__restrict__ part, int nblk, double *__restrict__ out) {
  const int i = threadIdx.x;
  if (i >= DIAG_N) return;
  double s = 0.0;
  for (int b = 0; b < nblk; b++) s = i == 13 ? fmax(s, part[(size_t)b * DIAG_N + i]) : s + part[(size_t)b * DIAG_N + i];
  out[i] = s;
}

// ------------------------------------------------------------------ remesh
// source/remesh/pmlib_remesh.f:84-226: a particle per kept cell, cells in k-j-i order
template <typename R>
__global__ void k_remesh_flag(PartGeom<R> g, const R *__restrict__ vort, const R *__restrict__ dvort,
                              const unsigned char *__restrict__ mask, R min_vort, R min_dvort, int incl_ghost,
                              unsigned *__restrict__ flag) {
  const size_t total = (size_t)g.ext[0] * g.ext[1] * g.ext[2];
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(t % g.ext[0]) + g.lo[0];
    const int j = (int)((t / g.ext[0]) % g.ext[1]) + g.lo[1];
    const int k = (int)(t / ((size_t)g.ext[0] * g.ext[1])) + g.lo[2];
    const int ii[3] = {i, j, k};
    bool place = true;
    for (int e = 0; e < 3; e++) {
      const bool in = (ii[e] >= 1 && ii[e] <= g.nint[e]) || (incl_ghost && ii[e] < 1 && g.bclo[e] == 0) ||
                      (incl_ghost && ii[e] > g.nint[e] && g.bchi[e] == 0);
      place = place && in;
    }
    const R *v = vort + 3 * t;
    const R s = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    R ds = R(0);
    if (dvort) {
      const R *dv = dvort + 3 * t;
      ds = sqrt(dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2]);
    }
    if (place && (s > min_vort || ds > min_dvort)) place = mask ? (mask[t] != 0) : true;
    else place = false;
    flag[t] = place ? 1u : 0u;
  }
}

template <typename R>
__global__ void k_remesh_fill(PartGeom<R> g, const R *__restrict__ vort, const R *__restrict__ dvort,
                              const R *__restrict__ vel, const unsigned *__restrict__ flag,
                              const unsigned *__restrict__ slot, R *__restrict__ pos, R *__restrict__ pv,
                              R *__restrict__ pdv, R *__restrict__ pvel) {
  const size_t total = (size_t)g.ext[0] * g.ext[1] * g.ext[2];
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
    if (!flag[t]) continue;
    const int ii[3] = {(int)(t % g.ext[0]) + g.lo[0], (int)((t / g.ext[0]) % g.ext[1]) + g.lo[1],
                       (int)(t / ((size_t)g.ext[0] * g.ext[1])) + g.lo[2]};
    const size_t q = 3 * (size_t)slot[t];
    for (int e = 0; e < 3; e++) {
      pos[q + e] = g.xmin[e] + ((R)(ii[e] - 1) + R(0.5)) * g.dx[e];
      pv[q + e] = vort[3 * t + e];
      if (pdv) pdv[q + e] = dvort ? dvort[3 * t + e] : R(0);
      if (pvel) pvel[q + e] = vel ? vel[3 * t + e] : R(0);
    }
  }
}

}  // namespace pmgpu
