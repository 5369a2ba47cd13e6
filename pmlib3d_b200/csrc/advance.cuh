// advance.cuh -- the particle time step around the solve: the vorticity right-hand
// side on the mesh (stretching + diffusion) and the Runge-Kutta stage update with
// the particle map (drop across free faces, wrap across periodic ones, reorder).
//
// Right-hand side (vortex_codes/vortex_structures/source/particle_derivatives/
// part_deriv_vorticity.f:57-193): one thread per interior cell,
//   dvort_l = visc (d2/dx2 + d2/dy2 + d2/dz2) vort_l + w . grad u_l
// with second- or fourth-order central differences; the neighbours come through
// the read-only cache (x neighbours share lines, y / z neighbours are reused by the
// CTA's other rows).
//
// Stage update (source/particles/pmlib_particles_advance.f:95-113) and map
// (pmlib_particles_map.f:63-127 with the communication order of one rank): the
// update uses unfused multiplies and adds in the reference's evaluation order, so
// positions, and with them the side a particle leaves on, are bit-identical to the
// reference arithmetic.  The reference maps the axes x, y, z in turn; one pass over
// an axis puts the low-side leavers first, then the high-side leavers, then the
// rest, and repeats while a particle is still outside a periodic side.  Pass t over
// an axis is a stable partition by the particle's class c_t in that pass (low 0,
// high 1, inside 2), so after K passes the order along the axis is lexicographic in
// (c_K, ..., c_1) and then the previous order.  Wraps only move a particle along
// their own axis, so a particle's classes on every axis follow from its own
// position, and the whole map is one stable sort by (key_z, key_y, key_x) with
// key_d = sum_t c_t 3^(t-1) over the K_d passes of axis d; particles that leave
// across a free side are dropped.  At most two passes per axis are supported (a
// particle moving more than a patch length in one step is reported as an error).
#pragma once

#include "common.cuh"

namespace pmgpu {

// ------------------------------------------------------------------ right-hand side
template <typename R> struct DerivGeom {
  int ext[3];      // cuboid extents including ghosts
  int ngl[3];      // low-face ghosts
  int nc[3];       // interior cells
  R c_1_dx2[3];    // 1 / dx^2
  R c_1_2dx[3];    // 1 / (2 dx)
  R visc;
};

template <typename R, int FD>
__global__ void __launch_bounds__(256) k_deriv_vorticity(DerivGeom<R> g, const R *__restrict__ vort,
                                                         const R *__restrict__ vel, R *__restrict__ dvort) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (i >= g.nc[0] || j >= g.nc[1]) return;
  const long long sx = 3, sy = 3LL * g.ext[0], sz = 3LL * g.ext[0] * g.ext[1];
  const long long m = (long long)(k + g.ngl[2]) * sz + (long long)(j + g.ngl[1]) * sy + (long long)(i + g.ngl[0]) * sx;
  const long long st[3] = {sx, sy, sz};
  const R w[3] = {__ldg(vort + m), __ldg(vort + m + 1), __ldg(vort + m + 2)};
#pragma unroll
  for (int l = 0; l < 3; l++) {
    const R *v = vort + m + l;
    const R *u = vel + m + l;
    const R v0 = __ldg(v);
    R dd[3], du[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
      const long long s = st[a];
      if constexpr (FD == 2) {
        dd[a] = (R(1) * __ldg(v - s) - R(2) * v0 + R(1) * __ldg(v + s)) * g.c_1_dx2[a];
        du[a] = (R(-1) * __ldg(u - s) + R(1) * __ldg(u + s)) * g.c_1_2dx[a];
      } else {
        const R c1 = R(-1) / R(12), c2 = R(4) / R(3), c3 = R(1) / R(6), c4 = R(4) / R(3);
        dd[a] = (c1 * __ldg(v - 2 * s) + c2 * __ldg(v - s) - R(2.5) * v0 + c2 * __ldg(v + s) + c1 * __ldg(v + 2 * s)) *
                g.c_1_dx2[a];
        du[a] = (c3 * __ldg(u - 2 * s) - c4 * __ldg(u - s) + c4 * __ldg(u + s) - c3 * __ldg(u + 2 * s)) * g.c_1_2dx[a];
      }
    }
    dvort[m + l] = g.visc * (dd[0] + dd[1] + dd[2]) + w[0] * du[0] + w[1] * du[1] + w[2] * du[2];
  }
}

// ------------------------------------------------------------------ stage update + map sides
template <typename R> struct AdvanceCoef {
  R a1, b1dt, c1, a2, b2dt, c2;  // b * dt formed in R as the reference does (b1(s)*dtime first)
  int zero_rk;                   // first-order scheme: the stage storage is cleared after the map
  R xmin[3], xmax[3];            // topology bounds: sides
  R pmin[3], pmax[3], plen[3];   // patch bounds and length: wraps
  int per_lo[3], per_hi[3];
};

__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }

constexpr unsigned ADV_REMOVED = 0x80000000u;
constexpr int ADV_PASSES = 2;  // map passes per axis the key holds

// Per particle: RK stage update in place, positions wrapped, and the map code: per
// axis 4 bits (bits 0-1 the class in pass 1, bits 2-3 in pass 2; 2 = inside), bit 31
// dropped.  stats[0] |= 1 when a particle leaves or is dropped, stats[1 + d] = the
// most passes axis d needs, stats[4] = 1 when a particle needs more than ADV_PASSES.
template <typename R>
__global__ void k_advance(AdvanceCoef<R> c, int n, R *__restrict__ pos, R *__restrict__ vort,
                          const R *__restrict__ vel, const R *__restrict__ dvort, R *__restrict__ vel_rk,
                          R *__restrict__ dvort_rk, unsigned *__restrict__ code, unsigned *__restrict__ stats) {
  const int stride = gridDim.x * blockDim.x;
  for (int p0 = blockIdx.x * blockDim.x; p0 < n; p0 += stride) {
    const int p = p0 + (int)threadIdx.x;
    unsigned cd = 0, np[3] = {0, 0, 0}, bad = 0;
    if (p < n) {
#pragma unroll
      for (int e = 0; e < 3; e++) {
        const size_t q = (size_t)3 * p + e;
        const R vr = add_rn(mul_rn(c.a1, vel_rk[q]), mul_rn(c.b1dt, vel[q]));
        const R dr = add_rn(mul_rn(c.a2, dvort_rk[q]), mul_rn(c.b2dt, dvort[q]));
        R x = add_rn(pos[q], mul_rn(c.c1, vr));
        vort[q] = add_rn(vort[q], mul_rn(c.c2, dr));
        vel_rk[q] = c.zero_rk ? R(0) : vr;
        dvort_rk[q] = c.zero_rk ? R(0) : dr;
        unsigned cls = 0xAu;  // both passes "inside"
        // pass t + 1 over this axis (a particle dropped on an earlier axis is gone)
        for (int t = 0; t <= ADV_PASSES && !(cd & ADV_REMOVED); t++) {
          const unsigned side = x < c.xmin[e] ? 0u : (x >= c.xmax[e] ? 1u : 2u);
          if (side == 2u) break;
          if ((side == 0u && !c.per_lo[e]) || (side == 1u && !c.per_hi[e])) {
            cd |= ADV_REMOVED;
            break;
          }
          if (t == ADV_PASSES) {
            bad = 1;
            break;
          }
          if (side == 0u && x < c.pmin[e]) x = add_rn(x, c.plen[e]);
          if (side == 1u && x >= c.pmax[e]) x = sub_rn(x, c.plen[e]);
          cls = (cls & ~(3u << (2 * t))) | (side << (2 * t));
          np[e] = t + 1;
        }
        pos[q] = x;
        cd |= cls << (4 * e);
      }
      code[p] = cd;
    }
    const unsigned moved = ((cd & ADV_REMOVED) || np[0] || np[1] || np[2]) ? 1u : 0u;
    const unsigned anym = __reduce_or_sync(0xffffffffu, moved | (bad << 1));
    if (anym) {
      const unsigned m0 = __reduce_max_sync(0xffffffffu, np[0]), m1 = __reduce_max_sync(0xffffffffu, np[1]),
                     m2 = __reduce_max_sync(0xffffffffu, np[2]);
      if ((threadIdx.x & 31) == 0) {
        if (anym & 1u) atomicOr(&stats[0], 1u);
        if (m0) atomicMax(&stats[1], m0);
        if (m1) atomicMax(&stats[2], m1);
        if (m2) atomicMax(&stats[3], m2);
        if (anym & 2u) atomicOr(&stats[4], 1u);
      }
    }
  }
}

// bucket of a particle from its map code; K[d] = passes over axis d (0..2); nbk =
// number of live buckets (the dropped go to bucket nbk)
__device__ __forceinline__ unsigned map_bucket(unsigned cd, const int K[3], unsigned nbk) {
  if (cd & ADV_REMOVED) return nbk;
  unsigned b = 0;
#pragma unroll
  for (int e = 2; e >= 0; e--) {
    const unsigned f = (cd >> (4 * e)) & 15u;
    unsigned key = 0;
    for (int t = K[e] - 1; t >= 0; t--) key = key * 3u + ((f >> (2 * t)) & 3u);
    unsigned pw = 1;
    for (int t = 0; t < K[e]; t++) pw *= 3u;
    b = b * pw + key;
  }
  return b;
}

// ------------------------------------------------------------------ stable partition
// A CTA owns MAP_CHUNK consecutive particles; its warps own MAP_CHUNK / 8 each.
constexpr int MAP_THREADS = 256;
constexpr int MAP_WARPS = MAP_THREADS / 32;
constexpr int MAP_CHUNK = 4096;
constexpr int MAP_MAX_BUCKETS = 730;  // two passes on every axis: 9^3 live buckets + dropped

// counts[b * nblk + blk]: particles of CTA blk in bucket b (bucket-major, so an
// exclusive scan gives every (bucket, CTA) its first output slot)
__global__ void __launch_bounds__(MAP_THREADS) k_map_count(const unsigned *__restrict__ code, int n, int K0, int K1,
                                                           int K2, unsigned nbk, unsigned *__restrict__ counts) {
  __shared__ unsigned h[MAP_MAX_BUCKETS];
  const int K[3] = {K0, K1, K2};
  for (int b = threadIdx.x; b <= (int)nbk; b += blockDim.x) h[b] = 0;
  __syncthreads();
  const int base = blockIdx.x * MAP_CHUNK;
  for (int t = threadIdx.x; t < MAP_CHUNK; t += blockDim.x) {
    const int p = base + t;
    if (p < n) atomicAdd(&h[map_bucket(code[p], K, nbk)], 1u);
  }
  __syncthreads();
  for (int b = threadIdx.x; b <= (int)nbk; b += blockDim.x) counts[(size_t)b * gridDim.x + blockIdx.x] = h[b];
}

// dest of every live particle: its (bucket, CTA) start + the particles of the same
// bucket before it in the CTA (stable: warps in order, lanes in order)
__global__ void __launch_bounds__(MAP_THREADS) k_map_scatter(const unsigned *__restrict__ code, int n, int K0, int K1,
                                                             int K2, unsigned nbk, const unsigned *__restrict__ start,
                                                             int *__restrict__ order) {
  __shared__ unsigned wc[MAP_WARPS][MAP_MAX_BUCKETS];
  const int K[3] = {K0, K1, K2};
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int i = threadIdx.x; i < MAP_WARPS * MAP_MAX_BUCKETS; i += blockDim.x) (&wc[0][0])[i] = 0;
  __syncthreads();
  constexpr int PER_WARP = MAP_CHUNK / MAP_WARPS;
  const int wbase = blockIdx.x * MAP_CHUNK + wid * PER_WARP;
  // 1. per-warp bucket counts
  for (int s = 0; s < PER_WARP; s += 32) {
    const int p = wbase + s + lane;
    const unsigned b = p < n ? map_bucket(code[p], K, nbk) : nbk + 1;
    const unsigned peers = __match_any_sync(0xffffffffu, b);
    if (b <= nbk && lane == __ffs(peers) - 1) wc[wid][b] += __popc(peers);
    __syncwarp();
  }
  __syncthreads();
  // 2. exclusive prefix over the warps of the CTA, per bucket
  for (int b = threadIdx.x; b <= (int)nbk; b += blockDim.x) {
    unsigned off = start[(size_t)b * gridDim.x + blockIdx.x];
    for (int w = 0; w < MAP_WARPS; w++) {
      const unsigned t = wc[w][b];
      wc[w][b] = off;
      off += t;
    }
  }
  __syncthreads();
  // 3. slots in order
  for (int s = 0; s < PER_WARP; s += 32) {
    const int p = wbase + s + lane;
    const unsigned b = p < n ? map_bucket(code[p], K, nbk) : nbk + 1;
    const unsigned peers = __match_any_sync(0xffffffffu, b);
    const int leader = __ffs(peers) - 1;
    if (b < nbk) order[wc[wid][b] + __popc(peers & ((1u << lane) - 1u))] = p;
    __syncwarp();
    if (b <= nbk && lane == leader) wc[wid][b] += __popc(peers);
    __syncwarp();
  }
}

// out[q] = in[order[q]] for (q, 3) arrays
template <typename R>
__global__ void k_gather3(const int *__restrict__ order, int n, const R *__restrict__ in, R *__restrict__ out) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
    const size_t s = (size_t)3 * order[q], d = (size_t)3 * q;
    out[d] = in[s];
    out[d + 1] = in[s + 1];
    out[d + 2] = in[s + 2];
  }
}

}  // namespace pmgpu
