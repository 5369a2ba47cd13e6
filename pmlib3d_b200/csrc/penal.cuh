// penal.cuh -- iterative Brinkman penalisation on a box of the main grid (the vortex
// client's penalisation_solve, vortex_codes/vortex_penalisation/source/penalisation/
// penalisation_solve.f): mesh maps between the main cuboid and the box, the masked
// velocity updates and the vorticity increment with its force moment.  Every sum is
// taken in FP64 in a fixed order (grid-stride loops of a fixed grid, a fixed tree in
// the CTA, a fixed tree over the CTAs), so a run gives the same bits every time.
#pragma once

#include "common.cuh"

namespace pmgpu {

constexpr int PEN_THREADS = 256;
constexpr int PEN_BLOCKS = 148 * 4;  // grid of the reducing kernels (fixed: fixed summation order)
constexpr int PEN_NV = 5;            // dforce x, y, z, residual enstrophy, enstrophy

// index ranges of one mesh map (source/mesh/pmlib_mesh_map.f:85-176, one rank):
// first sent / received point as array offsets (ghosts included) and counts
struct MapBox {
  int s0[3], r0[3], n[3];
  int es[3], er[3];  // extents of the two cuboids
};

template <typename R>
__global__ void k_mesh_map(MapBox m, int nv, const R *__restrict__ src, R *__restrict__ dst, int op) {
  const long long total = (long long)m.n[0] * m.n[1] * m.n[2];
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t % m.n[0]);
    const int j = (int)((t / m.n[0]) % m.n[1]);
    const int k = (int)(t / ((long long)m.n[0] * m.n[1]));
    const size_t si = (((size_t)(m.s0[2] + k) * m.es[1] + (m.s0[1] + j)) * m.es[0] + (m.s0[0] + i)) * nv;
    const size_t di = (((size_t)(m.r0[2] + k) * m.er[1] + (m.r0[1] + j)) * m.er[0] + (m.r0[0] + i)) * nv;
    for (int c = 0; c < nv; c++) dst[di + c] = op ? dst[di + c] + src[si + c] : src[si + c];
  }
}

// CTA sum of NV doubles a thread, fixed order; thread 0 writes part[blockIdx.x * NV + v]
template <int NV>
__device__ __forceinline__ void block_sum_fixed(double (&v)[NV], double *__restrict__ part) {
  __shared__ double sh[NV][PEN_THREADS / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < NV; q++) {
    double x = v[q];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if (lane == 0) sh[q][wid] = x;
  }
  __syncthreads();
  if (threadIdx.x < NV) {
    double s = 0.0;
    for (int w = 0; w < PEN_THREADS / 32; w++) s += sh[threadIdx.x][w];
    part[(size_t)blockIdx.x * NV + threadIdx.x] = s;
  }
}

// vel_pen = solid_vel - vel_pen, vel = solid vel_pen over the box with its ghosts;
// part: sum |vel| (penalisation_solve.f:84-107)
template <typename R>
__global__ void __launch_bounds__(PEN_THREADS) k_pen_init(long long np, const R *__restrict__ solid,
                                                          const R *__restrict__ svel, R *__restrict__ vel_pen,
                                                          R *__restrict__ vel, double *__restrict__ part) {
  double acc[1] = {0.0};
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < np; q += (long long)gridDim.x * blockDim.x) {
    const R s = solid[q];
    R u[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const R vp = svel[3 * q + c] - vel_pen[3 * q + c];
      vel_pen[3 * q + c] = vp;
      u[c] = s * vp;
      vel[3 * q + c] = u[c];
    }
    acc[0] += sqrt((double)u[0] * u[0] + (double)u[1] * u[1] + (double)u[2] * u[2]);
  }
  block_sum_fixed<1>(acc, part);
}

// vel = solid (vel_pen - vel) over the box with its ghosts; part: sum |vel| (:297-312)
template <typename R>
__global__ void __launch_bounds__(PEN_THREADS) k_pen_vel(long long np, const R *__restrict__ solid,
                                                         const R *__restrict__ vel_pen, R *__restrict__ vel,
                                                         double *__restrict__ part) {
  double acc[1] = {0.0};
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < np; q += (long long)gridDim.x * blockDim.x) {
    const R s = solid[q];
    R u[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
      u[c] = s * (vel_pen[3 * q + c] - vel[3 * q + c]);
      vel[3 * q + c] = u[c];
    }
    acc[0] += sqrt((double)u[0] * u[0] + (double)u[1] * u[1] + (double)u[2] * u[2]);
  }
  block_sum_fixed<1>(acc, part);
}

template <typename R> struct PenGeom {
  int ext[3], ngl[3], nc[3];
  R c_1_2dx[3];
  R xmin[3], dx[3];
  R relax;
};

// vort += relax curl(vel) on the interior of the box (FD 2 or 4, :145-250); part:
// sum x x dvort (3), sum |dvort|^2, sum |vort|^2
template <typename R, int FD>
__global__ void __launch_bounds__(PEN_THREADS) k_pen_curl(PenGeom<R> g, const R *__restrict__ vel,
                                                          R *__restrict__ vort, double *__restrict__ part) {
  double acc[PEN_NV] = {0.0, 0.0, 0.0, 0.0, 0.0};
  const long long total = (long long)g.nc[0] * g.nc[1] * g.nc[2];
  const long long sx = 3, sy = 3LL * g.ext[0], sz = 3LL * g.ext[0] * g.ext[1];
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t % g.nc[0]);
    const int j = (int)((t / g.nc[0]) % g.nc[1]);
    const int k = (int)(t / ((long long)g.nc[0] * g.nc[1]));
    const long long m = (long long)(k + g.ngl[2]) * sz + (long long)(j + g.ngl[1]) * sy + (long long)(i + g.ngl[0]) * sx;
    // d(component c)/d(axis a)
    auto d = [&](int c, int a, long long s) -> R {
      const R *u = vel + m + c;
      if constexpr (FD == 2) {
        return (R(-1) * u[-s] + R(1) * u[s]) * g.c_1_2dx[a];
      } else {
        const R c1 = R(1) / R(6), c2 = R(4) / R(3);
        return (c1 * u[-2 * s] - c2 * u[-s] + c2 * u[s] - c1 * u[2 * s]) * g.c_1_2dx[a];
      }
    };
    const R dvdx = d(1, 0, sx), dwdx = d(2, 0, sx), dudy = d(0, 1, sy), dwdy = d(2, 1, sy), dudz = d(0, 2, sz),
            dvdz = d(1, 2, sz);
    const R d0 = g.relax * (dwdy - dvdz), d1 = g.relax * (dudz - dwdx), d2 = g.relax * (dvdx - dudy);
    R *w = vort + m;
    const R w0 = w[0] + d0, w1 = w[1] + d1, w2 = w[2] + d2;
    w[0] = w0;
    w[1] = w1;
    w[2] = w2;
    const R px = g.xmin[0] + (R(i) + R(0.5)) * g.dx[0];
    const R py = g.xmin[1] + (R(j) + R(0.5)) * g.dx[1];
    const R pz = g.xmin[2] + (R(k) + R(0.5)) * g.dx[2];
    acc[0] += (double)py * d2 - (double)pz * d1;
    acc[1] += (double)pz * d0 - (double)px * d2;
    acc[2] += (double)px * d1 - (double)py * d0;
    acc[3] += (double)d0 * d0 + (double)d1 * d1 + (double)d2 * d2;
    acc[4] += (double)w0 * w0 + (double)w1 * w1 + (double)w2 * w2;
  }
  block_sum_fixed<PEN_NV>(acc, part);
}

// out[v] = sum over CTAs of part[b * nv + v], one warp a value, fixed order
__global__ void k_pen_final(const double *__restrict__ part, int nblk, int nv, double *__restrict__ out) {
  const int lane = threadIdx.x & 31, v = threadIdx.x >> 5;
  if (v >= nv) return;
  double s = 0.0;
  for (int b = lane; b < nblk; b += 32) s += part[(size_t)b * nv + v];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if (lane == 0) out[v] = s;
}

// free-stream velocity, added as the client adds it (penalisation_solve.f:415-419:
// the third statement adds vel_inf(3) to the second component)
template <typename R>
__global__ void k_add_vel_inf(long long nm, R *__restrict__ vel, R v0, R v1, R v2) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < nm; q += (long long)gridDim.x * blockDim.x) {
    vel[3 * q] = vel[3 * q] + v0;
    vel[3 * q + 1] = (vel[3 * q + 1] + v1) + v2;
  }
}

}  // namespace pmgpu
