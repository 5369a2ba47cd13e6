// common.cuh -- shared helpers for the B200 particle-mesh kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <string>

namespace pmgpu {

// complex type per precision: float2 / double2 (8 / 16 bytes, naturally aligned)
template <typename R> struct cplx_t;
template <> struct cplx_t<float> { typedef float2 type; };
template <> struct cplx_t<double> { typedef double2 type; };

template <typename C> struct real_of;
template <> struct real_of<float2> { typedef float type; };
template <> struct real_of<double2> { typedef double type; };

__host__ __device__ __forceinline__ float2 mk(float a, float b) { return make_float2(a, b); }
__host__ __device__ __forceinline__ double2 mk(double a, double b) { return make_double2(a, b); }

template <typename C> __host__ __device__ __forceinline__ C cadd(C a, C b) { return mk(a.x + b.x, a.y + b.y); }
template <typename C> __host__ __device__ __forceinline__ C csub(C a, C b) { return mk(a.x - b.x, a.y - b.y); }
template <typename C> __host__ __device__ __forceinline__ C cmul(C a, C b) {
  return mk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
template <typename C> __host__ __device__ __forceinline__ C cmulc(C a, C b) {
  return mk(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
template <typename C, typename R> __host__ __device__ __forceinline__ C cscale(C a, R s) {
  return mk(a.x * s, a.y * s);
}
// multiply by -i (forward) or +i (inverse)
template <int DIR, typename C> __host__ __device__ __forceinline__ C cmul_mi(C a) {
  return DIR > 0 ? mk(-a.y, a.x) : mk(a.y, -a.x);
}
template <typename C> __host__ __device__ __forceinline__ C cconj(C a) { return mk(a.x, -a.y); }

// kernel launch accounting (read by pmgpu_launch_count)
extern long long g_launches;

// error state shared with the C ABI
void set_error(const char *caller, const char *msg);
bool cuda_ok(cudaError_t e, const char *caller);

#define PM_LAUNCHED() (::pmgpu::g_launches++)

}  // namespace pmgpu
