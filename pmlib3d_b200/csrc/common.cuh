// common.cuh -- shared helpers for the B200 particle-mesh kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
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

// a + s * c for a complex s and a real c
template <typename C, typename R> __host__ __device__ __forceinline__ C cfma_r(C s, R c, C a) {
  return mk(a.x + s.x * c, a.y + s.y * c);
}

#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000
// FP32 complex values as one packed register pair: additions and real scalings are
// single FP32x2 instructions (same rounding as the two scalar operations)
template <> __device__ __forceinline__ float2 cadd<float2>(float2 a, float2 b) { return __fadd2_rn(a, b); }
template <> __device__ __forceinline__ float2 csub<float2>(float2 a, float2 b) {
  return __ffma2_rn(b, make_float2(-1.f, -1.f), a);
}
template <> __device__ __forceinline__ float2 cscale<float2, float>(float2 a, float s) {
  return __fmul2_rn(a, make_float2(s, s));
}
template <> __device__ __forceinline__ float2 cfma_r<float2, float>(float2 s, float c, float2 a) {
  return __ffma2_rn(s, make_float2(c, c), a);
}
#endif

// kernel launch accounting (read by pmgpu_launch_count)
extern std::atomic<long long> g_launches;

// error state shared with the C ABI
void set_error(const char *caller, const char *msg);
bool cuda_ok(cudaError_t e, const char *caller);

#define PM_LAUNCHED() (::pmgpu::g_launches++)

}  // namespace pmgpu
