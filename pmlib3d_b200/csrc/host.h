// host.h -- host-side declarations shared by the library's translation units:
// error reporting, launch accounting and per-kernel timing, and the FFT pass
// launchers that are compiled in their own units (passes_*.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <vector>

#include "../../include/pmlib_gpu.h"
#include "common.cuh"
#include "solve.cuh"

namespace pmgpu {

enum KClass { KC_BIN, KC_SCAN, KC_PLACE, KC_FIXUP, KC_DEPOSIT, KC_GADD, KC_XFWD, KC_YFWD, KC_ZPASS, KC_YINV,
              KC_XINV, KC_GFILL, KC_M2P, KC_DERIV, KC_ADVANCE, KC_MAP, KC_OTHER, KC_N };

// brackets one launch with CUDA events on its stream while timing is enabled
struct KTimer {
  int cls;
  cudaStream_t st;
  cudaEvent_t a = nullptr, b = nullptr;
  KTimer(int c, cudaStream_t s);
  ~KTimer();
};

#define CK(expr, caller)                         \
  do {                                           \
    if (!::pmgpu::cuda_ok((expr), (caller))) {   \
      return -1;                                 \
    }                                            \
  } while (0)
#define CKL(caller) CK(cudaGetLastError(), caller)

int num_sms();
// Raises a kernel's maximum dynamic shared memory to `bytes` if it is below: the
// attribute only grows, and it is set at most once per size increase and device, so
// launches of the same kernel on other streams are not held up by setting it again.
int smem_attr(const void *func, size_t bytes, const char *caller);

// shared-memory budget of one persistent pass CTA
constexpr size_t PASS_SMEM_BUDGET = 220 * 1024;

static inline size_t tw_bytes(int ntw, size_t csize) { return (size_t)((ntw + 7) & ~7) * csize; }

// kx tile of the Stockham y / z passes: the largest of 8, 4, 2, 1 whose three
// buffers fit (FP32 needs an even line count: two lines per 16-byte vector)
static inline int pick_tk(int n, int nc, size_t csize, int ntw) {
  for (int tk = 8; tk >= 1; tk /= 2) {
    if (csize == 8 && (nc * tk) % 2) continue;
    if (tw_bytes(ntw, csize) + 3 * (size_t)nc * tk * n * csize <= PASS_SMEM_BUDGET) return tk;
  }
  return 0;
}
static inline size_t lines_smem(int n, int nc, int tk, size_t csize, int ntw) {
  return tw_bytes(ntw, csize) + 3 * (size_t)nc * tk * n * csize;
}
// register engine: twiddles w_m^q + position table + wavenumbers (+ Bluestein chirp
// and spectrum) + one tile buffer; n = line length, m = transform length (m = n
// unless Bluestein)
static inline size_t reg_smem(int n, int m, int nc, int tk, size_t csize) {
  const size_t blue = m != n ? (((size_t)(n + m) * csize + 15) & ~(size_t)15) : 0;
  return (((size_t)m * csize + 15) & ~(size_t)15) + (((size_t)n * 4 + 15) & ~(size_t)15) +
         (((size_t)n * csize / 2 + 15) & ~(size_t)15) + blue + (size_t)nc * tk * m * csize;
}
// shared memory per CTA that lets the register-engine kernels run as many CTAs per
// SM as their register budget allows (FP32: 3, FP64: 2; 228 KB per SM)
static inline size_t reg_budget(size_t rsize) { return rsize == 4 ? (size_t)74 * 1024 : (size_t)112 * 1024; }
// the wide-radix FP32 kernels run two CTAs per SM
static inline size_t reg_budget_wide() { return (size_t)112 * 1024; }
// kx tile of the register engine: within the budget if possible, else one CTA per SM
static inline int pick_tk_reg(int n, int m, int nc, size_t csize, int Hp, size_t budget1) {
  for (size_t budget : {budget1, PASS_SMEM_BUDGET})
    for (int tk = 8; tk >= 1; tk /= 2) {
      if (Hp % tk) continue;
      if (reg_smem(n, m, nc, tk, csize) <= budget) return tk;
    }
  return 0;
}
// rows per tile of the register-engine x passes (table bytes + staging + buffer),
// two CTAs per SM if possible
static inline size_t rx_smem(int N, int m, int H, int P0, int Hp, int nc, int rb, size_t csize, size_t rsize,
                             bool inverse) {
  const size_t blue = m != N ? (((size_t)(N + m) * csize + 15) & ~(size_t)15) : 0;
  const size_t tabs = (((size_t)m * csize + 15) & ~(size_t)15) + (((size_t)H * csize + 15) & ~(size_t)15) +
                      (((size_t)N * 4 + 15) & ~(size_t)15) + blue;
  const size_t stage = inverse ? (size_t)rb * Hp * nc * csize : (((size_t)rb * P0 * nc * rsize + 15) / 16) * 16;
  return tabs + stage + (size_t)nc * rb * m * csize;
}
static inline int pick_rb_reg(int N, int m, int H, int P0, int Hp, int nc, size_t csize, size_t rsize, bool inverse,
                              size_t budget1) {
  for (size_t budget : {budget1, PASS_SMEM_BUDGET})
    for (int rb = 16; rb >= 1; rb--)
      if (rx_smem(N, m, H, P0, Hp, nc, rb, csize, rsize, inverse) <= budget) return rb;
  return 0;
}

// rows per tile of the x passes
static inline int pick_rb(int n2, int P0, int Hp, int nc, size_t csize, size_t rsize, int ntw, bool inverse) {
  for (int rb = 8; rb >= 1; rb--) {
    if (csize == 8 && (nc * rb) % 2) continue;
    const size_t stage = inverse ? (size_t)rb * Hp * nc * csize : (((size_t)rb * P0 * nc * rsize + 15) / 16) * 16;
    if (tw_bytes(ntw, csize) + stage + 2 * (size_t)nc * rb * n2 * csize <= PASS_SMEM_BUDGET) return rb;
  }
  return 0;
}

// ---- batches of patches: one launch per pass family (x forward, y forward, z pass,
// y inverse, x inverse) over the tiles of every patch, then the periodic ghost fill
// per axis.  The descriptors are built on the host once (batch_layout) and live in
// device memory; a solve passes the patches' arrays by value (BatchIo).
struct BatchPassInfo {
  size_t desc_off;  // byte offset of the pass's descriptors
  int nitems, chunk, wide;
  size_t smem;
};
struct BatchGhostInfo {
  size_t desc_off;
  int npatch;
  long long total;
};
struct BatchLayout {
  int npatch = 0;
  BatchPassInfo pass[5];
  BatchGhostInfo ghost[3];
  size_t bytes = 0;  // descriptor bytes
};

// ---- FFT passes (passes.cuh, instantiated per precision and component count)
// x then y forward: real cuboid (component stride cs) -> X -> Y
template <typename R, int NC>
int fwd_xy(SolveGeom<R> &g, const R *in, typename cplx_t<R>::type *X, typename cplx_t<R>::type *Y, cudaStream_t st,
           const char *caller, int cs = NC);
// z pass on rows_y spectrum rows: Z_VEL / Z_VORT / Z_VECPOT / Z_REGULARISE / Z_FORWARD
template <typename R, int NC>
int zpass(SolveGeom<R> &g, const typename cplx_t<R>::type *in, typename cplx_t<R>::type *out, int mode, int reproj,
          int use_zeta, int rows_y, cudaStream_t st, const char *caller);
// y then x inverse into the cuboid (periodic ghosts filled when `ghosts`)
template <typename R, int NC>
int inv_yx(SolveGeom<R> &g, const pmgpu_topo *topo, typename cplx_t<R>::type *Y, typename cplx_t<R>::type *X, R *out,
           cudaStream_t st, const char *caller, int cs = NC, bool ghosts = true);

// one pass along y (forward X -> Y, or inverse Y -> X)
// fills `desc` (host bytes) and `lay` for the velocity solve of n patches of
// geometries g[i] with work spectra X[i], Y[i] (run_solve's layout); -1 if a patch
// needs a pass the batched kernels do not run (the Stockham fallback)
template <typename R, int NC>
int batch_layout(int n, const SolveGeom<R> *g, typename cplx_t<R>::type *const *X,
                 typename cplx_t<R>::type *const *Y, const pmgpu_topo *const *topo, std::vector<unsigned char> &desc,
                 BatchLayout &lay, const char *caller);
// queues the batched solve: d_desc holds the descriptors, counters 5 zeroed words
template <typename R, int NC>
int batch_launch(const BatchLayout &lay, const void *d_desc, unsigned *counters, const void *const *vort,
                 void *const *vel, cudaStream_t st, const char *caller);
template <typename R, int NC>
int ypass(SolveGeom<R> &g, const typename cplx_t<R>::type *X, typename cplx_t<R>::type *Y, int inverse,
          cudaStream_t st, const char *caller);

// each pass unit holds its own copy of the DFT constant tables
int upload_cs_f32_1(const void *t32, const void *t64);
int upload_cs_f32_3(const void *t32, const void *t64);
int upload_cs_f64_1(const void *t32, const void *t64);
int upload_cs_f64_3(const void *t32, const void *t64);
int upload_cs_ct_f32(const void *t32, const void *t64);
int upload_cs_ct_f64(const void *t32, const void *t64);

// launches of the y / z line passes take a compile-time-plan kernel when one is
// compiled for the plan and kx tile (0: always the run-time engine)
extern int g_fft_ct;

}  // namespace pmgpu
