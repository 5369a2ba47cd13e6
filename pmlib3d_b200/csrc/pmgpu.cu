// pmgpu.cu -- C ABI of the B200 particle-mesh step: plans, particle kernels,
// Green's function set-up and the solve drivers.  The FFT pass kernels and their
// launchers are compiled in the passes_*.cu units (no relocatable device code:
// every unit registers its own kernels).
#include "../../include/pmlib_gpu.h"

#include "common.cuh"
#include "fft.cuh"
#include "green.cuh"
#include "host.h"
#include "particles.cuh"
#include "advance.cuh"
#include "penal.cuh"
#include "solve.cuh"

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <tuple>
#include <mutex>
#include <string>
#include <vector>

namespace pmgpu {

std::atomic<long long> g_launches{0};

// ------------------------------------------------------------------ per-kernel timing
// When enabled, every launch of the library is bracketed by CUDA events on its
// stream; pmgpu_timing_get sums the elapsed times per kernel class.
static const char *kc_names[KC_N] = {"bin", "scan", "place", "fixup", "deposit", "ghost_add",
                                     "x_fwd", "y_fwd", "z_pass", "y_inv", "x_inv", "ghost_fill", "m2p",
                                     "deriv_vorticity", "advance", "map", "other"};
static bool g_timing = false;
static std::mutex g_time_mu;  // the pending events (launches of several threads)
struct PendingEv {
  int cls;
  cudaEvent_t a, b;
};
static std::vector<PendingEv> g_pending;
static double g_kms[KC_N];
static long long g_kn[KC_N];

KTimer::KTimer(int c, cudaStream_t s) : cls(c), st(s) {
  if (g_timing) {
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a, st);
  }
}
KTimer::~KTimer() {
  if (g_timing && a) {
    cudaEventRecord(b, st);
    std::lock_guard<std::mutex> lk(g_time_mu);
    g_pending.push_back({cls, a, b});
  }
}
static void timing_collect() {
  std::lock_guard<std::mutex> lk(g_time_mu);
  for (auto &p : g_pending) {
    float ms = 0.f;
    cudaEventSynchronize(p.b);
    cudaEventElapsedTime(&ms, p.a, p.b);
    g_kms[p.cls] += ms;
    g_kn[p.cls] += 1;
    cudaEventDestroy(p.a);
    cudaEventDestroy(p.b);
  }
  g_pending.clear();
}

// The last error of the calling thread (plan set-up may run on another thread than
// the solves, see g_setup_mu).
static thread_local char g_err[512] = "";
// Entry points serialise on g_mu, except plan creation (pmgpu_poisson_setup*,
// pmgpu_batch_create) and the schedule table (pmgpu_fft_tune / _tuned /
// _set_schedule), which serialise on g_setup_mu: a plan can be set up while another
// thread queues solves of other plans.  The state both sides share is guarded on
// its own (device set-up, timing events, the launch counter, allocation injection).
static std::mutex g_mu;
static std::mutex g_setup_mu;
static std::mutex g_dev_mu;

// source/pmlib_write.f:40-48 format for rank 0
void set_error(const char *caller, const char *msg) {
  snprintf(g_err, sizeof(g_err), "[%04d](%s) : %s", 0, caller, msg);
  printf("%s\n", g_err);
  fflush(stdout);
}

bool cuda_ok(cudaError_t e, const char *caller) {
  if (e == cudaSuccess) return true;
  set_error(caller, cudaGetErrorString(e));
  return false;
}

// ------------------------------------------------------------------ per-device tables
static bool g_dev_ready[128];
// plans made while set use the out-of-place Stockham passes along y and z only
static int g_force_stockham = 0;

static int noalloc_reserve(int dev, const char *caller);

static int ensure_device(const char *caller) {
  int dev = 0;
  CK(cudaGetDevice(&dev), caller);
  std::lock_guard<std::mutex> lk(g_dev_mu);
  if (dev >= 0 && dev < 128 && g_dev_ready[dev]) return 0;
  if (noalloc_reserve(dev, caller)) return -1;
  static float t32[CS_R][CS_M][2];
  static double t64[CS_R][CS_M][2];
  const long double twopi = 2.0L * acosl(-1.0L);
  for (int R = 1; R < CS_R; R++)
    for (int m = 0; m < CS_M; m++) {
      long double a = (m < R) ? twopi * (long double)m / (long double)R : 0.0L;
      t64[R][m][0] = (double)cosl(a);
      t64[R][m][1] = (double)sinl(a);
      t32[R][m][0] = (float)cosl(a);
      t32[R][m][1] = (float)sinl(a);
    }
  if (upload_cs_f32_1(t32, t64) || upload_cs_f32_3(t32, t64) || upload_cs_f64_1(t32, t64) ||
      upload_cs_f64_3(t32, t64) || upload_cs_ct_f32(t32, t64) || upload_cs_ct_f64(t32, t64)) {
    set_error(caller, "could not upload the DFT constant tables.");
    return -1;
  }
  {
    // the Green's-function set-up takes its temporaries from the device's stream-
    // ordered pool; keep freed blocks in the pool instead of returning them to the
    // driver at every synchronisation (remapping gigabytes per plan)
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
      unsigned long long thr = ~0ull;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
  }
  if (dev >= 0 && dev < 128) g_dev_ready[dev] = true;
  return 0;
}

// ------------------------------------------------------------------ device buffers
// Device buffers come from the device's stream-ordered pool (freed blocks stay in
// the pool): allocating or freeing never synchronises the whole device, so plans can
// be created and destroyed while other streams run.  A buffer is freed in order on
// the legacy stream; its owner frees it only when no work using it is in flight.
// Injected allocation failure (pmgpu_inject_alloc_failure): the allocation that
// brings the countdown to zero reports cudaErrorMemoryAllocation; -1 = off.
static std::atomic<long long> g_fail_alloc{-1};

struct DevBuf {
  void *p = nullptr;
  size_t cap = 0;
  bool fixed = false;  // a view of preallocated memory: never allocates or frees
  bool stream_ordered = true;
  int ensure(size_t bytes, const char *caller) {
    if (bytes <= cap && p) return 0;
    if (fixed) {
      set_error(caller, "scratch size exceeds the fixed device scratch area.");
      return -1;
    }
    if (p) {
      if (stream_ordered) cudaFreeAsync(p, 0);
      else cudaFree(p);
    }
    p = nullptr;
    cap = 0;
    size_t b = std::max<size_t>(bytes, 256);
    if (g_fail_alloc.load() >= 0 && g_fail_alloc.fetch_sub(1) == 0) CK(cudaErrorMemoryAllocation, caller);
    if (stream_ordered) {
      CK(cudaMallocAsync(&p, b, 0), caller);
      CK(cudaStreamSynchronize(0), caller);  // usable from every stream from here on
    } else {
      CK(cudaMalloc(&p, b), caller);
    }
    cap = b;
    return 0;
  }
  void release() {
    if (p && !fixed) {
      if (stream_ordered) cudaFreeAsync(p, 0);
      else cudaFree(p);
    }
    p = nullptr;
    cap = 0;
  }
  template <typename T> T *as() const { return reinterpret_cast<T *>(p); }
};

// ------------------------------------------------------------------ FFT plans
typedef std::complex<long double> cld;

static bool supported_radix(int r) {
  return r == 2 || r == 3 || r == 4 || r == 5 || r == 7 || r == 8 || r == 11 || r == 13 || r == 16 || r == 17;
}

// radices: powers of two as 16, then 8/4/2; the other primes ascending
static bool make_fft(int n, int extM, FftDesc &d, std::vector<cld> &tw) {
  if (n < 1) return false;
  std::vector<int> pf;
  int m = n;
  for (int p = 2; (long long)p * p <= m; p++)
    while (m % p == 0) {
      pf.push_back(p);
      m /= p;
    }
  if (m > 1) pf.push_back(m);
  int c2 = (int)std::count(pf.begin(), pf.end(), 2);
  std::vector<int> rad;
  while (c2 >= 4) {
    rad.push_back(16);
    c2 -= 4;
  }
  if (c2 == 3) rad.push_back(8);
  else if (c2 == 2) rad.push_back(4);
  else if (c2 == 1) rad.push_back(2);
  std::vector<int> odd;
  for (int p : pf)
    if (p != 2) odd.push_back(p);
  std::sort(odd.begin(), odd.end());
  for (int p : odd) rad.push_back(p);
  if ((int)rad.size() > FFT_MAXPASS) return false;
  memset(&d, 0, sizeof(d));
  d.n = n;
  d.npass = (int)rad.size();
  const long double twopi = 2.0L * acosl(-1.0L);
  tw.clear();
  long long ns = 1;
  for (int p = 0; p < d.npass; p++) {
    const int R = rad[p];
    d.rad[p] = R;
    d.ns[p] = (int)ns;
    d.twoff[p] = (int)tw.size();
    const long long den = ns * R;
    for (long long k = 0; k < ns; k++)
      for (int r = 1; r < R; r++) {
        const long long q = (k * r) % den;
        const long double a = twopi * (long double)q / (long double)den;
        tw.push_back(cld(cosl(a), -sinl(a)));
      }
    d.rootoff[p] = (int)tw.size();
    if (!supported_radix(R))
      for (int q = 0; q < R; q++) {
        const long double a = twopi * (long double)q / (long double)R;
        tw.push_back(cld(cosl(a), -sinl(a)));
      }
    ns *= R;
  }
  d.ntw = (int)tw.size();
  d.extoff = 0;
  d.next = 0;
  if (extM > 0) {
    d.extoff = (int)tw.size();
    d.next = extM / 2 + 1;
    for (int k = 0; k < d.next; k++) {
      const long double a = twopi * (long double)k / (long double)extM;
      tw.push_back(cld(cosl(a), -sinl(a)));
    }
  }
  return true;
}

template <typename R> static int upload_tw(const std::vector<cld> &tw, DevBuf &buf, const char *caller) {
  typedef typename cplx_t<R>::type C;
  std::vector<C> h(tw.size() + 1);
  for (size_t i = 0; i < tw.size(); i++) h[i] = mk((R)tw[i].real(), (R)tw[i].imag());
  if (buf.ensure(sizeof(C) * h.size(), caller)) return -1;
  CK(cudaMemcpy(buf.p, h.data(), sizeof(C) * h.size(), cudaMemcpyHostToDevice), caller);
  return 0;
}

// ------------------------------------------------------------------ register-engine plans
// Factor n into at most three register radices; the score models per-point work
// (a shared-memory round trip + twiddles per phase, plus the DFT of the radix).
static double radix_cost(int r) {
  switch (r) {
    case 2: return 1.0;
    case 3: return 1.3;
    case 4: return 1.1;
    case 5: return 1.7;
    case 6: return 1.4;
    case 7: return 2.3;
    case 8: return 1.2;
    case 9: return 1.7;
    case 10: return 1.6;
    case 11: return 3.2;
    case 12: return 1.5;
    case 13: return 3.6;
    case 16: return 2.3;  // 16 and 17 exceed the register budget of two vectors a thread: spills
    case 17: return 5.4;
    default: return 1e9;
  }
}

// a plan from an explicit radix sequence (outermost first)
static void regplan_from(int n, const int *r, int np, RegPlan &pl) {
  memset(&pl, 0, sizeof(pl));
  pl.n = n;
  pl.np = np;
  int B = n;
  for (int p = 0; p < np; p++) {
    pl.rad[p] = r[p];
    pl.blk[p] = B;
    pl.str[p] = B / r[p];
    pl.twm[p] = n / B;
    pl.dstr[p] = make_fastdiv((unsigned)pl.str[p]);
    B /= r[p];
  }
}

// radix sequences of at most three register radices whose product is n, best model
// score first
struct RadixSeq {
  int np;
  int r[3];
  double cost;
};
static std::vector<RadixSeq> regplan_candidates(int n) {
  static const int S[] = {16, 17, 13, 12, 11, 10, 9, 8, 7, 6, 5, 4, 3, 2};
  std::vector<RadixSeq> out;
  auto add = [&](int np, int a, int b, int c) {
    RadixSeq q;
    q.np = np;
    q.r[0] = a;
    q.r[1] = b;
    q.r[2] = c;
    q.cost = 0.0;
    for (int i = 0; i < np; i++) q.cost += 1.5 + radix_cost(q.r[i]);
    if (a % 2) q.cost += 0.5;  // the zero half of a padded line is skipped only with an even first radix
    out.push_back(q);
  };
  for (int a : S) {
    if (n % a) continue;
    const int n1 = n / a;
    if (n1 == 1) {
      add(1, a, 0, 0);
      continue;
    }
    for (int b : S) {
      if (n1 % b) continue;
      const int n2 = n1 / b;
      if (n2 == 1) add(2, a, b, 0);
      else if (reg_radix(n2)) add(3, a, b, n2);
    }
  }
  std::stable_sort(out.begin(), out.end(), [](const RadixSeq &x, const RadixSeq &y) { return x.cost < y.cost; });
  return out;
}

// two-phase sequences with at least one wide composite radix (the wide FP32 kernel
// variant), fewest points per thread first; only the autotuner tries them
static std::vector<RadixSeq> regplan_candidates_wide(int n) {
  static const int S[] = {24, 22, 20, 18, 17, 16, 13, 12, 11, 10, 9, 8};
  std::vector<RadixSeq> out;
  for (int a : S) {
    if (n % a) continue;
    const int b = n / a;
    if (!(reg_radix(b) || reg_radix_wide(b)) || !(reg_radix_wide(a) || reg_radix_wide(b))) continue;
    RadixSeq q;
    q.np = 2;
    q.r[0] = a;
    q.r[1] = b;
    q.r[2] = 0;
    q.cost = (double)std::max(a, b) + (a % 2 ? 0.5 : 0.0);
    out.push_back(q);
  }
  std::stable_sort(out.begin(), out.end(), [](const RadixSeq &x, const RadixSeq &y) { return x.cost < y.cost; });
  return out;
}

// The same radices ordered for the fused middle of the z pass: the smallest radix
// that the registers take last, an even radix first where there is one (the zero half
// of a padded line is then skipped); any order of the radices is a valid plan.
static RadixSeq z_order(const RadixSeq &c, int rsize) {
  RadixSeq q = c;
  if (c.np < 2) return q;
  const int lim = rsize == 4 ? 8 : 6;
  int best = -1;
  for (int i = 0; i < c.np; i++)
    if (c.r[i] <= lim && (best < 0 || c.r[i] < c.r[best])) best = i;
  if (best < 0) return q;
  int rest[2], nr = 0;
  for (int i = 0; i < c.np; i++)
    if (i != best) rest[nr++] = c.r[i];
  if (nr == 2 && rest[0] % 2 && !(rest[1] % 2)) std::swap(rest[0], rest[1]);
  for (int i = 0; i < nr; i++) q.r[i] = rest[i];
  q.r[nr] = c.r[best];
  return q;
}

static bool make_regplan(int n, RegPlan &pl) {
  const std::vector<RadixSeq> c = regplan_candidates(n);
  if (c.empty()) return false;
  regplan_from(n, c[0].r, c[0].np, pl);
  return true;
}

// Autotuned schedules: (length, precision, axis) -> radix sequence and kx tile, the
// fastest measured forward pass among the candidates (process-wide, filled when
// plans are created while tuning is on).
struct TunedSchedule {
  int np;
  int r[3];
  int tk;
  double ms;
};
static std::map<std::tuple<int, int, int>, TunedSchedule> g_tuned;
static int g_tune = 0;

// position -> frequency index of the digit-reversed output of a plan
static std::vector<int> regplan_positions(const RegPlan &pl) {
  std::vector<int> k(pl.n);
  for (int q = 0; q < pl.n; q++) {
    int rem = q, mul = 1, f = 0;
    for (int p = 0; p < pl.np; p++) {
      const int sub = pl.blk[p] / pl.rad[p];
      const int d = rem / sub;
      rem -= d * sub;
      f += mul * d;
      mul *= pl.rad[p];
    }
    k[q] = f;
  }
  return k;
}

// forward DFT in long double, any length whose prime factors are small (mixed radix,
// decimation in time, recursive); used for the Bluestein spectra
static void host_dft(std::vector<cld> &a) {
  const size_t n = a.size();
  if (n <= 1) return;
  size_t p = 2;
  while (p * p <= n && n % p) p++;
  if (n % p) p = n;
  const size_t m = n / p;
  std::vector<std::vector<cld>> sub(p, std::vector<cld>(m));
  for (size_t j = 0; j < m; j++)
    for (size_t r = 0; r < p; r++) sub[r][j] = a[j * p + r];
  if (m > 1)
    for (size_t r = 0; r < p; r++) host_dft(sub[r]);
  const long double twopi = 2.0L * acosl(-1.0L);
  for (size_t k = 0; k < n; k++) {
    cld acc(0.0L, 0.0L);
    for (size_t r = 0; r < p; r++) {
      const long double ang = -twopi * (long double)((r * k) % n) / (long double)n;
      acc += sub[r][k % m] * cld(cosl(ang), sinl(ang));
    }
    a[k] = acc;
  }
}

// Bluestein plan for a line of length n: the convolution length m is the smallest
// m >= 2n - 1 with a register plan
static bool make_bluestein(int n, RegPlan &pl) {
  for (int m = 2 * n - 1; m <= 4 * n; m++)
    if (make_regplan(m, pl)) {
      pl.bl = 1;
      pl.bn = n;
      return true;
    }
  return false;
}

// chirp c[j] = exp(-i pi j^2 / n) and B = DFT_m of conj(c) wrapped (B[q] at the
// plan's position q)
template <typename C, typename R>
static void bluestein_tables(const RegPlan &pl, std::vector<C> &chirp, std::vector<C> &bpos) {
  const int n = pl.bn, m = pl.n;
  const long double pi = acosl(-1.0L);
  std::vector<cld> c(n), b(m, cld(0.0L, 0.0L));
  for (int j = 0; j < n; j++) {
    const long long q = ((long long)j * j) % (2LL * n);
    const long double a = -pi * (long double)q / (long double)n;
    c[j] = cld(cosl(a), sinl(a));
  }
  b[0] = std::conj(c[0]);
  for (int j = 1; j < n; j++) b[j] = b[m - j] = std::conj(c[j]);
  host_dft(b);
  const std::vector<int> kp = regplan_positions(pl);
  chirp.resize(n);
  bpos.resize(m);
  for (int j = 0; j < n; j++) chirp[j] = mk((R)c[j].real(), (R)c[j].imag());
  for (int q = 0; q < m; q++) bpos[q] = mk((R)b[kp[q]].real(), (R)b[kp[q]].imag());
}

static std::mutex g_attr_mu;
static std::map<std::pair<int, const void *>, size_t> g_smem_attr;
int smem_attr(const void *func, size_t bytes, const char *caller) {
  int dev = 0;
  CK(cudaGetDevice(&dev), caller);
  std::lock_guard<std::mutex> lk(g_attr_mu);
  size_t &cur = g_smem_attr[std::make_pair(dev, func)];
  if (bytes <= cur) return 0;
  CK(cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes), caller);
  cur = bytes;
  return 0;
}

static int g_nsm = 0;
int num_sms() {
  if (g_nsm == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&g_nsm, cudaDevAttrMultiProcessorCount, dev);
    if (g_nsm <= 0) g_nsm = 148;
  }
  return g_nsm;
}

}  // namespace pmgpu

using namespace pmgpu;

// ------------------------------------------------------------------ plan object
struct Geometry {
  int ext[3], off[3], P[3], M[3], H, Hp, N2;
  int allper;
};

// streams, events and double-buffered particle arrays of pmgpu_step_many
struct StepPipe {
  cudaStream_t s[3] = {nullptr, nullptr, nullptr};  // host->device, compute, device->host
  cudaEvent_t h2d[2] = {nullptr, nullptr}, comp[2] = {nullptr, nullptr}, d2h[2] = {nullptr, nullptr};
  DevBuf pos[2], val[2], out[2];
  ~StepPipe() {
    for (int i = 0; i < 3; i++)
      if (s[i]) cudaStreamSynchronize(s[i]);
    for (int i = 0; i < 2; i++) {
      pos[i].release();
      val[i].release();
      out[i].release();
      for (cudaEvent_t e : {h2d[i], comp[i], d2h[i]})
        if (e) cudaEventDestroy(e);
    }
    for (int i = 0; i < 3; i++)
      if (s[i]) cudaStreamDestroy(s[i]);
  }
};

struct pmgpu_plan {
  int prec;
  int green_mode = 0;  // 0: pmlib_poisson_setup's kernel; 1 / 2: the ppf / pff validation programs' kernels
  int pff_kx0 = 0;     // pff: treatment of the k_x = 0 plane (0 as written, 1 two-dimensional kernel)
  StepPipe pipe;
  pmgpu_patch patch;
  pmgpu_topo topo;
  pmgpu_params par;
  Geometry g;
  FftDesc fx, fy, fz;
  DevBuf twx, twy, twz;
  DevBuf kxt, kyt, kzt;
  DevBuf green;  // view of green_own (shared between plans of the same grid)
  std::shared_ptr<DevBuf> green_own;
  int gM1, gM2;
  double eps;
  DevBuf X, Y, Y2, Y3;
  // register-engine plans along y and z (in-place, digit-reversed spectra)
  int rx_ok, ry_ok, rz_ok;
  RegPlan rx, ry, rz;
  int tky = 0, tkz = 0;  // tuned kx tiles (0: chosen by shared memory)
  DevBuf rtwx, rtwy, rtwz, yk, zk, rextx, xpos;
  DevBuf rchx, rchy, rchz, rbx, rby, rbz;  // Bluestein chirps and spectra
  // the register-engine tables above are views of device tables shared by the plans
  // of the same transform length, precision and schedule; these keep them alive
  std::vector<std::shared_ptr<DevBuf>> tab_keep;
  DevBuf mesh_w, mesh_u, mesh_a, mesh_b;
  DevBuf h_pos, h_val, h_out;  // device mirrors used by host-pointer calls
  // particle scratch
  DevBuf key, val, key2, val2, counts, start, spart, hist;
  const int *perm;  // sorted order of the last deposit (device)
  int perm_n;
  ~pmgpu_plan() {
    DevBuf *bs[] = {&twx, &twy, &twz, &kxt, &kyt, &kzt, &X, &Y, &Y2, &Y3, &mesh_w, &mesh_u,
                    &mesh_a, &mesh_b, &h_pos, &h_val, &h_out, &key, &val, &key2, &val2, &counts,
                    &start, &spart, &hist, &rtwx, &rtwy, &rtwz, &yk, &zk, &rextx, &xpos,
                    &rchx, &rchy, &rchz, &rbx, &rby, &rbz};
    for (DevBuf *b : bs) b->release();
  }
};

namespace pmgpu {

// particle scratch shared by calls that have no plan
struct Scratch {
  DevBuf key, val, key2, val2, counts, start, spart, hist;
  DevBuf a, b, c, d, e, f, g, h;
  DevBuf diag;  // diagnostics partial sums
  DevBuf adv_code, adv_stats, adv_cnt, adv_start, adv_ord, adv_tmp;  // particle advance and map
  DevBuf pen_part, pen_out;                                           // penalisation sums
};
static Scratch &scratch() {
  static Scratch s;
  return s;
}

static size_t mesh_points(const pmgpu_topo *t) {
  size_t n = 1;
  for (int d = 0; d < 3; d++) n *= (size_t)(t->ncell[d] + t->nghost[2 * d] + t->nghost[2 * d + 1]);
  return n;
}

// ------------------------------------------------------------------ scans
static int exclusive_scan(const unsigned *in, unsigned *out, size_t n, DevBuf &part, cudaStream_t st,
                          const char *caller) {
  const size_t nb = (n + SCAN_TILE - 1) / SCAN_TILE;
  if (part.ensure(sizeof(unsigned) * (nb + 1), caller)) return -1;
  { KTimer kt_(KC_SCAN, st); k_scan_reduce<<<(unsigned)nb, SCAN_THREADS, 0, st>>>(in, n, part.as<unsigned>()); }
  PM_LAUNCHED();
  { KTimer kt_(KC_SCAN, st); k_scan_partials<<<1, SCAN_THREADS, 0, st>>>(part.as<unsigned>(), (int)nb); }
  PM_LAUNCHED();
  { KTimer kt_(KC_SCAN, st); k_scan_apply<<<(unsigned)nb, SCAN_THREADS, 0, st>>>(in, n, part.as<unsigned>(), out); }
  PM_LAUNCHED();
  CKL(caller);
  return 0;
}

template <typename R> static PartGeom<R> part_geom(const pmgpu_topo *t, int W) {
  PartGeom<R> g;
  memset(&g, 0, sizeof(g));
  unsigned long long nbins = 1;
  for (int e = 0; e < 3; e++) {
    g.ext[e] = t->ncell[e] + t->nghost[2 * e] + t->nghost[2 * e + 1];
    g.lo[e] = 1 - t->nghost[2 * e];
    g.nint[e] = t->ncell[e];
    g.nglo[e] = t->nghost[2 * e];
    g.bclo[e] = t->bound_cond[2 * e];
    g.bchi[e] = t->bound_cond[2 * e + 1];
    const int off = (W == 4) ? 1 : 2;
    g.blo[e] = g.lo[e] - (W - 1 - off);
    g.nb[e] = g.ext[e] + W - 1;
    nbins *= (unsigned long long)g.nb[e];
    g.xmin[e] = (R)t->xmin[e];
    g.xmax[e] = (R)t->xmax[e];
    g.dx[e] = (R)t->dx[e];
    g.c1dx[e] = R(1) / (R)t->dx[e];
  }
  g.nbins = (unsigned)nbins;
  return g;
}

struct PartScratchRefs {
  DevBuf *key, *val, *key2, *val2, *counts, *start, *spart, *hist;
};

// Bin keys and the stable sort of the particles by bin (the first half of P2M): on
// return s.key holds every particle's bin key (nbins for particles P2M skips) and
// s.val2 the sorted order, s.start the bin starts (nbins + 1 entries).
template <typename R>
static int run_bin_sort(const pmgpu_topo *t, int order, const R *pos, int n, PartScratchRefs s, cudaStream_t st,
                        const char *caller) {
  const int W = (order == 3) ? 4 : 6;
  PartGeom<R> g = part_geom<R>(t, W);
  const unsigned long long nb_total = (unsigned long long)g.nb[0] * g.nb[1] * g.nb[2];
  if (nb_total >= 0xFFFFFFF0ull) {
    set_error(caller, "Mesh too large for 32-bit bin keys.");
    return -1;
  }
  const size_t nn = (size_t)std::max(n, 1);
  if (s.key->ensure(sizeof(unsigned) * nn, caller) || s.val->ensure(sizeof(unsigned) * nn, caller) ||
      s.key2->ensure(sizeof(int) * nn, caller) || s.val2->ensure(sizeof(int) * nn, caller) ||
      s.hist->ensure(sizeof(unsigned) * (nn / (FIX_SMALL + 1) + 2), caller) ||
      s.counts->ensure(sizeof(unsigned) * (g.nbins + 1), caller) ||
      s.start->ensure(sizeof(unsigned) * (g.nbins + 1), caller))
    return -1;
  // counting sort by bin: provisional slots, bin starts, placement, stable fix-up
  CK(cudaMemsetAsync(s.counts->p, 0, sizeof(unsigned) * (g.nbins + 1), st), caller);
  CK(cudaMemsetAsync(s.hist->p, 0, sizeof(unsigned), st), caller);
  unsigned *keys = s.key->as<unsigned>(), *ranks = s.val->as<unsigned>();
  int *perm = s.val2->as<int>();
  if (n > 0) {
    const int nblk = std::min((n + 255) / 256, 148 * 32);
    if (W == 4) { KTimer kt_(KC_BIN, st); k_bin<R, 4><<<nblk, 256, 0, st>>>(g, pos, n, keys, ranks, s.counts->as<unsigned>()); }
    else { KTimer kt_(KC_BIN, st); k_bin<R, 6><<<nblk, 256, 0, st>>>(g, pos, n, keys, ranks, s.counts->as<unsigned>()); }
    PM_LAUNCHED();
    CKL(caller);
  }
  if (exclusive_scan(s.counts->as<unsigned>(), s.start->as<unsigned>(), (size_t)g.nbins + 1, *s.spart, st, caller))
    return -1;
  if (n > 0) {
    const int nblk = std::min((n + 255) / 256, 148 * 32);
    { KTimer kt_(KC_PLACE, st); k_place<<<nblk, 256, 0, st>>>(keys, ranks, n, s.start->as<unsigned>(), perm); }
    PM_LAUNCHED();
    const int nbb = (int)std::min<unsigned>(((g.nbins + 3) / 4 + 255) / 256, 148u * 32u);
    { KTimer kt_(KC_FIXUP, st); k_fixup_small<<<std::max(nbb, 1), 256, 0, st>>>(s.start->as<unsigned>(), g.nbins, perm, s.hist->as<unsigned>()); }
    PM_LAUNCHED();
    { KTimer kt_(KC_FIXUP, st); k_fixup_big<<<num_sms(), FIX_THREADS, 0, st>>>(s.start->as<unsigned>(), s.hist->as<unsigned>(), perm, s.key2->as<int>()); }
    PM_LAUNCHED();
    CKL(caller);
  }
  return 0;
}

// One deposition launch: a persistent grid of one CTA per SM (fewer for small
// grids), each taking an equal share of the cells.
template <typename R, int W, int NV>
static int launch_deposit(const PartGeom<R> &g, const R *pos, const R *vp, int vstride, PartScratchRefs s,
                          const int *perm, R *mp, int mstride, int clear_mode, cudaStream_t st, const char *caller) {
  const size_t smem = deposit_smem<R, W>();
  const int threads = dep_threads<R, W>();
  if (smem_attr((const void *)k_deposit<R, W, NV>, smem, caller)) return -1;
  // tiles of equal size: as many as 32 x CY tiles would need, cells spread evenly
  const int CY = dep_cells_y<R, W>();
  const long long ntx = (g.ext[0] + DEP_TX - 1) / DEP_TX, nty = (g.ext[1] + CY - 1) / CY;
  const int tw = (int)((g.ext[0] + ntx - 1) / ntx), th = (int)((g.ext[1] + nty - 1) / nty);
  const long long units = ntx * nty * g.ext[2];
  const int grid = (int)std::max<long long>(1, std::min<long long>(num_sms(), units));
  KTimer kt_(KC_DEPOSIT, st);
  k_deposit<R, W, NV><<<grid, threads, smem, st>>>(g, pos, vp, vstride, s.start->as<unsigned>(), perm, mp, mstride,
                                                    clear_mode, tw, th);
  PM_LAUNCHED();
  CKL(caller);
  return 0;
}

// P2M on device arrays.  clear_mode: 0 add, 1 clear, 2 clear ghosts.  On return
// *perm_out (if given) points at the sorted particle order.
template <typename R>
static int run_p2m(const pmgpu_topo *t, int order, const R *pos, const R *val, int nvar, int n, R *mesh,
                   int nvar_mesh, int clear_mode, PartScratchRefs s, cudaStream_t st, const int **perm_out,
                   const char *caller) {
  if (run_bin_sort<R>(t, order, pos, n, s, st, caller)) return -1;
  const int W = (order == 3) ? 4 : 6;
  PartGeom<R> g = part_geom<R>(t, W);
  const int *perm = s.val2->as<int>();
  // deposition, components in groups of at most three
  for (int c0 = 0; c0 < nvar;) {
    const int nv = (nvar - c0 >= 3) ? 3 : 1;
    const R *vp = val + c0;
    R *mp = mesh + c0;
    int rc = 0;
    if (W == 4) rc = (nv == 3) ? launch_deposit<R, 4, 3>(g, pos, vp, nvar, s, perm, mp, nvar_mesh, clear_mode, st, caller)
                               : launch_deposit<R, 4, 1>(g, pos, vp, nvar, s, perm, mp, nvar_mesh, clear_mode, st, caller);
    else rc = (nv == 3) ? launch_deposit<R, 6, 3>(g, pos, vp, nvar, s, perm, mp, nvar_mesh, clear_mode, st, caller)
                        : launch_deposit<R, 6, 1>(g, pos, vp, nvar, s, perm, mp, nvar_mesh, clear_mode, st, caller);
    if (rc) return -1;
    c0 += nv;
  }
  // components beyond nvar in the mesh are left alone; a wider mesh is an error upstream
  for (int d = 0; d < 3; d++) {
    if (t->bound_cond[2 * d] == 0 || t->bound_cond[2 * d + 1] == 0) continue;
    const int S = t->nghost[2 * d] + t->nghost[2 * d + 1];
    const long long total = (long long)S * g.ext[(d + 1) % 3] * g.ext[(d + 2) % 3];
    const int nblk = (int)std::min<long long>((total + 255) / 256, 148 * 16);
    { KTimer kt_(KC_GADD, st); k_ghost_add<R><<<std::max(nblk, 1), 256, 0, st>>>(mesh, g.ext[0], g.ext[1], g.ext[2], nvar_mesh, d,
                                                       t->ncell[d], t->nghost[2 * d], t->nghost[2 * d + 1]); }
    PM_LAUNCHED();
    CKL(caller);
  }
  if (perm_out) *perm_out = perm;
  return 0;
}

template <typename R>
static int run_m2p(const pmgpu_topo *t, int order, const R *pos, const int *ord, int n, const R *f0, const R *f1,
                   const R *f2, R *o0, R *o1, R *o2, cudaStream_t st, const char *caller) {
  if (n <= 0) return 0;
  const int W = (order == 3) ? 4 : 6;
  PartGeom<R> g = part_geom<R>(t, W);
  const int nblk = std::min((n + 127) / 128, 148 * 32);
  if (W == 4) { KTimer kt_(KC_M2P, st); k_m2p<R, 4><<<nblk, 128, 0, st>>>(g, pos, ord, n, nullptr, f0, f1, f2, o0, o1, o2); }
  else { KTimer kt_(KC_M2P, st); k_m2p<R, 6><<<nblk, 128, 0, st>>>(g, pos, ord, n, nullptr, f0, f1, f2, o0, o1, o2); }
  PM_LAUNCHED();
  CKL(caller);
  return 0;
}

// M2P of one field for particles already sorted by bin (perm, start of the
// deposition with the same positions): tiles of bins through shared memory, then
// the particles outside every bin (the tail of perm) one by one.
template <typename R, int W>
static int run_m2p_sorted_w(const pmgpu_topo *t, const R *pos, const unsigned *start, const int *perm, int n,
                            const R *f, R *o, cudaStream_t st, const char *caller) {
  PartGeom<R> g = part_geom<R>(t, W);
  const size_t sm = m2p_tile_smem<R, W>();
  if (smem_attr((const void *)k_m2p_tile<R, W>, sm, caller)) return -1;
  // tile edges on the bin of interior cell 1 (bin 1 - blo) along each axis
  auto org = [&](int e, int T) {
    const int r = (1 - g.blo[e]) % T;
    return r ? r - T : 0;
  };
  const int3 o3 = make_int3(org(0, M2P_TX), org(1, M2P_TY), org(2, M2P_TZ));
  dim3 grid((g.nb[0] - o3.x + M2P_TX - 1) / M2P_TX, (g.nb[1] - o3.y + M2P_TY - 1) / M2P_TY,
            (g.nb[2] - o3.z + M2P_TZ - 1) / M2P_TZ);
  { KTimer kt_(KC_M2P, st); k_m2p_tile<R, W><<<grid, M2P_THREADS, sm, st>>>(g, pos, start, perm, f, o, o3); }
  PM_LAUNCHED();
  const int nblk = std::min((n + 127) / 128, 148 * 8);
  { KTimer kt_(KC_M2P, st);
    k_m2p<R, W><<<nblk, 128, 0, st>>>(g, pos, perm, n, start + g.nbins, nullptr, nullptr, f, nullptr, nullptr, o); }
  PM_LAUNCHED();
  CKL(caller);
  return 0;
}
template <typename R>
static int run_m2p_sorted(const pmgpu_topo *t, int order, const R *pos, const unsigned *start, const int *perm,
                          int n, const R *f, R *o, cudaStream_t st, const char *caller) {
  if (n <= 0) return 0;
  return order == 3 ? run_m2p_sorted_w<R, 4>(t, pos, start, perm, n, f, o, st, caller)
                    : run_m2p_sorted_w<R, 6>(t, pos, start, perm, n, f, o, st, caller);
}

// ------------------------------------------------------------------ solve driver
template <typename R> static SolveGeom<R> solve_geom(const pmgpu_plan *pl) {
  typedef typename cplx_t<R>::type C;
  SolveGeom<R> g;
  memset(&g, 0, sizeof(g));
  for (int e = 0; e < 3; e++) {
    g.ext[e] = pl->g.ext[e];
    g.off[e] = pl->g.off[e];
    g.P[e] = pl->g.P[e];
    g.M[e] = pl->g.M[e];
  }
  g.H = pl->g.H;
  g.Hp = pl->g.Hp;
  g.N2 = pl->g.N2;
  g.fx = pl->fx;
  g.fy = pl->fy;
  g.fz = pl->fz;
  g.twx = pl->twx.as<C>();
  g.twy = pl->twy.as<C>();
  g.twz = pl->twz.as<C>();
  g.kxt = pl->kxt.as<R>();
  g.kyt = pl->kyt.as<R>();
  g.kzt = pl->kzt.as<R>();
  g.green = pl->green.as<R>();
  g.gM1 = pl->gM1;
  g.gM2 = pl->gM2;
  g.kernel2 = pl->par.poisson_kernel == 2;
  g.scale = (R)(1.0 / ((double)g.M[0] * (double)g.M[1] * (double)g.M[2]));
  g.eps2pi = (R)(2.0 * 3.14159265358979323846 * pl->eps);
  g.order = pl->par.poisson_order;
  g.allper = pl->g.allper;
  g.rchx = pl->rchx.as<C>();
  g.rchy = pl->rchy.as<C>();
  g.rchz = pl->rchz.as<C>();
  g.rbx = pl->rbx.as<C>();
  g.rby = pl->rby.as<C>();
  g.rbz = pl->rbz.as<C>();
  g.tky = pl->tky;
  g.tkz = pl->tkz;
  g.rx_ok = pl->rx_ok;
  g.rx = pl->rx;
  g.rtwx = pl->rtwx.as<C>();
  g.rextx = pl->rextx.as<C>();
  g.xpos = pl->xpos.as<int>();
  g.ry_ok = pl->ry_ok;
  g.rz_ok = pl->rz_ok;
  g.ry = pl->ry;
  g.rz = pl->rz;
  g.rtwy = pl->rtwy.as<C>();
  g.rtwz = pl->rtwz.as<C>();
  g.yk = pl->ry_ok ? pl->yk.as<int>() : nullptr;
  g.zk = pl->rz_ok ? pl->zk.as<int>() : nullptr;
  return g;
}

template <typename R>
static int run_solve(pmgpu_plan *pl, const R *vort, R *vel, R *vort_out, R *vecpot, int reg_vort, int reproj,
                     int calc_vecpot, cudaStream_t st, const char *caller) {
  typedef typename cplx_t<R>::type C;
  SolveGeom<R> g = solve_geom<R>(pl);
  const int ifft_vort = reg_vort || reproj;
  const int ifft_vecpot = calc_vecpot && pl->par.poisson_kernel == 1;
  const size_t nX = (size_t)g.P[1] * g.P[2] * g.Hp * 3, nY = (size_t)g.M[1] * g.P[2] * g.Hp * 3;
  if (pl->X.ensure(sizeof(C) * nX, caller) || pl->Y.ensure(sizeof(C) * nY, caller)) return -1;
  if (ifft_vort && pl->Y2.ensure(sizeof(C) * nY, caller)) return -1;
  if (ifft_vecpot && pl->Y3.ensure(sizeof(C) * nY, caller)) return -1;
  C *X = pl->X.as<C>(), *Y = pl->Y.as<C>();
  if (fwd_xy<R, 3>(g, vort, X, Y, st, caller)) return -1;
  if (ifft_vecpot && zpass<R, 3>(g, Y, pl->Y3.as<C>(), Z_VECPOT, 0, ifft_vort, g.M[1], st, caller)) return -1;
  if (ifft_vort && zpass<R, 3>(g, Y, pl->Y2.as<C>(), Z_VORT, reproj, 1, g.M[1], st, caller)) return -1;
  if (zpass<R, 3>(g, Y, Y, Z_VEL, 0, ifft_vort, g.M[1], st, caller)) return -1;
  if (inv_yx<R, 3>(g, &pl->topo, Y, X, vel, st, caller)) return -1;
  if (ifft_vort && inv_yx<R, 3>(g, &pl->topo, pl->Y2.as<C>(), X, vort_out, st, caller)) return -1;
  if (ifft_vecpot && vecpot && inv_yx<R, 3>(g, &pl->topo, pl->Y3.as<C>(), X, vecpot, st, caller)) return -1;
  return 0;
}

template <typename R, int NC>
static int run_regularise_nc(pmgpu_plan *pl, R *mesh, int cs, int reg_order, double fw, cudaStream_t st,
                             const char *caller) {
  typedef typename cplx_t<R>::type C;
  SolveGeom<R> g = solve_geom<R>(pl);
  g.order = reg_order;
  g.eps2pi = (R)(2.0 * 3.14159265358979323846 * fw);
  const size_t nX = (size_t)g.P[1] * g.P[2] * g.Hp * NC, nY = (size_t)g.M[1] * g.P[2] * g.Hp * NC;
  if (pl->X.ensure(sizeof(C) * nX, caller) || pl->Y.ensure(sizeof(C) * nY, caller)) return -1;
  C *X = pl->X.as<C>(), *Y = pl->Y.as<C>();
  if (fwd_xy<R, NC>(g, mesh, X, Y, st, caller, cs)) return -1;
  if (zpass<R, NC>(g, Y, Y, Z_REGULARISE, 0, 1, g.M[1], st, caller)) return -1;
  return inv_yx<R, NC>(g, &pl->topo, Y, X, mesh, st, caller, cs, false);
}

// pmlib_regularise on a device mesh of nvar components (ghost fill once at the end)
template <typename R>
static int run_regularise(pmgpu_plan *pl, R *mesh, int nvar, int reg_order, double fw, cudaStream_t st,
                          const char *caller) {
  if (nvar == 3) {
    if (run_regularise_nc<R, 3>(pl, mesh, 3, reg_order, fw, st, caller)) return -1;
  } else {
    for (int c = 0; c < nvar; c++)
      if (run_regularise_nc<R, 1>(pl, mesh + c, nvar, reg_order, fw, st, caller)) return -1;
  }
  const pmgpu_topo *topo = &pl->topo;
  for (int d = 0; d < 3; d++) {
    if (topo->bound_cond[2 * d] == 0 || topo->bound_cond[2 * d + 1] == 0) continue;
    const int ext[3] = {pl->g.ext[0], pl->g.ext[1], pl->g.ext[2]};
    const int S = topo->nghost[2 * d] + topo->nghost[2 * d + 1];
    const long long total = (long long)S * ext[(d + 1) % 3] * ext[(d + 2) % 3];
    const int nblk = (int)std::min<long long>((total + 255) / 256, 148 * 16);
    { KTimer kt_(KC_GFILL, st); k_ghost_fill<R><<<std::max(nblk, 1), 256, 0, st>>>(mesh, ext[0], ext[1], ext[2], nvar, d, topo->ncell[d],
                                                        topo->nghost[2 * d], topo->nghost[2 * d + 1]); }
    PM_LAUNCHED();
    CKL(caller);
  }
  return 0;
}

// ------------------------------------------------------------------ Green's function
// Spectra are shared by plans of the same grid, kernel parameters, precision and
// device: the cache holds weak references, a spectrum lives while a plan uses it.
static std::map<std::string, std::weak_ptr<DevBuf>> g_green_cache;

static std::string green_key(const pmgpu_plan *pl) {
  int dev = 0;
  cudaGetDevice(&dev);
  char b[512];
  const pmgpu_patch &p = pl->patch;
  snprintf(b, sizeof(b), "%d|%d.%d|%d|%a,%a,%a|%d,%d,%d|%d,%d,%d|%d,%d,%d,%d|%d,%d,%a", dev, pl->green_mode,
           pl->pff_kx0, pl->prec,
           p.dx[0], p.dx[1], p.dx[2], pl->g.M[0], pl->g.M[1], pl->g.M[2], p.bound_cond[0], p.bound_cond[1],
           p.bound_cond[2], p.ncell[0], p.ncell[1], p.ncell[2], p.nghost, pl->par.poisson_order,
           pl->par.poisson_kernel, pl->par.regularisation_radius);
  return std::string(b);
}

static void attach_green(pmgpu_plan *pl, const std::shared_ptr<DevBuf> &sp) {
  pl->green_own = sp;
  pl->green.p = sp->p;
  pl->green.cap = sp->cap;
  pl->green.fixed = true;
}

template <typename R> static int reg_tables(pmgpu_plan *pl, const char *caller, bool tune_ok);

template <typename R> static int setup_green(pmgpu_plan *pl, const char *caller) {
  const Geometry &G = pl->g;
  pl->gM1 = G.M[1] / 2 + 1;
  pl->gM2 = G.M[2] / 2 + 1;
  if (G.allper) return 0;
  const std::string key = green_key(pl);
  {
    auto it = g_green_cache.find(key);
    if (it != g_green_cache.end()) {
      if (auto sp = it->second.lock()) {
        attach_green(pl, sp);
        return 0;
      }
      g_green_cache.erase(it);
    }
  }
  std::shared_ptr<DevBuf> own(new DevBuf(), [](DevBuf *b) {
    b->release();
    delete b;
  });
  GreenParams gp;
  memset(&gp, 0, sizeof(gp));
  double mdx = 0.0;
  for (int e = 0; e < 3; e++) {
    gp.M[e] = G.M[e];
    gp.bc[e] = pl->patch.bound_cond[e] != 0 ? 1 : 0;
    gp.dx[e] = pl->patch.dx[e];
    gp.xmin[e] = -(0.5 * (double)G.M[e] + 0.5) * gp.dx[e];
    gp.plen[e] = pl->patch.bound_cond[e] == 0 ? gp.dx[e] * (double)(2 * (pl->patch.ncell[e] + 2 * pl->patch.nghost))
                                              : gp.dx[e] * (double)pl->patch.ncell[e];
    mdx = std::max(mdx, gp.dx[e]);
  }
  gp.mdx = mdx;
  gp.eps = pl->par.regularisation_radius * mdx;
  gp.order = pl->par.poisson_order;
  gp.kernel = pl->par.poisson_kernel;
  // FP64 transform of the sampled kernel on the full grid (ext = P = M): a temporary
  // FP64 plan provides the transform tables of the same lengths
  pmgpu_plan tmp;
  tmp.prec = PMGPU_FP64;
  tmp.g = G;
  for (int e = 0; e < 3; e++) {
    tmp.g.ext[e] = tmp.g.P[e] = G.M[e];
    tmp.g.off[e] = 0;
  }
  tmp.par = pl->par;
  tmp.eps = 0.0;
  tmp.perm = nullptr;
  tmp.perm_n = 0;
  tmp.gM1 = tmp.gM2 = 0;
  std::vector<cld> tw;
  // temporaries are stream-ordered on the legacy stream, so a set-up does not wait
  // for (or stall) solves running on other streams
  DevBuf gr, gX, gY, yinv, zinv;
  int rc = -1;
  do {
    if (!make_fft(G.N2, G.M[0], tmp.fx, tw) || upload_tw<double>(tw, tmp.twx, caller)) break;
    if (!make_fft(G.M[1], 0, tmp.fy, tw) || upload_tw<double>(tw, tmp.twy, caller)) break;
    if (!make_fft(G.M[2], 0, tmp.fz, tw) || upload_tw<double>(tw, tmp.twz, caller)) break;
    if (reg_tables<double>(&tmp, caller, false)) break;
    SolveGeom<double> gg = solve_geom<double>(&tmp);
    // spectrum rows after the y and z transforms: frequency -> row
    std::vector<int> yi(G.M[1]), zi(G.M[2]);
    bool rows_ok = true;
    for (int a = 0; a < 2 && rows_ok; a++) {
      const int n = G.M[1 + a];
      std::vector<int> &inv = a == 0 ? yi : zi;
      const int ok = a == 0 ? tmp.ry_ok : tmp.rz_ok;
      for (int q = 0; q < n; q++) inv[q] = q;
      if (ok) {
        std::vector<int> kp(n);
        rows_ok = cuda_ok(cudaMemcpy(kp.data(), (a == 0 ? tmp.yk : tmp.zk).p, sizeof(int) * n,
                                     cudaMemcpyDeviceToHost), caller);
        if (rows_ok)
          for (int q = 0; q < n; q++) inv[kp[q]] = q;
      }
    }
    if (!rows_ok) break;
    if (yinv.ensure(sizeof(int) * G.M[1], caller) || zinv.ensure(sizeof(int) * G.M[2], caller)) break;
    if (!cuda_ok(cudaMemcpy(yinv.p, yi.data(), sizeof(int) * G.M[1], cudaMemcpyHostToDevice), caller)) break;
    if (!cuda_ok(cudaMemcpy(zinv.p, zi.data(), sizeof(int) * G.M[2], cudaMemcpyHostToDevice), caller)) break;
    const size_t npts = (size_t)G.M[0] * G.M[1] * G.M[2];
    const size_t nspec = (size_t)G.M[2] * G.M[1] * G.Hp;
    if (gr.ensure(sizeof(double) * npts, caller) || gX.ensure(sizeof(double2) * nspec, caller) ||
        gY.ensure(sizeof(double2) * nspec, caller))
      break;
    const size_t noct = (size_t)pl->gM2 * pl->gM1 * G.H;
    const double f = pl->patch.dx[0] * pl->patch.dx[1] * pl->patch.dx[2] /
                     ((double)G.M[0] * (double)G.M[1] * (double)G.M[2]);
    const unsigned nb_real = (unsigned)std::min<size_t>((npts + 255) / 256, 148 * 64);
    const unsigned nb_oct = (unsigned)std::min<size_t>((noct + 255) / 256, 148 * 64);
    if (pl->green_mode == 2) {
      // the mixed-space kernel of the pff validation program: the x-transformed layout
      // (kx natural wavenumbers, y and z positions) is written directly, then y and z
      const unsigned nb_x = (unsigned)std::min<size_t>((nspec + 255) / 256, 148 * 64);
      k_green_pff<<<nb_x, 256>>>(gp, pl->pff_kx0, G.H, G.Hp, gX.as<double2>());
      PM_LAUNCHED();
      if (!cuda_ok(cudaGetLastError(), caller)) break;
      if (ypass<double, 1>(gg, gX.as<double2>(), gY.as<double2>(), 0, 0, caller)) break;
      if (zpass<double, 1>(gg, gY.as<double2>(), gY.as<double2>(), Z_FORWARD, 0, 0, G.M[1], 0, caller)) break;
      if (!cuda_ok(cudaStreamSynchronize(0), caller)) break;
      if (own->ensure(sizeof(R) * noct, caller)) break;
      attach_green(pl, own);
      k_green_octant<R><<<nb_oct, 256>>>(gY.as<double2>(), G.M[1], G.H, G.Hp, pl->gM1, pl->gM2, f, yinv.as<int>(),
                                         zinv.as<int>(), pl->green.as<R>());
      PM_LAUNCHED();
      if (!cuda_ok(cudaGetLastError(), caller)) break;
    } else if (pl->green_mode == 1) {
      // the spectral kernel of the ppf validation program: the y-transformed spectrum
      // (kx, ky natural wavenumbers, z positions) is written directly, then z only
      const unsigned nb_y = (unsigned)std::min<size_t>((nspec + 255) / 256, 148 * 64);
      k_green_ppf<<<nb_y, 256>>>(gp, G.H, G.Hp, tmp.ry_ok ? tmp.yk.as<int>() : nullptr, gY.as<double2>());
      PM_LAUNCHED();
      if (!cuda_ok(cudaGetLastError(), caller)) break;
      if (zpass<double, 1>(gg, gY.as<double2>(), gY.as<double2>(), Z_FORWARD, 0, 0, G.M[1], 0, caller)) break;
      if (!cuda_ok(cudaStreamSynchronize(0), caller)) break;
      if (own->ensure(sizeof(R) * noct, caller)) break;
      attach_green(pl, own);
      k_green_octant<R><<<nb_oct, 256>>>(gY.as<double2>(), G.M[1], G.H, G.Hp, pl->gM1, pl->gM2, f, yinv.as<int>(),
                                         zinv.as<int>(), pl->green.as<R>());
      PM_LAUNCHED();
      if (!cuda_ok(cudaGetLastError(), caller)) break;
    } else if (gp.kernel == 1) {
      k_green_real<<<nb_real, 256>>>(gp, gr.as<double>());
      PM_LAUNCHED();
      if (!cuda_ok(cudaGetLastError(), caller)) break;
      if (fwd_xy<double, 1>(gg, gr.as<double>(), gX.as<double2>(), gY.as<double2>(), 0, caller)) break;
      if (zpass<double, 1>(gg, gY.as<double2>(), gY.as<double2>(), Z_FORWARD, 0, 0, G.M[1], 0, caller)) break;
      if (!cuda_ok(cudaStreamSynchronize(0), caller)) break;
      if (own->ensure(sizeof(R) * noct, caller)) break;
      attach_green(pl, own);
      k_green_octant<R><<<nb_oct, 256>>>(gY.as<double2>(), G.M[1], G.H, G.Hp, pl->gM1, pl->gM2, f, yinv.as<int>(),
                                         zinv.as<int>(), pl->green.as<R>());
      PM_LAUNCHED();
      if (!cuda_ok(cudaGetLastError(), caller)) break;
    } else {
      // three octants S_x, S_y, S_z, then the planes E_x, E_y, E_z
      const size_t nE = (size_t)pl->gM2 * pl->gM1 + (size_t)pl->gM2 * G.H + (size_t)pl->gM1 * G.H;
      if (own->ensure(sizeof(R) * (3 * noct + nE), caller)) break;
      attach_green(pl, own);
      R *S = pl->green.as<R>(), *E = S + 3 * noct;
      R *Ec[3] = {E, E + (size_t)pl->gM2 * pl->gM1, E + (size_t)pl->gM2 * (pl->gM1 + G.H)};
      bool ok = true;
      for (int c = 0; c < 3 && ok; c++) {
        k_green_real2<<<nb_real, 256>>>(gp, c, gr.as<double>());
        PM_LAUNCHED();
        ok = cuda_ok(cudaGetLastError(), caller) &&
             !fwd_xy<double, 1>(gg, gr.as<double>(), gX.as<double2>(), gY.as<double2>(), 0, caller) &&
             !zpass<double, 1>(gg, gY.as<double2>(), gY.as<double2>(), Z_FORWARD, 0, 0, G.M[1], 0, caller);
        if (!ok) break;
        k_green2_split<R><<<nb_oct, 256>>>(gY.as<double2>(), c, G.M[0], G.M[1], G.M[2], G.H, G.Hp, pl->gM1, pl->gM2,
                                           f, yinv.as<int>(), zinv.as<int>(), S + c * noct, Ec[c]);
        PM_LAUNCHED();
        ok = cuda_ok(cudaGetLastError(), caller);
      }
      if (!ok) break;
    }
    if (!cuda_ok(cudaStreamSynchronize(0), caller)) break;
    g_green_cache[key] = own;
    rc = 0;
  } while (0);
  gr.release(); gX.release(); gY.release(); yinv.release(); zinv.release();
  cudaStreamSynchronize(0);
  return rc;
}

template <typename R> static int upload_wavenumbers(pmgpu_plan *pl, const char *caller) {
  DevBuf *bufs[3] = {&pl->kxt, &pl->kyt, &pl->kzt};
  for (int e = 0; e < 3; e++) {
    const int M = pl->g.M[e];
    const int cnt = (e == 0) ? pl->g.H : M;
    const double dx = pl->patch.dx[e];
    const double dk = 1.0 / ((double)M * dx);  // pmlib_poisson_solve.f:209-224, i_ptc = 0
    const double ksmp = 1.0 / (2.0 * dx);
    const double kmin = -ksmp;
    std::vector<R> h(cnt);
    for (int i = 0; i < cnt; i++) {
      const double k = (i + 1 <= M / 2) ? kmin + (double)i * dk + ksmp : kmin + (double)i * dk - ksmp;
      h[i] = (R)k;
    }
    if (bufs[e]->ensure(sizeof(R) * cnt, caller)) return -1;
    CK(cudaMemcpy(bufs[e]->p, h.data(), sizeof(R) * cnt, cudaMemcpyHostToDevice), caller);
  }
  return 0;
}

// Times the pass along `axis` of this plan's geometry (y: the forward pass; z: the
// fused transform / multiply / inverse pass of the velocity solve) for the candidate
// radix sequences (the five best by the model) and kx tiles, on scratch arrays; the
// fastest goes to the tuning table.  The plan's Green's function must exist.
template <typename R> static int tune_axis(pmgpu_plan *pl, int axis, TunedSchedule &best, const char *caller) {
  typedef typename cplx_t<R>::type C;
  const Geometry &G = pl->g;
  const int n = G.M[axis];
  std::vector<RadixSeq> cands = regplan_candidates(n);
  if (cands.size() > 5) cands.resize(5);
  if (axis == 2) {
    // the same radices ordered for the fused middle of the z pass
    const size_t nc = cands.size();
    for (size_t i = 0; i < nc; i++) {
      const RadixSeq q = z_order(cands[i], (int)sizeof(R));
      bool dup = false;
      for (const RadixSeq &o : cands)
        dup = dup || (o.np == q.np && o.r[0] == q.r[0] && o.r[1] == q.r[1] && o.r[2] == q.r[2]);
      if (!dup) cands.push_back(q);
    }
  }
  if (sizeof(R) == 4) {
    std::vector<RadixSeq> w = regplan_candidates_wide(n);
    if (w.size() > 3) w.resize(3);
    cands.insert(cands.end(), w.begin(), w.end());
  }
  DevBuf A, B, tw, kp;
  const size_t nx = (size_t)G.P[1] * G.P[2] * G.Hp * 3;
  const size_t ny = (size_t)G.M[1] * G.P[2] * G.Hp * 3;
  if ((axis == 1 && A.ensure(sizeof(C) * nx, caller)) || B.ensure(sizeof(C) * ny, caller)) return -1;
  if (axis == 1) CK(cudaMemsetAsync(A.p, 0, sizeof(C) * nx, 0), caller);
  CK(cudaMemsetAsync(B.p, 0, sizeof(C) * ny, 0), caller);
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0), caller);
  CK(cudaEventCreate(&e1), caller);
  best.ms = 1e30;
  best.np = 0;
  const long double twopi = 2.0L * acosl(-1.0L);
  for (const RadixSeq &c : cands) {
    RegPlan rp;
    regplan_from(n, c.r, c.np, rp);
    std::vector<C> t(n);
    for (int q = 0; q < n; q++) {
      const long double a = twopi * (long double)q / (long double)n;
      t[q] = mk((R)cosl(a), (R)-sinl(a));
    }
    const std::vector<int> pos = regplan_positions(rp);
    if (tw.ensure(sizeof(C) * n, caller) || kp.ensure(sizeof(int) * n, caller)) break;
    if (!cuda_ok(cudaMemcpy(tw.p, t.data(), sizeof(C) * n, cudaMemcpyHostToDevice), caller) ||
        !cuda_ok(cudaMemcpy(kp.p, pos.data(), sizeof(int) * n, cudaMemcpyHostToDevice), caller))
      break;
    for (int tk : {8, 4, 2}) {
      if (G.Hp % tk || reg_smem(n, n, 3, tk, sizeof(C)) > PASS_SMEM_BUDGET) continue;
      SolveGeom<R> g = solve_geom<R>(pl);
      if (axis == 1) {
        g.ry = rp;
        g.ry_ok = 1;
        g.rtwy = tw.as<C>();
        g.yk = kp.as<int>();
        g.tky = tk;
      } else {
        g.rz = rp;
        g.rz_ok = 1;
        g.rtwz = tw.as<C>();
        g.zk = kp.as<int>();
        g.tkz = tk;
      }
      auto run = [&]() {
        return axis == 1 ? ypass<R, 3>(g, A.as<C>(), B.as<C>(), 0, 0, caller)
                         : zpass<R, 3>(g, B.as<C>(), B.as<C>(), Z_VEL, 0, 0, G.M[1], 0, caller);
      };
      if (run()) continue;
      cudaEventRecord(e0, 0);
      bool ok = true;
      for (int r = 0; r < 3 && ok; r++) ok = run() == 0;
      cudaEventRecord(e1, 0);
      if (!ok || cudaEventSynchronize(e1) != cudaSuccess) continue;
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      if (ms / 3 < best.ms) {
        best.ms = ms / 3;
        best.np = c.np;
        for (int i = 0; i < 3; i++) best.r[i] = c.r[i];
        best.tk = tk;
      }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaGetLastError();
  return best.np > 0 ? 0 : -1;
}

// Device tables of the register engine, shared by every plan of the same transform
// length, precision and radix schedule (held by weak references, as the Green's
// spectra): a plan's set-up computes and uploads only the tables of lengths no live
// plan has.  Guarded by the set-up lock.
static std::map<std::string, std::weak_ptr<DevBuf>> g_tab_cache;
// the most recently used tables stay alive past their last plan (they are small), so
// that the FP64 transforms of the Green's set-up and plans of recurring lengths reuse
// them
// (never destroyed: freeing device memory from static destructors at exit could
// run after the runtime has unloaded)
static std::deque<std::shared_ptr<DevBuf>> &g_tab_recent = *new std::deque<std::shared_ptr<DevBuf>>();
constexpr size_t TAB_RECENT = 512;

static std::string regplan_key(const char *kind, int prec_bytes, int n, int extra, const RegPlan &rp) {
  char b[160];
  snprintf(b, sizeof(b), "%s|%d|%d|%d|%d:%d,%d,%d|%d,%d", kind, prec_bytes, n, extra, rp.np, rp.rad[0],
           rp.np > 1 ? rp.rad[1] : 0, rp.np > 2 ? rp.rad[2] : 0, rp.bl, rp.bn);
  return std::string(b);
}

// attaches `view` to the cached device table `key`, made by fill(host vector) and
// uploaded on a miss
template <typename T, typename Fill>
static int shared_table(pmgpu_plan *pl, const std::string &key, DevBuf &view, Fill fill, const char *caller) {
  std::shared_ptr<DevBuf> sp;
  auto it = g_tab_cache.find(key);
  if (it != g_tab_cache.end()) sp = it->second.lock();
  if (!sp) {
    std::vector<T> host;
    fill(host);
    sp = std::shared_ptr<DevBuf>(new DevBuf(), [](DevBuf *b) {
      b->release();
      delete b;
    });
    if (sp->ensure(sizeof(T) * std::max<size_t>(host.size(), 1), caller)) return -1;
    if (!host.empty()) CK(cudaMemcpy(sp->p, host.data(), sizeof(T) * host.size(), cudaMemcpyHostToDevice), caller);
    g_tab_cache[key] = sp;
    g_tab_recent.push_back(sp);
    if (g_tab_recent.size() > TAB_RECENT) g_tab_recent.pop_front();
  }
  view.release();
  view.p = sp->p;
  view.cap = sp->cap;
  view.fixed = true;
  pl->tab_keep.push_back(sp);
  return 0;
}

template <typename R> static int reg_tables(pmgpu_plan *pl, const char *caller, bool tune_ok) {
  typedef typename cplx_t<R>::type C;
  pl->rx_ok = pl->ry_ok = pl->rz_ok = 0;
  if (g_force_stockham) return 0;
  const long double twopi = 2.0L * acosl(-1.0L);
  const int pb = (int)sizeof(R);
  // twiddles w_m^q of a plan's transform length m
  auto twiddles = [&](int mm, std::vector<C> &tw) {
    tw.resize(mm);
    for (int q = 0; q < mm; q++) {
      const long double a = twopi * (long double)q / (long double)mm;
      tw[q] = mk((R)cosl(a), (R)-sinl(a));
    }
  };
  // Bluestein chirp and spectrum of a plan (nothing for a direct plan)
  auto upload_blue = [&](const std::string &key, const RegPlan &rp, DevBuf &ch, DevBuf &bp) -> int {
    if (!rp.bl) return 0;
    std::vector<C> c, b;
    bool made = false;
    auto make = [&]() {
      if (!made) bluestein_tables<C, R>(rp, c, b);
      made = true;
    };
    if (shared_table<C>(pl, key + "|ch", ch, [&](std::vector<C> &h) { make(); h = c; }, caller)) return -1;
    return shared_table<C>(pl, key + "|bp", bp, [&](std::vector<C> &h) { make(); h = b; }, caller);
  };
  pl->tab_keep.clear();
  {
    // x passes: half-length complex transform N = Mx / 2
    RegPlan rp;
    const int N = pl->g.N2, H = pl->g.H, Mx = pl->g.M[0];
    if (make_regplan(N, rp) || make_bluestein(N, rp)) {
      const std::string key = regplan_key("x", pb, N, Mx, rp);
      if (shared_table<C>(pl, key + "|tw", pl->rtwx, [&](std::vector<C> &h) { twiddles(rp.n, h); }, caller) ||
          shared_table<C>(pl, key + "|ext", pl->rextx,
                          [&](std::vector<C> &h) {
                            h.resize(H);
                            for (int k = 0; k < H; k++) {
                              const long double a = twopi * (long double)k / (long double)Mx;
                              h[k] = mk((R)cosl(a), (R)-sinl(a));
                            }
                          },
                          caller) ||
          shared_table<int>(pl, key + "|pos", pl->xpos,
                            [&](std::vector<int> &h) {
                              h.resize(N);
                              if (rp.bl) {
                                for (int q = 0; q < N; q++) h[q] = q;  // natural order
                              } else {
                                const std::vector<int> kp = regplan_positions(rp);
                                for (int q = 0; q < N; q++) h[kp[q]] = q;
                              }
                            },
                            caller) ||
          upload_blue(key, rp, pl->rchx, pl->rbx))
        return -1;
      pl->rx = rp;
      pl->rx_ok = 1;
    }
  }
  for (int axis = 1; axis <= 2; axis++) {
    RegPlan rp;
    const int n = pl->g.M[axis];
    if (!make_regplan(n, rp) && !make_bluestein(n, rp)) continue;
    bool tuned = false;
    if (!rp.bl && tune_ok) {
      // a schedule measured earlier for this length
      auto it = g_tuned.find(std::make_tuple(n, (int)sizeof(R), axis));
      if (it != g_tuned.end()) {
        regplan_from(n, it->second.r, it->second.np, rp);
        (axis == 1 ? pl->tky : pl->tkz) = it->second.tk;
        tuned = true;
      }
    }
    if (!rp.bl && !tuned && axis == 2) {
      // untuned z plans: the model's radices ordered for the fused middle
      RadixSeq c;
      c.np = rp.np;
      for (int i = 0; i < 3; i++) c.r[i] = i < rp.np ? rp.rad[i] : 0;
      c.cost = 0.0;
      const RadixSeq q = z_order(c, (int)sizeof(R));
      regplan_from(n, q.r, q.np, rp);
    }
    const std::string key = regplan_key("l", pb, n, 0, rp);
    DevBuf &tb = axis == 1 ? pl->rtwy : pl->rtwz;
    DevBuf &kb = axis == 1 ? pl->yk : pl->zk;
    if (shared_table<C>(pl, key + "|tw", tb, [&](std::vector<C> &h) { twiddles(rp.n, h); }, caller) ||
        shared_table<int>(pl, key + "|pos", kb,
                          [&](std::vector<int> &h) {
                            if (rp.bl) {
                              h.resize(n);
                              for (int q = 0; q < n; q++) h[q] = q;  // natural order
                            } else {
                              h = regplan_positions(rp);
                            }
                          },
                          caller) ||
        upload_blue(key, rp, axis == 1 ? pl->rchy : pl->rchz, axis == 1 ? pl->rby : pl->rbz))
      return -1;
    if (axis == 1) {
      pl->ry = rp;
      pl->ry_ok = 1;
    } else {
      pl->rz = rp;
      pl->rz_ok = 1;
    }
  }
  return 0;
}

// while tuning is on: measure the schedules of lengths not yet in the table, then
// rebuild the register plans from the table
template <typename R> static int apply_tuning(pmgpu_plan *pl, const char *caller) {
  if (!g_tune || g_force_stockham) return 0;
  bool fresh = false;
  for (int axis = 1; axis <= 2; axis++) {
    const RegPlan &rp = axis == 1 ? pl->ry : pl->rz;
    if (!(axis == 1 ? pl->ry_ok : pl->rz_ok) || rp.bl) continue;
    const auto key = std::make_tuple(pl->g.M[axis], (int)sizeof(R), axis);
    if (g_tuned.count(key)) continue;
    TunedSchedule ts;
    if (tune_axis<R>(pl, axis, ts, caller) == 0) {
      g_tuned.emplace(key, ts);
      fresh = true;
    }
  }
  return fresh ? reg_tables<R>(pl, caller, true) : 0;
}

template <typename R> static int plan_tables(pmgpu_plan *pl, const char *caller) {
  typedef typename cplx_t<R>::type C;
  std::vector<cld> tw;
  if (!make_fft(pl->g.N2, pl->g.M[0], pl->fx, tw) || upload_tw<R>(tw, pl->twx, caller)) return -1;
  if (!make_fft(pl->g.M[1], 0, pl->fy, tw) || upload_tw<R>(tw, pl->twy, caller)) return -1;
  if (!make_fft(pl->g.M[2], 0, pl->fz, tw) || upload_tw<R>(tw, pl->twz, caller)) return -1;
  if (upload_wavenumbers<R>(pl, caller)) return -1;
  if (reg_tables<R>(pl, caller, true)) return -1;
  if (setup_green<R>(pl, caller)) return -1;
  // the work spectra of a three-component solve, so that a plan's first solve (often
  // queued from another thread than the set-up) allocates nothing
  const Geometry &G = pl->g;
  const size_t nX = (size_t)G.P[1] * G.P[2] * G.Hp * 3, nY = (size_t)G.M[1] * G.P[2] * G.Hp * 3;
  if (pl->X.ensure(sizeof(C) * nX, caller) || pl->Y.ensure(sizeof(C) * nY, caller)) return -1;
  return apply_tuning<R>(pl, caller);
}

static int check_params(const pmgpu_params *par) {
  const char *caller = "pmlib_parameters_check";
  if (!par) {
    set_error(caller, "parameters missing.");
    return -1;
  }
  if (par->poisson_kernel != 1 && par->poisson_kernel != 2) {
    set_error(caller, "pmlib_poisson_kernel is incorrectly set.");
    return -1;
  }
  const int o = par->poisson_order;
  if (o != 0 && o != 2 && o != 4 && o != 6 && o != 8 && o != 10 && o != 100) {
    set_error(caller, "pmlib_poisson_order is incorrectly set.");
    return -1;
  }
  if (o > 0 && par->regularisation_radius < 1.0) {
    set_error(caller, "pmlib_regularisation_radius is incorrectly set.");
    return -1;
  }
  if (par->interpolation_order != 3 && par->interpolation_order != 4) {
    set_error(caller, "pmlib_interpolation_order is incorrectly set.");
    return -1;
  }
  return 0;
}

static int check_interp(const pmgpu_params *par, const char *caller) {
  if (!par || (par->interpolation_order != 3 && par->interpolation_order != 4)) {
    set_error(caller, "Interpolation scheme/order unknown.");
    return -1;
  }
  return 0;
}

}  // namespace pmgpu

// ====================================================================== C ABI
// (C linkage comes from the declarations in pmlib_gpu.h)

const char *pmgpu_last_error(void) { return pmgpu::g_err; }

long long pmgpu_launch_count(int reset) {
  const long long v = reset ? pmgpu::g_launches.exchange(0) : pmgpu::g_launches.load();
  return v;
}

int pmgpu_parameters_check(const pmgpu_params *par) { return check_params(par); }

int pmgpu_inject_alloc_failure(long long after) {
  g_fail_alloc.store(after < 0 ? -1 : after);
  return 0;
}

void pmgpu_timing_enable(int on) {
  std::lock_guard<std::mutex> lk(g_mu);
  timing_collect();
  g_timing = on != 0;
}

void pmgpu_timing_reset(void) {
  std::lock_guard<std::mutex> lk(g_mu);
  timing_collect();
  for (int i = 0; i < KC_N; i++) {
    g_kms[i] = 0.0;
    g_kn[i] = 0;
  }
}

int pmgpu_timing_get(int index, const char **name, double *ms_total, long long *launches) {
  std::lock_guard<std::mutex> lk(g_mu);
  timing_collect();
  if (index < 0 || index >= KC_N) return -1;
  if (name) *name = kc_names[index];
  if (ms_total) *ms_total = g_kms[index];
  if (launches) *launches = g_kn[index];
  return 0;
}

// source/patch/pmlib_patch_adjust.f:34-146
int pmgpu_patch_adjust(pmgpu_patch *p) {
  const char *caller = "pmlib_patch_adjust";
  int extend[3];
  for (int i = 0; i < 3; i++) {
    if (p->bound_cond[i] == 0) {
      const double centre = 0.5 * (p->xmax[i] + p->xmin[i]);
      int ncell = (int)std::ceil((p->xmax[i] - p->xmin[i]) / p->dx[i]);
      ncell = ncell + (16 - ((ncell + 2 * p->nghost) % 16));
      const double half = (double)std::lround(0.5 * (double)ncell);
      p->xmin[i] = centre - half * p->dx[i];
      p->xmax[i] = centre + half * p->dx[i];
      p->ncell[i] = (int)std::lround((p->xmax[i] - p->xmin[i]) / p->dx[i]);
      if (p->ncell[i] != ncell) {
        set_error(caller, "Failed to adjust the number of mesh cells");
        return -1;
      }
    } else {
      p->xmax[i] = p->xmin[i] + p->dx[i] * (double)std::lround((p->xmax[i] - p->xmin[i]) / p->dx[i]);
      p->ncell[i] = (int)std::lround((p->xmax[i] - p->xmin[i]) / p->dx[i]);
    }
  }
  for (int i = 0; i < 3; i++) extend[i] = p->bound_cond[i] == 0 ? 2 * p->ncell[i] : p->ncell[i];
  int s[3];
  if (extend[0] >= extend[1] && extend[0] >= extend[2]) {
    if (extend[1] >= extend[2]) { s[0] = 1; s[1] = 2; s[2] = 3; } else { s[0] = 1; s[1] = 3; s[2] = 2; }
  } else if (extend[1] >= extend[0] && extend[1] >= extend[2]) {
    if (extend[0] >= extend[2]) { s[0] = 2; s[1] = 1; s[2] = 3; } else { s[0] = 2; s[1] = 3; s[2] = 1; }
  } else if (extend[2] >= extend[0] && extend[2] >= extend[1]) {
    if (extend[0] >= extend[1]) { s[0] = 3; s[1] = 1; s[2] = 2; } else { s[0] = 3; s[1] = 2; s[2] = 1; }
  } else {
    set_error(caller, "Cant figure out fft sequence.");
    return -1;
  }
  for (int i = 0; i < 3; i++) p->fft_seq[i] = s[i];
  return 0;
}

// source/topology/pmlib_topology_cuboid.f:225-325 for one subdomain
int pmgpu_topology_cuboid(const pmgpu_patch *patch, int interpolation_order, pmgpu_topo *t) {
  const char *caller = "pmlib_topology_cuboid";
  int nghost_int;
  if (interpolation_order == 3) nghost_int = 2;
  else if (interpolation_order == 4) nghost_int = 3;
  else {
    set_error(caller, "Can not define number of ghost cells.");
    return -1;
  }
  memset(t, 0, sizeof(*t));
  for (int d = 0; d < 3; d++) {
    t->xmin[d] = patch->xmin[d];
    t->xmax[d] = patch->xmax[d];
    t->dx[d] = patch->dx[d];
    t->ncell[d] = patch->ncell[d];
    for (int s = 0; s < 2; s++) {
      t->bound_cond[2 * d + s] = patch->bound_cond[d] == 0 ? 0 : 1;
      t->nghost[2 * d + s] = patch->bound_cond[d] == 0 ? patch->nghost : nghost_int;
    }
  }
  return 0;
}

// ------------------------------------------------------------------ P2M / M2P (host pointers)
template <typename R>
static int p2m_host(const pmgpu_topo *t, const pmgpu_params *par, const R *xpart, const R *part, int nvar,
                    int npart, R *mesh, int nvar_mesh, int clear, int clear_ghost) {
  const char *caller = "pmlib_interp_particle_mesh";
  std::lock_guard<std::mutex> lk(g_mu);
  if (nvar != nvar_mesh) {
    set_error(caller, "Dimension of interpolation variables does not correspond.");
    return -1;
  }
  if (t->npart != npart) {
    set_error(caller, "Discrepancy in number of particles");
    return -1;
  }
  if (check_interp(par, caller) || ensure_device(caller)) return -1;
  Scratch &s = scratch();
  const size_t nm = mesh_points(t) * (size_t)nvar_mesh;
  if (s.a.ensure(sizeof(R) * 3 * (size_t)std::max(npart, 1), caller) ||
      s.b.ensure(sizeof(R) * (size_t)nvar * std::max(npart, 1), caller) || s.c.ensure(sizeof(R) * nm, caller))
    return -1;
  if (npart > 0) {
    CK(cudaMemcpy(s.a.p, xpart, sizeof(R) * 3 * (size_t)npart, cudaMemcpyHostToDevice), caller);
    CK(cudaMemcpy(s.b.p, part, sizeof(R) * (size_t)nvar * npart, cudaMemcpyHostToDevice), caller);
  }
  const int mode = clear ? 1 : (clear_ghost ? 2 : 0);
  if (mode != 1) CK(cudaMemcpy(s.c.p, mesh, sizeof(R) * nm, cudaMemcpyHostToDevice), caller);
  PartScratchRefs r{&s.key, &s.val, &s.key2, &s.val2, &s.counts, &s.start, &s.spart, &s.hist};
  if (run_p2m<R>(t, par->interpolation_order, s.a.as<R>(), s.b.as<R>(), nvar, npart, s.c.as<R>(), nvar_mesh, mode,
                 r, 0, nullptr, caller))
    return -1;
  CK(cudaMemcpy(mesh, s.c.p, sizeof(R) * nm, cudaMemcpyDeviceToHost), caller);
  return 0;
}

int pmgpu_interp_particle_mesh(const pmgpu_topo *topo, const pmgpu_params *par, const double *xpart,
                               const double *part, int nvar, int npart, double *mesh, int nvar_mesh, int clear,
                               int clear_ghost) {
  return p2m_host<double>(topo, par, xpart, part, nvar, npart, mesh, nvar_mesh, clear, clear_ghost);
}
int pmgpu_interp_particle_mesh_f32(const pmgpu_topo *topo, const pmgpu_params *par, const float *xpart,
                                   const float *part, int nvar, int npart, float *mesh, int nvar_mesh, int clear,
                                   int clear_ghost) {
  return p2m_host<float>(topo, par, xpart, part, nvar, npart, mesh, nvar_mesh, clear, clear_ghost);
}

// The bin keys and sorted particle order P2M deposits from (host arrays out)
template <typename R>
static int p2m_order_host(const pmgpu_topo *t, const pmgpu_params *par, const R *xpart, int npart, unsigned *keys,
                          int *order, unsigned *bin_start) {
  const char *caller = "pmgpu_p2m_sort_order";
  std::lock_guard<std::mutex> lk(g_mu);
  if (npart < 0) {
    set_error(caller, "Discrepancy in number of particles");
    return -1;
  }
  if (check_interp(par, caller) || ensure_device(caller)) return -1;
  Scratch &s = scratch();
  if (s.a.ensure(sizeof(R) * 3 * (size_t)std::max(npart, 1), caller)) return -1;
  if (npart > 0) CK(cudaMemcpy(s.a.p, xpart, sizeof(R) * 3 * (size_t)npart, cudaMemcpyHostToDevice), caller);
  PartScratchRefs r{&s.key, &s.val, &s.key2, &s.val2, &s.counts, &s.start, &s.spart, &s.hist};
  if (run_bin_sort<R>(t, par->interpolation_order, s.a.as<R>(), npart, r, 0, caller)) return -1;
  const PartGeom<R> g = part_geom<R>(t, par->interpolation_order == 3 ? 4 : 6);
  if (npart > 0 && keys) CK(cudaMemcpy(keys, s.key.p, sizeof(unsigned) * npart, cudaMemcpyDeviceToHost), caller);
  if (npart > 0 && order) CK(cudaMemcpy(order, s.val2.p, sizeof(int) * npart, cudaMemcpyDeviceToHost), caller);
  if (bin_start)
    CK(cudaMemcpy(bin_start, s.start.p, sizeof(unsigned) * ((size_t)g.nbins + 1), cudaMemcpyDeviceToHost), caller);
  return 0;
}

int pmgpu_p2m_sort_order(const pmgpu_topo *topo, const pmgpu_params *par, int precision, const void *xpart,
                         int npart, unsigned *keys, int *order, unsigned *bin_start) {
  if (precision == PMGPU_FP32)
    return p2m_order_host<float>(topo, par, static_cast<const float *>(xpart), npart, keys, order, bin_start);
  return p2m_order_host<double>(topo, par, static_cast<const double *>(xpart), npart, keys, order, bin_start);
}

template <typename R>
static int m2p_host(const pmgpu_topo *t, const pmgpu_params *par, const R *mvort, const R *mdvort, const R *mvel,
                    const R *pos, int npart, R *pv, R *pdv, R *pvel) {
  const char *caller = "pmlib_interp_mesh_particle";
  std::lock_guard<std::mutex> lk(g_mu);
  if (check_interp(par, caller) || ensure_device(caller)) return -1;
  Scratch &s = scratch();
  const size_t nm = mesh_points(t) * 3;
  const size_t np3 = 3 * (size_t)std::max(npart, 1);
  if (s.a.ensure(sizeof(R) * np3, caller)) return -1;
  const R *fin[3] = {mvort, mdvort, mvel};
  R *fout[3] = {pv, pdv, pvel};
  DevBuf *mb[3] = {&s.c, &s.d, &s.e};
  DevBuf *ob[3] = {&s.f, &s.g, &s.h};
  const R *df[3] = {nullptr, nullptr, nullptr};
  R *dof[3] = {nullptr, nullptr, nullptr};
  for (int f = 0; f < 3; f++) {
    if (!fin[f] || !fout[f]) continue;
    if (mb[f]->ensure(sizeof(R) * nm, caller) || ob[f]->ensure(sizeof(R) * np3, caller)) return -1;
    CK(cudaMemcpy(mb[f]->p, fin[f], sizeof(R) * nm, cudaMemcpyHostToDevice), caller);
    df[f] = mb[f]->as<R>();
    dof[f] = ob[f]->as<R>();
  }
  if (npart > 0) CK(cudaMemcpy(s.a.p, pos, sizeof(R) * 3 * (size_t)npart, cudaMemcpyHostToDevice), caller);
  if (run_m2p<R>(t, par->interpolation_order, s.a.as<R>(), nullptr, npart, df[0], df[1], df[2], dof[0], dof[1],
                 dof[2], 0, caller))
    return -1;
  for (int f = 0; f < 3; f++)
    if (dof[f] && npart > 0)
      CK(cudaMemcpy(fout[f], dof[f], sizeof(R) * 3 * (size_t)npart, cudaMemcpyDeviceToHost), caller);
  return 0;
}

int pmgpu_interp_mesh_particle(const pmgpu_topo *topo, const pmgpu_params *par, const double *mesh_vort,
                               const double *mesh_dvort, const double *mesh_vel, const double *pos, int npart,
                               double *part_vort, double *part_dvort, double *part_vel) {
  return m2p_host<double>(topo, par, mesh_vort, mesh_dvort, mesh_vel, pos, npart, part_vort, part_dvort, part_vel);
}
int pmgpu_interp_mesh_particle_f32(const pmgpu_topo *topo, const pmgpu_params *par, const float *mesh_vort,
                                   const float *mesh_dvort, const float *mesh_vel, const float *pos, int npart,
                                   float *part_vort, float *part_dvort, float *part_vel) {
  return m2p_host<float>(topo, par, mesh_vort, mesh_dvort, mesh_vel, pos, npart, part_vort, part_dvort, part_vel);
}

// ------------------------------------------------------------------ Poisson
// plan creation; the caller holds g_mu
static int g_pff_kx0 = 0;  // k_x = 0 treatment handed from pmgpu_poisson_setup_pff to create_plan (under g_setup_mu)
static int create_plan(const pmgpu_patch *patch, const pmgpu_topo *cuboid, const pmgpu_params *par, int precision,
                       pmgpu_plan **plan, const char *caller, int green_mode = 0) {
  if (!plan || !patch || !cuboid) {
    set_error(caller, "missing argument.");
    return -1;
  }
  *plan = nullptr;
  if (check_params(par)) return -1;
  if (precision != PMGPU_FP64 && precision != PMGPU_FP32) {
    set_error(caller, "precision unknown.");
    return -1;
  }
  int seen = 0;
  for (int i = 0; i < 3; i++) {
    if (patch->fft_seq[i] < 1 || patch->fft_seq[i] > 3) {
      set_error(caller, "fft direction unknown.");
      return -1;
    }
    seen |= 1 << patch->fft_seq[i];
  }
  if (seen != 0xE) {
    set_error(caller, "fft direction unknown.");
    return -1;
  }
  if (ensure_device(caller)) return -1;
  pmgpu_plan *pl = new pmgpu_plan();
  pl->prec = precision;
  pl->patch = *patch;
  pl->topo = *cuboid;
  pl->par = *par;
  pl->perm = nullptr;
  pl->perm_n = 0;
  double mdx = 0.0;
  int allper = 1;
  for (int e = 0; e < 3; e++) {
    const bool freeax = patch->bound_cond[e] == 0;
    pl->g.ext[e] = cuboid->ncell[e] + cuboid->nghost[2 * e] + cuboid->nghost[2 * e + 1];
    pl->g.off[e] = freeax ? 0 : cuboid->nghost[2 * e];
    pl->g.P[e] = freeax ? pl->g.ext[e] : cuboid->ncell[e];
    pl->g.M[e] = freeax ? 2 * pl->g.P[e] : pl->g.P[e];
    if (pl->g.M[e] % 2 != 0 || pl->g.M[e] < 2) {
      delete pl;
      set_error("pmlib_fft", "nfft is an odd number.");
      return -1;
    }
    if (freeax) allper = 0;
    mdx = std::max(mdx, patch->dx[e]);
  }
  pl->g.H = pl->g.M[0] / 2 + 1;
  pl->g.Hp = (pl->g.H + 7) / 8 * 8;
  pl->g.N2 = pl->g.M[0] / 2;
  pl->g.allper = allper;
  pl->eps = par->regularisation_radius * mdx;
  pl->green_mode = green_mode;
  pl->pff_kx0 = green_mode == 2 ? g_pff_kx0 : 0;
  const int rc = (precision == PMGPU_FP64) ? plan_tables<double>(pl, caller) : plan_tables<float>(pl, caller);
  if (rc) {
    delete pl;
    return -1;
  }
  *plan = pl;
  return 0;
}

int pmgpu_poisson_setup(const pmgpu_patch *patch, const pmgpu_topo *cuboid, const pmgpu_params *par,
                        int precision, pmgpu_plan **plan) {
  std::lock_guard<std::mutex> lk(g_setup_mu);
  return create_plan(patch, cuboid, par, precision, plan, "pmlib_poisson_setup");
}

int pmgpu_poisson_setup_ppf(const pmgpu_patch *patch, const pmgpu_topo *cuboid, const pmgpu_params *par,
                            int precision, pmgpu_plan **plan) {
  const char *caller = "pmlib_poisson_setup";
  std::lock_guard<std::mutex> lk(g_setup_mu);
  if (!patch || !par || !plan) {
    set_error(caller, "missing argument.");
    return -1;
  }
  if (!(patch->bound_cond[0] != 0 && patch->bound_cond[1] != 0 && patch->bound_cond[2] == 0)) {
    set_error(caller, "The spectral kernel needs periodic x and y and a free z.");
    return -1;
  }
  if (par->poisson_kernel == 2) {  // poisson_setup_ppf.f: no velocity kernel
    set_error(caller, "Velocity kernel is not implemented.");
    return -1;
  }
  if (par->poisson_order == 100) {
    set_error(caller, "Integration kernel unknown - change POISSON ORDER.");
    return -1;
  }
  return create_plan(patch, cuboid, par, precision, plan, caller, 1);
}

int pmgpu_poisson_setup_pff(const pmgpu_patch *patch, const pmgpu_topo *cuboid, const pmgpu_params *par,
                            int precision, int kx0, pmgpu_plan **plan) {
  const char *caller = "pmlib_poisson_setup";
  std::lock_guard<std::mutex> lk(g_setup_mu);
  if (!patch || !par || !plan) {
    set_error(caller, "missing argument.");
    return -1;
  }
  if (!(patch->bound_cond[0] != 0 && patch->bound_cond[1] == 0 && patch->bound_cond[2] == 0)) {
    set_error(caller, "The spectral kernel needs a periodic x and free y and z.");
    return -1;
  }
  if (par->poisson_kernel == 2) {  // poisson_setup_pff.f: no velocity kernel
    set_error(caller, "Velocity kernel is not implemented.");
    return -1;
  }
  if (par->poisson_order == 100) {
    set_error(caller, "Integration kernel unknown - change POISSON ORDER.");
    return -1;
  }
  if (kx0 != PMGPU_PFF_AS_WRITTEN && kx0 != PMGPU_PFF_LOG2D) {
    set_error(caller, "Unknown treatment of the kx = 0 plane.");
    return -1;
  }
  g_pff_kx0 = kx0;
  const int rc = create_plan(patch, cuboid, par, precision, plan, caller, 2);
  g_pff_kx0 = 0;
  return rc;
}

void pmgpu_plan_destroy(pmgpu_plan *plan) {
  std::lock_guard<std::mutex> lk(g_mu);
  delete plan;
}

template <typename R>
static int solve_host(pmgpu_plan *pl, R *vort, R *vel, R *vecpot, int reg_vort, int reproj, int calc_vecpot) {
  const char *caller = "pmlib_poisson_solve";
  std::lock_guard<std::mutex> lk(g_mu);
  if (!pl) {
    set_error(caller, "plan missing.");
    return -1;
  }
  if ((pl->prec == PMGPU_FP64) != (sizeof(R) == 8)) {
    set_error(caller, "plan precision does not match the arrays.");
    return -1;
  }
  if (ensure_device(caller)) return -1;
  const size_t nm = mesh_points(&pl->topo) * 3;
  const int ifft_vort = reg_vort || reproj;
  const int ifft_vecpot = calc_vecpot && pl->par.poisson_kernel == 1 && vecpot;
  if (pl->mesh_w.ensure(sizeof(R) * nm, caller) || pl->mesh_u.ensure(sizeof(R) * nm, caller)) return -1;
  if (ifft_vecpot && pl->mesh_a.ensure(sizeof(R) * nm, caller)) return -1;
  CK(cudaMemcpy(pl->mesh_w.p, vort, sizeof(R) * nm, cudaMemcpyHostToDevice), caller);
  if (run_solve<R>(pl, pl->mesh_w.as<R>(), pl->mesh_u.as<R>(), pl->mesh_w.as<R>(),
                   ifft_vecpot ? pl->mesh_a.as<R>() : nullptr, reg_vort, reproj, ifft_vecpot, 0, caller))
    return -1;
  CK(cudaMemcpy(vel, pl->mesh_u.p, sizeof(R) * nm, cudaMemcpyDeviceToHost), caller);
  if (ifft_vort) CK(cudaMemcpy(vort, pl->mesh_w.p, sizeof(R) * nm, cudaMemcpyDeviceToHost), caller);
  if (ifft_vecpot) CK(cudaMemcpy(vecpot, pl->mesh_a.p, sizeof(R) * nm, cudaMemcpyDeviceToHost), caller);
  return 0;
}

int pmgpu_poisson_solve_dev(pmgpu_plan *plan, void *d_vort, void *d_vel, void *d_vecpot, int reg_vort, int reproj,
                            int calc_vecpot, void *stream) {
  const char *caller = "pmlib_poisson_solve";
  std::lock_guard<std::mutex> lk(g_mu);
  if (!plan || !d_vort || !d_vel) {
    set_error(caller, "missing argument.");
    return -1;
  }
  if (ensure_device(caller)) return -1;
  const int vp = calc_vecpot && d_vecpot ? 1 : 0;
  cudaStream_t st = (cudaStream_t)stream;
  if (plan->prec == PMGPU_FP64)
    return run_solve<double>(plan, (const double *)d_vort, (double *)d_vel, (double *)d_vort, (double *)d_vecpot,
                             reg_vort, reproj, vp, st, caller);
  return run_solve<float>(plan, (const float *)d_vort, (float *)d_vel, (float *)d_vort, (float *)d_vecpot, reg_vort,
                          reproj, vp, st, caller);
}

int pmgpu_poisson_solve(pmgpu_plan *plan, double *vort, double *vel, double *vecpot, int reg_vort, int reproj,
                        int calc_vecpot) {
  return solve_host<double>(plan, vort, vel, vecpot, reg_vort, reproj, calc_vecpot);
}
int pmgpu_poisson_solve_f32(pmgpu_plan *plan, float *vort, float *vel, float *vecpot, int reg_vort, int reproj,
                            int calc_vecpot) {
  return solve_host<float>(plan, vort, vel, vecpot, reg_vort, reproj, calc_vecpot);
}

template <typename R>
static int regularise_host(pmgpu_plan *pl, R *mesh, int nvar, int reg_order, double fw) {
  const char *caller = "pmlib_regularise";
  std::lock_guard<std::mutex> lk(g_mu);
  if (!pl) {
    set_error(caller, "plan missing.");
    return -1;
  }
  if ((pl->prec == PMGPU_FP64) != (sizeof(R) == 8)) {
    set_error(caller, "plan precision does not match the arrays.");
    return -1;
  }
  if (nvar > 3) {
    set_error(caller, "Cant regularise variables of ndim > 3.");
    return -1;
  }
  if (nvar < 1 || (reg_order != 0 && reg_order != 2 && reg_order != 4 && reg_order != 6 && reg_order != 8 &&
                   reg_order != 10)) {
    set_error(caller, "Regularisation order unknown.");
    return -1;
  }
  if (ensure_device(caller)) return -1;
  const size_t nm = mesh_points(&pl->topo) * nvar;
  if (pl->mesh_w.ensure(sizeof(R) * nm, caller)) return -1;
  CK(cudaMemcpy(pl->mesh_w.p, mesh, sizeof(R) * nm, cudaMemcpyHostToDevice), caller);
  if (run_regularise<R>(pl, pl->mesh_w.as<R>(), nvar, reg_order, fw, 0, caller)) return -1;
  CK(cudaMemcpy(mesh, pl->mesh_w.p, sizeof(R) * nm, cudaMemcpyDeviceToHost), caller);
  return 0;
}

int pmgpu_regularise(pmgpu_plan *plan, double *mesh, int nvar, int reg_order, double filter_width) {
  return regularise_host<double>(plan, mesh, nvar, reg_order, filter_width);
}
int pmgpu_regularise_f32(pmgpu_plan *plan, float *mesh, int nvar, int reg_order, double filter_width) {
  return regularise_host<float>(plan, mesh, nvar, reg_order, filter_width);
}

// ------------------------------------------------------------------ the step
template <typename R>
static int step_dev(pmgpu_plan *pl, const R *pos, const R *pv, int n, R *pvel, cudaStream_t st) {
  const char *caller = "pmgpu_step";
  const size_t nm = mesh_points(&pl->topo) * 3;
  if (pl->mesh_w.ensure(sizeof(R) * nm, caller) || pl->mesh_u.ensure(sizeof(R) * nm, caller)) return -1;
  pmgpu_topo t = pl->topo;
  t.npart = n;
  PartScratchRefs r{&pl->key, &pl->val, &pl->key2, &pl->val2, &pl->counts, &pl->start, &pl->spart, &pl->hist};
  const int *perm = nullptr;
  if (run_p2m<R>(&t, pl->par.interpolation_order, pos, pv, 3, n, pl->mesh_w.as<R>(), 3, 1, r, st, &perm, caller))
    return -1;
  if (run_solve<R>(pl, pl->mesh_w.as<R>(), pl->mesh_u.as<R>(), nullptr, nullptr, 0, 0, 0, st, caller)) return -1;
  if (run_m2p_sorted<R>(&t, pl->par.interpolation_order, pos, pl->start.as<unsigned>(), perm, n,
                        pl->mesh_u.as<R>(), pvel, st, caller))
    return -1;
  return 0;
}

int pmgpu_step_dev(pmgpu_plan *plan, const void *d_pos, const void *d_part_vort, int npart, void *d_part_vel,
                   void *stream) {
  const char *caller = "pmgpu_step";
  std::lock_guard<std::mutex> lk(g_mu);
  if (!plan) {
    set_error(caller, "plan missing.");
    return -1;
  }
  if (ensure_device(caller)) return -1;
  cudaStream_t st = (cudaStream_t)stream;
  if (plan->prec == PMGPU_FP64)
    return step_dev<double>(plan, (const double *)d_pos, (const double *)d_part_vort, npart, (double *)d_part_vel, st);
  return step_dev<float>(plan, (const float *)d_pos, (const float *)d_part_vort, npart, (float *)d_part_vel, st);
}

// Grows every buffer a step of up to n particles uses, so that steps queued on other
// streams never reallocate (a reallocation frees on the legacy stream).
template <typename R> static int ensure_step_scratch(pmgpu_plan *pl, int n, const char *caller) {
  const size_t nm = mesh_points(&pl->topo) * 3;
  const int W = pl->par.interpolation_order == 3 ? 4 : 6;
  PartGeom<R> g = part_geom<R>(&pl->topo, W);
  const size_t nn = (size_t)std::max(n, 1);
  typedef typename cplx_t<R>::type C;
  const Geometry &G = pl->g;
  const size_t nX = (size_t)G.P[1] * G.P[2] * G.Hp * 3, nY = (size_t)G.M[1] * G.P[2] * G.Hp * 3;
  if (pl->mesh_w.ensure(sizeof(R) * nm, caller) || pl->mesh_u.ensure(sizeof(R) * nm, caller) ||
      pl->X.ensure(sizeof(C) * nX, caller) || pl->Y.ensure(sizeof(C) * nY, caller) ||
      pl->key.ensure(sizeof(unsigned) * nn, caller) || pl->val.ensure(sizeof(unsigned) * nn, caller) ||
      pl->key2.ensure(sizeof(int) * nn, caller) || pl->val2.ensure(sizeof(int) * nn, caller) ||
      pl->hist.ensure(sizeof(unsigned) * (nn / (FIX_SMALL + 1) + 2), caller) ||
      pl->counts.ensure(sizeof(unsigned) * (g.nbins + 1), caller) ||
      pl->start.ensure(sizeof(unsigned) * (g.nbins + 1), caller))
    return -1;
  const size_t nb = (g.nbins + 1 + SCAN_TILE - 1) / SCAN_TILE;
  return pl->spart.ensure(sizeof(unsigned) * (nb + 1), caller);
}

int pmgpu_step_many(pmgpu_plan *plan, int nsteps, const void *const *pos, const void *const *part_vort,
                    const int *npart, void *const *part_vel) {
  const char *caller = "pmgpu_step";
  std::lock_guard<std::mutex> lk(g_mu);
  if (!plan || nsteps < 0 || (nsteps > 0 && (!pos || !part_vort || !npart || !part_vel))) {
    set_error(caller, "missing argument.");
    return -1;
  }
  if (ensure_device(caller)) return -1;
  int nmax = 0;
  for (int i = 0; i < nsteps; i++) {
    if (npart[i] < 0 || (npart[i] > 0 && (!pos[i] || !part_vort[i] || !part_vel[i]))) {
      set_error(caller, "missing argument.");
      return -1;
    }
    nmax = std::max(nmax, npart[i]);
  }
  const bool f64 = plan->prec == PMGPU_FP64;
  const size_t es = f64 ? 8 : 4;
  if ((f64 ? ensure_step_scratch<double>(plan, nmax, caller) : ensure_step_scratch<float>(plan, nmax, caller)))
    return -1;
  StepPipe &P = plan->pipe;
  if (!P.s[0]) {
    for (int i = 0; i < 3; i++) CK(cudaStreamCreateWithFlags(&P.s[i], cudaStreamNonBlocking), caller);
    for (int i = 0; i < 2; i++) {
      CK(cudaEventCreateWithFlags(&P.h2d[i], cudaEventDisableTiming), caller);
      CK(cudaEventCreateWithFlags(&P.comp[i], cudaEventDisableTiming), caller);
      CK(cudaEventCreateWithFlags(&P.d2h[i], cudaEventDisableTiming), caller);
    }
  }
  const size_t nb = es * 3 * (size_t)std::max(nmax, 1);
  for (int i = 0; i < 2; i++)
    if (P.pos[i].ensure(nb, caller) || P.val[i].ensure(nb, caller) || P.out[i].ensure(nb, caller)) return -1;
  cudaStream_t sh = P.s[0], sc = P.s[1], sd = P.s[2];
  for (int i = 0; i < nsteps; i++) {
    const int b = i & 1, n = npart[i];
    const size_t bytes = es * 3 * (size_t)n;
    // the slot's inputs are free once step i-2 has computed, its output once copied out
    if (i >= 2) CK(cudaStreamWaitEvent(sh, P.comp[b], 0), caller);
    if (n > 0) {
      CK(cudaMemcpyAsync(P.pos[b].p, pos[i], bytes, cudaMemcpyHostToDevice, sh), caller);
      CK(cudaMemcpyAsync(P.val[b].p, part_vort[i], bytes, cudaMemcpyHostToDevice, sh), caller);
    }
    CK(cudaEventRecord(P.h2d[b], sh), caller);
    CK(cudaStreamWaitEvent(sc, P.h2d[b], 0), caller);
    if (i >= 2) CK(cudaStreamWaitEvent(sc, P.d2h[b], 0), caller);
    const int rc = f64 ? step_dev<double>(plan, P.pos[b].as<double>(), P.val[b].as<double>(), n,
                                          P.out[b].as<double>(), sc)
                       : step_dev<float>(plan, P.pos[b].as<float>(), P.val[b].as<float>(), n, P.out[b].as<float>(), sc);
    if (rc) {
      cudaStreamSynchronize(sh);
      cudaStreamSynchronize(sc);
      cudaStreamSynchronize(sd);
      return -1;
    }
    CK(cudaEventRecord(P.comp[b], sc), caller);
    CK(cudaStreamWaitEvent(sd, P.comp[b], 0), caller);
    if (n > 0) CK(cudaMemcpyAsync(part_vel[i], P.out[b].p, bytes, cudaMemcpyDeviceToHost, sd), caller);
    CK(cudaEventRecord(P.d2h[b], sd), caller);
  }
  CK(cudaStreamSynchronize(sd), caller);
  CK(cudaStreamSynchronize(sc), caller);
  CK(cudaStreamSynchronize(sh), caller);
  return 0;
}

int pmgpu_step(pmgpu_plan *plan, const void *pos, const void *part_vort, int npart, void *part_vel) {
  const char *caller = "pmgpu_step";
  std::lock_guard<std::mutex> lk(g_mu);
  if (!plan) {
    set_error(caller, "plan missing.");
    return -1;
  }
  if (ensure_device(caller)) return -1;
  const size_t es = plan->prec == PMGPU_FP64 ? 8 : 4;
  const size_t nb = es * 3 * (size_t)std::max(npart, 1);
  if (plan->h_pos.ensure(nb, caller) || plan->h_val.ensure(nb, caller) || plan->h_out.ensure(nb, caller)) return -1;
  cudaStream_t st = 0;
  if (npart > 0) {
    CK(cudaMemcpyAsync(plan->h_pos.p, pos, es * 3 * (size_t)npart, cudaMemcpyHostToDevice, st), caller);
    CK(cudaMemcpyAsync(plan->h_val.p, part_vort, es * 3 * (size_t)npart, cudaMemcpyHostToDevice, st), caller);
  }
  int rc;
  if (plan->prec == PMGPU_FP64)
    rc = step_dev<double>(plan, plan->h_pos.as<double>(), plan->h_val.as<double>(), npart, plan->h_out.as<double>(), st);
  else
    rc = step_dev<float>(plan, plan->h_pos.as<float>(), plan->h_val.as<float>(), npart, plan->h_out.as<float>(), st);
  if (rc) return -1;
  if (npart > 0) CK(cudaMemcpyAsync(part_vel, plan->h_out.p, es * 3 * (size_t)npart, cudaMemcpyDeviceToHost, st), caller);
  CK(cudaStreamSynchronize(st), caller);
  return 0;
}

// ------------------------------------------------------------------ remesh
int pmgpu_remesh(const pmgpu_topo *topo, const double *mesh_vort, const double *mesh_dvort, const double *mesh_vel,
                 const unsigned char *mask, double min_vort, double min_dvort, int incl_ghost, int max_part,
                 double *pos, double *part_vort, double *part_dvort, double *part_vel, int *npart) {
  const char *caller = "pmlib_remesh_particles";
  std::lock_guard<std::mutex> lk(g_mu);
  if (!topo || !mesh_vort || !npart) {
    set_error(caller, "missing argument.");
    return -1;
  }
  if (ensure_device(caller)) return -1;
  Scratch &s = scratch();
  const size_t nc = mesh_points(topo);
  PartGeom<double> g = part_geom<double>(topo, 4);
  if (s.c.ensure(sizeof(double) * 3 * nc, caller) || s.counts.ensure(sizeof(unsigned) * (nc + 1), caller) ||
      s.start.ensure(sizeof(unsigned) * (nc + 1), caller))
    return -1;
  CK(cudaMemcpy(s.c.p, mesh_vort, sizeof(double) * 3 * nc, cudaMemcpyHostToDevice), caller);
  const double *ddv = nullptr, *dvel = nullptr;
  const unsigned char *dmask = nullptr;
  if (mesh_dvort) {
    if (s.d.ensure(sizeof(double) * 3 * nc, caller)) return -1;
    CK(cudaMemcpy(s.d.p, mesh_dvort, sizeof(double) * 3 * nc, cudaMemcpyHostToDevice), caller);
    ddv = s.d.as<double>();
  }
  if (mesh_vel) {
    if (s.e.ensure(sizeof(double) * 3 * nc, caller)) return -1;
    CK(cudaMemcpy(s.e.p, mesh_vel, sizeof(double) * 3 * nc, cudaMemcpyHostToDevice), caller);
    dvel = s.e.as<double>();
  }
  if (mask) {
    if (s.h.ensure(nc, caller)) return -1;
    CK(cudaMemcpy(s.h.p, mask, nc, cudaMemcpyHostToDevice), caller);
    dmask = s.h.as<unsigned char>();
  }
  const int nblk = (int)std::min<size_t>((nc + 255) / 256, 148 * 32);
  CK(cudaMemset(s.counts.p, 0, sizeof(unsigned) * (nc + 1)), caller);
  k_remesh_flag<double><<<nblk, 256>>>(g, s.c.as<double>(), ddv, dmask, min_vort, min_dvort, incl_ghost,
                                       s.counts.as<unsigned>());
  PM_LAUNCHED();
  CKL(caller);
  if (exclusive_scan(s.counts.as<unsigned>(), s.start.as<unsigned>(), nc + 1, s.spart, 0, caller)) return -1;
  unsigned total = 0;
  CK(cudaMemcpy(&total, s.start.as<unsigned>() + nc, sizeof(unsigned), cudaMemcpyDeviceToHost), caller);
  *npart = (int)total;
  if (!pos) return 0;
  if ((int)total > max_part) {
    set_error(caller, "particle arrays too small.");
    return -1;
  }
  const size_t np3 = 3 * (size_t)std::max<unsigned>(total, 1);
  if (s.f.ensure(sizeof(double) * np3 * 4, caller)) return -1;
  double *dpos = s.f.as<double>(), *dpv = dpos + np3, *dpdv = dpv + np3, *dpvel = dpdv + np3;
  k_remesh_fill<double><<<nblk, 256>>>(g, s.c.as<double>(), ddv, dvel, s.counts.as<unsigned>(),
                                       s.start.as<unsigned>(), dpos, dpv, dpdv, dpvel);
  PM_LAUNCHED();
  CKL(caller);
  if (total > 0) {
    const size_t b = sizeof(double) * 3 * (size_t)total;
    CK(cudaMemcpy(pos, dpos, b, cudaMemcpyDeviceToHost), caller);
    if (part_vort) CK(cudaMemcpy(part_vort, dpv, b, cudaMemcpyDeviceToHost), caller);
    if (part_dvort) CK(cudaMemcpy(part_dvort, dpdv, b, cudaMemcpyDeviceToHost), caller);
    if (part_vel) CK(cudaMemcpy(part_vel, dpvel, b, cudaMemcpyDeviceToHost), caller);
  }
  return 0;
}


// ------------------------------------------------------------------ allocation-free P2M
// Some callers cannot allocate device memory while they run: a host program that
// reserved the GPU's memory up front (a fixed-budget pool or another runtime owning
// the allocator), or a loop that must not risk the implicit synchronisation and
// failure modes of cudaMalloc / cudaFree.  This variant of the deposition keeps all
// of its scratch (bin keys, particle order, bin counts and starts, the list of
// crowded bins) in one static device array, and takes only device pointers from the
// caller.  The module loads lazily, so the array exists on a device only once code
// of this file has been used there: the library's first call on a device (any entry
// point) looks up its address, which makes the driver reserve it then.
namespace pmgpu {
constexpr size_t NOALLOC_MAX_PART = size_t(1) << 18;  // particles per call
constexpr size_t NOALLOC_MAX_BINS = size_t(1) << 19;  // (nx' + 3)(ny' + 3)(nz' + 3) for M4'
constexpr size_t NA_PART_BYTES = NOALLOC_MAX_PART * 4;
constexpr size_t NA_BIN_BYTES = (NOALLOC_MAX_BINS + 256) * 4;
// the overflow list of the stable fix-up: a count and the bins that hold more than
// FIX_SMALL particles, at most NOALLOC_MAX_PART / (FIX_SMALL + 1) of them
constexpr size_t NA_HIST_BYTES = ((NOALLOC_MAX_PART / (FIX_SMALL + 1) + 2) * 4 + 255) / 256 * 256;
constexpr size_t NA_SPART_BYTES = size_t(1) << 12;
constexpr size_t NOALLOC_BYTES = 4 * NA_PART_BYTES + 2 * NA_BIN_BYTES + NA_HIST_BYTES + NA_SPART_BYTES;
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_BYTES];
static void *g_noalloc_addr[128];

// once per device, with that device current: the host-side symbol is only a
// stand-in, the kernels need the device address of the array
static int noalloc_reserve(int dev, const char *caller) {
  if (dev < 0 || dev >= 128 || g_noalloc_addr[dev]) return 0;
  void *ptr = nullptr;
  CK(cudaGetSymbolAddress(&ptr, g_noalloc_scratch), caller);
  g_noalloc_addr[dev] = ptr;
  return 0;
}
}  // namespace pmgpu

int pmgpu_interp_particle_mesh_noalloc(const pmgpu_topo *topo, const pmgpu_params *par, const double *d_xpart,
                                       const double *d_part, int nvar, int npart, double *d_mesh, int nvar_mesh,
                                       int clear, int clear_ghost, void *stream) {
  const char *caller = "pmlib_interp_particle_mesh";
  std::lock_guard<std::mutex> lk(g_mu);
  if (!topo) {
    set_error(caller, "missing argument.");
    return -1;
  }
  if (nvar != nvar_mesh) {
    set_error(caller, "Dimension of interpolation variables does not correspond.");
    return -1;
  }
  if (topo->npart != npart) {
    set_error(caller, "Discrepancy in number of particles");
    return -1;
  }
  if (check_interp(par, caller)) return -1;
  const int W = par->interpolation_order == 3 ? 4 : 6;
  unsigned long long nbins = 1;
  for (int e = 0; e < 3; e++)
    nbins *= (unsigned long long)(topo->ncell[e] + topo->nghost[2 * e] + topo->nghost[2 * e + 1] + W - 1);
  if (npart < 0 || (size_t)npart > NOALLOC_MAX_PART || nbins > NOALLOC_MAX_BINS) {
    char msg[200];
    snprintf(msg, sizeof(msg),
             "allocation-free deposition is limited to %zu particles and %zu bins (got %d particles, %llu bins).",
             (size_t)NOALLOC_MAX_PART, (size_t)NOALLOC_MAX_BINS, npart, nbins);
    set_error(caller, msg);
    return -1;
  }
  if (ensure_device(caller)) return -1;
  int dev = 0;
  CK(cudaGetDevice(&dev), caller);
  if (dev < 0 || dev >= 128) {
    set_error(caller, "device index out of range.");
    return -1;
  }
  if (noalloc_reserve(dev, caller)) return -1;
  unsigned char *base = reinterpret_cast<unsigned char *>(g_noalloc_addr[dev]);
  DevBuf key, val, key2, val2, counts, start, spart, hist;
  DevBuf *views[] = {&key, &val, &key2, &val2};
  size_t off = 0;
  for (DevBuf *v : views) {
    v->p = base + off;
    v->cap = NA_PART_BYTES;
    v->fixed = true;
    off += NA_PART_BYTES;
  }
  DevBuf *bviews[] = {&counts, &start};
  for (DevBuf *v : bviews) {
    v->p = base + off;
    v->cap = NA_BIN_BYTES;
    v->fixed = true;
    off += NA_BIN_BYTES;
  }
  hist.p = base + off;
  hist.cap = NA_HIST_BYTES;
  hist.fixed = true;
  off += NA_HIST_BYTES;
  spart.p = base + off;
  spart.cap = NA_SPART_BYTES;
  spart.fixed = true;
  PartScratchRefs r{&key, &val, &key2, &val2, &counts, &start, &spart, &hist};
  const int mode = clear ? 1 : (clear_ghost ? 2 : 0);
  return run_p2m<double>(topo, par->interpolation_order, d_xpart, d_part, nvar, npart, d_mesh, nvar_mesh, mode, r,
                         (cudaStream_t)stream, nullptr, caller);
}

int pmgpu_fft_engine(int engine) {
  std::lock_guard<std::mutex> lk(g_setup_mu);
  const int old = g_force_stockham;
  g_force_stockham = engine == 1 ? 1 : 0;
  return old;
}

namespace pmgpu {
int g_fft_ct = 1;
}

int pmgpu_fft_specialised(int on) {
  std::lock_guard<std::mutex> lk(g_mu);
  const int old = g_fft_ct;
  g_fft_ct = on ? 1 : 0;
  return old;
}

// ------------------------------------------------------------------ batches of patches
// Independent solves of patches of uneven sizes and boundary types.  Each patch has
// its own plan (work buffers; the Green's spectra are shared through the cache when
// grids coincide).  Patches are spread over a few internal streams, largest first
// onto the least loaded stream, so small solves overlap on the device; the whole
// batch is captured once into a CUDA graph and replayed while the caller passes the
// same arrays on the same stream.
static int g_batch_fuse = 1;  // batches made while set run the batched passes

struct pmgpu_batch {
  int prec = 0;
  std::vector<pmgpu_plan *> plans;
  // the batched passes: one launch per pass family over the tiles of every patch
  // (unless a patch needs the Stockham fallback or there are more than BATCH_MAX
  // patches: then each patch runs its own passes on the internal streams)
  bool fused = false;
  pmgpu::BatchLayout lay;
  DevBuf desc, counters;
  std::vector<int> lane;  // internal stream of each patch
  std::vector<cudaStream_t> aux;
  std::vector<cudaEvent_t> ev;  // [0] fork, [1 + k] join of stream k
  bool warm = false;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaStream_t gstream = nullptr;
  std::vector<void *> gptr;  // arrays the graph was captured with
  ~pmgpu_batch() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    for (cudaEvent_t e : ev) cudaEventDestroy(e);
    for (cudaStream_t s : aux) cudaStreamDestroy(s);
    for (pmgpu_plan *p : plans) delete p;
    desc.release();
    counters.release();
  }
};

namespace pmgpu {
// sets up the batched passes: every plan's work spectra, then the descriptors of
// the five pass families in device memory; leaves b->fused false when a patch needs
// a pass the batched kernels do not run
template <typename R> static int batch_fuse(pmgpu_batch *b, const char *caller) {
  typedef typename cplx_t<R>::type C;
  const int n = (int)b->plans.size();
  std::vector<SolveGeom<R>> geo(n);
  std::vector<C *> X(n), Y(n);
  std::vector<const pmgpu_topo *> topo(n);
  for (int i = 0; i < n; i++) {
    pmgpu_plan *pl = b->plans[i];
    geo[i] = solve_geom<R>(pl);
    const size_t nX = (size_t)geo[i].P[1] * geo[i].P[2] * geo[i].Hp * 3;
    const size_t nY = (size_t)geo[i].M[1] * geo[i].P[2] * geo[i].Hp * 3;
    if (pl->X.ensure(sizeof(C) * nX, caller) || pl->Y.ensure(sizeof(C) * nY, caller)) return -1;
    X[i] = pl->X.as<C>();
    Y[i] = pl->Y.as<C>();
    topo[i] = &pl->topo;
  }
  std::vector<unsigned char> host;
  if (batch_layout<R, 3>(n, geo.data(), X.data(), Y.data(), topo.data(), host, b->lay, caller)) return 0;
  if (b->desc.ensure(host.size(), caller) || b->counters.ensure(5 * sizeof(unsigned), caller)) return -1;
  CK(cudaMemcpy(b->desc.p, host.data(), host.size(), cudaMemcpyHostToDevice), caller);
  b->fused = true;
  return 0;
}

// queue every patch's solve: the batched passes, or each patch's own passes with the
// internal streams forked off `st` and joined back
static int batch_enqueue(pmgpu_batch *b, void *const *d_vort, void *const *d_vel, cudaStream_t st,
                         const char *caller) {
  if (b->fused)
    return b->prec == PMGPU_FP64
               ? batch_launch<double, 3>(b->lay, b->desc.p, b->counters.as<unsigned>(), d_vort, d_vel, st, caller)
               : batch_launch<float, 3>(b->lay, b->desc.p, b->counters.as<unsigned>(), d_vort, d_vel, st, caller);
  CK(cudaEventRecord(b->ev[0], st), caller);
  for (cudaStream_t s : b->aux) CK(cudaStreamWaitEvent(s, b->ev[0], 0), caller);
  for (size_t i = 0; i < b->plans.size(); i++) {
    pmgpu_plan *pl = b->plans[i];
    cudaStream_t s = b->aux[b->lane[i]];
    const int rc = b->prec == PMGPU_FP64
                       ? run_solve<double>(pl, (const double *)d_vort[i], (double *)d_vel[i], nullptr, nullptr, 0, 0,
                                           0, s, caller)
                       : run_solve<float>(pl, (const float *)d_vort[i], (float *)d_vel[i], nullptr, nullptr, 0, 0, 0,
                                          s, caller);
    if (rc) return -1;
  }
  for (size_t k = 0; k < b->aux.size(); k++) {
    CK(cudaEventRecord(b->ev[1 + k], b->aux[k]), caller);
    CK(cudaStreamWaitEvent(st, b->ev[1 + k], 0), caller);
  }
  return 0;
}
}  // namespace pmgpu

int pmgpu_batch_create(int npatch, const pmgpu_patch *patches, const pmgpu_topo *cuboids,
                       const pmgpu_params *par, int precision, pmgpu_batch **batch) {
  const char *caller = "pmgpu_batch_create";
  std::lock_guard<std::mutex> lk(g_mu);
  std::lock_guard<std::mutex> lk2(g_setup_mu);  // it creates plans
  if (!batch || npatch <= 0 || !patches || !cuboids) {
    set_error(caller, "missing argument.");
    return -1;
  }
  *batch = nullptr;
  pmgpu_batch *b = new pmgpu_batch();
  b->prec = precision;
  for (int i = 0; i < npatch; i++) {
    pmgpu_plan *pl = nullptr;
    if (create_plan(&patches[i], &cuboids[i], par, precision, &pl, caller)) {
      delete b;
      return -1;
    }
    b->plans.push_back(pl);
  }
  const int ns = std::min(npatch, 8);
  std::vector<int> order(npatch);
  for (int i = 0; i < npatch; i++) order[i] = i;
  auto work = [&](int i) {
    const Geometry &G = b->plans[i]->g;
    return (double)G.M[0] * G.M[1] * G.M[2];
  };
  std::sort(order.begin(), order.end(), [&](int a, int c) { return work(a) > work(c); });
  std::vector<double> load(ns, 0.0);
  b->lane.assign(npatch, 0);
  for (int i : order) {
    const int k = (int)(std::min_element(load.begin(), load.end()) - load.begin());
    b->lane[i] = k;
    load[k] += work(i);
  }
  b->aux.resize(ns);
  b->ev.resize(ns + 1);
  for (int k = 0; k < ns; k++)
    if (!cuda_ok(cudaStreamCreateWithFlags(&b->aux[k], cudaStreamNonBlocking), caller)) {
      b->aux.resize(k);
      delete b;
      return -1;
    }
  for (int k = 0; k <= ns; k++)
    if (!cuda_ok(cudaEventCreateWithFlags(&b->ev[k], cudaEventDisableTiming), caller)) {
      b->ev.resize(k);
      delete b;
      return -1;
    }
  if (g_batch_fuse) {
    const int rc = precision == PMGPU_FP64 ? batch_fuse<double>(b, caller) : batch_fuse<float>(b, caller);
    if (rc) {
      delete b;
      return -1;
    }
  }
  *batch = b;
  return 0;
}

int pmgpu_batch_fused(const pmgpu_batch *b) { return b && b->fused ? 1 : 0; }

int pmgpu_batch_mode(int fused) {
  std::lock_guard<std::mutex> lk(g_mu);
  const int old = g_batch_fuse;
  g_batch_fuse = fused ? 1 : 0;
  return old;
}

int pmgpu_batch_solve(pmgpu_batch *b, void *const *d_vort, void *const *d_vel, void *stream) {
  const char *caller = "pmgpu_batch_solve";
  std::lock_guard<std::mutex> lk(g_mu);
  if (!b || !d_vort || !d_vel) {
    set_error(caller, "missing argument.");
    return -1;
  }
  if (ensure_device(caller)) return -1;
  cudaStream_t st = (cudaStream_t)stream;
  const size_t np = b->plans.size();
  std::vector<void *> ptrs(d_vort, d_vort + np);
  ptrs.insert(ptrs.end(), d_vel, d_vel + np);
  if (b->exec && b->gstream == st && b->gptr == ptrs) {
    CK(cudaGraphLaunch(b->exec, st), caller);
    return 0;
  }
  if (!b->warm || st == nullptr) {
    // first call (allocates the work buffers) or the legacy stream: run directly
    if (batch_enqueue(b, d_vort, d_vel, st, caller)) return -1;
    b->warm = true;
    return 0;
  }
  if (b->exec) {
    cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
  }
  if (b->graph) {
    cudaGraphDestroy(b->graph);
    b->graph = nullptr;
  }
  CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed), caller);
  const int rc = batch_enqueue(b, d_vort, d_vel, st, caller);
  cudaGraph_t g = nullptr;
  const cudaError_t e = cudaStreamEndCapture(st, &g);
  if (rc || e != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    if (!rc) cuda_ok(e, caller);
    return -1;
  }
  b->graph = g;
  CK(cudaGraphInstantiate(&b->exec, g, 0), caller);
  b->gstream = st;
  b->gptr = ptrs;
  CK(cudaGraphLaunch(b->exec, st), caller);
  return 0;
}

int pmgpu_batch_size(const pmgpu_batch *b) { return b ? (int)b->plans.size() : 0; }

pmgpu_plan *pmgpu_batch_plan(pmgpu_batch *b, int i) {
  if (!b || i < 0 || i >= (int)b->plans.size()) return nullptr;
  return b->plans[i];
}

void pmgpu_batch_destroy(pmgpu_batch *b) {
  std::lock_guard<std::mutex> lk(g_mu);
  delete b;
}

int pmgpu_fft_tune(int on) {
  std::lock_guard<std::mutex> lk(g_setup_mu);
  const int old = g_tune;
  g_tune = on ? 1 : 0;
  return old;
}

int pmgpu_fft_tuned(int index, int *length, int *precision, int *axis, int *radices, int *tile, double *ms) {
  std::lock_guard<std::mutex> lk(g_setup_mu);
  if (index < 0 || index >= (int)g_tuned.size()) return -1;
  auto it = g_tuned.begin();
  std::advance(it, index);
  if (length) *length = std::get<0>(it->first);
  if (precision) *precision = std::get<1>(it->first) == 8 ? PMGPU_FP64 : PMGPU_FP32;
  if (axis) *axis = std::get<2>(it->first);
  if (radices)
    for (int i = 0; i < 3; i++) radices[i] = i < it->second.np ? it->second.r[i] : 0;
  if (tile) *tile = it->second.tk;
  if (ms) *ms = it->second.ms;
  return 0;
}

int pmgpu_fft_set_schedule(int length, int precision, int axis, const int *radices, int tile) {
  const char *caller = "pmgpu_fft_set_schedule";
  std::lock_guard<std::mutex> lk(g_setup_mu);
  if ((precision != PMGPU_FP32 && precision != PMGPU_FP64) || (axis != 1 && axis != 2) || length < 2) {
    set_error(caller, "length, precision or axis out of range.");
    return -1;
  }
  const auto key = std::make_tuple(length, precision == PMGPU_FP64 ? 8 : 4, axis);
  if (!radices) {
    g_tuned.erase(key);
    return 0;
  }
  TunedSchedule ts;
  ts.np = 0;
  long long prod = 1;
  for (int i = 0; i < 3 && radices[i] > 0; i++) {
    const int r = radices[i];
    if (!(reg_radix(r) || (precision == PMGPU_FP32 && reg_radix_wide(r)))) {
      set_error(caller, "radix not available.");
      return -1;
    }
    ts.r[ts.np++] = r;
    prod *= r;
  }
  for (int i = ts.np; i < 3; i++) ts.r[i] = 0;
  if (ts.np == 0 || prod != length || (tile != 0 && tile != 1 && tile != 2 && tile != 4 && tile != 8)) {
    set_error(caller, "radices do not multiply to the length, or tile not in {0, 1, 2, 4, 8}.");
    return -1;
  }
  ts.tk = tile;
  ts.ms = 0.0;
  g_tuned[key] = ts;
  return 0;
}

// ------------------------------------------------------------------ diagnostics
int pmgpu_particle_diagnostics(const double dx[3], const void *d_pos, const void *d_vel, const void *d_vort,
                               int npart, int precision, double out[14], void *stream) {
  const char *caller = "pmgpu_particle_diagnostics";
  std::lock_guard<std::mutex> lk(g_mu);
  if (!dx || !out || npart < 0 || (npart > 0 && (!d_pos || !d_vel || !d_vort))) {
    set_error(caller, "missing argument.");
    return -1;
  }
  if (ensure_device(caller)) return -1;
  Scratch &s = scratch();
  const int nblk = 2 * num_sms();
  if (s.diag.ensure(sizeof(double) * ((size_t)nblk * DIAG_N + DIAG_N), caller)) return -1;
  double *part = s.diag.as<double>(), *dout = part + (size_t)nblk * DIAG_N;
  cudaStream_t st = (cudaStream_t)stream;
  const double dv = dx[0] * dx[1] * dx[2];
  if (precision == PMGPU_FP64)
    k_diag_partial<double><<<nblk, DIAG_THREADS, 0, st>>>((const double *)d_pos, (const double *)d_vel,
                                                          (const double *)d_vort, npart, dv, part);
  else
    k_diag_partial<float><<<nblk, DIAG_THREADS, 0, st>>>((const float *)d_pos, (const float *)d_vel,
                                                         (const float *)d_vort, npart, dv, part);
  PM_LAUNCHED();
  k_diag_final<<<1, 32, 0, st>>>(part, nblk, dout);
  PM_LAUNCHED();
  CKL(caller);
  double h[DIAG_N];
  CK(cudaMemcpyAsync(h, dout, sizeof(h), cudaMemcpyDeviceToHost, st), caller);
  CK(cudaStreamSynchronize(st), caller);
  for (int i = 0; i < DIAG_N; i++) out[i] = h[i];
  if (h[7] > 0.0) {
    for (int i = 9; i < 13; i++) out[i] = h[i] / h[7];  // centroid and ring radius (diagnostics_knot.f:171-175)
  }
  return 0;
}

// ------------------------------------------------------------------ particle step around the solve
// dvort = visc lap(vort) + (vort . grad) vel on the interior, then the periodic ghost
// map (the client's part_deriv_vorticity, vortex_structures/source/particle_derivatives/
// part_deriv_vorticity.f:57-206) on device meshes (3, nx', ny', nz')
template <typename R>
static int run_deriv_vorticity(const pmgpu_topo *t, int fd_order, double visc, const R *vort, const R *vel, R *dvort,
                               cudaStream_t st, const char *caller) {
  if (fd_order != 2 && fd_order != 4) {
    set_error("pmlib_parameters_check", "pmlib_fd_order is incorrectly set.");
    return -1;
  }
  DerivGeom<R> g;
  for (int e = 0; e < 3; e++) {
    g.ext[e] = t->ncell[e] + t->nghost[2 * e] + t->nghost[2 * e + 1];
    g.ngl[e] = t->nghost[2 * e];
    g.nc[e] = t->ncell[e];
    if (t->nghost[2 * e] < fd_order / 2 || t->nghost[2 * e + 1] < fd_order / 2) {
      set_error(caller, "Too few ghost cells for the finite differences.");
      return -1;
    }
    g.c_1_dx2[e] = R(1) / ((R)t->dx[e] * (R)t->dx[e]);
    g.c_1_2dx[e] = R(1) / (R(2) * (R)t->dx[e]);
  }
  g.visc = (R)visc;
  if (g.nc[0] > 0 && g.nc[1] > 0 && g.nc[2] > 0) {
    const dim3 blk(32, 8), grid((g.nc[0] + 31) / 32, (g.nc[1] + 7) / 8, g.nc[2]);
    KTimer kt_(KC_DERIV, st);
    if (fd_order == 2) k_deriv_vorticity<R, 2><<<grid, blk, 0, st>>>(g, vort, vel, dvort);
    else k_deriv_vorticity<R, 4><<<grid, blk, 0, st>>>(g, vort, vel, dvort);
    PM_LAUNCHED();
    CKL(caller);
  }
  for (int d = 0; d < 3; d++) {
    if (t->bound_cond[2 * d] == 0 || t->bound_cond[2 * d + 1] == 0) continue;
    const int S = t->nghost[2 * d] + t->nghost[2 * d + 1];
    const long long total = (long long)S * g.ext[(d + 1) % 3] * g.ext[(d + 2) % 3];
    const int nblk = (int)std::min<long long>((total + 255) / 256, 148 * 16);
    { KTimer kt_(KC_GFILL, st); k_ghost_fill<R><<<std::max(nblk, 1), 256, 0, st>>>(dvort, g.ext[0], g.ext[1], g.ext[2], 3, d,
                                                                                    t->ncell[d], t->nghost[2 * d],
                                                                                    t->nghost[2 * d + 1]); }
    PM_LAUNCHED();
    CKL(caller);
  }
  return 0;
}

// Runge-Kutta coefficients of source/particles/pmlib_particles_advance.f:49-88 in the
// working precision (the reference forms them as REAL(MK) constants)
template <typename R> static int rk_coef(int order, int stage, int euler, R &a1, R &b1, R &c1, R &a2, R &b2, R &c2) {
  const R z = R(0), o = R(1), h = R(0.5);
  R A1[3] = {z, z, z}, B1[3] = {z, z, z}, C1[3] = {z, z, z}, A2[3] = {z, z, z}, B2[3] = {z, z, z}, C2[3] = {z, z, z};
  if (order == 1) {
    B1[0] = C1[0] = B2[0] = C2[0] = o;
  } else if (order == 2) {
    A1[1] = -h; B1[0] = B1[1] = o; C1[0] = h; C1[1] = o;
    if (euler) { A2[1] = o; B2[0] = o; C2[0] = h; C2[1] = h; }
    else { A2[1] = -h; B2[0] = B2[1] = o; C2[0] = h; C2[1] = o; }
  } else if (order == 3) {
    A1[1] = R(-5) / R(9); A1[2] = R(-153) / R(128);
    B1[0] = B1[1] = B1[2] = o;
    C1[0] = R(1) / R(3); C1[1] = R(15) / R(16); C1[2] = R(8) / R(15);
    if (euler) { A2[1] = A2[2] = o; B2[0] = o; C2[0] = C2[1] = C2[2] = R(1) / R(3); }
    else {
      A2[1] = R(-5) / R(9); A2[2] = R(-153) / R(128);
      B2[0] = B2[1] = B2[2] = o;
      C2[0] = R(1) / R(3); C2[1] = R(15) / R(16); C2[2] = R(8) / R(15);
    }
  } else {
    return -1;
  }
  if (stage < 1 || stage > order) return -2;
  a1 = A1[stage - 1]; b1 = B1[stage - 1]; c1 = C1[stage - 1];
  a2 = A2[stage - 1]; b2 = B2[stage - 1]; c2 = C2[stage - 1];
  return 0;
}

// pmlib_particles_advance (source/particles/pmlib_particles_advance.f:5-213, one rank)
// on device arrays (3, npart): stage update in place, then the map as one stable
// bucket sort of the survivors (arrays compacted in place).  Waits for the stream:
// the new count is needed on the host.
template <typename R>
static int run_advance(const pmgpu_patch *pa, pmgpu_topo *t, int order, int stage, double dtime, int euler, R *pos,
                       R *vort, const R *vel, const R *dvort, R *vel_rk, R *dvort_rk, int n, int *nout,
                       cudaStream_t st, const char *caller) {
  AdvanceCoef<R> c;
  memset(&c, 0, sizeof(c));
  R b1, b2;
  const int rc = rk_coef<R>(order, stage, euler, c.a1, b1, c.c1, c.a2, b2, c.c2);
  if (rc == -1) {
    // the message of source/parameters/pmlib_parameters_check.f:90-96
    set_error("pmlib_parameters_check", "pmlib_interpolation_order is incorrectly set.");
    return -1;
  }
  if (rc == -2) {
    set_error(caller, "Time stage out of range.");
    return -1;
  }
  if (n < 0 || (n > 0 && (!pos || !vort || !vel || !dvort || !vel_rk || !dvort_rk))) {
    set_error(caller, "missing argument.");
    return -1;
  }
  c.b1dt = b1 * (R)dtime;
  c.b2dt = b2 * (R)dtime;
  c.zero_rk = order == 1;
  for (int e = 0; e < 3; e++) {
    c.xmin[e] = (R)t->xmin[e];
    c.xmax[e] = (R)t->xmax[e];
    c.pmin[e] = (R)pa->xmin[e];
    c.pmax[e] = (R)pa->xmax[e];
    c.plen[e] = (R)pa->xmax[e] - (R)pa->xmin[e];
    c.per_lo[e] = t->bound_cond[2 * e] != 0;
    c.per_hi[e] = t->bound_cond[2 * e + 1] != 0;
  }
  *nout = n;
  if (n == 0) {
    t->npart = 0;
    return 0;
  }
  Scratch &s = scratch();
  if (s.adv_code.ensure(sizeof(unsigned) * (size_t)n, caller) || s.adv_stats.ensure(sizeof(unsigned) * 8, caller))
    return -1;
  unsigned *stats = s.adv_stats.as<unsigned>();
  CK(cudaMemsetAsync(stats, 0, sizeof(unsigned) * 8, st), caller);
  const int nblk = std::min((n + 255) / 256, 148 * 16);
  { KTimer kt_(KC_ADVANCE, st); k_advance<R><<<nblk, 256, 0, st>>>(c, n, pos, vort, vel, dvort, vel_rk, dvort_rk,
                                                                   s.adv_code.as<unsigned>(), stats); }
  PM_LAUNCHED();
  CKL(caller);
  unsigned h[8];
  CK(cudaMemcpyAsync(h, stats, sizeof(h), cudaMemcpyDeviceToHost, st), caller);
  CK(cudaStreamSynchronize(st), caller);
  if (h[4]) {
    set_error(caller, "A particle moved more than one patch length in one step.");
    return -1;
  }
  if (!h[0]) {  // nobody left or was dropped: the order stays
    t->npart = n;
    return 0;
  }
  const int K0 = (int)h[1], K1 = (int)h[2], K2 = (int)h[3];
  unsigned nbk = 1;
  for (int k : {K0, K1, K2})
    for (int i = 0; i < k; i++) nbk *= 3u;
  const int nb = (n + MAP_CHUNK - 1) / MAP_CHUNK;
  const size_t ncnt = (size_t)(nbk + 1) * nb;
  if (s.adv_cnt.ensure(sizeof(unsigned) * (ncnt + 1), caller) ||
      s.adv_start.ensure(sizeof(unsigned) * (ncnt + 1), caller) || s.adv_ord.ensure(sizeof(int) * (size_t)n, caller) ||
      s.adv_tmp.ensure(sizeof(R) * 3 * (size_t)n, caller))
    return -1;
  { KTimer kt_(KC_MAP, st); k_map_count<<<nb, MAP_THREADS, 0, st>>>(s.adv_code.as<unsigned>(), n, K0, K1, K2, nbk,
                                                                    s.adv_cnt.as<unsigned>()); }
  PM_LAUNCHED();
  CKL(caller);
  if (exclusive_scan(s.adv_cnt.as<unsigned>(), s.adv_start.as<unsigned>(), ncnt, s.spart, st, caller)) return -1;
  { KTimer kt_(KC_MAP, st); k_map_scatter<<<nb, MAP_THREADS, 0, st>>>(s.adv_code.as<unsigned>(), n, K0, K1, K2, nbk,
                                                                      s.adv_start.as<unsigned>(),
                                                                      s.adv_ord.as<int>()); }
  PM_LAUNCHED();
  CKL(caller);
  unsigned live = 0;  // first slot of the dropped bucket = survivors
  CK(cudaMemcpyAsync(&live, s.adv_start.as<unsigned>() + (size_t)nbk * nb, sizeof(unsigned), cudaMemcpyDeviceToHost,
                     st), caller);
  CK(cudaStreamSynchronize(st), caller);
  const int m = (int)live;
  R *arrs[4] = {pos, vort, vel_rk, dvort_rk};
  for (R *a : arrs) {
    if (m > 0) {
      { KTimer kt_(KC_MAP, st); k_gather3<R><<<std::min((m + 255) / 256, 148 * 16), 256, 0, st>>>(
          s.adv_ord.as<int>(), m, a, s.adv_tmp.as<R>()); }
      PM_LAUNCHED();
      CK(cudaMemcpyAsync(a, s.adv_tmp.p, sizeof(R) * 3 * (size_t)m, cudaMemcpyDeviceToDevice, st), caller);
    }
  }
  CKL(caller);
  CK(cudaStreamSynchronize(st), caller);
  *nout = m;
  t->npart = m;
  return 0;
}

template <typename R>
static int deriv_host(const pmgpu_topo *t, int fd_order, double visc, const R *vort, const R *vel, R *dvort) {
  const char *caller = "part_deriv_vorticity";
  std::lock_guard<std::mutex> lk(g_mu);
  if (!t || !vort || !vel || !dvort) {
    set_error(caller, "missing argument.");
    return -1;
  }
  if (ensure_device(caller)) return -1;
  Scratch &s = scratch();
  const size_t nm = mesh_points(t) * 3;
  if (s.c.ensure(sizeof(R) * nm, caller) || s.d.ensure(sizeof(R) * nm, caller) || s.e.ensure(sizeof(R) * nm, caller))
    return -1;
  CK(cudaMemcpy(s.c.p, vort, sizeof(R) * nm, cudaMemcpyHostToDevice), caller);
  CK(cudaMemcpy(s.d.p, vel, sizeof(R) * nm, cudaMemcpyHostToDevice), caller);
  CK(cudaMemcpy(s.e.p, dvort, sizeof(R) * nm, cudaMemcpyHostToDevice), caller);  // free-axis ghosts are kept
  if (run_deriv_vorticity<R>(t, fd_order, visc, s.c.as<R>(), s.d.as<R>(), s.e.as<R>(), 0, caller)) return -1;
  CK(cudaMemcpy(dvort, s.e.p, sizeof(R) * nm, cudaMemcpyDeviceToHost), caller);
  return 0;
}

int pmgpu_deriv_vorticity(const pmgpu_topo *topo, int fd_order, double visc, const double *mesh_vort,
                          const double *mesh_vel, double *mesh_dvort) {
  return deriv_host<double>(topo, fd_order, visc, mesh_vort, mesh_vel, mesh_dvort);
}
int pmgpu_deriv_vorticity_f32(const pmgpu_topo *topo, int fd_order, double visc, const float *mesh_vort,
                              const float *mesh_vel, float *mesh_dvort) {
  return deriv_host<float>(topo, fd_order, visc, mesh_vort, mesh_vel, mesh_dvort);
}
int pmgpu_deriv_vorticity_dev(const pmgpu_topo *topo, int fd_order, double visc, int precision, const void *d_vort,
                              const void *d_vel, void *d_dvort, void *stream) {
  const char *caller = "part_deriv_vorticity";
  std::lock_guard<std::mutex> lk(g_mu);
  if (!topo || !d_vort || !d_vel || !d_dvort) {
    set_error(caller, "missing argument.");
    return -1;
  }
  if (ensure_device(caller)) return -1;
  cudaStream_t st = (cudaStream_t)stream;
  if (precision == PMGPU_FP64)
    return run_deriv_vorticity<double>(topo, fd_order, visc, (const double *)d_vort, (const double *)d_vel,
                                       (double *)d_dvort, st, caller);
  if (precision == PMGPU_FP32)
    return run_deriv_vorticity<float>(topo, fd_order, visc, (const float *)d_vort, (const float *)d_vel,
                                      (float *)d_dvort, st, caller);
  set_error(caller, "precision unknown.");
  return -1;
}

template <typename R>
static int advance_host(const pmgpu_patch *pa, pmgpu_topo *t, int order, int stage, double dtime, int euler, R *pos,
                        R *vort, const R *vel, const R *dvort, R *vel_rk, R *dvort_rk, int npart, int *nout) {
  const char *caller = "pmlib_particles_advance";
  std::lock_guard<std::mutex> lk(g_mu);
  if (!pa || !t || !nout || npart < 0) {
    set_error(caller, "missing argument.");
    return -1;
  }
  if (ensure_device(caller)) return -1;
  Scratch &s = scratch();
  const size_t b = sizeof(R) * 3 * (size_t)std::max(npart, 1);
  DevBuf *bufs[6] = {&s.c, &s.d, &s.e, &s.f, &s.g, &s.h};
  for (DevBuf *d : bufs)
    if (d->ensure(b, caller)) return -1;
  const R *src[6] = {pos, vort, vel, dvort, vel_rk, dvort_rk};
  for (int i = 0; i < 6; i++)
    if (npart > 0 && src[i]) CK(cudaMemcpy(bufs[i]->p, src[i], sizeof(R) * 3 * (size_t)npart, cudaMemcpyHostToDevice), caller);
  if (npart > 0 && (!pos || !vort || !vel || !dvort || !vel_rk || !dvort_rk)) {
    set_error(caller, "missing argument.");
    return -1;
  }
  if (run_advance<R>(pa, t, order, stage, dtime, euler, s.c.as<R>(), s.d.as<R>(), s.e.as<R>(), s.f.as<R>(),
                     s.g.as<R>(), s.h.as<R>(), npart, nout, 0, caller))
    return -1;
  R *dst[4] = {pos, vort, vel_rk, dvort_rk};
  DevBuf *from[4] = {&s.c, &s.d, &s.g, &s.h};
  for (int i = 0; i < 4; i++)
    if (*nout > 0) CK(cudaMemcpy(dst[i], from[i]->p, sizeof(R) * 3 * (size_t)*nout, cudaMemcpyDeviceToHost), caller);
  return 0;
}

int pmgpu_particles_advance(const pmgpu_patch *patch, pmgpu_topo *topo, int time_order, int itimestage,
                            double dtime, int euler_vort, double *pos, double *vort, const double *vel,
                            const double *dvort, double *vel_rk, double *dvort_rk, int npart, int *npart_out) {
  return advance_host<double>(patch, topo, time_order, itimestage, dtime, euler_vort, pos, vort, vel, dvort, vel_rk,
                              dvort_rk, npart, npart_out);
}
int pmgpu_particles_advance_f32(const pmgpu_patch *patch, pmgpu_topo *topo, int time_order, int itimestage,
                                double dtime, int euler_vort, float *pos, float *vort, const float *vel,
                                const float *dvort, float *vel_rk, float *dvort_rk, int npart, int *npart_out) {
  return advance_host<float>(patch, topo, time_order, itimestage, dtime, euler_vort, pos, vort, vel, dvort, vel_rk,
                             dvort_rk, npart, npart_out);
}
int pmgpu_particles_advance_dev(const pmgpu_patch *patch, pmgpu_topo *topo, int time_order, int itimestage,
                                double dtime, int euler_vort, int precision, void *d_pos, void *d_vort,
                                const void *d_vel, const void *d_dvort, void *d_vel_rk, void *d_dvort_rk, int npart,
                                int *npart_out, void *stream) {
  const char *caller = "pmlib_particles_advance";
  std::lock_guard<std::mutex> lk(g_mu);
  if (!patch || !topo || !npart_out) {
    set_error(caller, "missing argument.");
    return -1;
  }
  if (ensure_device(caller)) return -1;
  cudaStream_t st = (cudaStream_t)stream;
  if (precision == PMGPU_FP64)
    return run_advance<double>(patch, topo, time_order, itimestage, dtime, euler_vort, (double *)d_pos,
                               (double *)d_vort, (const double *)d_vel, (const double *)d_dvort, (double *)d_vel_rk,
                               (double *)d_dvort_rk, npart, npart_out, st, caller);
  if (precision == PMGPU_FP32)
    return run_advance<float>(patch, topo, time_order, itimestage, dtime, euler_vort, (float *)d_pos,
                              (float *)d_vort, (const float *)d_vel, (const float *)d_dvort, (float *)d_vel_rk,
                              (float *)d_dvort_rk, npart, npart_out, st, caller);
  set_error(caller, "precision unknown.");
  return -1;
}

// ------------------------------------------------------------------ one stage of the vortex client
// The stage of vortex_codes/vortex_structures/source/main.f:396-510 without remeshing
// and diagnostics, from this library's pieces: P2M of the particle vorticity (mesh
// cleared first), the solve for the mesh velocity, the vorticity right-hand side on
// the mesh (its free-face ghosts start at zero), M2P of velocity and right-hand side
// in the bin order of the deposition, and the stage update with the particle map.
template <typename R>
static int vortex_stage(pmgpu_plan *pl, int order, int stage, double dtime, int euler, int fd_order, double visc,
                        R *pos, R *vort, R *vel_rk, R *dvort_rk, int n, R *pvel, R *pdvort, int *nout,
                        cudaStream_t st) {
  const char *caller = "pmgpu_vortex_stage";
  const size_t nm = mesh_points(&pl->topo) * 3;
  if (pl->mesh_w.ensure(sizeof(R) * nm, caller) || pl->mesh_u.ensure(sizeof(R) * nm, caller) ||
      pl->mesh_a.ensure(sizeof(R) * nm, caller))
    return -1;
  pmgpu_topo t = pl->topo;
  t.npart = n;
  PartScratchRefs r{&pl->key, &pl->val, &pl->key2, &pl->val2, &pl->counts, &pl->start, &pl->spart, &pl->hist};
  const int *perm = nullptr;
  if (run_p2m<R>(&t, pl->par.interpolation_order, pos, vort, 3, n, pl->mesh_w.as<R>(), 3, 1, r, st, &perm, caller))
    return -1;
  if (run_solve<R>(pl, pl->mesh_w.as<R>(), pl->mesh_u.as<R>(), nullptr, nullptr, 0, 0, 0, st, caller)) return -1;
  CK(cudaMemsetAsync(pl->mesh_a.p, 0, sizeof(R) * nm, st), caller);
  if (run_deriv_vorticity<R>(&t, fd_order, visc, pl->mesh_w.as<R>(), pl->mesh_u.as<R>(), pl->mesh_a.as<R>(), st,
                             caller))
    return -1;
  if (run_m2p_sorted<R>(&t, pl->par.interpolation_order, pos, pl->start.as<unsigned>(), perm, n, pl->mesh_u.as<R>(),
                        pvel, st, caller) ||
      run_m2p_sorted<R>(&t, pl->par.interpolation_order, pos, pl->start.as<unsigned>(), perm, n, pl->mesh_a.as<R>(),
                        pdvort, st, caller))
    return -1;
  return run_advance<R>(&pl->patch, &t, order, stage, dtime, euler, pos, vort, pvel, pdvort, vel_rk, dvort_rk, n,
                        nout, st, caller);
}

int pmgpu_vortex_stage_dev(pmgpu_plan *plan, int time_order, int itimestage, double dtime, int euler_vort,
                           int fd_order, double visc, void *d_pos, void *d_vort, void *d_vel_rk, void *d_dvort_rk,
                           int npart, void *d_part_vel, void *d_part_dvort, int *npart_out, void *stream) {
  const char *caller = "pmgpu_vortex_stage";
  std::lock_guard<std::mutex> lk(g_mu);
  if (!plan || !npart_out || npart < 0 ||
      (npart > 0 && (!d_pos || !d_vort || !d_vel_rk || !d_dvort_rk || !d_part_vel || !d_part_dvort))) {
    set_error(caller, "missing argument.");
    return -1;
  }
  if (ensure_device(caller)) return -1;
  cudaStream_t st = (cudaStream_t)stream;
  if (plan->prec == PMGPU_FP64)
    return vortex_stage<double>(plan, time_order, itimestage, dtime, euler_vort, fd_order, visc, (double *)d_pos,
                                (double *)d_vort, (double *)d_vel_rk, (double *)d_dvort_rk, npart,
                                (double *)d_part_vel, (double *)d_part_dvort, npart_out, st);
  return vortex_stage<float>(plan, time_order, itimestage, dtime, euler_vort, fd_order, visc, (float *)d_pos,
                             (float *)d_vort, (float *)d_vel_rk, (float *)d_dvort_rk, npart, (float *)d_part_vel,
                             (float *)d_part_dvort, npart_out, st);
}

// ------------------------------------------------------------------ Brinkman penalisation
static int nint_d(double x) { return (int)lround(x); }

// index ranges of source/mesh/pmlib_mesh_map.f:85-176 (one rank), as array offsets
static int mesh_map_box(const pmgpu_topo *s, const pmgpu_topo *r, int map_ghost, MapBox &m, const char *caller) {
  for (int i = 0; i < 3; i++) {
    const double dx = r->dx[i];
    if (dx != s->dx[i]) {
      set_error("pmlib_mesh_map", "Mesh cell size does not coinside.");
      return -1;
    }
    if (nint_d((r->xmax[i] - s->xmin[i]) / dx) <= 0 || nint_d((s->xmax[i] - r->xmin[i]) / dx) <= 0) {
      set_error(caller, "The penalisation box does not intersect the grid.");
      return -1;
    }
    const int ds = nint_d((r->xmin[i] - s->xmin[i]) / dx);
    const int ngs_lo = s->nghost[2 * i], ngs_hi = s->nghost[2 * i + 1];
    const int ngr_lo = r->nghost[2 * i], ngr_hi = r->nghost[2 * i + 1];
    int ng, smin, rmin, smax, rmax;
    if (ds == 0) {
      ng = (map_ghost && r->bound_cond[2 * i] == 0) ? std::min(ngr_lo, ngs_lo) : 0;
      smin = 1 - ng;
      rmin = 1 - ng;
    } else if (ds < 0) {  // the sender starts inside the receiver
      ng = (map_ghost && s->bound_cond[2 * i] == 0) ? std::min(ngs_lo, -ds + ngr_lo) : 0;
      smin = 1 - ng;
      rmin = 1 - ds - ng;
    } else {
      ng = (map_ghost && r->bound_cond[2 * i] == 0) ? std::min(ngr_lo, ds + ngs_lo) : 0;
      smin = 1 + ds - ng;
      rmin = 1 - ng;
    }
    const int de = nint_d((r->xmax[i] - s->xmax[i]) / dx);
    if (de == 0) {
      ng = (map_ghost && r->bound_cond[2 * i + 1] == 0) ? std::min(ngr_hi, ngs_hi) : 0;
      smax = s->ncell[i] + ng;
      rmax = r->ncell[i] + ng;
    } else if (de > 0) {  // the receiver reaches beyond the sender
      ng = (map_ghost && s->bound_cond[2 * i + 1] == 0) ? std::min(ngs_hi, de + ngr_hi) : 0;
      smax = s->ncell[i] + ng;
      rmax = nint_d((s->xmax[i] - r->xmin[i]) / dx) + ng;
    } else {
      ng = (map_ghost && r->bound_cond[2 * i + 1] == 0) ? std::min(ngr_hi, -de + ngs_hi) : 0;
      smax = nint_d((r->xmax[i] - s->xmin[i]) / dx) + ng;
      rmax = r->ncell[i] + ng;
    }
    if (smax - smin != rmax - rmin || smax < smin) {
      set_error("pmlib_mesh_map", "Number of sended and recieved cells does not correspond");
      return -1;
    }
    m.s0[i] = smin - 1 + s->nghost[2 * i];
    m.r0[i] = rmin - 1 + r->nghost[2 * i];
    m.n[i] = smax - smin + 1;
    m.es[i] = s->ncell[i] + s->nghost[2 * i] + s->nghost[2 * i + 1];
    m.er[i] = r->ncell[i] + r->nghost[2 * i] + r->nghost[2 * i + 1];
    if (m.s0[i] < 0 || m.r0[i] < 0 || m.s0[i] + m.n[i] > m.es[i] || m.r0[i] + m.n[i] > m.er[i]) {
      set_error("pmlib_mesh_map", "Sending or receiving index out of range");
      return -1;
    }
  }
  return 0;
}

template <typename R>
static int launch_mesh_map(const MapBox &m, const R *src, R *dst, int op, cudaStream_t st, const char *caller) {
  const long long total = (long long)m.n[0] * m.n[1] * m.n[2];
  if (total <= 0) return 0;
  { KTimer kt_(KC_OTHER, st);
    k_mesh_map<R><<<(unsigned)std::min<long long>((total + 255) / 256, 148 * 16), 256, 0, st>>>(m, 3, src, dst, op); }
  PM_LAUNCHED();
  CKL(caller);
  return 0;
}

// The vortex client's iterative Brinkman penalisation (vortex_codes/vortex_penalisation/
// source/penalisation/penalisation_solve.f:5-430, one rank) on device arrays: the box
// is the penalisation plan's cuboid, the box fields live in that plan's mesh buffers
// (vel_pen, vel, vort), and its Poisson solves are that plan's solves.
template <typename R>
static int run_penal(pmgpu_plan *pm, pmgpu_plan *pp, const R *solid, const R *svel, double relax, double tol,
                     int max_iter, double dtime, int fd_order, int reproject, const double vel_inf[3], R *vort,
                     R *vel, double force[3], int *niter, double resid[3], cudaStream_t st) {
  const char *caller = "penalisation";
  if (fd_order != 2 && fd_order != 4) {
    set_error("pmlib_parameters_check", "pmlib_fd_order is incorrectly set.");
    return -1;
  }
  for (int e = 0; e < 3; e++)
    if (pp->topo.nghost[2 * e] < fd_order / 2 || pp->topo.nghost[2 * e + 1] < fd_order / 2) {
      set_error(caller, "Too few ghost cells in the penalisation box for the finite differences.");
      return -1;
    }
  MapBox to_box, to_main;
  if (mesh_map_box(&pm->topo, &pp->topo, 1, to_box, caller) || mesh_map_box(&pp->topo, &pm->topo, 1, to_main, caller))
    return -1;
  const size_t npp = mesh_points(&pp->topo), npm = mesh_points(&pm->topo);
  if (pp->mesh_a.ensure(sizeof(R) * 3 * npp, caller) || pp->mesh_u.ensure(sizeof(R) * 3 * npp, caller) ||
      pp->mesh_w.ensure(sizeof(R) * 3 * npp, caller))
    return -1;
  Scratch &sc = scratch();
  if (sc.pen_part.ensure(sizeof(double) * PEN_BLOCKS * PEN_NV, caller) || sc.pen_out.ensure(sizeof(double) * 8, caller))
    return -1;
  R *vel_pen = pp->mesh_a.as<R>(), *pvel = pp->mesh_u.as<R>(), *pvort = pp->mesh_w.as<R>();
  double *part = sc.pen_part.as<double>(), *dout = sc.pen_out.as<double>();
  auto sums = [&](int nv, double *h) -> int {
    k_pen_final<<<1, 32 * nv, 0, st>>>(part, PEN_BLOCKS, nv, dout);
    PM_LAUNCHED();
    CK(cudaMemcpyAsync(h, dout, sizeof(double) * nv, cudaMemcpyDeviceToHost, st), caller);
    CK(cudaStreamSynchronize(st), caller);
    return 0;
  };
  // :61-107 main velocity onto the cleared box; vel_pen = solid_vel - vel; vel = solid vel_pen
  CK(cudaMemsetAsync(vel_pen, 0, sizeof(R) * 3 * npp, st), caller);
  CK(cudaMemsetAsync(pvort, 0, sizeof(R) * 3 * npp, st), caller);
  if (launch_mesh_map<R>(to_box, vel, vel_pen, 0, st, caller)) return -1;
  { KTimer kt_(KC_OTHER, st);
    k_pen_init<R><<<PEN_BLOCKS, PEN_THREADS, 0, st>>>((long long)npp, solid, svel, vel_pen, pvel, part); }
  PM_LAUNCHED();
  CKL(caller);
  double sum_vel_pen = 0.0;
  if (sums(1, &sum_vel_pen)) return -1;
  PenGeom<R> g;
  for (int e = 0; e < 3; e++) {
    g.ext[e] = pp->topo.ncell[e] + pp->topo.nghost[2 * e] + pp->topo.nghost[2 * e + 1];
    g.ngl[e] = pp->topo.nghost[2 * e];
    g.nc[e] = pp->topo.ncell[e];
    g.c_1_2dx[e] = R(1) / (R(2) * (R)pp->topo.dx[e]);
    g.xmin[e] = (R)pp->topo.xmin[e];
    g.dx[e] = (R)pp->topo.dx[e];
  }
  g.relax = (R)relax;
  const double dvol = pp->topo.dx[0] * pp->topo.dx[1] * pp->topo.dx[2], c_1_dt = 1.0 / dtime;
  double residual_force = 0.0, residual_vel = 0.0, residual_enst = 0.0;
  int npen = 0;
  for (int c = 0; c < 3; c++) force[c] = 0.0;
  while ((residual_force > tol && npen < max_iter) || npen == 0) {
    npen++;
    { KTimer kt_(KC_OTHER, st);
      if (fd_order == 2) k_pen_curl<R, 2><<<PEN_BLOCKS, PEN_THREADS, 0, st>>>(g, pvel, pvort, part);
      else k_pen_curl<R, 4><<<PEN_BLOCKS, PEN_THREADS, 0, st>>>(g, pvel, pvort, part); }
    PM_LAUNCHED();
    CKL(caller);
    double h[PEN_NV];
    if (sums(PEN_NV, h)) return -1;
    if (run_solve<R>(pp, pvort, pvel, nullptr, nullptr, 0, 0, 0, st, caller)) return -1;
    { KTimer kt_(KC_OTHER, st);
      k_pen_vel<R><<<PEN_BLOCKS, PEN_THREADS, 0, st>>>((long long)npp, solid, vel_pen, pvel, part); }
    PM_LAUNCHED();
    CKL(caller);
    double res_vel = 0.0;
    if (sums(1, &res_vel)) return -1;
    double df[3];
    for (int c = 0; c < 3; c++) {
      df[c] = -h[c] * dvol * c_1_dt;
      force[c] = force[c] + df[c];
    }
    residual_enst = h[3] / h[4];
    residual_vel = res_vel / sum_vel_pen;
    residual_force = sqrt(df[0] * df[0] + df[1] * df[1] + df[2] * df[2]) /
                     sqrt(force[0] * force[0] + force[1] * force[1] + force[2] * force[2]);
  }
  // :345-360 box vorticity added to the main vorticity, then the main ghost map
  if (launch_mesh_map<R>(to_main, pvort, vort, 1, st, caller)) return -1;
  const pmgpu_topo *t = &pm->topo;
  for (int d = 0; d < 3; d++) {
    if (t->bound_cond[2 * d] == 0 || t->bound_cond[2 * d + 1] == 0) continue;
    const int ext[3] = {to_main.er[0], to_main.er[1], to_main.er[2]};
    const int S = t->nghost[2 * d] + t->nghost[2 * d + 1];
    const long long total = (long long)S * ext[(d + 1) % 3] * ext[(d + 2) % 3];
    const int nblk = (int)std::min<long long>((total + 255) / 256, 148 * 16);
    { KTimer kt_(KC_GFILL, st);
      k_ghost_fill<R><<<std::max(nblk, 1), 256, 0, st>>>(vort, ext[0], ext[1], ext[2], 3, d, t->ncell[d],
                                                         t->nghost[2 * d], t->nghost[2 * d + 1]); }
    PM_LAUNCHED();
    CKL(caller);
  }
  // :364-419 main solve (vorticity reprojected when asked), free-stream velocity
  if (run_solve<R>(pm, vort, vel, reproject ? vort : nullptr, nullptr, 0, reproject ? 1 : 0, 0, st, caller))
    return -1;
  { KTimer kt_(KC_OTHER, st);
    k_add_vel_inf<R><<<(unsigned)std::min<size_t>((npm + 255) / 256, 148 * 16), 256, 0, st>>>(
        (long long)npm, vel, (R)vel_inf[0], (R)vel_inf[1], (R)vel_inf[2]); }
  PM_LAUNCHED();
  CKL(caller);
  CK(cudaStreamSynchronize(st), caller);
  *niter = npen;
  resid[0] = residual_vel;
  resid[1] = residual_force;
  resid[2] = residual_enst;
  return 0;
}

int pmgpu_penalisation_solve_dev(pmgpu_plan *plan, pmgpu_plan *penal_plan, const void *d_solid,
                                 const void *d_solid_vel, double relaxation, double tolerance, int max_iter,
                                 double dtime, int fd_order, int reproject, const double vel_inf[3], void *d_vort,
                                 void *d_vel, double force[3], int *niter, double residuals[3], void *stream) {
  const char *caller = "penalisation";
  std::lock_guard<std::mutex> lk(g_mu);
  if (!plan || !penal_plan || !d_solid || !d_solid_vel || !vel_inf || !d_vort || !d_vel || !force || !niter ||
      !residuals || max_iter < 1 || !(dtime != 0.0)) {
    set_error(caller, "missing or invalid argument.");
    return -1;
  }
  if (plan->prec != penal_plan->prec) {
    set_error(caller, "the grid and the penalisation box plans differ in precision.");
    return -1;
  }
  if (ensure_device(caller)) return -1;
  cudaStream_t st = (cudaStream_t)stream;
  if (plan->prec == PMGPU_FP64)
    return run_penal<double>(plan, penal_plan, (const double *)d_solid, (const double *)d_solid_vel, relaxation,
                             tolerance, max_iter, dtime, fd_order, reproject, vel_inf, (double *)d_vort,
                             (double *)d_vel, force, niter, residuals, st);
  return run_penal<float>(plan, penal_plan, (const float *)d_solid, (const float *)d_solid_vel, relaxation, tolerance,
                          max_iter, dtime, fd_order, reproject, vel_inf, (float *)d_vort, (float *)d_vel, force,
                          niter, residuals, st);
}

// ------------------------------------------------------------------ one stage of the penalisation client
namespace pmgpu {
// pmlib_remesh on device fields (source/remesh/pmlib_remesh.f:84-226, one rank): one
// particle at the centre of every kept cell in k-j-i order into arrays of capacity
// max_part; the count comes back to the host (the stream is synchronised)
template <typename R>
static int run_remesh_dev(pmgpu_plan *pl, const pmgpu_topo *t, const R *vort, const R *dvort, const R *vel,
                          double min_vort, double min_dvort, int max_part, R *pos, R *pv, R *pdv, R *pvel, int *np,
                          cudaStream_t st, const char *caller) {
  const size_t nc = mesh_points(t);
  PartGeom<R> g = part_geom<R>(t, 4);
  if (pl->counts.ensure(sizeof(unsigned) * (nc + 1), caller) || pl->start.ensure(sizeof(unsigned) * (nc + 1), caller))
    return -1;
  const int nblk = (int)std::min<size_t>((nc + 255) / 256, 148 * 32);
  CK(cudaMemsetAsync(pl->counts.p, 0, sizeof(unsigned) * (nc + 1), st), caller);
  k_remesh_flag<R><<<nblk, 256, 0, st>>>(g, vort, dvort, nullptr, (R)min_vort, (R)min_dvort, 0,
                                         pl->counts.as<unsigned>());
  PM_LAUNCHED();
  CKL(caller);
  if (exclusive_scan(pl->counts.as<unsigned>(), pl->start.as<unsigned>(), nc + 1, pl->spart, st, caller)) return -1;
  unsigned total = 0;
  CK(cudaMemcpyAsync(&total, pl->start.as<unsigned>() + nc, sizeof(unsigned), cudaMemcpyDeviceToHost, st), caller);
  CK(cudaStreamSynchronize(st), caller);
  if ((long long)total > (long long)max_part) {
    char msg[160];
    snprintf(msg, sizeof(msg), "remeshing makes %u particles, more than the arrays hold (%d).", total, max_part);
    set_error(caller, msg);
    return -1;
  }
  k_remesh_fill<R><<<nblk, 256, 0, st>>>(g, vort, dvort, vel, pl->counts.as<unsigned>(), pl->start.as<unsigned>(),
                                         pos, pv, pdv, pvel);
  PM_LAUNCHED();
  CKL(caller);
  *np = (int)total;
  return 0;
}

// One stage of the penalisation client's time loop (vortex_codes/vortex_penalisation/
// source/main.f:343-492, one rank, no repatching, diagnostics or output) on the plan's
// mesh buffers: P2M of the particle vorticity (cleared), the solve (reprojected when
// the client asks or on the first stage of the first step, the vorticity pulled back
// then), the free-stream velocity added, the iterative penalisation on the first
// stage, the vorticity right-hand side, then a remesh from the mesh fields (first
// stage of a remeshing step or of the first step; thresholds remesh_trunc and
// remesh_trunc / dtime, velocity and right-hand side copied) or M2P of the velocity
// and the right-hand side, and the stage update with the particle map.
template <typename R>
static int penal_stage(pmgpu_plan *pm, pmgpu_plan *pp, const R *solid, const R *svel, const pmgpu_penal_stage_args &a,
                       R *pos, R *vort, R *vel_rk, R *dvort_rk, int n, int max_part, R *pvel, R *pdvort, int *nout,
                       double force[3], int *niter, double resid[3], cudaStream_t st) {
  const char *caller = "pmgpu_penalisation_stage";
  const size_t nmp = mesh_points(&pm->topo), nm = nmp * 3;
  if (pm->mesh_w.ensure(sizeof(R) * nm, caller) || pm->mesh_u.ensure(sizeof(R) * nm, caller) ||
      pm->mesh_a.ensure(sizeof(R) * nm, caller))
    return -1;
  R *w = pm->mesh_w.as<R>(), *u = pm->mesh_u.as<R>(), *dw = pm->mesh_a.as<R>();
  pmgpu_topo t = pm->topo;
  t.npart = n;
  PartScratchRefs r{&pm->key, &pm->val, &pm->key2, &pm->val2, &pm->counts, &pm->start, &pm->spart, &pm->hist};
  const int *perm = nullptr;
  if (run_p2m<R>(&t, pm->par.interpolation_order, pos, vort, 3, n, w, 3, 1, r, st, &perm, caller)) return -1;
  const int first = a.first_step && a.itimestage == 1;
  const int reproj = a.reproject || first;
  const int back = reproj || a.regularise_vort;
  if (run_solve<R>(pm, w, u, back ? w : nullptr, nullptr, a.regularise_vort, reproj, 0, st, caller)) return -1;
  if (a.vel_inf[0] != 0.0 || a.vel_inf[1] != 0.0 || a.vel_inf[2] != 0.0) {
    const int nblk = (int)std::min<size_t>((nmp + 255) / 256, 148 * 16);
    k_add_vec3<R><<<nblk, 256, 0, st>>>(u, nmp, (R)a.vel_inf[0], (R)a.vel_inf[1], (R)a.vel_inf[2]);
    PM_LAUNCHED();
    CKL(caller);
  }
  force[0] = force[1] = force[2] = 0.0;
  resid[0] = resid[1] = resid[2] = 0.0;
  *niter = 0;
  if (a.itimestage == 1 && pp && solid &&
      run_penal<R>(pm, pp, solid, svel, a.relaxation, a.tolerance, a.max_iter, a.dtime, a.fd_order, a.reproject,
                   a.vel_inf, w, u, force, niter, resid, st))
    return -1;
  CK(cudaMemsetAsync(dw, 0, sizeof(R) * nm, st), caller);
  if (run_deriv_vorticity<R>(&t, a.fd_order, a.visc, w, u, dw, st, caller)) return -1;
  if ((a.remesh || a.first_step) && a.itimestage == 1) {
    int m = 0;
    if (run_remesh_dev<R>(pm, &t, w, dw, u, a.remesh_trunc, a.remesh_trunc / a.dtime, max_part, pos, vort, pdvort, pvel,
                          &m, st, caller))
      return -1;
    if (m > 0) {
      CK(cudaMemsetAsync(vel_rk, 0, sizeof(R) * 3 * (size_t)m, st), caller);
      CK(cudaMemsetAsync(dvort_rk, 0, sizeof(R) * 3 * (size_t)m, st), caller);
    }
    n = m;
    t.npart = m;
  } else if (run_m2p_sorted<R>(&t, pm->par.interpolation_order, pos, pm->start.as<unsigned>(), perm, n, dw, pdvort, st,
                               caller) ||
             run_m2p_sorted<R>(&t, pm->par.interpolation_order, pos, pm->start.as<unsigned>(), perm, n, u, pvel, st,
                               caller)) {
    return -1;
  }
  return run_advance<R>(&pm->patch, &t, a.time_order, a.itimestage, a.dtime, 0, pos, vort, pvel, pdvort, vel_rk,
                        dvort_rk, n, nout, st, caller);
}
}  // namespace pmgpu

int pmgpu_penalisation_stage_dev(pmgpu_plan *plan, pmgpu_plan *penal_plan, const void *d_solid,
                                 const void *d_solid_vel, const pmgpu_penal_stage_args *args, void *d_pos,
                                 void *d_vort, void *d_vel_rk, void *d_dvort_rk, int npart, int max_part,
                                 void *d_part_vel, void *d_part_dvort, int *npart_out, double force[3], int *niter,
                                 double residuals[3], void *stream) {
  const char *caller = "pmgpu_penalisation_stage";
  std::lock_guard<std::mutex> lk(g_mu);
  if (!plan || !args || !npart_out || !force || !niter || !residuals || npart < 0 || max_part < npart ||
      (max_part > 0 && (!d_pos || !d_vort || !d_vel_rk || !d_dvort_rk || !d_part_vel || !d_part_dvort)) ||
      !(args->dtime != 0.0) || args->itimestage < 1 || args->itimestage > args->time_order) {
    set_error(caller, "missing or invalid argument.");
    return -1;
  }
  if (penal_plan && (!d_solid || !d_solid_vel || penal_plan->prec != plan->prec || args->max_iter < 1)) {
    set_error(caller, "missing or invalid penalisation argument.");
    return -1;
  }
  if (ensure_device(caller)) return -1;
  cudaStream_t st = (cudaStream_t)stream;
  if (plan->prec == PMGPU_FP64)
    return penal_stage<double>(plan, penal_plan, (const double *)d_solid, (const double *)d_solid_vel, *args,
                               (double *)d_pos, (double *)d_vort, (double *)d_vel_rk, (double *)d_dvort_rk, npart,
                               max_part, (double *)d_part_vel, (double *)d_part_dvort, npart_out, force, niter,
                               residuals, st);
  return penal_stage<float>(plan, penal_plan, (const float *)d_solid, (const float *)d_solid_vel, *args,
                            (float *)d_pos, (float *)d_vort, (float *)d_vel_rk, (float *)d_dvort_rk, npart, max_part,
                            (float *)d_part_vel, (float *)d_part_dvort, npart_out, force, niter, residuals, st);
}
