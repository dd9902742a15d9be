// solver.cu — host side of the C ABI (include/mmp.h): parameter checks, the
// reference's setup arithmetic, device state, CUDA-graph replay of RK steps.
//
// The setup follows the reference's constructor step by step
// (src/MultimodePropagation.cpp:4-56, :100-155, :165-199) in FP64 on the host;
// everything per step runs on the device in the kernels of stage_kernels.cuh.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#ifndef MMP_NO_NVTX
#include <nvtx3/nvToolsExt.h>
#endif

#include "kernel_table.h"
#include "mmp.h"
#include "stage_kernels.cuh"

using namespace mmp;

// ---------------------------------------------------------------------------------------
// instantiated kernel sets (kern_inst.cu objects)
#define MMP_DECL(tag, L, X) KernelSet make_kernels_##tag##_##L##_##X();
#define MMP_DECL_ALL(tag) \
  MMP_DECL(tag, 6, 0) MMP_DECL(tag, 7, 0) MMP_DECL(tag, 8, 0) MMP_DECL(tag, 9, 0) MMP_DECL(tag, 10, 0) \
  MMP_DECL(tag, 11, 0) MMP_DECL(tag, 12, 0) MMP_DECL(tag, 13, 0) MMP_DECL(tag, 14, 0) MMP_DECL(tag, 15, 0) \
  MMP_DECL(tag, 16, 0)
namespace mmp {
MMP_DECL_ALL(f32)
MMP_DECL_ALL(f64)
MMP_DECL(f32, 12, 1) MMP_DECL(f32, 13, 1) MMP_DECL(f32, 14, 1) MMP_DECL(f32, 15, 1) MMP_DECL(f32, 16, 1)
MMP_DECL(f64, 11, 1) MMP_DECL(f64, 12, 1) MMP_DECL(f64, 13, 1) MMP_DECL(f64, 14, 1)

KernelSet kernels_for(int fp64, int logn, int xc) {
#define MMP_CASE(tag, L, X) case L: return make_kernels_##tag##_##L##_##X();
  if (xc == 1) {
    if (fp64) {
      switch (logn) {
        MMP_CASE(f64, 11, 1) MMP_CASE(f64, 12, 1) MMP_CASE(f64, 13, 1) MMP_CASE(f64, 14, 1)
        default: return KernelSet();
      }
    }
    switch (logn) {
      MMP_CASE(f32, 12, 1) MMP_CASE(f32, 13, 1) MMP_CASE(f32, 14, 1) MMP_CASE(f32, 15, 1) MMP_CASE(f32, 16, 1)
      default: return KernelSet();
    }
  }
  if (xc != 0) return KernelSet();
  if (fp64) {
    switch (logn) {
      MMP_CASE(f64, 6, 0) MMP_CASE(f64, 7, 0) MMP_CASE(f64, 8, 0) MMP_CASE(f64, 9, 0) MMP_CASE(f64, 10, 0)
      MMP_CASE(f64, 11, 0) MMP_CASE(f64, 12, 0) MMP_CASE(f64, 13, 0) MMP_CASE(f64, 14, 0) MMP_CASE(f64, 15, 0)
      MMP_CASE(f64, 16, 0)
      default: return KernelSet();
    }
  }
  switch (logn) {
    MMP_CASE(f32, 6, 0) MMP_CASE(f32, 7, 0) MMP_CASE(f32, 8, 0) MMP_CASE(f32, 9, 0) MMP_CASE(f32, 10, 0)
    MMP_CASE(f32, 11, 0) MMP_CASE(f32, 12, 0) MMP_CASE(f32, 13, 0) MMP_CASE(f32, 14, 0) MMP_CASE(f32, 15, 0)
    MMP_CASE(f32, 16, 0)
    default: return KernelSet();
  }
#undef MMP_CASE
}
}  // namespace mmp

namespace {

std::atomic<uint64_t> g_launches{0};
// Text of the calling thread's last failure (mmp_last_error). A fixed buffer, so that
// recording a failure never allocates (mmp_dft_noalloc reports through it too).
thread_local char g_last_error[512];

int fail_c(int code, const char* msg) {
  std::snprintf(g_last_error, sizeof(g_last_error), "%s", msg ? msg : "");
  return code;
}
int fail(int code, const std::string& msg) { return fail_c(code, msg.c_str()); }

}  // namespace

namespace mmp_detail {
// NVTX range over a host-side phase (create, autotune, propagate, result, ...), for
// timeline tools: a push and a pop of a named range, no-ops unless a tool is attached.
// Build with -DMMP_NO_NVTX to leave them out.
struct Range {
#ifndef MMP_NO_NVTX
  explicit Range(const char* name) { nvtxRangePushA(name); }
  ~Range() { nvtxRangePop(); }
#else
  explicit Range(const char*) {}
#endif
  Range(const Range&) = delete;
  Range& operator=(const Range&) = delete;
};
// for the other units (io.cpp, noalloc.cu): record the text mmp_last_error returns
int set_error(int code, const std::string& msg) { return fail(code, msg); }
int set_error_c(int code, const char* msg) { return fail_c(code, msg); }
// a kernel launched outside launch() (noalloc.cu), counted in mmp_kernel_launch_count
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
}  // namespace mmp_detail

namespace {

#define CUDA_TRY(expr)                                                                 \
  do {                                                                                   \
    cudaError_t e_ = (expr);                                                             \
    if (e_ != cudaSuccess) {                                                             \
      return fail(e_ == cudaErrorMemoryAllocation ? MMP_ENOMEM : MMP_ECUDA,              \
                  std::string(#expr) + ": " + cudaGetErrorString(e_));                   \
    }                                                                                    \
  } while (0)

// *flag = 1 if any of the n complex values is NaN or infinite (set_fields' input check,
// on the device copy of the fields: a host scan of a 28-mode, 65536-sample member took
// 4.5 ms on one core).
__global__ void __launch_bounds__(256) k_check_finite(const double2* __restrict__ x, size_t n, int* flag) {
  bool bad = false;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const double2 v = x[i];
    bad = bad || !isfinite(v.x) || !isfinite(v.y);
  }
  if (__syncthreads_or(bad) && threadIdx.x == 0) *flag = 1;
}

// ---- device allocations: every one goes through dev_malloc / dev_free ------------------
// Failure injection for tests (mmp_debug_fail_alloc): after `g_fail_after` more
// successful allocations the next one fails as cudaErrorMemoryAllocation (-1: never).
// g_live counts the allocations not yet freed (mmp_debug_live_allocations).
std::atomic<int64_t> g_fail_after{-1};
std::atomic<int64_t> g_live{0};

cudaError_t dev_malloc(void** p, size_t bytes, cudaMemPool_t pool = nullptr, cudaStream_t st = nullptr) {
  int64_t n = g_fail_after.load();
  while (n >= 0 && !g_fail_after.compare_exchange_weak(n, n - 1)) {
  }
  if (n == 0) {
    *p = nullptr;
    return cudaErrorMemoryAllocation;
  }
  const cudaError_t e = pool ? cudaMallocFromPoolAsync(p, bytes, pool, st) : cudaMalloc(p, bytes);
  if (e == cudaSuccess) g_live.fetch_add(1);
  else *p = nullptr;
  return e;
}
void dev_free(void* p, cudaStream_t st = nullptr, bool pooled = false) {
  if (!p) return;
  if (pooled) cudaFreeAsync(p, st);
  else cudaFree(p);
  g_live.fetch_sub(1);
}

// shared memory of k_raman_scan: a 128 KB segment of V, padded
constexpr int kScanSmem = padded_len(128 * 1024 / 8) * 8;
// Dynamic shared memory k_contract may take (the 227 KB per block, less its static part)
constexpr size_t kContractSmemMax = 226 * 1024;

// ---- per-device resources: twiddle tables, kernel attributes ------------------------------
struct DeviceRes {
  bool ready = false;
  TwTables tw{};
  void* tw_mem = nullptr;
};
std::mutex g_dev_mu;
std::map<int, DeviceRes> g_dev;

int ensure_device(int dev, DeviceRes** out) {
  std::lock_guard<std::mutex> lk(g_dev_mu);
  DeviceRes& r = g_dev[dev];
  if (r.ready) { *out = &r; return MMP_OK; }
  cudaDeviceProp prop;
  CUDA_TRY(cudaGetDeviceProperties(&prop, dev));
  if (prop.major < 10) return fail(MMP_ENODEV, "device is not sm_100 (compute capability " +
                                   std::to_string(prop.major) + "." + std::to_string(prop.minor) + ")");
  // twiddle tables w_L[m] = exp(-2 pi i m / 2^L), L = 1..16, in FP64 and FP32
  size_t n_tot = 0;
  for (int L = 1; L <= kMaxLogN; ++L) n_tot += (size_t)1 << L;
  std::vector<double2> hd(n_tot);
  std::vector<float2> hf(n_tot);
  size_t off = 0;
  std::vector<size_t> offs(kMaxLogN + 1, 0);
  for (int L = 1; L <= kMaxLogN; ++L) {
    offs[L] = off;
    const size_t n = (size_t)1 << L;
    for (size_t m = 0; m < n; ++m) {
      const double a = -2.0 * M_PI * (double)m / (double)n;
      hd[off + m] = make_double2(std::cos(a), std::sin(a));
      hf[off + m] = make_float2((float)hd[off + m].x, (float)hd[off + m].y);
    }
    off += n;
  }
  // the split rows' combine tables, [n][kl] = w_L[n kl] (n < CG, kl < 2^L / CG), gathered
  // from the tables above, so that they hold the same values
  struct Cmb { int fp64, L, xc; size_t off; };
  std::vector<Cmb> cm;
  size_t cbytes = 0;
  for (int fp64 = 0; fp64 < 2; ++fp64)
    for (int L = kMinLogN; L <= kMaxLogN; ++L)
      for (int xc = 0; xc < 2; ++xc) {
        const KernelSet ks = kernels_for(fp64, L, xc);
        if (!ks.prime || ks.C < 2) continue;
        cm.push_back({fp64, L, xc, cbytes});
        cbytes += ((size_t)1 << L) * (fp64 ? sizeof(double2) : sizeof(float2));
      }
  std::vector<unsigned char> hc(cbytes);
  for (const Cmb& c : cm) {
    const KernelSet ks = kernels_for(c.fp64, c.L, c.xc);
    const size_t n = (size_t)1 << c.L;
    const size_t CG = (size_t)ks.C * (c.fp64 ? 2 : 4);  // C times the run length G (32 bytes)
    for (size_t kl = 0; kl < n / CG; ++kl)
      for (size_t q = 0; q < CG; ++q) {
        const size_t m = q * kl, e = q * (n / CG) + kl;
        if (c.fp64) reinterpret_cast<double2*>(hc.data() + c.off)[e] = hd[offs[c.L] + m];
        else reinterpret_cast<float2*>(hc.data() + c.off)[e] = hf[offs[c.L] + m];
      }
  }
  // one allocation: FP64 tables | FP32 tables | combine tables
  void* mem = nullptr;
  CUDA_TRY(dev_malloc(&mem, n_tot * (sizeof(double2) + sizeof(float2)) + cbytes));
  double2* dd = (double2*)mem;
  float2* df = (float2*)(dd + n_tot);
  unsigned char* dc = (unsigned char*)(df + n_tot);
  cudaError_t ce = cudaMemcpy(dd, hd.data(), n_tot * sizeof(double2), cudaMemcpyHostToDevice);
  if (ce == cudaSuccess) ce = cudaMemcpy(df, hf.data(), n_tot * sizeof(float2), cudaMemcpyHostToDevice);
  if (ce == cudaSuccess && cbytes) ce = cudaMemcpy(dc, hc.data(), cbytes, cudaMemcpyHostToDevice);
  if (ce != cudaSuccess) {
    dev_free(mem);
    return fail(MMP_ECUDA, std::string("twiddle upload: ") + cudaGetErrorString(ce));
  }
  for (int L = 0; L <= kMaxLogN; ++L) {
    r.tw.d[L] = L ? dd + offs[L] : nullptr;
    r.tw.f[L] = L ? df + offs[L] : nullptr;
  }
  for (const Cmb& c : cm) {
    if (c.fp64) r.tw.cd[c.L][c.xc] = (const double2*)(dc + c.off);
    else r.tw.cf[c.L][c.xc] = (const float2*)(dc + c.off);
  }
  r.tw_mem = mem;
  // dynamic shared memory opt-in for every instantiated kernel
  for (int fp64 = 0; fp64 < 2; ++fp64)
    for (int L = kMinLogN; L <= kMaxLogN; ++L)
      for (int xc = 0; xc < 2; ++xc) {
        KernelSet ks = kernels_for(fp64, L, xc);
        if (!ks.prime) continue;
        std::vector<const void*> fns = {ks.prime, ks.pair, ks.nu, ks.result, ks.dft_fwd, ks.dft_inv};
        for (const void* f : ks.nu_mid) if (f) fns.push_back(f);
        for (const void* f : ks.nu_last) if (f) fns.push_back(f);
        for (const void* f : fns)
          CUDA_TRY(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, ks.smem));
      }
  const void* contract_fns[] = {(const void*)&k_contract<float, 0>,  (const void*)&k_contract<float, 1>,
                                (const void*)&k_contract<float, 2>,  (const void*)&k_contract<double, 0>,
                                (const void*)&k_contract<double, 1>, (const void*)&k_contract<double, 2>};
  for (const void* f : contract_fns)
    CUDA_TRY(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kContractSmemMax));
  CUDA_TRY(cudaFuncSetAttribute((const void*)&k_contract_pc<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                110 * 1024));
  CUDA_TRY(cudaFuncSetAttribute((const void*)&k_contract_pc<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                110 * 1024));
  CUDA_TRY(cudaFuncSetAttribute((const void*)&k_contract_tc<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                227 * 1024 - 256));
  CUDA_TRY(cudaFuncSetAttribute((const void*)&k_contract_sr<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                227 * 1024));
  CUDA_TRY(cudaFuncSetAttribute((const void*)&k_contract_sr<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                227 * 1024));
  CUDA_TRY(cudaFuncSetAttribute((const void*)&k_raman_scan<float>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, kScanSmem));
  CUDA_TRY(cudaFuncSetAttribute((const void*)&k_raman_scan<double>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, kScanSmem));
  CUDA_TRY(cudaFuncSetAttribute((const void*)&k_raman_agg<float>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
  CUDA_TRY(cudaFuncSetAttribute((const void*)&k_raman_agg<double>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
  r.ready = true;
  *out = &r;
  return MMP_OK;
}

cudaError_t launch(const void* fn, dim3 grid, int nthr, int smem, int C, cudaStream_t st, void** args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = dim3((unsigned)nthr, 1, 1);
  cfg.dynamicSmemBytes = (size_t)smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  cfg.numAttrs = 0;
  if (C > 1) {
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
  }
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return cudaLaunchKernelExC(&cfg, fn, args);
}

int ilog2_exact(uint32_t n) {
  if (n == 0 || (n & (n - 1))) return -1;
  int l = 0;
  while ((1u << l) < n) ++l;
  return l;
}

// ---- RK tableaus: src/RungeKutta.cpp ------------------------------------------------------
void set_tableau(Tableau& t, const std::vector<std::vector<double>>& a, const std::vector<double>& b,
                 const std::vector<double>& c) {
  std::memset(&t, 0, sizeof(t));
  t.s = (int)b.size();
  for (size_t i = 0; i < a.size(); ++i)
    for (size_t j = 0; j < a[i].size(); ++j) t.a[i][j] = a[i][j];
  for (size_t i = 0; i < b.size(); ++i) t.b[i] = b[i];
  for (size_t i = 0; i < (size_t)t.s; ++i) t.c[i] = c[i];
  t.last_b = 0;
  for (int i = 0; i < t.s; ++i)
    if (t.b[i] != 0.0) t.last_b = i;
}

void tableau_for(const mmp_params* p, Tableau& t) {
  const double s = std::sqrt(21.0);
  if (p->rk_variant == MMP_RK_BUTCHER7_LAMBDA_MU) {
    // src/RungeKutta.cpp:75-122
    const double lam = p->rk_lambda, mu = p->rk_mu;
    set_tableau(t,
                {{0.},
                 {mu},
                 {2 / 3. - 2. / (9. * mu), 2. / (9. * mu)},
                 {5 / 12. - 1. / (9 * mu), 1. / (9 * mu), -1 / 12.},
                 {17 / 16. - 3. / (8. * mu), 3. / (8. * mu), -3 / 16., -3 / 8.},
                 {17 / 16. - 3. / (8 * mu) + 1. / (4. * lam), 3. / (8. * mu), -3 / 16. - 3. / (4. * lam),
                  -3 / 8. - 3. / (2. * lam), 2. / lam},
                 {-27 / 44. + 3. / (11. * mu), -3. / (11. * mu), 63 / 44., 18 / 11., 4. * ((lam - 4.) / 11.),
                  -(4. * lam) / 11.}},
                {1 / 120., 0., 27 / 40., 27 / 40., (lam - 8.) / 15., -lam / 15., 11 / 120.},
                {0., mu, 2 / 3., 1 / 3., 1 / 2., 1 / 2., 1.});
    return;
  }
  switch (p->method_order) {
    case 8:  // Butcher11, src/RungeKutta.cpp:125-175
      set_tableau(
          t,
          {{0.},
           {1 / 2.},
           {1 / 4., 1 / 4.},
           {1 / 7., (-7. + 3. * s) / 98., (21. - 5. * s) / 49.},
           {(11. - s) / 84., 0., (18. - 4. * s) / 63., (21. + s) / 252.},
           {(5. - s) / 48., 0., (9. - s) / 36., (-231. - 14. * s) / 360., (63. + 7. * s) / 80.},
           {(10. + s) / 42., 0., (-432. - 92. * s) / 315., (633. + 145. * s) / 90., (-504. - 115. * s) / 70.,
            (63. + 13. * s) / 35.},
           {1 / 14., 0., 0., 0., (14. + 3. * s) / 126., (13. + 3. * s) / 63., 1 / 9.},
           {1 / 32., 0., 0., 0., (91. + 21. * s) / 576., 11 / 72., (-385. + 75. * s) / 1152.,
            (63. - 13. * s) / 128.},
           {1 / 14., 0., 0., 0., 1 / 9., (-733. + 147. * s) / 2205., (515. - 111. * s) / 504.,
            (-51. + 11. * s) / 56., (132. - 28. * s) / 245.},
           {0., 0., 0., 0., (-42. - 7. * s) / 18., (-18. - 28. * s) / 45., (-273. + 53. * s) / 72.,
            (301. - 53. * s) / 72., (28. + 28. * s) / 45., (49. + 7. * s) / 18.}},
          {1 / 20., 0., 0., 0., 0., 0., 0., 49 / 180., 16 / 45., 49 / 180., 1 / 20.},
          {0., 1 / 2., 1 / 2., (7. - s) / 14., (7. - s) / 14., 1 / 2., (7. + s) / 14., (7. + s) / 14., 1 / 2.,
           (7. - s) / 14., 1.});
      return;
    case 6: {  // Butcher7(nu = 1), src/RungeKutta.cpp:24-72
      const double nu = 1.0;
      set_tableau(t,
                  {{0.},
                   {nu},
                   {(4. * nu - 1.) / (8. * nu), 1. / (8. * nu)},
                   {(10. * nu - 2.) / (27. * nu), 2. / (27. * nu), (8. * nu) / (27. * nu)},
                   {(56. - 77. * nu + (8. - 17. * nu) * s) / (392. * nu), (-8. * (7. + s)) / (392. * nu),
                    (48. * (7. + s) * nu) / (392. * nu), (-3. * (21. + s) * nu) / (392. * nu)},
                   {(-5. * (287. * nu - 56. - (59. * nu - 8.) * s)) / (1960. * nu), (-40. * (7. - s)) / (1960. * nu),
                    (320. * s * nu) / (1960. * nu), (3. * (21. - 121. * s) * nu) / (1960. * nu),
                    (392. * (6. - s) * nu) / (1960. * nu)},
                   {(15. * ((30. * nu - 8.) - 7. * nu * s)) / (180. * nu), 120. / (180. * nu),
                    (-40. * (5. + 7. * s) * nu) / (180. * nu), (63. * (2. + 3. * s) * nu) / (180. * nu),
                    (-14. * (49. - 9. * s) * nu) / (180. * nu), (70. * (7. + s) * nu) / (180. * nu)}},
                  {9 / 180., 0., 64 / 180., 0., 49 / 180., 49 / 180., 9 / 180.},
                  {0., nu, 1 / 2., 2 / 3., (7. + s) / 14., (7. - s) / 14., 1.});
      return;
    }
    default:  // Butcher4, src/RungeKutta.cpp:3-21
      set_tableau(t, {{0.}, {1 / 2.}, {0., 1 / 2.}, {0., 0., 1.}}, {1 / 6., 1 / 3., 1 / 3., 1 / 6.},
                  {0., 1 / 2., 1 / 2., 1.});
      return;
  }
}

// ---- one solve: host setup and device buffers ---------------------------------------------
struct Member {
  uint32_t M = 0, nt = 0, n_beta = 0, n_steps = 0;
  double T0 = 0, LD = 0, t_final = 0, delta_t = 0, z_final = 0, delta_z = 0, cf = 0;
  double fiber_length = 0;  // m (snapshot positions)
  double max_beta2 = 0, max_Q = 0, sgn_gamma = 1, fR = 0, omega0 = 0;
  std::vector<uint32_t> unique_pairs;
  std::vector<int2> pairs;
  std::vector<Term> terms;
  std::vector<int> term_off;
  // terms merged per (p, k, pair field) for k_contract_sr: coefficients (a, b), k | q << 16,
  // offsets per p, modes by descending merged-term count
  std::vector<double> sr_ab;
  std::vector<unsigned> sr_kq;
  std::vector<int> sr_off;    // [M + 1]
  std::vector<int4> sr_plan;  // k_contract_sr's group plan (SolveDesc::sr_plan)
  int sr_rounds = 0;
  std::vector<double> poly;
  bool quirk = false;
  bool dense_ok = false;  // the dense contraction form is built for this solve
  uint32_t flags = 0;
  // device
  void* block = nullptr;  // one allocation for all per-solve buffers
  SolveDesc desc{};
  unsigned long long* counters = nullptr;  // step, total, done_ctr|status
  double* energy = nullptr;
  double* photons = nullptr;
  unsigned long long mon_cap = 0;
  unsigned long long total_host = 0;  // steps enqueued since creation
  unsigned long long step_host = 0;   // steps since the last z reset
  size_t bytes = 0;                   // device bytes of `block`
};

int validate(const mmp_params* p, std::string& why) {
  if (!p) { why = "params is NULL"; return MMP_EINVAL; }
  if (p->n_modes == 0) { why = "n_modes must be >= 1"; return MMP_EINVAL; }
  if (p->nt == 0) { why = "nt must be >= 1"; return MMP_EINVAL; }
  if (!p->dispersion) { why = "dispersion_coefficients is NULL"; return MMP_EINVAL; }
  if (p->n_beta < 3) {
    why = "dispersion_coefficients needs >= 3 orders per mode (beta[p][2] is read, src/MultimodePropagation.cpp:71)";
    return MMP_EINVAL;
  }
  if (p->n_beta > (uint32_t)kMaxBeta) { why = "at most 13 dispersion orders (int factorial of the reference overflows beyond 12!)"; return MMP_EINVAL; }
  if (!p->initial_fields) { why = "initial_fields is NULL"; return MMP_EINVAL; }
  if (p->n_nonzeros && !p->coupling) { why = "coupling is NULL with n_nonzeros > 0"; return MMP_EINVAL; }
  if (!(p->pulse_width > 0) || !std::isfinite(p->pulse_width)) { why = "pulse_width must be > 0"; return MMP_EINVAL; }
  if (!(p->time_window > 0) || !std::isfinite(p->time_window)) { why = "time_window must be > 0"; return MMP_EINVAL; }
  if (!(p->fiber_length > 0) || !std::isfinite(p->fiber_length)) { why = "fiber_length must be > 0"; return MMP_EINVAL; }
  if (p->n_steps == 0) { why = "n_steps must be >= 1"; return MMP_EINVAL; }
  if (!std::isfinite(p->nonlinearity_const)) { why = "nonlinearity_const must be finite"; return MMP_EINVAL; }
  if (p->nonlinearity_const == 0) {
    // the reference then scales the fields by 0 and its getResult divides by 0: all NaN
    // (src/MultimodePropagation.cpp:53, :61; src/MultimodePropagation_CPU.cpp:100)
    why = "nonlinearity_const is 0: the conversion factor sqrt(|gamma| LD) sqrt(max|Q|) is 0";
    return MMP_EINVAL;
  }
  double mb2 = 0, mq = 0;
  for (uint32_t m = 0; m < p->n_modes; ++m) {
    for (uint32_t i = 0; i < p->n_beta; ++i)
      if (!std::isfinite(p->dispersion[m * p->n_beta + i])) { why = "dispersion coefficient not finite"; return MMP_EINVAL; }
    mb2 = std::max(mb2, std::fabs(p->dispersion[m * p->n_beta + 2]));
  }
  if (mb2 == 0) { why = "max |beta2| is 0: the reference's dispersion length T0^2/max|beta2| is infinite"; return MMP_EINVAL; }
  for (uint32_t j = 0; j < p->n_nonzeros; ++j) {
    const mmp_nz& e = p->coupling[j];
    if (e.p >= p->n_modes || e.k >= p->n_modes || e.l >= p->n_modes || e.m >= p->n_modes) {
      why = "coupling index out of range (entry " + std::to_string(j) + ")";
      return MMP_EINVAL;
    }
    if (!std::isfinite(e.value)) { why = "coupling value not finite (entry " + std::to_string(j) + ")"; return MMP_EINVAL; }
    mq = std::max(mq, std::fabs(e.value));
  }
  if (mq == 0) { why = "max |Q| is 0: the reference divides Q by it (src/MultimodePropagation.cpp:117-136)"; return MMP_EINVAL; }
  if (p->raman) {
    if (!p->raman_response) { why = "raman_response is NULL for a Raman-on solver"; return MMP_EINVAL; }
    if (!std::isfinite(p->raman_proportion)) { why = "raman_proportion not finite"; return MMP_EINVAL; }
    for (uint32_t t = 0; t < p->nt; ++t)
      if (!std::isfinite(p->raman_response[t])) { why = "raman_response not finite"; return MMP_EINVAL; }
  }
  for (size_t t = 0; t < 2 * (size_t)p->n_modes * p->nt; ++t)
    if (!std::isfinite(p->initial_fields[t])) { why = "initial_fields not finite"; return MMP_EINVAL; }
  if (p->rk_variant == MMP_RK_BUTCHER7_LAMBDA_MU && (p->rk_lambda == 0 || p->rk_mu == 0)) {
    why = "Butcher7(lambda, mu) needs lambda != 0 and mu != 0"; return MMP_EINVAL;
  }
  if (p->rk_variant != MMP_RK_BY_ORDER && p->rk_variant != MMP_RK_BUTCHER7_LAMBDA_MU) {
    why = "unknown rk_variant"; return MMP_EINVAL;
  }
  const int lg = ilog2_exact(p->nt);
  if (lg < kMinLogN || lg > kMaxLogN) {
    why = "nt must be a power of two in [64, 65536] in this build";
    return MMP_ENOTSUP;
  }
  return MMP_OK;
}

// k_contract_sr's phase B plan: kSrGroups groups of eight lanes per round, as many rounds as
// modes need. Groups left over after one per mode go to the modes with the most merged terms,
// which are split in two halves in adjacent groups of one warp (pairs of groups 0-1 or 2-3);
// the units are placed in descending term count so that groups of similar length share a
// warp. Entry: (p, first term, end, role), role 0 whole, 1 lower half, 2 upper half, 3 empty.
void sr_make_plan(Member& s) {
  const int M = (int)s.M;
  const int rounds = std::max(1, (M + kSrGroups - 1) / kSrGroups);
  const int S = rounds * kSrGroups;
  std::vector<int> order(M);
  for (int q = 0; q < M; ++q) order[q] = q;
  auto cnt = [&](int q) { return s.sr_off[q + 1] - s.sr_off[q]; };
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return cnt(x) > cnt(y); });
  struct Unit { int p, n0, n1, halves, cost; };
  std::vector<Unit> units;
  int spare = S - M;
  for (int q : order) {
    const bool split = spare > 0 && cnt(q) >= 2;
    if (split) --spare;
    units.push_back({q, s.sr_off[q], s.sr_off[q + 1], split ? 2 : 1, split ? (cnt(q) + 1) / 2 : cnt(q)});
  }
  std::stable_sort(units.begin(), units.end(), [](const Unit& a, const Unit& b) { return a.cost > b.cost; });
  s.sr_plan.assign(S, make_int4(0, 0, 0, 3));
  std::vector<char> used(S, 0);
  for (const Unit& u : units) {
    int slot = -1;
    if (u.halves == 2)
      for (int g = 0; g + 1 < S && slot < 0; g += 2)
        if (!used[g] && !used[g + 1]) slot = g;
    if (slot >= 0) {
      const int mid = u.n0 + (u.n1 - u.n0 + 1) / 2;
      s.sr_plan[slot] = make_int4(u.p, u.n0, mid, 1);
      s.sr_plan[slot + 1] = make_int4(u.p, mid, u.n1, 2);
      used[slot] = used[slot + 1] = 1;
      continue;
    }
    for (int g = 0; g < S && slot < 0; ++g)  // whole (also a split that found no aligned pair)
      if (!used[g]) slot = g;
    s.sr_plan[slot] = make_int4(u.p, u.n0, u.n1, 0);
    used[slot] = 1;
  }
  s.sr_rounds = rounds;
}

// The reference's setup, in FP64 with the same expressions.
void host_setup(const mmp_params* p, Member& s) {
  const uint32_t M = p->n_modes, L = p->n_beta;
  s.M = M; s.nt = p->nt; s.n_beta = L; s.n_steps = p->n_steps; s.flags = p->flags;
  s.T0 = p->pulse_width;
  const double gamma = p->nonlinearity_const;
  s.sgn_gamma = gamma >= 0 ? 1.0 : -1.0;                              // :34
  double max_beta2 = 0;                                                // :67-77
  for (uint32_t q = 0; q < M; ++q) max_beta2 = std::max(max_beta2, std::fabs(p->dispersion[q * L + 2]));
  double max_Q = 0;                                                    // :81-97
  for (uint32_t j = 0; j < p->n_nonzeros; ++j) max_Q = std::max(max_Q, std::fabs(p->coupling[j].value));
  s.max_beta2 = max_beta2;
  s.max_Q = max_Q;
  s.LD = (s.T0 * s.T0) / max_beta2;                                    // :42
  std::vector<double> c(L);
  for (uint32_t i = 0; i < L; ++i) c[i] = 1. / std::pow(s.T0, (double)i) * s.LD;  // :100-106
  s.t_final = p->time_window / s.T0;                                   // :47-48
  s.delta_t = s.t_final / s.nt;
  s.z_final = p->fiber_length / s.LD;                                  // :50-51
  s.fiber_length = p->fiber_length;
  s.delta_z = s.z_final / p->n_steps;
  s.cf = std::sqrt(std::fabs(gamma) * s.LD) * std::sqrt(max_Q);        // :53
  s.fR = p->raman ? p->raman_proportion : 0.0;
  s.omega0 = p->center_frequency;
  // Im L_p(alpha) = bt0 - bt1 alpha - bt2/2 alpha^2 + sum_{k>=3} (-1)^k bt_k/k! alpha^k (:165-187)
  s.poly.assign((size_t)M * L, 0.0);
  for (uint32_t q = 0; q < M; ++q) {
    for (uint32_t i = 0; i < L; ++i) {
      const double bt = p->dispersion[q * L + i] * c[i];
      double coef;
      if (i == 0) coef = bt;
      else if (i == 1) coef = -bt;
      else if (i == 2) coef = -bt / 2;
      else {
        double fact = 1;
        for (uint32_t f = 2; f <= i; ++f) fact *= f;
        coef = ((i % 2) ? -1.0 : 1.0) * bt / fact;
      }
      s.poly[q * L + i] = coef;
    }
  }
  // unique_pairs: p outer, insertion order inner (:139-155)
  std::vector<std::vector<const mmp_nz*>> byp(M);
  for (uint32_t j = 0; j < p->n_nonzeros; ++j) byp[p->coupling[j].p].push_back(&p->coupling[j]);
  std::map<uint32_t, uint32_t> slot_of;
  for (uint32_t q = 0; q < M; ++q)
    for (const mmp_nz* e : byp[q]) {
      const uint32_t code = e->l + e->m * M;
      if (!slot_of.count(code)) {
        slot_of[code] = (uint32_t)s.unique_pairs.size();
        s.unique_pairs.push_back(code);
      }
    }
  const bool physical = (p->flags & MMP_F_PHYSICAL_PAIRS) != 0;
  s.quirk = false;
  for (size_t i = 0; i < s.unique_pairs.size(); ++i)
    if (s.unique_pairs[i] != i) s.quirk = !physical;
  // contraction terms with the pair each one actually reads
  // (reference CPU: V[slot] = U[slot % M] conj(U[slot / M]), :126-133, :195-205)
  auto pair_of = [&](const mmp_nz* e, int& le, int& me) {
    const uint32_t code = e->l + e->m * M;
    const uint32_t src = physical ? code : slot_of[code];
    le = (int)(src % M);
    me = (int)(src / M);
    return std::make_pair(std::min(le, me), std::max(le, me));
  };
  // the pair fields the non-zero terms read, numbered block by block over the (l, m)
  // triangle, blocks of 8 l by 2 m: a warp's 32 consecutive pair fields (one per lane in
  // k_contract_sr and k_raman_agg_sr) then read few distinct U rows, whose 16-byte loads
  // share wavefronts (the rows start 4 banks apart). Measured on the 28-mode sweep against
  // (l, m) order: k_raman_agg_sr 0.544 -> 0.469 ms, k_contract_sr 2.08 -> 2.02 ms.
  std::map<std::pair<int, int>, int> pair_idx;
  for (uint32_t q = 0; q < M; ++q)
    for (const mmp_nz* e : byp[q]) {
      int le, me;
      if (e->value != 0.0) pair_idx[pair_of(e, le, me)] = 0;
    }
  {
    std::vector<std::pair<int, int>> order;
    for (const auto& kv : pair_idx) order.push_back(kv.first);
    auto key = [](const std::pair<int, int>& x) {
      return std::make_tuple(x.first / 8, x.second / 2, x.first % 8, x.second % 2);
    };
    std::stable_sort(order.begin(), order.end(),
                     [&](const std::pair<int, int>& a, const std::pair<int, int>& b) { return key(a) < key(b); });
    for (const auto& lm : order) {
      pair_idx[lm] = (int)s.pairs.size();
      s.pairs.push_back(make_int2(lm.first, lm.second));
    }
  }
  s.term_off.assign(M + 1, 0);
  for (uint32_t q = 0; q < M; ++q) {
    s.term_off[q] = (int)s.terms.size();
    for (const mmp_nz* e : byp[q]) {
      if (e->value == 0.0) continue;  // contributes exactly 0
      int le, me;
      const int idx = pair_idx[pair_of(e, le, me)];
      Term t;
      t.k = (unsigned short)e->k;
      t.l = (unsigned short)le;
      t.m = (unsigned short)me;
      t.pc = (unsigned short)(idx | (le > me ? 0x8000 : 0));  // R_ml = conj(R_lm): h_R is real
      t.q = e->value / max_Q;                                  // Q_tilde (:117-136)
      s.terms.push_back(t);
    }
    // each p's terms in pair-field order (stable): the pair-chunked contraction walks
    // them chunk by chunk with one cursor
    std::stable_sort(s.terms.begin() + s.term_off[q], s.terms.end(),
                     [](const Term& a, const Term& b) { return (a.pc & 0x7fff) < (b.pc & 0x7fff); });
  }
  s.term_off[M] = (int)s.terms.size();
  // merged terms: Q1 W + Q2 conj(W) = (Q1 + Q2) Re W + i (Q1 - Q2) Im W for the terms of p
  // with the same k and pair field (both readings of a symmetric coupling), one record each
  s.sr_ab.clear();
  s.sr_kq.clear();
  s.sr_off.assign(M + 1, 0);
  for (uint32_t q = 0; q < M; ++q) {
    s.sr_off[q] = (int)s.sr_kq.size();
    std::map<std::pair<int, int>, std::pair<double, double>> merged;  // (k, pair) -> (a, b)
    for (int j = s.term_off[q]; j < s.term_off[q + 1]; ++j) {
      const Term& t = s.terms[j];
      auto& ab = merged[std::make_pair((int)t.k, (int)(t.pc & 0x7fff))];
      ab.first += t.q;
      ab.second += (t.pc & 0x8000) ? -t.q : t.q;
    }
    for (const auto& e : merged) {
      s.sr_ab.push_back(e.second.first);
      s.sr_ab.push_back(e.second.second);
      s.sr_kq.push_back((unsigned)e.first.second | ((unsigned)e.first.first << 16));
    }
  }
  s.sr_off[M] = (int)s.sr_kq.size();
  sr_make_plan(s);
}

size_t align_up(size_t x) { return (x + 255) & ~(size_t)255; }

}  // namespace

// ---------------------------------------------------------------------------------------
struct mmp_batch {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool fp64 = false, raman = false;
  uint32_t nt = 0;
  int logn = 0;
  Tableau tab{};
  // Slots: `capacity` descriptors on the device; members[i] is in use when active[i].
  // An ordinary batch fills every slot; a served pool admits and retires solves
  // between graph replays, and the kernels skip empty slots (M = 0).
  uint32_t capacity = 0;
  std::vector<Member> members;
  std::vector<uint8_t> active;
  SolveDesc* d_descs = nullptr;
  int* d_flag = nullptr;  // set_fields' non-finite-input flag (in the d_descs allocation)
  uint32_t span = 0;  // slots the kernels are launched over: highest active slot + 1
  // Served pools take solve state from a stream-ordered pool (no device-wide
  // synchronisation when a solve is admitted or retired); null: cudaMalloc/cudaFree.
  cudaMemPool_t mempool = nullptr;
  // graph branches: solves split into `groups` independent kernel chains (capture_steps)
  uint32_t groups = 1;
  bool raman_iir = false;  // every solve's h_R is a damped sinusoid: pair fields by k_raman_scan
  bool raman_fused = false;  // ... and the recurrence runs inside the contraction tiles
  int dense = 0;  // contraction form: 0 term loop, 1 dense (k_contract<T, 1>), 2 per solve
  bool tc = false;  // dense form on the tensor cores (k_contract_tc)
  int pchunk = 0;   // > 0: pair fields per chunk of the pair-chunked contraction (k_contract_pc)
  bool sr = false;  // serial-recurrence contraction in sub-blocks (k_contract_sr)
  int tile_req = 0;  // contraction tile asked for by the autotuner (0: batch_shape's own)
  int tuned = 0;     // 1: launch parameters chosen by timing (autotune)
  std::vector<cudaStream_t> branch;
  std::vector<cudaEvent_t> branch_ev;
  cudaEvent_t fork_ev = nullptr;
  int Mmax = 0, Pmax = 0;
  int TT = 32;
  int stage_terms = 0;
  size_t contract_smem = 0;
  KernelSet ks{}, ks64{};
  DeviceRes* dev = nullptr;
  cudaGraphExec_t graph = nullptr;
  int graph_steps = 0;
  int kernels_per_step = 0;
};

struct mmp_solver {
  mmp_batch* b = nullptr;
};

namespace {

void* T2ptr(void* base, size_t off) { return (char*)base + off; }

int upload_desc(mmp_batch* b) {
  std::vector<SolveDesc> h(b->capacity);
  for (size_t i = 0; i < b->capacity; ++i) {
    if (b->active[i]) {
      h[i] = b->members[i].desc;
    } else {
      std::memset(&h[i], 0, sizeof(SolveDesc));  // empty slot: M = 0, every kernel skips it
    }
  }
  CUDA_TRY(cudaMemcpyAsync(b->d_descs, h.data(), h.size() * sizeof(SolveDesc), cudaMemcpyHostToDevice,
                           b->stream));
  CUDA_TRY(cudaStreamSynchronize(b->stream));  // h is a host temporary
  return MMP_OK;
}

int grow_monitors(mmp_batch* b, Member& s, unsigned long long need) {
  if (need <= s.mon_cap) return MMP_OK;
  unsigned long long cap = std::max<unsigned long long>(need, s.mon_cap * 2);
  cap = std::max<unsigned long long>(cap, 1024);
  double* mem = nullptr;
  CUDA_TRY(dev_malloc((void**)&mem, 2 * cap * sizeof(double)));
  cudaError_t e = cudaMemsetAsync(mem, 0, 2 * cap * sizeof(double), b->stream);
  if (s.mon_cap) {
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(mem, s.energy, s.mon_cap * sizeof(double), cudaMemcpyDeviceToDevice, b->stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(mem + cap, s.photons, s.mon_cap * sizeof(double), cudaMemcpyDeviceToDevice, b->stream);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
  if (e != cudaSuccess) {
    dev_free(mem);
    return fail(MMP_ECUDA, std::string("monitor buffers: ") + cudaGetErrorString(e));
  }
  dev_free(s.energy);
  s.energy = mem;
  s.photons = mem + cap;
  s.mon_cap = cap;
  s.desc.energy = s.energy;
  s.desc.photons = s.photons;
  s.desc.mon_cap = cap;
  return upload_desc(b);
}

// launch helpers ------------------------------------------------------------------------
KParams kparams(mmp_batch* b, int stage, const SolveDesc* descs) {
  KParams kp;
  std::memset(&kp, 0, sizeof(kp));
  kp.descs = descs;
  kp.tw = b->dev->tw;
  kp.tab = b->tab;
  kp.stage = stage;
  return kp;
}

int launch_row_kernel(mmp_batch* b, const KernelSet& ks, const void* fn, int rows, int nsolves, int stage,
                      const SolveDesc* descs, cudaStream_t st = nullptr) {
  if (rows <= 0 || nsolves <= 0) return MMP_OK;
  KParams kp = kparams(b, stage, descs);
  void* args[] = {&kp};
  dim3 grid((unsigned)(rows * ks.C), (unsigned)nsolves, 1);
  CUDA_TRY(launch(fn, grid, ks.nthr, ks.smem, ks.C, st ? st : b->stream, args));
  return MMP_OK;
}

// contraction over solves [first, first + count) (default: every slot)
int launch_contract(mmp_batch* b, uint32_t first = 0, uint32_t count = ~0u, cudaStream_t st = nullptr) {
  if (count == ~0u) count = b->span;
  if (count == 0) return MMP_OK;
  const SolveDesc* descs = b->d_descs + first;
  int nt = (int)b->nt, TT = b->TT, sterms = b->stage_terms;
  int mode = !b->raman ? 0 : (b->raman_fused ? 2 : 1);
  void* args[] = {(void*)&descs, &nt, &TT, &sterms, &mode};
  dim3 grid((unsigned)(b->nt / b->TT), count, 1);
  const void* f32[] = {(const void*)&k_contract<float, 0>, (const void*)&k_contract<float, 1>,
                       (const void*)&k_contract<float, 2>};
  const void* f64[] = {(const void*)&k_contract<double, 0>, (const void*)&k_contract<double, 1>,
                       (const void*)&k_contract<double, 2>};
  if (b->sr) {
    int tb = b->TT;
    void* sargs[] = {(void*)&descs, &nt, &tb, &mode};
    const void* fsr = b->fp64 ? (const void*)&k_contract_sr<double> : (const void*)&k_contract_sr<float>;
    CUDA_TRY(launch(fsr, grid, kSrThreads, (int)b->contract_smem, 1, st ? st : b->stream, sargs));
    return MMP_OK;
  }
  if (b->pchunk) {
    int pc = b->pchunk;
    void* pargs[] = {(void*)&descs, &nt, &TT, &pc};
    const void* fpc = b->fp64 ? (const void*)&k_contract_pc<double> : (const void*)&k_contract_pc<float>;
    CUDA_TRY(launch(fpc, grid, 256, (int)b->contract_smem, 1, st ? st : b->stream, pargs));
    return MMP_OK;
  }
  if (b->tc) {
    void* targs[] = {(void*)&descs, &nt, &mode};
    CUDA_TRY(launch((const void*)&k_contract_tc<float>, grid, 512, (int)b->contract_smem, 1, st ? st : b->stream, targs));
    return MMP_OK;
  }
  const void* fn = b->fp64 ? f64[b->dense] : f32[b->dense];
  CUDA_TRY(launch(fn, grid, 256, (int)b->contract_smem, 1, st ? st : b->stream, args));
  return MMP_OK;
}

// The k_nu instantiation for stage i: a stage whose count of stored N_hat_j terms (the
// count k_nu's thread 0 derives) has a specialised body built takes it; every other
// stage the generic one.
const void* nu_kernel(const KernelSet& ks, const Tableau& tab, int i) {
  const bool last = i == tab.s - 1;
  int nq = 0;
  if (last) {
    for (int j = 0; j < tab.s; ++j) nq += (j != i && tab.b[j] != 0.0);
  } else {
    for (int j = 0; j < i; ++j) nq += (tab.a[i + 1][j] != 0.0);
  }
  if (!last && nq < 6 && ks.nu_mid[nq]) return ks.nu_mid[nq];
  if (last && nq < 5 && ks.nu_last[nq]) return ks.nu_last[nq];
  return ks.nu;
}

// Raman pair fields for `nsolves` solves from descs: with the recurrence fused into the
// contraction, its tile aggregates and carries; else the recurrence as a row scan when
// every solve's h_R is a damped sinusoid; else the FFT convolution of kernel set ks.
int launch_pairs(mmp_batch* b, const KernelSet& ks, int nsolves, int stage, const SolveDesc* descs,
                 cudaStream_t st = nullptr) {
  if (!(b->raman && b->Pmax > 0) || nsolves <= 0) return MMP_OK;
  if (!b->raman_iir) return launch_row_kernel(b, ks, ks.pair, b->Pmax, nsolves, stage, descs, st);
  int nt = (int)b->nt;
  if (b->raman_fused) {
    const size_t t2 = b->fp64 ? sizeof(double2) : sizeof(float2);
    int TT = b->TT;
    const SolveDesc* dd = descs;
    void* args[] = {(void*)&dd, &nt, &TT};
    if (b->sr) {  // one thread per pair field through the tile (k_contract_sr's tiles)
      const int smem = (int)(2 * (size_t)b->Mmax * (kSrSub / 2 + 1) * 2 * t2);
      const void* fa = b->fp64 ? (const void*)&k_raman_agg_sr<double> : (const void*)&k_raman_agg_sr<float>;
      CUDA_TRY(launch(fa, dim3((unsigned)(nt / TT), (unsigned)nsolves, 1), kSrThreads, smem, 1,
                      st ? st : b->stream, args));
    } else {
      const int smem = (int)(((size_t)b->Mmax * TT + TT) * t2);  // U tile and the weight table
      const void* fa = b->fp64 ? (const void*)&k_raman_agg<double> : (const void*)&k_raman_agg<float>;
      CUDA_TRY(launch(fa, dim3((unsigned)(nt / TT), (unsigned)nsolves, 1), 256, smem, 1, st ? st : b->stream, args));
    }
    const void* fc = b->fp64 ? (const void*)&k_raman_carry<double> : (const void*)&k_raman_carry<float>;
    CUDA_TRY(launch(fc, dim3((unsigned)b->Pmax, (unsigned)nsolves, 1), 32, 0, 1, st ? st : b->stream, args));
    return MMP_OK;
  }
  // segments of at most 128 KB of V staged in shared memory
  const size_t t2 = b->fp64 ? sizeof(double2) : sizeof(float2);
  int seg = std::min(nt, (int)((128 * 1024) / t2));
  const int thr = std::max(32, std::min(512, seg / 8));
  const int smem = padded_len(seg) * (int)t2;
  const SolveDesc* dd = descs;
  void* args[] = {(void*)&dd, &nt, &seg};
  const void* fn = b->fp64 ? (const void*)&k_raman_scan<double> : (const void*)&k_raman_scan<float>;
  CUDA_TRY(launch(fn, dim3((unsigned)b->Pmax, (unsigned)nsolves, 1), thr, smem, 1, st ? st : b->stream, args));
  return MMP_OK;
}

// One RK step for solves [first, first + count) on stream st (default: all, batch stream).
int enqueue_step(mmp_batch* b, uint32_t first = 0, uint32_t count = ~0u, cudaStream_t st = nullptr) {
  if (count == ~0u) count = b->span;
  const SolveDesc* descs = b->d_descs + first;
  for (int i = 0; i < b->tab.s; ++i) {
    int rc = launch_pairs(b, b->ks, (int)count, i, descs, st);
    if (rc) return rc;
    rc = launch_contract(b, first, count, st);
    if (rc) return rc;
    rc = launch_row_kernel(b, b->ks, nu_kernel(b->ks, b->tab, i), b->Mmax, (int)count, i, descs, st);
    if (rc) return rc;
  }
  return MMP_OK;
}

// Capture `steps` RK steps. With b->groups > 1 the solves are split into that many
// contiguous groups whose kernel chains are independent branches of the graph: the
// solves of a batch never depend on one another, so one group's launches fill the
// SMs that another group's launch tail leaves idle.
int capture_steps(mmp_batch* b, int steps) {
  const uint32_t G = std::max<uint32_t>(1, std::min<uint32_t>(b->groups, b->span));
  if (G == 1) {
    int rc = MMP_OK;
    for (int k = 0; k < steps && rc == MMP_OK; ++k) rc = enqueue_step(b);
    return rc;
  }
  while (b->branch.size() < G) {
    cudaStream_t s = nullptr;
    CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    b->branch.push_back(s);
    cudaEvent_t e = nullptr;
    CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    b->branch_ev.push_back(e);
  }
  if (!b->fork_ev) CUDA_TRY(cudaEventCreateWithFlags(&b->fork_ev, cudaEventDisableTiming));
  cudaEvent_t fork = b->fork_ev;
  CUDA_TRY(cudaEventRecord(fork, b->stream));
  int rc = MMP_OK;
  for (uint32_t g = 0; g < G && rc == MMP_OK; ++g) {
    const uint32_t lo = g * b->span / G, hi = (g + 1) * b->span / G;
    CUDA_TRY(cudaStreamWaitEvent(b->branch[g], fork, 0));
    for (int k = 0; k < steps && rc == MMP_OK; ++k) rc = enqueue_step(b, lo, hi - lo, b->branch[g]);
  }
  for (uint32_t g = 0; g < G; ++g) {  // join (also on error: the capture must close)
    CUDA_TRY(cudaEventRecord(b->branch_ev[g], b->branch[g]));
    CUDA_TRY(cudaStreamWaitEvent(b->stream, b->branch_ev[g], 0));
  }
  return rc;
}

int build_graph(mmp_batch* b, int steps) {
  if (b->graph && b->graph_steps == steps) return MMP_OK;
  mmp_detail::Range range("mmp.capture_graph");
  if (b->graph) {
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
  }
  cudaGraph_t g = nullptr;
  const uint64_t counted = g_launches.load();
  CUDA_TRY(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
  int rc = capture_steps(b, steps);
  cudaError_t e = cudaStreamEndCapture(b->stream, &g);
  g_launches.store(counted);  // captured launches run (and are counted) at replay
  if (rc) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (e != cudaSuccess) return fail(MMP_ECUDA, std::string("stream capture: ") + cudaGetErrorString(e));
  e = cudaGraphInstantiate(&b->graph, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return fail(MMP_ECUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
  b->graph_steps = steps;
  return MMP_OK;
}

int check_status(mmp_batch* b) {
  int bad = 0;
  for (auto& s : b->members) {
    if (!s.block) continue;  // empty slot
    int st = 0;
    CUDA_TRY(cudaMemcpy(&st, (char*)s.counters + 3 * sizeof(unsigned long long), sizeof(int),
                        cudaMemcpyDeviceToHost));
    bad |= st;
  }
  if (bad & kStatusTimeout) return fail(MMP_ETIMEOUT, "a device-side bounded wait gave up");
  if (bad & kStatusNonFinite) return fail(MMP_ENONFINITE, "the field became NaN/Inf during propagation");
  if (bad & kStatusDrift)
    return fail(MMP_EDRIFT, "the FP64 energy monitor left the band set by mmp_set_energy_drift_limit");
  return MMP_OK;
}

int batch_propagate_async(mmp_batch* b, uint32_t nz) {
  if (!b) return fail(MMP_EINVAL, "NULL batch");
  mmp_detail::Range range("mmp.propagate");
  CUDA_TRY(cudaSetDevice(b->device));
  for (auto& s : b->members) {
    if (!s.block) continue;  // empty slot
    const bool continuous = (s.flags & MMP_F_CONTINUOUS) != 0;
    if (!continuous) {
      // initLawsonRK: z = 0 (src/MultimodePropagation.cpp:158-163)
      CUDA_TRY(cudaMemsetAsync(s.counters, 0, sizeof(unsigned long long), b->stream));
      s.step_host = 0;
    }
    if (!(s.flags & MMP_F_NO_MONITORS)) {
      int rc = grow_monitors(b, s, s.total_host + nz);
      if (rc) return rc;
    }
  }
  if (nz == 0) return MMP_OK;
  // U for stage 0 at the current z
  int rc = launch_row_kernel(b, b->ks, b->ks.prime, b->Mmax, (int)b->span, 0, b->d_descs);
  if (rc) return rc;
  const int G = 8;  // steps per captured graph
  uint32_t left = nz;
  if (left >= (uint32_t)G) {
    rc = build_graph(b, G);
    if (rc) return rc;
    while (left >= (uint32_t)G) {
      CUDA_TRY(cudaGraphLaunch(b->graph, b->stream));
      g_launches.fetch_add((uint64_t)G * b->kernels_per_step, std::memory_order_relaxed);
      left -= G;
    }
  }
  for (uint32_t k = 0; k < left; ++k) {
    rc = enqueue_step(b);
    if (rc) return rc;
  }
  for (auto& s : b->members) {
    s.total_host += nz;
    s.step_host += nz;
  }
  return MMP_OK;
}

int batch_sync(mmp_batch* b) {
  mmp_detail::Range range("mmp.synchronize");
  CUDA_TRY(cudaSetDevice(b->device));
  CUDA_TRY(cudaStreamSynchronize(b->stream));
  return check_status(b);
}

int member_result(mmp_batch* b, uint32_t idx, double* out) {
  if (!b || idx >= b->members.size() || !out) return fail(MMP_EINVAL, "bad result arguments");
  mmp_detail::Range range("mmp.get_result");
  CUDA_TRY(cudaSetDevice(b->device));
  Member& s = b->members[idx];
  int rc = launch_row_kernel(b, b->ks64, b->ks64.result, (int)s.M, 1, 0, b->d_descs + idx);
  if (rc) return rc;
  CUDA_TRY(cudaMemcpyAsync(out, s.desc.io, (size_t)s.M * s.nt * sizeof(double2), cudaMemcpyDeviceToHost,
                           b->stream));
  CUDA_TRY(cudaStreamSynchronize(b->stream));
  return MMP_OK;
}

int member_set_fields(mmp_batch* b, uint32_t idx, const double* phi0) {
  if (!b || idx >= b->members.size() || !phi0) return fail(MMP_EINVAL, "bad set_fields arguments");
  mmp_detail::Range range("mmp.set_fields");
  CUDA_TRY(cudaSetDevice(b->device));
  Member& s = b->members[idx];
  const size_t bytes = (size_t)s.M * s.nt * sizeof(double2);
  CUDA_TRY(cudaMemcpyAsync(s.desc.io, phi0, bytes, cudaMemcpyHostToDevice, b->stream));
  {
    // the fields are checked on the device copy, before anything of the solve changes
    CUDA_TRY(cudaMemsetAsync(b->d_flag, 0, sizeof(int), b->stream));
    const double2* io = s.desc.io;
    size_t n = (size_t)s.M * s.nt;
    int* flag = b->d_flag;
    void* args[] = {(void*)&io, &n, &flag};
    CUDA_TRY(launch((const void*)&k_check_finite, dim3(1184, 1, 1), 256, 0, 1, b->stream, args));
    int bad = 0;
    CUDA_TRY(cudaMemcpyAsync(&bad, b->d_flag, sizeof(int), cudaMemcpyDeviceToHost, b->stream));
    CUDA_TRY(cudaStreamSynchronize(b->stream));
    if (bad) return fail(MMP_EINVAL, "initial fields not finite");
  }
  // psi_hat = FFT(cf * phi0)   (src/MultimodePropagation.cpp:59-63 in the frequency domain)
  DftArgs a;
  std::memset(&a, 0, sizeof(a));
  a.in = s.desc.io;
  a.out = s.desc.psi_hat;
  a.rows = (int)s.M;
  a.scale = s.cf;
  a.tw = b->dev->tw;
  void* args[] = {&a};
  CUDA_TRY(launch(b->ks64.dft_fwd, dim3((unsigned)(s.M * b->ks64.C), 1, 1), b->ks64.nthr, b->ks64.smem,
                  b->ks64.C, b->stream, args));
  if (!b->fp64) {  // psi_hat rounded to T
    const double2* src = s.desc.psi_hat;
    float2* dst = (float2*)s.desc.psi_t;
    size_t n = (size_t)s.M * s.nt;
    void* cargs[] = {(void*)&src, &dst, &n};
    CUDA_TRY(launch((const void*)&k_to_t2<float>, dim3(1184, 1, 1), 256, 0, 1, b->stream, cargs));
  }
  CUDA_TRY(cudaMemsetAsync(s.counters, 0, sizeof(unsigned long long), b->stream));  // z = 0
  CUDA_TRY(cudaMemsetAsync((char*)s.counters + 3 * sizeof(unsigned long long), 0, sizeof(int), b->stream));
  // the drift check's reference energy: the first step's energy from these fields on
  CUDA_TRY(cudaMemsetAsync((char*)s.counters + 4 * sizeof(unsigned long long), 0, sizeof(double), b->stream));
  s.step_host = 0;
  return MMP_OK;
}

// Batch-wide state every member shares: device resources, kernel sets, stream.
int batch_open(mmp_batch* b, const mmp_params* p0, const Tableau& tab0) {
  int dev = 0;
  CUDA_TRY(cudaGetDevice(&dev));
  DeviceRes* res = nullptr;
  int rc = ensure_device(dev, &res);
  if (rc) return rc;
  b->device = dev;
  b->dev = res;
  b->fp64 = (p0->flags & MMP_F_FP64) != 0;
  b->raman = p0->raman != 0;
  b->nt = p0->nt;
  b->logn = ilog2_exact(p0->nt);
  b->tab = tab0;
  b->ks = kernels_for(b->fp64 ? 1 : 0, b->logn);
  if (const char* env = std::getenv("MMP_ROW_SPLIT"))  // 1: rows split over twice the CTAs, where built
    if (std::atoi(env) == 1 && kernels_for(b->fp64 ? 1 : 0, b->logn, 1).prime)
      b->ks = kernels_for(b->fp64 ? 1 : 0, b->logn, 1);
  b->ks64 = kernels_for(1, b->logn);
  if (!b->ks.prime || !b->ks64.prime) return fail(MMP_ENOTSUP, "no kernels built for this nt");
  b->kernels_per_step = b->tab.s * ((b->raman ? 1 : 0) + 2);
  CUDA_TRY(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
  CUDA_TRY(dev_malloc((void**)&b->d_descs, (size_t)b->capacity * sizeof(SolveDesc) + 16));
  b->d_flag = reinterpret_cast<int*>(b->d_descs + b->capacity);
  return MMP_OK;
}

bool same_shape(const mmp_batch* b, const mmp_params* p) {
  Tableau t;
  tableau_for(p, t);
  return p->nt == b->nt && ((p->flags & MMP_F_FP64) != 0) == b->fp64 && (p->raman != 0) == b->raman &&
         std::memcmp(&t, &b->tab, sizeof(t)) == 0;
}

// Tensor-core form of the dense coefficients (SolveDesc::dense_tc): floats per solve, and
// the matrices themselves from the FP64 dense form A[p][q][0..31]. Per chunk of kTcChunk
// pair fields: four K-major matrices [Re hi, Re lo, Im hi, Im lo][kTcChunk/4][N = 16 M][4],
// row n = 16 p + k, each value split x = hi + lo with hi = x rounded to TF32 (nearest, ties
// away, as the device's cvt.rna) and lo = x - hi in FP32; rows k >= M and fields q >= P are 0.
size_t tc_floats(size_t M, size_t P) {
  const size_t nch = (P + kTcChunk - 1) / kTcChunk;
  return nch * 4 * kTcChunk * 16 * M;
}
float tf32_round(float x) {
  uint32_t u;
  std::memcpy(&u, &x, 4);
  u = (u + 0x1000u) & 0xFFFFE000u;
  std::memcpy(&x, &u, 4);
  return x;
}
std::vector<float> tc_operand(const std::vector<double>& A, int M, int P) {
  constexpr int K = kDenseMaxModes, KC = kTcChunk;
  const int N = 16 * M, nch = (P + KC - 1) / KC;
  std::vector<float> B(tc_floats(M, P), 0.0f);
  for (int c = 0; c < nch; ++c)
    for (int m = 0; m < 4; ++m)
      for (int jq = 0; jq < KC / 4; ++jq)
        for (int n = 0; n < N; ++n)
          for (int i = 0; i < 4; ++i) {
            const int q = c * KC + 4 * jq + i, p = n / 16, k = n % 16;
            if (q >= P || k >= M) continue;
            const double x = A[((size_t)p * P + q) * 2 * K + (m < 2 ? 0 : K) + k];
            const float hi = tf32_round((float)x);
            B[((((size_t)c * 4 + m) * (KC / 4) + jq) * N + n) * 4 + i] = (m & 1) ? (float)(x - (double)hi) : hi;
          }
  return B;
}

// Build the dense contraction form for this solve? Per sample, the register-blocked
// product spends about 36 instructions on every (p, pair field) couple (all kDenseMaxModes
// k at once), the term loop about 7 on every term, so the dense form pays from 5 M P
// terms on. MMP_DENSE=0 / 1 forces the choice (M <= 16 either way).
bool dense_wanted(const mmp_batch* b, const Member& s) {
  (void)b;
  if (s.M > (uint32_t)kDenseMaxModes || s.pairs.empty()) return false;
  if (const char* env = std::getenv("MMP_DENSE"))
    if (*env) return std::atoi(env) == 1;
  return s.terms.size() > 5 * (size_t)s.M * s.pairs.size();
}

// step, total, done counter | status, drift reference energy, spare
constexpr int kCounterWords = 6;

// Polls the contraction kernels give the first wait for their tile copy: far above any
// copy time. MMP_TILE_WAIT_POLLS (read when a solve is created) lowers it, for tests that
// make that bounded wait run out and check that the call reports MMP_ETIMEOUT.
unsigned tile_wait_polls() {
  if (const char* env = std::getenv("MMP_TILE_WAIT_POLLS"))
    if (*env) return (unsigned)std::strtoul(env, nullptr, 10);
  return kMaxWaitPolls;
}

size_t member_bytes(const mmp_batch* b, const Member& s) {
  const size_t t2 = b->fp64 ? sizeof(double2) : sizeof(float2);
  const size_t nt = b->nt, M = s.M, P = s.pairs.size(), S = (size_t)b->tab.s;
  size_t off = 0;
  off = align_up(off + M * nt * sizeof(double2));                               // psi_hat
  off = align_up(off + (b->fp64 ? 0 : M * nt * t2));                            // psi_hat in T
  off = align_up(off + M * nt * sizeof(double2));                               // io
  off = align_up(off + S * M * nt * t2);                                        // Nh
  off = align_up(off + M * nt * t2);                                            // U
  off = align_up(off + M * nt * t2);                                            // sigma
  off = align_up(off + (b->raman ? P : 0) * nt * t2);                           // W (R)
  off = align_up(off + (b->raman ? nt : 0) * std::max(t2, sizeof(double2)));    // H
  off = align_up(off + (b->raman ? P * (nt / 16) * 2 : 0) * t2);                // Raman tile carries
  off = align_up(off + (b->raman ? kRamanPow : 0) * t2);                         // powers of lambda
  off = align_up(off + (dense_wanted(b, s) ? M * P * 2 * kDenseMaxModes * (t2 / 2) : 0));  // dense form
  off = align_up(off + (dense_wanted(b, s) && !b->fp64 ? tc_floats(M, P) * sizeof(float) : 0));  // tensor-core form
  off = align_up(off + s.poly.size() * sizeof(double));
  off = align_up(off + std::max<size_t>(P, 1) * sizeof(int2));
  off = align_up(off + std::max<size_t>(s.terms.size(), 1) * sizeof(Term));
  off = align_up(off + (M + 1) * sizeof(int));
  off = align_up(off + std::max<size_t>(s.sr_kq.size(), 1) * 16);                // merged coefficients
  off = align_up(off + std::max<size_t>(s.sr_kq.size(), 1) * sizeof(unsigned));  // their k | q << 16
  off = align_up(off + s.sr_plan.size() * sizeof(int4));                         // group plan
  off = align_up(off + kCounterWords * sizeof(unsigned long long));
  return off;
}

// Does the sampled Raman response satisfy h_i = Im(c lambda^i) for every i < n (a damped
// sinusoid, |lambda| < 1)? Then its circular convolution is a periodic first-order
// recurrence (k_raman_scan). lambda is the complex root of z^2 = alpha z + beta, the
// recurrence h_i = alpha h_{i-1} + beta h_{i-2} read off h_0..h_3; c follows from h_0, h_1.
// Accepted when every sample matches the model to 1e-10 of max|h| (the sampled model
// itself, evaluated in FP64, matches to ~1e-12 at NT = 2^16).
bool fit_damped_sinusoid(const double* h, uint32_t n, std::complex<double>& lam, std::complex<double>& c) {
  if (n < 16) return false;
  double hmax = 0;
  for (uint32_t i = 0; i < n; ++i) {
    if (!std::isfinite(h[i])) return false;
    hmax = std::max(hmax, std::fabs(h[i]));
  }
  if (hmax == 0) return false;
  const double det = h[1] * h[1] - h[0] * h[2];
  if (std::fabs(det) < 1e-300) return false;
  const double alpha = (h[2] * h[1] - h[3] * h[0]) / det;
  const double beta = (h[1] * h[3] - h[2] * h[2]) / det;
  const double disc = alpha * alpha + 4 * beta;
  if (!(disc < 0)) return false;  // real roots: not an oscillating response
  lam = std::complex<double>(alpha / 2, std::sqrt(-disc) / 2);
  if (!(std::abs(lam) < 1)) return false;
  // Im(c) = h_0, Im(c lambda) = c.re lambda.im + c.im lambda.re = h_1
  c = std::complex<double>((h[1] - h[0] * lam.real()) / lam.imag(), h[0]);
  std::complex<double> m = c;
  const double tol = 1e-10 * hmax;
  for (uint32_t i = 0; i < n; ++i) {
    if (std::fabs(h[i] - m.imag()) > tol) return false;
    m *= lam;
  }
  return true;
}

// Host setup, device state and uploads for slot idx from params p; leaves the solve
// at z = 0 with its initial fields transformed. One cudaMalloc for all of it.
int member_init(mmp_batch* b, uint32_t idx, const mmp_params* p) {
  Member& s = b->members[idx];
  s = Member();
  host_setup(p, s);
  const size_t t2 = b->fp64 ? sizeof(double2) : sizeof(float2);
  const size_t nt = b->nt, M = s.M, P = s.pairs.size(), S = (size_t)b->tab.s;
  // one allocation: psi_hat | psi_hat in T | io | Nh | U | sigma | W | H | tiles | poly | pairs | terms |
  // term_off | counters
  size_t off = 0;
  const size_t o_psi = off; off = align_up(off + M * nt * sizeof(double2));
  const size_t o_pst = off; off = align_up(off + (b->fp64 ? 0 : M * nt * t2));
  const size_t o_io = off; off = align_up(off + M * nt * sizeof(double2));
  const size_t o_nh = off; off = align_up(off + S * M * nt * t2);
  const size_t o_u = off; off = align_up(off + M * nt * t2);
  const size_t o_sig = off; off = align_up(off + M * nt * t2);
  const size_t o_w = off; off = align_up(off + (b->raman ? P : 0) * nt * t2);
  const size_t o_h = off; off = align_up(off + (b->raman ? nt : 0) * std::max(t2, sizeof(double2)));
  const size_t o_rt = off; off = align_up(off + (b->raman ? P * (nt / 16) * 2 : 0) * t2);
  const size_t o_rp = off; off = align_up(off + (b->raman ? kRamanPow : 0) * t2);
  s.dense_ok = dense_wanted(b, s);
  const size_t o_dq = off; off = align_up(off + (s.dense_ok ? M * P * 2 * kDenseMaxModes * (t2 / 2) : 0));
  const bool tc_ok = s.dense_ok && !b->fp64;
  const size_t o_tc = off; off = align_up(off + (tc_ok ? tc_floats(M, P) * sizeof(float) : 0));
  const size_t o_poly = off; off = align_up(off + s.poly.size() * sizeof(double));
  const size_t o_pairs = off; off = align_up(off + std::max<size_t>(P, 1) * sizeof(int2));
  const size_t o_terms = off; off = align_up(off + std::max<size_t>(s.terms.size(), 1) * sizeof(Term));
  const size_t o_toff = off; off = align_up(off + (M + 1) * sizeof(int));
  const size_t nsr = s.sr_kq.size();
  const size_t o_src = off; off = align_up(off + std::max<size_t>(nsr, 1) * 16);
  const size_t o_skq = off; off = align_up(off + std::max<size_t>(nsr, 1) * sizeof(unsigned));
  const size_t o_splan = off; off = align_up(off + s.sr_plan.size() * sizeof(int4));
  const size_t o_cnt = off; off = align_up(off + kCounterWords * sizeof(unsigned long long));
  cudaError_t e = dev_malloc(&s.block, off, b->mempool, b->stream);
  if (e != cudaSuccess) {
    s.block = nullptr;
    return fail(MMP_ENOMEM, "allocating solver state: " + std::string(cudaGetErrorString(e)));
  }
  s.bytes = off;
  CUDA_TRY(cudaMemsetAsync(s.block, 0, off, b->stream));
  SolveDesc& d = s.desc;
  std::memset(&d, 0, sizeof(d));
  d.M = (int)M;
  d.P = (int)P;
  d.n_beta = (int)s.n_beta;
  d.raman = b->raman ? 1 : 0;
  d.alpha_scale = 2 * M_PI / s.t_final;
  d.dz = s.delta_z;
  d.sgn_gamma = s.sgn_gamma;
  d.one_minus_fR = b->raman ? (1.0 - s.fR) : 1.0;
  d.inv_nt = 1.0 / (double)nt;
  d.result_scale = 1.0 / ((double)nt * s.cf);
  d.energy_scale = s.delta_t * s.T0 / (s.cf * s.cf * (double)nt);
  d.omega0_T0 = s.omega0 * s.T0;
  d.photon_scale = d.energy_scale * s.T0 / 1.054571817e-10;
  d.poly = (const double*)T2ptr(s.block, o_poly);
  d.psi_hat = (double2*)T2ptr(s.block, o_psi);
  d.psi_t = b->fp64 ? (void*)d.psi_hat : T2ptr(s.block, o_pst);
  d.io = (double2*)T2ptr(s.block, o_io);
  d.Nh = T2ptr(s.block, o_nh);
  d.U = T2ptr(s.block, o_u);
  d.sigma = T2ptr(s.block, o_sig);
  d.W = T2ptr(s.block, o_w);
  d.H = b->raman ? T2ptr(s.block, o_h) : nullptr;
  d.raman_tiles = b->raman ? T2ptr(s.block, o_rt) : nullptr;
  d.raman_pow = b->raman ? T2ptr(s.block, o_rp) : nullptr;
  d.dense_q = s.dense_ok ? T2ptr(s.block, o_dq) : nullptr;
  d.dense_tc = tc_ok ? (const float*)T2ptr(s.block, o_tc) : nullptr;
  d.pairs = (const int2*)T2ptr(s.block, o_pairs);
  d.terms = (const Term*)T2ptr(s.block, o_terms);
  d.term_off = (const int*)T2ptr(s.block, o_toff);
  d.sr_coef = T2ptr(s.block, o_src);
  d.sr_kq = (const unsigned*)T2ptr(s.block, o_skq);
  d.sr_plan = (const int4*)T2ptr(s.block, o_splan);
  d.sr_terms = (int)nsr;
  d.sr_rounds = s.sr_rounds;
  s.counters = (unsigned long long*)T2ptr(s.block, o_cnt);
  d.step = s.counters;
  d.total = s.counters + 1;
  d.done_ctr = (unsigned int*)(s.counters + 2);
  d.status = (int*)(s.counters + 3);
  d.drift_ref = (double*)(s.counters + 4);
  d.drift_tol = 0.0;
  d.monitors = (s.flags & MMP_F_NO_MONITORS) ? 0 : 1;
  d.step_limit = ~0ull;
  d.tile_wait_polls = tile_wait_polls();
  if (b->raman) {
    std::complex<double> lam, c;
    if (fit_damped_sinusoid(p->raman_response, (uint32_t)nt, lam, c)) {
      // R = w sum_i h_i V[n - i], w = Delta_t T0 f_R (the scale the spectrum H carries)
      const std::complex<double> lamN = std::pow(lam, (double)nt);
      const std::complex<double> kap = (s.delta_t * s.T0 * s.fR) * c * (1.0 - lamN);
      const std::complex<double> inv = 1.0 / (1.0 - lamN);
      d.iir = 1;
      d.iir_lambda = make_double2(lam.real(), lam.imag());
      d.iir_kappa = make_double2(kap.real(), kap.imag());
      d.iir_inv_one_minus = make_double2(inv.real(), inv.imag());
      // lambda^j, j < kRamanPow, by binary powering in FP64 (the tile aggregates' weights)
      std::vector<double2> pw64(kRamanPow);
      std::vector<float2> pw32(kRamanPow);
      for (int j = 0; j < kRamanPow; ++j) {
        std::complex<double> r(1.0, 0.0), base = lam;
        for (int e = j; e; e >>= 1) {
          if (e & 1) r *= base;
          base *= base;
        }
        pw64[j] = make_double2(r.real(), r.imag());
        pw32[j] = make_float2((float)r.real(), (float)r.imag());
      }
      if (b->fp64)
        CUDA_TRY(cudaMemcpyAsync((void*)d.raman_pow, pw64.data(), kRamanPow * sizeof(double2), cudaMemcpyHostToDevice,
                                 b->stream));
      else
        CUDA_TRY(cudaMemcpyAsync((void*)d.raman_pow, pw32.data(), kRamanPow * sizeof(float2), cudaMemcpyHostToDevice,
                                 b->stream));
      CUDA_TRY(cudaStreamSynchronize(b->stream));  // the tables are host temporaries
    }
  }
  CUDA_TRY(cudaMemcpyAsync((void*)d.poly, s.poly.data(), s.poly.size() * sizeof(double), cudaMemcpyHostToDevice, b->stream));
  if (P) CUDA_TRY(cudaMemcpyAsync((void*)d.pairs, s.pairs.data(), P * sizeof(int2), cudaMemcpyHostToDevice, b->stream));
  if (!s.terms.empty())
    CUDA_TRY(cudaMemcpyAsync((void*)d.terms, s.terms.data(), s.terms.size() * sizeof(Term), cudaMemcpyHostToDevice, b->stream));
  CUDA_TRY(cudaMemcpyAsync((void*)d.term_off, s.term_off.data(), (M + 1) * sizeof(int), cudaMemcpyHostToDevice, b->stream));
  {
    // merged terms (k_contract_sr): records (a, b) in T
    std::vector<float> cf32;
    if (!b->fp64) cf32.assign(s.sr_ab.begin(), s.sr_ab.end());
    if (nsr) {
      CUDA_TRY(cudaMemcpyAsync((void*)d.sr_coef, b->fp64 ? (const void*)s.sr_ab.data() : (const void*)cf32.data(),
                               nsr * t2, cudaMemcpyHostToDevice, b->stream));
      CUDA_TRY(cudaMemcpyAsync((void*)d.sr_kq, s.sr_kq.data(), nsr * sizeof(unsigned), cudaMemcpyHostToDevice,
                               b->stream));
    }
    CUDA_TRY(cudaMemcpyAsync((void*)d.sr_plan, s.sr_plan.data(), s.sr_plan.size() * sizeof(int4),
                             cudaMemcpyHostToDevice, b->stream));
    CUDA_TRY(cudaStreamSynchronize(b->stream));  // the staging vectors are host temporaries
  }
  if (s.dense_ok) {
    // A[p][q][k] += Q, A[p][q][16 + k] += Q or -Q (terms that read conj of pair field q)
    constexpr int K = kDenseMaxModes;
    std::vector<double> A((size_t)M * P * 2 * K, 0.0);
    for (uint32_t p = 0; p < M; ++p)
      for (int j = s.term_off[p]; j < s.term_off[p + 1]; ++j) {
        const Term& t = s.terms[j];
        const size_t q = t.pc & 0x7fff;
        const double v = t.q;
        A[((size_t)p * P + q) * 2 * K + t.k] += v;
        A[((size_t)p * P + q) * 2 * K + K + t.k] += (t.pc & 0x8000) ? -v : v;
      }
    const size_t n = A.size();
    if (b->fp64) {
      CUDA_TRY(cudaMemcpyAsync((void*)d.dense_q, A.data(), n * sizeof(double), cudaMemcpyHostToDevice, b->stream));
      CUDA_TRY(cudaStreamSynchronize(b->stream));  // A is a host temporary
    } else {
      std::vector<float> Af(A.begin(), A.end());
      CUDA_TRY(cudaMemcpyAsync((void*)d.dense_q, Af.data(), n * sizeof(float), cudaMemcpyHostToDevice, b->stream));
      const std::vector<float> B = tc_operand(A, (int)M, (int)P);
      CUDA_TRY(cudaMemcpyAsync((void*)d.dense_tc, B.data(), B.size() * sizeof(float), cudaMemcpyHostToDevice,
                               b->stream));
      CUDA_TRY(cudaStreamSynchronize(b->stream));  // Af and B are host temporaries
    }
  }
  if (b->raman) {
    // Raman spectrum: H = FFT(h_R) * dt * T0 * fR / NT  (src/MultimodePropagation_CPU.cpp:170-176, :241-251)
    std::vector<double2> hr(nt);
    for (size_t t = 0; t < nt; ++t) hr[t] = make_double2(p->raman_response[t], 0.0);
    double2* tmp = d.io;                 // staging
    double2* h64 = (double2*)d.Nh;       // FP64 spectrum scratch (Nh is large enough and unused yet)
    CUDA_TRY(cudaMemcpyAsync(tmp, hr.data(), nt * sizeof(double2), cudaMemcpyHostToDevice, b->stream));
    CUDA_TRY(cudaStreamSynchronize(b->stream));  // hr is a host temporary
    DftArgs a;
    std::memset(&a, 0, sizeof(a));
    a.in = tmp;
    a.out = h64;
    a.rows = 1;
    a.scale = s.delta_t * s.T0 * s.fR / (double)nt;
    a.tw = b->dev->tw;
    void* args[] = {&a};
    CUDA_TRY(launch(b->ks64.dft_fwd, dim3((unsigned)b->ks64.C, 1, 1), b->ks64.nthr, b->ks64.smem, b->ks64.C, b->stream, args));
    const void* conv = b->fp64 ? (const void*)&k_to_t2<double> : (const void*)&k_to_t2<float>;
    const double2* cin = h64;
    void* cout_ = (void*)d.H;
    size_t cnt = nt;
    void* cargs[] = {(void*)&cin, &cout_, &cnt};
    CUDA_TRY(launch(conv, dim3(64, 1, 1), 256, 0, 1, b->stream, cargs));
    CUDA_TRY(cudaMemsetAsync(d.Nh, 0, S * M * nt * t2, b->stream));
  }
  b->active[idx] = 1;
  int rc = upload_desc(b);
  if (rc) return rc;
  return member_set_fields(b, idx, p->initial_fields);
}

// Launch geometry that depends on the members: largest M and P, contraction tile and
// its shared memory. Returns true when it changed (captured graphs are then stale).
// What a batch's launch shape depends on: maxima (and minima) over its solves.
struct ShapeStats {
  int Mmax = 0, Mmin = 1 << 30, Pmax = 0, Pall = 0;
  size_t max_terms = 0, max_sr_terms = 0;
  bool iir = true, all_dense = true, any_dense = false;
  uint32_t span = 0;
};

// One solve's part in them: what its host setup gives (see solve_counts).
struct SolveCounts {
  int M = 0;
  size_t pairs = 0, terms = 0, sr_terms = 0;
  bool iir = false, dense_ok = false;
};

void add_stats(ShapeStats& st, const mmp_batch* b, const SolveCounts& c, uint32_t span) {
  st.iir = st.iir && c.iir;
  st.all_dense = st.all_dense && c.dense_ok;
  st.any_dense = st.any_dense || c.dense_ok;
  st.span = std::max(st.span, span);
  st.Mmax = std::max(st.Mmax, c.M);
  st.Mmin = std::min(st.Mmin, c.M);
  st.Pmax = std::max(st.Pmax, (int)(b->raman ? c.pairs : 0));
  st.Pall = std::max(st.Pall, (int)c.pairs);
  st.max_terms = std::max(st.max_terms, c.terms);
  st.max_sr_terms = std::max(st.max_sr_terms, c.sr_terms);
}

SolveCounts member_counts(const Member& s) {
  SolveCounts c;
  c.M = (int)s.M;
  c.pairs = s.pairs.size();
  c.terms = s.terms.size();
  c.sr_terms = s.sr_kq.size();
  c.iir = s.desc.iir != 0;
  c.dense_ok = s.dense_ok;
  return c;
}

ShapeStats batch_stats(const mmp_batch* b) {
  ShapeStats st;
  for (size_t i = 0; i < b->members.size(); ++i)
    if (b->active[i]) add_stats(st, b, member_counts(b->members[i]), (uint32_t)i + 1);
  return st;
}

// A batch's launch shape: the contraction form and tile, the Raman route and the shared
// memory they take, chosen from its statistics alone.
struct Shape {
  int Mmax = 0, Pmax = 0, TT = 32, dense = 0, pchunk = 0, stage_terms = 0;
  bool tc = false, sr = false, fused = false, iir = false;
  size_t smem = 0;
  uint32_t span = 0;
};

// Shapes that run the same kernels with the same tiles on a solve (so give it the same bits).
bool same_kernels(const Shape& x, const Shape& y) {
  return x.TT == y.TT && x.dense == y.dense && x.pchunk == y.pchunk && x.stage_terms == y.stage_terms &&
         x.tc == y.tc && x.sr == y.sr && x.fused == y.fused && x.iir == y.iir;
}

Shape choose_shape(const mmp_batch* b, const ShapeStats& st) {
  const size_t t2 = b->fp64 ? sizeof(double2) : sizeof(float2);
  const int Mmax = st.Mmax, Pmax = st.Pmax, Pall = st.Pall, Mmin = st.Mmin;
  const uint32_t span = st.span;
  const size_t max_terms = st.max_terms, max_sr_terms = st.max_sr_terms;
  bool iir = b->raman && st.iir;
  const bool all_dense = st.all_dense, any_dense = st.any_dense;
  // contraction tile: the largest power of two <= 256 whose U + pair-field tile fits in
  // 100 KB (the pair fields are formed in the tile with Raman on and off)
  const int rows = std::max(Mmax + Pall, 1);
  int TT = 256;
  while (TT > 32 && (size_t)rows * TT * t2 > 100 * 1024) TT >>= 1;
  while (TT > 2 && (size_t)rows * TT * t2 > 200 * 1024) TT >>= 1;  // >= 2: 16-byte bulk copies
  while (TT > (int)b->nt) TT >>= 1;
  int tile_req = b->tile_req;  // the autotuner's tile, else MMP_CONTRACT_TILE
  if (!tile_req)
    if (const char* env = std::getenv("MMP_CONTRACT_TILE")) tile_req = std::atoi(env);
  if (tile_req >= 64 && tile_req < TT) TT = tile_req;
  size_t smem = (size_t)rows * TT * t2;
  if (const char* env = std::getenv("MMP_RAMAN_FFT"))  // 1 forces the FFT convolution
    if (std::atoi(env) == 1) iir = false;
  // the recurrence runs inside the contraction tiles when a lane gets 2..8 samples
  // (64 <= TT <= 256); MMP_RAMAN_FUSED=0 keeps the row scan
  bool fused = iir && TT >= 64 && (int)b->nt >= TT;
  if (const char* env = std::getenv("MMP_RAMAN_FUSED"))
    if (std::atoi(env) == 0) fused = false;
  if (fused) smem += 2 * (size_t)Pmax * t2;  // the tile's carries (k_contract, raman_mode 2)
  int dense = (span == 0 || TT < 64 || !any_dense) ? 0 : (all_dense ? 1 : 2);
  // FP32 batches whose every solve has the dense form with at least kTcMinModes modes run
  // it on the tensor cores (k_contract_tc, tiles of kTcTile samples) when the pair fields
  // come from inside the tile or from U alone (Raman off); MMP_TC=0 keeps the
  // register-blocked form. A batch that mixes in any other solve keeps the latter for all.
  bool tc = !b->fp64 && span > 0 && all_dense && Mmin >= kTcMinModes && (int)b->nt >= kTcTile &&
            (!b->raman || iir);
  if (const char* env = std::getenv("MMP_TC"))
    if (std::atoi(env) == 0) tc = false;
  if (const char* env = std::getenv("MMP_RAMAN_FUSED"))  // the kernel forms the Raman fields itself
    if (std::atoi(env) == 0 && b->raman) tc = false;
  if (tc) {
    TT = kTcTile;
    fused = b->raman;
    dense = 1;
    smem = ((size_t)Mmax * TT + (b->raman ? 2 * (size_t)Pmax : 0)) * sizeof(float2) +
           2 * 4 * (size_t)kTcChunk * (TT + 16 * (size_t)Mmax) * sizeof(float) +  // two operand buffers
           1024;                                                                  // their alignment
  } else if (dense) {
    smem += 8 * 2 * (size_t)kDenseChunk * 2 * kDenseMaxModes * (t2 / 2);  // staged coefficient rows
  }
  // terms follow the tiles in shared memory, coefficient in T, when they fit (else they
  // are read through L1 from the FP64 table); the dense form reads no terms
  const size_t staged = b->fp64 ? sizeof(StagedTerm<double>) : sizeof(StagedTerm<float>);
  // Tall tiles (the U tile and every pair field do not fit at 64 samples or more): the
  // pair-chunked contraction keeps the recurrence in the tiles with only a chunk of pair
  // fields in shared memory (3 CTAs per SM in FP32, 2 in FP64), instead of the row scan
  // writing P Raman rows to HBM for the contraction to read back. MMP_PAIR_CHUNK=0 keeps
  // the row scan.
  int pchunk = 0;
  bool pc_ok = iir && !fused && !any_dense && span > 0;
  if (const char* env = std::getenv("MMP_RAMAN_FUSED"))
    if (std::atoi(env) == 0) pc_ok = false;
  if (const char* env = std::getenv("MMP_PAIR_CHUNK"))
    if (std::atoi(env) == 0) pc_ok = false;
  if (pc_ok) {
    int tc_tt = 256;  // items per thread: M TT / 2 <= kPcItems * 256
    while (tc_tt > 64 && (size_t)Mmax * tc_tt > 2 * kPcItems * 256) tc_tt >>= 1;
    while (tc_tt > (int)b->nt) tc_tt >>= 1;
    const size_t budget = b->fp64 ? 110 * 1024 : 72 * 1024;
    const size_t fixed = (size_t)Mmax * tc_tt * t2 + max_terms * staged + 2 * (size_t)Pmax * t2;
    if (tc_tt >= 64 && (size_t)Mmax * tc_tt <= 2 * kPcItems * 256 && fixed + 8 * (size_t)tc_tt * t2 <= budget) {
      pchunk = (int)std::min<size_t>((size_t)std::max(Pmax, 1), (budget - fixed) / ((size_t)tc_tt * t2));
      TT = tc_tt;
      fused = true;
      smem = fixed + (size_t)pchunk * tc_tt * t2;
    }
  }
  // Tall tiles with every pair field formed in the contraction (Raman off, or the
  // recurrence fused): the serial-recurrence contraction in sub-blocks of kSrSub samples
  // (k_contract_sr, tiles of up to 256 samples) when its shared memory fits, in place of the
  // pair-chunked one. MMP_CONTRACT_SR=0 keeps the latter.
  bool sr = false;
  {
    const bool tall = (size_t)rows * 64 * t2 > 100 * 1024;
    bool ok = tall && span > 0 && !any_dense && Mmax <= kSrMaxModes &&
              Pall <= kSrPairsPerThread * kSrThreads && (!b->raman || iir) && (int)b->nt >= kSrSub * 4;
    if (const char* env = std::getenv("MMP_CONTRACT_SR"))
      if (std::atoi(env) == 0) ok = false;
    if (const char* env = std::getenv("MMP_RAMAN_FUSED"))
      if (std::atoi(env) == 0 && b->raman) ok = false;
    const size_t sp = 2 * t2;  // one sample pair of one row
    const size_t rs = kSrSub / 2 + 1;
    const size_t plan = (size_t)((Mmax + kSrGroups - 1) / kSrGroups) * kSrGroups * sizeof(int4);
    const size_t need = (2 * (size_t)Mmax + (size_t)Pall) * rs * sp + plan + max_sr_terms * 2 * t2;  // SrRec
    if (ok && need <= 227 * 1024) {
      sr = true;
      pchunk = 0;
      TT = std::min(tile_req >= 64 ? std::min(tile_req, 256) : 256, (int)b->nt);
      fused = b->raman;
      smem = (need + 15) & ~(size_t)15;
    }
  }
  const int stage_terms = sr ? 0 : (pchunk ? 1 : (dense != 1 && !tc && smem + max_terms * staged <= 200 * 1024 ? 1 : 0));
  if (stage_terms && !pchunk) smem += max_terms * staged;
  Shape sh;
  sh.Mmax = Mmax;
  sh.Pmax = Pmax;
  sh.TT = TT;
  sh.dense = dense;
  sh.pchunk = pchunk;
  sh.stage_terms = stage_terms;
  sh.tc = tc;
  sh.sr = sr;
  sh.fused = fused;
  sh.iir = iir;
  sh.smem = smem;
  sh.span = span;
  return sh;
}

// Would the solve with counts `c` run in batch `b` (a served pool) on exactly the kernels and tiles it
// runs alone? True when a batch of it alone, `b` with it added and `b` as it is all have
// the same shape (an empty `b`: the first two). The shape depends on maxima over the
// solves (the tile shrinks as rows grow, tall tiles take the serial-recurrence form, dense Q
// the dense form), so a solve joins only pools whose maxima lead to its own choices, and
// since every solve in a pool then has the pool's shape alone, one leaving does not change
// it either.
// A solve's counts from its parameters alone (the host setup a member gets at creation).
SolveCounts solve_counts(const mmp_params* p) {
  Member m;
  host_setup(p, m);
  SolveCounts c = member_counts(m);
  c.iir = false;
  if (p->raman && p->raman_response) {
    std::complex<double> lam, cc;
    c.iir = fit_damped_sinusoid(p->raman_response, p->nt, lam, cc);
  }
  c.dense_ok = dense_wanted(nullptr, m);
  return c;
}

bool joins_same_kernels(const mmp_batch* b, const SolveCounts& c) {
  ShapeStats alone;
  add_stats(alone, b, c, 1);
  ShapeStats with = batch_stats(b);
  const bool empty = with.span == 0;
  add_stats(with, b, c, 1);
  const Shape w = choose_shape(b, with);
  if (!same_kernels(choose_shape(b, alone), w)) return false;
  return empty || same_kernels(choose_shape(b, batch_stats(b)), w);
}

bool batch_shape(mmp_batch* b) {
  const Shape sh = choose_shape(b, batch_stats(b));
  const bool changed = sh.Mmax != b->Mmax || sh.Pmax != b->Pmax || sh.TT != b->TT || sh.smem != b->contract_smem ||
                       sh.stage_terms != b->stage_terms || sh.span != b->span || sh.iir != b->raman_iir ||
                       sh.fused != b->raman_fused || sh.dense != b->dense || sh.tc != b->tc ||
                       sh.pchunk != b->pchunk || sh.sr != b->sr;
  b->dense = sh.dense;
  b->tc = sh.tc;
  b->pchunk = sh.pchunk;
  b->sr = sh.sr;
  b->raman_iir = sh.iir;
  b->raman_fused = sh.fused;
  b->kernels_per_step = b->tab.s * ((b->raman ? (sh.fused ? 2 : 1) : 0) + 2);
  b->span = sh.span;
  b->Mmax = sh.Mmax;
  b->Pmax = sh.Pmax;
  b->TT = sh.TT;
  b->contract_smem = sh.smem;
  b->stage_terms = sh.stage_terms;
  if (changed && b->graph) {
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
    b->graph_steps = 0;
  }
  return changed;
}

// ---- autotuner -------------------------------------------------------------------------
// Three launch parameters are chosen by timing whole RK steps of this batch on its own
// buffers, one parameter after the other (each timed with the others at their current
// choice):
//   1. the per-mode transform kernels: each row on the minimal set of CTAs, or split over
//      twice as many (a cluster twice as wide: one more radix-2 exchange across CTAs and
//      half the shared memory per CTA, so two CTAs share an SM), where that set is built;
//   2. the contraction tile: samples per CTA of k_contract (64 / 128 / 256, as many as fit
//      its shared memory) or of k_contract_sr (64 / 128 / 256);
//   3. the graph branches: the batch's solves split into 1, 2 or 4 independent kernel
//      chains per captured step.
// The timed steps advance the solves; afterwards every member gets its initial fields
// back at z = 0 with its counters cleared, as if nothing had run. The choice is cached
// per shape (device, precision, NT, tableau size, largest M and P, batch size, Raman,
// contraction form, candidate lists). Batches of one solve are not tuned: they keep the
// default parameters, the ones the serving loop's pools use, so that a served solve and
// the same solve run alone give the same bits. MMP_ROW_SPLIT, MMP_CONTRACT_TILE and
// MMP_GROUPS each fix one parameter instead.
struct TuneChoice {
  int xc = 0, tile = 0, groups = 1;
};
std::mutex g_tune_mu;
std::map<std::vector<int>, TuneChoice> g_tune_cache;

// Device time per RK step of `reps` steps after one warm-up step.
int time_steps(mmp_batch* b, int reps, float* ms) {
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  CUDA_TRY(cudaEventCreate(&e0));
  cudaError_t e = cudaEventCreate(&e1);
  int rc = e == cudaSuccess ? capture_steps(b, 1) : fail(MMP_ECUDA, cudaGetErrorString(e));
  if (rc == MMP_OK) {
    cudaEventRecord(e0, b->stream);
    rc = capture_steps(b, reps);
    cudaEventRecord(e1, b->stream);
  }
  float f = 0.f;
  if (rc == MMP_OK) {
    e = cudaEventSynchronize(e1);
    if (e == cudaSuccess) e = cudaEventElapsedTime(&f, e0, e1);
    if (e != cudaSuccess) rc = fail(MMP_ECUDA, cudaGetErrorString(e));
  } else {
    cudaStreamSynchronize(b->stream);
  }
  cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  *ms = f / (float)reps;
  return rc;
}

// Contraction tiles worth timing for the form batch_shape chose (first: its own choice).
std::vector<int> tile_candidates(const mmp_batch* b) {
  std::vector<int> t = {b->TT};
  if (b->tc || b->pchunk) return t;  // fixed tiles
  if (b->sr || b->TT >= 64)
    for (int c = 256; c >= 64; c >>= 1)
      if (c != b->TT && c <= (b->sr ? 256 : b->TT) && c <= (int)b->nt) t.push_back(c);
  return t;
}

int restore_members(mmp_batch* b, const mmp_params* const* params) {
  for (uint32_t i = 0; i < b->members.size(); ++i) {
    if (!b->active[i]) continue;
    int rc = member_set_fields(b, i, params[i]->initial_fields);
    if (rc) return rc;
    CUDA_TRY(cudaMemsetAsync(b->members[i].counters, 0, kCounterWords * sizeof(unsigned long long), b->stream));
  }
  CUDA_TRY(cudaStreamSynchronize(b->stream));
  return MMP_OK;
}

int autotune(mmp_batch* b, const mmp_params* const* params) {
  mmp_detail::Range range("mmp.autotune");
  const KernelSet base = kernels_for(b->fp64 ? 1 : 0, b->logn, 0);
  const KernelSet alt = kernels_for(b->fp64 ? 1 : 0, b->logn, 1);
  std::vector<int> xcs = {0}, tiles = tile_candidates(b), gs = {1};
  if (alt.prime) xcs.push_back(1);
  const int g0 = b->span >= 16 ? 4 : (b->span >= 4 ? 2 : 1);  // the untuned default
  gs = {g0};
  for (int g : {1, 2, 4})
    if (g != g0 && (uint32_t)g <= b->span) gs.push_back(g);
  if (const char* env = std::getenv("MMP_ROW_SPLIT"))
    if (*env) xcs = {std::atoi(env) == 1 && alt.prime ? 1 : 0};
  if (const char* env = std::getenv("MMP_CONTRACT_TILE"))
    if (*env) tiles = {std::atoi(env)};
  if (const char* env = std::getenv("MMP_GROUPS"))
    if (*env) gs = {std::max(1, std::atoi(env))};
  auto apply = [&](const TuneChoice& c) {
    b->ks = c.xc ? alt : base;
    b->tile_req = c.tile;
    batch_shape(b);
    b->groups = (uint32_t)c.groups;
  };
  TuneChoice c;
  c.xc = xcs[0];
  c.tile = tiles[0];
  c.groups = gs[0];
  b->tuned = 0;
  if (b->span < 2 || (xcs.size() == 1 && tiles.size() == 1 && gs.size() == 1)) {
    apply(c);
    return MMP_OK;
  }
  std::vector<int> key = {b->device, b->fp64 ? 1 : 0, b->logn, b->tab.s, b->Mmax, b->Pmax,
                          (int)b->span, b->raman ? 1 : 0, b->tc ? 1 : 0, b->sr ? 1 : 0,
                          b->pchunk ? 1 : 0, b->dense, -1};
  for (const std::vector<int>* v : {&xcs, &tiles, &gs}) {
    key.insert(key.end(), v->begin(), v->end());
    key.push_back(-1);
  }
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) {
      apply(it->second);
      b->tuned = 1;
      return MMP_OK;
    }
  }
  const uint64_t counted = g_launches.load();
  int rc = MMP_OK;
  auto sweep = [&](int TuneChoice::*field, const std::vector<int>& vals) {
    if (vals.size() < 2 || rc) return;
    float best = 0.f;
    int pick = c.*field;
    for (size_t i = 0; i < vals.size() && rc == MMP_OK; ++i) {
      TuneChoice t = c;
      t.*field = vals[i];
      apply(t);
      float ms = 0.f;
      rc = time_steps(b, 3, &ms);
      if (rc == MMP_OK && (i == 0 || ms < best)) {
        best = ms;
        pick = vals[i];
      }
    }
    c.*field = pick;
  };
  apply(c);
  sweep(&TuneChoice::xc, xcs);
  sweep(&TuneChoice::tile, tiles);
  sweep(&TuneChoice::groups, gs);
  g_launches.store(counted);  // tuning launches are not solver work
  if (rc) return rc;
  apply(c);
  rc = restore_members(b, params);
  if (rc) return rc;
  b->tuned = 1;
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune_cache[key] = c;
  return MMP_OK;
}

int create_batch(const mmp_params* const* params, uint32_t n, mmp_batch** out) {
  if (!out) return fail(MMP_EINVAL, "out is NULL");
  *out = nullptr;
  if (!params || n == 0) return fail(MMP_EINVAL, "empty batch");
  mmp_detail::Range range("mmp.create");
  for (uint32_t i = 0; i < n; ++i) {
    std::string why;
    int rc = validate(params[i], why);
    if (rc) return fail(rc, "member " + std::to_string(i) + ": " + why);
  }
  Tableau tab0;
  tableau_for(params[0], tab0);
  mmp_batch* b = new mmp_batch();
  b->capacity = n;
  b->members.resize(n);
  b->active.assign(n, 0);
  int rc = batch_open(b, params[0], tab0);
  for (uint32_t i = 1; i < n && rc == MMP_OK; ++i)
    if (!same_shape(b, params[i]))
      rc = fail(MMP_EINVAL, "batch members must share nt, precision, raman and the RK tableau");
  for (uint32_t i = 0; i < n && rc == MMP_OK; ++i) rc = member_init(b, i, params[i]);
  if (rc == MMP_OK) {
    batch_shape(b);
    rc = autotune(b, params);
  }
  if (rc == MMP_OK) {
    cudaError_t e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess) rc = fail(MMP_ECUDA, cudaGetErrorString(e));
  }
  if (rc != MMP_OK) {
    mmp_batch_destroy(b);
    return rc;
  }
  *out = b;
  return MMP_OK;
}

void fill_info(mmp_batch* b, const Member& s, mmp_info* info) {
  std::memset(info, 0, sizeof(*info));
  info->n_modes = s.M;
  info->nt = s.nt;
  info->n_stages = (uint32_t)b->tab.s;
  info->n_pairs = (uint32_t)s.unique_pairs.size();
  info->n_pair_fields = (uint32_t)s.pairs.size();
  info->pair_quirk_active = s.quirk ? 1u : 0u;
  info->t_final = s.t_final;
  info->delta_t = s.delta_t;
  info->z_final = s.z_final;
  info->delta_z = s.delta_z;
  info->z = (double)s.step_host * s.delta_z;
  info->LD = s.LD;
  info->conversion_factor = s.cf;
  info->max_beta2 = s.max_beta2;
  info->max_Q = s.max_Q;
  info->steps_done = s.total_host;
  info->fp64 = b->fp64 ? 1u : 0u;
  info->cluster_ctas = (uint32_t)b->ks.C;
  info->raman_recurrence = b->raman_fused ? 2u : (b->raman_iir ? 1u : 0u);
  info->graph_branches = b->groups;
  info->dense_contraction = (b->dense == 1 || (b->dense == 2 && s.dense_ok)) ? 1u : 0u;
  info->tensor_core_contraction = b->tc ? 1u : 0u;
  info->contract_pair_chunk = (uint32_t)b->pchunk;
  info->contract_sub_block = b->sr ? (uint32_t)kSrSub : 0u;
  info->contract_tile = (uint32_t)b->TT;
  info->autotuned = (uint32_t)b->tuned;
}

}  // namespace

// ---------------------------------------------------------------------------------------
// C ABI
extern "C" {

int mmp_validate_params(const mmp_params* params, char* msg, size_t msg_len) {
  std::string why;
  int rc = validate(params, why);
  if (msg && msg_len) {
    std::snprintf(msg, msg_len, "%s", rc ? why.c_str() : "");
  }
  if (rc) fail(rc, why);
  return rc;
}

int mmp_batch_create(const mmp_params* const* params, uint32_t n, mmp_batch** out) {
  return create_batch(params, n, out);
}

int mmp_batch_propagate_async(mmp_batch* b, uint32_t nz) { return batch_propagate_async(b, nz); }

int mmp_batch_synchronize(mmp_batch* b) {
  if (!b) return fail(MMP_EINVAL, "NULL batch");
  return batch_sync(b);
}

int mmp_batch_propagate(mmp_batch* b, uint32_t nz) {
  int rc = batch_propagate_async(b, nz);
  if (rc) return rc;
  return batch_sync(b);
}

int mmp_batch_get_result(mmp_batch* b, uint32_t index, double* out) { return member_result(b, index, out); }

int mmp_batch_set_fields(mmp_batch* b, uint32_t index, const double* phi0) {
  int rc = member_set_fields(b, index, phi0);
  if (rc) return rc;
  return MMP_OK;
}

int mmp_batch_get_info(mmp_batch* b, uint32_t index, mmp_info* info) {
  if (!b || index >= b->members.size() || !info) return fail(MMP_EINVAL, "bad info arguments");
  fill_info(b, b->members[index], info);
  return MMP_OK;
}

uint32_t mmp_batch_size(const mmp_batch* b) { return b ? (uint32_t)b->members.size() : 0u; }

int mmp_batch_set_energy_drift_limit(mmp_batch* b, uint32_t index, double rel_tol) {
  if (!b || index >= b->members.size() || !b->active[index]) return fail(MMP_EINVAL, "bad drift-limit arguments");
  if (!(rel_tol >= 0.0) || !std::isfinite(rel_tol)) return fail(MMP_EINVAL, "drift limit must be finite and >= 0");
  Member& s = b->members[index];
  if (rel_tol > 0.0 && (s.flags & MMP_F_NO_MONITORS))
    return fail(MMP_ESTATE, "the drift check reads the energy monitor, which MMP_F_NO_MONITORS turns off");
  CUDA_TRY(cudaSetDevice(b->device));
  CUDA_TRY(cudaStreamSynchronize(b->stream));  // no launch in flight reads the old descriptor
  s.desc.drift_tol = rel_tol;
  return upload_desc(b);
}

int mmp_batch_propagate_timed(mmp_batch* b, uint32_t nz, uint32_t repeats, double* ms) {
  if (!b || !ms) return fail(MMP_EINVAL, "bad timed-propagate arguments");
  CUDA_TRY(cudaSetDevice(b->device));
  cudaEvent_t e0, e1;
  CUDA_TRY(cudaEventCreate(&e0));
  CUDA_TRY(cudaEventCreate(&e1));
  int rc = MMP_OK;
  cudaError_t e = cudaEventRecord(e0, b->stream);
  for (uint32_t r = 0; r < repeats && rc == MMP_OK && e == cudaSuccess; ++r) rc = batch_propagate_async(b, nz);
  if (e == cudaSuccess) e = cudaEventRecord(e1, b->stream);
  if (e == cudaSuccess) e = cudaEventSynchronize(e1);
  float f = 0.f;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&f, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc;
  if (e != cudaSuccess) return fail(MMP_ECUDA, cudaGetErrorString(e));
  *ms = f;
  return check_status(b);
}

int mmp_batch_profile(mmp_batch* b, uint32_t nz, double* ms_per_launch, uint32_t* launches) {
  if (!b || !ms_per_launch || !launches) return fail(MMP_EINVAL, "bad profile arguments");
  mmp_detail::Range range("mmp.profile");
  CUDA_TRY(cudaSetDevice(b->device));
  for (int k = 0; k < 3; ++k) { ms_per_launch[k] = 0.0; launches[k] = 0; }
  for (auto& s : b->members) {
    if (!(s.flags & MMP_F_CONTINUOUS)) {
      CUDA_TRY(cudaMemsetAsync(s.counters, 0, sizeof(unsigned long long), b->stream));
      s.step_host = 0;
    }
    if (!(s.flags & MMP_F_NO_MONITORS)) {
      int rc = grow_monitors(b, s, s.total_host + nz);
      if (rc) return rc;
    }
  }
  const int nsol = (int)b->span;
  int rc = launch_row_kernel(b, b->ks, b->ks.prime, b->Mmax, nsol, 0, b->d_descs);
  if (rc) return rc;
  cudaEvent_t ev[2];
  CUDA_TRY(cudaEventCreate(&ev[0]));
  CUDA_TRY(cudaEventCreate(&ev[1]));
  double acc[3] = {0, 0, 0};
  for (uint32_t n = 0; n < nz && rc == MMP_OK; ++n) {
    for (int i = 0; i < b->tab.s && rc == MMP_OK; ++i) {
      for (int kind = 0; kind < 3 && rc == MMP_OK; ++kind) {
        if (kind == 0 && !(b->raman && b->Pmax > 0)) continue;
        cudaError_t e = cudaEventRecord(ev[0], b->stream);
        if (e != cudaSuccess) { rc = fail(MMP_ECUDA, cudaGetErrorString(e)); break; }
        if (kind == 0) rc = launch_pairs(b, b->ks, nsol, i, b->d_descs);
        else if (kind == 1) rc = launch_contract(b);
        else rc = launch_row_kernel(b, b->ks, nu_kernel(b->ks, b->tab, i), b->Mmax, nsol, i, b->d_descs);
        if (rc) break;
        e = cudaEventRecord(ev[1], b->stream);
        if (e == cudaSuccess) e = cudaEventSynchronize(ev[1]);
        float f = 0.f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&f, ev[0], ev[1]);
        if (e != cudaSuccess) { rc = fail(MMP_ECUDA, cudaGetErrorString(e)); break; }
        acc[kind] += f;
        launches[kind] += 1;
      }
    }
  }
  cudaEventDestroy(ev[0]);
  cudaEventDestroy(ev[1]);
  if (rc) return rc;
  for (auto& s : b->members) {
    s.total_host += nz;
    s.step_host += nz;
  }
  for (int k = 0; k < 3; ++k) ms_per_launch[k] = launches[k] ? acc[k] / launches[k] : 0.0;
  return batch_sync(b);
}

void mmp_batch_destroy(mmp_batch* b) {
  if (!b) return;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  if (b->graph) cudaGraphExecDestroy(b->graph);
  for (auto& s : b->members) {
    dev_free(s.block, b->stream, b->mempool != nullptr);
    dev_free(s.energy);
  }
  if (b->mempool && b->stream) cudaStreamSynchronize(b->stream);
  for (cudaStream_t s : b->branch) cudaStreamDestroy(s);
  for (cudaEvent_t e : b->branch_ev) cudaEventDestroy(e);
  if (b->fork_ev) cudaEventDestroy(b->fork_ev);
  dev_free(b->d_descs);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
}

int mmp_solver_create(const mmp_params* params, mmp_solver** out) {
  if (!out) return fail(MMP_EINVAL, "out is NULL");
  *out = nullptr;
  const mmp_params* arr[1] = {params};
  mmp_batch* b = nullptr;
  int rc = create_batch(arr, 1, &b);
  if (rc) return rc;
  mmp_solver* s = new mmp_solver();
  s->b = b;
  *out = s;
  return MMP_OK;
}

int mmp_propagate(mmp_solver* s, uint32_t nz) {
  if (!s) return fail(MMP_EINVAL, "NULL solver");
  return mmp_batch_propagate(s->b, nz);
}

int mmp_propagate_async(mmp_solver* s, uint32_t nz) {
  if (!s) return fail(MMP_EINVAL, "NULL solver");
  return batch_propagate_async(s->b, nz);
}

int mmp_synchronize(mmp_solver* s) {
  if (!s) return fail(MMP_EINVAL, "NULL solver");
  return batch_sync(s->b);
}

int mmp_propagate_default(mmp_solver* s) {
  if (!s) return fail(MMP_EINVAL, "NULL solver");
  const Member& m = s->b->members[0];
  // src/MultimodePropagation.cpp:213-216
  const unsigned nz = (unsigned)std::floor(m.z_final / m.delta_z);
  return mmp_batch_propagate(s->b, nz);
}

int mmp_get_result(mmp_solver* s, double* out) {
  if (!s) return fail(MMP_EINVAL, "NULL solver");
  return member_result(s->b, 0, out);
}

int mmp_propagate_snapshots(mmp_solver* sol, uint32_t n_save, int z_mode, double* fields, double* Z,
                            double* elapsed_s) {
  if (!sol) return fail(MMP_EINVAL, "NULL solver");
  if (n_save == 0) return fail(MMP_EINVAL, "n_save must be >= 1");
  mmp_detail::Range range("mmp.snapshots");
  if (z_mode != 0 && z_mode != 1) return fail(MMP_EINVAL, "z_mode must be 0 (continuous) or 1 (reference)");
  const auto t0 = std::chrono::steady_clock::now();
  mmp_batch* b = sol->b;
  Member& s = b->members[0];
  // matlab/mm_propagation.cpp:61-91: n_save - 1 chunks of n_steps / n_save steps, then
  // one of n_steps / n_save + n_steps % n_save; Z += nz * fiber_length / n_steps
  const uint32_t nz = s.n_steps / n_save;
  const double delta_Z = s.fiber_length / s.n_steps;
  const uint32_t flags0 = s.flags;
  const size_t row = (size_t)2 * s.M * s.nt;
  double z_acc = 0.0;
  for (uint32_t i = 0; i < n_save; ++i) {
    const uint32_t n = (i + 1 < n_save) ? nz : nz + s.n_steps % n_save;
    if (z_mode == 0 && i > 0) s.flags |= MMP_F_CONTINUOUS;  // later chunks carry z on
    int rc = batch_propagate_async(b, n);
    s.flags = flags0;
    if (rc == MMP_OK) rc = batch_sync(b);
    if (rc == MMP_OK && fields) rc = member_result(b, 0, fields + i * row);
    if (rc) return rc;
    z_acc += n * delta_Z;
    if (Z) Z[i] = z_acc;
    if (elapsed_s) elapsed_s[i] = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
  return MMP_OK;
}

int mmp_set_fields(mmp_solver* s, const double* phi0) {
  if (!s) return fail(MMP_EINVAL, "NULL solver");
  int rc = member_set_fields(s->b, 0, phi0);
  if (rc) return rc;
  CUDA_TRY(cudaStreamSynchronize(s->b->stream));
  return MMP_OK;
}

int mmp_get_monitors(mmp_solver* s, double* energy, double* photons, uint64_t max_steps, uint64_t* n_written) {
  if (!s) return fail(MMP_EINVAL, "NULL solver");
  mmp_batch* b = s->b;
  Member& m = b->members[0];
  CUDA_TRY(cudaSetDevice(b->device));
  CUDA_TRY(cudaStreamSynchronize(b->stream));
  uint64_t n = std::min<uint64_t>(max_steps, std::min<uint64_t>(m.total_host, m.mon_cap));
  if (m.flags & MMP_F_NO_MONITORS) n = 0;
  if (n && energy) CUDA_TRY(cudaMemcpy(energy, m.energy, n * sizeof(double), cudaMemcpyDeviceToHost));
  if (n && photons) CUDA_TRY(cudaMemcpy(photons, m.photons, n * sizeof(double), cudaMemcpyDeviceToHost));
  if (n_written) *n_written = n;
  return MMP_OK;
}

int mmp_set_energy_drift_limit(mmp_solver* s, double rel_tol) {
  if (!s) return fail(MMP_EINVAL, "NULL solver");
  return mmp_batch_set_energy_drift_limit(s->b, 0, rel_tol);
}

int mmp_get_info(mmp_solver* s, mmp_info* info) {
  if (!s || !info) return fail(MMP_EINVAL, "bad info arguments");
  fill_info(s->b, s->b->members[0], info);
  return MMP_OK;
}

void mmp_solver_destroy(mmp_solver* s) {
  if (!s) return;
  mmp_batch_destroy(s->b);
  delete s;
}

int mmp_tableau(uint32_t method_order, int32_t rk_variant, double rk_lambda, double rk_mu, uint32_t* s,
                double* a, double* b, double* c) {
  if (rk_variant != MMP_RK_BY_ORDER && rk_variant != MMP_RK_BUTCHER7_LAMBDA_MU)
    return fail(MMP_EINVAL, "unknown rk_variant");
  mmp_params p;
  std::memset(&p, 0, sizeof(p));
  p.method_order = method_order;
  p.rk_variant = rk_variant;
  p.rk_lambda = rk_lambda;
  p.rk_mu = rk_mu;
  Tableau t;
  tableau_for(&p, t);
  if (s) *s = (uint32_t)t.s;
  for (int i = 0; i < kMaxStages; ++i) {
    for (int j = 0; j < kMaxStages; ++j)
      if (a) a[i * kMaxStages + j] = t.a[i][j];
    if (b) b[i] = t.b[i];
    if (c) c[i] = t.c[i];
  }
  return MMP_OK;
}

int mmp_dft(uint32_t n, uint32_t rows, int direction, int fp64, const double* in, double* out) {
  if (!in || !out || rows == 0) return fail(MMP_EINVAL, "bad dft arguments");
  if (direction != -1 && direction != 1) return fail(MMP_EINVAL, "direction must be -1 or +1");
  mmp_detail::Range range("mmp.dft");
  const int lg = ilog2_exact(n);
  if (lg < kMinLogN || lg > kMaxLogN) return fail(MMP_ENOTSUP, "n must be a power of two in [64, 65536]");
  int dev = 0;
  CUDA_TRY(cudaGetDevice(&dev));
  DeviceRes* res = nullptr;
  int rc = ensure_device(dev, &res);
  if (rc) return rc;
  KernelSet ks = kernels_for(fp64 ? 1 : 0, lg);
  const size_t bytes = (size_t)rows * n * sizeof(double2);
  double2* d_in = nullptr;
  double2* d_out = nullptr;
  cudaStream_t st = nullptr;
  CUDA_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  cudaError_t e = dev_malloc((void**)&d_in, bytes);
  if (e == cudaSuccess) e = dev_malloc((void**)&d_out, bytes);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_in, in, bytes, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) {
    DftArgs a;
    std::memset(&a, 0, sizeof(a));
    a.in = d_in;
    a.out = d_out;
    a.rows = (int)rows;
    a.scale = direction < 0 ? 1.0 : 1.0 / (double)n;
    a.tw = res->tw;
    void* args[] = {&a};
    e = launch(direction < 0 ? ks.dft_fwd : ks.dft_inv, dim3(rows * (unsigned)ks.C, 1, 1), ks.nthr,
               ks.smem, ks.C, st, args);
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(out, d_out, bytes, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  dev_free(d_in);
  dev_free(d_out);
  cudaStreamDestroy(st);
  if (e != cudaSuccess)
    return fail(e == cudaErrorMemoryAllocation ? MMP_ENOMEM : MMP_ECUDA, std::string("mmp_dft: ") + cudaGetErrorString(e));
  return MMP_OK;
}

const char* mmp_strerror(int code) {
  switch (code) {
    case MMP_OK: return "ok";
    case MMP_EINVAL: return "invalid parameters";
    case MMP_ENOMEM: return "out of memory";
    case MMP_ECUDA: return "CUDA runtime error";
    case MMP_ENONFINITE: return "field became non-finite";
    case MMP_ETIMEOUT: return "timed out";
    case MMP_ENOTSUP: return "not supported by this build";
    case MMP_ENODEV: return "no sm_100 device";
    case MMP_ESTATE: return "invalid state for this call";
    case MMP_EDRIFT: return "energy drift above the set limit";
    default: return "unknown error";
  }
}

const char* mmp_last_error(void) { return g_last_error; }

const char* mmp_version(void) { return "mmp_b200 0.1.0 (sm_100a)"; }

uint64_t mmp_kernel_launch_count(void) { return g_launches.load(); }

int mmp_debug_fail_alloc(int64_t after) {
  g_fail_after.store(after < 0 ? -1 : after);
  return MMP_OK;
}

int64_t mmp_debug_live_allocations(void) { return g_live.load(); }

}  // extern "C"

// serving loop (mmp_server_*): slot pools built on the batch machinery above
#include "server.cuh"
