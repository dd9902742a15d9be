// noalloc.cu — mmp_dft_noalloc: the batched transform of mmp_dft without any
// device (or host) memory allocation.
//
// Who needs this: code that may not call cudaMalloc at the point where it wants a
// transform — for example a host that has handed the whole device memory pool to
// its own caching allocator (so a fresh cudaMalloc fails or fragments the pool),
// a latency-bound loop that cannot afford the implicit device synchronisation a
// cudaMalloc/cudaFree pair can cause, or a plugin whose memory budget is fixed
// when the library is loaded. mmp_dft allocates a device copy of the input and
// output on every call; this entry point stages them in memory reserved when
// the library is loaded instead.
//
// Memory: one file-scope static device array (kArenaBytes, about 19 MiB) holds
// the FP64 and FP32 twiddle tables for every supported size followed by a
// staging buffer of kMaxSamples complex FP64 samples. Every GPU that loads this
// library holds the array until the process exits. The transform runs in place
// in the staging buffer (each row is read whole into shared memory before any
// of it is written), so no second buffer is needed.
//
// Set-up: the first call on a device, with that device current, looks up the
// array's device address with cudaGetSymbolAddress (host code may not use the
// array's name as a device address) and fills the twiddle tables with one
// kernel launch. Make that first call before any stream capture.
//
// Sharing: all calls on a device share the one staging buffer and leave their
// data in it. Nothing in it needs to start at zero (each call writes every sample
// it reads), but calls that overlap on the GPU — from several host threads — race
// on it; serialise them.
//
// Errors are reported like every other entry point's: a negative MMP_E* code, and
// the text in mmp_last_error() on the calling thread (recorded into a fixed buffer,
// without allocating). Its kernel launches are counted in mmp_kernel_launch_count().
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "kernel_table.h"
#include "mmp.h"
#include "stage_kernels.cuh"

using namespace mmp;

namespace {

constexpr size_t kTwEntries = ((size_t)1 << (kMaxLogN + 1)) - 2;  // sum over L = 1..16 of 2^L
constexpr size_t kMaxSamples = (size_t)1 << 20;                  // complex FP64 staging samples
constexpr size_t kTwD = kTwEntries * sizeof(double2);
constexpr size_t kTwF = kTwEntries * sizeof(float2);
constexpr size_t kStageOff = ((kTwD + kTwF) + 255) & ~(size_t)255;
constexpr size_t kArenaBytes = kStageOff + kMaxSamples * sizeof(double2);

static __device__ __align__(256) unsigned char g_noalloc_arena[kArenaBytes];

// w_L[m] = exp(-2 pi i m / 2^L) for L = 1..16; table L starts at entry 2^L - 2.
__global__ void k_fill_twiddles(double2* d, float2* f) {
  for (size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x; g < kTwEntries;
       g += (size_t)gridDim.x * blockDim.x) {
    int L = 1;
    while (((size_t)1 << (L + 1)) - 2 <= g) ++L;
    const size_t m = g - (((size_t)1 << L) - 2);
    double s, c;
    sincospi(-2.0 * (double)m / (double)((size_t)1 << L), &s, &c);
    d[g] = make_double2(c, s);
    f[g] = make_float2((float)c, (float)s);
  }
}

struct NoallocDevice {
  bool ready = false;
  unsigned char* base = nullptr;
  TwTables tw{};
};
std::mutex g_mu;
constexpr int kMaxDevices = 64;
NoallocDevice g_devs[kMaxDevices];  // fixed table: no allocation on any call

}  // namespace

namespace mmp_detail {
int set_error_c(int code, const char* msg);  // solver.cu: the text mmp_last_error returns
void count_launch();                          // solver.cu: mmp_kernel_launch_count
}  // namespace mmp_detail

namespace {

int fail(int code, const char* msg) { return mmp_detail::set_error_c(code, msg); }

int setup(int dev, NoallocDevice** out) {
  if (dev < 0 || dev >= kMaxDevices) return fail(MMP_ENODEV, "device ordinal out of range");
  std::lock_guard<std::mutex> lk(g_mu);
  NoallocDevice& r = g_devs[dev];
  if (r.ready) { *out = &r; return MMP_OK; }
  int major = 0;
  if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev) != cudaSuccess || major < 10)
    return fail(MMP_ENODEV, "no sm_100 device");
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_arena);
  if (e != cudaSuccess || !p) return fail(MMP_ECUDA, cudaGetErrorString(e));
  r.base = static_cast<unsigned char*>(p);
  double2* d = reinterpret_cast<double2*>(r.base);
  float2* f = reinterpret_cast<float2*>(r.base + kTwD);
  k_fill_twiddles<<<256, 256>>>(d, f);
  e = cudaGetLastError();
  if (e == cudaSuccess) mmp_detail::count_launch();
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e != cudaSuccess) return fail(MMP_ECUDA, cudaGetErrorString(e));
  for (int L = 0; L <= kMaxLogN; ++L) {
    r.tw.d[L] = L ? d + (((size_t)1 << L) - 2) : nullptr;
    r.tw.f[L] = L ? f + (((size_t)1 << L) - 2) : nullptr;
  }
  for (int fp64 = 0; fp64 < 2; ++fp64)
    for (int L = kMinLogN; L <= kMaxLogN; ++L) {
      KernelSet ks = kernels_for(fp64, L);
      if (!ks.dft_fwd) continue;
      if (cudaFuncSetAttribute(ks.dft_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, ks.smem) != cudaSuccess ||
          cudaFuncSetAttribute(ks.dft_inv, cudaFuncAttributeMaxDynamicSharedMemorySize, ks.smem) != cudaSuccess)
        return fail(MMP_ECUDA, "cudaFuncSetAttribute failed");
    }
  r.ready = true;
  *out = &r;
  return MMP_OK;
}

}  // namespace

extern "C" {

int mmp_dft_noalloc(uint32_t n, uint32_t rows, int direction, int fp64, const double* in, double* out) {
  if (!in || !out || rows == 0) return fail(MMP_EINVAL, "bad dft arguments");
  if (direction != -1 && direction != 1) return fail(MMP_EINVAL, "direction must be -1 or +1");
  if (n == 0 || (n & (n - 1))) return fail(MMP_ENOTSUP, "n must be a power of two in [64, 65536]");
  int lg = 0;
  while ((1u << lg) < n) ++lg;
  if (lg < kMinLogN || lg > kMaxLogN) return fail(MMP_ENOTSUP, "n must be a power of two in [64, 65536]");
  if ((size_t)rows * n > kMaxSamples)
    return fail(MMP_EINVAL, "rows * n exceeds the 2^20-sample static staging buffer of mmp_dft_noalloc");
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return fail(MMP_ECUDA, "cudaGetDevice failed");
  NoallocDevice* r = nullptr;
  int rc = setup(dev, &r);
  if (rc) return rc;
  const KernelSet ks = kernels_for(fp64 ? 1 : 0, lg);
  double2* stage = reinterpret_cast<double2*>(r->base + kStageOff);
  const size_t bytes = (size_t)rows * n * sizeof(double2);
  cudaError_t e = cudaMemcpy(stage, in, bytes, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    DftArgs a;
    std::memset(&a, 0, sizeof(a));
    a.in = stage;
    a.out = stage;
    a.rows = (int)rows;
    a.scale = direction < 0 ? 1.0 : 1.0 / (double)n;
    a.tw = r->tw;
    void* args[] = {&a};
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(rows * (unsigned)ks.C, 1, 1);
    cfg.blockDim = dim3((unsigned)ks.nthr, 1, 1);
    cfg.dynamicSmemBytes = (size_t)ks.smem;
    cfg.stream = 0;
    cudaLaunchAttribute attr[1];
    if (ks.C > 1) {
      attr[0].id = cudaLaunchAttributeClusterDimension;
      attr[0].val.clusterDim.x = (unsigned)ks.C;
      attr[0].val.clusterDim.y = 1;
      attr[0].val.clusterDim.z = 1;
      cfg.attrs = attr;
      cfg.numAttrs = 1;
    }
    e = cudaLaunchKernelExC(&cfg, direction < 0 ? ks.dft_fwd : ks.dft_inv, args);
    if (e == cudaSuccess) mmp_detail::count_launch();
  }
  if (e == cudaSuccess) e = cudaMemcpy(out, stage, bytes, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return fail(MMP_ECUDA, cudaGetErrorString(e));
  return MMP_OK;
}

}  // extern "C"
