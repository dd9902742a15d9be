// kern_inst.cu — compiled once per (precision, log2 NT) with
//   -DMMP_REAL=float|double -DMMP_LOGN=<6..16> -DMMP_TAG=f32|f64
// so that the heavily unrolled FFT kernels build in parallel.
#include "kernel_table.h"
#include "stage_kernels.cuh"

#define MMP_CAT3_(a, b, c) a##b##_##c
#define MMP_CAT3(a, b, c) MMP_CAT3_(a, b, c)

namespace mmp {

KernelSet MMP_CAT3(make_kernels_, MMP_TAG, MMP_LOGN)() {
  using T = MMP_REAL;
  constexpr int L = MMP_LOGN;
  using Gm = Geo<T, L>;
  KernelSet k;
  k.prime = (const void*)&k_prime<T, L>;
  k.pair = (const void*)&k_pair<T, L>;
  k.nu = (const void*)&k_nu<T, L>;
  k.result = (const void*)&k_result<T, L>;
  k.dft_fwd = (const void*)&k_dft<T, L, false>;
  k.dft_inv = (const void*)&k_dft<T, L, true>;
  k.C = Gm::C;
  k.nthr = Gm::NTHR;
  k.smem = Gm::SMEM_BYTES;
  k.logn = L;
  k.fp64 = sizeof(T) == 8;
  return k;
}

}  // namespace mmp
