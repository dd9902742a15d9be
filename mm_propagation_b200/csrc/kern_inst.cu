// kern_inst.cu — compiled once per (precision, log2 NT, row split) with
//   -DMMP_REAL=float|double -DMMP_LOGN=<6..16> -DMMP_TAG=f32|f64 -DMMP_XC=<0|1>
// so that the heavily unrolled FFT kernels build in parallel. MMP_XC = 1 splits
// every row over twice as many CTAs (a cluster), halving each CTA's shared memory
// and registers so that two CTAs share an SM; the solver times both and keeps the
// faster (see solver.cu, autotune).
#include "kernel_table.h"
#include "stage_kernels.cuh"

#ifndef MMP_XC
#define MMP_XC 0
#endif

#define MMP_CAT4_(a, b, c, d) a##b##_##c##_##d
#define MMP_CAT4(a, b, c, d) MMP_CAT4_(a, b, c, d)

namespace mmp {

KernelSet MMP_CAT4(make_kernels_, MMP_TAG, MMP_LOGN, MMP_XC)() {
  using T = MMP_REAL;
  constexpr int L = MMP_LOGN;
  constexpr int X = MMP_XC;
  using Gm = Geo<T, L, X>;
  KernelSet k;
  k.prime = (const void*)&k_prime<T, L, X>;
  k.pair = (const void*)&k_pair<T, L, X>;
  k.nu = (const void*)&k_nu<T, L, X, -1>;
  // specialised stage bodies: RK4's (0 and last-3) in both precisions, the order-6 and
  // order-8 tableaus' (intermediate 1..5, last 4) in FP32
  k.nu_mid[0] = (const void*)&k_nu<T, L, X, 0>;
  k.nu_last[3] = (const void*)&k_nu<T, L, X, kNuLastBody + 3>;
  if constexpr (sizeof(T) == 4) {
    k.nu_mid[1] = (const void*)&k_nu<T, L, X, 1>;
    k.nu_mid[2] = (const void*)&k_nu<T, L, X, 2>;
    k.nu_mid[3] = (const void*)&k_nu<T, L, X, 3>;
    k.nu_mid[4] = (const void*)&k_nu<T, L, X, 4>;
    k.nu_mid[5] = (const void*)&k_nu<T, L, X, 5>;
    k.nu_last[4] = (const void*)&k_nu<T, L, X, kNuLastBody + 4>;
  }
  k.result = (const void*)&k_result<T, L, X>;
  k.dft_fwd = (const void*)&k_dft<T, L, X, false>;
  k.dft_inv = (const void*)&k_dft<T, L, X, true>;
  k.C = Gm::C;
  k.nthr = Gm::NTHR;
  k.smem = Gm::SMEM_BYTES;
  k.logn = L;
  k.fp64 = sizeof(T) == 8;
  k.xc = X;
  return k;
}

}  // namespace mmp
