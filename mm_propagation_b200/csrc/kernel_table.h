// kernel_table.h — host-visible handles to the kernels instantiated for one
// (precision, log2 NT) pair by kern_inst.cu.
#pragma once

namespace mmp {

struct KernelSet {
  const void* prime = nullptr;
  const void* pair = nullptr;
  const void* nu = nullptr;          // k_nu for any stage
  const void* nu_mid[6] = {};        // ... for intermediate stages reading n stored N_hat_j
  const void* nu_last[5] = {};       // ... for last stages reading n (null: not built)
  const void* result = nullptr;
  const void* dft_fwd = nullptr;
  const void* dft_inv = nullptr;
  int C = 0;      // CTAs per row (cluster size)
  int nthr = 0;   // threads per CTA
  int smem = 0;   // dynamic shared memory per CTA, bytes
  int logn = 0;
  int fp64 = 0;
  int xc = 0;     // rows split over 2^xc times the minimal number of CTAs
};

constexpr int kMinLogN = 6;
constexpr int kMaxLogN = 16;

// Row-split variants built besides xc = 0 (FP32 / FP64 ranges of log2 NT).
constexpr int kSplitMinLogN32 = 12, kSplitMaxLogN32 = 16;
constexpr int kSplitMinLogN64 = 11, kSplitMaxLogN64 = 14;

// Defined in the kern_inst.cu objects; returns an empty set for variants not built.
KernelSet kernels_for(int fp64, int logn, int xc = 0);

}  // namespace mmp
