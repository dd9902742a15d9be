// kernel_table.h — host-visible handles to the kernels instantiated for one
// (precision, log2 NT) pair by kern_inst.cu.
#pragma once

namespace mmp {

struct KernelSet {
  const void* prime = nullptr;
  const void* pair = nullptr;
  const void* nu = nullptr;
  const void* result = nullptr;
  const void* dft_fwd = nullptr;
  const void* dft_inv = nullptr;
  int C = 0;      // CTAs per row (cluster size)
  int nthr = 0;   // threads per CTA
  int smem = 0;   // dynamic shared memory per CTA, bytes
  int logn = 0;
  int fp64 = 0;
};

constexpr int kMinLogN = 6;
constexpr int kMaxLogN = 16;

// Defined in the kern_inst.cu objects; returns an empty set for sizes not built.
KernelSet kernels_for(int fp64, int logn);

}  // namespace mmp
