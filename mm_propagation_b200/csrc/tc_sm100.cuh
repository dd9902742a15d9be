// tc_sm100.cuh — the 5th-generation tensor core (tcgen05) of sm_100a as inline PTX: tensor
// memory (TMEM) allocation, shared-memory matrix descriptors, the TF32 MMA with FP32
// accumulators in TMEM, its completion on an mbarrier, and TMEM loads.
//
// Two operand layouts are described here. K-major without swizzle (desc_kmajor): a matrix
// of R rows by K 32-bit values stored as [K/4][R][4], i.e. for every group of 4 consecutive
// K values the R rows follow each other 16 bytes apart; the hardware's 8-row x 16-byte core
// matrices are then contiguous 128-byte blocks (stride-byte offset SBO = 128 between 8-row
// groups) and the two 16-byte K halves of one MMA (K = 8 for TF32) are R * 16 bytes apart
// (leading-byte offset LBO), so the MMA's K step advances the start address by 2 R 16 bytes.
// MN-major TF32 (desc_mn_tf32, mn_tf32_offset): see below.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace mmp {
namespace tc {

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor (64 bits): start address, LBO and SBO in 16-byte units
// (14 bits each, at bits 0, 16 and 32), descriptor version 1 at bit 46, base offset 0,
// layout type 0 (no swizzle) in bits 61-63.
__device__ __forceinline__ uint64_t desc_kmajor(const void* base, uint32_t lbo_bytes, uint32_t sbo_bytes) {
  uint64_t d = (uint64_t)((smem_u32(base) >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// MN-major TF32 operand (the one swizzled layout the tensor core takes for MN-major 32-bit
// operands, "128B with 32-byte atoms"): atoms of 4 K-rows x 128 bytes (32 values along M or
// N), 512-byte aligned, in which the 32-byte chunk index (address bits 5-6) is XORed with
// the row index (bits 7-8). LBO = bytes between consecutive atoms along M/N, SBO = bytes
// between consecutive 4-row groups along K; layout type 1 in bits 61-63.
__device__ __forceinline__ uint64_t desc_mn_tf32(const void* base, uint32_t lbo_bytes, uint32_t sbo_bytes) {
  return desc_kmajor(base, lbo_bytes, sbo_bytes) | ((uint64_t)1 << 61);
}
// Byte offset of element (mn, k) in such an operand.
__host__ __device__ __forceinline__ uint32_t mn_tf32_offset(int mn, int k, uint32_t lbo, uint32_t sbo) {
  const int r = k & 3, chunk = (mn >> 3) & 3;
  return (uint32_t)(k >> 2) * sbo + (uint32_t)(mn >> 5) * lbo + (uint32_t)r * 128u +
         (uint32_t)((chunk ^ r) << 5) + (uint32_t)((mn & 7) << 2);
}

// Instruction descriptor (32 bits): FP32 accumulator (bits 4-5 = 1), A and B in TF32
// (bits 7-9 and 10-12 = 2), A K-major (bit 15 = 0) or MN-major (1), B K-major (bit 16 = 0),
// N / 8 at bit 17, M / 16 at bit 24.
__host__ __device__ constexpr uint32_t idesc_tf32(int M, int N, bool a_mn_major = false) {
  return (1u << 4) | (2u << 7) | (2u << 10) | (a_mn_major ? (1u << 15) : 0u) | ((uint32_t)(N >> 3) << 17) |
         ((uint32_t)(M >> 4) << 24);
}

// D[tmem] (+)= A * B^T for one K step of 8; issued by a single thread.
__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
  const uint32_t z = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z)
      : "memory");
}

// The mbarrier at bar gets one arrival once every MMA this thread issued before has completed.
__device__ __forceinline__ void commit(unsigned long long* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

// TMEM allocation by one full warp: ncols (a power of two, 32..512) columns of all 128
// lanes; the base address is written to *dst in shared memory.
__device__ __forceinline__ void alloc(uint32_t* dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)), "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy shared-memory writes become visible to the tensor core (async proxy)
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 16 consecutive 32-bit columns of this thread's TMEM lane (warp w reads lanes
// 32 (w % 4) .. + 31; taddr carries that lane base in bits 16-31), then wait for them.
__device__ __forceinline__ void ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// x rounded to TF32 (10 explicit mantissa bits, nearest, ties away from zero) in a 32-bit
// container, and the FP32 remainder: x = hi + lo exactly, |lo| <= 2^-11 |x|.
__device__ __forceinline__ float tf32_hi(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

}  // namespace tc
}  // namespace mmp
