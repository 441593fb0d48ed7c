// umma_core.cuh — the tcgen05 building blocks shared by this library's
// tensor-core kernels (the bf16 GEMM of umma_gemm.cuh and the INT8
// correlation of corr_i8.cuh): shared-memory addresses and no-swizzle matrix
// descriptors, the commit of issued MMAs to an mbarrier, and bounded
// mbarrier waits.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace umma {

constexpr long long kSpinLimit = 20000000;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor, SWIZZLE_NONE, K-major (core matrices of
// 8 rows x 16 bytes; used by the INT8 correlation kernel).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version for sm_100
  return d;                // base offset 0, legacy LBO mode, layout type 0 (no swizzle)
}

__device__ __forceinline__ void commit_to(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ bool try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// bounded wait; false after kSpinLimit polls
__device__ __forceinline__ bool wait_parity(uint64_t* bar, uint32_t parity) {
  for (long long i = 0; i < kSpinLimit; ++i)
    if (try_wait(bar, parity)) return true;
  return false;
}

}  // namespace umma
