// tma.cuh -- mbarrier and bulk-copy (cp.async.bulk) helpers for kernels that
// stage contiguous records in shared memory.  Every wait is bounded: on
// expiry the caller records an error and leaves instead of spinning.
#pragma once
#include "maspcg_internal.cuh"

namespace maspcg {

constexpr long long kWaitLimit = 1ll << 26;

__device__ __forceinline__ unsigned smem_addr(const void* p)
{
  return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes)
{
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}

// Global -> shared bulk copy completing on `bar`; dst, src and bytes must be
// multiples of 16.
__device__ __forceinline__ void tma_bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar)
{
  asm volatile(
      "cp.async.bulk.shared::cta.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

// Bounded wait for the phase `parity` of the barrier; false on expiry.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity)
{
  const unsigned a = smem_addr(bar);
  for (long long it = 0; it < kWaitLimit; ++it) {
    unsigned done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

}  // namespace maspcg
