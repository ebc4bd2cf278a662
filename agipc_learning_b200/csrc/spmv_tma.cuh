// spmv_tma.cuh -- BCSR SpMV with the block stream staged by TMA bulk copies.
//
// Persistent CTAs walk 32-row chunks.  For each chunk one thread issues two
// cp.async.bulk copies (values and column indices of the chunk's blocks, a
// contiguous byte range each) into a shared-memory stage tracked by an
// mbarrier; the next chunk is in flight while the current one is computed.
// 16 lanes own one block row and read its blocks from shared memory (stride
// of 9 words: conflict free); x is gathered through L1/L2.  A chunk whose
// blocks do not fit a stage is computed straight from global memory.
// Every mbarrier wait is bounded; on expiry the kernel records an error and
// leaves.
#pragma once
#include "maspcg_internal.cuh"
#include "spmv_row.cuh"

namespace maspcg {

constexpr int kTmaRows = 32;        // block rows per chunk
constexpr int kTmaThreads = 512;    // 16 lanes per row
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

template <typename Tm>
struct TmaStage {
  static constexpr int kCap = sizeof(Tm) == 4 ? 1024 : 512;      // blocks per stage
  static constexpr int kValBytes = kCap * 9 * (int)sizeof(Tm) + 32;
  static constexpr int kColBytes = kCap * 4 + 32;
};

template <typename Tm>
__device__ __forceinline__ void chunk_issue(int chunk, int nrows, const int* __restrict__ rowptr, const Tm* val,
                                            const int* colidx, unsigned char* sval, unsigned char* scol, uint64_t* bar)
{
  const int r0 = chunk * kTmaRows, r1 = min(r0 + kTmaRows, nrows);
  const int b0 = rowptr[r0], b1 = rowptr[r1];
  if (b1 - b0 > TmaStage<Tm>::kCap || b1 == b0) return;  // oversized or empty: computed from global
  const size_t vs = ((size_t)b0 * 9 * sizeof(Tm)) & ~(size_t)15;
  const size_t ve = ((size_t)b1 * 9 * sizeof(Tm) + 15) & ~(size_t)15;
  const size_t cs = ((size_t)b0 * 4) & ~(size_t)15;
  const size_t ce = ((size_t)b1 * 4 + 15) & ~(size_t)15;
  mbar_expect_tx(bar, (unsigned)((ve - vs) + (ce - cs)));
  tma_bulk_g2s(sval, reinterpret_cast<const unsigned char*>(val) + vs, (unsigned)(ve - vs), bar);
  tma_bulk_g2s(scol, reinterpret_cast<const unsigned char*>(colidx) + cs, (unsigned)(ce - cs), bar);
}

}  // namespace maspcg
