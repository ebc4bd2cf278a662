// pcg_device.cuh -- grid reductions with a last-block epilogue and the
// device-side PCG scalar updates shared by the iteration kernels.
#pragma once
#include "maspcg_internal.cuh"

namespace maspcg {

constexpr int kRedTpb = 256;

// Block-sum v, store it in partial[slot]; the last block to arrive (counted
// on *ticket against `expected` blocks) sums partial[0..total_parts) in a
// fixed order.  Returns true in every thread of that last block; the sum is
// valid in thread 0.  NT must equal blockDim.x (the block reduction sizes
// its shared array and its final warp from it).
template <typename Tacc, int NT = kRedTpb>
__device__ __forceinline__ bool grid_finish(Tacc v, Tacc* partial, int slot, int total_parts, unsigned* ticket,
                                            unsigned expected, Tacc& total)
{
  static_assert(NT % 32 == 0 && NT >= 32 && NT <= 1024, "block size");
  __shared__ Tacc red[NT / 32];
  __shared__ int last;
  const Tacc b = block_sum<Tacc, NT>(v, red);
  if (threadIdx.x == 0) {
    partial[slot] = b;
    __threadfence();
    const unsigned t = atomicAdd(ticket, 1u);
    last = (t == expected - 1) ? 1 : 0;
  }
  __syncthreads();
  if (!last) return false;
  __threadfence();
  Tacc s = 0;
  for (int i = threadIdx.x; i < total_parts; i += blockDim.x) s += __ldcg(partial + i);
  s = block_sum<Tacc, NT>(s, red);
  if (threadIdx.x == 0) {
    total = s;
    *ticket = 0u;
  }
  return true;
}

// End of the preconditioner apply: r^T z of this iteration.
// mode 1: initial apply (rz0); mode 2: inside the loop (beta, k++).
__device__ __forceinline__ void rz_update(PcgScalars* s, double rz_new, int mode)
{
  s->rz_new = rz_new;
  if (mode == 1 && rz_new == 0.0 && s->bb == 0.0) {  // b = 0: x = 0 is exact
    s->rz = s->rz0 = 0.0;
    s->k = 0;
    s->status = MASPCG_SOLVE_CONVERGED;
    s->iterations = 0;
    return;
  }
  if (!isfinite(rz_new)) {
    s->status = MASPCG_SOLVE_NONFINITE;
    s->iterations = s->k;
    return;
  }
  if (!(rz_new > 0.0)) {
    s->status = MASPCG_SOLVE_INVALID_RZ;
    s->iterations = s->k;
    return;
  }
  if (mode == 1) {
    s->rz = rz_new;
    s->rz0 = rz_new;
    s->k = 1;
    s->beta = 0.0;
  } else {
    s->beta = rz_new / s->rz;
    s->rz = rz_new;
    s->k += 1;
  }
  if (s->k >= s->max_iter) {
    s->status = MASPCG_SOLVE_ITERATION_CAP;
    s->iterations = s->max_iter;
  }
}

// Grid-wide barrier of a cooperative launch (every CTA resident).  The last
// CTA to arrive resets the count and advances the generation word the
// others wait on.  The wait is bounded: on expiry the CTA records error 3
// and the barrier returns false (the caller then leaves; the host reports
// the error after the graph).
constexpr long long kBarrierLimit = 1ll << 24;

__device__ __forceinline__ bool grid_barrier(PcgScalars* s, int* err)
{
  __shared__ int ok_s;
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned* gen = &s->barrier_gen;
    const unsigned g0 = *gen;
    __threadfence();
    int ok = 1;
    if (atomicAdd(&s->tickets[kTicketBarrier], 1u) == gridDim.x - 1) {
      s->tickets[kTicketBarrier] = 0u;
      __threadfence();
      atomicAdd(&s->barrier_gen, 1u);
    } else {
      long long it = 0;
      while (*gen == g0) {
        if (++it > kBarrierLimit) {
          ok = 0;
          atomicExch(err, 3);
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
    ok_s = ok;
  }
  __syncthreads();
  return ok_s != 0;
}

// r.z summed by two concurrent kernels (the level-0 apply and the coarse
// levels): each stores its part and takes a ticket; the second adds the two
// parts in a fixed order and updates the scalars (mode as in rz_update).
__device__ __forceinline__ void rz_part_done(PcgScalars* s, int part, double value, int mode)
{
  s->rz_part[part] = value;
  __threadfence();
  const unsigned t = atomicAdd(&s->tickets[kTicketPair], 1u);
  if (t == 1u) {
    __threadfence();
    const double total = __ldcg(&s->rz_part[0]) + __ldcg(&s->rz_part[1]);
    s->tickets[kTicketPair] = 0u;
    if (mode > 0) rz_update(s, total, mode);
  }
}

// ---- padded search direction: one 16-byte (FP32) / 32-byte (FP64) slot per
// block row, so the SpMV gathers a column's three entries with one vector load.
template <typename T>
struct P4;
template <>
struct P4<float> {
  float x, y, z, w;
};
template <>
struct P4<double> {
  double x, y, z, w;
};

__device__ __forceinline__ P4<float> ld_p4(const float* p4, int v)
{
  const float4 q = __ldg(reinterpret_cast<const float4*>(p4) + v);
  return {q.x, q.y, q.z, q.w};
}
__device__ __forceinline__ P4<double> ld_p4(const double* p4, int v)
{
  const double2 a = __ldg(reinterpret_cast<const double2*>(p4) + 2 * v);
  const double2 b = __ldg(reinterpret_cast<const double2*>(p4) + 2 * v + 1);
  return {a.x, a.y, b.x, b.y};
}
__device__ __forceinline__ void st_p4(float* p4, int v, float x, float y, float z)
{
  reinterpret_cast<float4*>(p4)[v] = make_float4(x, y, z, 0.f);
}
__device__ __forceinline__ void st_p4(double* p4, int v, double x, double y, double z)
{
  reinterpret_cast<double2*>(p4)[2 * v] = make_double2(x, y);
  reinterpret_cast<double2*>(p4)[2 * v + 1] = make_double2(z, 0.0);
}

}  // namespace maspcg
