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

// The stopping gate after the x / r update of iteration k (PCGSolver::pcg,
// pcg_solver.cu:277-282: tested with the r.z of before the update): the rz
// gate |r.z| <= tol r0.z0, or the Euclidean ||r|| <= tol ||b|| on rr.  MIXED:
// a met gate asks for the FP64 true residual instead of stopping.  Returns
// true when the loop stops here (gate met or rr not finite).
__device__ __forceinline__ bool gate_check(PcgScalars* s, double rr, int mixed)
{
  s->rr = rr;
  s->rr_peak = fmax(s->rr_peak, rr);
  if (!isfinite(rr)) {
    s->status = MASPCG_SOLVE_NONFINITE;
    s->iterations = s->k;
    return true;
  }
  const bool conv = (s->gate == MASPCG_GATE_RZ) ? (fabs(s->rz) <= s->tol * s->rz0) : (rr <= s->tol * s->tol * s->bb);
  if (!conv) return false;
  if (mixed) {
    s->status = kNeedTrue;
  } else {
    s->status = MASPCG_SOLVE_CONVERGED;
    s->iterations = s->k;
  }
  return true;
}

// Modes of the r.z completion (the end of a preconditioner apply).
enum RzMode {
  kRzNone = 0,      // standalone apply: no scalar update
  kRzInitial = 1,   // initial apply: rz0, k = 1
  kRzLoop = 2,      // in the loop: beta = r.z / previous r.z, k++
  kRzFusedStd = 4,  // the apply ran behind the iteration's x / r update: the r buffers swap and the gate on s->rr
                    // comes first, then as kRzLoop
  kRzFusedMix = 5   // the same in MIXED precision (a met gate asks for the FP64 true residual)
};

// End of the preconditioner apply: r^T z of this iteration (mode: RzMode).
__device__ __forceinline__ void rz_update(PcgScalars* s, double rz_new, int mode)
{
  if (mode == kRzFusedStd || mode == kRzFusedMix) {
    s->rbuf ^= 1;
    if (gate_check(s, s->rr, mode == kRzFusedMix)) return;
    mode = kRzLoop;
  }
  s->rz_new = rz_new;
  if (mode == kRzInitial && rz_new == 0.0 && s->bb == 0.0) {  // b = 0: x = 0 is exact
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
  if (mode == kRzInitial) {
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

// The x / r update of a PCG iteration fused into the preconditioner apply
// that follows it (the kernels that read r to precondition it update their
// own rows first):
//   x += alpha p,   r' = r - alpha Ap
// r is double-buffered (cur = s->rbuf): the coarse levels, beside the level-0
// apply, restrict r' formed again from r and Ap (the same FMA, so the same
// bits) while the apply writes it; the r.z completion swaps the buffers.
struct FusedArgs {
  const float* p4;  // search direction, padded 4 per row
  const float* ap;  // A p, 3 per row
  float* x;
  float* r[2];
  int update;       // 1: the update first; 0: r[cur] is already the residual to precondition
};

// The scalars a fused kernel reads once at entry (nothing changes them until
// every kernel of the iteration has passed its rows).
struct FusedScal {
  int cur;
  float alpha;
};
__device__ __forceinline__ FusedScal fused_scalars(const PcgScalars* s) { return FusedScal{s->rbuf, (float)s->alpha}; }

// The residual the apply of one row starts from: r' of the update (written,
// with x, when `write`: the kernel that owns the row), or r[cur] when the
// update ran before (update == 0).
__device__ __forceinline__ void fused_input_row(const FusedArgs& f, const FusedScal& fs, int row, bool write,
                                                float rn[3])
{
  const size_t b = 3 * (size_t)row;
  if (!f.update) {
#pragma unroll
    for (int q = 0; q < 3; ++q) rn[q] = f.r[fs.cur][b + q];
    return;
  }
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    rn[q] = fmaf(-fs.alpha, f.ap[b + q], f.r[fs.cur][b + q]);
    if (write) {
      f.x[b + q] = fmaf(fs.alpha, f.p4[4 * (size_t)row + q], f.x[b + q]);
      f.r[fs.cur ^ 1][b + q] = rn[q];
    }
  }
}

// Grid-wide barrier of a cooperative launch (every CTA resident).  The last
// CTA to arrive resets the count and advances the generation word the
// others wait on.  The wait is bounded (s->barrier_limit spins): on expiry
// the CTA records error 3, stops the solve and the barrier returns false
// (the caller then leaves; the host reports the error after the graph).
__device__ __forceinline__ bool grid_barrier(PcgScalars* s, int* err)
{
  __shared__ int ok_s;
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned* gen = &s->barrier_gen;
    const unsigned g0 = *gen;
    const long long limit = s->barrier_limit;
    const unsigned expected = gridDim.x + (unsigned)s->barrier_extra;
    __threadfence();
    int ok = 1;
    if (atomicAdd(&s->tickets[kTicketBarrier], 1u) == expected - 1) {
      s->tickets[kTicketBarrier] = 0u;
      __threadfence();
      atomicAdd(&s->barrier_gen, 1u);
    } else {
      long long it = 0;
      while (*gen == g0) {
        if (++it > limit) {
          // give up: record the error and stop the solve, so every later
          // kernel returns at entry and the host reads the error after this
          // graph launch
          ok = 0;
          atomicExch(err, 3);
          atomicExch(&s->status, (int)MASPCG_SOLVE_NONFINITE);
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
