// residual_noalloc.cu -- FP64 residual norms ||b_j - A x_j|| and ||b_j|| of up
// to MASPCG_RESIDUAL_MAX_VECTORS device-resident vectors, without allocating.
//
// This is the allocation-free variant of the FP64 true-residual kernel of the
// PCG loop (k_true_residual in pcg.cu).  That kernel works on vectors already
// permuted into the internal row order and keeps its per-block partial sums
// in buffers owned by the handle; maspcg_spmv, the public way to form
// b - A x, stages host vectors in buffers it grows on demand.  Here x and b
// stay in the caller's row order (the kernel gathers through row_of_int) and
// every byte of scratch lives in one file-scope device array:
//
//   g_residual_scratch, 65,696 bytes per device (doubles):
//     [0, 8192)           partial[block < 512][vector < 8][2]: per-block sums
//                         of r^2 and b^2
//     [8192, 8208)        result[vector][2]: ||r||, ||b||
//     [8208]              low 32 bits: completion ticket
//
// The ticket must be zero when a launch starts.  Static device storage starts
// at zero, set-up (the first call that sees the array at a new device address)
// zeroes it once more, and the last block of every launch puts it back to
// zero.  The partial sums and results need no initial value.
//
// One scratch per device and process: two launches that overlapped on one
// device would race on it.  The host entry point therefore holds a per-device
// lock from set-up to the end of its stream synchronisation.
#include <mutex>

#include "maspcg_internal.cuh"

namespace maspcg {
namespace {

constexpr int kResTpb = 256;
constexpr int kResLpr = 16;  // lanes per block row
constexpr int kResGroups = kResTpb / kResLpr;
constexpr int kResMaxVectors = MASPCG_RESIDUAL_MAX_VECTORS;
constexpr int kResMaxBlocks = 512;
constexpr size_t kResResultOffset = (size_t)kResMaxBlocks * kResMaxVectors * 2;
constexpr size_t kResTicketOffset = kResResultOffset + 2 * kResMaxVectors;
constexpr size_t kResScratchDoubles = kResTicketOffset + 4;  // whole 32-byte tail
constexpr int kMaxDevices = 64;

static_assert(kResScratchDoubles * sizeof(double) == 65696, "scratch size stated in the header comment");

static __device__ __align__(256) double g_residual_scratch[kResScratchDoubles];

// One 16-lane group per internal block row (grid-stride).  Padding rows
// (row_of_int < 0) contribute nothing; x and b are read in the caller's order.
__global__ void __launch_bounds__(kResTpb)
    k_residual_noalloc(const int* __restrict__ rowptr, const int* __restrict__ colidx, const double* __restrict__ val,
                       const int* __restrict__ row_of_int, int nrows, const double* __restrict__ x,
                       const double* __restrict__ b, long long ld, int count, double* scratch)
{
  __shared__ double red[kResTpb / 32][2 * kResMaxVectors];
  __shared__ int last;
  const int sub = threadIdx.x % kResLpr;
  double r2[kResMaxVectors], b2[kResMaxVectors];
#pragma unroll
  for (int j = 0; j < kResMaxVectors; ++j) r2[j] = b2[j] = 0.0;

  const int iters = (nrows + gridDim.x * kResGroups - 1) / (gridDim.x * kResGroups);
  for (int it = 0; it < iters; ++it) {
    const int row = (it * gridDim.x + blockIdx.x) * kResGroups + threadIdx.x / kResLpr;
    const int orig = row < nrows ? row_of_int[row] : -1;
    const int rs = orig >= 0 ? rowptr[row] : 0, re = orig >= 0 ? rowptr[row + 1] : 0;
    double acc[kResMaxVectors][3];
#pragma unroll
    for (int j = 0; j < kResMaxVectors; ++j) acc[j][0] = acc[j][1] = acc[j][2] = 0.0;
    for (int t = rs + sub; t < re; t += kResLpr) {
      const int oc = row_of_int[colidx[t]];
      if (oc < 0) continue;
      const double* B = val + 9 * (size_t)t;
      const double m0 = B[0], m1 = B[1], m2 = B[2], m3 = B[3], m4 = B[4], m5 = B[5], m6 = B[6], m7 = B[7], m8 = B[8];
#pragma unroll
      for (int j = 0; j < kResMaxVectors; ++j) {
        if (j < count) {
          const double* xs = x + j * ld + 3 * (size_t)oc;
          const double x0 = xs[0], x1 = xs[1], x2 = xs[2];
          acc[j][0] += m0 * x0 + m1 * x1 + m2 * x2;
          acc[j][1] += m3 * x0 + m4 * x1 + m5 * x2;
          acc[j][2] += m6 * x0 + m7 * x1 + m8 * x2;
        }
      }
    }
#pragma unroll
    for (int j = 0; j < kResMaxVectors; ++j) {
      if (j < count) {  // uniform: every lane of the warp takes the same branch
#pragma unroll
        for (int o = kResLpr / 2; o > 0; o >>= 1) {
          acc[j][0] += __shfl_xor_sync(kFull, acc[j][0], o, kResLpr);
          acc[j][1] += __shfl_xor_sync(kFull, acc[j][1], o, kResLpr);
          acc[j][2] += __shfl_xor_sync(kFull, acc[j][2], o, kResLpr);
        }
        if (orig >= 0 && sub < 3) {
          const double ax = sub == 0 ? acc[j][0] : (sub == 1 ? acc[j][1] : acc[j][2]);
          const double bv = b[j * ld + 3 * (size_t)orig + sub];
          const double v = bv - ax;
          r2[j] += v * v;
          b2[j] += bv * bv;
        }
      }
    }
  }

  // block sums -> partial[block][j][2]
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
#pragma unroll
  for (int j = 0; j < kResMaxVectors; ++j) {
    if (j < count) {
      const double a = warp_sum(r2[j]), c = warp_sum(b2[j]);
      if (l == 0) {
        red[w][2 * j] = a;
        red[w][2 * j + 1] = c;
      }
    }
  }
  __syncthreads();
  unsigned* ticket = reinterpret_cast<unsigned*>(scratch + kResTicketOffset);
  if (threadIdx.x < 2 * count) {
    double s = 0.0;
    for (int q = 0; q < kResTpb / 32; ++q) s += red[q][threadIdx.x];
    scratch[((size_t)blockIdx.x * kResMaxVectors) * 2 + threadIdx.x] = s;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = (atomicAdd(ticket, 1u) == gridDim.x - 1) ? 1 : 0;
  __syncthreads();
  if (!last) return;
  __threadfence();
  // last block: fixed-order sums over the blocks
  if (threadIdx.x < 2 * count) {
    double s = 0.0;
    for (unsigned q = 0; q < gridDim.x; ++q) s += __ldcg(scratch + ((size_t)q * kResMaxVectors) * 2 + threadIdx.x);
    scratch[kResResultOffset + threadIdx.x] = sqrt(s);
  }
  if (threadIdx.x == 0) *ticket = 0u;
}

std::mutex g_res_lock[kMaxDevices];
double* g_res_scratch[kMaxDevices] = {};

}  // namespace

void residual_norms_noalloc(maspcg_handle* h, int count, const double* x, const double* b, double* residual_norms,
                            double* rhs_norms)
{
  MREQ(h->device >= 0 && h->device < kMaxDevices, MASPCG_ERR_UNSUPPORTED, "device ordinal beyond the scratch table");
  std::lock_guard<std::mutex> lock(g_res_lock[h->device]);
  // The array's device address is looked up on every call (a lookup, not an
  // allocation): a context created again on this device (after
  // cudaDeviceReset, or a handle on a non-primary context) loads the module
  // again at another address, and a cached address would then be stale.
  void* p = nullptr;
  MCK(cudaGetSymbolAddress(&p, g_residual_scratch));
  double*& seen = g_res_scratch[h->device];
  if (seen != static_cast<double*>(p)) {
    // set-up for this module instance, with h->device current: a freshly
    // loaded array is zero already; the ticket is cleared once more
    MCK(cudaMemsetAsync(static_cast<double*>(p) + kResTicketOffset, 0, sizeof(double), h->stream));
    MCK(cudaStreamSynchronize(h->stream));
    seen = static_cast<double*>(p);
  }
  double* scratch = seen;
  const int grid = std::max(1, std::min(std::min(2 * h->sm_count, kResMaxBlocks), ceil_div(h->nb_int, kResGroups)));
  k_residual_noalloc<<<grid, kResTpb, 0, h->stream>>>(h->rowptr.get(), h->colidx.get(), h->val64.get(),
                                                      h->row_of_int.get(), h->nb_int, x, b, 3LL * h->nb, count,
                                                      scratch);
  MLAUNCHED(h);
  MCK(cudaGetLastError());
  double out[2 * kResMaxVectors];
  MCK(cudaMemcpyAsync(out, scratch + kResResultOffset, 2 * (size_t)count * sizeof(double), cudaMemcpyDeviceToHost,
                      h->stream));
  MCK(cudaStreamSynchronize(h->stream));
  for (int j = 0; j < count; ++j) {
    residual_norms[j] = out[2 * j];
    if (rhs_norms) rhs_norms[j] = out[2 * j + 1];
  }
}

}  // namespace maspcg
