// contact.cu -- the per-triplet fix-ups between the contact/element Hessian
// producers and the triplet merge, in place on the device:
//
// * adjust_contacts: adjust_fem_fem_contact_indices_kernel (StiffGIPC/
//   GIPC.cu:10130-10160).  A barrier Hessian contributes the full 4x4 block
//   pattern of its pair, so every off-diagonal coupling appears twice, as
//   (a, b) and (b, a).  The lower copy (row > col) is moved onto the upper
//   slot and its value cleared, so only the upper copy carries the block;
//   an upper triplet touching a vertex with a nonzero boundary type is
//   cleared too; both indices move into the global Hessian numbering by the
//   FEM offset.
// * zero_boundary: zero_fem_boundary_hessian_kernel (GIPC.cu:10162-10181):
//   element triplets touching a boundary vertex are cleared.
// * gather_triplets: a subsystem's triplets picked from the global list by
//   index and shifted into the subsystem's numbering, as
//   LocalPreconditioner::calculate_subsystem_bcoo_indices and
//   setPreconditioner_bcoo pick them (i_preconditioner.cu:54-89).
//
// Integer work plus stores of +0.0, so the outputs are bit-exact.  The
// reference reads bd_type without a bound check; here an index outside
// [0, n_vertices) skips that triplet and the call reports it.
#include "maspcg_internal.cuh"

namespace maspcg {
namespace {

constexpr int kContactTpb = 256;

// Clears values9[9 t .. 9 t + 8] for the triplets t of this warp whose
// `clear` flag is set: the warp's 32 x 9 doubles are written as coalesced
// runs, each lane taking every 32nd double of the warp's span.
__device__ __forceinline__ void clear_flagged(double* values9, int warp_first, int n, bool clear)
{
  const unsigned mask = __ballot_sync(kFull, clear);
  if (!mask) return;
  const int lane = threadIdx.x & 31;
  const int count = min(32, n - warp_first);
  for (int e = lane; e < 9 * count; e += 32)
    if ((mask >> (e / 9)) & 1u) values9[9 * (size_t)warp_first + e] = 0.0;
}

__global__ void __launch_bounds__(kContactTpb) k_adjust_contacts(int n, int* rows, int* cols, double* values9,
                                                                   const int* __restrict__ bd_type, int n_vertices,
                                                                   int offset, int* bad)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int warp_first = i & ~31;
  if (warp_first >= n) return;  // whole warp past the end
  bool clear = false;
  if (i < n) {
    const int r = rows[i], c = cols[i];
    if (r < 0 || c < 0 || r >= n_vertices || c >= n_vertices) {
      atomicExch(bad, 1);
    } else if (r <= c) {
      rows[i] = r + offset;
      cols[i] = c + offset;
      clear = bd_type[r] != 0 || bd_type[c] != 0;
    } else {
      rows[i] = c + offset;
      cols[i] = r + offset;
      clear = true;
    }
  }
  clear_flagged(values9, warp_first, n, clear);
}

__global__ void __launch_bounds__(kContactTpb) k_zero_boundary(int n, const int* __restrict__ rows,
                                                                 const int* __restrict__ cols, double* values9,
                                                                 const int* __restrict__ bd_type, int n_vertices,
                                                                 int offset, int* bad)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int warp_first = i & ~31;
  if (warp_first >= n) return;
  bool clear = false;
  if (i < n) {
    const int a = rows[i] - offset, b = cols[i] - offset;
    if (a < 0 || b < 0 || a >= n_vertices || b >= n_vertices)
      atomicExch(bad, 1);
    else
      clear = bd_type[a] != 0 || bd_type[b] != 0;
  }
  clear_flagged(values9, warp_first, n, clear);
}

// Triplet t of a sub-range: the source triplet idx[t] (t itself without an
// index list) with both indices moved down by `offset`.  An index past the
// source gives the row -1, which the matrix build reports as out of range.
// Without rows_out only the values are gathered.
__global__ void __launch_bounds__(kContactTpb) k_gather_triplets(int n, const unsigned* __restrict__ idx,
                                                                   const int* __restrict__ rows,
                                                                   const int* __restrict__ cols,
                                                                   const double* __restrict__ vals9,
                                                                   long long source, int offset, int* rows_out,
                                                                   int* cols_out, double* vals_out)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const long long t = idx ? (long long)idx[i] : (long long)i;
  if (t >= source) {
    if (rows_out) rows_out[i] = cols_out[i] = -1;
    return;
  }
  if (rows_out) {
    rows_out[i] = rows[t] - offset;
    cols_out[i] = cols[t] - offset;
  }
#pragma unroll
  for (int e = 0; e < 9; ++e) vals_out[9 * (size_t)i + e] = vals9[9 * (size_t)t + e];
}

}  // namespace

bool adjust_contacts(maspcg_handle* h, int n, int* rows, int* cols, double* values9, const int* bd_type,
                     int n_vertices, int offset, bool zero_boundary_only)
{
  h->asm_flags.resize(4);
  int* bad = h->asm_flags.get();
  MCK(cudaMemsetAsync(bad, 0, sizeof(int), h->stream));
  const int grid = ceil_div(n, kContactTpb);
  if (zero_boundary_only)
    k_zero_boundary<<<grid, kContactTpb, 0, h->stream>>>(n, rows, cols, values9, bd_type, n_vertices, offset, bad);
  else
    k_adjust_contacts<<<grid, kContactTpb, 0, h->stream>>>(n, rows, cols, values9, bd_type, n_vertices, offset, bad);
  MLAUNCHED(h);
  MCK(cudaGetLastError());
  int flag = 0;
  MCK(cudaMemcpyAsync(&flag, bad, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  MCK(cudaStreamSynchronize(h->stream));
  return flag == 0;
}

void gather_triplets(maspcg_handle* h, int n, const unsigned* idx, const int* rows, const int* cols,
                     const double* vals9, long long source, int offset, int* rows_out, int* cols_out,
                     double* vals_out)
{
  k_gather_triplets<<<ceil_div(n, kContactTpb), kContactTpb, 0, h->stream>>>(n, idx, rows, cols, vals9, source, offset,
                                                                             rows_out, cols_out, vals_out);
  MLAUNCHED(h);
  MCK(cudaGetLastError());
}

}  // namespace maspcg
