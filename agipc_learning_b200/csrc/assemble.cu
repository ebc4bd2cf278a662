// assemble.cu -- the two triplet steps in front of the solve, on the device:
//
// * convert_bcoo: Converter::convert (StiffGIPC/linear_system/utils/
//   converter.cu:137-284).  Triplets keyed (row << 32) + col (packed into as
//   few bits as the indices need: the same order) are radix-sorted (stable), runs of equal keys are found with head flags and an exclusive
//   scan, and each run's 3x3 blocks are summed.  The reference sums a run with
//   a warp head-segmented reduction plus FP64 atomics, whose order varies;
//   here one thread sums its run in the stable sort order, so the result is
//   deterministic (and equal to a sequential sum in input order within each
//   key).
// * partition_contacts: GIPC::partitionContactHessian (StiffGIPC/GIPC.cu:
//   9952-10128 with _partition_collision_triplets and _reorder_triplets at
//   :218-283).  Contact triplets carry a type hash (0 FEM-FEM, 1 ABD-FEM,
//   2 FEM-ABD, 3 ABD-ABD); a stable radix sort on it groups them by type
//   in that order, and the per-type counts come back with the reordered
//   triplets.
//
// Both are integer, bit-exact work apart from the FP64 sums.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "maspcg_internal.cuh"

namespace maspcg {
namespace {

constexpr int kAsmTpb = 256;

// Largest row and column index (for the key width), and a flag for
// negative indices.
__global__ void k_conv_range(const int* __restrict__ rows, const int* __restrict__ cols, int n, int* flags)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  int r = -1, c = -1;
  if (i < n) {
    r = rows[i];
    c = cols[i];
    if (r < 0 || c < 0) atomicExch(flags, 1);
  }
  r = __reduce_max_sync(0xffffffffu, (unsigned)max(r, 0));
  c = __reduce_max_sync(0xffffffffu, (unsigned)max(c, 0));
  if ((threadIdx.x & 31) == 0) {
    atomicMax(flags + 1, r);
    atomicMax(flags + 2, c);
  }
}

// Key (row << col_bits) + col: the order of (row << 32) + col in as few bits
// as the indices need, so the radix sort runs only the passes it must.
__global__ void k_conv_keys(const int* __restrict__ rows, const int* __restrict__ cols, int n, int col_bits,
                            unsigned long long* keys, int* idx)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  keys[i] = ((unsigned long long)(unsigned)rows[i] << col_bits) + (unsigned long long)(unsigned)cols[i];
  idx[i] = i;
}

__global__ void k_conv_heads(const unsigned long long* __restrict__ keys, int n, int* heads)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) heads[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1 : 0;
}

// start[u] = first sorted position of unique key u; start[count] = n
__global__ void k_conv_starts(const int* __restrict__ heads, const int* __restrict__ pos, int n, int* start)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && heads[i]) start[pos[i]] = i;
  if (i == n - 1) start[pos[i] + heads[i]] = n;
}

// One thread per unique key: its row and column, and the sum of its run's
// blocks in sorted (stable) order.
__global__ void k_conv_sum(const unsigned long long* __restrict__ keys, const int* __restrict__ perm,
                           const int* __restrict__ start, int count, int col_bits, const double* __restrict__ vals,
                           int* rows_out, int* cols_out, double* vals_out)
{
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= count) return;
  const int s = start[u], e = start[u + 1];
  const unsigned long long k = keys[s];
  rows_out[u] = (int)(k >> col_bits);
  cols_out[u] = (int)(k & ((1ull << col_bits) - 1ull));
  double a[9];
#pragma unroll
  for (int q = 0; q < 9; ++q) a[q] = 0.0;
  for (int t = s; t < e; ++t) {
    const double* v = vals + 9 * (size_t)perm[t];
#pragma unroll
    for (int q = 0; q < 9; ++q) a[q] = a[q] + v[q];
  }
#pragma unroll
  for (int q = 0; q < 9; ++q) vals_out[9 * (size_t)u + q] = a[q];
}

__global__ void k_part_keys(const unsigned long long* __restrict__ types, int n, unsigned* keys, int* idx, int* bad,
                            int* counts)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const unsigned long long t = types[i];
  if (t > 3ull) atomicExch(bad, 1);
  const unsigned k = (unsigned)(t & 3ull);
  keys[i] = k;
  idx[i] = i;
  atomicAdd(counts + k, 1);
}

__global__ void k_gather_triplets(const int* __restrict__ perm, int n, const int* __restrict__ rows,
                                  const int* __restrict__ cols, const double* __restrict__ vals, int* rows_out,
                                  int* cols_out, double* vals_out)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int p = perm[i];
  rows_out[i] = rows[p];
  cols_out[i] = cols[p];
#pragma unroll
  for (int q = 0; q < 9; ++q) vals_out[9 * (size_t)i + q] = vals[9 * (size_t)p + q];
}

}  // namespace

int convert_bcoo(maspcg_handle* h, const int* rows, const int* cols, const double* vals, int n, int* rows_out,
                 int* cols_out, double* vals_out)
{
  if (n <= 0) return 0;
  cudaStream_t st = h->stream;
  h->asm_keys.resize(2 * (size_t)n);
  h->asm_idx.resize(2 * (size_t)n);
  h->asm_flags.resize(2 * (size_t)n + 4);
  unsigned long long* k0 = h->asm_keys.get();
  unsigned long long* k1 = k0 + n;
  int* i0 = h->asm_idx.get();
  int* i1 = i0 + n;
  int* heads = h->asm_flags.get();
  int* pos = heads + n;
  int* flags = pos + n;  // negative index, max row, max col
  MCK(cudaMemsetAsync(flags, 0, 3 * sizeof(int), st));
  const int grid = ceil_div(n, kAsmTpb);
  k_conv_range<<<grid, kAsmTpb, 0, st>>>(rows, cols, n, flags); MLAUNCHED(h);
  int fl[3] = {0, 0, 0};
  MCK(cudaMemcpyAsync(fl, flags, 3 * sizeof(int), cudaMemcpyDeviceToHost, st));
  MCK(cudaStreamSynchronize(st));
  MREQ(fl[0] == 0, MASPCG_ERR_INVALID_ARGUMENT, "negative row or column index");
  auto bits = [](unsigned v) {
    int b = 1;
    while (b < 32 && (v >> b) != 0u) ++b;
    return b;
  };
  const int col_bits = bits((unsigned)fl[2]), key_bits = col_bits + bits((unsigned)fl[1]);
  k_conv_keys<<<grid, kAsmTpb, 0, st>>>(rows, cols, n, col_bits, k0, i0); MLAUNCHED(h);
  size_t need = 0;
  MCK(cub::DeviceRadixSort::SortPairs(nullptr, need, k0, k1, i0, i1, n, 0, key_bits, st));
  size_t need2 = 0;
  MCK(cub::DeviceScan::ExclusiveSum(nullptr, need2, heads, pos, n, st));
  h->cub_tmp.resize(std::max(std::max(need, need2), h->cub_tmp.n));
  size_t tb = h->cub_tmp.cap;
  MCK(cub::DeviceRadixSort::SortPairs(h->cub_tmp.get(), tb, k0, k1, i0, i1, n, 0, key_bits, st));
  k_conv_heads<<<grid, kAsmTpb, 0, st>>>(k1, n, heads); MLAUNCHED(h);
  tb = h->cub_tmp.cap;
  MCK(cub::DeviceScan::ExclusiveSum(h->cub_tmp.get(), tb, heads, pos, n, st));
  int last[2] = {0, 0};
  MCK(cudaMemcpyAsync(&last[0], pos + (n - 1), sizeof(int), cudaMemcpyDeviceToHost, st));
  MCK(cudaMemcpyAsync(&last[1], heads + (n - 1), sizeof(int), cudaMemcpyDeviceToHost, st));
  MCK(cudaStreamSynchronize(st));
  const int count = last[0] + last[1];
  h->asm_start.resize((size_t)count + 1);
  k_conv_starts<<<grid, kAsmTpb, 0, st>>>(heads, pos, n, h->asm_start.get()); MLAUNCHED(h);
  k_conv_sum<<<ceil_div(count, kAsmTpb), kAsmTpb, 0, st>>>(k1, i1, h->asm_start.get(), count, col_bits, vals,
                                                          rows_out, cols_out, vals_out); MLAUNCHED(h);
  MCK(cudaGetLastError());
  return count;
}

void partition_contacts(maspcg_handle* h, const int* rows, const int* cols, const double* vals,
                        const unsigned long long* types, int n, int* rows_out, int* cols_out, double* vals_out,
                        int counts[4])
{
  counts[0] = counts[1] = counts[2] = counts[3] = 0;
  if (n <= 0) return;
  cudaStream_t st = h->stream;
  h->asm_keys.resize((size_t)n);  // two 32-bit key arrays
  h->asm_idx.resize(2 * (size_t)n);
  h->asm_flags.resize(8);
  unsigned* k0 = reinterpret_cast<unsigned*>(h->asm_keys.get());
  unsigned* k1 = k0 + n;
  int* i0 = h->asm_idx.get();
  int* i1 = i0 + n;
  int* bad = h->asm_flags.get();
  int* dcount = bad + 1;
  MCK(cudaMemsetAsync(bad, 0, 5 * sizeof(int), st));
  const int grid = ceil_div(n, kAsmTpb);
  k_part_keys<<<grid, kAsmTpb, 0, st>>>(types, n, k0, i0, bad, dcount); MLAUNCHED(h);
  size_t need = 0;
  MCK(cub::DeviceRadixSort::SortPairs(nullptr, need, k0, k1, i0, i1, n, 0, 2, st));
  h->cub_tmp.resize(std::max(need, h->cub_tmp.n));
  size_t tb = h->cub_tmp.cap;
  MCK(cub::DeviceRadixSort::SortPairs(h->cub_tmp.get(), tb, k0, k1, i0, i1, n, 0, 2, st));
  int flags[5] = {0, 0, 0, 0, 0};
  MCK(cudaMemcpyAsync(flags, bad, 5 * sizeof(int), cudaMemcpyDeviceToHost, st));
  MCK(cudaStreamSynchronize(st));
  MREQ(flags[0] == 0, MASPCG_ERR_INVALID_ARGUMENT, "contact type hash outside 0..3");
  k_gather_triplets<<<grid, kAsmTpb, 0, st>>>(i1, n, rows, cols, vals, rows_out, cols_out, vals_out); MLAUNCHED(h);
  MCK(cudaGetLastError());
  for (int t = 0; t < 4; ++t) counts[t] = flags[1 + t];
}

}  // namespace maspcg
