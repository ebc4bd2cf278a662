// galerkin.cu -- the AGIPC coarse system on the device (StiffGIPC/agipc/
// agipc_galerkin.cu): A_c = P^T A P and b_c = P^T b for the mixed
// prolongation P of the coarse mapping, and x = P x_c back.
//
// The mapping (agipc_criterion.cuh:13-25, transform_for_block at
// agipc_galerkin.cu:200-219): fine blocks [0, prefix) pass through unchanged
// (coarse block = fine block); fine FEM node k = block prefix + k belongs to
// coarse node fine_to_coarse[k], whose blocks start at prefix +
// coarse_block_bases[c] and whose basis is the subset `basis_masks[c]` of
// (1, x, y, z) at the node's rest position: a translational node keeps 1, an
// affine node all four.  A fine block (i, j) therefore expands into
// width_i x width_j coarse blocks phi_i[a] phi_j[b] A_ij (count_expanded_blocks
// and emit_expanded_blocks, :221-283): a diagonal fine block keeps a <= b; an
// off-diagonal one that lands on a coarse diagonal block adds its transpose;
// one that lands below the diagonal is transposed to (col, row).  The
// expanded triplets are then merged like any triplet list (assemble.cu).
#include <cub/device/device_scan.cuh>

#include "maspcg_internal.cuh"

namespace maspcg {

namespace {

constexpr int kGalTpb = 256;

__device__ __forceinline__ void transform_block(const GalerkinMap& m, int block, int& base, int& width, double phi[4])
{
  phi[0] = 1.0;
  phi[1] = phi[2] = phi[3] = 0.0;
  if (block < m.prefix) {
    base = block;
    width = 1;
    return;
  }
  const int k = block - m.prefix;
  const int c = m.fine_to_coarse[k];
  base = m.prefix + m.coarse_block_bases[c];
  const int mask = m.basis_masks[c];
  width = __popc((unsigned)mask & 15u);
  const double raw[4] = {1.0, m.rest[3 * (size_t)k], m.rest[3 * (size_t)k + 1], m.rest[3 * (size_t)k + 2]};
  int o = 0;
#pragma unroll
  for (int q = 0; q < 4; ++q)
    if (mask & (1 << q)) phi[o++] = raw[q];
}

__global__ void k_gal_count(GalerkinMap m, const int* __restrict__ rows, const int* __restrict__ cols, int n,
                            int* counts, int* bad)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int r = rows[i], c = cols[i];
  if (r < 0 || c < 0 || r >= m.fine_blocks || c >= m.fine_blocks) {
    atomicExch(bad, 1);
    counts[i] = 0;
    return;
  }
  int rb, rw, cb, cw;
  double rp[4], cp[4];
  transform_block(m, r, rb, rw, rp);
  transform_block(m, c, cb, cw, cp);
  counts[i] = r == c ? rw * (rw + 1) / 2 : rw * cw;
}

// values Eigen column-major: element (row i, col j) at i + 3j
__global__ void k_gal_emit(GalerkinMap m, const double* __restrict__ vals, const int* __restrict__ rows,
                           const int* __restrict__ cols, const int* __restrict__ offsets, int n, double* out_vals,
                           int* out_rows, int* out_cols, int* bad)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int r = rows[i], c = cols[i];
  if (r < 0 || c < 0 || r >= m.fine_blocks || c >= m.fine_blocks) return;
  int rb, rw, cb, cw;
  double rp[4], cp[4];
  transform_block(m, r, rb, rw, rp);
  transform_block(m, c, cb, cw, cp);
  double in[9];
#pragma unroll
  for (int e = 0; e < 9; ++e) in[e] = vals[9 * (size_t)i + e];
  int o = offsets[i];
  for (int a = 0; a < rw; ++a)
    for (int b = 0; b < cw; ++b) {
      if (r == c && a > b) continue;
      int mr = rb + a, mc = cb + b;
      const double w = rp[a] * cp[b];
      double v[9];
#pragma unroll
      for (int e = 0; e < 9; ++e) v[e] = w * in[e];
      if (r != c && mr == mc) {
        double t[9];
#pragma unroll
        for (int ii = 0; ii < 3; ++ii)
#pragma unroll
          for (int jj = 0; jj < 3; ++jj) t[ii + 3 * jj] = v[ii + 3 * jj] + v[jj + 3 * ii];
#pragma unroll
        for (int e = 0; e < 9; ++e) v[e] = t[e];
      } else if (mr > mc) {
        const int s = mr;
        mr = mc;
        mc = s;
        double t[9];
#pragma unroll
        for (int ii = 0; ii < 3; ++ii)
#pragma unroll
          for (int jj = 0; jj < 3; ++jj) t[ii + 3 * jj] = v[jj + 3 * ii];
#pragma unroll
        for (int e = 0; e < 9; ++e) v[e] = t[e];
      }
      out_rows[o] = mr;
      out_cols[o] = mc;
#pragma unroll
      for (int e = 0; e < 9; ++e) {
        out_vals[9 * (size_t)o + e] = v[e];
        if (!isfinite(v[e])) atomicExch(bad, 2);
      }
      ++o;
    }
}

// b_c = P^T b (FP64 atomics, as reduce_mixed_rhs at agipc_galerkin.cu:285-306)
__global__ void k_gal_restrict(GalerkinMap m, const double* __restrict__ fine, double* coarse, int* bad)
{
  const int block = blockIdx.x * blockDim.x + threadIdx.x;
  if (block >= m.fine_blocks) return;
  int base, width;
  double phi[4];
  transform_block(m, block, base, width, phi);
  for (int comp = 0; comp < 3; ++comp) {
    const double v = fine[3 * (size_t)block + comp];
    if (!isfinite(v)) {
      atomicExch(bad, 2);
      continue;
    }
    for (int a = 0; a < width; ++a) atomicAdd(coarse + 3 * (size_t)(base + a) + comp, phi[a] * v);
  }
}

// x = P x_c (prolongate_mixed, agipc_galerkin.cu:355-369)
__global__ void k_gal_prolong(GalerkinMap m, const double* __restrict__ coarse, double* fine)
{
  const int block = blockIdx.x * blockDim.x + threadIdx.x;
  if (block >= m.fine_blocks) return;
  int base, width;
  double phi[4];
  transform_block(m, block, base, width, phi);
  for (int comp = 0; comp < 3; ++comp) {
    double v = 0.0;
    for (int a = 0; a < width; ++a) v += phi[a] * coarse[3 * (size_t)(base + a) + comp];
    fine[3 * (size_t)block + comp] = v;
  }
}

int read_int(maspcg_handle* h, const int* d)
{
  int v = 0;
  MCK(cudaMemcpyAsync(&v, d, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  MCK(cudaStreamSynchronize(h->stream));
  return v;
}

}  // namespace

// Expanded (unmerged) coarse triplets into the handle's scratch; returns
// their count and points *v, *r, *c at them.
int galerkin_expand(maspcg_handle* h, const GalerkinMap& m, const double* vals, const int* rows, const int* cols,
                    int n, const double** v, const int** r, const int** c)
{
  cudaStream_t st = h->stream;
  h->gal_counts.resize(2 * (size_t)n + 2);
  int* counts = h->gal_counts.get();
  int* offsets = counts + n;
  int* bad = offsets + n;
  MCK(cudaMemsetAsync(bad, 0, sizeof(int), st));
  const int grid = ceil_div(n, kGalTpb);
  k_gal_count<<<grid, kGalTpb, 0, st>>>(m, rows, cols, n, counts, bad); MLAUNCHED(h);
  size_t need = 0;
  MCK(cub::DeviceScan::ExclusiveSum(nullptr, need, counts, offsets, n, st));
  h->cub_tmp.resize(std::max(need, h->cub_tmp.n));
  size_t tb = h->cub_tmp.cap;
  MCK(cub::DeviceScan::ExclusiveSum(h->cub_tmp.get(), tb, counts, offsets, n, st));
  MREQ(read_int(h, bad) == 0, MASPCG_ERR_INVALID_ARGUMENT, "fine block index outside [0, fine_blocks)");
  int last[2] = {0, 0};
  MCK(cudaMemcpyAsync(&last[0], offsets + (n - 1), sizeof(int), cudaMemcpyDeviceToHost, st));
  MCK(cudaMemcpyAsync(&last[1], counts + (n - 1), sizeof(int), cudaMemcpyDeviceToHost, st));
  MCK(cudaStreamSynchronize(st));
  const long long expanded = (long long)last[0] + last[1];
  MREQ(expanded <= 0x3fffffffLL, MASPCG_ERR_CAPACITY, "expanded coarse triplets exceed 2^30");
  h->gal_vals.resize(9 * (size_t)std::max(expanded, 1LL));
  h->gal_rows.resize((size_t)std::max(expanded, 1LL));
  h->gal_cols.resize((size_t)std::max(expanded, 1LL));
  k_gal_emit<<<grid, kGalTpb, 0, st>>>(m, vals, rows, cols, offsets, n, h->gal_vals.get(), h->gal_rows.get(),
                                       h->gal_cols.get(), bad); MLAUNCHED(h);
  MREQ(read_int(h, bad) == 0, MASPCG_ERR_INVALID_ARGUMENT, "non-finite coarse matrix entry");
  *v = h->gal_vals.get();
  *r = h->gal_rows.get();
  *c = h->gal_cols.get();
  return (int)expanded;
}

void galerkin_restrict(maspcg_handle* h, const GalerkinMap& m, const double* fine, double* coarse, int coarse_blocks)
{
  cudaStream_t st = h->stream;
  h->gal_counts.resize(std::max<size_t>(h->gal_counts.n, 1));
  int* bad = h->gal_counts.get();
  MCK(cudaMemsetAsync(bad, 0, sizeof(int), st));
  MCK(cudaMemsetAsync(coarse, 0, sizeof(double) * 3 * (size_t)coarse_blocks, st));
  if (m.fine_blocks > 0) {
    k_gal_restrict<<<ceil_div(m.fine_blocks, kGalTpb), kGalTpb, 0, st>>>(m, fine, coarse, bad); MLAUNCHED(h);
  }
  MREQ(read_int(h, bad) == 0, MASPCG_ERR_INVALID_ARGUMENT, "non-finite fine right-hand side");
}

void galerkin_prolong(maspcg_handle* h, const GalerkinMap& m, const double* coarse, double* fine)
{
  if (m.fine_blocks <= 0) return;
  k_gal_prolong<<<ceil_div(m.fine_blocks, kGalTpb), kGalTpb, 0, h->stream>>>(m, coarse, fine); MLAUNCHED(h);
  MCK(cudaGetLastError());
}

}  // namespace maspcg
