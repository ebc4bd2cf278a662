// matrix.cu -- assembled BCOO -> internal full BCSR, FP64 SpMV, permutations,
// block-Jacobi (3x3) and affine-body (12x12) inverses.
//
// The conversion follows Converter::convert (converter.cu:137-284): a stable
// radix sort on a (row,col) key and a segmented sum of equal keys, so the
// block structure is bit-exact and FP64 sums are taken in input order.  It
// differs in what it produces: both triangles (the symmetric SpMV of
// spmv.cu:28-53 scatters B^T with atomics; a row-owned BCSR needs none) and
// rows renumbered into the MAS partition order.
#include <algorithm>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "maspcg_internal.cuh"
#include "spmv_row.cuh"

namespace maspcg {
namespace {

constexpr int kTpb = 256;
constexpr unsigned long long kSentinel = ~0ull;

__global__ void k_make_keys(const int* __restrict__ rows, const int* __restrict__ cols, int n, int nb,
                            const int* __restrict__ int_of_row, int bits, unsigned long long* keys, int* vals,
                            int* bad)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int r = rows[i], c = cols[i];
  if (r < 0 || c < 0 || r >= nb || c >= nb) {
    atomicAdd(bad, 1);
    keys[2 * (size_t)i] = kSentinel;
    keys[2 * (size_t)i + 1] = kSentinel;
    return;
  }
  const unsigned long long ri = (unsigned)int_of_row[r], ci = (unsigned)int_of_row[c];
  keys[2 * (size_t)i] = (ri << bits) | ci;
  vals[2 * (size_t)i] = i << 1;  // A_rc = H
  if (r != c) {
    keys[2 * (size_t)i + 1] = (ci << bits) | ri;
    vals[2 * (size_t)i + 1] = (i << 1) | 1;  // A_cr = H^T
  } else {
    keys[2 * (size_t)i + 1] = kSentinel;
    vals[2 * (size_t)i + 1] = -1;
    atomicAdd(bad + 2, 1);
  }
}

__global__ void k_heads(const unsigned long long* __restrict__ keys, int m, int* head)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const unsigned long long k = keys[i];
  head[i] = (k != kSentinel && (i == 0 || k != keys[i - 1])) ? 1 : 0;
}

__global__ void k_fill_structure(const unsigned long long* __restrict__ keys, const int* __restrict__ head,
                                 const int* __restrict__ uidx, int m, int bits, int* colidx, int* seg_start,
                                 int* row_count)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  if (!head[i]) return;
  const unsigned long long k = keys[i];
  const int u = uidx[i];
  const int row = (int)(k >> bits);
  colidx[u] = (int)(k & ((1ull << bits) - 1));
  seg_start[u] = i;
  atomicAdd(row_count + row, 1);
}

// One thread per stored block: sum its input blocks in sorted (= input) order.
__global__ void k_fill_values(const unsigned long long* __restrict__ keys, const int* __restrict__ vals_sorted,
                              const int* __restrict__ seg_start, int nnzb, int m_valid,
                              const double* __restrict__ in_vals, double* val64, float* val32,
                              unsigned short* val_lo)
{
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= nnzb) return;
  const int s = seg_start[u];
  const int e = (u + 1 < nnzb) ? seg_start[u + 1] : m_valid;
  double a[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int i = s; i < e; ++i) {
    const int v = vals_sorted[i];
    const double* H = in_vals + 9 * (size_t)(v >> 1);  // Eigen column-major
    if (v & 1) {
      // transpose: (r,c) of A_cr = H(c,r) = H[c + 3r]
#pragma unroll
      for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) a[3 * r + c] += H[c + 3 * r];
    } else {
#pragma unroll
      for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) a[3 * r + c] += H[r + 3 * c];
    }
  }
#pragma unroll
  for (int q = 0; q < 9; ++q) {
    val64[9 * (size_t)u + q] = a[q];
    const size_t at = (size_t)(u >> 5) * 288 + 32 * q + (u & 31);  // tiles of 32 blocks, element-major
    const float hi = (float)a[q];
    val32[at] = hi;
    // the remainder a - hi is exact in FP64; its BF16 rounding carries A to
    // about 2^-32 relative
    if (val_lo) val_lo[at] = __bfloat16_as_ushort(__float2bfloat16_rn((float)(a[q] - (double)hi)));
  }
}

// y = a*A*x + b*y, FP64, half-warp per block row.
__global__ void k_spmv64(const int* __restrict__ rowptr, const int* __restrict__ colidx, const double* __restrict__ val,
                         const double* __restrict__ x, double* y, double a, double b, int nrows)
{
  constexpr int LPR = 16;
  const int gl = blockIdx.x * blockDim.x + threadIdx.x;
  const int row = gl / LPR, sub = gl % LPR;
  const bool ok = row < nrows;
  const int rs = ok ? rowptr[row] : 0, re = ok ? rowptr[row + 1] : 0;
  double acc[3];
  row_product<double, double, LPR>(rs, re, colidx, val, x, sub, acc);
  if (ok && sub < 3) {
    const double prev = (b != 0.0) ? b * y[3 * (size_t)row + sub] : 0.0;
    y[3 * (size_t)row + sub] = a * acc[sub] + prev;
  }
}

__global__ void k_permute_in(const double* __restrict__ src, double* dst, const int* __restrict__ row_of_int, int nb_int)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 3 * nb_int) return;
  const int r = row_of_int[i / 3];
  dst[i] = r >= 0 ? src[3 * (size_t)r + i % 3] : 0.0;
}

__global__ void k_permute_out(const double* __restrict__ src, double* dst, const int* __restrict__ int_of_row, int nb)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 3 * nb) return;
  dst[i] = src[3 * (size_t)int_of_row[i / 3] + i % 3];
}

// DiagPreconditioner (diag_preconditioner.cu:10-39): 3x3 inverse of the
// diagonal block, identity where it is missing.
__global__ void k_diag3(const int* __restrict__ rowptr, const int* __restrict__ colidx, const double* __restrict__ val,
                        int nrows, double* inv64, float* inv32)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nrows) return;
  int lo = rowptr[i], hi = rowptr[i + 1] - 1, t = -1;
  while (lo <= hi) {
    const int mid = (lo + hi) >> 1;
    const int c = colidx[mid];
    if (c == i) {
      t = mid;
      break;
    }
    if (c < i)
      lo = mid + 1;
    else
      hi = mid - 1;
  }
  double o[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  if (t >= 0) {
    const double* m = val + 9 * (size_t)t;  // row-major
    const double a = m[0], b = m[1], c = m[2], d = m[3], e = m[4], f = m[5], g = m[6], hh = m[7], k = m[8];
    const double A = e * k - f * hh, B = -(d * k - f * g), C = d * hh - e * g;
    const double det = a * A + b * B + c * C;
    const double id = 1.0 / det;
    o[0] = A * id;
    o[1] = -(b * k - c * hh) * id;
    o[2] = (b * f - c * e) * id;
    o[3] = B * id;
    o[4] = (a * k - c * g) * id;
    o[5] = -(a * f - c * d) * id;
    o[6] = C * id;
    o[7] = -(a * hh - b * g) * id;
    o[8] = (a * e - b * d) * id;
  }
  for (int q = 0; q < 9; ++q) {
    inv64[9 * (size_t)i + q] = o[q];
    inv32[9 * (size_t)i + q] = (float)o[q];
  }
}

// ABDPreconditioner (setup_abd_system_gradient_and_hessian.cu:407-441): gather
// the body's 12x12 diagonal block from the blocks with row/4 == col/4 and
// invert it (Gauss-Jordan, partial pivoting), row-major.
__global__ void k_abd_inverse(const int* __restrict__ rowptr, const int* __restrict__ colidx,
                              const double* __restrict__ val, int bodies, double* inv64, float* inv32, int* failed)
{
  const int bdy = blockIdx.x * blockDim.x + threadIdx.x;
  if (bdy >= bodies) return;
  double a[12][24];
  for (int r = 0; r < 12; ++r)
    for (int c = 0; c < 24; ++c) a[r][c] = (c - 12 == r) ? 1.0 : 0.0;
  for (int q = 0; q < 4; ++q) {
    const int row = 4 * bdy + q;
    for (int t = rowptr[row]; t < rowptr[row + 1]; ++t) {
      const int c = colidx[t];
      if (c / 4 != bdy) continue;
      const double* m = val + 9 * (size_t)t;
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) a[3 * q + i][3 * (c % 4) + j] = m[3 * i + j];
    }
  }
  bool ok = true;
  for (int k = 0; k < 12; ++k) {
    int piv = k;
    for (int r = k + 1; r < 12; ++r)
      if (fabs(a[r][k]) > fabs(a[piv][k])) piv = r;
    if (a[piv][k] == 0.0) {
      ok = false;
      break;
    }
    if (piv != k)
      for (int c = 0; c < 24; ++c) {
        const double t = a[k][c];
        a[k][c] = a[piv][c];
        a[piv][c] = t;
      }
    const double inv = 1.0 / a[k][k];
    for (int c = 0; c < 24; ++c) a[k][c] *= inv;
    for (int r = 0; r < 12; ++r) {
      if (r == k) continue;
      const double f = a[r][k];
      if (f == 0.0) continue;
      for (int c = 0; c < 24; ++c) a[r][c] -= f * a[k][c];
    }
  }
  if (!ok) atomicAdd(failed, 1);
  for (int r = 0; r < 12; ++r)
    for (int c = 0; c < 12; ++c) {
      const double v = ok ? a[r][c + 12] : (r == c ? 1.0 : 0.0);
      inv64[144 * (size_t)bdy + 12 * r + c] = v;
      inv32[144 * (size_t)bdy + 12 * r + c] = (float)v;
    }
}

size_t cub_bytes_sort(int m, int end_bit)
{
  size_t b = 0;
  MCK(cub::DeviceRadixSort::SortPairs(nullptr, b, (const unsigned long long*)nullptr, (unsigned long long*)nullptr,
                                      (const int*)nullptr, (int*)nullptr, m, 0, end_bit));
  return b;
}

}  // namespace

void build_internal_matrix(maspcg_handle* h, const double* vals, const int* rows, const int* cols, int n)
{
  cudaStream_t st = h->stream;
  const int nb = h->nb;
  // ---- internal row order
  std::vector<int> iof(nb);
  h->mas_layout = (h->cfg.preconditioner == MASPCG_PRECOND_MAS32 || h->cfg.preconditioner == MASPCG_PRECOND_MAS16) &&
                  h->has_graph && h->nv > 0;
  int nb_int = nb;
  if (h->mas_layout) {
    MREQ(h->fem_off + h->nv <= nb, MASPCG_ERR_INVALID_ARGUMENT, "FEM range exceeds the block rows");
    const int shift = h->c0 - h->nv;
    for (int r = 0; r < nb; ++r) {
      if (r < h->fem_off)
        iof[r] = r;
      else if (r < h->fem_off + h->nv)
        iof[r] = h->fem_off + h->h_rmp[r - h->fem_off];
      else
        iof[r] = r + shift;
    }
    nb_int = nb + shift;
  } else {
    for (int r = 0; r < nb; ++r) iof[r] = r;
  }
  std::vector<int> roi(nb_int, -1);
  for (int r = 0; r < nb; ++r) roi[iof[r]] = r;
  h->nb_int = nb_int;
  h->int_of_row.resize(nb);
  h->row_of_int.resize(nb_int);
  MCK(cudaMemcpyAsync(h->int_of_row.get(), iof.data(), sizeof(int) * nb, cudaMemcpyHostToDevice, st));
  MCK(cudaMemcpyAsync(h->row_of_int.get(), roi.data(), sizeof(int) * nb_int, cudaMemcpyHostToDevice, st));

  // ---- keys
  int bits = 1;
  while ((1ll << bits) <= nb_int) ++bits;
  MREQ(2 * bits <= 62, MASPCG_ERR_CAPACITY, "too many block rows");
  const int m = 2 * n;
  h->keys.resize(m);
  h->keys_sorted.resize(m);
  h->kv.resize(m);
  h->kv_sorted.resize(m);
  h->seg_head.resize(m);
  h->seg_start.resize(m + 1);
  h->failed.resize(8);
  MCK(cudaMemsetAsync(h->failed.get(), 0, sizeof(int) * 8, st));
  k_make_keys<<<ceil_div(n, kTpb), kTpb, 0, st>>>(rows, cols, n, nb, h->int_of_row.get(), bits, h->keys.get(),
                                                 h->kv.get(), h->failed.get()); MLAUNCHED(h);
  // keys use 2*bits bits; the all-ones sentinel still sorts last on 2*bits+1
  const int end_bit = 2 * bits + 1;
  size_t need = cub_bytes_sort(m, end_bit);
  size_t scan_b = 0;
  MCK(cub::DeviceScan::ExclusiveSum(nullptr, scan_b, (const int*)nullptr, (int*)nullptr, m));
  need = std::max(need, scan_b);
  h->cub_tmp.resize(need);
  size_t tb = h->cub_tmp.cap;
  MCK(cub::DeviceRadixSort::SortPairs(h->cub_tmp.get(), tb, h->keys.get(), h->keys_sorted.get(), h->kv.get(),
                                      h->kv_sorted.get(), m, 0, end_bit, st));
  k_heads<<<ceil_div(m, kTpb), kTpb, 0, st>>>(h->keys_sorted.get(), m, h->seg_head.get()); MLAUNCHED(h);
  // unique index = exclusive scan of heads (reuse kv as output)
  tb = h->cub_tmp.cap;
  MCK(cub::DeviceScan::ExclusiveSum(h->cub_tmp.get(), tb, h->seg_head.get(), h->kv.get(), m, st));
  int tail[2] = {0, 0}, flags[3] = {0, 0, 0};
  MCK(cudaMemcpyAsync(&tail[0], h->kv.get() + (m - 1), sizeof(int), cudaMemcpyDeviceToHost, st));
  MCK(cudaMemcpyAsync(&tail[1], h->seg_head.get() + (m - 1), sizeof(int), cudaMemcpyDeviceToHost, st));
  MCK(cudaMemcpyAsync(flags, h->failed.get(), 3 * sizeof(int), cudaMemcpyDeviceToHost, st));
  MCK(cudaStreamSynchronize(st));
  MREQ(flags[0] == 0, MASPCG_ERR_INVALID_ARGUMENT, "matrix block index out of range");
  const int nnzb = tail[0] + tail[1];
  const int m_valid = m - flags[2];  // sentinels (one per diagonal input block) sort last
  h->m_valid = m_valid;
  h->nnzb = nnzb;
  h->colidx.resize(nnzb, 4);  // 16-byte tail for TMA bulk copies
  h->val64.resize((size_t)9 * nnzb, 2);
  h->val32.resize((size_t)9 * (((size_t)nnzb + 31) / 32 * 32));
  if (h->cfg.matrix_form == MASPCG_MATRIX_F32_SPLIT) h->val_lo.resize(h->val32.n);
  h->row_count.resize(nb_int + 1);
  h->rowptr.resize(nb_int + 1);
  MCK(cudaMemsetAsync(h->row_count.get(), 0, sizeof(int) * (nb_int + 1), st));
  k_fill_structure<<<ceil_div(m, kTpb), kTpb, 0, st>>>(h->keys_sorted.get(), h->seg_head.get(), h->kv.get(), m, bits,
                                                      h->colidx.get(), h->seg_start.get(), h->row_count.get()); MLAUNCHED(h);
  // rowptr = exclusive scan of the per-row counts (the extra entry gives nnzb)
  tb = h->cub_tmp.cap;
  MCK(cub::DeviceScan::ExclusiveSum(h->cub_tmp.get(), tb, h->row_count.get(), h->rowptr.get(), nb_int + 1, st));
  if (h->vals_pending) {  // host values copied on the side stream
    MCK(cudaStreamWaitEvent(st, h->ev_join, 0));
    h->vals_pending = false;
  }
  k_fill_values<<<ceil_div(nnzb, kTpb), kTpb, 0, st>>>(h->keys_sorted.get(), h->kv_sorted.get(), h->seg_start.get(),
                                                      nnzb, m_valid, vals, h->val64.get(), h->val32.get(),
                                                      h->cfg.matrix_form == MASPCG_MATRIX_F32_SPLIT ? h->val_lo.get()
                                                                                                    : nullptr);
  MLAUNCHED(h);
  MCK(cudaGetLastError());
}

void refresh_internal_values(maspcg_handle* h, const double* vals)
{
  cudaStream_t st = h->stream;
  if (h->vals_pending) {  // host values copied on the side stream
    MCK(cudaStreamWaitEvent(st, h->ev_join, 0));
    h->vals_pending = false;
  }
  k_fill_values<<<ceil_div(h->nnzb, kTpb), kTpb, 0, st>>>(h->keys_sorted.get(), h->kv_sorted.get(),
                                                          h->seg_start.get(), h->nnzb, h->m_valid, vals,
                                                          h->val64.get(), h->val32.get(),
                                                          h->cfg.matrix_form == MASPCG_MATRIX_F32_SPLIT
                                                              ? h->val_lo.get()
                                                              : nullptr);
  MLAUNCHED(h);
  MCK(cudaGetLastError());
}

void launch_spmv64(maspcg_handle* h, const double* x, double* y, double a, double b)
{
  const long long threads = (long long)h->nb_int * 16;
  k_spmv64<<<ceil_div(threads, kTpb), kTpb, 0, h->stream>>>(h->rowptr.get(), h->colidx.get(), h->val64.get(), x, y, a,
                                                           b, h->nb_int); MLAUNCHED(h);
  MCK(cudaGetLastError());
}

void permute_in(maspcg_handle* h, const double* src, double* dst)
{
  k_permute_in<<<ceil_div(3LL * h->nb_int, kTpb), kTpb, 0, h->stream>>>(src, dst, h->row_of_int.get(), h->nb_int); MLAUNCHED(h);
  MCK(cudaGetLastError());
}

void permute_out(maspcg_handle* h, const double* src, double* dst)
{
  k_permute_out<<<ceil_div(3LL * h->nb, kTpb), kTpb, 0, h->stream>>>(src, dst, h->int_of_row.get(), h->nb); MLAUNCHED(h);
  MCK(cudaGetLastError());
}

void build_block_jacobi(maspcg_handle* h)
{
  cudaStream_t st = h->stream;
  if (h->cfg.preconditioner == MASPCG_PRECOND_BLOCK_JACOBI) {
    h->diag_inv64.resize((size_t)9 * h->nb_int);
    h->diag_inv32.resize((size_t)9 * h->nb_int);
    k_diag3<<<ceil_div(h->nb_int, kTpb), kTpb, 0, st>>>(h->rowptr.get(), h->colidx.get(), h->val64.get(), h->nb_int,
                                                       h->diag_inv64.get(), h->diag_inv32.get()); MLAUNCHED(h);
  }
  if (h->abd_bodies > 0 && h->cfg.preconditioner != MASPCG_PRECOND_NONE) {
    h->abd_inv64.resize((size_t)144 * h->abd_bodies);
    h->abd_inv32.resize((size_t)144 * h->abd_bodies);
    k_abd_inverse<<<ceil_div(h->abd_bodies, 64), 64, 0, st>>>(h->rowptr.get(), h->colidx.get(), h->val64.get(),
                                                            h->abd_bodies, h->abd_inv64.get(), h->abd_inv32.get(),
                                                            h->failed.get() + 1); MLAUNCHED(h);
  }
  MCK(cudaGetLastError());
}

}  // namespace maspcg
