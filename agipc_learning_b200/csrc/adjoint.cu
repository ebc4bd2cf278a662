// adjoint.cu -- the matrix adjoint of the differentiable Newton-step solve.
//
// For L(x) with x = A^-1 b and lam = A^-1 dL/dx (A is symmetric, so the
// adjoint solve reuses the same operator and preconditioner), dL/dA = -lam x^T.
// A is given as upper BCOO blocks (row <= col) where block (r, c) holds A_rc
// and stands for A_cr = A_rc^T as well, so the gradient of one input block is
//   r != c:  G = -(lam_r x_c^T + x_r lam_c^T)
//   r == c:  G = -lam_r x_r^T
// written column-major like the block values (element (i, j) at i + 3j).
// Repeated (r, c) entries each get the full G, as each one adds into A_rc.
#include "maspcg_internal.cuh"

namespace maspcg {
namespace {

constexpr int kAdjTpb = 256;

__global__ void __launch_bounds__(kAdjTpb) k_bcoo_gradient(const int* __restrict__ rows, const int* __restrict__ cols,
                                                          int n, const double* __restrict__ lam,
                                                          const double* __restrict__ x, double* grad)
{
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int r = rows[t], c = cols[t];
  const double lr[3] = {lam[3 * (size_t)r], lam[3 * (size_t)r + 1], lam[3 * (size_t)r + 2]};
  const double xc[3] = {x[3 * (size_t)c], x[3 * (size_t)c + 1], x[3 * (size_t)c + 2]};
  double g[9];
#pragma unroll
  for (int j = 0; j < 3; ++j)
#pragma unroll
    for (int i = 0; i < 3; ++i) g[i + 3 * j] = -lr[i] * xc[j];
  if (r != c) {
    const double xr[3] = {x[3 * (size_t)r], x[3 * (size_t)r + 1], x[3 * (size_t)r + 2]};
    const double lc[3] = {lam[3 * (size_t)c], lam[3 * (size_t)c + 1], lam[3 * (size_t)c + 2]};
#pragma unroll
    for (int j = 0; j < 3; ++j)
#pragma unroll
      for (int i = 0; i < 3; ++i) g[i + 3 * j] -= xr[i] * lc[j];
  }
  double* o = grad + 9 * (size_t)t;
#pragma unroll
  for (int e = 0; e < 9; ++e) o[e] = g[e];
}

}  // namespace

void bcoo_gradient(maspcg_handle* h, const int* rows, const int* cols, int n, const double* lam, const double* x,
                   double* grad)
{
  if (n <= 0) return;
  k_bcoo_gradient<<<ceil_div(n, kAdjTpb), kAdjTpb, 0, h->stream>>>(rows, cols, n, lam, x, grad);
  MLAUNCHED(h);
  MCK(cudaGetLastError());
}

}  // namespace maspcg
