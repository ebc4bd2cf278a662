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

// The same outer products chained through the element blocks to each tet's
// Young's modulus: a tet's blocks are linear in its modulus E_t (the Lame pair
// is linear in E, and the PSD projection commutes with a positive scale), so
// dL/dE_t = sum over its blocks k of <G_k, V_k> / E_t with G_k as above; the
// G_k are never stored.  Blocks [bpt t, bpt t + bpt) of the list are tet t's.
// One warp per tet: lanes take the blocks, a shuffle sum, lane 0 writes.
__global__ void __launch_bounds__(kAdjTpb) k_modulus_gradient(const int* __restrict__ rows,
                                                             const int* __restrict__ cols,
                                                             const double* __restrict__ vals, int ntet, int bpt,
                                                             const double* __restrict__ lam,
                                                             const double* __restrict__ x,
                                                             const double* __restrict__ E, double* gE)
{
  const int t = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (t >= ntet) return;  // whole warp
  double acc = 0.0;
  for (int q = lane; q < bpt; q += 32) {
    const size_t k = (size_t)t * bpt + q;
    const int r = rows[k], c = cols[k];
    const double* V = vals + 9 * k;  // column-major: element (i, j) at i + 3j
    double s = 0.0;
#pragma unroll
    for (int j = 0; j < 3; ++j)
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        double g = lam[3 * (size_t)r + i] * x[3 * (size_t)c + j];
        if (r != c) g += x[3 * (size_t)r + i] * lam[3 * (size_t)c + j];
        s -= g * V[i + 3 * j];
      }
    acc += s;
  }
  acc = warp_sum(acc);
  if (lane == 0) gE[t] = acc / E[t];
}

}  // namespace

void modulus_gradient(maspcg_handle* h, const int* rows, const int* cols, const double* vals, int ntet, int bpt,
                      const double* lam, const double* x, const double* E, double* gE)
{
  if (ntet <= 0) return;
  k_modulus_gradient<<<ceil_div(32LL * ntet, kAdjTpb), kAdjTpb, 0, h->stream>>>(rows, cols, vals, ntet, bpt, lam, x, E,
                                                                              gE);
  MLAUNCHED(h);
  MCK(cudaGetLastError());
}

void bcoo_gradient(maspcg_handle* h, const int* rows, const int* cols, int n, const double* lam, const double* x,
                   double* grad)
{
  if (n <= 0) return;
  k_bcoo_gradient<<<ceil_div(n, kAdjTpb), kAdjTpb, 0, h->stream>>>(rows, cols, n, lam, x, grad);
  MLAUNCHED(h);
  MCK(cudaGetLastError());
}

}  // namespace maspcg
