// diagnostics.cu -- per-domain numerical checks of the MAS preconditioner:
// check_local_matrices / gpu_local_checks and the local part of
// numerical_diagnostics (StiffGIPC/TraditionalMAS32Preconditioner.cu:76-147,
// :149-180, :2727-2887).
//
// For every domain, with A its assembled FP64 matrix (zero diagonal entries
// set to 1, as the inversion does) and M its stored inverse (decoded to FP32):
//   * finiteness of A and M, the smallest diagonal entry of each;
//   * A SPD: an FP64 Cholesky without pivoting meets only positive pivots;
//   * the inverse residual ||A M - I||_F / sqrt(n);
//   * M SPD: implied when A is SPD and the residual is <= 1e-3 (for
//     symmetric M, A SPD and ||I - A M||_2 < 1 make M SPD), else checked by
//     its own Cholesky.
// One CTA per domain; A and M are held in shared memory as dense n x n FP64
// (n = 96 for 32-slot banks: 147 KB), the Cholesky runs in place column by
// column, and the product A M reads both from shared memory.
#include <cmath>
#include <limits>

#include "maspcg_internal.cuh"

namespace maspcg {
namespace {

constexpr int kDiagTpb = 256;

template <int B>
__device__ __forceinline__ int packed_index(int row, int col)
{
  int br = row / 3, bc = col / 3, rr = row % 3, cc = col % 3;
  if (br > bc) {
    int t = br;
    br = bc;
    bc = t;
    t = rr;
    rr = cc;
    cc = t;
  }
  return (B * br - br * (br + 1) / 2 + bc) * 9 + rr + 3 * cc;  // column-major 3x3 blocks
}

// In-place lower Cholesky of the n x n matrix w (row-major); *ok is cleared
// at the first pivot that is not finite and positive.
template <int N>
__device__ void cholesky_check(double* w, int* ok)
{
  for (int k = 0; k < N; ++k) {
    if (threadIdx.x == 0) {
      const double piv = w[k * N + k];
      if (!isfinite(piv) || piv <= 0.0)
        *ok = 0;
      else
        w[k * N + k] = sqrt(piv);
    }
    __syncthreads();
    if (!*ok) return;  // uniform: read after the barrier
    const double d = w[k * N + k];
    for (int r = k + 1 + threadIdx.x; r < N; r += blockDim.x) w[r * N + k] /= d;
    __syncthreads();
    const int m = N - k - 1;
    const int pairs = m * (m + 1) / 2;
    for (int t = threadIdx.x; t < pairs; t += blockDim.x) {
      int r = (int)((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);
      while (r * (r + 1) / 2 > t) --r;
      while ((r + 1) * (r + 2) / 2 <= t) ++r;
      const int c = t - r * (r + 1) / 2;
      const int rr = k + 1 + r, cc = k + 1 + c;
      w[rr * N + cc] -= w[rr * N + k] * w[cc * N + k];
    }
    __syncthreads();
  }
}

template <typename T>
__device__ __forceinline__ T block_min(T v, T* red)
{
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(kFull, v, o));
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) red[w] = v;
  __syncthreads();
  T s = red[0];
  for (int i = 1; i < (int)(blockDim.x >> 5); ++i) s = fmin(s, red[i]);
  __syncthreads();
  return s;
}

// results: 7 doubles per domain (local finite, inverse finite, local SPD,
// inverse SPD, min local diagonal, min inverse diagonal, inverse residual).
template <int B>
__global__ void __launch_bounds__(kDiagTpb) k_local_checks(const double* __restrict__ packed64,
                                                           const float* __restrict__ inverse32, double* results)
{
  constexpr int N = 3 * B;
  constexpr int P = B * (B + 1) / 2;
  extern __shared__ double smem[];
  double* w = smem;          // N x N: A, then its factor
  double* mv = smem + N * N;  // N x N: M
  __shared__ int finite_a, finite_b, pos_a, pos_b;
  __shared__ double red[kDiagTpb / 32];
  const double* A = packed64 + (size_t)blockIdx.x * P * 9;
  const float* M = inverse32 + (size_t)blockIdx.x * P * 9;
  if (threadIdx.x == 0) finite_a = finite_b = 1;
  __syncthreads();
  double da = (double)INFINITY, db = (double)INFINITY;
  for (int i = threadIdx.x; i < N * N; i += blockDim.x) {
    const int row = i / N, col = i % N;
    double a = A[packed_index<B>(row, col)];
    const double b = (double)M[packed_index<B>(row, col)];
    if (row == col && a == 0.0) a = 1.0;
    if (!isfinite(a)) atomicExch(&finite_a, 0);
    if (!isfinite(b)) atomicExch(&finite_b, 0);
    w[i] = a;
    mv[i] = b;
    if (row == col) {
      da = fmin(da, a);
      db = fmin(db, b);
    }
  }
  da = block_min(da, red);
  db = block_min(db, red);
  if (threadIdx.x == 0) {
    pos_a = finite_a;
    pos_b = finite_b;
  }
  __syncthreads();
  if (finite_a) cholesky_check<N>(w, &pos_a);
  __syncthreads();
  // A again, for the product
  for (int i = threadIdx.x; i < N * N; i += blockDim.x) {
    const int row = i / N, col = i % N;
    double a = A[packed_index<B>(row, col)];
    if (row == col && a == 0.0) a = 1.0;
    w[i] = a;
  }
  __syncthreads();
  double sum = 0.0;
  if (finite_a && finite_b)
    for (int i = threadIdx.x; i < N * N; i += blockDim.x) {
      const int row = i / N, col = i % N;
      double prod = 0.0;
      for (int k = 0; k < N; ++k) prod += w[row * N + k] * mv[k * N + col];
      const double e = prod - (row == col ? 1.0 : 0.0);
      sum += e * e;
    }
  sum = block_sum<double, kDiagTpb>(sum, red);
  __shared__ double residual;
  if (threadIdx.x == 0) residual = sqrt(sum / N);
  __syncthreads();
  const bool need_b = finite_b && !(pos_a && residual <= 1e-3);
  if (need_b) cholesky_check<N>(mv, &pos_b);  // uniform condition
  __syncthreads();
  if (threadIdx.x == 0) {
    double* o = results + 7 * (size_t)blockIdx.x;
    o[0] = finite_a;
    o[1] = finite_b;
    o[2] = pos_a;
    o[3] = pos_b;
    o[4] = da;
    o[5] = db;
    o[6] = residual;  // 0 when A or M is not finite, as the reference reports it
  }
}

}  // namespace

void check_local_matrices(maspcg_handle* h, int count, int bank, const double* packed64_dev,
                          const float* inverse32_dev, double* results_dev)
{
  if (count <= 0) return;
  cudaStream_t st = h->stream;
  if (bank == 32) {
    constexpr int bytes = 2 * 96 * 96 * sizeof(double);
    static bool cfg = false;
    if (!cfg) {
      MCK(cudaFuncSetAttribute(k_local_checks<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
      cfg = true;
    }
    k_local_checks<32><<<count, kDiagTpb, bytes, st>>>(packed64_dev, inverse32_dev, results_dev);
  } else {
    constexpr int bytes = 2 * 48 * 48 * sizeof(double);
    k_local_checks<16><<<count, kDiagTpb, bytes, st>>>(packed64_dev, inverse32_dev, results_dev);
  }
  MLAUNCHED(h);
  MCK(cudaGetLastError());
}

}  // namespace maspcg
