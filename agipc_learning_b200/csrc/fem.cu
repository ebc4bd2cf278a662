// fem.cu -- the producer of the FEM part of A: per-tet gradient and
// PSD-projected Hessian of the stable Neo-Hookean energy (SNK1),
// _calculate_fem_gradient_hessian (StiffGIPC/femEnergy.cu:1720-1856) with
// __computePEPF_StableNHK3D1_double (:432-455), __computePFPX3D_Eigen_double
// (:1389), BuildTwistAndFlipEigenvectors (:1593-1639) and
// __project_StabbleNHK_H_3D1_makePD (:1641-1717).
//
// Per tet: F = Ds Dm^-1, energy u/2 (I2 - 3) + r/2 (I3 - 1 - u/r)^2 with the
// Lame rates u (length) and r (volume).  The gradient dt^2 V dF/dx^T P(F) is
// accumulated into the vertex gradient with FP64 atomics (as the reference
// does).  The 9x9 Hessian in F is projected through its closed-form
// eigensystem: six twist/flip pairs from the signed SVD F = U diag(S) V^T,
// and three scaling modes from a 3x3 eigenproblem; negative eigenvalues are
// clamped to zero.  The 12x12 element Hessian dt^2 V dF/dx^T H_F dF/dx is
// written as the 10 upper 3x3 blocks of the tet, rows <= cols (a block below
// the diagonal is transposed), values Eigen column-major.
//
// One thread per tet, FP64 throughout.
#include "maspcg_internal.cuh"

namespace maspcg {
namespace {

constexpr int kFemTpb = 128;

// Cyclic Jacobi on a symmetric 3x3 (row-major a, destroyed): eigenvalues d,
// eigenvectors in the columns of v (row-major).
__device__ void sym3_eigen(double a[9], double d[3], double v[9])
{
#pragma unroll
  for (int i = 0; i < 9; ++i) v[i] = (i % 4 == 0) ? 1.0 : 0.0;
  for (int sweep = 0; sweep < 32; ++sweep) {
    const double off = a[1] * a[1] + a[2] * a[2] + a[5] * a[5];
    const double dia = a[0] * a[0] + a[4] * a[4] + a[8] * a[8];
    if (off <= 1e-34 * dia || off == 0.0) break;
#pragma unroll
    for (int pr = 0; pr < 3; ++pr) {
      const int p = pr == 2 ? 1 : 0, q = pr == 0 ? 1 : 2;
      const double apq = a[3 * p + q];
      if (apq == 0.0) continue;
      const double theta = (a[3 * q + q] - a[3 * p + p]) / (2.0 * apq);
      const double t = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
      const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
#pragma unroll
      for (int k = 0; k < 3; ++k) {  // columns p, q of a
        const double akp = a[3 * k + p], akq = a[3 * k + q];
        a[3 * k + p] = c * akp - s * akq;
        a[3 * k + q] = s * akp + c * akq;
      }
#pragma unroll
      for (int k = 0; k < 3; ++k) {  // rows p, q of a
        const double apk = a[3 * p + k], aqk = a[3 * q + k];
        a[3 * p + k] = c * apk - s * aqk;
        a[3 * q + k] = s * apk + c * aqk;
      }
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const double vkp = v[3 * k + p], vkq = v[3 * k + q];
        v[3 * k + p] = c * vkp - s * vkq;
        v[3 * k + q] = s * vkp + c * vkq;
      }
    }
  }
  d[0] = a[0];
  d[1] = a[4];
  d[2] = a[8];
}

__device__ __forceinline__ void cross3(const double* a, const double* b, double* o)
{
  o[0] = a[1] * b[2] - a[2] * b[1];
  o[1] = a[2] * b[0] - a[0] * b[2];
  o[2] = a[0] * b[1] - a[1] * b[0];
}

// Signed SVD of a 3x3 (row-major): F = U diag(S) V^T with U, V rotations and
// S[2] carrying the sign of det F.  V from the eigenvectors of F^T F
// (descending), U and S from a Gram-Schmidt QR of F V.
__device__ void signed_svd3(const double F[9], double U[9], double S[3], double V[9])
{
  double c[9];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) c[3 * i + j] = F[i] * F[j] + F[3 + i] * F[3 + j] + F[6 + i] * F[6 + j];
  double d[3], w[9];
  sym3_eigen(c, d, w);
  int o[3] = {0, 1, 2};  // descending order
  if (d[o[0]] < d[o[1]]) { const int t = o[0]; o[0] = o[1]; o[1] = t; }
  if (d[o[1]] < d[o[2]]) { const int t = o[1]; o[1] = o[2]; o[2] = t; }
  if (d[o[0]] < d[o[1]]) { const int t = o[0]; o[0] = o[1]; o[1] = t; }
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int k = 0; k < 3; ++k) V[3 * i + k] = w[3 * i + o[k]];
  const double detv = V[0] * (V[4] * V[8] - V[5] * V[7]) - V[1] * (V[3] * V[8] - V[5] * V[6]) +
                      V[2] * (V[3] * V[7] - V[4] * V[6]);
  if (detv < 0.0) V[2] = -V[2], V[5] = -V[5], V[8] = -V[8];
  double b[3][3];  // columns of F V
#pragma unroll
  for (int k = 0; k < 3; ++k)
#pragma unroll
    for (int i = 0; i < 3; ++i) b[k][i] = F[3 * i] * V[k] + F[3 * i + 1] * V[3 + k] + F[3 * i + 2] * V[6 + k];
  double u0[3], u1[3], u2[3];
  double n0 = sqrt(b[0][0] * b[0][0] + b[0][1] * b[0][1] + b[0][2] * b[0][2]);
  if (n0 > 0.0) {
    for (int i = 0; i < 3; ++i) u0[i] = b[0][i] / n0;
  } else {
    u0[0] = 1.0, u0[1] = 0.0, u0[2] = 0.0;
  }
  const double p = u0[0] * b[1][0] + u0[1] * b[1][1] + u0[2] * b[1][2];
  double r1[3] = {b[1][0] - p * u0[0], b[1][1] - p * u0[1], b[1][2] - p * u0[2]};
  double n1 = sqrt(r1[0] * r1[0] + r1[1] * r1[1] + r1[2] * r1[2]);
  if (!(n1 > 1e-300)) {  // any unit vector orthogonal to u0
    const double e[3] = {fabs(u0[0]) < 0.9 ? 1.0 : 0.0, fabs(u0[0]) < 0.9 ? 0.0 : 1.0, 0.0};
    cross3(u0, e, r1);
    n1 = sqrt(r1[0] * r1[0] + r1[1] * r1[1] + r1[2] * r1[2]);
    for (int i = 0; i < 3; ++i) r1[i] /= n1;
    n1 = 0.0;
    for (int i = 0; i < 3; ++i) u1[i] = r1[i];
  } else {
    for (int i = 0; i < 3; ++i) u1[i] = r1[i] / n1;
  }
  cross3(u0, u1, u2);
  S[0] = n0;
  S[1] = n1;
  S[2] = u2[0] * b[2][0] + u2[1] * b[2][1] + u2[2] * b[2][2];
  for (int i = 0; i < 3; ++i) {
    U[3 * i] = u0[i];
    U[3 * i + 1] = u1[i];
    U[3 * i + 2] = u2[i];
  }
}

__global__ void __launch_bounds__(kFemTpb) k_fem_snk1(int ntet, const unsigned* __restrict__ tets,
                                                      const double* __restrict__ x, const double* __restrict__ dm_inv,
                                                      const double* __restrict__ volume,
                                                      const double* __restrict__ len_rate,
                                                      const double* __restrict__ vol_rate, double dt2, int offset,
                                                      int nverts, double* gradient, int* rows, int* cols,
                                                      double* vals, int* bad)
{
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ntet) return;
  const unsigned v[4] = {tets[4 * (size_t)t], tets[4 * (size_t)t + 1], tets[4 * (size_t)t + 2],
                         tets[4 * (size_t)t + 3]};
  if (v[0] >= (unsigned)nverts || v[1] >= (unsigned)nverts || v[2] >= (unsigned)nverts || v[3] >= (unsigned)nverts) {
    atomicExch(bad, 1);  // the tet is skipped; the call reports the error
    return;
  }
  const double* Di = dm_inv + 9 * (size_t)t;  // row-major Dm^-1
  double Ds[9];
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) Ds[3 * r + c] = x[3 * (size_t)v[c + 1] + r] - x[3 * (size_t)v[0] + r];
  double F[9];
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) F[3 * r + c] = Ds[3 * r] * Di[c] + Ds[3 * r + 1] * Di[3 + c] + Ds[3 * r + 2] * Di[6 + c];
  const double u = len_rate[t], rr = vol_rate[t], vol = volume[t];
  // dI3/dF (cofactor matrix) and I3
  double g[9];
  g[0] = F[4] * F[8] - F[5] * F[7];
  g[1] = F[5] * F[6] - F[3] * F[8];
  g[2] = F[3] * F[7] - F[4] * F[6];
  g[3] = F[7] * F[2] - F[8] * F[1];
  g[4] = F[8] * F[0] - F[6] * F[2];
  g[5] = F[6] * F[1] - F[7] * F[0];
  g[6] = F[1] * F[5] - F[4] * F[2];
  g[7] = F[2] * F[3] - F[0] * F[5];
  g[8] = F[0] * F[4] - F[1] * F[3];
  const double I3 = F[0] * g[0] + F[1] * g[1] + F[2] * g[2];
  // dF_ij / dx_{a,i} = cf[a][j]
  double cf[4][3];
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    cf[1][j] = Di[j];
    cf[2][j] = Di[3 + j];
    cf[3][j] = Di[6 + j];
    cf[0][j] = -(cf[1][j] + cf[2][j] + cf[3][j]);
  }
  const double scale = dt2 * vol;
  // gradient: P = u F + (r (I3 - 1) - u) dI3/dF
  {
    const double k = rr * (I3 - 1.0) - u;
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        double f = 0.0;
#pragma unroll
        for (int j = 0; j < 3; ++j) f += cf[a][j] * (u * F[3 * i + j] + k * g[3 * i + j]);
        atomicAdd(gradient + 3 * (size_t)v[a] + i, scale * f);
      }
  }
  // eigensystem of the 9x9 Hessian in F (vec column-major: index i + 3j)
  double U[9], S[3], V[9];
  signed_svd3(F, U, S, V);
  const double J = I3;
  double lam[9];
  const double ev1 = rr * (J - 1.0) - u;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    lam[i] = u + S[i] * ev1;      // twist
    lam[3 + i] = u - S[i] * ev1;  // flip
  }
  double A[9];
  const double ev2 = rr * (2.0 * J - 1.0) - u;
  A[0] = u + rr * S[1] * S[1] * S[2] * S[2];
  A[4] = u + rr * S[0] * S[0] * S[2] * S[2];
  A[8] = u + rr * S[0] * S[0] * S[1] * S[1];
  A[1] = A[3] = ev2 * S[2];
  A[2] = A[6] = ev2 * S[1];
  A[5] = A[7] = ev2 * S[0];
  double sd[3], sv[9];
  sym3_eigen(A, sd, sv);
  lam[6] = sd[0];
  lam[7] = sd[1];
  lam[8] = sd[2];
  // eigenvector k as a 3x3 matrix Q_k (row-major, Q[i][j] = q[i + 3j]) and
  // its image w_k = dF/dx^T q_k (12 entries), accumulated into the blocks
  const double h = 0.70710678118654752440;  // 1/sqrt(2)
  double Hb[10][9];
#pragma unroll
  for (int b = 0; b < 10; ++b)
#pragma unroll
    for (int e = 0; e < 9; ++e) Hb[b][e] = 0.0;
#pragma unroll 1
  for (int k = 0; k < 9; ++k) {
    const double l = lam[k] > 0.0 ? lam[k] : 0.0;
    if (l == 0.0) continue;
    double Q[9];
    if (k < 6) {
      // twist / flip for the axis pair (p, q) opposite axis m
      const int m = k % 3;
      const int p = m == 0 ? 1 : 0, q = m == 2 ? 1 : 2;
      const double sg = k < 3 ? -1.0 : 1.0;  // twist: U_q V_p^T - U_p V_q^T; flip: the sum
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
          Q[3 * i + j] = h * (U[3 * i + q] * V[3 * j + p] + sg * U[3 * i + p] * V[3 * j + q]);
    } else {
      const int c = k - 6;
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
          Q[3 * i + j] = U[3 * i] * sv[c] * V[3 * j] + U[3 * i + 1] * sv[3 + c] * V[3 * j + 1] +
                         U[3 * i + 2] * sv[6 + c] * V[3 * j + 2];
    }
    double w[12];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int i = 0; i < 3; ++i) w[3 * a + i] = cf[a][0] * Q[3 * i] + cf[a][1] * Q[3 * i + 1] + cf[a][2] * Q[3 * i + 2];
    int bi = 0;
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = a; b < 4; ++b, ++bi)
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
          for (int j = 0; j < 3; ++j) Hb[bi][3 * i + j] += l * w[3 * a + i] * w[3 * b + j];
  }
  // triplets: 10 upper blocks, rows <= cols, Eigen column-major values
  int bi = 0;
  const size_t base = 10 * (size_t)t;
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = a; b < 4; ++b, ++bi) {
      const int ra = (int)v[a] + offset, rb = (int)v[b] + offset;
      const bool swap = ra > rb;
      rows[base + bi] = swap ? rb : ra;
      cols[base + bi] = swap ? ra : rb;
      double* o = vals + 9 * (base + bi);
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) o[i + 3 * j] = scale * (swap ? Hb[bi][3 * j + i] : Hb[bi][3 * i + j]);
    }
}

}  // namespace

void fem_snk1(maspcg_handle* h, int ntet, int nverts, const unsigned* tets, const double* x, const double* dm_inv,
              const double* volume, const double* len_rate, const double* vol_rate, double dt, int offset,
              double* gradient, int* rows, int* cols, double* vals)
{
  if (ntet <= 0) return;
  h->asm_flags.resize(std::max<size_t>(h->asm_flags.n, 1));
  int* bad = h->asm_flags.get();
  MCK(cudaMemsetAsync(bad, 0, sizeof(int), h->stream));
  k_fem_snk1<<<ceil_div(ntet, kFemTpb), kFemTpb, 0, h->stream>>>(ntet, tets, x, dm_inv, volume, len_rate, vol_rate,
                                                                 dt * dt, offset, nverts, gradient, rows, cols, vals,
                                                                 bad);
  MLAUNCHED(h);
  MCK(cudaGetLastError());
  int flag = 0;
  MCK(cudaMemcpyAsync(&flag, bad, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  MCK(cudaStreamSynchronize(h->stream));
  MREQ(flag == 0, MASPCG_ERR_INVALID_ARGUMENT, "tet vertex id out of range");
}

}  // namespace maspcg
