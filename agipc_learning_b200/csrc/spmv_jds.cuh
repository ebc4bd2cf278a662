// spmv_jds.cuh -- the FP32 matrix of the PCG iteration in a sliced
// jagged-diagonal layout, and the SpMV over it.
//
// Layout (built by build_jds in matrix.cu from the FP64 full BCSR):
//   * a slice is 32 consecutive internal block rows (one MAS level-0 domain
//     when the rows follow the MAS partition); inside a slice the rows are
//     ranked by length, longest first (ties by row), and perm[32 s + i] holds
//     the slice-local row at rank i (bit 7 set: the rank writes nothing, its
//     row lies past the end or takes the FP64 row path);
//   * column k of a slice holds the k-th block (ascending column) of every
//     ranked row longer than k: those are ranks [0, n_k), stored at
//     base[s] + coff[cbase[s] + k] + i, so column k of a slice is one
//     contiguous run and a warp reads it with consecutive addresses; the
//     layout stores no padding;
//   * an entry is 40 bytes over three planes: a (elements 0-3 of the
//     row-major 3x3 block), b (elements 4-7) and c (element 8 and the column
//     index as a float bit pattern), so a lane reads a block with two 16-byte
//     and one 8-byte load;
//   * rows of the affine bodies, and rows longer than kJdsMaxLen blocks, are
//     not in the slices: they are listed in xrows and multiplied from the FP64
//     BCSR with FP64 sums (a body's 12x12 block spans ~1e11 between its
//     orthogonality stiffness and its mass-only rotation modes, more than
//     FP32 values keep positive definite).
// The SpMV gives a warp SL slices at once, lane i the row of rank i, and
// walks the columns U at a time: each step issues the loads of SL x U blocks
// before their gathers of the search direction, with no cross-lane reduction
// and no row-pointer reads.
#pragma once
#include <type_traits>

#include "maspcg_internal.cuh"
#include "pcg_device.cuh"

namespace maspcg {

constexpr int kJdsMaxLen = 64;  // longer rows take the FP64 row path
#ifndef MASPCG_JDS_SL
#define MASPCG_JDS_SL 1
#endif
#ifndef MASPCG_JDS_U
#define MASPCG_JDS_U 4
#endif
#ifndef MASPCG_JDS_ACC64
#define MASPCG_JDS_ACC64 0
#endif
constexpr int kJdsSlicesPerWarp = MASPCG_JDS_SL;  // slices a warp walks at once
constexpr int kJdsColumnsPerStep = MASPCG_JDS_U;  // columns of each slice whose loads go out together

struct JdsArgs {
  const int* base;             // slices + 1: first entry of each slice
  const int* cbase;            // slices + 1: first column offset of each slice (width + 1 offsets per slice)
  const int* coff;             // per slice: entries in the columns before column k, k = 0..width
  const unsigned char* perm;   // 32 per slice: slice-local row of each rank, bit 7 = writes nothing
  const float4* a;
  const float4* b;
  const float2* c;
  const int* xrows;            // rows on the FP64 row path
  int slices;
  int nx;
};

inline JdsArgs jds_args(const maspcg_handle* h)
{
  JdsArgs j{};
  j.base = h->jds_base.get();
  j.cbase = h->jds_cbase.get();
  j.coff = h->jds_coff.get();
  j.perm = h->jds_perm.get();
  j.a = h->jds_a.get();
  j.b = h->jds_b.get();
  j.c = h->jds_c.get();
  j.xrows = h->jds_xrows.get();
  j.slices = h->jds_slices;
  j.nx = h->jds_nx;
  return j;
}

// Ap for the slices of this warp; returns this thread's share of p.Ap.
template <typename Tacc, int SL, int U>
__device__ __forceinline__ Tacc spmv_jds(const JdsArgs& j, const float* __restrict__ p4, float* ap)
{
  const int lane = threadIdx.x & 31;
  const int gw = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int nw = (int)((gridDim.x * blockDim.x) >> 5);
  Tacc dot = 0;
  for (int s0 = gw * SL; s0 < j.slices; s0 += nw * SL) {
    using RowAcc = typename std::conditional<MASPCG_JDS_ACC64 != 0, double, float>::type;
    int base[SL], cb[SL], width[SL], prow[SL];
    bool wr[SL];
    RowAcc acc[SL][3];
    int wmax = 0;
#pragma unroll
    for (int q = 0; q < SL; ++q) {
      const int s = s0 + q;
      const bool valid = s < j.slices;
      base[q] = valid ? __ldg(j.base + s) : 0;
      cb[q] = valid ? __ldg(j.cbase + s) : 0;
      width[q] = valid ? __ldg(j.cbase + s + 1) - cb[q] - 1 : 0;
      const unsigned pm = valid ? __ldg(j.perm + 32 * (size_t)s + lane) : 0x80u;
      prow[q] = 32 * s + (int)(pm & 31u);
      wr[q] = valid && !(pm & 0x80u);
      acc[q][0] = acc[q][1] = acc[q][2] = 0.f;
      wmax = max(wmax, width[q]);
    }
    for (int c0 = 0; c0 < wmax; c0 += 32) {
      int off[SL], cnt[SL];
#pragma unroll
      for (int q = 0; q < SL; ++q) {
        const int k = c0 + lane;
        const bool in = k < width[q];
        off[q] = in ? __ldg(j.coff + cb[q] + k) : 0;
        cnt[q] = in ? __ldg(j.coff + cb[q] + k + 1) - off[q] : 0;
      }
      const int nk = min(32, wmax - c0);
      for (int kk = 0; kk < nk; kk += U) {
        float4 A[SL][U], B[SL][U];
        float2 C[SL][U];
        bool act[SL][U];
#pragma unroll
        for (int q = 0; q < SL; ++q)
#pragma unroll
          for (int u = 0; u < U; ++u) {
            const int k = (kk + u) & 31;
            const int o = __shfl_sync(kFull, off[q], k);
            const int n = __shfl_sync(kFull, cnt[q], k);
            act[q][u] = kk + u < nk && lane < n;
            if (act[q][u]) {
              const size_t e = (size_t)base[q] + o + lane;
              C[q][u] = __ldcs(j.c + e);
              A[q][u] = __ldcs(j.a + e);
              B[q][u] = __ldcs(j.b + e);
            }
          }
#pragma unroll
        for (int q = 0; q < SL; ++q)
#pragma unroll
          for (int u = 0; u < U; ++u)
            if (act[q][u]) {
              const P4<float> x = ld_p4(p4, __float_as_int(C[q][u].y));
              const float4 m0 = A[q][u], m1 = B[q][u];
              acc[q][0] += (RowAcc)(m0.x * x.x + m0.y * x.y + m0.z * x.z);
              acc[q][1] += (RowAcc)(m0.w * x.x + m1.x * x.y + m1.y * x.z);
              acc[q][2] += (RowAcc)(m1.z * x.x + m1.w * x.y + C[q][u].x * x.z);
            }
      }
    }
#pragma unroll
    for (int q = 0; q < SL; ++q)
      if (wr[q]) {
        float* y = ap + 3 * (size_t)prow[q];
        const float y0 = (float)acc[q][0], y1 = (float)acc[q][1], y2 = (float)acc[q][2];
        y[0] = y0;
        y[1] = y1;
        y[2] = y2;
        const P4<float> pr = ld_p4(p4, prow[q]);
        dot += (Tacc)pr.x * (Tacc)y0 + (Tacc)pr.y * (Tacc)y1 + (Tacc)pr.z * (Tacc)y2;
      }
  }
  return dot;
}

// Ap for the listed rows from the FP64 BCSR with FP64 sums (LPR lanes per
// row); returns this thread's share of p.Ap.
template <typename Tacc, int LPR>
__device__ __forceinline__ Tacc spmv_rows_listed(const int* __restrict__ rowptr, const int* __restrict__ colidx,
                                                 const double* __restrict__ val64, const int* __restrict__ xrows,
                                                 int nx, const float* __restrict__ p4, float* ap)
{
  const int sub = threadIdx.x % LPR;
  const int groups = (int)(gridDim.x * blockDim.x) / LPR;
  const int g0 = (int)(blockIdx.x * blockDim.x + threadIdx.x) / LPR;
  double dot = 0.0;
  // the loop runs while any group of the warp has a row: the shuffles below
  // take all 32 lanes
  for (int i = g0; __any_sync(kFull, i < nx); i += groups) {
    const bool ok = i < nx;
    const int row = ok ? __ldg(xrows + i) : 0;
    double a0 = 0.0, a1 = 0.0, a2 = 0.0;
    if (ok) {
      const int re = __ldg(rowptr + row + 1);
      for (int t = __ldg(rowptr + row) + sub; t < re; t += LPR) {
        const double* m = val64 + 9 * (size_t)t;
        const P4<float> x = ld_p4(p4, __ldg(colidx + t));
        a0 += __ldcs(m) * (double)x.x + __ldcs(m + 1) * (double)x.y + __ldcs(m + 2) * (double)x.z;
        a1 += __ldcs(m + 3) * (double)x.x + __ldcs(m + 4) * (double)x.y + __ldcs(m + 5) * (double)x.z;
        a2 += __ldcs(m + 6) * (double)x.x + __ldcs(m + 7) * (double)x.y + __ldcs(m + 8) * (double)x.z;
      }
    }
#pragma unroll
    for (int o = LPR / 2; o > 0; o >>= 1) {
      a0 += __shfl_xor_sync(kFull, a0, o, LPR);
      a1 += __shfl_xor_sync(kFull, a1, o, LPR);
      a2 += __shfl_xor_sync(kFull, a2, o, LPR);
    }
    if (ok && sub < 3) {
      const float y = (float)(sub == 0 ? a0 : (sub == 1 ? a1 : a2));
      ap[3 * (size_t)row + sub] = y;
      const P4<float> pr = ld_p4(p4, row);
      dot += (double)(sub == 0 ? pr.x : (sub == 1 ? pr.y : pr.z)) * (double)y;
    }
  }
  return (Tacc)dot;
}

}  // namespace maspcg
