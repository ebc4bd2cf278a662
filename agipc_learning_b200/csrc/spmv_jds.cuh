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
//     ranked row longer than k: those are ranks [0, n_k), entries
//     coff[k] + i of the slice, so column k is one contiguous run read with
//     consecutive addresses; nothing is padded;
//   * a slice is one contiguous record of 40 bytes per entry: plane a
//     (elements 0-3 of the row-major 3x3 block, 16 B per entry), plane b
//     (elements 4-7) and plane c (element 8 and the column index as a float
//     bit pattern, 8 B), each plane E entries long with E the entry count
//     rounded up to even, so a record is a multiple of 16 bytes and can be
//     moved by one bulk copy;
//   * a 64-int header per slice: E, the width (longest row) and coff[0..width];
//     the record's byte offset in srec;
//   * rows of the affine bodies, and rows longer than kJdsMaxLen blocks, are
//     not in the slices: they are listed in xrows and multiplied from the FP64
//     BCSR with FP64 sums (a body's 12x12 block spans ~1e11 between its
//     orthogonality stiffness and its mass-only rotation modes, more than
//     FP32 values keep positive definite).
// Each lane takes the row of one rank and walks the columns U at a time: the
// loads of U blocks go out before their gathers of the search direction; the
// 3x3 products are FP32 and each block's three results are added into FP64
// row sums (the sum over the row's blocks cancels between the mass and the
// elastic and contact terms, which FP32 sums do not resolve); no cross-lane
// reduction, no row pointers.
#pragma once
#include <type_traits>

#include "maspcg_internal.cuh"
#include "pcg_device.cuh"
#include "tma.cuh"

namespace maspcg {

constexpr int kJdsMaxLen = 61;  // longer rows take the FP64 row path (the header holds coff[0..61])
constexpr int kJdsHeader = 64;  // ints per slice header
#ifndef MASPCG_JDS_U
#define MASPCG_JDS_U 4
#endif
#ifndef MASPCG_JDS_STAGED
#define MASPCG_JDS_STAGED 1
#endif
#ifndef MASPCG_JDS_G
#define MASPCG_JDS_G 16
#endif
constexpr int kJdsColumnsPerStep = MASPCG_JDS_U;  // direct form: columns whose loads go out together
constexpr int kJdsGather = MASPCG_JDS_G;          // staged form: columns whose gathers go out together
// Staged form: warps per CTA and the two record slots of each warp.
constexpr int kJdsWarps = 4;
constexpr int kJdsSlotBytes = 24576;  // slices of more than 614 entries are read from global memory
constexpr int kJdsSmem = kJdsWarps * 2 * kJdsSlotBytes;

struct JdsArgs {
  const int* hdr;              // kJdsHeader ints per slice
  const long long* srec;       // slices + 1: byte offset of each slice's record
  const unsigned char* perm;   // 32 per slice: slice-local row of each rank, bit 7 = writes nothing
  const unsigned char* data;   // the records
  const int* xrows;            // rows on the FP64 row path
  int slices;
  int nx;
};

// The vector side of one SpMV: y = A x with x gathered from one padded
// vector, or (kTwo) from the sum of two, x4 + x4b; xsum (kTwo) receives that
// sum for the rows the SpMV writes (3 per row).
struct SpmvVec {
  const float* x4;
  const float* x4b;
  float* y;
  float* xsum;
};

template <bool kTwo>
__device__ __forceinline__ P4<float> spmv_x(const SpmvVec& v, int c)
{
  P4<float> x = ld_p4(v.x4, c);
  if constexpr (kTwo) {
    const P4<float> b = ld_p4(v.x4b, c);
    x.x += b.x;
    x.y += b.y;
    x.z += b.z;
  }
  return x;
}

// y for one row and its share of x.y (xsum written for kTwo).
template <bool kTwo, typename Tacc>
__device__ __forceinline__ Tacc spmv_store_row(const SpmvVec& v, int row, float y0, float y1, float y2)
{
  float* y = v.y + 3 * (size_t)row;
  y[0] = y0;
  y[1] = y1;
  y[2] = y2;
  const P4<float> xr = spmv_x<kTwo>(v, row);
  if constexpr (kTwo) {
    float* z = v.xsum + 3 * (size_t)row;
    z[0] = xr.x;
    z[1] = xr.y;
    z[2] = xr.z;
  }
  return (Tacc)xr.x * (Tacc)y0 + (Tacc)xr.y * (Tacc)y1 + (Tacc)xr.z * (Tacc)y2;
}

inline JdsArgs jds_args(const maspcg_handle* h)
{
  JdsArgs j{};
  j.hdr = h->jds_hdr.get();
  j.srec = h->jds_srec.get();
  j.perm = h->jds_perm.get();
  j.data = h->jds_data.get();
  j.xrows = h->jds_xrows.get();
  j.slices = h->jds_slices;
  j.nx = h->jds_nx;
  return j;
}

// Slice metadata held by a warp: lane l holds header words l and 32 + l and
// the rank byte of rank l.
struct JdsMeta {
  int v0, v1;
  unsigned pm;
  long long rec;
};

__device__ __forceinline__ JdsMeta jds_meta(const JdsArgs& j, int s, int lane)
{
  JdsMeta m{0, 0, 0x80u, 0};
  if (s < j.slices) {
    const int* hd = j.hdr + (size_t)kJdsHeader * s;
    m.v0 = __ldg(hd + lane);
    m.v1 = __ldg(hd + 32 + lane);
    m.pm = __ldg(j.perm + 32 * (size_t)s + lane);
    m.rec = __ldg(j.srec + s);
  }
  return m;
}

// coff[k] of the slice (k <= kJdsMaxLen): header word 2 + k.
__device__ __forceinline__ int jds_coff(const JdsMeta& m, int k)
{
  const int a = __shfl_sync(kFull, m.v0, (k + 2) & 31);
  const int b = __shfl_sync(kFull, m.v1, (k + 2) & 31);
  return k + 2 < 32 ? a : b;
}

template <bool kShared>
__device__ __forceinline__ float4 jds_ld4(const unsigned char* p)
{
  if constexpr (kShared)
    return *reinterpret_cast<const float4*>(p);
  else
    return __ldcs(reinterpret_cast<const float4*>(p));
}
template <bool kShared>
__device__ __forceinline__ float2 jds_ld2(const unsigned char* p)
{
  if constexpr (kShared)
    return *reinterpret_cast<const float2*>(p);
  else
    return __ldcs(reinterpret_cast<const float2*>(p));
}

// One slice: Ap for its rows from the record at `rec` (shared memory when
// kShared, else global); returns this lane's share of p.Ap.
template <typename Tacc, int U, bool kShared, bool kTwo>
__device__ __forceinline__ Tacc jds_slice(const JdsMeta& m, int s, const unsigned char* rec, const SpmvVec& v,
                                          int lane)
{
  const int ep = __shfl_sync(kFull, m.v0, 0);
  const int width = __shfl_sync(kFull, m.v0, 1);
  const unsigned char* pa = rec;
  const unsigned char* pb = rec + 16 * (size_t)ep;
  const unsigned char* pc = rec + 32 * (size_t)ep;
  double acc0 = 0.0, acc1 = 0.0, acc2 = 0.0;
  int o_next = jds_coff(m, 0);
  for (int kk = 0; kk < width; kk += U) {
    float4 A[U], B[U];
    float2 C[U];
    bool act[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int k = kk + u;
      const int o = o_next;
      o_next = jds_coff(m, k + 1);
      act[u] = k < width && lane < o_next - o;
      if (act[u]) {
        const int e = o + lane;
        C[u] = jds_ld2<kShared>(pc + 8 * (size_t)e);
        A[u] = jds_ld4<kShared>(pa + 16 * (size_t)e);
        B[u] = jds_ld4<kShared>(pb + 16 * (size_t)e);
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u)
      if (act[u]) {
        const P4<float> x = spmv_x<kTwo>(v, __float_as_int(C[u].y));
        const float4 m0 = A[u], m1 = B[u];
        acc0 += (double)(m0.x * x.x + m0.y * x.y + m0.z * x.z);
        acc1 += (double)(m0.w * x.x + m1.x * x.y + m1.y * x.z);
        acc2 += (double)(m1.z * x.x + m1.w * x.y + C[u].x * x.z);
      }
  }
  Tacc dot = 0;
  if (!(m.pm & 0x80u))
    dot = spmv_store_row<kTwo, Tacc>(v, 32 * s + (int)(m.pm & 31u), (float)acc0, (float)acc1, (float)acc2);
  return dot;
}

// One slice from its record in shared memory: the column indices are read
// first and the gathers of the search direction for G columns go out
// together (one L2 round trip per G columns); the block values are read from
// shared memory afterwards.  Returns this lane's share of p.Ap.
template <typename Tacc, int G, bool kTwo>
__device__ __forceinline__ Tacc jds_slice_smem(const JdsMeta& m, int s, const unsigned char* rec, const SpmvVec& v,
                                               int lane)
{
  const int ep = __shfl_sync(kFull, m.v0, 0);
  const int width = __shfl_sync(kFull, m.v0, 1);
  const float4* pa = reinterpret_cast<const float4*>(rec);
  const float4* pb = reinterpret_cast<const float4*>(rec + 16 * (size_t)ep);
  const float2* pc = reinterpret_cast<const float2*>(rec + 32 * (size_t)ep);
  double acc0 = 0.0, acc1 = 0.0, acc2 = 0.0;
  int o_next = jds_coff(m, 0);
  for (int kk = 0; kk < width; kk += G) {
    int e[G];
    float c8[G];
    P4<float> x[G];
#pragma unroll
    for (int u = 0; u < G; ++u) {
      const int k = kk + u;
      const int o = o_next;
      o_next = jds_coff(m, k + 1);
      e[u] = (k < width && lane < o_next - o) ? o + lane : -1;
      if (e[u] >= 0) {
        const float2 c = pc[e[u]];
        c8[u] = c.x;
        x[u] = spmv_x<kTwo>(v, __float_as_int(c.y));
      }
    }
#pragma unroll
    for (int u = 0; u < G; ++u)
      if (e[u] >= 0) {
        const float4 m0 = pa[e[u]], m1 = pb[e[u]];
        acc0 += (double)(m0.x * x[u].x + m0.y * x[u].y + m0.z * x[u].z);
        acc1 += (double)(m0.w * x[u].x + m1.x * x[u].y + m1.y * x[u].z);
        acc2 += (double)(m1.z * x[u].x + m1.w * x[u].y + c8[u] * x[u].z);
      }
  }
  Tacc dot = 0;
  if (!(m.pm & 0x80u))
    dot = spmv_store_row<kTwo, Tacc>(v, 32 * s + (int)(m.pm & 31u), (float)acc0, (float)acc1, (float)acc2);
  return dot;
}

// Ap for the slices of this warp, records read from global memory; the next
// slice's metadata is fetched while the current one is computed.
template <typename Tacc, int U, bool kTwo>
__device__ __forceinline__ Tacc spmv_jds_direct(const JdsArgs& j, const SpmvVec& v)
{
  const int lane = threadIdx.x & 31;
  const int gw = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int nw = (int)((gridDim.x * blockDim.x) >> 5);
  Tacc dot = 0;
  JdsMeta next = jds_meta(j, gw, lane);
  for (int s = gw; s < j.slices; s += nw) {
    const JdsMeta m = next;
    next = jds_meta(j, s + nw, lane);
    dot += jds_slice<Tacc, U, false, kTwo>(m, s, j.data + m.rec, v, lane);
  }
  return dot;
}

// Staged form: each warp owns two record slots in shared memory; the record
// of its next-but-one slice is bulk-copied into the slot its current slice
// frees, so the copies run ahead of the arithmetic and hold no registers.
// Records larger than a slot are read from global memory.  Every wait is
// bounded: on expiry the warp records error 1, drains its copies in flight
// (bounded), and returns false.
template <typename Tacc, int U, bool kTwo>
__device__ __forceinline__ bool spmv_jds_staged(const JdsArgs& j, const SpmvVec& v, unsigned char* slots,
                                                uint64_t* bars, int* err, Tacc& dot)
{
  const int lane = threadIdx.x & 31, lw = threadIdx.x >> 5;
  const int gw = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int nw = (int)((gridDim.x * blockDim.x) >> 5);
  unsigned char* slot[2] = {slots + (size_t)lw * 2 * kJdsSlotBytes, slots + (size_t)(2 * lw + 1) * kJdsSlotBytes};
  uint64_t* bar = bars + 2 * lw;
  // issue the record copy of slice s into slot q (lane 0); true when issued
  auto issue = [&](int s, int q) -> bool {
    bool staged = false;
    if (s < j.slices) {
      const long long r0 = __ldg(j.srec + s), r1 = __ldg(j.srec + s + 1);
      const long long bytes = r1 - r0;
      staged = bytes > 0 && bytes <= kJdsSlotBytes;
      if (staged && lane == 0) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_expect_tx(&bar[q], (unsigned)bytes);
        tma_bulk_g2s(slot[q], j.data + r0, (unsigned)bytes, &bar[q]);
      }
    }
    return staged;
  };
  if (lane == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncwarp();
  bool pending[2];
  unsigned ph[2] = {0u, 0u};
  pending[0] = issue(gw, 0);
  pending[1] = issue(gw + nw, 1);
  JdsMeta next = jds_meta(j, gw, lane);
  bool ok = true;
  int i = 0;
  for (int s = gw; s < j.slices; s += nw, ++i) {
    const int q = i & 1;
    const JdsMeta m = next;
    next = jds_meta(j, s + nw, lane);
    if (pending[q]) {
      const bool w = mbar_wait(&bar[q], ph[q]);
      if (!__all_sync(kFull, w)) {
        ok = false;
        break;
      }
      ph[q] ^= 1u;
      pending[q] = false;
      dot += jds_slice_smem<Tacc, kJdsGather, kTwo>(m, s, slot[q], v, lane);
      __syncwarp();  // every lane is done with the slot before it is refilled
    } else {
      dot += jds_slice<Tacc, U, false, kTwo>(m, s, j.data + m.rec, v, lane);
    }
    pending[q] = issue(s + 2 * nw, q);
  }
  if (!ok && lane == 0) {
    atomicExch(err, 1);
#pragma unroll
    for (int q = 0; q < 2; ++q)
      if (pending[q]) mbar_wait(&bar[q], ph[q]);
  }
  return ok;
}

// Ap for the listed rows from the FP64 BCSR with FP64 sums (LPR lanes per
// row); returns this thread's share of p.Ap.
template <typename Tacc, int LPR, bool kTwo>
__device__ __forceinline__ Tacc spmv_rows_listed(const int* __restrict__ rowptr, const int* __restrict__ colidx,
                                                 const double* __restrict__ val64, const int* __restrict__ xrows,
                                                 int nx, const SpmvVec& v)
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
        const P4<float> x = spmv_x<kTwo>(v, __ldg(colidx + t));
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
    if (ok && sub == 0) dot += (double)spmv_store_row<kTwo, double>(v, row, (float)a0, (float)a1, (float)a2);
  }
  return (Tacc)dot;
}

}  // namespace maspcg
