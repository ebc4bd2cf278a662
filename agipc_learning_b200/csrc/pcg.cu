// pcg.cu -- the PCG iteration of PCGSolver::pcg (pcg_solver.cu:192-326) on
// the device.
//
// The reference runs one host-driven iteration with three reduction trees and
// two blocking device-to-host copies.  Here the scalars (rz, alpha, beta, the
// iteration counter and a status word) live on the device, every reduction is
// finished by the last block of the kernel that produces it (fixed order, so
// results are deterministic), and a fixed number of iterations is captured in
// one CUDA graph; once the status leaves RUNNING every later kernel returns at
// entry.  The host reads the status once per graph launch.
//
// Per iteration: p = z + beta p | Ap = A p, p.Ap, alpha | x += alpha p,
// r -= alpha Ap, r.r and the stopping gate | z = M^-1 r, r.z, beta.
// Precision modes: REFERENCE (FP64 matrix/vectors/dots, FP32 MAS), FP32
// (everything FP32), MIXED (FP32 matrix/vectors, 16-bit domain inverses, FP64
// dots, FP64 residual replacement every period with x accumulated in FP64).
#include <algorithm>
#include <cmath>
#include <type_traits>

#include "maspcg_internal.cuh"
#include "pcg_device.cuh"
#include "mas_args.cuh"
#include "spmv_row.cuh"

namespace maspcg {

template <typename Tv, typename Tacc>
void mas_apply(maspcg_handle* h, const Tv* r, Tv* z, Tacc* partial, int part_base, int total_parts, int mode,
               int grid0, PcgScalars* s, bool overlap);

template <typename Tv, typename Tacc>
void mas_level0_only(maspcg_handle* h, const Tv* r, Tv* z, Tacc* partial, int grid0, PcgScalars* s, int variant);
template <typename Tacc>
void mas_apply_fused(maspcg_handle* h, const FusedArgs& fa, float* z, Tacc* partial, double* partial_rr, int part_base,
                     int total_parts, int mode, int grid0, PcgScalars* s, bool overlap);
void launch_factor(maspcg_handle* h, double* assembled_out);
int mas_level0_grid(maspcg_handle* h);
template <typename Tv, typename Tacc>
void mas16_apply(maspcg_handle* h, const Tv* r, Tv* z, Tacc* partial, int part_base, int total_parts, int mode,
                 int grid, PcgScalars* s, bool overlap);
int mas16_grid(maspcg_handle* h);

namespace {

constexpr int kTpb = kRedTpb;

__device__ __forceinline__ bool running(const PcgScalars* s) { return s->status == MASPCG_SOLVE_RUNNING; }

// x = 0, r = b, (x_hi = 0), b.b
template <typename Tv>
__global__ void __launch_bounds__(kTpb) k_init(const double* __restrict__ b, Tv* x, Tv* r, double* xhi, int n,
                                                double* partial, PcgScalars* s)
{
  double acc = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double v = b[i];
    x[i] = Tv(0);
    r[i] = (Tv)v;
    if (xhi) xhi[i] = 0.0;
    acc += v * v;
  }
  double total = 0.0;
  if (grid_finish<double>(acc, partial, blockIdx.x, gridDim.x, &s->tickets[kTicketAux], gridDim.x, total) &&
      threadIdx.x == 0) {
    s->bb = total;
    s->rr_peak = total;
  }
}

// Entries [4q, 4q + 4) of a vector as 16-byte (FP32) / 2 x 16-byte (FP64)
// accesses.
template <typename T>
__device__ __forceinline__ void ld4(const T* p, int q, T o[4])
{
  if constexpr (sizeof(T) == 4) {
    const float4 w = reinterpret_cast<const float4*>(p)[q];
    o[0] = w.x, o[1] = w.y, o[2] = w.z, o[3] = w.w;
  } else {
    const double2 a = reinterpret_cast<const double2*>(p)[2 * q], b = reinterpret_cast<const double2*>(p)[2 * q + 1];
    o[0] = a.x, o[1] = a.y, o[2] = b.x, o[3] = b.y;
  }
}
template <typename T>
__device__ __forceinline__ void st4(T* p, int q, const T o[4])
{
  if constexpr (sizeof(T) == 4) {
    reinterpret_cast<float4*>(p)[q] = make_float4(o[0], o[1], o[2], o[3]);
  } else {
    reinterpret_cast<double2*>(p)[2 * q] = make_double2(o[0], o[1]);
    reinterpret_cast<double2*>(p)[2 * q + 1] = make_double2(o[2], o[3]);
  }
}

// ---- the three steps of one iteration head as device bodies, shared by
// the separate kernels and by the fused cooperative kernel below.

// p = z (k == 1) or z + beta p for the rows this thread strides over, written
// into the padded layout.  With `coarse` the MAS rows first add the coarse
// correction (the overlapped apply leaves it out of z).
template <typename Tv, bool kCoarse>
__device__ __forceinline__ void update_p_rows(const ApplyArgs& a, const Tv* __restrict__ z, Tv* p4, int nrows,
                                              bool first, Tv beta)
{
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < nrows; v += gridDim.x * blockDim.x) {
    Tv z0 = z[3 * (size_t)v], z1 = z[3 * (size_t)v + 1], z2 = z[3 * (size_t)v + 2];
    if (kCoarse) {
      const int slot = v - a.fem_off;
      if (slot >= 0 && slot < a.c0) {
        float cc[3];
        if (coarse_correction(a, slot, cc)) {
          z0 += (Tv)cc[0];
          z1 += (Tv)cc[1];
          z2 += (Tv)cc[2];
        }
      }
    }
    if (first) {
      st_p4(p4, v, z0, z1, z2);
    } else {
      const P4<Tv> o = ld_p4(p4, v);
      st_p4(p4, v, z0 + beta * o.x, z1 + beta * o.y, z2 + beta * o.z);
    }
  }
}

template <typename Tv, bool kCoarse>
__global__ void __launch_bounds__(kTpb) k_update_p(ApplyArgs a, const Tv* __restrict__ z, Tv* p4, int nrows,
                                                    const PcgScalars* s)
{
  pdl_wait();
  if (!running(s)) return;
  update_p_rows<Tv, kCoarse>(a, z, p4, nrows, s->k == 1, (Tv)s->beta);
}

// One 3x3 block of the matrix.  FP32: tiles of 32 blocks stored element-major
// (element e of block t at (t/32)*288 + 32e + t%32), so a warp's element loads
// are coalesced and a tile is one contiguous 1152-byte run.  FP64: row-major
// blocks.
template <bool kTiled, typename Tm>
__device__ __forceinline__ void load_block(const Tm* __restrict__ val, int t, Tm m[9])
{
  if (kTiled) {
    const Tm* b = val + (size_t)(t >> 5) * 288 + (t & 31);
#pragma unroll
    for (int e = 0; e < 9; ++e) m[e] = __ldcs(b + 32 * e);
  } else {
#pragma unroll
    for (int e = 0; e < 9; ++e) m[e] = __ldcs(val + 9 * (size_t)t + e);
  }
}

// The BF16 remainder of an FP32 tile block (MASPCG_MATRIX_F32_SPLIT), at the
// same positions as load_block's tiles.
__device__ __forceinline__ void load_block_lo(const unsigned short* __restrict__ lo, int t, float m[9])
{
  const unsigned short* b = lo + (size_t)(t >> 5) * 288 + (t & 31);
#pragma unroll
  for (int e = 0; e < 9; ++e) m[e] = __uint_as_float((uint32_t)__ldcs(b + 32 * e) << 16);
}

// Accumulator of the SpMV rows: the matrix's own type (FP32 tiles, FP64
// matrix).  The FP32 forms with accurate sums add a low part beside it.
template <typename Tm, int kForm>
using SpmvAcc = typename AccOf<Tm>::type;

// hi + lo += t, the sum's rounding error kept by TwoSum (round-to-nearest
// intrinsics, so the compiler cannot contract the steps).
__device__ __forceinline__ void two_sum_add(float& hi, float& lo, float t)
{
  const float s = __fadd_rn(hi, t);
  const float bp = __fsub_rn(s, hi);
  lo = __fadd_rn(lo, __fadd_rn(__fsub_rn(hi, __fsub_rn(s, bp)), __fsub_rn(t, bp)));
  hi = s;
}

// hi + lo += a b with the product exact and the sum compensated: the
// product's rounding error from one FMA, the sum's from TwoSum (Ogita, Rump
// and Oishi's Dot2), so a row accumulates its products to about 2^-48 of the
// sum of their magnitudes without leaving FP32.  The round-to-nearest
// intrinsics keep the compiler from contracting the steps into FMAs, which
// would change the error terms.
__device__ __forceinline__ void dot2_add(float& hi, float& lo, float a, float b)
{
  const float p = __fmul_rn(a, b);
  const float e = fmaf(a, b, -p);
  const float s = __fadd_rn(hi, p);
  const float bp = __fsub_rn(s, hi);
  const float err = __fadd_rn(__fsub_rn(hi, __fsub_rn(s, bp)), __fsub_rn(p, bp));
  hi = s;
  lo = __fadd_rn(lo, __fadd_rn(err, e));
}

// Ap = A p for block rows [lo, nrows); returns this thread's share of p.Ap.
// LPR lanes per block row and two row groups per thread in flight at once
// (rows r and r + stride); each lane takes kPer blocks of each row per step
// and issues all their loads before the arithmetic.  kForm (FP32 tiles): the
// maspcg_matrix_form, i.e. FP32 sums or compensated sums of exact products
// (dot2_add), and with the split form the BF16 remainder's products added to
// the low parts.
template <typename Tm, typename Tv, typename Tacc, bool kTiled, int LPR, int kForm>
__device__ __forceinline__ Tacc spmv_rows(const int* __restrict__ rowptr, const int* __restrict__ colidx,
                                          const Tm* __restrict__ val, const unsigned short* __restrict__ val_lo,
                                          const Tv* __restrict__ p4, Tv* ap, int lo, int nrows)
{
  using A = SpmvAcc<Tm, kForm>;
  constexpr bool kSplit = kTiled && kForm == MASPCG_MATRIX_F32_SPLIT;
  constexpr bool kDot2 = kTiled && kForm != MASPCG_MATRIX_F32;  // compensated sums (below)
  // COMPENSATED: each block row's three products by an FP32 FMA chain, only
  // the sum across blocks compensated; the other forms: every product exact
  constexpr bool kBlockFma = kForm == MASPCG_MATRIX_F32_COMPENSATED;
  constexpr int kRows = kTpb / LPR;
  const int sub = threadIdx.x % LPR;
  const int step = gridDim.x * kRows;
  Tacc dot = 0;
  // row extents of the first step; each step fetches the next step's
  auto extent = [&](int row, int& b, int& e) {
    const bool ok = row < nrows;
    b = ok ? __ldg(rowptr + row) : 0;
    e = ok ? __ldg(rowptr + row + 1) : 0;
  };
  int nsa, nea, nsb, neb;
  extent(lo + blockIdx.x * kRows + threadIdx.x / LPR, nsa, nea);
  extent(lo + blockIdx.x * kRows + threadIdx.x / LPR + step, nsb, neb);
  constexpr int kPer = 2;
  constexpr int kIn = 2 * kPer;  // blocks in flight per step
  for (int row0 = lo + blockIdx.x * kRows; row0 < nrows; row0 += 2 * step) {
    const int ra = row0 + threadIdx.x / LPR, rb = ra + step;
    const int sa = nsa, ea = nea, sb = nsb, eb = neb;
    extent(ra + 2 * step, nsa, nea);
    extent(rb + 2 * step, nsb, neb);
    A a[2][3] = {{0, 0, 0}, {0, 0, 0}};
    float al[2][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}};  // kDot2: the low parts (and the remainder's products)
    const int na = (ea - sa + kPer * LPR - 1) / (kPer * LPR), nbk = (eb - sb + kPer * LPR - 1) / (kPer * LPR);
    const int steps = max(__reduce_max_sync(kFull, (unsigned)na), __reduce_max_sync(kFull, (unsigned)nbk));
    for (int k = 0; k < steps; ++k) {
      // blocks j < kPer of row a, the rest of row b
      int tt[kIn];
      bool in[kIn];
#pragma unroll
      for (int j = 0; j < kIn; ++j) {
        const int half = j / kPer, i = j % kPer;
        tt[j] = (half ? sb : sa) + sub + kPer * LPR * k + i * LPR;
        in[j] = tt[j] < (half ? eb : ea);
      }
      Tm m[kIn][9];
      int c[kIn];
#pragma unroll
      for (int j = 0; j < kIn; ++j) {
        c[j] = in[j] ? __ldcs(colidx + tt[j]) : 0;
        if (in[j]) {
          load_block<kTiled>(val, tt[j], m[j]);
        } else {
#pragma unroll
          for (int e = 0; e < 9; ++e) m[j][e] = Tm(0);
        }
      }
#pragma unroll
      for (int j = 0; j < kIn; ++j) {
        const P4<Tv> x = ld_p4(p4, c[j]);
        A* o = a[j / kPer];
        if constexpr (kDot2) {
          float* ol = al[j / kPer];
          const float xv[3] = {(float)x.x, (float)x.y, (float)x.z};
#pragma unroll
          for (int i = 0; i < 3; ++i) {
            if constexpr (kBlockFma) {
              two_sum_add(o[i], ol[i], fmaf(m[j][3 * i], xv[0], fmaf(m[j][3 * i + 1], xv[1],
                                                                     __fmul_rn(m[j][3 * i + 2], xv[2]))));
            } else {
#pragma unroll
              for (int t = 0; t < 3; ++t) dot2_add(o[i], ol[i], m[j][3 * i + t], xv[t]);
            }
          }
        } else {
          o[0] += (A)m[j][0] * (A)x.x + (A)m[j][1] * (A)x.y + (A)m[j][2] * (A)x.z;
          o[1] += (A)m[j][3] * (A)x.x + (A)m[j][4] * (A)x.y + (A)m[j][5] * (A)x.z;
          o[2] += (A)m[j][6] * (A)x.x + (A)m[j][7] * (A)x.y + (A)m[j][8] * (A)x.z;
        }
        if constexpr (kSplit) {
          float w[9];
          if (in[j]) {
            load_block_lo(val_lo, tt[j], w);
          } else {
#pragma unroll
            for (int e = 0; e < 9; ++e) w[e] = 0.f;
          }
          float* ol = al[j / kPer];
          ol[0] += w[0] * (float)x.x + w[1] * (float)x.y + w[2] * (float)x.z;
          ol[1] += w[3] * (float)x.x + w[4] * (float)x.y + w[5] * (float)x.z;
          ol[2] += w[6] * (float)x.x + w[7] * (float)x.y + w[8] * (float)x.z;
        }
      }
    }
    // lane partial sums of each row component, added across the row's LPR
    // lanes (in FP64 when the sums are compensated: hi + lo, then exact adds)
    using R = typename std::conditional<kDot2, double, A>::type;
    R u[2][3];
#pragma unroll
    for (int h = 0; h < 2; ++h)
#pragma unroll
      for (int q = 0; q < 3; ++q) u[h][q] = kDot2 ? (R)a[h][q] + (R)al[h][q] : (R)a[h][q];
#pragma unroll
    for (int h = 0; h < 2; ++h)
#pragma unroll
      for (int o = LPR / 2; o > 0; o >>= 1) {
        u[h][0] += __shfl_xor_sync(kFull, u[h][0], o, LPR);
        u[h][1] += __shfl_xor_sync(kFull, u[h][1], o, LPR);
        u[h][2] += __shfl_xor_sync(kFull, u[h][2], o, LPR);
      }
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int row = h ? rb : ra;
      if (row < nrows && sub < 3) {
        const Tv y = (Tv)(sub == 0 ? u[h][0] : (sub == 1 ? u[h][1] : u[h][2]));
        ap[3 * (size_t)row + sub] = y;
        const P4<Tv> pr = ld_p4(p4, row);
        const Tv pv = sub == 0 ? pr.x : (sub == 1 ? pr.y : pr.z);
        dot += (Tacc)pv * (Tacc)y;
      }
    }
  }
  return dot;
}

// Last block of the SpMV: p.Ap and alpha (or a stop on curvature / NaN).
__device__ __forceinline__ void spmv_finish(PcgScalars* s, double pap)
{
  s->pap = pap;
  if (!isfinite(pap)) {
    s->status = MASPCG_SOLVE_NONFINITE;
    s->iterations = s->k;
  } else if (!(pap > 0.0)) {
    s->status = MASPCG_SOLVE_NONPOSITIVE_CURVATURE;
    s->iterations = s->k;
  } else {
    s->alpha = s->rz / pap;
  }
}

// Ap for block rows [0, n64) from the FP64 matrix with FP64 sums, used when
// the iteration runs on the FP32 tiles: these are the affine-body rows, whose
// 12x12 blocks carry the orthogonality stiffness (~1e7 on the diagonal)
// beside rotation modes held only by the mass (~1e-4), a spread FP32 values
// or sums cannot keep positive definite.  A body row also holds the coupling
// blocks of every FEM vertex in contact with the body (tens of blocks), so
// each row takes a whole warp, two blocks per lane per step with all their
// loads issued before the arithmetic.
template <typename Tv, typename Tacc>
__device__ __forceinline__ Tacc spmv_rows_exact(const int* __restrict__ rowptr, const int* __restrict__ colidx,
                                                const double* __restrict__ val64, const Tv* __restrict__ p4, Tv* ap,
                                                int n64)
{
  constexpr int LPR = 32, kPer = 2;
  constexpr int kRows = kTpb / LPR;
  const int lane = threadIdx.x % LPR;
  double dot = 0.0;
  for (int row0 = blockIdx.x * kRows; row0 < n64; row0 += gridDim.x * kRows) {
    const int row = row0 + threadIdx.x / LPR;  // warp-uniform
    double a0 = 0.0, a1 = 0.0, a2 = 0.0;
    if (row < n64) {
      const int rs = __ldg(rowptr + row), re = __ldg(rowptr + row + 1);
      for (int t0 = rs + lane; t0 < re; t0 += kPer * LPR) {
        double m[kPer][9];
        int c[kPer];
#pragma unroll
        for (int j = 0; j < kPer; ++j) {
          const int t = t0 + j * LPR;
          c[j] = t < re ? __ldcs(colidx + t) : 0;
          if (t < re) {
            load_block<false>(val64, t, m[j]);
          } else {
#pragma unroll
            for (int e = 0; e < 9; ++e) m[j][e] = 0.0;
          }
        }
#pragma unroll
        for (int j = 0; j < kPer; ++j) {
          const P4<Tv> x = ld_p4(p4, c[j]);
          a0 += m[j][0] * (double)x.x + m[j][1] * (double)x.y + m[j][2] * (double)x.z;
          a1 += m[j][3] * (double)x.x + m[j][4] * (double)x.y + m[j][5] * (double)x.z;
          a2 += m[j][6] * (double)x.x + m[j][7] * (double)x.y + m[j][8] * (double)x.z;
        }
      }
    }
#pragma unroll
    for (int o = LPR / 2; o > 0; o >>= 1) {
      a0 += __shfl_xor_sync(kFull, a0, o, LPR);
      a1 += __shfl_xor_sync(kFull, a1, o, LPR);
      a2 += __shfl_xor_sync(kFull, a2, o, LPR);
    }
    if (row < n64 && lane < 3) {
      const Tv y = (Tv)(lane == 0 ? a0 : (lane == 1 ? a1 : a2));
      ap[3 * (size_t)row + lane] = y;
      const P4<Tv> pr = ld_p4(p4, row);
      dot += (double)(lane == 0 ? pr.x : (lane == 1 ? pr.y : pr.z)) * (double)y;
    }
  }
  return (Tacc)dot;
}

// Both parts of the product: rows [0, n64) exact (n64 is 0 for the FP64
// matrix), the rest from `val`.
template <typename Tm, typename Tv, typename Tacc, bool kTiled, int LPR, int kForm>
__device__ __forceinline__ Tacc spmv_all(const int* __restrict__ rowptr, const int* __restrict__ colidx,
                                         const Tm* __restrict__ val, const unsigned short* __restrict__ val_lo,
                                         const double* __restrict__ val64, int n64, const Tv* __restrict__ p4,
                                         Tv* ap, int nrows)
{
  Tacc dot = 0;
  if (n64 > 0) dot = spmv_rows_exact<Tv, Tacc>(rowptr, colidx, val64, p4, ap, n64);
  return dot + spmv_rows<Tm, Tv, Tacc, kTiled, LPR, kForm>(rowptr, colidx, val, val_lo, p4, ap, n64, nrows);
}

// Resident CTAs per SM the SpMV asks of the register allocator: three (80
// registers) for the FP32 tiles in every form, two for the FP64 matrix.
template <typename Tm, int kForm>
constexpr int spmv_min_ctas() { return std::is_same<Tm, float>::value ? 3 : 2; }

template <typename Tm, typename Tv, typename Tacc, bool kTiled, int LPR, int kForm>
__global__ void __launch_bounds__(kTpb, spmv_min_ctas<Tm, kForm>()) k_spmv(const int* __restrict__ rowptr, const int* __restrict__ colidx,
                                                const Tm* __restrict__ val, const unsigned short* __restrict__ val_lo,
                                                const double* __restrict__ val64, int n64,
                                                const Tv* __restrict__ p4, Tv* ap, int nrows, Tacc* partial,
                                                PcgScalars* s)
{
  pdl_wait();
  if (!running(s)) return;
  const Tacc dot = spmv_all<Tm, Tv, Tacc, kTiled, LPR, kForm>(rowptr, colidx, val, val_lo, val64, n64, p4, ap, nrows);
  pdl_trigger();
  Tacc total = 0;
  if (grid_finish<Tacc>(dot, partial, blockIdx.x, gridDim.x, &s->tickets[kTicketSpmv], gridDim.x, total) &&
      threadIdx.x == 0)
    spmv_finish(s, (double)total);
}

// x += alpha p, r -= alpha Ap for the entries this thread strides over;
// returns its share of r.r.  Four consecutive entries of x, r and Ap per
// step (16-byte accesses) with the matching entries of the padded p; a
// scalar tail covers n % 4.
template <typename Tv, typename Tacc>
__device__ __forceinline__ Tacc update_xr_rows(Tv* x, Tv* r, const Tv* __restrict__ p4, const Tv* __restrict__ ap,
                                               int nrows, Tv alpha)
{
  Tacc acc = 0;
  const int n = 3 * nrows, n4 = n >> 2;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n4; q += gridDim.x * blockDim.x) {
    Tv xx[4], rr[4], ww[4], pp[4];
    ld4(x, q, xx);
    ld4(r, q, rr);
    ld4(ap, q, ww);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int j = 4 * q + k;
      pp[k] = p4[4 * (j / 3) + j % 3];
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      xx[k] = xx[k] + alpha * pp[k];
      rr[k] = rr[k] - alpha * ww[k];
      acc += (Tacc)rr[k] * (Tacc)rr[k];
    }
    st4(x, q, xx);
    st4(r, q, rr);
  }
  for (int j = 4 * n4 + blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    const Tv pv = p4[4 * (j / 3) + j % 3];
    x[j] = x[j] + alpha * pv;
    const Tv rn = r[j] - alpha * ap[j];
    r[j] = rn;
    acc += (Tacc)rn * (Tacc)rn;
  }
  return acc;
}

template <typename Tv, typename Tacc>
__global__ void __launch_bounds__(kTpb) k_update_xr(Tv* x, Tv* r, const Tv* __restrict__ p4, const Tv* __restrict__ ap,
                                                     int nrows, int mixed, Tacc* partial, PcgScalars* s)
{
  pdl_wait();
  if (!running(s)) return;
  const Tacc acc = update_xr_rows<Tv, Tacc>(x, r, p4, ap, nrows, (Tv)s->alpha);
  pdl_trigger();
  Tacc total = 0;
  if (grid_finish<Tacc>(acc, partial, blockIdx.x, gridDim.x, &s->tickets[kTicketXr], gridDim.x, total) &&
      threadIdx.x == 0)
    gate_check(s, (double)total, mixed);
}

// The iteration head as one cooperative kernel (every CTA resident): the p
// update, a grid barrier, the SpMV with p.Ap and alpha, a grid barrier, the
// x/r update with r.r and the gate.  Saves two kernel boundaries per
// iteration; the barriers are bounded (grid_barrier).
template <typename Tm, typename Tv, typename Tacc, bool kTiled, int LPR, bool kCoarse, int kForm>
__global__ void __launch_bounds__(kTpb) k_iteration_head(ApplyArgs a, const int* __restrict__ rowptr,
                                                          const int* __restrict__ colidx, const Tm* __restrict__ val,
                                                          const unsigned short* __restrict__ val_lo,
                                                          const double* __restrict__ val64, int n64,
                                                          const Tv* __restrict__ z, Tv* p4, Tv* ap, Tv* x, Tv* r,
                                                          int nrows, int mixed, Tacc* partial, PcgScalars* s, int* err)
{
  if (!running(s)) return;  // uniform: no CTA of this launch has written the status yet
  update_p_rows<Tv, kCoarse>(a, z, p4, nrows, s->k == 1, (Tv)s->beta);
  if (!grid_barrier(s, err)) return;
  const Tacc dot = spmv_all<Tm, Tv, Tacc, kTiled, LPR, kForm>(rowptr, colidx, val, val_lo, val64, n64, p4, ap, nrows);
  Tacc total = 0;
  if (grid_finish<Tacc>(dot, partial, blockIdx.x, gridDim.x, &s->tickets[kTicketSpmv], gridDim.x, total) &&
      threadIdx.x == 0)
    spmv_finish(s, (double)total);
  if (!grid_barrier(s, err)) return;
  // status and alpha were written by another CTA before the barrier: read
  // them past L1 (this CTA cached the scalars' line at entry)
  if (__ldcg(&s->status) != MASPCG_SOLVE_RUNNING) return;  // uniform
  const Tacc acc = update_xr_rows<Tv, Tacc>(x, r, p4, ap, nrows, (Tv)__ldcg(&s->alpha));
  total = 0;
  if (grid_finish<Tacc>(acc, partial, blockIdx.x, gridDim.x, &s->tickets[kTicketXr], gridDim.x, total) &&
      threadIdx.x == 0)
    gate_check(s, (double)total, mixed);
}

// The end of one batch inside the device-side solve loop: run the next batch
// while the solve is running and the batch cap is not reached.
__global__ void k_loop_condition(cudaGraphConditionalHandle handle, PcgScalars* s)
{
  const int n = ++s->graph_launches;
  cudaGraphSetConditional(handle, (s->status == MASPCG_SOLVE_RUNNING && n < s->max_launches) ? 1u : 0u);
}

// MIXED: fold the FP32 correction into the FP64 iterate.
__global__ void __launch_bounds__(kTpb) k_fold_x(double* xhi, float* xlo, int n, int force, const PcgScalars* s)
{
  pdl_wait();
  if (!force && !(s->status == MASPCG_SOLVE_RUNNING || s->status == kNeedTrue)) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    xhi[i] += (double)xlo[i];
    xlo[i] = 0.f;
  }
}

// MIXED, at the end of each graph of refinement_period iterations: is the
// recursive residual replaced by the FP64 true residual now?  Always when the
// recursive gate was met (kNeedTrue: the true residual decides the stop).
// MASPCG_REPLACE_PERIODIC: at every graph end.  MASPCG_REPLACE_RELIABLE: once
// ||r|| has fallen to kReliableDrop of the largest ||r|| since the last
// replacement (a reliable update in the sense of Sleijpen and van der Vorst,
// 1996): each replacement perturbs the Krylov recurrence by the gap between
// the recursive and the true residual, so it is made where the residual has
// shrunk enough that the gap is worth closing, a few times per decade of
// reduction rather than every period.  Read at entry by both kernels of the
// step; neither writes the scalars before its last block.
constexpr double kReliableDrop = 0.1;
__device__ __forceinline__ bool replace_due(const PcgScalars* s)
{
  if (s->status == kNeedTrue) return true;
  if (s->status != MASPCG_SOLVE_RUNNING) return false;
  return s->replace_mode == MASPCG_REPLACE_PERIODIC || s->rr <= kReliableDrop * kReliableDrop * s->rr_peak;
}

// MIXED: r = b - A x_hi in FP64 with the FP64 matrix; FP32 copy for the
// iteration; last block: stop on the true residual or resume.
template <int LPR>
__global__ void __launch_bounds__(kTpb) k_true_residual(const int* __restrict__ rowptr, const int* __restrict__ colidx,
                                                         const double* __restrict__ val, const double* __restrict__ xhi,
                                                         const double* __restrict__ b, float* r32, float* r32b,
                                                         int nrows, double* partial, PcgScalars* s)
{
  pdl_wait();
  if (!replace_due(s)) return;
  (void)r32b;
  const int groups_per_block = kTpb / LPR;
  const int sub = threadIdx.x % LPR;
  double acc2 = 0.0;
  const int iters = (nrows + gridDim.x * groups_per_block - 1) / (gridDim.x * groups_per_block);
  for (int it = 0; it < iters; ++it) {
    const int row = (it * gridDim.x + blockIdx.x) * groups_per_block + threadIdx.x / LPR;
    const bool ok = row < nrows;
    const int rs = ok ? rowptr[row] : 0, re = ok ? rowptr[row + 1] : 0;
    double acc[3];
    row_product<double, double, LPR>(rs, re, colidx, val, xhi, sub, acc);
    if (ok && sub < 3) {
      const double v = b[3 * (size_t)row + sub] - acc[sub];
      r32[3 * (size_t)row + sub] = (float)v;
      acc2 += v * v;
    }
  }
  pdl_trigger();
  double total = 0.0;
  if (grid_finish<double>(acc2, partial, blockIdx.x, gridDim.x, &s->tickets[kTicketTrue], gridDim.x, total) &&
      threadIdx.x == 0) {
    s->rr_true = total;
    s->rr = total;
    s->rr_peak = total;
    s->refinements += 1;
    s->rbuf = 0;  // the replaced residual lives in the first r buffer
    if (!isfinite(total)) {
      s->status = MASPCG_SOLVE_NONFINITE;
      s->iterations = s->k;
    } else if (total <= s->tol * s->tol * s->bb) {
      s->status = MASPCG_SOLVE_CONVERGED;
      s->iterations = s->k;
    } else {
      s->status = MASPCG_SOLVE_RUNNING;
    }
  }
}

// Rows outside the MAS range: affine bodies (12x12 inverse), the 3x3
// block-Jacobi rows, identity elsewhere (global_linear_system.cu:293-306).
// When `finalize` is set this kernel completes the r.z reduction.
template <typename Tv, typename Tacc, typename Tinv>
__global__ void __launch_bounds__(kTpb) k_other_apply(const Tv* __restrict__ r, Tv* z, int nb_int, int mas_lo,
                                                       int mas_hi, int bodies, const Tinv* __restrict__ abd_inv,
                                                       const Tinv* __restrict__ diag_inv, Tacc* partial, int part_base,
                                                       int total_parts, int finalize, int mode, PcgScalars* s)
{
  pdl_wait();
  if (s && s->status != MASPCG_SOLVE_RUNNING) return;
  Tacc dot = 0;
  const int stride = gridDim.x * blockDim.x;
  // bodies: one thread per body
  for (int bdy = blockIdx.x * blockDim.x + threadIdx.x; bdy < bodies; bdy += stride) {
    const Tinv* P = abd_inv + 144 * (size_t)bdy;
    Tv in[12];
#pragma unroll
    for (int c = 0; c < 12; ++c) in[c] = r[12 * (size_t)bdy + c];
#pragma unroll 1
    for (int a = 0; a < 12; ++a) {
      Tinv acc = 0;
#pragma unroll
      for (int c = 0; c < 12; ++c) acc += P[12 * a + c] * (Tinv)in[c];
      z[12 * (size_t)bdy + a] = (Tv)acc;
      dot += (Tacc)in[a] * (Tacc)(Tv)acc;
    }
  }
  // remaining rows
  const int first = 4 * bodies;
  for (int row = first + blockIdx.x * blockDim.x + threadIdx.x; row < nb_int; row += stride) {
    if (row >= mas_lo && row < mas_hi) continue;
    const Tv r0 = r[3 * (size_t)row], r1 = r[3 * (size_t)row + 1], r2 = r[3 * (size_t)row + 2];
    Tv z0 = r0, z1 = r1, z2 = r2;
    if (diag_inv) {
      const Tinv* D = diag_inv + 9 * (size_t)row;
      z0 = (Tv)(D[0] * (Tinv)r0 + D[1] * (Tinv)r1 + D[2] * (Tinv)r2);
      z1 = (Tv)(D[3] * (Tinv)r0 + D[4] * (Tinv)r1 + D[5] * (Tinv)r2);
      z2 = (Tv)(D[6] * (Tinv)r0 + D[7] * (Tinv)r1 + D[8] * (Tinv)r2);
    }
    z[3 * (size_t)row] = z0;
    z[3 * (size_t)row + 1] = z1;
    z[3 * (size_t)row + 2] = z2;
    dot += (Tacc)r0 * (Tacc)z0 + (Tacc)r1 * (Tacc)z1 + (Tacc)r2 * (Tacc)z2;
  }
  if (!partial) return;
  if (!finalize) {
    __shared__ Tacc red[kTpb / 32];
    const Tacc bsum = block_sum<Tacc, kTpb>(dot, red);
    if (threadIdx.x == 0) partial[part_base + blockIdx.x] = bsum;
    return;
  }
  pdl_trigger();
  Tacc total = 0;
  if (grid_finish<Tacc>(dot, partial, part_base + blockIdx.x, total_parts, &s->tickets[kTicketRz], gridDim.x, total) &&
      threadIdx.x == 0 && mode > 0)
    rz_update(s, (double)total, mode);
}

// y = b - y (in place), ||y||^2
__global__ void __launch_bounds__(kTpb) k_residual_norm(const double* __restrict__ b, double* y, int n, double* partial,
                                                         PcgScalars* s)
{
  double acc = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double v = b[i] - y[i];
    y[i] = v;
    acc += v * v;
  }
  double total = 0.0;
  if (grid_finish<double>(acc, partial, blockIdx.x, gridDim.x, &s->tickets[kTicketAux], gridDim.x, total) &&
      threadIdx.x == 0)
    s->rr_true = total;
}

template <typename Tv>
__global__ void k_to_f64(const Tv* __restrict__ x, double* y, int n)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] = (double)x[i];
}

template <typename Tv>
__global__ void k_from_f64(const double* __restrict__ x, Tv* y, int n)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] = (Tv)x[i];
}

// FP64 vector (3 per block row) into the padded search-direction layout.
template <typename Tv>
__global__ void k_to_p4(const double* __restrict__ x, Tv* p4, int nrows)
{
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v < nrows) st_p4(p4, v, (Tv)x[3 * (size_t)v], (Tv)x[3 * (size_t)v + 1], (Tv)x[3 * (size_t)v + 2]);
}

// Reads `n` 16-byte words through L2 (evicting what was cached) without
// dirtying any line; writes only if the data is nonzero (never, in use).
__global__ void __launch_bounds__(kTpb) k_l2_evict(const uint4* __restrict__ p, size_t n, unsigned* sink)
{
  unsigned acc = 0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const uint4 v = __ldcg(p + i);
    acc |= v.x | v.y | v.z | v.w;
  }
  if (acc == 0xffffffffu) *sink = acc;
}

// Rows outside the MAS range behind the iteration's fused x / r update
// (fa.update): the update of the row, then its preconditioner (affine bodies:
// 12x12 inverse; other rows: identity, as in the reference) into z; per-CTA
// r.z and r.r partials (the level-0 apply completes both).
template <typename Tacc, typename Tinv>
__global__ void __launch_bounds__(kTpb) k_other_apply_fused(FusedArgs fa, float* z, int nb_int, int mas_lo,
                                                             int mas_hi, int bodies, const Tinv* __restrict__ abd_inv,
                                                             Tacc* partial, double* partial_rr, PcgScalars* s)
{
  pdl_wait();
  if (s->status != MASPCG_SOLVE_RUNNING) return;
  const FusedScal fs = fused_scalars(s);
  Tacc dot = 0;
  double rr = 0.0;
  const int stride = gridDim.x * blockDim.x;
  for (int bdy = blockIdx.x * blockDim.x + threadIdx.x; bdy < bodies; bdy += stride) {
    const Tinv* P = abd_inv + 144 * (size_t)bdy;
    float in[12];
#pragma unroll
    for (int q = 0; q < 4; ++q) fused_input_row(fa, fs, 4 * bdy + q, true, in + 3 * q);
#pragma unroll 1
    for (int a = 0; a < 12; ++a) {
      Tinv acc = 0;
#pragma unroll
      for (int col = 0; col < 12; ++col) acc += P[12 * a + col] * (Tinv)in[col];
      const float zv = (float)acc;
      z[12 * (size_t)bdy + a] = zv;
      dot += (Tacc)in[a] * (Tacc)zv;
      rr += (double)in[a] * in[a];
    }
  }
  for (int row = 4 * bodies + blockIdx.x * blockDim.x + threadIdx.x; row < nb_int; row += stride) {
    if (row >= mas_lo && row < mas_hi) continue;
    float r3[3];
    fused_input_row(fa, fs, row, true, r3);
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      z[3 * (size_t)row + i] = r3[i];
      dot += (Tacc)r3[i] * (Tacc)r3[i];
      rr += (double)r3[i] * r3[i];
    }
  }
  __shared__ Tacc red[kTpb / 32];
  __shared__ double red2[kTpb / 32];
  const Tacc bsum = block_sum<Tacc, kTpb>(dot, red);
  const double bsum2 = block_sum<double, kTpb>(rr, red2);
  if (threadIdx.x == 0) {
    partial[blockIdx.x] = bsum;
    if (fa.update) partial_rr[blockIdx.x] = bsum2;
  }
}

// The x / r update of the last iteration of a MIXED batch, whose FP64
// residual replacement comes between the update and the apply: r' of the
// current buffer into the first one, x, r.r and the stopping gate.
template <typename Tacc>
__global__ void __launch_bounds__(kTpb) k_update_xr_fused(FusedArgs fa, int nrows, int mixed, Tacc* partial,
                                                           PcgScalars* s)
{
  pdl_wait();
  if (s->status != MASPCG_SOLVE_RUNNING) return;
  const FusedScal fs = fused_scalars(s);
  Tacc acc = 0;
  for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < nrows; row += gridDim.x * blockDim.x) {
    const size_t b = 3 * (size_t)row;
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      const float rq = fmaf(-fs.alpha, fa.ap[b + q], fa.r[fs.cur][b + q]);
      fa.x[b + q] = fmaf(fs.alpha, fa.p4[4 * (size_t)row + q], fa.x[b + q]);
      fa.r[0][b + q] = rq;
      acc += (Tacc)rq * (Tacc)rq;
    }
  }
  pdl_trigger();
  Tacc total = 0;
  if (grid_finish<Tacc>(acc, partial, blockIdx.x, gridDim.x, &s->tickets[kTicketXr], gridDim.x, total) &&
      threadIdx.x == 0) {
    s->rbuf = 0;
    gate_check(s, (double)total, mixed);
  }
}

// ----------------------------------------------------------------- engine --

// Everything a captured solve graph depends on besides device data: the
// buffer allocation count (addresses), the stream, the sizes, the level table
// of the hierarchy, the configuration and the launch options.  A graph is
// re-captured only when this changes (or graph_dirty is set), so a Newton
// step that refreshes values or rebuilds the preconditioner on the same
// structure reuses it.
std::vector<unsigned long long> graph_signature(const maspcg_handle* h)
{
  std::vector<unsigned long long> s = {g_buf_epoch.load(), (unsigned long long)(uintptr_t)h->stream,
                                       (unsigned long long)h->nb, (unsigned long long)h->nb_int,
                                       (unsigned long long)h->n_in, (unsigned long long)h->nnzb,
                                       (unsigned long long)h->fem_off, (unsigned long long)h->abd_bodies,
                                       (unsigned long long)h->c0, (unsigned long long)h->mas_layout,
                                       (unsigned long long)h->has_precond, (unsigned long long)h->use_pdl,
                                       (unsigned long long)h->fused_head, (unsigned long long)h->overlap_coarse,
                                       (unsigned long long)h->apply_variant, (unsigned long long)h->fuse_update,
                                       (unsigned long long)h->nv, (unsigned long long)h->bank};
  auto bytes = [&s](const void* p, size_t n) {
    const unsigned char* c = static_cast<const unsigned char*>(p);
    for (size_t i = 0; i < n; i += 8) {
      unsigned long long w = 0;
      std::memcpy(&w, c + i, std::min<size_t>(8, n - i));
      s.push_back(w);
    }
  };
  bytes(&h->cfg, sizeof(h->cfg));
  bytes(&h->lv, sizeof(h->lv));
  return s;
}

template <typename Tm, typename Tv, typename Tacc>
struct Engine {
  maspcg_handle* h;
  int n, gstream, gspmv, grows, gl0, gother, parts_other, parts_total;
  bool mas, mas16, mixed, ovl;
  bool fused;  // the x / r update runs inside the apply kernels (FP32 matrix, MAS32)

  explicit Engine(maspcg_handle* hh) : h(hh)
  {
    n = 3 * h->nb_int;
    mas = h->mas_layout && h->cfg.preconditioner == MASPCG_PRECOND_MAS32;
    mas16 = h->mas_layout && h->cfg.preconditioner == MASPCG_PRECOND_MAS16;
    mixed = h->cfg.precision == MASPCG_PREC_MIXED;
    gstream = h->grid_stream;
    gspmv = std::max(1, std::min(ceil_div(h->nb_int, kTpb / 16), 4 * h->sm_count));
    grows = std::max(1, std::min(ceil_div(h->nb_int, kTpb), 8 * h->sm_count));
    gl0 = mas ? mas_level0_grid(h) : (mas16 ? mas16_grid(h) : 0);
    ovl = (mas || mas16) && h->lv.levelnum > 1 && h->overlap_coarse;
    const bool other = !(mas || mas16) || h->abd_bodies > 0 || h->fem_off > 0 || h->nb_int > h->fem_off + h->c0;
    gother = other ? std::max(1, std::min(ceil_div(std::max(h->nb_int, 1), kTpb), 2 * h->sm_count)) : 0;
    parts_other = gother;
    parts_total = gother + gl0;
    fused = std::is_same<Tm, float>::value && mas && h->fuse_update && !h->fused_head;
  }
  Tv* V(maspcg::DBuf<unsigned char>& b) { return reinterpret_cast<Tv*>(b.get()); }
  static float* Vf(maspcg::DBuf<unsigned char>& b) { return reinterpret_cast<float*>(b.get()); }
  Tacc* partial() { return reinterpret_cast<Tacc*>(h->partial.get()); }
  Tacc* partial_rz() { return reinterpret_cast<Tacc*>(h->partial_rz.get()); }

  FusedArgs fused_args(int update)
  {
    FusedArgs f{};
    f.p4 = Vf(h->vp4);
    f.ap = Vf(h->vap);
    f.x = Vf(h->vx);
    f.r[0] = Vf(h->vr);
    f.r[1] = Vf(h->vr2);
    f.update = update;
    return f;
  }

  // The preconditioner apply behind the iteration's fused x / r update
  // (mode: RzMode).
  void fused_precondition(int mode, PcgScalars* s)
  {
    const FusedArgs f = fused_args(1);
    if (gother) {
      const int bodies = h->abd_bodies;
      const int mas_lo = h->fem_off, mas_hi = h->fem_off + h->c0;
      if (bodies > 0)
        launch_pdl(h, k_other_apply_fused<Tacc, double>, dim3(gother), dim3(kTpb), 0, f, Vf(h->vz), h->nb_int, mas_lo,
                   mas_hi, bodies, (const double*)h->abd_inv64.get(), partial_rz(), h->partial_rr.get(), s);
      else
        launch_pdl(h, k_other_apply_fused<Tacc, float>, dim3(gother), dim3(kTpb), 0, f, Vf(h->vz), h->nb_int, mas_lo,
                   mas_hi, bodies, (const float*)h->abd_inv32.get(), partial_rz(), h->partial_rr.get(), s);
    }
    mas_apply_fused<Tacc>(h, f, Vf(h->vz), partial_rz(), h->partial_rr.get(), parts_other, parts_total, mode, gl0, s,
                          ovl);
    MCK(cudaGetLastError());
  }

  // overlap: the coarse levels run beside the level-0 apply and z leaves the
  // coarse correction to the next p update (inside the solve only).
  void precondition(const Tv* r, Tv* z, int mode, PcgScalars* s, bool overlap = false)
  {
    const bool ref = h->cfg.precision == MASPCG_PREC_REFERENCE;
    if (gother) {
      const bool bj = h->cfg.preconditioner == MASPCG_PRECOND_BLOCK_JACOBI;
      const bool any_mas = mas || mas16;
      const int mas_lo = any_mas ? h->fem_off : 0, mas_hi = any_mas ? h->fem_off + h->c0 : 0;
      const int bodies = (h->cfg.preconditioner == MASPCG_PRECOND_NONE) ? 0 : h->abd_bodies;
      // affine bodies always apply their FP64 inverses: the 12x12 inverse
      // spans the same ~1e11 spread as the body's Hessian block
      if (ref || bodies > 0)
        launch_pdl(h, k_other_apply<Tv, Tacc, double>, dim3(gother), dim3(kTpb), 0, 
            r, z, h->nb_int, mas_lo, mas_hi, bodies, h->abd_inv64.get(), bj ? h->diag_inv64.get() : nullptr,
            s ? partial_rz() : nullptr, 0, parts_total, any_mas ? 0 : 1, mode, s);
      else
        launch_pdl(h, k_other_apply<Tv, Tacc, float>, dim3(gother), dim3(kTpb), 0, 
            r, z, h->nb_int, mas_lo, mas_hi, bodies, h->abd_inv32.get(), bj ? h->diag_inv32.get() : nullptr,
            s ? partial_rz() : nullptr, 0, parts_total, any_mas ? 0 : 1, mode, s);
    }
    if (mas) mas_apply<Tv, Tacc>(h, r, z, s ? partial_rz() : nullptr, parts_other, parts_total, mode, gl0, s, overlap);
    if (mas16)
      mas16_apply<Tv, Tacc>(h, r, z, s ? partial_rz() : nullptr, parts_other, parts_total, mode, gl0, s, overlap);
    MCK(cudaGetLastError());
  }

  void iteration_head(PcgScalars* s)
  {
    if (h->fused_head) {
      fused_head(s);
      return;
    }
    const ApplyArgs a = ovl ? mas_apply_args(h) : ApplyArgs{};
    if (ovl)
      launch_pdl(h, k_update_p<Tv, true>, dim3(grows), dim3(kTpb), 0, a, V(h->vz), V(h->vp4), h->nb_int, s);
    else
      launch_pdl(h, k_update_p<Tv, false>, dim3(grows), dim3(kTpb), 0, a, V(h->vz), V(h->vp4), h->nb_int, s);
    spmv(s);
    launch_pdl(h, k_update_xr<Tv, Tacc>, dim3(grows), dim3(kTpb), 0, V(h->vx), V(h->vr), V(h->vp4), V(h->vap),
               h->nb_int, mixed ? 1 : 0, partial(), s);
  }

  // The iteration head as one cooperative launch: one resident wave of CTAs.
  template <bool kCoarse, int kForm>
  void fused_head_t(PcgScalars* s, const ApplyArgs& a)
  {
    constexpr bool kTiled = std::is_same<Tm, float>::value;
    auto kern = k_iteration_head<Tm, Tv, Tacc, kTiled, kSpmvLanes, kCoarse, kForm>;
    static int per_sm = 0;
    if (!per_sm) {
      MCK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kTpb, 0));
      MREQ(per_sm > 0, MASPCG_ERR_CUDA, "fused iteration kernel cannot be resident");
    }
    const int grid = std::max(1, std::min(ceil_div(h->nb_int, kTpb / kSpmvLanes), per_sm * h->sm_count));
    launch_cooperative(h, kern, dim3(grid), dim3(kTpb), 0, a, h->rowptr.get(), h->colidx.get(), matrix(),
                       matrix_lo(), h->val64.get(), exact_rows(), V(h->vz), V(h->vp4), V(h->vap), V(h->vx), V(h->vr), h->nb_int, mixed ? 1 : 0, partial(), s,
                       h->failed.get() + 4);
  }

  template <int kForm>
  void fused_head_f(PcgScalars* s)
  {
    if (ovl)
      fused_head_t<true, kForm>(s, mas_apply_args(h));
    else
      fused_head_t<false, kForm>(s, ApplyArgs{});
  }

  void fused_head(PcgScalars* s)
  {
    switch (form()) {
      case MASPCG_MATRIX_F32_ACCURATE: fused_head_f<MASPCG_MATRIX_F32_ACCURATE>(s); break;
      case MASPCG_MATRIX_F32_COMPENSATED: fused_head_f<MASPCG_MATRIX_F32_COMPENSATED>(s); break;
      case MASPCG_MATRIX_F32_SPLIT: fused_head_f<MASPCG_MATRIX_F32_SPLIT>(s); break;
      default: fused_head_f<MASPCG_MATRIX_F32>(s); break;
    }
  }

  const Tm* matrix();
  // the BF16 remainder of the split form (else unused)
  const unsigned short* matrix_lo() const { return h->val_lo.get(); }
  // the matrix form the FP32 tiles run in; the FP64 matrix has one form
  int form() const { return std::is_same<Tm, float>::value ? h->cfg.matrix_form : (int)MASPCG_MATRIX_F32; }
  // block rows the FP32-tile SpMV takes from the FP64 matrix (the affine bodies)
  int exact_rows() const { return std::is_same<Tm, float>::value ? 4 * h->abd_bodies : 0; }

  // SpMV rows per CTA step: kTpb / kSpmvLanes.
  static constexpr int kSpmvLanes = 8;

  template <int kForm>
  void spmv_t(PcgScalars* s)
  {
    constexpr bool kTiled = std::is_same<Tm, float>::value;
    constexpr int rows = kTpb / kSpmvLanes;
    auto kern = k_spmv<Tm, Tv, Tacc, kTiled, kSpmvLanes, kForm>;
    // one wave of resident CTAs; the kernel strides over the rest
    static int per_sm = 0;
    if (!per_sm) {
      MCK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kTpb, 0));
      per_sm = std::max(per_sm, 1);
    }
    const int grid = std::max(1, std::min(ceil_div(h->nb_int, rows), per_sm * h->sm_count));
    launch_pdl(h, kern, dim3(grid), dim3(kTpb), 0, h->rowptr.get(), h->colidx.get(), matrix(), matrix_lo(),
               h->val64.get(), exact_rows(), V(h->vp4), V(h->vap), h->nb_int, partial(), s);
  }

  void spmv(PcgScalars* s)
  {
    if constexpr (std::is_same<Tm, float>::value) {
      switch (form()) {
        case MASPCG_MATRIX_F32_ACCURATE: spmv_t<MASPCG_MATRIX_F32_ACCURATE>(s); return;
        case MASPCG_MATRIX_F32_SPLIT: spmv_t<MASPCG_MATRIX_F32_SPLIT>(s); return;
        case MASPCG_MATRIX_F32_COMPENSATED: spmv_t<MASPCG_MATRIX_F32_COMPENSATED>(s); return;
        default: break;
      }
    }
    spmv_t<MASPCG_MATRIX_F32>(s);
  }



  void true_residual(PcgScalars* s)
  {
    launch_pdl(h, k_fold_x, dim3(gstream), dim3(kTpb), 0, h->x64.get(), reinterpret_cast<float*>(h->vx.get()), n, 0, s);
    launch_pdl(h, k_true_residual<16>, dim3(gspmv), dim3(kTpb), 0, h->rowptr.get(), h->colidx.get(), h->val64.get(),
               h->x64.get(), h->b64.get(), reinterpret_cast<float*>(h->vr.get()),
               (float*)nullptr, h->nb_int, h->partial.get(), s);
  }

  // y = A x through the iteration's own SpMV kernel: x (internal order, FP64)
  // rounded into the padded search-direction layout, the kernel run once,
  // its working-precision output widened into y.
  void spmv_working(const double* x_int, double* y_int)
  {
    cudaStream_t st = h->stream;
    PcgScalars* s = h->scal.get();
    PcgScalars init{};
    init.status = MASPCG_SOLVE_RUNNING;
    init.k = 2;
    init.rz = 1.0;
    init.max_iter = 1 << 30;
    MCK(cudaMemcpyAsync(s, &init, sizeof(init), cudaMemcpyHostToDevice, st));
    k_to_p4<Tv><<<ceil_div(h->nb_int, kTpb), kTpb, 0, st>>>(x_int, V(h->vp4), h->nb_int);
    MLAUNCHED(h);
    const bool pdl = h->use_pdl;
    h->use_pdl = false;
    spmv(s);
    h->use_pdl = pdl;
    k_to_f64<Tv><<<ceil_div(n, kTpb), kTpb, 0, st>>>(V(h->vap), y_int, n);
    MLAUNCHED(h);
    MCK(cudaGetLastError());
  }

  // The solve loop as one graph: a conditional WHILE node whose body is one
  // batch followed by k_loop_condition, so the batches repeat on the device
  // with no host round trip between them.  Where the driver does not take a
  // conditional node, the graph is the batch alone and the host relaunches
  // it after each status read.
  void build_graph(int batch, PcgScalars* s)
  {
    cudaStream_t st = h->stream;
    if (h->graph_exec) cudaGraphExecDestroy(h->graph_exec);
    h->graph_exec = nullptr;
    h->graph_loop = false;
    const long long launches_before = h->kernel_launches;
    auto capture = [&](cudaGraph_t into, cudaGraphConditionalHandle handle, bool loop) -> cudaGraph_t {
      cudaGraph_t g = nullptr;
      if (loop)
        MCK(cudaStreamBeginCaptureToGraph(st, into, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
      else
        MCK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
      try {
        record_batch(batch, s);
        if (loop) {
          k_loop_condition<<<1, 1, 0, st>>>(handle, s);
          MLAUNCHED(h);
          MCK(cudaGetLastError());
        }
      } catch (...) {
        cudaStreamEndCapture(st, &g);
        if (g && !loop) cudaGraphDestroy(g);
        h->kernel_launches = launches_before;
        throw;
      }
      MCK(cudaStreamEndCapture(st, &g));
      return g;
    };
    cudaGraph_t parent = nullptr;
    bool loop = (h->cfg.flags & MASPCG_FLAG_HOST_LOOP) == 0 && cudaGraphCreate(&parent, 0) == cudaSuccess;
    cudaGraphConditionalHandle handle{};
    cudaGraph_t body = nullptr;
    if (loop) {
      cudaGraphNodeParams p{};
      p.type = cudaGraphNodeTypeConditional;
      cudaGraphNode_t node;
      loop = cudaGraphConditionalHandleCreate(&handle, parent, 1, cudaGraphCondAssignDefault) == cudaSuccess;
      if (loop) {
        p.conditional.handle = handle;
        p.conditional.type = cudaGraphCondTypeWhile;
        p.conditional.size = 1;
        loop = cudaGraphAddNode(&node, parent, nullptr, 0, &p) == cudaSuccess;
        if (loop) body = p.conditional.phGraph_out[0];
      }
      if (!loop) {
        cudaGetLastError();  // the driver does not take conditional nodes: the host loop it is
        cudaGraphDestroy(parent);
        parent = nullptr;
      }
    }
    cudaGraph_t g = loop ? (capture(body, handle, true), parent) : capture(nullptr, handle, false);
    h->graph_kernels = h->kernel_launches - launches_before;
    h->kernel_launches = launches_before;
    const cudaError_t e = cudaGraphInstantiate(&h->graph_exec, g, 0);
    cudaGraphDestroy(g);
    MCK(e);
    h->graph_loop = loop;
    h->graph_batch = batch;
    h->graph_dirty = false;
    h->graph_sig = graph_signature(h);
    ++h->graph_captures;
  }

  // One graph = `batch` iterations.
  void record_batch(int batch, PcgScalars* s)
  {
    for (int it = 0; it < batch; ++it) {
      if (fused) {
        const ApplyArgs a = ovl ? mas_apply_args(h) : ApplyArgs{};
        if (ovl)
          launch_pdl(h, k_update_p<Tv, true>, dim3(grows), dim3(kTpb), 0, a, V(h->vz), V(h->vp4), h->nb_int, s);
        else
          launch_pdl(h, k_update_p<Tv, false>, dim3(grows), dim3(kTpb), 0, a, V(h->vz), V(h->vp4), h->nb_int, s);
        spmv(s);
        if (mixed && it == batch - 1) {
          // x / r update, FP64 residual replacement, then the apply of the new r
          launch_pdl(h, k_update_xr_fused<Tacc>, dim3(grows), dim3(kTpb), 0, fused_args(1), h->nb_int, 1, partial(),
                     s);
          true_residual(s);
          precondition(V(h->vr), V(h->vz), 2, s, ovl);
        } else {
          fused_precondition(mixed ? kRzFusedMix : kRzFusedStd, s);
        }
        continue;
      }
      iteration_head(s);
      if (mixed && it == batch - 1) true_residual(s);
      precondition(V(h->vr), V(h->vz), 2, s, ovl);
    }
  }

  // Mean device time of one stage over `repeats` launches.  Before every
  // launch a 256 MB zero buffer is read through L2 (clean lines only, so the
  // timed launch pays no write-back), so each launch starts cold as it does
  // inside the solve, where the SpMV streams more than L2 between two
  // applies.  The stage's time is (evict + stage) x repeats minus
  // evict x repeats, each pair of events around a back-to-back sequence, so
  // no per-launch event overhead is counted.  Programmatic dependent launch
  // is off while timing.
  double time_stage(int stage, int repeats)
  {
    cudaStream_t st = h->stream;
    PcgScalars* s = h->scal.get();
    PcgScalars init{};
    init.status = MASPCG_SOLVE_RUNNING;
    init.k = 2;
    init.rz = 1.0;
    init.rz0 = 1.0;
    init.max_iter = 1 << 30;
    init.tol = 0.0;
    init.gate = MASPCG_GATE_EUCLID;
    MREQ(stage != 3 || mas || mas16, MASPCG_ERR_NOT_READY, "stage 3 needs a MAS preconditioner");
    MREQ(stage != 2 || mas, MASPCG_ERR_NOT_READY, "stage 2 needs a MAS32 preconditioner");
    MREQ(stage < 4 || stage > 6 || mas, MASPCG_ERR_NOT_READY, "stages 4-6 need a MAS32 preconditioner");
    MREQ(stage != 7 || mixed, MASPCG_ERR_NOT_READY, "stage 7 needs the mixed precision");
    MREQ(stage >= 0 && stage <= 7, MASPCG_ERR_INVALID_ARGUMENT, "unknown stage");
    constexpr size_t kFlushBytes = 256u << 20;
    if (h->l2_flush.n < kFlushBytes) {
      h->l2_flush.resize(kFlushBytes);
      MCK(cudaMemsetAsync(h->l2_flush.get(), 0, kFlushBytes, st));
    }
    MCK(cudaMemcpyAsync(s, &init, sizeof(init), cudaMemcpyHostToDevice, st));
    auto once = [&]() {
      switch (stage) {
        case 0: spmv(s); break;
        case 1: precondition(V(h->vr), V(h->vz), 0, s); break;
        case 2: mas_level0_only<Tv, Tacc>(h, V(h->vr), V(h->vz), partial_rz(), gl0, s, -1); break;
        case 3: launch_factor(h, nullptr); break;
        case 7: true_residual(s); break;
        default: mas_level0_only<Tv, Tacc>(h, V(h->vr), V(h->vz), partial_rz(), gl0, s, stage == 6 ? 0 : stage - 3);
      }
    };
    const bool pdl = h->use_pdl;
    h->use_pdl = false;
    auto evict = [&]() {
      k_l2_evict<<<4 * h->sm_count, kTpb, 0, st>>>(reinterpret_cast<const uint4*>(h->l2_flush.get()),
                                                   kFlushBytes / 16, reinterpret_cast<unsigned*>(h->l2_flush.get()));
      MLAUNCHED(h);
    };
    auto timed = [&](bool with_stage) {
      MCK(cudaEventRecord(h->ev0, st));
      for (int i = 0; i < repeats; ++i) {
        evict();
        if (with_stage) once();
      }
      MCK(cudaEventRecord(h->ev1, st));
      MCK(cudaEventSynchronize(h->ev1));
      float ms = 0.f;
      MCK(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
      return (double)ms;
    };
    double total = 0.0;
    try {
      once();  // warm
      evict();
      const double both = timed(true);
      const double alone = timed(false);
      total = std::max(0.0, both - alone);
    } catch (...) {
      h->use_pdl = pdl;
      throw;
    }
    h->use_pdl = pdl;
    MCK(cudaMemcpyAsync(h->h_scal, s, sizeof(PcgScalars), cudaMemcpyDeviceToHost, st));
    MCK(cudaStreamSynchronize(st));
    MCK(cudaGetLastError());
    if (h->h_scal->status != MASPCG_SOLVE_RUNNING)
      throw Error(MASPCG_ERR_NOT_READY, "stage " + std::to_string(stage) + " left status " +
                                            std::to_string(h->h_scal->status) + " (pAp " +
                                            std::to_string(h->h_scal->pap) + ", rz_new " +
                                            std::to_string(h->h_scal->rz_new) + "): solve once first");
    return total / std::max(1, repeats);
  }

  void run(const double* b_int, maspcg_result* res)
  {
    cudaStream_t st = h->stream;
    PcgScalars* s = h->scal.get();
    const int max_iter = h->cfg.max_iterations > 0 ? h->cfg.max_iterations
                                                   : (int)(h->cfg.max_iter_ratio * (double)(3 * h->nb));
    PcgScalars init{};
    init.status = MASPCG_SOLVE_RUNNING;
    init.max_iter = max_iter;
    init.replace_mode = h->cfg.residual_replacement;
    init.graph_launches = 0;
    init.max_launches = max_iter / (mixed ? std::max(1, h->cfg.refinement_period)
                                          : std::max(1, h->cfg.iterations_per_launch)) + 4;
    init.gate = mixed ? MASPCG_GATE_EUCLID : h->cfg.gate;
    init.tol = h->cfg.tolerance;
    init.barrier_limit = h->barrier_limit;
    init.barrier_extra = h->barrier_extra;
    MCK(cudaMemcpyAsync(s, &init, sizeof(init), cudaMemcpyHostToDevice, st));
    MCK(cudaMemsetAsync(h->failed.get() + 4, 0, sizeof(int), st));
    MCK(cudaEventRecord(h->ev0, st));
    k_init<Tv><<<gstream, kTpb, 0, st>>>(b_int, V(h->vx), V(h->vr), mixed ? h->x64.get() : nullptr, n,
                                         h->partial_rz.get(), s); MLAUNCHED(h);
    precondition(V(h->vr), V(h->vz), 1, s, ovl);
    // graph of one batch
    const int batch = mixed ? std::max(1, h->cfg.refinement_period) : std::max(1, h->cfg.iterations_per_launch);
    if (h->graph_dirty || h->graph_batch != batch || graph_signature(h) != h->graph_sig) build_graph(batch, s);
    int launches = 0;
    const int max_launches = max_iter / batch + 4;
    if (h->graph_loop) {
      // one launch: the batches repeat on the device until the status leaves
      // RUNNING (or the cap).  Nothing waits on the host between the start
      // and the end of the solve: a solve already stopped at entry runs one
      // batch whose kernels return at once, and the status, the batch count
      // and the error word are read once at the end.
      MCK(cudaGraphLaunch(h->graph_exec, st));
    } else {
      // the host loop: a status read before each launch (the first also
      // covers the initial apply)
      MCK(cudaMemcpyAsync(h->h_scal, s, sizeof(PcgScalars), cudaMemcpyDeviceToHost, st));
      MCK(cudaStreamSynchronize(st));
      while (h->h_scal->status == MASPCG_SOLVE_RUNNING && launches < max_launches) {
        MCK(cudaGraphLaunch(h->graph_exec, st));
        h->kernel_launches += h->graph_kernels;
        ++launches;
        MCK(cudaMemcpyAsync(h->h_scal, s, sizeof(PcgScalars), cudaMemcpyDeviceToHost, st));
        MCK(cudaStreamSynchronize(st));
      }
    }
    // final FP64 iterate
    if (mixed) {
      launch_pdl(h, k_fold_x, dim3(gstream), dim3(kTpb), 0, h->x64.get(), reinterpret_cast<float*>(h->vx.get()), n, 1, s);
    } else {
      k_to_f64<Tv><<<ceil_div(n, kTpb), kTpb, 0, st>>>(V(h->vx), h->x64.get(), n); MLAUNCHED(h);
    }
    MCK(cudaEventRecord(h->ev1, st));
    // FP64 true residual with the FP64 matrix (reporting)
    launch_spmv64(h, h->x64.get(), h->r64.get(), 1.0, 0.0);
    k_residual_norm<<<gstream, kTpb, 0, st>>>(h->b64.get(), h->r64.get(), n, h->partial_rz.get(), s); MLAUNCHED(h);
    MCK(cudaMemcpyAsync(h->h_scal, s, sizeof(PcgScalars), cudaMemcpyDeviceToHost, st));
    MCK(cudaMemcpyAsync(h->h_err, h->failed.get() + 4, sizeof(int), cudaMemcpyDeviceToHost, st));
    MCK(cudaStreamSynchronize(st));
    if (h->graph_loop) {
      launches = h->h_scal->graph_launches;
      h->kernel_launches += h->graph_kernels * launches;
    }
    {
      const int terr = *h->h_err;
      MREQ(terr == 0, MASPCG_ERR_CUDA,
           terr == 2   ? "coarse-level dataflow queue overflow in the preconditioner apply"
           : terr == 3 ? "a grid barrier of the fused iteration kernel timed out"
                       : "a TMA mbarrier wait expired in the preconditioner apply");
    }
    float ms = 0.f;
    MCK(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
    if (res) {
      const PcgScalars& hs = *h->h_scal;
      res->iterations = hs.status == MASPCG_SOLVE_RUNNING ? hs.k : hs.iterations;
      res->status = hs.status == kNeedTrue ? MASPCG_SOLVE_RUNNING : hs.status;
      res->refinements = hs.refinements;
      res->launches = launches;
      res->rz0 = hs.rz0;
      res->rz_final = hs.rz;
      res->rel_res_recursive = hs.bb > 0 ? std::sqrt(hs.rr / hs.bb) : 0.0;
      res->rel_res_true = hs.bb > 0 ? std::sqrt(hs.rr_true / hs.bb) : std::sqrt(hs.rr_true);
      res->solve_ms = ms;
      res->fp64_gate_met = (std::isfinite(res->rel_res_true) && res->rel_res_true <= h->cfg.tolerance) ? 1 : 0;
    }
  }
};

template <>
const double* Engine<double, double, double>::matrix()
{
  return h->val64.get();
}
template <>
const float* Engine<float, float, float>::matrix()
{
  return h->val32.get();
}
template <>
const float* Engine<float, float, double>::matrix()
{
  return h->val32.get();
}

}  // namespace

size_t vec_elem_size(const maspcg_handle* h) { return h->cfg.precision == MASPCG_PREC_REFERENCE ? 8 : 4; }

double time_stage(maspcg_handle* h, int stage, int repeats)
{
  switch (h->cfg.precision) {
    case MASPCG_PREC_REFERENCE: return Engine<double, double, double>(h).time_stage(stage, repeats);
    case MASPCG_PREC_FP32: return Engine<float, float, float>(h).time_stage(stage, repeats);
    default: return Engine<float, float, double>(h).time_stage(stage, repeats);
  }
}

void solve(maspcg_handle* h, const double* b_int, double* x_int, maspcg_result* res)
{
  switch (h->cfg.precision) {
    case MASPCG_PREC_REFERENCE: {
      Engine<double, double, double> e(h);
      e.run(b_int, res);
      break;
    }
    case MASPCG_PREC_FP32: {
      Engine<float, float, float> e(h);
      e.run(b_int, res);
      break;
    }
    default: {
      Engine<float, float, double> e(h);
      e.run(b_int, res);
      break;
    }
  }
  MCK(cudaMemcpyAsync(x_int, h->x64.get(), sizeof(double) * 3 * (size_t)h->nb_int, cudaMemcpyDeviceToDevice,
                      h->stream));
}

void spmv_working(maspcg_handle* h, const double* x_int, double* y_int)
{
  switch (h->cfg.precision) {
    case MASPCG_PREC_REFERENCE: Engine<double, double, double>(h).spmv_working(x_int, y_int); break;
    case MASPCG_PREC_FP32: Engine<float, float, float>(h).spmv_working(x_int, y_int); break;
    default: Engine<float, float, double>(h).spmv_working(x_int, y_int); break;
  }
}

// z = M^-1 r on internal-order FP64 vectors (standalone apply).
void apply_preconditioner64(maspcg_handle* h, const double* r_int, double* z_int)
{
  cudaStream_t st = h->stream;
  const int n = 3 * h->nb_int;
  if (h->cfg.precision == MASPCG_PREC_REFERENCE) {
    Engine<double, double, double> e(h);
    e.precondition(r_int, z_int, 0, nullptr);
  } else {
    float* r32 = reinterpret_cast<float*>(h->vr.get());
    float* z32 = reinterpret_cast<float*>(h->vz.get());
    k_from_f64<float><<<ceil_div(n, kTpb), kTpb, 0, st>>>(r_int, r32, n); MLAUNCHED(h);
    if (h->cfg.precision == MASPCG_PREC_FP32) {
      Engine<float, float, float> e(h);
      e.precondition(r32, z32, 0, nullptr);
    } else {
      Engine<float, float, double> e(h);
      e.precondition(r32, z32, 0, nullptr);
    }
    k_to_f64<float><<<ceil_div(n, kTpb), kTpb, 0, st>>>(z32, z_int, n); MLAUNCHED(h);
  }
  MCK(cudaGetLastError());
}

}  // namespace maspcg
