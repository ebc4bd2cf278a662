// mas.cu -- MAS domain matrices, inverses and the preconditioner apply:
// TraditionalMAS32 (32-slot banks, 96x96 domains) and, where marked, CEMAS16
// (16-slot banks, 48x48 domains, MASPreconditioner.cu).
//
// Build (once per Newton step, after the hierarchy):
//   * member lists: for every coarse level a stable radix sort of the fine
//     slots by their level node, so each coarse node owns a contiguous,
//     fixed-order list of fine rows;
//   * one CTA per domain (all levels in one launch): warp a owns destination
//     block-row a; it walks the fine rows of its node and every block whose
//     column node lies in the same bank is added by the lane that owns that
//     column -- the Galerkin sum P^T A P of prepare_hessian_bcoo_kernel and
//     prepare_hessian_bcoo_sum_kernel (TraditionalMAS32Preconditioner.cu:
//     2234-2464) without atomics and in a fixed order;
//   * the 96x96 FP64 matrix stays in registers (thread (a,b) holds block
//     (a,b)); zero diagonals become 1 (expand_symmetric_mas32 :1062-1096);
//     FP32 storage inverts it in place by Gauss-Jordan elimination without
//     pivoting, as __inverse6_P96x96 (:1099-1146) does, with the pivot (=
//     the squared Cholesky diagonal) checked > 0, and stores 17 wrapped
//     diagonals x 9 elements x 32 lanes; 16-bit storage writes the lower
//     blocks out and k_domain_chol16 factors them (scaled BF16/FP16 tiles);
//   * CEMAS16: the same with 16-slot banks (48x48, FP32, 9 wrapped
//     diagonals), with its assembly and store rules.
// Apply (every PCG iteration): MAS32 runs the coarse levels as one dataflow
// kernel beside a tensor-core level-0 apply of the 16-bit records (or a warp
// per domain on FP32 records, each stored block used for both triangles
// through a shuffle); CEMAS16 runs half a warp per domain (see the CEMAS16
// apply kernels).
#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <cmath>
#include <type_traits>

#include "maspcg_internal.cuh"
#include "pcg_device.cuh"
#include "tma.cuh"
#include "mas_args.cuh"

namespace maspcg {
namespace {

constexpr int kTpb = 256;

template <typename T>
__device__ __forceinline__ T from_d(double v);
template <>
__device__ __forceinline__ float from_d<float>(double v) { return (float)v; }
template <>
__device__ __forceinline__ __nv_bfloat16 from_d<__nv_bfloat16>(double v) { return __float2bfloat16_rn((float)v); }
template <>
__device__ __forceinline__ __half from_d<__half>(double v) { return __float2half_rn((float)v); }


// ------------------------------------------------------------------ build --

__global__ void k_member_keys(const int* __restrict__ cmap, int c0, int count, unsigned* keys, int* vals)
{
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= c0) return;
  const int c = cmap[s];
  keys[s] = c >= 0 ? (unsigned)c : (unsigned)count;
  vals[s] = s;
}

__global__ void k_member_offsets(const unsigned* __restrict__ keys, int nreal, int count, int* off)
{
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= nreal) return;
  const unsigned k = keys[p];
  if (p == 0 || keys[p - 1] != k) off[k] = p;
  if (p == nreal - 1) off[count] = nreal;
}

template <int kB>
__device__ __forceinline__ int pkb(int a, int b) { return kB * a - a * (a + 1) / 2 + b; }

// CEMAS16 assembly (MASPreconditioner.cu prepare_hessian_bcoo_kernel
// :1822-1914 and prepare_hessian_bcoo_sum_kernel :1916-2037) differs from
// MAS32 on the entries (rs, u) of a fine row whose column lies in the row's
// own level-0 bank (rs, u: level-0 slots):
//  * an in-bank upper block is kept only when its column's slot is not
//    below its row's: a pair whose slot order runs against its vertex order
//    is not transposed (MAS32 transposes it) but dropped, at every level;
//  * in a bank that is one component, the coarse diagonal block receives
//    the entries of rows (2k, 2k+1) through the entry (2k, 0), so a row
//    whose even partner slot is padding adds nothing to the coarse levels.
// pmr: part_map_real; prefix_orig: components per level-0 bank (null for
// the level-0 domain itself).
__device__ __forceinline__ bool cemas16_drops(int rs, int u, const int* __restrict__ pmr,
                                              const int* __restrict__ prefix_orig)
{
  if ((u >> 4) != (rs >> 4)) return false;
  if (u != rs && ((pmr[rs] < pmr[u]) != (rs < u))) return true;
  return prefix_orig && prefix_orig[rs >> 4] == 1 && pmr[rs & ~1] < 0;
}

// Accumulate the fine row `row` into the owner lanes: every block whose
// column's level node `B` lies in bank `bank` is added by lane B % kB.
// Staging: 16 blocks per chunk through the warp's shared-memory slots, so
// the 9 doubles of a block are read coalesced and summed in block order.
// kB = 16 applies the CEMAS16 rules (pmr non-null).
template <int kB>
__device__ __forceinline__ void gather_row(const int* __restrict__ rowptr, const int* __restrict__ colidx,
                                           const double* __restrict__ val64, const int* __restrict__ cmap, int row,
                                           int fem_off, int c0, int bank, int lane, double* stage, int* sdest,
                                           double acc[9], const int* __restrict__ pmr = nullptr,
                                           const int* __restrict__ prefix_orig = nullptr)
{
  const int rs = rowptr[row], re = rowptr[row + 1];
  for (int t0 = rs; t0 < re; t0 += 16) {
    const int nblk = min(16, re - t0);
    if (lane < nblk) {
      int dest = -1;
      const int u = colidx[t0 + lane] - fem_off;
      if (u >= 0 && u < c0) {
        const int B = cmap ? cmap[u] : u;
        if (B >= 0 && B / kB == bank) dest = B % kB;
        if (kB == 16 && dest >= 0 && cemas16_drops(row - fem_off, u, pmr, prefix_orig)) dest = -1;
      }
      sdest[lane] = dest;
    }
    const double* src = val64 + 9 * (size_t)t0;
    for (int q = lane; q < nblk * 9; q += 32) stage[q] = src[q];
    __syncwarp();
    for (int j = 0; j < nblk; ++j) {
      if (sdest[j] == lane) {
#pragma unroll
        for (int e = 0; e < 9; ++e) acc[e] += stage[9 * j + e];
      }
    }
    __syncwarp();
  }
}

struct CoarseArgs {
  const int* pmr;          // CEMAS16 rules (bank 16 only)
  const int* prefix_orig;
  const int* perm[kMaxLevels];
  const int* cmap[kMaxLevels];
  int slice_base[kMaxLevels + 1];  // first warp item of each level (levels >= 1)
  int dom_begin[kMaxLevels + 1];
  int levelnum;
  int slice_rows;
  int nv;
  const int* rowptr;
  const int* colidx;
  const double* val64;
  int fem_off, c0;
  double* coarse64;  // (domains - dom_begin[1]) x kB x kB blocks, row-major 3x3
};

// Coarse-level Galerkin sums: one warp per slice of a level's member list
// (fine rows grouped by node); the slice's partial block-row is reduced in
// registers and added to the FP64 coarse domain matrix once per node.
template <int kB>
__global__ void __launch_bounds__(256) k_coarse_assemble(CoarseArgs a)
{
  __shared__ double stage_s[8][16 * 9];
  __shared__ int sdest_s[8][16];
  const int item = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31, lw = threadIdx.x >> 5;
  int L = 1;
  while (L + 1 < a.levelnum && item >= a.slice_base[L + 1]) ++L;
  if (item >= a.slice_base[a.levelnum]) return;
  const int sl = item - a.slice_base[L];
  const int p0 = sl * a.slice_rows, p1 = min(p0 + a.slice_rows, a.nv);
  const int* perm = a.perm[L];
  const int* cmap = a.cmap[L];
  double acc[9];
#pragma unroll
  for (int e = 0; e < 9; ++e) acc[e] = 0.0;
  int node = -1;
  auto flush = [&](int A) {
    if (lane >= kB) return;
    const int local = a.dom_begin[L] + A / kB - a.dom_begin[1];
    double* dst = a.coarse64 + (((size_t)local * kB + A % kB) * kB + lane) * 9;
#pragma unroll
    for (int e = 0; e < 9; ++e)
      if (acc[e] != 0.0) atomicAdd(dst + e, acc[e]);
  };
  for (int pos = p0; pos < p1; ++pos) {
    const int v = perm[pos];
    const int A = cmap[v];
    if (A != node) {
      if (node >= 0) flush(node);
#pragma unroll
      for (int e = 0; e < 9; ++e) acc[e] = 0.0;
      node = A;
    }
    gather_row<kB>(a.rowptr, a.colidx, a.val64, cmap, a.fem_off + v, a.fem_off, a.c0, A / kB, lane, stage_s[lw],
                   sdest_s[lw], acc, a.pmr, a.prefix_orig);
  }
  if (node >= 0) flush(node);
}

// One CTA per domain; thread (w,lane) owns block (w,lane) of the 3kB x 3kB
// FP64 matrix (one warp per block row; for kB = 16 lanes 16..31 only help
// stage the gathered rows).  FP32 storage: in-place Gauss-Jordan inverse,
// symmetric layout.  16-bit storage (kB = 32): Cholesky A = L L^T,
// W = L^-1, stored W S^-1 with column scales S, so the applied operator
// S (W S^-1)^T (W S^-1) S stays SPD whatever the rounding.
template <typename TI, bool kAssembled, int kB>
__global__ void __launch_bounds__(1024, 1) k_domain_factor(FactorArgs a, int dom_offset)
{
  __shared__ double buf[2][96];
  __shared__ double stage[32][16 * 9];
  __shared__ int sdest[32][16];
  __shared__ float sscale[96];
  __shared__ unsigned smax[96];
  __shared__ double spiv[2][2];  // per step: 1/pivot (GJ) or {sqrt(pivot), 1/sqrt(pivot)} (Cholesky)
  __shared__ int fail;

  const int g = blockIdx.x + dom_offset;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) fail = 0;
  if (threadIdx.x < 96) smax[threadIdx.x] = 0u;

  double acc[9];
#pragma unroll
  for (int e = 0; e < 9; ++e) acc[e] = 0.0;
  const int d0 = a.lv.dom_begin[1];
  if (g < d0) {
    const int slot = kB * g + w;
    if (a.pmr[slot] >= 0)
      gather_row<kB>(a.rowptr, a.colidx, a.val64, nullptr, a.fem_off + slot, a.fem_off, a.c0, g, lane, stage[w],
                     sdest[w], acc, a.pmr);
  } else if (lane < kB) {
    const double* src = a.coarse64 + (((size_t)(g - d0) * kB + w) * kB + lane) * 9;
#pragma unroll
    for (int e = 0; e < 9; ++e) acc[e] = src[e];
  }
  if (kAssembled && lane >= w && lane < kB) {
    double* o = a.assembled + ((size_t)g * (kB * (kB + 1) / 2) + pkb<kB>(w, lane)) * 9;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) o[i + 3 * j] = acc[3 * i + j];
  }
  if (kAssembled && a.gather_only) return;  // uniform: no barrier has run yet
  if (lane == w) {
    if (acc[0] == 0.0) acc[0] = 1.0;
    if (acc[4] == 0.0) acc[4] = 1.0;
    if (acc[8] == 0.0) acc[8] = 1.0;
  }
  constexpr bool kFactored = !std::is_same<TI, float>::value;
  static_assert(kB == 32 || !kFactored, "16-slot banks store FP32 inverses");
  TI* out = reinterpret_cast<TI*>(a.inv) + (size_t)g * (kB == 32 ? inv_elems<TI>() : kMas16InvElems);

  if (!kFactored) {
    // ---- in-place Gauss-Jordan inversion (the elimination of __inverse6_P96x96)
    for (int q = 0; q < kB; ++q) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const int j = 3 * q + c;
        double* pr = buf[j & 1];
        if (w == q) {
          pr[3 * lane + 0] = acc[3 * c + 0];
          pr[3 * lane + 1] = acc[3 * c + 1];
          pr[3 * lane + 2] = acc[3 * c + 2];
          if (lane == q) {  // the pivot's owner inverts it once for the CTA
            double pv = acc[4 * c];
            if (!(pv > 0.0) || !isfinite(pv)) {
              fail = 1;
              pv = 1.0;
            }
            spiv[j & 1][0] = 1.0 / pv;
          }
        }
        const double m0 = __shfl_sync(kFull, acc[c], q);
        const double m1 = __shfl_sync(kFull, acc[3 + c], q);
        const double m2 = __shfl_sync(kFull, acc[6 + c], q);
        __syncthreads();
        const double inv = spiv[j & 1][0];
        const double p[3] = {pr[3 * lane], pr[3 * lane + 1], pr[3 * lane + 2]};
        const double mm[3] = {m0, m1, m2};
#pragma unroll
        for (int i = 0; i < 3; ++i) {
          const bool rowj = (w == q) && (i == c);
          const double f = mm[i] * inv;
#pragma unroll
          for (int jj = 0; jj < 3; ++jj) {
            const bool colj = (lane == q) && (jj == c);
            double& x = acc[3 * i + jj];
            if (rowj && colj)
              x = inv;
            else if (rowj)
              x = p[jj] * inv;
            else if (colj)
              x = -f;
            else
              x = fma(-f, p[jj], x);
          }
        }
      }
    }
    __syncthreads();
    if (threadIdx.x == 0 && fail) atomicAdd(a.failed, 1);
    const int d = (lane - w) & (kB - 1);
    if (lane < kB && d <= kB / 2) {
      const bool zero = (d == kB / 2) && (w >= kB / 2);
      if (kB == 16 && d == 0) {
        // CEMAS16 stores the diagonal blocks with their lower elements
        // taken from the upper ones (MASPreconditioner.cu:705-711)
        acc[3] = acc[1];
        acc[6] = acc[2];
        acc[7] = acc[5];
      }
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) out[(d * 9 + 3 * i + j) * kB + w] = from_d<TI>(zero ? 0.0 : acc[3 * i + j]);
    }
    return;
  }
  if constexpr (kFactored) {
    // 16-bit storage: the lower blocks go to dom64 for k_domain_chol16
    if (lane <= w) {
      double* o = a.dom64 + ((size_t)g * kPacked + w * (w + 1) / 2 + lane) * 9;
#pragma unroll
      for (int e = 0; e < 9; ++e) o[e] = acc[e];
    }
  }
}

// 16-bit storage, second pass: the Cholesky factor of one domain from its
// lower FP64 blocks (dom64, written by k_domain_factor), then W = L^-1 and
// the scaled tile store.  Thread t < 528 owns lower block (w, lane),
// t = w(w+1)/2 + lane; only the lower triangle takes part, so two CTAs fit
// on an SM and hide each other's step latency.  The steps talk through
// shared memory only, so the thread layout is free.
constexpr int kCholThreads = 544;  // 528 lower blocks in 17 warps
template <typename TI>
__global__ void __launch_bounds__(kCholThreads, 2) k_domain_chol16(FactorArgs a, int dom_offset)
{
  __shared__ double dinv[kBank][9];      // L_qq^-1 (lower, row-major), kept for W below
  __shared__ double panel[2][kBank][9];  // L_wq
  __shared__ double wrow[2][kBank][9];   // W_ql
  __shared__ float sscale[96];
  __shared__ unsigned smax[96];
  __shared__ int fail;
  const int g = blockIdx.x + dom_offset;
  const bool act = threadIdx.x < kPacked;
  int w = -1, lane = -1;
  if (act) {
    const int t = threadIdx.x;
    w = (int)((sqrtf(8.f * t + 1.f) - 1.f) * 0.5f);
    while (w * (w + 1) / 2 > t) --w;
    while ((w + 1) * (w + 2) / 2 <= t) ++w;
    lane = t - w * (w + 1) / 2;
  }
  if (threadIdx.x == 0) fail = 0;
  if (threadIdx.x < 96) smax[threadIdx.x] = 0u;
  double acc[9];
  if (act) {
    const double* src = a.dom64 + ((size_t)g * kPacked + threadIdx.x) * 9;
#pragma unroll
    for (int e = 0; e < 9; ++e) acc[e] = src[e];
  } else {
#pragma unroll
    for (int e = 0; e < 9; ++e) acc[e] = 0.0;
  }
  __syncthreads();
  // ---- blocked Cholesky, right-looking over the 32 block columns: thread
  // (q,q) factors its 3x3 diagonal block and inverts the factor, the block
  // column below it is solved against that factor, then the trailing lower
  // blocks take the rank-3 update.  Lower blocks (w >= lane) hold L after.
  for (int q = 0; q < kBank; ++q) {
    const int b = q & 1;
    if (w == q && lane == q) {
      double p0 = acc[0];
      if (!(p0 > 0.0) || !isfinite(p0)) fail = 1, p0 = 1.0;
      const double l00 = sqrt(p0), i00 = 1.0 / l00;
      const double l10 = acc[3] * i00, l20 = acc[6] * i00;
      double p1 = acc[4] - l10 * l10;
      if (!(p1 > 0.0) || !isfinite(p1)) fail = 1, p1 = 1.0;
      const double l11 = sqrt(p1), i11 = 1.0 / l11;
      const double l21 = (acc[7] - l20 * l10) * i11;
      double p2 = acc[8] - l20 * l20 - l21 * l21;
      if (!(p2 > 0.0) || !isfinite(p2)) fail = 1, p2 = 1.0;
      const double l22 = sqrt(p2), i22 = 1.0 / l22;
      const double i10 = -(l10 * i00) * i11;
      const double i21 = -(l21 * i11) * i22;
      const double i20 = -(l20 * i00 + l21 * i10) * i22;
      const double L[9] = {l00, 0.0, 0.0, l10, l11, 0.0, l20, l21, l22};
      const double I[9] = {i00, 0.0, 0.0, i10, i11, 0.0, i20, i21, i22};
#pragma unroll
      for (int e = 0; e < 9; ++e) {
        acc[e] = L[e];
        dinv[q][e] = I[e];
      }
    }
    __syncthreads();
    if (lane == q && w > q) {  // L_wq = A_wq L_qq^-T
      double l[9];
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
          l[3 * i + j] = acc[3 * i] * dinv[q][3 * j] + acc[3 * i + 1] * dinv[q][3 * j + 1] +
                         acc[3 * i + 2] * dinv[q][3 * j + 2];
#pragma unroll
      for (int e = 0; e < 9; ++e) {
        acc[e] = l[e];
        panel[b][w][e] = l[e];
      }
    }
    __syncthreads();
    if (w > q && lane > q && lane <= w) {  // A_wl -= L_wq L_lq^T
      const double* pw = panel[b][w];
      const double* pl = panel[b][lane];
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
          acc[3 * i + j] -= pw[3 * i] * pl[3 * j] + pw[3 * i + 1] * pl[3 * j + 1] + pw[3 * i + 2] * pl[3 * j + 2];
    }
  }
  // ---- W = L^-1 by blocked forward substitution on the identity: row
  // block q of W is L_qq^-1 times the current right-hand side, which is then
  // eliminated from the rows below.
  double xr[9];
#pragma unroll
  for (int e = 0; e < 9; ++e) xr[e] = (w == lane && (e % 4) == 0) ? 1.0 : 0.0;
  for (int q = 0; q < kBank; ++q) {
    const int b = q & 1;
    if (lane == q && w > q) {
#pragma unroll
      for (int e = 0; e < 9; ++e) panel[b][w][e] = acc[e];  // L_wq
    }
    if (w == q && lane <= q) {  // W_ql = L_qq^-1 X_ql
      double y[9];
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
          y[3 * i + j] = dinv[q][3 * i] * xr[j] + dinv[q][3 * i + 1] * xr[3 + j] + dinv[q][3 * i + 2] * xr[6 + j];
#pragma unroll
      for (int e = 0; e < 9; ++e) {
        xr[e] = y[e];
        wrow[b][lane][e] = y[e];
      }
    }
    __syncthreads();
    if (w > q && lane <= q) {  // X_wl -= L_wq W_ql
      const double* lw = panel[b][w];
      const double* wl = wrow[b][lane];
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
          xr[3 * i + j] -= lw[3 * i] * wl[j] + lw[3 * i + 1] * wl[3 + j] + lw[3 * i + 2] * wl[6 + j];
    }
  }
  __syncthreads();
  // ---- column scales and factored store (lower blocks only)
  if (act) {
#pragma unroll
    for (int jj = 0; jj < 3; ++jj) {
      const float m = (float)fmax(fmax(fabs(xr[jj]), fabs(xr[3 + jj])), fabs(xr[6 + jj]));
      atomicMax(smax + 3 * lane + jj, __float_as_uint(m));
    }
  }
  __syncthreads();
  if (threadIdx.x < 96) {
    float sv = __uint_as_float(smax[threadIdx.x]);
    if (!(sv > 0.f) || !isfinite(sv)) sv = 1.f;
    sscale[threadIdx.x] = sv;
    a.scale[(size_t)g * 96 + threadIdx.x] = sv;
  }
  __syncthreads();
  if (threadIdx.x == 0 && fail) atomicAdd(a.failed, 1);
  // tile store: lower blocks, and zeros for the upper elements that fall in
  // a diagonal tile
  if (!act) return;
  TI* out = reinterpret_cast<TI*>(a.inv) + (size_t)g * kInvElems16;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int jj = 0; jj < 3; ++jj) {
      // (an upper element outside the diagonal tiles has no slot: a 3x3
      // diagonal block can straddle a tile boundary)
      const int row = 3 * w + i, col = 3 * lane + jj;
      if (row >= col)
        out[inv16_pos(row, col)] = from_d<TI>(xr[3 * i + jj] / (double)sscale[3 * lane + jj]);
      else if ((row >> 4) == (col >> 4))
        out[inv16_pos(row, col)] = from_d<TI>(0.0);
      // the mirror upper block (lane, w): its elements inside a diagonal tile are zero
      const int mr = 3 * lane + i, mc = 3 * w + jj;
      if (w > lane && (mr >> 4) == (mc >> 4)) out[inv16_pos(mr, mc)] = from_d<TI>(0.0);
    }
}

// ------------------------------------------------------------------ apply --

// z = (M x) for one domain held by one warp, FP32 storage: the symmetric
// inverse, lane l holding block (l, (l + d) % 32) of diagonal d = 0..16, each
// stored block serving both triangles through a shuffle.  x, y: the lane's
// three rows.
__device__ __forceinline__ void domain_apply(const float* __restrict__ inv, int lane, const float x[3], float y[3])
{
  const float x0 = x[0], x1 = x[1], x2 = x[2];
  float y0 = 0.f, y1 = 0.f, y2 = 0.f;
#pragma unroll
  for (int d = 0; d < kDiags; ++d) {
    const int c = (lane + d) & 31;
    const float c0 = __shfl_sync(kFull, x0, c), c1 = __shfl_sync(kFull, x1, c), c2 = __shfl_sync(kFull, x2, c);
    float B[9];
#pragma unroll
    for (int e = 0; e < 9; ++e) B[e] = inv[(d * 9 + e) * kBank + lane];
    y0 += B[0] * c0 + B[1] * c1 + B[2] * c2;
    y1 += B[3] * c0 + B[4] * c1 + B[5] * c2;
    y2 += B[6] * c0 + B[7] * c1 + B[8] * c2;
    if (d != 0) {
      const float t0 = B[0] * x0 + B[3] * x1 + B[6] * x2;
      const float t1 = B[1] * x0 + B[4] * x1 + B[7] * x2;
      const float t2 = B[2] * x0 + B[5] * x1 + B[8] * x2;
      const int src = (lane - d) & 31;
      y0 += __shfl_sync(kFull, t0, src);
      y1 += __shfl_sync(kFull, t1, src);
      y2 += __shfl_sync(kFull, t2, src);
    }
  }
  y[0] = y0;
  y[1] = y1;
  y[2] = y2;
}

// ---- tensor-core apply of a 16-bit factored record -------------------------
//
// M = S V^T V S with V the scaled lower factor (96 x 96, 21 tiles of 16 x 16
// in shared memory, inv16_pos).  Pass 1, t = V (S x), multiplies each tile by
// the matching 16 entries of the vector with mma.m16n8k16 (the tile as A);
// pass 2, z = V^T t, does the same with the tiles loaded transposed
// (ldmatrix .trans).  The FP32 vector enters the 16-bit B operand as three
// terms, hi + mid + lo (each the rounding of what the previous ones leave),
// in columns 0, 1, 2 of B, so the products carry the vector to FP32 precision
// and the FP32 accumulators of the three columns are added afterwards.  FP16
// records scale the vector by a power of two (its largest entry to [1, 2))
// first, as FP16 has a narrow exponent range; the scaling is exact.
constexpr int kPartStride = 104;             // 16-bit split terms: 3 rows of 104 (bank spread)
constexpr int kApplyScratch = 1024;          // per warp: 96 FP32 + 3 x 104 16-bit
constexpr int kRecBytes16 = kInvElems16 * 2;  // 10,752

template <typename TI>
struct Mma16;
template <>
struct Mma16<__nv_bfloat16> {
  static constexpr bool kNormalize = false;
  static __device__ __forceinline__ void mma(float c[4], const uint32_t a[4], uint32_t b0, uint32_t b1)
  {
    asm("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
  }
  static __device__ __forceinline__ unsigned short to16(float v) { return __bfloat16_as_ushort(__float2bfloat16_rn(v)); }
  static __device__ __forceinline__ float from16(unsigned short u) { return __uint_as_float((uint32_t)u << 16); }
};
template <>
struct Mma16<__half> {
  static constexpr bool kNormalize = true;
  static __device__ __forceinline__ void mma(float c[4], const uint32_t a[4], uint32_t b0, uint32_t b1)
  {
    asm("mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
  }
  static __device__ __forceinline__ unsigned short to16(float v) { return __half_as_ushort(__float2half_rn(v)); }
  static __device__ __forceinline__ float from16(unsigned short u) { return __half2float(__ushort_as_half(u)); }
};

__device__ __forceinline__ void ldsm(uint32_t addr, uint32_t a[4])
{
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];"
               : "=r"(a[0]), "=r"(a[1]), "=r"(a[2]), "=r"(a[3])
               : "r"(addr)
               : "memory");
}
__device__ __forceinline__ void ldsm_t(uint32_t addr, uint32_t a[4])
{
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];"
               : "=r"(a[0]), "=r"(a[1]), "=r"(a[2]), "=r"(a[3])
               : "r"(addr)
               : "memory");
}

// Power-of-two factor taking the warp's largest |v| to [1, 2) (1 when the
// vector is zero or not finite), and its inverse.
__device__ __forceinline__ void pow2_normalizer(const float v[3], float& f, float& fi)
{
  const float m = fmaxf(fabsf(v[0]), fmaxf(fabsf(v[1]), fabsf(v[2])));
  const unsigned mb = __reduce_max_sync(kFull, __float_as_uint(m));
  int ex = (int)(mb >> 23) - 127;
  if (mb == 0u || mb >= 0x7f800000u) ex = 0;
  ex = max(-120, min(120, ex));
  f = __uint_as_float((unsigned)(127 - ex) << 23);
  fi = __uint_as_float((unsigned)(127 + ex) << 23);
}

// Three 16-bit terms of each of the lane's three entries (rows 3 lane + i).
template <typename TI>
__device__ __forceinline__ void split_store(unsigned short* part, int lane, const float v[3])
{
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    float r = v[i];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const unsigned short u = Mma16<TI>::to16(r);
      part[k * kPartStride + 3 * lane + i] = u;
      r -= Mma16<TI>::from16(u);
    }
  }
}

// B operand of the 16 vector entries [16 K, 16 K + 16): thread (g, q) holds
// column g (split term g; zero for g >= 3), rows 2q, 2q+1 and 2q+8, 2q+9.
__device__ __forceinline__ void b_frag(const unsigned short* part, int K, int g, int q, uint32_t& b0, uint32_t& b1)
{
  b0 = b1 = 0u;
  if (g < 3) {
    const unsigned short* p = part + g * kPartStride + 16 * K + 2 * q;
    b0 = *reinterpret_cast<const uint32_t*>(p);
    b1 = *reinterpret_cast<const uint32_t*>(p + 8);
  }
}

// Sum of the three split-term columns of 6 accumulator tiles into out[96]:
// thread (g, q = 0) holds columns 0-1 of rows g and g + 8, thread (g, 1)
// column 2.
__device__ __forceinline__ void reduce_columns(float acc[6][4], float* out, int g, int q)
{
#pragma unroll
  for (int I = 0; I < 6; ++I) {
    float t0 = acc[I][0] + acc[I][1], t1 = acc[I][2] + acc[I][3];
    t0 += __shfl_down_sync(kFull, t0, 1);
    t1 += __shfl_down_sync(kFull, t1, 1);
    if (q == 0) {
      out[16 * I + g] = t0;
      out[16 * I + g + 8] = t1;
    }
  }
}

// y = (M x) for one domain held by one warp: rec is the 16-bit record in
// shared memory, scratch this warp's kApplyScratch bytes of shared memory,
// sc the lane's three column scales.
template <typename TI>
__device__ __forceinline__ void domain_apply16(const TI* rec, unsigned char* scratch, const float sc[3], int lane,
                                               const float x[3], float y[3])
{
  using M = Mma16<TI>;
  float* vf = reinterpret_cast<float*>(scratch);
  unsigned short* part = reinterpret_cast<unsigned short*>(scratch + 96 * sizeof(float));
  const int g = lane >> 2, q = lane & 3;
  const int m = lane >> 3, rr = lane & 7;
  const uint32_t base = (uint32_t)__cvta_generic_to_shared(rec);
  const uint32_t off_n = ((((m & 1) << 3) + rr) << 5) + ((((m >> 1) ^ (rr >> 2)) & 1) << 4);
  const uint32_t off_t = ((((m >> 1) << 3) + rr) << 5) + ((((m & 1) ^ (rr >> 2)) & 1) << 4);
  const float s0 = sc[0], s1 = sc[1], s2 = sc[2];
  float v[3] = {x[0] * s0, x[1] * s1, x[2] * s2};
  float f1 = 1.f, fi1 = 1.f;
  if constexpr (M::kNormalize) {
    pow2_normalizer(v, f1, fi1);
    v[0] *= f1;
    v[1] *= f1;
    v[2] *= f1;
  }
  split_store<TI>(part, lane, v);
  __syncwarp();
  // pass 1: t = V v
  {
    float acc[6][4];
#pragma unroll
    for (int I = 0; I < 6; ++I) acc[I][0] = acc[I][1] = acc[I][2] = acc[I][3] = 0.f;
#pragma unroll
    for (int K = 0; K < 6; ++K) {
      uint32_t b0, b1;
      b_frag(part, K, g, q, b0, b1);
#pragma unroll
      for (int I = K; I < 6; ++I) {
        uint32_t a[4];
        ldsm(base + (uint32_t)((I * (I + 1) / 2 + K) * 512) + off_n, a);
        M::mma(acc[I], a, b0, b1);
      }
    }
    reduce_columns(acc, vf, g, q);
  }
  __syncwarp();
  v[0] = vf[3 * lane];
  v[1] = vf[3 * lane + 1];
  v[2] = vf[3 * lane + 2];
  float f2 = 1.f, fi2 = 1.f;
  if constexpr (M::kNormalize) {
    pow2_normalizer(v, f2, fi2);
    v[0] *= f2;
    v[1] *= f2;
    v[2] *= f2;
  }
  split_store<TI>(part, lane, v);
  __syncwarp();
  // pass 2: z = V^T t
  {
    float acc[6][4];
#pragma unroll
    for (int J = 0; J < 6; ++J) acc[J][0] = acc[J][1] = acc[J][2] = acc[J][3] = 0.f;
#pragma unroll
    for (int K = 0; K < 6; ++K) {
      uint32_t b0, b1;
      b_frag(part, K, g, q, b0, b1);
#pragma unroll
      for (int J = 0; J <= K; ++J) {
        uint32_t a[4];
        ldsm_t(base + (uint32_t)((K * (K + 1) / 2 + J) * 512) + off_t, a);
        M::mma(acc[J], a, b0, b1);
      }
    }
    reduce_columns(acc, vf, g, q);
  }
  __syncwarp();
  const float back = fi1 * fi2;
  y[0] = vf[3 * lane] * back * s0;
  y[1] = vf[3 * lane + 1] * back * s1;
  y[2] = vf[3 * lane + 2] * back * s2;
}

// Leader of each key group gets the group sum: with kFast a butterfly when
// the whole warp is one group (the common case at level 0: one coarse node
// per bank), else the group's lanes in ascending order.  Both orders are
// fixed.  (The walk over coarse levels uses the general form only: ptxas
// fails to allocate registers for the butterfly inside that loop.)
template <bool kFast>
__device__ __forceinline__ void group_sum(int key, const float v[3], float out[3], bool& leader)
{
  const unsigned grp = __match_any_sync(kFull, key);
  float s0, s1, s2;
  if (kFast && grp == kFull) {  // warp-uniform
    s0 = v[0], s1 = v[1], s2 = v[2];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      s0 += __shfl_xor_sync(kFull, s0, o);
      s1 += __shfl_xor_sync(kFull, s1, o);
      s2 += __shfl_xor_sync(kFull, s2, o);
    }
  } else {
    s0 = s1 = s2 = 0.f;
    for (int src = 0; src < 32; ++src) {
      const float a0 = __shfl_sync(kFull, v[0], src), a1 = __shfl_sync(kFull, v[1], src),
                  a2 = __shfl_sync(kFull, v[2], src);
      if ((grp >> src) & 1u) {
        s0 += a0;
        s1 += a1;
        s2 += a2;
      }
    }
  }
  out[0] = s0;
  out[1] = s1;
  out[2] = s2;
  leader = (__ffs(grp) - 1) == (int)(threadIdx.x & 31);
}

// Copy a 16-bit domain record to a warp's shared-memory slot with coalesced
// 16-byte loads (streaming: a record is read once per apply).
__device__ __forceinline__ void stage_record(const uint4* __restrict__ src, unsigned char* slot, int lane)
{
  uint4* dst = reinterpret_cast<uint4*>(slot);
  __syncwarp();
#pragma unroll 7
  for (int k = lane; k < kRecBytes16 / 16; k += 32) dst[k] = __ldcs(src + k);
  __syncwarp();
}

// Domain-apply kernels: 4 warps per CTA.  16-bit records are staged in
// shared memory (a record and the apply scratch per warp: 47,104 bytes per
// CTA, four CTAs per SM).
constexpr int kApplyTpb = 128;
constexpr int kDirectSmem16 = (kApplyTpb / 32) * (kRecBytes16 + kApplyScratch);
#define MAS_APPLY_BOUNDS(TI) __launch_bounds__(kApplyTpb, 4)

// ---- coarse levels in one kernel (restriction + coarse domain applies) ----
//
// BuildMultiLevelR and the coarse part of _schwarzLocalXSym6 as a dataflow
// over the hierarchy.  CTA c restricts level-0 banks [16c, 16c + 16) (two
// per warp, so one resident wave of CTAs covers them) into level-1 nodes.  A coarse domain (32 consecutive nodes of level
// l >= 1) is complete once every unit that writes one of its nodes has
// finished; each unit counts itself into the domains its parents fall in,
// and the unit that completes a domain processes it in the same CTA:
// restricts its nodes into level l + 1 (which may complete further domains)
// and applies the domain's inverse.  Sums run in a fixed order (group sums
// in lane order), so the result does not depend on which CTA finishes last;
// nothing waits.  Counters return to zero as they complete.
constexpr int kChainWarps = 8;
constexpr int kChainBanks = 2;                          // level-0 banks each warp restricts
constexpr int kChainUnitBanks = kChainWarps * kChainBanks;  // banks per CTA: one resident wave covers them
constexpr int kChainQueue = 64;
constexpr int kChainApplySlots = 4;  // 16-bit domain records staged in shared memory at a time

// Dynamic shared memory of k_coarse_chain: 16-bit records are staged (their
// two passes then read shared memory), FP32 records are read from global.
template <typename TI>
constexpr int chain_smem_bytes() { return sizeof(TI) == 2 ? kChainApplySlots * (kRecBytes16 + kApplyScratch) : 0; }

// One thread counts a finished unit, whose parents span global slots
// [lo, hi], into the parent domains; domains it completes are appended to
// the CTA's queue (the thread's `tail`).  Release before the counts, acquire
// after a completion.
__device__ __forceinline__ void chain_arrive(const ApplyArgs& a, int lo, int hi, int* queue, int& tail)
{
  const int d1 = a.lv.dom_begin[1];
  __threadfence();
  for (int g = lo / kBank; g <= hi / kBank; ++g) {
    const int old = atomicAdd(a.chain_count + (g - d1), 1);
    if (old + 1 == a.chain_target[g - d1]) {
      a.chain_count[g - d1] = 0;
      if (tail < kChainQueue)
        queue[tail++] = g;
      else
        atomicExch(a.err, 2);
    }
  }
  __threadfence();
}

// Level of a coarse domain g.
__device__ __forceinline__ int domain_level(const LevelInfo& lv, int g)
{
  int l = 1;
  while (l + 1 < lv.levelnum && g >= lv.dom_begin[l + 1]) ++l;
  return l;
}

// pair: the level-0 apply runs concurrently and leaves the coarse correction
// to the p update; this kernel then also sums r.z of the coarse levels,
// sum over domains of R.Z (= r . P Z), and completes r.z with the level-0
// part (rz_part_done, mode as in rz_update).
template <typename TI, typename Tv, bool kFused>
__global__ void __launch_bounds__(kChainWarps * 32) k_coarse_chain(ApplyArgs a, const Tv* __restrict__ r,
                                                                  PcgScalars* s, int mode, int pair, FusedArgs fa)
{
  __shared__ int queue[kChainQueue];
  __shared__ int tail_s, lo_s, hi_s;
  pdl_wait();
  if (s && s->status != MASPCG_SOLVE_RUNNING) return;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    tail_s = 0;
    lo_s = INT_MAX;
    hi_s = -1;
  }
  __syncthreads();
  FusedScal fs{};
  if constexpr (kFused) fs = fused_scalars(s);
  // level 0 -> level 1 (RestrictR of the fine residual); a level-1 node's
  // children all lie in one bank, so its sum is written, not accumulated
#pragma unroll
  for (int k = 0; k < kChainBanks; ++k) {
    const int bank = blockIdx.x * kChainUnitBanks + k * kChainWarps + w;
    if (bank < a.c0 / kBank) {
      const int slot = bank * kBank + lane;
      const int key = a.cmap1[slot];
      float v[3];
      if constexpr (kFused) {
        // r' of the iteration's update, formed as the level-0 apply forms it
        fused_input_row(fa, fs, a.fem_off + slot, false, v);
      } else {
        const Tv* rp = r + 3 * (size_t)(a.fem_off + slot);
        v[0] = (float)rp[0];
        v[1] = (float)rp[1];
        v[2] = (float)rp[2];
      }
      float o[3];
      bool leader;
      group_sum<true>(key >= 0 ? key : -1 - lane, v, o, leader);
      if (leader && key >= 0) {
        float* d = a.coarse_r + 3 * (size_t)key;
        d[0] = o[0];
        d[1] = o[1];
        d[2] = o[2];
      }
      const int lo = (int)__reduce_min_sync(kFull, key >= 0 ? (unsigned)key : 0x7fffffffu);
      const int hi = (int)__reduce_max_sync(kFull, key >= 0 ? (unsigned)key : 0u);
      const bool any = __any_sync(kFull, key >= 0);  // every lane votes
      if (lane == 0 && any) {
        atomicMin(&lo_s, a.c0 + lo);
        atomicMax(&hi_s, a.c0 + hi);
      }
    }
  }
  pdl_trigger();
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0 && hi_s >= 0) {
    int t = 0;
    chain_arrive(a, lo_s, hi_s, queue, t);
    tail_s = t;
  }
  __syncthreads();
  const int tail0 = tail_s;
  if (tail0 == 0) return;
  // warp 0: walk up the levels, restricting every completed domain.  Lane 0
  // owns the queue tail; the loop bound is broadcast from it every step so
  // the warp never diverges on it.
  if (w == 0) {
    int t = tail0;  // meaningful in lane 0
    for (int i = 0; i < __shfl_sync(kFull, t, 0); ++i) {
      const int g = queue[i];
      const int l = domain_level(a.lv, g);
      if (l + 1 >= a.lv.levelnum) continue;  // top level: nothing above
      const int sg = g * kBank + lane;         // global slot of the node
      const bool valid = sg - a.lv.begin[l] < a.lv.count[l];
      float v[3] = {0.f, 0.f, 0.f};
      int key = -1 - lane;
      if (valid) {
        const float* src = a.coarse_r + 3 * (size_t)(sg - a.c0);
        v[0] = __ldcg(src);
        v[1] = __ldcg(src + 1);
        v[2] = __ldcg(src + 2);
        key = a.going_next[sg];
      }
      float o[3];
      bool leader;
      group_sum<false>(key, v, o, leader);
      if (leader && valid) {
        float* d = a.coarse_r + 3 * (size_t)(key - a.c0);
        d[0] = o[0];
        d[1] = o[1];
        d[2] = o[2];
      }
      const int lo = (int)__reduce_min_sync(kFull, valid ? (unsigned)key : 0x7fffffffu);
      const int hi = (int)__reduce_max_sync(kFull, valid ? (unsigned)key : 0u);
      if (lane == 0 && lo <= hi) chain_arrive(a, lo, hi, queue, t);
      __syncwarp();
    }
    if (lane == 0) tail_s = t;
  }
  __syncthreads();
  // apply the completed domains' inverses: 16-bit records are copied into a
  // shared-memory slot per warp with 77 coalesced loads per lane, so the
  // tensor-core passes read it there
  extern __shared__ __align__(16) unsigned char chain_slots[];
  const int n = tail_s;
  constexpr bool kStage = sizeof(TI) == 2;
  constexpr int kSlots = kStage ? kChainApplySlots : kChainWarps;
  if (w < kSlots) {
    for (int i = w; i < n; i += kSlots) {
      const int g = queue[i];
      const size_t base = (size_t)(kBank * g + lane - a.c0) * 3;
      const float x[3] = {__ldcg(a.coarse_r + base), __ldcg(a.coarse_r + base + 1), __ldcg(a.coarse_r + base + 2)};
      float y[3];
      if constexpr (kStage) {
        unsigned char* slot = chain_slots + (size_t)w * (kRecBytes16 + kApplyScratch);
        stage_record(reinterpret_cast<const uint4*>(a.inv) + (size_t)g * (kRecBytes16 / 16), slot, lane);
        const float* scg = a.scale + (size_t)g * 96 + 3 * lane;
        const float sc[3] = {scg[0], scg[1], scg[2]};
        domain_apply16<TI>(reinterpret_cast<const TI*>(slot), slot + kRecBytes16, sc, lane, x, y);
      } else {
        domain_apply(reinterpret_cast<const float*>(a.inv) + (size_t)g * kInvElems, lane, x, y);
      }
      a.coarse_z[base] = y[0];
      a.coarse_z[base + 1] = y[1];
      a.coarse_z[base + 2] = y[2];
      if (pair && s) {
        // this domain's R.Z; the warp applying the last coarse domain adds
        // them up in domain order and completes r.z
        const int d1 = a.lv.dom_begin[1], nd = a.lv.domains - d1;
        const double dz = warp_sum((double)x[0] * y[0] + (double)x[1] * y[1] + (double)x[2] * y[2]);
        int last = 0;
        if (lane == 0) {
          a.chain_dot[g - d1] = dz;
          __threadfence();
          last = atomicAdd(&s->tickets[kTicketCoarse], 1u) == (unsigned)nd - 1u;
        }
        if (__shfl_sync(kFull, last, 0)) {
          __threadfence();
          double t = 0.0;
          for (int q = lane; q < nd; q += 32) t += __ldcg(a.chain_dot + q);
          t = warp_sum(t);
          if (lane == 0) {
            s->tickets[kTicketCoarse] = 0u;
            rz_part_done(s, 1, t, mode);
          }
        }
      }
    }
  }
}

// Expected arrivals per coarse domain: the same unit/parent-range rule as
// k_coarse_chain, counted once per build.
__global__ void k_chain_targets(ApplyArgs a, int* target)
{
  const int lane = threadIdx.x & 31;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int d1 = a.lv.dom_begin[1];
  const int units0 = (a.c0 / kBank + kChainUnitBanks - 1) / kChainUnitBanks;
  int lo = 0x7fffffff, hi = -1;
  if (gw < units0) {
    for (int b = gw * kChainUnitBanks; b < min((gw + 1) * kChainUnitBanks, a.c0 / kBank); ++b) {
      const int key = a.cmap1[b * kBank + lane];
      const int l2 = (int)__reduce_min_sync(kFull, key >= 0 ? (unsigned)key : 0x7fffffffu);
      const int h2 = (int)__reduce_max_sync(kFull, key >= 0 ? (unsigned)key : 0u);
      const bool any = __any_sync(kFull, key >= 0);
      if (any) {
        lo = min(lo, a.c0 + l2);
        hi = max(hi, a.c0 + h2);
      }
    }
  } else {
    const int g = d1 + (gw - units0);  // a coarse domain as a unit
    if (g >= a.lv.domains) return;
    const int l = domain_level(a.lv, g);
    if (l + 1 >= a.lv.levelnum) return;
    const int sg = g * kBank + lane;
    const bool valid = sg - a.lv.begin[l] < a.lv.count[l];
    const int key = valid ? a.going_next[sg] : 0;
    lo = (int)__reduce_min_sync(kFull, valid ? (unsigned)key : 0x7fffffffu);
    hi = (int)__reduce_max_sync(kFull, valid ? (unsigned)key : 0u);
    if (!__any_sync(kFull, valid)) return;
  }
  if (lane == 0 && hi >= 0)
    for (int g = lo / kBank; g <= hi / kBank; ++g) atomicAdd(target + (g - d1), 1);
}

// ---- CEMAS16 apply (MASPreconditioner::preconditioning, :2250-2291) -------
//
// Over 16-slot banks:
//   * the restriction, one launch per coarse level (L-1 launches): a node of
//     level l+1 is a connected component inside one bank of level l, so its
//     children sit in one half-warp; each group is summed in lane order and
//     its lowest lane writes the parent's R once (no atomics; the reference
//     adds the same FP32 terms with atomics, __buildMultiLevelR_optimized_new
//     :729-847);
//   * the coarse domain applies (levels >= 1) and the level-0 domain apply:
//     half a warp per 48x48 domain, lane l holding block (l, (l + d) % 16) of
//     the wrapped diagonals d = 0..8, each stored block serving both
//     triangles through a shuffle of width 16 (_schwarzLocalXSym6 :957-1027);
//   * the prolongation: a vertex's z is its level-0 result plus the coarse
//     results along its coarse table, in level order (__collectFinalZ_new
//     :850-881), with r.z.  Sequentially it is fused into the level-0 apply;
//     with the coarse levels on the side stream beside the level-0 apply it
//     is a pass of its own after the join (the same FP32 sums either way).
struct Mas16Args {
  const int* pmr;
  const int* going_next;
  const int* coarse_table;  // 6 global slots per vertex (levels 1..L-1)
  LevelInfo lv;
  const float* inv;  // kMas16InvElems per domain
  float* coarse_r;   // (total_clusters - c0) x 3
  float* coarse_z;
  int fem_off, c0;
};

// R of level l+1 from level l (l = 0: from r).
template <typename Tv>
__global__ void __launch_bounds__(kTpb) k16_restrict(Mas16Args a, const Tv* __restrict__ r, int level, PcgScalars* s)
{
  pdl_wait();
  if (s && s->status != MASPCG_SOLVE_RUNNING) return;
  const int count = level == 0 ? a.c0 : a.lv.count[level];
  const int padded = (count + 15) & ~15;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if ((t & ~31) >= padded) return;  // whole warp past the level
  float v[3] = {0.f, 0.f, 0.f};
  int parent = -1;
  if (t < count) {
    if (level == 0) {
      const int vtx = a.pmr[t];
      if (vtx >= 0) {
        const size_t base = 3 * (size_t)(a.fem_off + t);
        v[0] = (float)r[base];
        v[1] = (float)r[base + 1];
        v[2] = (float)r[base + 2];
        parent = a.going_next[vtx];
      }
    } else {
      const int slot = a.lv.begin[level] + t;
      const float* x = a.coarse_r + 3 * (size_t)(slot - a.c0);
      v[0] = x[0];
      v[1] = x[1];
      v[2] = x[2];
      parent = a.going_next[slot];
    }
  }
  float o[3];
  bool leader;
  group_sum<false>(parent >= 0 ? parent : -1 - (int)(threadIdx.x & 31), v, o, leader);
  if (parent >= 0 && leader) {
    float* d = a.coarse_r + 3 * (size_t)(parent - a.c0);
    d[0] = o[0];
    d[1] = o[1];
    d[2] = o[2];
  }
}

// y = M x for the domain of this half-warp (lane = t & 15); x of the lane's
// node; all 32 lanes of the warp take part (in = false: x = 0, no loads).
// The lane's 81 record elements are all loaded before the arithmetic, so a
// warp has its whole 10 KB in flight at once.
__device__ __forceinline__ void domain_apply16(const float* __restrict__ inv, bool in, int lane, const float x[3],
                                               float y[3])
{
  float Bm[kMas16Diags * 9];
#pragma unroll
  for (int k = 0; k < kMas16Diags * 9; ++k) Bm[k] = in ? __ldcs(inv + k * 16 + lane) : 0.f;
  float y0 = 0.f, y1 = 0.f, y2 = 0.f;
#pragma unroll
  for (int d = 0; d < kMas16Diags; ++d) {
    const int c = (lane + d) & 15;
    const float c0 = __shfl_sync(kFull, x[0], c, 16), c1 = __shfl_sync(kFull, x[1], c, 16),
                c2 = __shfl_sync(kFull, x[2], c, 16);
    const float* B = Bm + 9 * d;
    y0 += B[0] * c0 + B[1] * c1 + B[2] * c2;
    y1 += B[3] * c0 + B[4] * c1 + B[5] * c2;
    y2 += B[6] * c0 + B[7] * c1 + B[8] * c2;
    if (d != 0) {
      const float t0 = B[0] * x[0] + B[3] * x[1] + B[6] * x[2];
      const float t1 = B[1] * x[0] + B[4] * x[1] + B[7] * x[2];
      const float t2 = B[2] * x[0] + B[5] * x[1] + B[8] * x[2];
      const int src = (lane - d) & 15;
      y0 += __shfl_sync(kFull, t0, src, 16);
      y1 += __shfl_sync(kFull, t1, src, 16);
      y2 += __shfl_sync(kFull, t2, src, 16);
    }
  }
  y[0] = y0;
  y[1] = y1;
  y[2] = y2;
}

// All coarse domains (levels >= 1).  pair: the grid's R.Z (= r . P Z, the
// coarse part of r.z) completes part 1 of the pair r.z.
template <typename Tacc>
__global__ void __launch_bounds__(kTpb, 2) k16_apply_coarse(Mas16Args a, Tacc* cpart, PcgScalars* s, int mode,
                                                           int pair)
{
  pdl_wait();
  if (s && s->status != MASPCG_SOLVE_RUNNING) return;  // uniform: nothing changes the status meanwhile
  const int d1 = a.lv.dom_begin[1];
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int g = d1 + (t >> 4), lane = t & 15;
  const bool in = g < a.lv.domains;
  const size_t base = 3 * (size_t)(16 * g + lane - a.c0);
  float x[3] = {0.f, 0.f, 0.f}, y[3];
  if (in) {
    x[0] = a.coarse_r[base];
    x[1] = a.coarse_r[base + 1];
    x[2] = a.coarse_r[base + 2];
  }
  domain_apply16(a.inv + (size_t)(in ? g : 0) * kMas16InvElems, in, lane, x, y);
  Tacc dot = 0;
  if (in) {
    a.coarse_z[base] = y[0];
    a.coarse_z[base + 1] = y[1];
    a.coarse_z[base + 2] = y[2];
    dot = (Tacc)x[0] * (Tacc)y[0] + (Tacc)x[1] * (Tacc)y[1] + (Tacc)x[2] * (Tacc)y[2];
  }
  if (!pair || !s) return;
  Tacc total = 0;
  if (grid_finish<Tacc>(dot, cpart, blockIdx.x, gridDim.x, &s->tickets[kTicketCoarse], gridDim.x, total) &&
      threadIdx.x == 0)
    rz_part_done(s, 1, (double)total, mode);
}

// CTAs of k16_apply_coarse.
inline int mas16_coarse_grid(const maspcg_handle* h)
{
  return std::max(1, ceil_div((long long)(h->lv.domains - h->lv.dom_begin[1]) * 16, kTpb));
}

// The coarse correction and r.z of one slot's z (y holds the level-0 result
// in FP32 precision).
template <typename Tv, typename Tacc>
__device__ __forceinline__ Tacc prolong16(const Mas16Args& a, int vtx, const Tv rv[3], float y[3], Tv* zp)
{
  if (vtx >= 0) {
    const int* ct = a.coarse_table + 6 * (size_t)vtx;
    for (int l = 1; l < a.lv.levelnum; ++l) {
      const float* zc = a.coarse_z + 3 * (size_t)(ct[l - 1] - a.c0);
      y[0] += zc[0];
      y[1] += zc[1];
      y[2] += zc[2];
    }
  } else {
    y[0] = y[1] = y[2] = 0.f;
  }
  Tacc dot = 0;
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    const Tv zv = (Tv)y[q];
    zp[q] = zv;
    dot += (Tacc)rv[q] * (Tacc)zv;
  }
  return dot;
}

template <typename Tacc>
__device__ __forceinline__ void rz_finish(Tacc dot, Tacc* partial, int part_base, int total_parts, int mode,
                                          PcgScalars* s)
{
  if (!partial) return;
  Tacc total = 0;
  if (grid_finish<Tacc>(dot, partial, part_base + blockIdx.x, total_parts, &s->tickets[kTicketRz], gridDim.x, total) &&
      threadIdx.x == 0 && mode > 0)
    rz_update(s, (double)total, mode);
}

// kProlong: add the coarse correction and sum r.z (the coarse levels ran
// before).  Else z = the level-0 result (the next p update adds the coarse
// correction), and r.z0 completes part 0 of the pair r.z.
template <typename Tv, typename Tacc, bool kProlong>
__global__ void __launch_bounds__(kTpb, 2) k16_apply_level0(Mas16Args a, const Tv* __restrict__ r, Tv* z, Tacc* partial,
                                                         int part_base, int total_parts, int mode, PcgScalars* s)
{
  pdl_wait();
  if (s && s->status != MASPCG_SOLVE_RUNNING) return;
  const int d0 = a.lv.dom_begin[1];
  Tacc dot = 0;
  const int stride = gridDim.x * blockDim.x;
  const int span = (d0 * 16 + 31) & ~31;  // whole warps
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < span; t += stride) {
    const int g = t >> 4, lane = t & 15;
    const bool in = g < d0;
    const int slot = 16 * g + lane;
    const int vtx = in ? a.pmr[slot] : -1;
    const size_t base = 3 * (size_t)(a.fem_off + slot);
    Tv rv[3] = {0, 0, 0};
    float x[3] = {0.f, 0.f, 0.f}, y[3];
    if (vtx >= 0) {
      rv[0] = r[base];
      rv[1] = r[base + 1];
      rv[2] = r[base + 2];
      x[0] = (float)rv[0];
      x[1] = (float)rv[1];
      x[2] = (float)rv[2];
    }
    domain_apply16(a.inv + (size_t)(in ? g : 0) * kMas16InvElems, in, lane, x, y);
    if (!in) continue;
    if (kProlong) {
      dot += prolong16<Tv, Tacc>(a, vtx, rv, y, z + base);
    } else {
      const bool real = vtx >= 0;
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        const Tv zv = real ? (Tv)y[q] : Tv(0);
        z[base + q] = zv;
        dot += (Tacc)rv[q] * (Tacc)zv;
      }
    }
  }
  pdl_trigger();
  if (kProlong) {
    rz_finish(dot, partial, part_base, total_parts, mode, s);
  } else if (partial) {
    Tacc total = 0;
    if (grid_finish<Tacc>(dot, partial, part_base + blockIdx.x, total_parts, &s->tickets[kTicketRz], gridDim.x,
                          total) &&
        threadIdx.x == 0)
      rz_part_done(s, 0, (double)total, mode);
  }
}

Mas16Args make_mas16_args(maspcg_handle* h)
{
  Mas16Args a{};
  a.pmr = h->pmr.get();
  a.going_next = h->going_next.get();
  a.coarse_table = h->coarse_table.get();
  a.lv = h->lv;
  a.inv = reinterpret_cast<const float*>(h->inv.get());
  a.coarse_r = h->coarse_r.get();
  a.coarse_z = h->coarse_z.get();
  a.fem_off = h->fem_off;
  a.c0 = h->c0;
  return a;
}

}  // namespace

// Level-0 apply + prolongation + r.z; with `partial` set, the last block
// completes the r.z reduction over [0, total_parts) and, for mode > 0,
// updates the PCG scalars (rz0 / beta / k).
template <typename TI, typename Tv, typename Tacc, bool kFused>
__global__ void MAS_APPLY_BOUNDS(TI) k_level0_apply(ApplyArgs a, const Tv* __restrict__ r, Tv* z, Tacc* partial,
                                                      int part_base, int total_parts, int mode, PcgScalars* s,
                                                      int coarse_add, int pair, FusedArgs fa, double* partial_rr)
{
  pdl_wait();
  if (s && s->status != MASPCG_SOLVE_RUNNING) return;
  const int lane = threadIdx.x & 31;
  const int warps_total = gridDim.x * (blockDim.x >> 5);
  Tacc dot = 0;
  double rr = 0.0;
  FusedScal fs{};
  if constexpr (kFused) fs = fused_scalars(s);
  for (int g = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; g < a.lv.dom_begin[1]; g += warps_total) {
    const int slot = kBank * g + lane;
    const size_t row3 = 3 * (size_t)(a.fem_off + slot);
    Tv r0, r1, r2;
    if constexpr (kFused) {
      float rn[3];
      fused_input_row(fa, fs, a.fem_off + slot, true, rn);
      r0 = rn[0], r1 = rn[1], r2 = rn[2];
      if (fa.update) rr += (double)rn[0] * rn[0] + (double)rn[1] * rn[1] + (double)rn[2] * rn[2];
    } else {
      r0 = r[row3], r1 = r[row3 + 1], r2 = r[row3 + 2];
    }
    const float x[3] = {(float)r0, (float)r1, (float)r2};
    float y[3];
    if constexpr (sizeof(TI) == 2) {
      extern __shared__ __align__(16) unsigned char direct_slots[];
      unsigned char* slot = direct_slots + (size_t)(threadIdx.x >> 5) * (kRecBytes16 + kApplyScratch);
      stage_record(reinterpret_cast<const uint4*>(a.inv) + (size_t)g * (kRecBytes16 / 16), slot, lane);
      const float* scg = a.scale + (size_t)g * 96 + 3 * lane;
      const float sc[3] = {scg[0], scg[1], scg[2]};
      domain_apply16<TI>(reinterpret_cast<const TI*>(slot), slot + kRecBytes16, sc, lane, x, y);
    } else {
      domain_apply(reinterpret_cast<const float*>(a.inv) + (size_t)g * kInvElems, lane, x, y);
    }
    float cc[3];
    const bool real = coarse_add ? coarse_correction(a, slot, cc) : a.pmr[slot] >= 0;
    if (!real) {
      y[0] = y[1] = y[2] = 0.f;
    } else if (coarse_add) {
      y[0] += cc[0];
      y[1] += cc[1];
      y[2] += cc[2];
    }
    z[row3] = (Tv)y[0];
    z[row3 + 1] = (Tv)y[1];
    z[row3 + 2] = (Tv)y[2];
    dot += (Tacc)r0 * (Tacc)(Tv)y[0] + (Tacc)r1 * (Tacc)(Tv)y[1] + (Tacc)r2 * (Tacc)(Tv)y[2];
  }
  pdl_trigger();
  if (kFused && fa.update) {
    double rt = 0.0;
    if (grid_finish<double, kApplyTpb>(rr, partial_rr, part_base + blockIdx.x, total_parts, &s->tickets[kTicketXr],
                                       gridDim.x, rt) &&
        threadIdx.x == 0)
      s->rr = rt;
  }
  if (partial) {
    Tacc total = 0;
    if (grid_finish<Tacc, kApplyTpb>(dot, partial, part_base + blockIdx.x, total_parts, &s->tickets[kTicketRz], gridDim.x,
                          total) &&
        threadIdx.x == 0 && mode > 0) {
      if (pair)
        rz_part_done(s, 0, (double)total, mode);
      else
        rz_update(s, (double)total, mode);
    }
  }
}

// Domain apply with the inverse staged by TMA: each warp streams its
// domains' stored records (one contiguous bulk copy per domain) into kBuf
// shared-memory slots of its own and applies them from there, so the two
// passes of the factored form read global memory once.  kBuf = 2 overlaps a
// warp's next copy with its arithmetic; kBuf = 1 halves the shared memory per
// warp and fits more warps per SM.  Level 0 reads r / writes z (plus the
// coarse correction and r.z); coarse levels read and write the coarse R/Z
// arrays.  Every wait is bounded; on expiry the warp drains its copies,
// records the error and the whole CTA leaves.
constexpr int kApplyWarps = 4;

template <typename TI, typename Tv, typename Tacc, bool kLevel0, int kBuf, bool kFused>
__global__ void __launch_bounds__(kApplyWarps * 32, kBuf == 1 ? 4 : 2)
    k_apply_tma(ApplyArgs a, const Tv* __restrict__ r, Tv* z, Tacc* partial, int part_base, int total_parts, int mode,
                PcgScalars* s, int g_begin, int g_end, int* err, int coarse_add, int pair, FusedArgs fa,
                double* partial_rr)
{
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ __align__(8) uint64_t bar[kApplyWarps][kBuf];
  pdl_wait();
  if (s && s->status != MASPCG_SOLVE_RUNNING) return;
  static_assert(sizeof(TI) == 2, "the staged apply holds 16-bit records");
  constexpr unsigned kBytes = kRecBytes16;
  const int lw = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int warps_total = gridDim.x * kApplyWarps;
  const int gw = blockIdx.x * kApplyWarps + lw;
  unsigned char* buf = smem + (size_t)lw * (kBuf * kBytes + kApplyScratch);
  const TI* inv = reinterpret_cast<const TI*>(a.inv);
  if (lane == 0) {
#pragma unroll
    for (int j = 0; j < kBuf; ++j) mbar_init(&bar[lw][j], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
#pragma unroll
    for (int j = 0; j < kBuf; ++j) {
      const int gj = g_begin + gw + j * warps_total;
      if (gj < g_end) {
        mbar_expect_tx(&bar[lw][j], kBytes);
        tma_bulk_g2s(buf + j * kBytes, inv + (size_t)gj * inv_elems<TI>(), kBytes, &bar[lw][j]);
      }
    }
  }
  __syncwarp();
  unsigned ph[kBuf];
#pragma unroll
  for (int j = 0; j < kBuf; ++j) ph[j] = 0;
  Tacc dot = 0;
  double rr = 0.0;
  FusedScal fs{};
  if constexpr (kFused) fs = fused_scalars(s);
  int i = 0;
  bool ok = true;
  for (int g = g_begin + gw; g < g_end; g += warps_total, ++i) {
    const int st = kBuf == 1 ? 0 : (i & 1);
    // loads that do not depend on the record go out before its wait
    const float* scg = a.scale + (size_t)g * 96 + 3 * lane;
    const float sc[3] = {__ldg(scg), __ldg(scg + 1), __ldg(scg + 2)};
    float x[3], y[3];
    Tv rv[3];
    size_t base;
    if (kLevel0) {
      base = 3 * (size_t)(a.fem_off + kBank * g + lane);
      if constexpr (kFused) {
        float rn[3];
        fused_input_row(fa, fs, a.fem_off + kBank * g + lane, true, rn);
        rv[0] = rn[0];
        rv[1] = rn[1];
        rv[2] = rn[2];
        if (fa.update) rr += (double)rn[0] * rn[0] + (double)rn[1] * rn[1] + (double)rn[2] * rn[2];
      } else {
        rv[0] = r[base];
        rv[1] = r[base + 1];
        rv[2] = r[base + 2];
      }
      x[0] = (float)rv[0];
      x[1] = (float)rv[1];
      x[2] = (float)rv[2];
    } else {
      base = (size_t)(kBank * g + lane - a.c0) * 3;
      x[0] = a.coarse_r[base];
      x[1] = a.coarse_r[base + 1];
      x[2] = a.coarse_r[base + 2];
      rv[0] = rv[1] = rv[2] = Tv(0);
    }
    const bool padded = kLevel0 && !coarse_add && a.pmr[kBank * g + lane] < 0;
    const bool w = mbar_wait(&bar[lw][st], ph[st]);
    if (w) ph[st] ^= 1u;
    if (!__all_sync(kFull, w)) {
      ok = false;
      break;
    }
    const TI* blk = reinterpret_cast<const TI*>(buf + st * kBytes);
    domain_apply16<TI>(blk, buf + kBuf * kBytes, sc, lane, x, y);
    __syncwarp();
    const int gn = g + kBuf * warps_total;
    if (lane == 0 && gn < g_end) {
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      mbar_expect_tx(&bar[lw][st], kBytes);
      tma_bulk_g2s(buf + st * kBytes, inv + (size_t)gn * inv_elems<TI>(), kBytes, &bar[lw][st]);
    }
    if (kLevel0) {
      const int slot = kBank * g + lane;
      float cc[3];
      const bool real = coarse_add ? coarse_correction(a, slot, cc) : !padded;
      if (!real) {
        y[0] = y[1] = y[2] = 0.f;
      } else if (coarse_add) {
        y[0] += cc[0];
        y[1] += cc[1];
        y[2] += cc[2];
      }
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        const Tv zv = (Tv)y[q];
        z[base + q] = zv;
        dot += (Tacc)rv[q] * (Tacc)zv;
      }
    } else {
      a.coarse_z[base] = y[0];
      a.coarse_z[base + 1] = y[1];
      a.coarse_z[base + 2] = y[2];
    }
  }
  pdl_trigger();
  if (!ok && lane == 0) {
    // drain this warp's copies still in flight (bounded), report
    atomicExch(err, 1);
#pragma unroll
    for (int j = 0; j < kBuf; ++j) {
      const int gj = g_begin + gw + (i + j) * warps_total;
      const int sj = kBuf == 1 ? 0 : ((i + j) & 1);
      if (gj < g_end) mbar_wait(&bar[lw][sj], ph[sj]);
    }
    if (s) s->status = MASPCG_SOLVE_NONFINITE;
  }
  if (__syncthreads_or(!ok)) return;  // the whole CTA leaves together
  if (kFused && kLevel0 && fa.update) {
    // r.r of the updated residual first: its last block stores it before its
    // arrival on the r.z ticket, so the r.z completion below sees it
    double rt = 0.0;
    if (grid_finish<double, kApplyWarps * 32>(rr, partial_rr, part_base + blockIdx.x, total_parts,
                                              &s->tickets[kTicketXr], gridDim.x, rt) &&
        threadIdx.x == 0)
      s->rr = rt;
  }
  if (kLevel0 && partial) {
    Tacc total = 0;
    if (grid_finish<Tacc, kApplyWarps * 32>(dot, partial, part_base + blockIdx.x, total_parts, &s->tickets[kTicketRz],
                                            gridDim.x, total) &&
        threadIdx.x == 0 && mode > 0) {
      if (pair)
        rz_part_done(s, 0, (double)total, mode);
      else
        rz_update(s, (double)total, mode);
    }
  }
}

void launch_factor(maspcg_handle* h, double* assembled_out);
namespace {
ApplyArgs make_apply_args(maspcg_handle* h);
}

void build_mas_domains(maspcg_handle* h, double* assembled_out)
{
  cudaStream_t st = h->stream;
  const LevelInfo& lv = h->lv;
  const int c0 = h->c0;
  // member lists per coarse level
  h->sort_keys.resize(c0);
  h->sort_keys_out.resize(c0);
  h->sort_vals.resize(c0);
  size_t need = 0;
  MCK(cub::DeviceRadixSort::SortPairs(nullptr, need, (const unsigned*)nullptr, (unsigned*)nullptr, (const int*)nullptr,
                                      (int*)nullptr, c0, 0, 32));
  h->cub_tmp.resize(std::max(need, h->cub_tmp.n));
  for (int l = 1; l < lv.levelnum; ++l) {
    const int count = lv.count[l];
    int bits = 1;
    while ((1ll << bits) <= count) ++bits;
    k_member_keys<<<ceil_div(c0, kTpb), kTpb, 0, st>>>(h->cmap[l].get(), c0, count,
                                                      reinterpret_cast<unsigned*>(h->sort_keys.get()),
                                                      h->sort_vals.get()); MLAUNCHED(h);
    h->perm[l].resize(c0);
    h->off[l].resize(count + 1);
    size_t tb = h->cub_tmp.cap;
    MCK(cub::DeviceRadixSort::SortPairs(h->cub_tmp.get(), tb, reinterpret_cast<const unsigned*>(h->sort_keys.get()),
                                        reinterpret_cast<unsigned*>(h->sort_keys_out.get()), h->sort_vals.get(),
                                        h->perm[l].get(), c0, 0, bits, st));
    k_member_offsets<<<ceil_div(h->nv, kTpb), kTpb, 0, st>>>(
        reinterpret_cast<const unsigned*>(h->sort_keys_out.get()), h->nv, count, h->off[l].get()); MLAUNCHED(h);
  }
  // storage (16-slot banks: FP32 only)
  const int storage = h->bank == 16 ? (int)MASPCG_INV_FP32 : h->cfg.inverse_storage;
  const size_t esize = storage == MASPCG_INV_FP32 ? 4 : 2;
  h->inv.resize((size_t)lv.domains * (h->bank == 16 ? kMas16InvElems : inv_elems_for(storage)) * esize, 16);
  if (storage != MASPCG_INV_FP32) h->inv_scale.resize((size_t)lv.domains * 96);
  MCK(cudaMemsetAsync(h->failed.get() + 3, 0, sizeof(int), st));
  launch_factor(h, assembled_out);
  // coarse work vectors (padding entries stay zero)
  const size_t coarse = (size_t)(lv.total_clusters - c0) * 3;
  h->coarse_r.resize(coarse > 0 ? coarse : 3);
  h->coarse_z.resize(coarse > 0 ? coarse : 3);
  if (h->bank == 16) {
    h->chain_dot.resize((size_t)mas16_coarse_grid(h));  // k16_apply_coarse's R.Z partials
    MCK(cudaMemsetAsync(h->coarse_r.get(), 0, h->coarse_r.bytes(), st));
    MCK(cudaMemsetAsync(h->coarse_z.get(), 0, h->coarse_z.bytes(), st));
    int f = 0;
    MCK(cudaMemcpyAsync(&f, h->failed.get() + 3, sizeof(int), cudaMemcpyDeviceToHost, st));
    MCK(cudaStreamSynchronize(st));
    h->failed_domains = f;
    return;
  }
  const int coarse_domains = lv.domains - lv.dom_begin[1];
  h->chain_count.resize((size_t)std::max(coarse_domains, 1));
  h->chain_target.resize((size_t)std::max(coarse_domains, 1));
  h->chain_dot.resize((size_t)std::max(coarse_domains, 1));
  MCK(cudaMemsetAsync(h->chain_count.get(), 0, h->chain_count.bytes(), st));
  MCK(cudaMemsetAsync(h->chain_target.get(), 0, h->chain_target.bytes(), st));
  if (lv.levelnum > 1) {
    const ApplyArgs aa = make_apply_args(h);
    const long long units = (c0 / kBank + kChainUnitBanks - 1) / kChainUnitBanks + coarse_domains;
    k_chain_targets<<<ceil_div(units * 32, kTpb), kTpb, 0, st>>>(aa, h->chain_target.get());
    MLAUNCHED(h);
  }
  MCK(cudaMemsetAsync(h->coarse_r.get(), 0, h->coarse_r.bytes(), st));
  MCK(cudaMemsetAsync(h->coarse_z.get(), 0, h->coarse_z.bytes(), st));
  int f = 0;
  MCK(cudaMemcpyAsync(&f, h->failed.get() + 3, sizeof(int), cudaMemcpyDeviceToHost, st));
  MCK(cudaStreamSynchronize(st));
  h->failed_domains = f;
}

template <int kB>
void launch_factor_t(maspcg_handle* h, double* assembled_out, bool gather_only = false)
{
  cudaStream_t st = h->stream;
  const LevelInfo& lv = h->lv;
  const int c0 = h->c0;
  const int storage = kB == 16 ? (int)MASPCG_INV_FP32 : h->cfg.inverse_storage;
  const int d0 = lv.dom_begin[1];
  const int coarse_domains = lv.domains - d0;
  // coarse-level Galerkin sums (kept from the build when only gathering)
  if (!gather_only) h->coarse64.resize((size_t)std::max(coarse_domains, 1) * kB * kB * 9);
  CoarseArgs ca{};
  ca.pmr = h->pmr.get();
  ca.prefix_orig = h->prefix_orig.get();
  ca.levelnum = lv.levelnum;
  ca.slice_rows = 64;
  ca.nv = h->nv;
  int items = 0;
  for (int l = 1; l < lv.levelnum; ++l) {
    ca.perm[l] = h->perm[l].get();
    ca.cmap[l] = h->cmap[l].get();
    ca.slice_base[l] = items;
    items += ceil_div(h->nv, ca.slice_rows);
  }
  ca.slice_base[lv.levelnum] = items;
  for (int l = 0; l <= lv.levelnum; ++l) ca.dom_begin[l] = lv.dom_begin[l];
  ca.rowptr = h->rowptr.get();
  ca.colidx = h->colidx.get();
  ca.val64 = h->val64.get();
  ca.fem_off = h->fem_off;
  ca.c0 = c0;
  ca.coarse64 = h->coarse64.get();
  // The coarse sums feed only the coarse domains: with level-0 domains to
  // factor they are assembled on the side stream meanwhile, and the coarse
  // domains are factored after the join.
  const bool split = !gather_only && items > 0 && d0 > 0 && coarse_domains > 0;
  if (!gather_only) {
    cudaStream_t cs = st;
    if (split) {
      MCK(cudaEventRecord(h->ev_fork, st));
      MCK(cudaStreamWaitEvent(h->side_stream, h->ev_fork, 0));
      cs = h->side_stream;
    }
    MCK(cudaMemsetAsync(h->coarse64.get(), 0, (size_t)coarse_domains * kB * kB * 9 * sizeof(double), cs));
    if (items > 0) {
      k_coarse_assemble<kB><<<ceil_div((long long)items * 32, 256), 256, 0, cs>>>(ca);
      MLAUNCHED(h);
    }
    if (split) MCK(cudaEventRecord(h->ev_join, cs));
  }
  FactorArgs fa{};
  fa.lv = lv;
  for (int l = 1; l < lv.levelnum; ++l) {
    fa.cmap[l] = h->cmap[l].get();
    fa.perm[l] = h->perm[l].get();
    fa.off[l] = h->off[l].get();
  }
  fa.pmr = h->pmr.get();
  fa.rowptr = h->rowptr.get();
  fa.colidx = h->colidx.get();
  fa.val64 = h->val64.get();
  fa.fem_off = h->fem_off;
  fa.c0 = c0;
  fa.inv = h->inv.get();
  fa.scale = storage == MASPCG_INV_FP32 ? nullptr : h->inv_scale.get();
  fa.failed = h->failed.get() + 3;
  fa.assembled = assembled_out;
  fa.coarse64 = h->coarse64.get();
  fa.gather_only = gather_only ? 1 : 0;
  if (kB == 32 && storage != MASPCG_INV_FP32 && !gather_only) {
    h->dom64.resize((size_t)lv.domains * kPacked * 9);
    fa.dom64 = h->dom64.get();
  }
  // domains [g0, g0 + n): gather / Gauss-Jordan, then the 16-bit Cholesky
  auto factor = [&](int g0, int n) {
    if (n <= 0) return;
#define MAS_FACTOR(TI, ASM) k_domain_factor<TI, ASM, kB><<<n, 32 * kB, 0, st>>>(fa, g0)
    if constexpr (kB == 16) {
      if (assembled_out)
        MAS_FACTOR(float, true);
      else
        MAS_FACTOR(float, false);
    } else if (assembled_out) {
      if (storage == MASPCG_INV_FP32)
        MAS_FACTOR(float, true);
      else if (storage == MASPCG_INV_BF16)
        MAS_FACTOR(__nv_bfloat16, true);
      else
        MAS_FACTOR(__half, true);
    } else {
      if (storage == MASPCG_INV_FP32)
        MAS_FACTOR(float, false);
      else if (storage == MASPCG_INV_BF16)
        MAS_FACTOR(__nv_bfloat16, false);
      else
        MAS_FACTOR(__half, false);
    }
#undef MAS_FACTOR
    MLAUNCHED(h);
    if (gather_only) return;
    if constexpr (kB == 32) {
      if (storage == MASPCG_INV_BF16) {
        k_domain_chol16<__nv_bfloat16><<<n, kCholThreads, 0, st>>>(fa, g0);
        MLAUNCHED(h);
      } else if (storage == MASPCG_INV_FP16) {
        k_domain_chol16<__half><<<n, kCholThreads, 0, st>>>(fa, g0);
        MLAUNCHED(h);
      }
    }
  };
  if (split) {
    factor(0, d0);
    MCK(cudaStreamWaitEvent(st, h->ev_join, 0));
    factor(d0, lv.domains - d0);
  } else {
    factor(0, lv.domains);
  }
  MCK(cudaGetLastError());
}

void launch_factor(maspcg_handle* h, double* assembled_out)
{
  if (h->bank == 16)
    launch_factor_t<16>(h, assembled_out);
  else
    launch_factor_t<32>(h, assembled_out);
}

void gather_mas_domains(maspcg_handle* h, double* assembled_out)
{
  if (h->bank == 16)
    launch_factor_t<16>(h, assembled_out, true);
  else
    launch_factor_t<32>(h, assembled_out, true);
}

namespace {
ApplyArgs make_apply_args(maspcg_handle* h)
{
  ApplyArgs a{};
  a.cmap1 = h->cmap[1].get();
  a.going_next = h->going_next.get();
  a.coarse_r = h->coarse_r.get();
  a.coarse_z = h->coarse_z.get();
  for (int l = 1; l < h->lv.levelnum && l < kMaxLevels; ++l) a.cmap[l] = h->cmap[l].get();
  a.pmr = h->pmr.get();
  a.chain_count = h->chain_count.get();
  a.chain_target = h->chain_target.get();
  a.chain_dot = h->chain_dot.get();
  a.err = h->failed.get() + 4;
  a.inv = h->inv.get();
  a.scale = h->cfg.inverse_storage == MASPCG_INV_FP32 ? nullptr : h->inv_scale.get();
  a.fem_off = h->fem_off;
  a.c0 = h->c0;
  a.lv = h->lv;
  return a;
}

// Level-0 domain apply variants (the solve uses h->apply_variant).
enum ApplyVariant { kApplyDirect = 0, kApplyStaged2 = 1, kApplyStaged1 = 2 };

template <typename TI, typename Tv, typename Tacc, bool kLevel0, int kBuf, bool kFused = false>
void launch_apply_tma(maspcg_handle* h, const ApplyArgs& a, const Tv* r, Tv* z, Tacc* partial, int part_base,
                      int total_parts, int mode, PcgScalars* s, int g_begin, int g_end, int grid, int coarse_add,
                      int pair, const FusedArgs& fa = FusedArgs{}, double* partial_rr = nullptr)
{
  constexpr int bytes = kApplyWarps * (kBuf * kRecBytes16 + kApplyScratch);
  auto kern = k_apply_tma<TI, Tv, Tacc, kLevel0, kBuf, kFused>;
  static bool configured = false;
  if (!configured) {
    MCK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    configured = true;
  }
  launch_pdl(h, kern, dim3(grid), dim3(kApplyWarps * 32), bytes, a, r, z, partial, part_base, total_parts, mode, s,
             g_begin, g_end, h->failed.get() + 4, coarse_add, pair, fa, partial_rr);
}

// CTAs of a staged apply over `domains` domains: one wave of resident CTAs.
inline int staged_grid(const maspcg_handle* h, int domains, int kbuf)
{
  return std::max(1, std::min(ceil_div(domains, kApplyWarps), (kbuf == 1 ? 4 : 2) * h->sm_count));
}

// CTAs of the level-0 apply in a variant.  The r.z partial sums occupy one
// slot per CTA, so the PCG engine sizes its reduction with this same count.
inline int level0_grid(const maspcg_handle* h, int variant)
{
  const int d0 = h->lv.dom_begin[1];
  if (h->cfg.inverse_storage == MASPCG_INV_FP32) variant = kApplyDirect;
  switch (variant) {
    case kApplyStaged2: return staged_grid(h, d0, 2);
    case kApplyStaged1: return staged_grid(h, d0, 1);
    default:
      return std::max(1, std::min(ceil_div((long long)d0 * 32, kApplyTpb),
                                  (h->cfg.inverse_storage == MASPCG_INV_FP32 ? 16 : 4) * h->sm_count));
  }
}

// Level-0 apply (with r.z) in the given variant; coarse_add: z includes the
// coarse correction (else the p update adds it); pair: r.z is completed
// together with the concurrently running coarse levels.
template <typename TI, typename Tv, typename Tacc, bool kFused = false>
void level0_apply(maspcg_handle* h, const ApplyArgs& a, int variant, const Tv* r, Tv* z, Tacc* partial, int part_base,
                  int total_parts, int mode, PcgScalars* s, int grid0, int coarse_add = 1, int pair = 0,
                  const FusedArgs& fa = FusedArgs{}, double* partial_rr = nullptr)
{
  const int d0 = h->lv.dom_begin[1];
  if (std::is_same<TI, float>::value) variant = kApplyDirect;
  // grid0 == level0_grid(h, variant): every CTA owns one r.z slot
  switch (variant) {
    case kApplyStaged2:
      if constexpr (sizeof(TI) == 2)
        launch_apply_tma<TI, Tv, Tacc, true, 2, kFused>(h, a, r, z, partial, part_base, total_parts, mode, s, 0, d0,
                                                        grid0, coarse_add, pair, fa, partial_rr);
      break;
    case kApplyStaged1:
      if constexpr (sizeof(TI) == 2)
        launch_apply_tma<TI, Tv, Tacc, true, 1, kFused>(h, a, r, z, partial, part_base, total_parts, mode, s, 0, d0,
                                                        grid0, coarse_add, pair, fa, partial_rr);
      break;

    default:
      launch_pdl(h, k_level0_apply<TI, Tv, Tacc, kFused>, dim3(grid0), dim3(kApplyTpb),
                 sizeof(TI) == 2 ? kDirectSmem16 : 0, a, r, z, partial, part_base, total_parts, mode, s, coarse_add,
                 pair, fa, partial_rr);
      break;
  }
}

template <typename TI, typename Tv, bool kFused = false>
void launch_chain(maspcg_handle* h, cudaStream_t st, const ApplyArgs& a, const Tv* r, PcgScalars* s, int mode, int pair,
                  const FusedArgs& fa = FusedArgs{})
{
  constexpr int bytes = chain_smem_bytes<TI>();
  auto kern = k_coarse_chain<TI, Tv, kFused>;
  static bool configured = false;
  if (!configured && bytes > 48 * 1024)
    MCK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  configured = true;
  launch_pdl_on(h, st, kern, dim3(ceil_div(h->c0 / kBank, kChainUnitBanks)), dim3(kChainWarps * 32), bytes, a, r, s,
                mode, pair, fa);
}

// The MAS apply.  Sequential form: the coarse levels, then the level-0 apply
// adding the coarse correction.  Overlapped form (inside the solve): the
// coarse levels run on the side stream beside the level-0 apply, the two
// complete r.z together, and the next p update adds the coarse correction.
template <typename TI, typename Tv, typename Tacc>
void mas_apply_t(maspcg_handle* h, const Tv* r, Tv* z, Tacc* partial, int part_base, int total_parts, int mode,
                 int grid0, PcgScalars* s, bool overlap)
{
  ApplyArgs a = make_apply_args(h);
  const LevelInfo& lv = h->lv;
  const int variant = std::is_same<TI, float>::value ? (int)kApplyDirect : h->apply_variant;
  if (lv.levelnum <= 1) {
    level0_apply<TI, Tv, Tacc>(h, a, variant, r, z, partial, part_base, total_parts, mode, s, grid0);
    return;
  }
  if (!overlap || !s) {
    launch_chain<TI, Tv>(h, h->stream, a, r, s, mode, 0);
    level0_apply<TI, Tv, Tacc>(h, a, variant, r, z, partial, part_base, total_parts, mode, s, grid0);
    return;
  }
  MCK(cudaEventRecord(h->ev_fork, h->stream));
  MCK(cudaStreamWaitEvent(h->side_stream, h->ev_fork, 0));
  launch_chain<TI, Tv>(h, h->side_stream, a, r, s, mode, 1);
  MCK(cudaEventRecord(h->ev_join, h->side_stream));
  level0_apply<TI, Tv, Tacc>(h, a, variant, r, z, partial, part_base, total_parts, mode, s, grid0, 0, 1);
  MCK(cudaStreamWaitEvent(h->stream, h->ev_join, 0));
}

// The MAS apply behind the iteration's fused x / r update (fa.update; else
// fa.r[cur] is the residual): the level-0 apply updates its rows and
// preconditions r', the coarse levels restrict the same r' formed again.
// Overlapped (inside the solve, outside the reference precision): the coarse
// levels run on the side stream, r.z is completed from the two parts and the
// next p update adds the coarse correction; else they run first and the
// level-0 apply adds it.  r.r of the update comes from the level-0 apply.
template <typename TI, typename Tacc>
void mas_apply_fused_t(maspcg_handle* h, const FusedArgs& fa, float* z, Tacc* partial, double* partial_rr,
                       int part_base, int total_parts, int mode, int grid0, PcgScalars* s, bool overlap)
{
  ApplyArgs a = make_apply_args(h);
  const LevelInfo& lv = h->lv;
  const int variant = std::is_same<TI, float>::value ? (int)kApplyDirect : h->apply_variant;
  if (lv.levelnum <= 1) {
    level0_apply<TI, float, Tacc, true>(h, a, variant, nullptr, z, partial, part_base, total_parts, mode, s, grid0, 1,
                                        0, fa, partial_rr);
    return;
  }
  if (!overlap) {
    launch_chain<TI, float, true>(h, h->stream, a, nullptr, s, mode, 0, fa);
    level0_apply<TI, float, Tacc, true>(h, a, variant, nullptr, z, partial, part_base, total_parts, mode, s, grid0, 1,
                                        0, fa, partial_rr);
    return;
  }
  MCK(cudaEventRecord(h->ev_fork, h->stream));
  MCK(cudaStreamWaitEvent(h->side_stream, h->ev_fork, 0));
  launch_chain<TI, float, true>(h, h->side_stream, a, nullptr, s, mode, 1, fa);
  MCK(cudaEventRecord(h->ev_join, h->side_stream));
  level0_apply<TI, float, Tacc, true>(h, a, variant, nullptr, z, partial, part_base, total_parts, mode, s, grid0, 0, 1,
                                      fa, partial_rr);
  MCK(cudaStreamWaitEvent(h->stream, h->ev_join, 0));
}

}  // namespace

ApplyArgs mas_apply_args(maspcg_handle* h) { return make_apply_args(h); }



// Explicit launcher used by pcg.cu.
template <typename Tv, typename Tacc>
void mas_apply(maspcg_handle* h, const Tv* r, Tv* z, Tacc* partial, int part_base, int total_parts, int mode,
               int grid0, PcgScalars* s, bool overlap)
{
  switch (h->cfg.inverse_storage) {
    case MASPCG_INV_BF16:
      mas_apply_t<__nv_bfloat16, Tv, Tacc>(h, r, z, partial, part_base, total_parts, mode, grid0, s, overlap);
      break;
    case MASPCG_INV_FP16:
      mas_apply_t<__half, Tv, Tacc>(h, r, z, partial, part_base, total_parts, mode, grid0, s, overlap);
      break;
    default: mas_apply_t<float, Tv, Tacc>(h, r, z, partial, part_base, total_parts, mode, grid0, s, overlap); break;
  }
  MCK(cudaGetLastError());
}

template <typename Tacc>
void mas_apply_fused(maspcg_handle* h, const FusedArgs& fa, float* z, Tacc* partial, double* partial_rr, int part_base,
                     int total_parts, int mode, int grid0, PcgScalars* s, bool overlap)
{
  switch (h->cfg.inverse_storage) {
    case MASPCG_INV_BF16:
      mas_apply_fused_t<__nv_bfloat16, Tacc>(h, fa, z, partial, partial_rr, part_base, total_parts, mode, grid0, s,
                                             overlap);
      break;
    case MASPCG_INV_FP16:
      mas_apply_fused_t<__half, Tacc>(h, fa, z, partial, partial_rr, part_base, total_parts, mode, grid0, s, overlap);
      break;
    default:
      mas_apply_fused_t<float, Tacc>(h, fa, z, partial, partial_rr, part_base, total_parts, mode, grid0, s, overlap);
      break;
  }
  MCK(cudaGetLastError());
}
template void mas_apply_fused<float>(maspcg_handle*, const FusedArgs&, float*, float*, double*, int, int, int, int,
                                     PcgScalars*, bool);
template void mas_apply_fused<double>(maspcg_handle*, const FusedArgs&, float*, double*, double*, int, int, int, int,
                                      PcgScalars*, bool);

// Stage timing helpers: the level-0 domain apply alone, and the domain
// assembly + inversion alone (member lists from the last build).
template <typename Tv, typename Tacc>
void mas_level0_only(maspcg_handle* h, const Tv* r, Tv* z, Tacc* partial, int grid0, PcgScalars* s, int variant)
{
  ApplyArgs a = make_apply_args(h);
  if (variant < 0) variant = h->apply_variant;
  const int grid = level0_grid(h, variant);
  (void)grid0;
  switch (h->cfg.inverse_storage) {
    case MASPCG_INV_BF16:
      level0_apply<__nv_bfloat16, Tv, Tacc>(h, a, variant, r, z, partial, 0, grid, 0, s, grid);
      break;
    case MASPCG_INV_FP16: level0_apply<__half, Tv, Tacc>(h, a, variant, r, z, partial, 0, grid, 0, s, grid); break;
    default:
      MREQ(variant == kApplyDirect || variant == h->apply_variant, MASPCG_ERR_UNSUPPORTED,
           "the staged apply exists for 16-bit inverses only");
      level0_apply<float, Tv, Tacc>(h, a, kApplyDirect, r, z, partial, 0, grid, 0, s, grid);
      break;
  }
  MCK(cudaGetLastError());
}
template void mas_level0_only<float, float>(maspcg_handle*, const float*, float*, float*, int, PcgScalars*, int);
template void mas_level0_only<float, double>(maspcg_handle*, const float*, float*, double*, int, PcgScalars*, int);
template void mas_level0_only<double, double>(maspcg_handle*, const double*, double*, double*, int, PcgScalars*,
                                              int);

template void mas_apply<float, float>(maspcg_handle*, const float*, float*, float*, int, int, int, int, PcgScalars*,
                                      bool);
template void mas_apply<float, double>(maspcg_handle*, const float*, float*, double*, int, int, int, int, PcgScalars*,
                                       bool);
template void mas_apply<double, double>(maspcg_handle*, const double*, double*, double*, int, int, int, int,
                                        PcgScalars*, bool);

int mas_level0_grid(maspcg_handle* h) { return level0_grid(h, h->apply_variant); }

// CTAs of the kernel that completes r.z (level-0 apply or prolongation).
// CTAs of the level-0 apply, which completes r.z (or part 0 of it).  When
// the coarse levels run beside it (inside the solve, outside the reference
// precision) it leaves 16 SMs' worth of CTA slots free: its CTAs take every
// register of an SM, two per SM, so the chain's small launches start at once
// instead of after the apply drains.
int mas16_grid(maspcg_handle* h)
{
  const int sms = (h->overlap_coarse && h->lv.levelnum > 1) ? std::max(h->sm_count - 16, 1) : 4 * h->sm_count;
  return std::max(1, std::min(ceil_div(h->c0, kTpb), 2 * sms));
}

// CEMAS16 apply.  Sequential: the restriction level by level, the coarse
// domain applies, then the level-0 apply with the prolongation and r.z.
// overlap (with s): the restriction and the coarse applies on the side
// stream beside the level-0 apply; z leaves the coarse correction to the
// next p update (as the MAS32 apply does) and r.z is completed from a pair
// of parts, r.z0 over the fine rows and R.Z over the coarse domains.
template <typename Tv, typename Tacc>
void mas16_apply(maspcg_handle* h, const Tv* r, Tv* z, Tacc* partial, int part_base, int total_parts, int mode,
                 int grid, PcgScalars* s, bool overlap)
{
  const Mas16Args a = make_mas16_args(h);
  const LevelInfo& lv = h->lv;
  const bool pair = overlap && s && lv.levelnum > 1;
  auto coarse_levels = [&](cudaStream_t st) {
    for (int l = 0; l + 1 < lv.levelnum; ++l) {
      const int count = l == 0 ? h->c0 : lv.count[l];
      launch_pdl_on(h, st, k16_restrict<Tv>, dim3(std::max(1, ceil_div((count + 15) & ~15, kTpb))), dim3(kTpb), 0,
                    a, r, l, s);
    }
    launch_pdl_on(h, st, k16_apply_coarse<Tacc>, dim3(mas16_coarse_grid(h)), dim3(kTpb), 0, a,
                  reinterpret_cast<Tacc*>(h->chain_dot.get()), s, mode, pair ? 1 : 0);
  };
  if (pair) {
    MCK(cudaEventRecord(h->ev_fork, h->stream));
    MCK(cudaStreamWaitEvent(h->side_stream, h->ev_fork, 0));
    coarse_levels(h->side_stream);
    MCK(cudaEventRecord(h->ev_join, h->side_stream));
    launch_pdl(h, k16_apply_level0<Tv, Tacc, false>, dim3(grid), dim3(kTpb), 0, a, r, z, partial, part_base,
               total_parts, mode, s);
    MCK(cudaStreamWaitEvent(h->stream, h->ev_join, 0));
  } else {
    if (lv.levelnum > 1) coarse_levels(h->stream);
    launch_pdl(h, k16_apply_level0<Tv, Tacc, true>, dim3(grid), dim3(kTpb), 0, a, r, z, partial, part_base,
               total_parts, mode, s);
  }
  MCK(cudaGetLastError());
}
template void mas16_apply<float, float>(maspcg_handle*, const float*, float*, float*, int, int, int, int,
                                        PcgScalars*, bool);
template void mas16_apply<float, double>(maspcg_handle*, const float*, float*, double*, int, int, int, int,
                                         PcgScalars*, bool);
template void mas16_apply<double, double>(maspcg_handle*, const double*, double*, double*, int, int, int, int,
                                          PcgScalars*, bool);

// Decode the stored inverses into the reference's packed FP32 layout.
void decode_inverses(maspcg_handle* h, float* out)
{
  const int D = h->lv.domains;
  const int storage = h->bank == 16 ? (int)MASPCG_INV_FP32 : h->cfg.inverse_storage;
  const size_t esize = storage == MASPCG_INV_FP32 ? 4 : 2;
  std::vector<unsigned char> raw((size_t)D * (h->bank == 16 ? kMas16InvElems : inv_elems_for(storage)) * esize);
  std::vector<float> sc;
  MCK(cudaMemcpyAsync(raw.data(), h->inv.get(), raw.size(), cudaMemcpyDeviceToHost, h->stream));
  if (storage != MASPCG_INV_FP32) {
    sc.resize((size_t)D * 96);
    MCK(cudaMemcpyAsync(sc.data(), h->inv_scale.get(), sc.size() * 4, cudaMemcpyDeviceToHost, h->stream));
  }
  MCK(cudaStreamSynchronize(h->stream));
  auto elem = [&](size_t idx) -> float {
    if (storage == MASPCG_INV_FP32) {
      float f;
      std::memcpy(&f, raw.data() + idx * 4, 4);
      return f;
    }
    uint16_t u;
    std::memcpy(&u, raw.data() + idx * 2, 2);
    if (storage == MASPCG_INV_BF16) {
      uint32_t w = (uint32_t)u << 16;
      float f;
      std::memcpy(&f, &w, 4);
      return f;
    }
    // IEEE half -> float
    const uint32_t sign = (u >> 15) & 1, ex = (u >> 10) & 0x1f, man = u & 0x3ff;
    float f;
    if (ex == 0)
      f = std::ldexp((float)man, -24);
    else if (ex == 31)
      f = man ? NAN : INFINITY;
    else
      f = std::ldexp((float)(man | 0x400), (int)ex - 25);
    return sign ? -f : f;
  };
  if (h->bank == 16) {
    for (int g = 0; g < D; ++g)
      for (int a = 0; a < 16; ++a)
        for (int b = a; b < 16; ++b) {
          const int d = b - a;
          const bool direct = d <= 8;
          const int lane = direct ? a : b, dd = direct ? d : 16 - d;
          float* o = out + ((size_t)g * kMas16Packed + (16 * a - a * (a + 1) / 2 + b)) * 9;
          for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
              const int ei = direct ? 3 * i + j : 3 * j + i;
              o[i + 3 * j] = elem((size_t)g * kMas16InvElems + (size_t)(dd * 9 + ei) * 16 + lane);
            }
        }
    return;
  }
  if (storage == MASPCG_INV_FP32) {
    for (int g = 0; g < D; ++g)
      for (int a = 0; a < kBank; ++a)
        for (int b = a; b < kBank; ++b) {
          // block (a,b) lives at lane a, diagonal b-a when that is <= 16, else it
          // is the transpose of (b,a) at lane b, diagonal 32-(b-a).
          const int d = b - a;
          const bool direct = d <= 16;
          const int lane = direct ? a : b, dd = direct ? d : 32 - d;
          float* o = out + ((size_t)g * kPacked + (kBank * a - a * (a + 1) / 2 + b)) * 9;
          for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
              const int ei = direct ? 3 * i + j : 3 * j + i;
              o[i + 3 * j] = elem((size_t)g * kInvElems + (size_t)(dd * 9 + ei) * kBank + lane);
            }
        }
    return;
  }
  // factored storage: rebuild W (lower, column-scaled) and form W^T W
  std::vector<double> W(96 * 96), M(96 * 96);
  for (int g = 0; g < D; ++g) {
    std::fill(W.begin(), W.end(), 0.0);
    const float* scg = sc.data() + (size_t)g * 96;
    for (int i = 0; i < 96; ++i)
      for (int j = 0; j <= i; ++j)
        W[i * 96 + j] = (double)elem((size_t)g * kInvElems16 + (size_t)inv16_pos(i, j)) * scg[j];
    for (int r = 0; r < 96; ++r)
      for (int q = r; q < 96; ++q) {
        double acc = 0;
        for (int k = std::max(r, q); k < 96; ++k) acc += W[k * 96 + r] * W[k * 96 + q];
        M[r * 96 + q] = M[q * 96 + r] = acc;
      }
    for (int a = 0; a < kBank; ++a)
      for (int b = a; b < kBank; ++b) {
        float* o = out + ((size_t)g * kPacked + (kBank * a - a * (a + 1) / 2 + b)) * 9;
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j) o[i + 3 * j] = (float)M[(3 * a + i) * 96 + 3 * b + j];
      }
  }
}

}  // namespace maspcg
