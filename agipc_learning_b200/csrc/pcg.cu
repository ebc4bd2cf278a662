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

#include "maspcg_internal.cuh"
#include "pcg_device.cuh"
#include "spmv_row.cuh"
#include "spmv_tma.cuh"

namespace maspcg {

template <typename Tv, typename Tacc>
void mas_apply(maspcg_handle* h, const Tv* r, Tv* z, Tacc* partial, int part_base, int total_parts, int mode,
               int grid0, PcgScalars* s);
template <typename Tv, typename Tacc>
void mas_level0_only(maspcg_handle* h, const Tv* r, Tv* z, Tacc* partial, int grid0, PcgScalars* s);
void launch_factor(maspcg_handle* h, double* assembled_out);
int mas_level0_grid(maspcg_handle* h);

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
      threadIdx.x == 0)
    s->bb = total;
}

// p = z (k == 1) or z + beta p
template <typename Tv>
__global__ void __launch_bounds__(kTpb) k_update_p(const Tv* __restrict__ z, Tv* p, int n, const PcgScalars* s)
{
  pdl_enter();
  if (!running(s)) return;
  const bool first = s->k == 1;
  const Tv beta = (Tv)s->beta;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    p[i] = first ? z[i] : z[i] + beta * p[i];
}

// Ap = A p (LPR lanes per block row) and p.Ap; last block: alpha.
template <typename Tm, typename Tv, typename Tacc, int LPR>
__global__ void __launch_bounds__(kTpb) k_spmv_dot(const int* __restrict__ rowptr, const int* __restrict__ colidx,
                                                    const Tm* __restrict__ val, const Tv* __restrict__ p, Tv* ap,
                                                    int nrows, Tacc* partial, PcgScalars* s)
{
  if (!running(s)) return;
  const int groups_per_block = kTpb / LPR;
  const int sub = threadIdx.x % LPR;
  Tacc dot = 0;
  const int iters = (nrows + gridDim.x * groups_per_block - 1) / (gridDim.x * groups_per_block);
  for (int it = 0; it < iters; ++it) {
    const int row = (it * gridDim.x + blockIdx.x) * groups_per_block + threadIdx.x / LPR;
    const bool ok = row < nrows;
    const int rs = ok ? rowptr[row] : 0, re = ok ? rowptr[row + 1] : 0;
    typename AccOf<Tm>::type acc[3];
    row_product<Tm, Tv, LPR>(rs, re, colidx, val, p, sub, acc);
    if (ok && sub < 3) {
      const Tv y = (Tv)acc[sub];
      ap[3 * (size_t)row + sub] = y;
      dot += (Tacc)p[3 * (size_t)row + sub] * (Tacc)y;
    }
  }
  Tacc total = 0;
  if (grid_finish<Tacc>(dot, partial, blockIdx.x, gridDim.x, &s->tickets[kTicketSpmv], gridDim.x, total) &&
      threadIdx.x == 0) {
    const double pap = (double)total;
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
}

// Ap = A p with the block stream staged by TMA (spmv_tma.cuh) and p.Ap;
// last block: alpha.  `err` records an expired mbarrier wait.
template <typename Tm, typename Tv, typename Tacc>
__global__ void __launch_bounds__(kTmaThreads, 2)
    k_spmv_tma(const int* __restrict__ rowptr, const int* __restrict__ colidx, const Tm* __restrict__ val,
               const Tv* __restrict__ p, Tv* ap, int nrows, Tacc* partial, PcgScalars* s, int* err)
{
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ __align__(8) uint64_t bar[2];
  pdl_enter();
  if (!running(s)) return;
  using St = TmaStage<Tm>;
  unsigned char* sval0 = smem;
  unsigned char* sval1 = smem + St::kValBytes;
  unsigned char* scol0 = smem + 2 * St::kValBytes;
  unsigned char* scol1 = smem + 2 * St::kValBytes + St::kColBytes;
  const int nchunks = (nrows + kTmaRows - 1) / kTmaRows;
  const int tid = threadIdx.x, grp = tid >> 4, sub = tid & 15;
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  auto staged = [&](int chunk) {
    const int r0 = chunk * kTmaRows, r1 = min(r0 + kTmaRows, nrows);
    const int nb = rowptr[r1] - rowptr[r0];
    return nb > 0 && nb <= St::kCap;
  };
  if (tid == 0) {
    const int c0 = blockIdx.x, c1 = blockIdx.x + gridDim.x;
    if (c0 < nchunks) chunk_issue<Tm>(c0, nrows, rowptr, val, colidx, sval0, scol0, &bar[0]);
    if (c1 < nchunks) chunk_issue<Tm>(c1, nrows, rowptr, val, colidx, sval1, scol1, &bar[1]);
  }
  unsigned phase0 = 0, phase1 = 0;
  Tacc dot = 0;
  int i = 0;
  bool ok = true;
  for (int chunk = blockIdx.x; chunk < nchunks; chunk += gridDim.x, ++i) {
    const int st = i & 1;
    const int r0 = chunk * kTmaRows, r1 = min(r0 + kTmaRows, nrows);
    const int b0 = rowptr[r0];
    const bool stg = staged(chunk);
    if (stg) {
      const bool w = mbar_wait(st ? &bar[1] : &bar[0], st ? phase1 : phase0);
      if (w) {
        if (st)
          phase1 ^= 1u;
        else
          phase0 ^= 1u;
      }
      if (!__syncthreads_and(w)) {
        ok = false;
        break;
      }
    }
    const int row = r0 + grp;
    const bool has = row < r1;
    const int rs = has ? rowptr[row] : 0, re = has ? rowptr[row + 1] : 0;
    typename AccOf<Tm>::type acc[3];
    if (stg) {
      using A = typename AccOf<Tm>::type;
      const unsigned char* sv = st ? sval1 : sval0;
      const unsigned char* sc = st ? scol1 : scol0;
      const Tm* vb = reinterpret_cast<const Tm*>(sv + (((size_t)b0 * 9 * sizeof(Tm)) & 15));
      const int* cb = reinterpret_cast<const int*>(sc + (((size_t)b0 * 4) & 15));
      A a0 = 0, a1 = 0, a2 = 0;
      for (int t = rs + sub; t < re; t += 16) {
        const int lt = t - b0;
        const int c = cb[lt];
        const Tm* B = vb + 9 * lt;
        const A x0 = (A)ldv(p + 3 * (size_t)c), x1 = (A)ldv(p + 3 * (size_t)c + 1), x2 = (A)ldv(p + 3 * (size_t)c + 2);
        a0 += (A)B[0] * x0 + (A)B[1] * x1 + (A)B[2] * x2;
        a1 += (A)B[3] * x0 + (A)B[4] * x1 + (A)B[5] * x2;
        a2 += (A)B[6] * x0 + (A)B[7] * x1 + (A)B[8] * x2;
      }
#pragma unroll
      for (int o = 8; o > 0; o >>= 1) {
        a0 += __shfl_xor_sync(kFull, a0, o, 16);
        a1 += __shfl_xor_sync(kFull, a1, o, 16);
        a2 += __shfl_xor_sync(kFull, a2, o, 16);
      }
      acc[0] = a0;
      acc[1] = a1;
      acc[2] = a2;
    } else {
      row_product<Tm, Tv, 16>(rs, re, colidx, val, p, sub, acc);
    }
    if (has && sub < 3) {
      const Tv y = (Tv)acc[sub];
      ap[3 * (size_t)row + sub] = y;
      dot += (Tacc)p[3 * (size_t)row + sub] * (Tacc)y;
    }
    __syncthreads();  // the stage is free again
    if (tid == 0) {
      const int nxt = chunk + 2 * gridDim.x;
      if (nxt < nchunks) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        chunk_issue<Tm>(nxt, nrows, rowptr, val, colidx, st ? sval1 : sval0, st ? scol1 : scol0,
                        st ? &bar[1] : &bar[0]);
      }
    }
  }
  if (!ok) {
    // drain the copies this CTA still has in flight (bounded), report, leave
    if (tid == 0) {
      atomicExch(err, 1);
      for (int j = 0; j < 2; ++j) {
        const int chunk = blockIdx.x + (i + j) * gridDim.x;
        if (chunk < nchunks && staged(chunk)) {
          const int stj = (i + j) & 1;
          mbar_wait(stj ? &bar[1] : &bar[0], stj ? phase1 : phase0);
        }
      }
      s->status = MASPCG_SOLVE_NONFINITE;
    }
    return;
  }
  Tacc total = 0;
  if (grid_finish<Tacc, kTmaThreads>(dot, partial, blockIdx.x, gridDim.x, &s->tickets[kTicketSpmv], gridDim.x, total) &&
      threadIdx.x == 0) {
    const double pap = (double)total;
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
}

// x += alpha p, r -= alpha Ap, r.r; last block: stopping gate.
// MIXED: x is the FP32 correction since the last replacement and a met gate
// asks for the FP64 true residual instead of stopping.
template <typename Tv, typename Tacc>
__global__ void __launch_bounds__(kTpb) k_update_xr(Tv* x, Tv* r, const Tv* __restrict__ p, const Tv* __restrict__ ap,
                                                     int n, int mixed, Tacc* partial, PcgScalars* s)
{
  pdl_enter();
  if (!running(s)) return;
  const Tv alpha = (Tv)s->alpha;
  Tacc acc = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    x[i] += alpha * p[i];
    const Tv ri = r[i] - alpha * ap[i];
    r[i] = ri;
    acc += (Tacc)ri * (Tacc)ri;
  }
  Tacc total = 0;
  if (grid_finish<Tacc>(acc, partial, blockIdx.x, gridDim.x, &s->tickets[kTicketXr], gridDim.x, total) &&
      threadIdx.x == 0) {
    const double rr = (double)total;
    s->rr = rr;
    if (!isfinite(rr)) {
      s->status = MASPCG_SOLVE_NONFINITE;
      s->iterations = s->k;
      return;
    }
    const bool conv = (s->gate == MASPCG_GATE_RZ) ? (fabs(s->rz) <= s->tol * s->rz0) : (rr <= s->tol * s->tol * s->bb);
    if (conv) {
      if (mixed) {
        s->status = kNeedTrue;
      } else {
        s->status = MASPCG_SOLVE_CONVERGED;
        s->iterations = s->k;
      }
    }
  }
}

// MIXED: fold the FP32 correction into the FP64 iterate.
__global__ void __launch_bounds__(kTpb) k_fold_x(double* xhi, float* xlo, int n, int force, const PcgScalars* s)
{
  pdl_enter();
  if (!force && !(s->status == MASPCG_SOLVE_RUNNING || s->status == kNeedTrue)) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    xhi[i] += (double)xlo[i];
    xlo[i] = 0.f;
  }
}

// MIXED: r = b - A x_hi in FP64 with the FP64 matrix; FP32 copy for the
// iteration; last block: stop on the true residual or resume.
template <int LPR>
__global__ void __launch_bounds__(kTpb) k_true_residual(const int* __restrict__ rowptr, const int* __restrict__ colidx,
                                                         const double* __restrict__ val, const double* __restrict__ xhi,
                                                         const double* __restrict__ b, float* r32, int nrows,
                                                         double* partial, PcgScalars* s)
{
  pdl_enter();
  if (!(s->status == MASPCG_SOLVE_RUNNING || s->status == kNeedTrue)) return;
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
  double total = 0.0;
  if (grid_finish<double>(acc2, partial, blockIdx.x, gridDim.x, &s->tickets[kTicketTrue], gridDim.x, total) &&
      threadIdx.x == 0) {
    s->rr_true = total;
    s->rr = total;
    s->refinements += 1;
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
  pdl_enter();
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

// ----------------------------------------------------------------- engine --

template <typename Tm, typename Tv, typename Tacc>
struct Engine {
  maspcg_handle* h;
  int n, gstream, gspmv, gl0, gother, parts_other, parts_total;
  bool mas, mixed;

  explicit Engine(maspcg_handle* hh) : h(hh)
  {
    n = 3 * h->nb_int;
    mas = h->mas_layout && h->cfg.preconditioner == MASPCG_PRECOND_MAS32;
    mixed = h->cfg.precision == MASPCG_PREC_MIXED;
    gstream = h->grid_stream;
    gspmv = std::max(1, std::min(ceil_div(h->nb_int, kTpb / 16), 4 * h->sm_count));
    gl0 = mas ? mas_level0_grid(h) : 0;
    const bool other = !mas || h->abd_bodies > 0 || h->fem_off > 0 || h->nb_int > h->fem_off + h->c0;
    gother = other ? std::max(1, std::min(ceil_div(std::max(h->nb_int, 1), kTpb), 2 * h->sm_count)) : 0;
    parts_other = gother;
    parts_total = gother + gl0;
  }
  Tv* V(maspcg::DBuf<unsigned char>& b) { return reinterpret_cast<Tv*>(b.get()); }
  Tacc* partial() { return reinterpret_cast<Tacc*>(h->partial.get()); }
  Tacc* partial_rz() { return reinterpret_cast<Tacc*>(h->partial_rz.get()); }

  void precondition(const Tv* r, Tv* z, int mode, PcgScalars* s)
  {
    const bool ref = h->cfg.precision == MASPCG_PREC_REFERENCE;
    if (gother) {
      const bool bj = h->cfg.preconditioner == MASPCG_PRECOND_BLOCK_JACOBI;
      const int mas_lo = mas ? h->fem_off : 0, mas_hi = mas ? h->fem_off + h->c0 : 0;
      const int bodies = (h->cfg.preconditioner == MASPCG_PRECOND_NONE) ? 0 : h->abd_bodies;
      if (ref)
        launch_pdl(h, k_other_apply<Tv, Tacc, double>, dim3(gother), dim3(kTpb), 0, 
            r, z, h->nb_int, mas_lo, mas_hi, bodies, h->abd_inv64.get(), bj ? h->diag_inv64.get() : nullptr,
            s ? partial_rz() : nullptr, 0, parts_total, mas ? 0 : 1, mode, s);
      else
        launch_pdl(h, k_other_apply<Tv, Tacc, float>, dim3(gother), dim3(kTpb), 0, 
            r, z, h->nb_int, mas_lo, mas_hi, bodies, h->abd_inv32.get(), bj ? h->diag_inv32.get() : nullptr,
            s ? partial_rz() : nullptr, 0, parts_total, mas ? 0 : 1, mode, s);
      MLAUNCHED(h);
    }
    if (mas) mas_apply<Tv, Tacc>(h, r, z, s ? partial_rz() : nullptr, parts_other, parts_total, mode, gl0, s);
    MCK(cudaGetLastError());
  }

  void iteration_head(PcgScalars* s)
  {
    launch_pdl(h, k_update_p<Tv>, dim3(gstream), dim3(kTpb), 0, V(h->vz), V(h->vp), n, s);
    spmv_tma(s);
    launch_pdl(h, k_update_xr<Tv, Tacc>, dim3(gstream), dim3(kTpb), 0, V(h->vx), V(h->vr), V(h->vp), V(h->vap), n, mixed ? 1 : 0,
                                                   partial(), s);
  }

  const Tm* matrix();

  void spmv_tma(PcgScalars* s)
  {
    using St = TmaStage<Tm>;
    constexpr int bytes = 2 * (St::kValBytes + St::kColBytes);
    static bool configured = false;
    if (!configured) {
      MCK(cudaFuncSetAttribute(k_spmv_tma<Tm, Tv, Tacc>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
      configured = true;
    }
    const int grid = std::max(1, std::min(2 * h->sm_count, ceil_div(h->nb_int, kTmaRows)));
    launch_pdl(h, k_spmv_tma<Tm, Tv, Tacc>, dim3(grid), dim3(kTmaThreads), bytes, h->rowptr.get(), h->colidx.get(), matrix(),
                                                                      V(h->vp), V(h->vap), h->nb_int, partial(), s,
                                                                      h->failed.get() + 4);
    MLAUNCHED(h);
  }

  void true_residual(PcgScalars* s)
  {
    launch_pdl(h, k_fold_x, dim3(gstream), dim3(kTpb), 0, h->x64.get(), reinterpret_cast<float*>(h->vx.get()), n, 0, s);
    launch_pdl(h, k_true_residual<16>, dim3(gspmv), dim3(kTpb), 0, h->rowptr.get(), h->colidx.get(), h->val64.get(), h->x64.get(),
                                               h->b64.get(), reinterpret_cast<float*>(h->vr.get()), h->nb_int,
                                               h->partial.get(), s);
  }

  // One graph = `batch` iterations.
  void record_batch(int batch, PcgScalars* s)
  {
    for (int it = 0; it < batch; ++it) {
      iteration_head(s);
      if (mixed && it == batch - 1) true_residual(s);
      precondition(V(h->vr), V(h->vz), 2, s);
    }
  }

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
    MCK(cudaMemcpyAsync(s, &init, sizeof(init), cudaMemcpyHostToDevice, st));
    MREQ(stage != 3 || mas, MASPCG_ERR_NOT_READY, "stage 3 needs a MAS32 preconditioner");
    MREQ(stage != 2 || mas, MASPCG_ERR_NOT_READY, "stage 2 needs a MAS32 preconditioner");
    auto once = [&]() {
      switch (stage) {
        case 0: spmv_tma(s); break;
        case 4:
          k_spmv_dot<Tm, Tv, Tacc, 16><<<gspmv, kTpb, 0, st>>>(h->rowptr.get(), h->colidx.get(), matrix(), V(h->vp),
                                                              V(h->vap), h->nb_int, partial(), s);
          MLAUNCHED(h);
          break;
        case 1: precondition(V(h->vr), V(h->vz), 0, s); break;
        case 2: mas_level0_only<Tv, Tacc>(h, V(h->vr), V(h->vz), partial_rz(), gl0, s); break;
        case 3: launch_factor(h, nullptr); break;
        default: throw Error(MASPCG_ERR_INVALID_ARGUMENT, "unknown stage");
      }
    };
    once();  // warm
    MCK(cudaEventRecord(h->ev0, st));
    for (int i = 0; i < repeats; ++i) once();
    MCK(cudaEventRecord(h->ev1, st));
    MCK(cudaMemcpyAsync(h->h_scal, s, sizeof(PcgScalars), cudaMemcpyDeviceToHost, st));
    MCK(cudaStreamSynchronize(st));
    MCK(cudaGetLastError());
    MREQ(h->h_scal->status == MASPCG_SOLVE_RUNNING, MASPCG_ERR_NOT_READY,
         "stage timing needs finite vectors: solve once first");
    float ms = 0.f;
    MCK(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
    return (double)ms / std::max(1, repeats);
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
    init.gate = mixed ? MASPCG_GATE_EUCLID : h->cfg.gate;
    init.tol = h->cfg.tolerance;
    MCK(cudaMemcpyAsync(s, &init, sizeof(init), cudaMemcpyHostToDevice, st));
    MCK(cudaMemsetAsync(h->failed.get() + 4, 0, sizeof(int), st));
    MCK(cudaEventRecord(h->ev0, st));
    k_init<Tv><<<gstream, kTpb, 0, st>>>(b_int, V(h->vx), V(h->vr), mixed ? h->x64.get() : nullptr, n,
                                         h->partial_rz.get(), s); MLAUNCHED(h);
    precondition(V(h->vr), V(h->vz), 1, s);
    // graph of one batch
    const int batch = mixed ? std::max(1, h->cfg.refinement_period) : std::max(1, h->cfg.iterations_per_launch);
    if (h->graph_dirty || h->graph_batch != batch) {
      if (h->graph_exec) cudaGraphExecDestroy(h->graph_exec);
      h->graph_exec = nullptr;
      cudaGraph_t g = nullptr;
      const long long launches_before = h->kernel_launches;
      MCK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
      try {
        record_batch(batch, s);
      } catch (...) {
        cudaStreamEndCapture(st, &g);
        if (g) cudaGraphDestroy(g);
        h->kernel_launches = launches_before;
        throw;
      }
      MCK(cudaStreamEndCapture(st, &g));
      h->graph_kernels = h->kernel_launches - launches_before;
      h->kernel_launches = launches_before;
      MCK(cudaGraphInstantiate(&h->graph_exec, g, 0));
      cudaGraphDestroy(g);
      h->graph_batch = batch;
      h->graph_dirty = false;
    }
    int launches = 0;
    // The first status read also covers the initial apply.
    MCK(cudaMemcpyAsync(h->h_scal, s, sizeof(PcgScalars), cudaMemcpyDeviceToHost, st));
    MCK(cudaStreamSynchronize(st));
    const int max_launches = max_iter / batch + 4;
    while (h->h_scal->status == MASPCG_SOLVE_RUNNING && launches < max_launches) {
      MCK(cudaGraphLaunch(h->graph_exec, st));
      h->kernel_launches += h->graph_kernels;
      ++launches;
      MCK(cudaMemcpyAsync(h->h_scal, s, sizeof(PcgScalars), cudaMemcpyDeviceToHost, st));
      MCK(cudaStreamSynchronize(st));
    }
    {
      int terr = 0;
      MCK(cudaMemcpy(&terr, h->failed.get() + 4, sizeof(int), cudaMemcpyDeviceToHost));
      MREQ(terr == 0, MASPCG_ERR_CUDA, "a TMA mbarrier wait expired in the SpMV");
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
    MCK(cudaStreamSynchronize(st));
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
