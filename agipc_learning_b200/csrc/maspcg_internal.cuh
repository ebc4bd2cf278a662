// maspcg_internal.cuh -- shared definitions of the B200 MAS-PCG library.
//
// Data layout (HBM):
//   * Internal block-row order: [rows before the FEM range][the part_map_size
//     MAS slots of the FEM range, in partition order, padding slots empty]
//     [rows after the FEM range].  A level-0 MAS domain is 32 consecutive
//     internal rows, so restriction and prolongation at level 0 are the
//     identity and a domain's residual is 96 contiguous floats.
//   * Matrix: full block-CSR (both triangles) over internal rows, 3x3 blocks
//     row-major; FP64 copy (reference precision, true residual) and FP32 copy
//     (inner iterations).
//   * Domain inverses: 17 "diagonals" x 9 elements x 32 lanes per domain;
//     element (i,j) of block (l, (l+d) mod 32) at [d][3i+j][l]; diagonal 16 is
//     stored for l < 16 only (zeros above).  16-bit storage is symmetrically
//     scaled: S^-1 A^-1 S^-1 with S = diag(sqrt(diag A^-1)), scales in FP32.
#pragma once

#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <stdint.h>

#include <atomic>
#include <cstring>
#include <utility>
#include <stdexcept>
#include <string>
#include <vector>

#include "maspcg.h"

namespace maspcg {

constexpr int kBank = 32;
constexpr int kPacked = kBank * (kBank + 1) / 2;  // 528
constexpr int kDiags = 17;
constexpr int kInvElems = kDiags * 9 * kBank;      // 4896 stored elements per domain (FP32)
// 16-bit storage holds the lower triangle of the scaled 96x96 factor as the
// 21 tiles (I >= J, tile T = I(I+1)/2 + J) of 16x16 elements that the
// tensor-core apply reads with ldmatrix: row r of a tile at 16 r elements,
// its two 8-element halves swapped when bit 2 of r is set, so the eight rows
// of one 8x8 ldmatrix operand fall in distinct shared-memory banks.  Upper
// elements of the diagonal tiles are zero.  A domain record is 10,752 bytes,
// copied to shared memory as one bulk copy.
constexpr int kTiles16 = 21;
constexpr int kInvElems16 = kTiles16 * 256;  // 5376 stored 16-bit elements per domain

// CEMAS16 (16-slot banks, 48x48 domains): FP32 inverses stored as 9 wrapped
// diagonals x 9 elements x 16 lanes, lane l holding block (l, (l + d) % 16).
constexpr int kMas16Packed = 16 * 17 / 2;                 // 136 packed upper blocks
constexpr int kMas16Diags = 9;
constexpr int kMas16InvElems = kMas16Diags * 9 * 16;      // 1296 per domain

// Stored elements per domain for an inverse element type.
template <typename TI>
constexpr int inv_elems() { return sizeof(TI) == 4 ? kInvElems : kInvElems16; }
inline int inv_elems_for(int storage) { return storage == MASPCG_INV_FP32 ? kInvElems : kInvElems16; }

// Position of element (i, j) of a 16-bit domain record: i >= j, or i < j
// inside a diagonal tile.
__host__ __device__ __forceinline__ int inv16_pos(int i, int j)
{
  const int I = i >> 4, J = j >> 4, r = i & 15, c = j & 15;
  return (I * (I + 1) / 2 + J) * 256 + r * 16 + ((((c >> 3) ^ (r >> 2)) & 1) << 3) + (c & 7);
}
constexpr int kMaxLevels = 6;
constexpr unsigned kFull = 0xffffffffu;

struct Error : std::runtime_error {
  maspcg_status status;
  Error(maspcg_status s, const std::string& m) : std::runtime_error(m), status(s) {}
};

#define MCK(expr)                                                                                  \
  do {                                                                                             \
    cudaError_t e_ = (expr);                                                                       \
    if (e_ != cudaSuccess) {                                                                       \
      throw ::maspcg::Error(e_ == cudaErrorMemoryAllocation ? MASPCG_ERR_OUT_OF_MEMORY : MASPCG_ERR_CUDA, \
                            std::string(#expr) + ": " + cudaGetErrorString(e_));                  \
    }                                                                                              \
  } while (0)

#define MREQ(cond, status, msg)                         \
  do {                                                  \
    if (!(cond)) throw ::maspcg::Error((status), (msg)); \
  } while (0)

// Counts device-buffer (re)allocations and releases in the process: a
// captured solve graph holds buffer addresses, so a graph captured at one
// count is reused only while the count is unchanged.
inline std::atomic<unsigned long long> g_buf_epoch{0};

// Grow-only device buffer.  A function-local temporary, which no solve graph
// can hold, is made uncounted (DBuf<T> b{false}).
template <typename T>
struct DBuf {
  T* p = nullptr;
  size_t cap = 0;
  size_t n = 0;
  bool counted = true;  // (re)allocations advance g_buf_epoch
  DBuf() = default;
  explicit DBuf(bool count) : counted(count) {}
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  ~DBuf() { release(); }
  void release()
  {
    if (p) {
      cudaFree(p);
      if (counted) ++g_buf_epoch;
    }
    p = nullptr;
    cap = n = 0;
  }
  // `pad` extra elements keep 16-byte vector loads of the tail in bounds.
  void resize(size_t count, size_t pad = 0)
  {
    const size_t need = count + pad;
    if (need > cap) {
      if (p) cudaFree(p);
      p = nullptr;
      cap = 0;
      if (counted) ++g_buf_epoch;
      if (need) {
        MCK(cudaMalloc(reinterpret_cast<void**>(&p), need * sizeof(T)));
        cap = need;
      }
    }
    n = count;
  }
  T* get() const { return p; }
  size_t bytes() const { return n * sizeof(T); }
};

// Device-resident PCG state; every iteration kernel reads it, only the last
// block of a reduction writes it.
struct PcgScalars {
  double rz, rz0, rz_new, pap, alpha, beta, rr, bb, rr_true;
  int k;          // current iteration (1-based, PCGSolver::pcg's k)
  int status;     // maspcg_solve_status, plus kNeedTrue
  int max_iter;   // PCGSolver: loop while k < max_iter
  int refinements;
  int iterations; // reported iteration count once stopped
  int gate;
  double tol;
  double rz_part[2];  // r.z of the level-0 apply (0) and of the coarse levels (1) when they run concurrently
  unsigned tickets[10];
  unsigned barrier_gen;  // generation of the grid barrier of the fused iteration kernel
  int rbuf;              // fused x / r update: which of the two r buffers holds the current residual
  long long barrier_limit;  // spins a grid-barrier wait may take before it gives up (maspcg_set_wait_test_hooks)
  int barrier_extra;        // arrivals a grid barrier expects beyond the grid (test hook: > 0 never completes)
  double rr_peak;           // MIXED: largest r.r since the last residual replacement (b.b at the start)
  int replace_mode;         // MIXED: maspcg_replacement
  int graph_launches;       // batches run by the device-side solve loop
  int max_launches;         // ... and the most it may run
};

constexpr int kNeedTrue = 16;  // MIXED: recursive gate met or period end; true residual pending
constexpr int kCapPending = 32;

enum Ticket { kTicketSpmv = 0, kTicketXr = 1, kTicketRz = 2, kTicketTrue = 3, kTicketAux = 4, kTicketPair = 5,
              kTicketCoarse = 6, kTicketBarrier = 7 };

struct LevelInfo {
  int levelnum;
  int count[kMaxLevels + 1];      // nodes per level (level 0: part_map_size slots)
  int begin[kMaxLevels + 1];      // first global cluster slot of the level
  int dom_begin[kMaxLevels + 1];  // first domain of the level
  int total_clusters;
  int domains;
};

// Pointers used by the domain factorisation kernel, one entry per level.
struct FactorArgs {
  LevelInfo lv;
  const int* cmap[kMaxLevels];   // fine slot -> level-L local node (-1 padding); level 0 unused
  const int* perm[kMaxLevels];   // level-L member lists (fine slots), level >= 1
  const int* off[kMaxLevels];    // level-L member offsets [count+1], level >= 1
  const int* pmr;                // part_map_real
  const int* rowptr;
  const int* colidx;
  const double* val64;           // row-major blocks
  int fem_off;
  int c0;
  void* inv;                     // inv_elems<TI>() per domain, type per storage
  float* scale;                  // 96 per domain (16-bit storage)
  int* failed;                   // count of domains with a pivot <= 0
  double* assembled;             // optional: packed FP64 domain matrices (reference layout)
  const double* coarse64;        // coarse-level domain matrices (32x32 blocks, row-major 3x3)
  double* dom64;                 // 16-bit storage: lower FP64 blocks per domain (kPacked x 9, row-major)
  int gather_only;               // write `assembled` and stop: the stored inverses are left as they are
};

}  // namespace maspcg

// ---------------------------------------------------------------- handle ---
struct maspcg_handle {
  maspcg_config cfg{};
  cudaStream_t stream = nullptr;
  cudaStream_t own_stream = nullptr;
  cudaStream_t side_stream = nullptr;       // the coarse levels run here beside the level-0 apply
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  int device = 0;
  int sm_count = 148;
  std::string last_error;

  // ---- graph (set_graph)
  int bank = 32;  // MAS bank: 32 (TraditionalMAS32) or 16 (CEMAS16)
  bool has_graph = false;
  int nv = 0, c0 = 0, levelnum = 0, node_offset = 0, nlist_size = 0;
  long long gn_cap = 0;
  maspcg::DBuf<uint32_t> nstart, nnum_init, nlist_init, nnum, nlist;
  maspcg::DBuf<int> pmr, rmp;
  std::vector<int> h_pmr, h_rmp;
  maspcg::DBuf<int> pairs;
  int n_pairs = 0;

  // ---- hierarchy (build)
  maspcg::DBuf<uint32_t> fine_mask, next_mask, next_prefix, next_prefix_sum;
  maspcg::DBuf<int> prefix_orig, prefix_sum_orig, cst, going_next, coarse_table, level_size;
  maspcg::LevelInfo lv{};
  maspcg::DBuf<int> cmap[maspcg::kMaxLevels], perm[maspcg::kMaxLevels], off[maspcg::kMaxLevels];
  maspcg::DBuf<int> sort_keys, sort_vals, sort_keys_out;
  maspcg::DBuf<unsigned char> cub_tmp;
  maspcg::DBuf<int> scan_tmp;

  // ---- matrix (set_matrix_bcoo)
  bool has_matrix = false;
  int nb = 0, fem_off = 0, abd_bodies = 0, nb_int = 0, n_in = 0, nnzb = 0;
  int m_valid = 0;  // sorted (key, block) pairs that carry a block (the merge of set_matrix_bcoo)
  bool mas_layout = false;  // internal order uses the MAS partition
  maspcg::DBuf<int> int_of_row, row_of_int;
  maspcg::DBuf<int> rowptr, colidx;
  maspcg::DBuf<double> val64;     // row-major 3x3 blocks
  maspcg::DBuf<float> val32;      // tiles of 32 blocks, element-major: (t/32)*288 + 32e + t%32
  maspcg::DBuf<unsigned short> val_lo;  // MASPCG_MATRIX_F32_SPLIT: BF16 of A - A32, laid out as val32
  maspcg::DBuf<unsigned long long> keys, keys_sorted;
  maspcg::DBuf<int> kv, kv_sorted, seg_head, seg_start, row_count;
  maspcg::DBuf<double> in_vals;
  maspcg::DBuf<int> in_rows, in_cols;

  // ---- preconditioner (build)
  bool has_precond = false;
  maspcg::DBuf<unsigned char> inv;  // domain inverses
  maspcg::DBuf<float> inv_scale;
  maspcg::DBuf<int> failed;
  int failed_domains = 0;
  maspcg::DBuf<float> coarse_r, coarse_z;
  maspcg::DBuf<int> chain_count, chain_target;  // coarse-level dataflow counters (per coarse domain)
  maspcg::DBuf<double> chain_dot;               // per coarse domain: R.Z (r.z of the coarse levels)
  maspcg::DBuf<double> coarse64;
  maspcg::DBuf<double> dom64;  // 16-bit storage: assembled lower blocks between the two factor passes
  maspcg::DBuf<double> abd_inv64;
  maspcg::DBuf<float> abd_inv32;
  maspcg::DBuf<double> diag_inv64;
  maspcg::DBuf<float> diag_inv32;

  // ---- PCG
  maspcg::DBuf<unsigned char> vx, vr, vz, vap;      // vectors in the working precision, 3 per block row
  maspcg::DBuf<unsigned char> vp4;                  // search direction, padded to 4 per block row
  maspcg::DBuf<double> b64, x64, r64;               // FP64: rhs, x (hi), residual scratch
  maspcg::DBuf<double> partial, partial_rz, partial_rr;
  maspcg::DBuf<unsigned char> vr2;  // second residual buffer of the fused x / r update (FP32 / MIXED)
  maspcg::DBuf<maspcg::PcgScalars> scal;
  maspcg::PcgScalars* h_scal = nullptr;  // pinned mirror
  int* h_err = nullptr;                  // pinned mirror of the solve's kernel error word
  maspcg::DBuf<double> io_a, io_b;       // staging for host pointers / permutations
  maspcg::DBuf<unsigned char> l2_flush;  // maspcg_time_stage only: written between timed launches
  maspcg::DBuf<int> adj_rows, adj_cols;   // maspcg_bcoo_gradient staging for host arguments
  maspcg::DBuf<double> adj_lam, adj_x, adj_grad;
  // maspcg_convert_bcoo / maspcg_partition_contact_triplets: sort keys and
  // permutation, head flags and scan, run starts, and host-argument staging
  maspcg::DBuf<unsigned long long> asm_keys, asm_types;
  maspcg::DBuf<int> asm_idx, asm_flags, asm_start, asm_rows, asm_cols, asm_rows_out, asm_cols_out;
  maspcg::DBuf<double> asm_vals, asm_vals_out;
  // maspcg_galerkin_*: expansion counts/offsets, expanded triplets, staging
  maspcg::DBuf<int> gal_counts, gal_rows, gal_cols, gal_in_rows, gal_in_cols, gal_f2c, gal_bases, gal_masks,
      gal_out_rows, gal_out_cols;
  maspcg::DBuf<double> gal_vals, gal_in_vals, gal_rest, gal_vec_in, gal_vec_out, gal_out_vals;
  // maspcg_fem_snk1_gradient_hessian host-argument staging
  maspcg::DBuf<unsigned> fem_tets;
  maspcg::DBuf<double> fem_x, fem_dminv, fem_vol, fem_len, fem_volr, fem_grad;
  cudaGraphExec_t graph_exec = nullptr;
  int graph_batch = 0;
  std::vector<unsigned long long> graph_sig;  // what graph_exec was captured against (graph_signature)
  long long graph_captures = 0;               // solve graphs captured and instantiated
  bool graph_dirty = true;
  bool graph_loop = false;        // graph_exec runs the whole solve loop (a conditional WHILE node)
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  int grid_stream = 0;  // CTAs for grid-stride kernels
  long long kernel_launches = 0;  // this library's kernels launched on the handle
  long long graph_kernels = 0;    // kernel nodes of the captured batch graph
  bool use_pdl = false;           // programmatic dependent launch for the iteration kernels (MASPCG_FLAG_PDL)
  bool fused_head = false;        // p update + SpMV + x/r update as one cooperative kernel (MASPCG_FLAG_FUSED_HEAD)
  bool vals_pending = false;      // set_matrix_bcoo: host values still copying on side_stream (ev_join)
  bool overlap_coarse = true;     // coarse levels beside the level-0 apply (off: MASPCG_FLAG_SEQUENTIAL_COARSE)
  int apply_variant = 2;          // 16-bit level-0 apply: 0 direct loads, 1 TMA-staged x2 buffers, 2 TMA-staged x1
  bool fuse_update = false;       // x / r update inside the apply kernels (MASPCG_FLAG_FUSED_UPDATE)
  long long barrier_limit = 1ll << 24;  // grid-barrier wait bound (spins of 64 ns sleeps)
  int barrier_extra = 0;                // test hook: extra arrivals a grid barrier waits for
};

namespace maspcg {

// hierarchy.cu
void build_hierarchy(maspcg_handle* h);

// matrix.cu
void build_internal_matrix(maspcg_handle* h, const double* vals_dev, const int* rows_dev, const int* cols_dev, int n);
// New values for the structure of the last build_internal_matrix (same
// triplets in the same order): the FP64 BCSR values and the FP32 layout.
void refresh_internal_values(maspcg_handle* h, const double* vals_dev);
void launch_spmv64(maspcg_handle* h, const double* x, double* y, double a, double b);  // internal order
void permute_in(maspcg_handle* h, const double* src_orig, double* dst_int);
void permute_out(maspcg_handle* h, const double* src_int, double* dst_orig);
void build_block_jacobi(maspcg_handle* h);

// mas.cu
void build_mas_domains(maspcg_handle* h, double* assembled_out);
// The packed FP64 domain matrices the stored inverses were built from: level
// 0 gathered again (a fixed order), the coarse levels from the build's own
// Galerkin sums; neither the sums nor the inverses are recomputed.
void gather_mas_domains(maspcg_handle* h, double* assembled_out);
void mas_apply_launch(maspcg_handle* h, const void* r, void* z, bool finalize_rz);
void decode_inverses(maspcg_handle* h, float* out_host);

// Count one launch of this library (graph captures are corrected afterwards).
#define MLAUNCHED(h) (++(h)->kernel_launches)

// pcg.cu
double time_stage(maspcg_handle* h, int stage, int repeats);
void solve(maspcg_handle* h, const double* b_dev, double* x_dev, maspcg_result* res);
void spmv_working(maspcg_handle* h, const double* x_int, double* y_int);  // internal order, FP64 in/out

// adjoint.cu (device pointers, caller's row order)
void bcoo_gradient(maspcg_handle* h, const int* rows, const int* cols, int n, const double* lam, const double* x,
                   double* grad);
void modulus_gradient(maspcg_handle* h, const int* rows, const int* cols, const double* vals, int ntet, int bpt,
                      const double* lam, const double* x, const double* E, double* gE);

// assemble.cu (device pointers; returns the unique count / the type counts)
int convert_bcoo(maspcg_handle* h, const int* rows, const int* cols, const double* vals, int n, int* rows_out,
                 int* cols_out, double* vals_out);
void partition_contacts(maspcg_handle* h, const int* rows, const int* cols, const double* vals,
                        const unsigned long long* types, int n, int* rows_out, int* cols_out, double* vals_out,
                        int counts[4]);

// contact.cu (device pointers, in place).  zero_boundary_only: clear the
// triplets touching a boundary vertex (indices minus `offset`); else the
// contact adjustment (lower copies moved up and cleared, boundary pairs
// cleared, indices plus `offset`).  Returns false when an index fell outside
// [0, n_vertices) (that triplet is left as it was).
bool adjust_contacts(maspcg_handle* h, int n, int* rows, int* cols, double* values9, const int* bd_type,
                     int n_vertices, int offset, bool zero_boundary_only);
// Sub-range triplets (device pointers): out[t] = source[idx ? idx[t] : t]
// with indices - offset; an index >= source gives rows_out -1.
void gather_triplets(maspcg_handle* h, int n, const unsigned* idx, const int* rows, const int* cols,
                     const double* vals9, long long source, int offset, int* rows_out, int* cols_out,
                     double* vals_out);

// galerkin.cu (device pointers).  The AGIPC mapping: fine blocks [0, prefix)
// pass through; FEM node k (block prefix + k) maps to coarse node
// fine_to_coarse[k], whose blocks start at prefix + coarse_block_bases[c]
// with the basis subset basis_masks[c] of (1, x, y, z) at rest[3k..3k+2].
struct GalerkinMap {
  const int* fine_to_coarse;
  const int* coarse_block_bases;
  const int* basis_masks;
  const double* rest;
  int prefix;
  int fine_blocks;
};
int galerkin_expand(maspcg_handle* h, const GalerkinMap& m, const double* vals, const int* rows, const int* cols,
                    int n, const double** v, const int** r, const int** c);
void galerkin_restrict(maspcg_handle* h, const GalerkinMap& m, const double* fine, double* coarse, int coarse_blocks);
void galerkin_prolong(maspcg_handle* h, const GalerkinMap& m, const double* coarse, double* fine);

// fem.cu (device pointers)
void fem_snk1(maspcg_handle* h, int ntet, int nverts, const unsigned* tets, const double* x, const double* dm_inv,
              const double* volume, const double* len_rate, const double* vol_rate, double dt, int offset,
              double* gradient, int* rows, int* cols, double* vals);

// diagnostics.cu (device pointers): 7 doubles per domain into results
void check_local_matrices(maspcg_handle* h, int count, int bank, const double* packed64_dev,
                          const float* inverse32_dev, double* results_dev);

// residual_noalloc.cu
void residual_norms_noalloc(maspcg_handle* h, int count, const double* x, const double* b, double* residual_norms,
                            double* rhs_norms);
void apply_preconditioner64(maspcg_handle* h, const double* r_int, double* z_int);
size_t vec_elem_size(const maspcg_handle* h);

// common device helpers
template <typename T>
__device__ __forceinline__ T warp_sum(T v)
{
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}

template <typename T, int NT>
__device__ __forceinline__ T block_sum(T v, T* smem /* NT/32 */)
{
  v = warp_sum(v);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) smem[w] = v;
  __syncthreads();
  T s = 0;
  if (w == 0) {
    s = (l < NT / 32) ? smem[l] : T(0);
    s = warp_sum(s);
  }
  __syncthreads();
  return s;  // valid in warp 0
}

inline int ceil_div(long long a, long long b) { return (int)((a + b - 1) / b); }

// Programmatic dependent launch.  An iteration kernel waits at entry for its
// predecessor's completion (and memory) before touching anything it
// produced, and lets its successor be scheduled once its own main loop is
// done, so the successor's launch overlaps this kernel's tail (the last-block
// reduction) without its CTAs taking SM resources from the main loop.
// Without the launch attribute both instructions are no-ops.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

template <typename... KArgs, typename... Args>
void launch_pdl_on(maspcg_handle* h, cudaStream_t stream, void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem,
                   Args&&... args)
{
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = h->use_pdl ? 1 : 0;
  MCK(cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...));
  ++h->kernel_launches;
}

// Cooperative launch (all CTAs resident at once) for kernels with a grid
// barrier; the caller sizes the grid from the occupancy API.
template <typename... KArgs, typename... Args>
void launch_cooperative(maspcg_handle* h, void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, Args&&... args)
{
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = h->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  MCK(cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...));
  ++h->kernel_launches;
}

template <typename... KArgs, typename... Args>
void launch_pdl(maspcg_handle* h, void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, Args&&... args)
{
  launch_pdl_on(h, h->stream, kernel, grid, block, smem, std::forward<Args>(args)...);
}

}  // namespace maspcg
