/*
 * maspcg.h -- C ABI of the B200 MAS-preconditioned PCG for StiffGIPC's
 * Newton-step linear solve.
 *
 * One handle owns one linear system on one GPU: the neighbour graph and
 * partition of the FEM vertices (MAS hierarchy input), the contact pairs of
 * the current Newton step, the assembled block-sparse Hessian, the
 * preconditioner built from it, and the PCG work space.  All entry points
 * return a maspcg_status; none aborts or exits.  A handle is thread-compatible
 * (one host thread at a time), not thread-safe.  All device work is issued on
 * the handle's stream.
 *
 * Pointers: every array argument may be a host pointer or a device pointer
 * (detected with cudaPointerGetAttributes); host arrays are copied in/out
 * inside the call.
 *
 * Layouts restated from the reference (KLBSTL/AGIPC_LEARNING):
 *   - 3x3 block: 9 doubles, Eigen::Matrix3d column-major, element (r,c) at
 *     r + 3c (StiffGIPC/linear_system/linear_system/global_matrix.h:18-25);
 *   - matrix: upper BCOO, row <= col, block (r,c) holds A_rc and implies
 *     A_cr = A_rc^T (StiffGIPC/linear_system/utils/spmv.cu:28-53);
 *   - vectors: double, 3 per block row (double3 in the reference);
 *   - contact pairs: int4 with IPC's sign encoding
 *     (StiffGIPC/TraditionalMAS32Preconditioner.cu:1550-1962).
 */
#ifndef MASPCG_H
#define MASPCG_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define MASPCG_API __attribute__((visibility("default")))
#else
#define MASPCG_API
#endif

typedef struct maspcg_handle maspcg_handle;

typedef enum {
  MASPCG_OK = 0,
  MASPCG_ERR_INVALID_ARGUMENT = 1,
  MASPCG_ERR_NULL_HANDLE = 2,
  MASPCG_ERR_CUDA = 3,
  MASPCG_ERR_OUT_OF_MEMORY = 4,
  MASPCG_ERR_NOT_READY = 5, /* call order: graph -> matrix -> build -> solve */
  MASPCG_ERR_CAPACITY = 6,  /* hierarchy / size overflow (gipc::hierarchy_capacity) */
  MASPCG_ERR_NO_DEVICE = 7,
  MASPCG_ERR_UNSUPPORTED = 8
} maspcg_status;

/* Preconditioner ids follow the reference's P_type (gl_main.cu:1248-1250). */
typedef enum {
  MASPCG_PRECOND_BLOCK_JACOBI = 0, /* DiagPreconditioner: 3x3 block inverse */
  MASPCG_PRECOND_MAS16 = 1,        /* MASPreconditioner (CEMAS16, 16-vertex banks) on the FEM range + ABD 12x12 */
  MASPCG_PRECOND_MAS32 = 2,        /* TraditionalMAS32 on the FEM range + ABD 12x12 */
  MASPCG_PRECOND_NONE = 3
} maspcg_preconditioner;

typedef enum {
  /* FP64 matrix, vectors and dots; FP32 MAS apply: the reference's arithmetic */
  MASPCG_PREC_REFERENCE = 0,
  /* everything FP32 (matrix, vectors, dots, FP32 domain inverses) */
  MASPCG_PREC_FP32 = 1,
  /* FP32 matrix and vectors, 16-bit domain inverses with FP32 accumulation,
   * FP64 dots, the FP32 x folded into an FP64 x every refinement_period
   * iterations and the recursive residual replaced by the FP64 true residual
   * as residual_replacement says; stops on the FP64 true residual */
  MASPCG_PREC_MIXED = 2
} maspcg_precision;

typedef enum {
  MASPCG_GATE_RZ = 0,    /* PCGSolver::pcg: |r^T z| <= tol * r0^T z0, tested after the update */
  MASPCG_GATE_EUCLID = 1 /* ||r|| <= tol * ||b|| */
} maspcg_gate;

typedef enum { MASPCG_INV_FP32 = 0, MASPCG_INV_BF16 = 1, MASPCG_INV_FP16 = 2 } maspcg_inverse_storage;

typedef struct {
  double tolerance;      /* PCGSolverConfig::global_tol_rate (1e-4) */
  double max_iter_ratio; /* PCGSolverConfig::max_iter_ratio (0.3): max_iter = ratio * dof */
  int max_iterations;    /* > 0 overrides max_iter_ratio */
  int gate;              /* maspcg_gate */
  int precision;         /* maspcg_precision */
  int inverse_storage;   /* maspcg_inverse_storage (FP32 unless MIXED; always FP32 for CEMAS16) */
  int preconditioner;    /* maspcg_preconditioner */
  int refinement_period; /* MIXED: iterations between checks for an FP64 true residual (default 16) */
  int bank_size;         /* MAS bank: 32 (GPU_MAS_BANKSIZE) for MAS32, 16 (BANKSIZE) for CEMAS16 */
  int iterations_per_launch; /* PCG iterations per CUDA-graph launch (default 8) */
  int flags;             /* maspcg_flags: kernel-schedule choices, 0 = defaults */
  int matrix_form;       /* maspcg_matrix_form: the iteration matrix of FP32 / MIXED precision */
  int residual_replacement; /* maspcg_replacement: when MIXED replaces the recursive residual */
} maspcg_config;

/* When MIXED precision replaces the recursive residual r by the FP64 true
 * residual b - A x (checked at the end of every graph of refinement_period
 * iterations; always when the recursive gate is met, where the true residual
 * decides the stop).  x_hi += x_lo is folded at every check either way. */
typedef enum {
  MASPCG_REPLACE_PERIODIC = 0, /* at every check (the default: the fewest iterations on every system measured) */
  MASPCG_REPLACE_RELIABLE = 1  /* once ||r|| has fallen to 0.1 of its largest value since the last replacement: a
                                  few FP64 residuals per decade of reduction instead of one per period, but with
                                  FP32 sums the recursive residual can drift between them (more iterations on
                                  contact-dense systems) */
} maspcg_replacement;

/* How FP32 and MIXED precision store the iteration's matrix and sum its
 * products (maspcg_config.matrix_form).  The reference precision always runs
 * the FP64 matrix with FP64 sums, and the affine-body rows always take the
 * FP64 matrix.  MASPCG_MATRIX_F32_ACCURATE forms each FP32 x FP32 product
 * exactly (its rounding error from one FMA) and sums them compensated in
 * pairs of FP32 numbers (Ogita, Rump and Oishi's Dot2), so the FP32-valued
 * operator A32 p is computed to about 2^-48 of the sum of the terms'
 * magnitudes before the single rounding of the result: on stiff contact rows
 * (barrier blocks beside a soft mass term) FP32 sums lose more than the FP32
 * values themselves do. */
typedef enum {
  MASPCG_MATRIX_F32 = 0,       /* FP32 values, products and sums (the default: the fewest instructions) */
  MASPCG_MATRIX_F32_ACCURATE = 1, /* FP32 values; exact products, compensated sums */
  MASPCG_MATRIX_F32_SPLIT = 2, /* FP32 values plus BF16 values of the remainder A - A32, so the operator is A to
                                  about 2^-32 relative: for systems whose stiffness spread FP32 values cannot
                                  carry (18 more bytes per block); sums as MASPCG_MATRIX_F32_ACCURATE */
  MASPCG_MATRIX_F32_COMPENSATED = 3 /* FP32 values; each block row's three products by FMA in FP32, the blocks of a
                                       row summed compensated (TwoSum): cheaper than ACCURATE, enough for contact-
                                       dense systems with periodic replacement */
} maspcg_matrix_form;

/* Kernel-schedule choices (bits of maspcg_config.flags); results do not depend
 * on them beyond floating-point summation order. */
typedef enum {
  MASPCG_FLAG_PDL = 1,                 /* launch iteration kernels with programmatic dependent launch */
  MASPCG_FLAG_APPLY_STAGED2 = 2,       /* 16-bit level-0 apply: two TMA slots per warp */
  MASPCG_FLAG_APPLY_DIRECT = 4,        /* 16-bit level-0 apply: records staged by per-lane loads, no TMA */
  MASPCG_FLAG_SEQUENTIAL_COARSE = 8,   /* run the MAS coarse levels before the level-0 apply, not beside it
                                          (always so in MASPCG_PREC_REFERENCE, whose r.z is then summed over
                                          the fine rows as the reference sums it) */
  MASPCG_FLAG_FUSED_HEAD = 16,         /* p update, SpMV and x/r update as one cooperative kernel with grid barriers */
  MASPCG_FLAG_FUSED_UPDATE = 32,       /* FP32 / MIXED with MAS32: the x / r update run by the preconditioner's apply
                                          kernels on their own rows instead of a kernel of its own (measured slower:
                                          the latency-bound apply kernels take longer than the update they absorb) */
  MASPCG_FLAG_HOST_LOOP = 64           /* the solve loop as a graph of one batch relaunched by the host after each
                                          status read, instead of one graph with a conditional WHILE node (the path
                                          drivers without conditional nodes take; per-kernel profilers cannot see
                                          inside a graph with conditional nodes) */
} maspcg_flags;

typedef struct {
  int iterations;           /* PCGSolver::pcg return value semantics */
  int status;               /* maspcg_solve_status: which gate stopped the loop (see below) */
  int refinements;          /* FP64 true-residual replacements (MIXED) */
  int launches;             /* CUDA-graph launches */
  double rz0;               /* r0^T z0 */
  double rz_final;          /* last r^T z used by the gate */
  double rel_res_recursive; /* ||r_k|| / ||b|| of the recursive residual */
  double rel_res_true;      /* ||b - A x|| / ||b|| in FP64 with the FP64 input matrix */
  double solve_ms;          /* device time of maspcg_solve (events) */
  /* 1 when rel_res_true <= tolerance: the returned x meets the Euclidean
   * tolerance checked in FP64 against the FP64 input matrix.  MASPCG_SOLVE_
   * CONVERGED alone says only that the configured gate was met by the loop's
   * own quantities (the recursive residual or r^T z), which in FP32 can stop
   * far above the tolerance; a Newton loop that needs the FP64 guarantee
   * reads this field (MIXED stops on the FP64 residual, so there the two
   * agree). */
  int fp64_gate_met;
} maspcg_result;

typedef enum {
  MASPCG_SOLVE_RUNNING = 0,
  MASPCG_SOLVE_CONVERGED = 1,
  MASPCG_SOLVE_ITERATION_CAP = 2,
  MASPCG_SOLVE_NONPOSITIVE_CURVATURE = 3, /* p^T A p <= 0 */
  MASPCG_SOLVE_NONFINITE = 4,
  MASPCG_SOLVE_INVALID_RZ = 5 /* r^T z <= 0 or non-finite: preconditioner not SPD */
} maspcg_solve_status;

/* Defaults of PCGSolverConfig (pcg_solver.h:7-17) and the app
 * (Assets/scene/parameterSetting.txt:14): tol 1e-4, ratio 0.3, rz gate,
 * reference precision, MAS32. */
MASPCG_API void maspcg_config_default(maspcg_config* cfg);

MASPCG_API const char* maspcg_status_string(int status);
/* Message of the last failing call on this handle ("" if none); NULL handle:
 * the last failure of maspcg_create on this thread. */
MASPCG_API const char* maspcg_last_error(const maspcg_handle* h);

/* Replaces GlobalLinearSystem::create<PCGSolver>(PCGSolverConfig) and the
 * preconditioner factory (StiffGIPC/gipc/gipc.cu:67-100,
 * linear_system/solver/pcg_solver.h:7-24).  Uses the current CUDA device. */
MASPCG_API maspcg_status maspcg_create(const maspcg_config* cfg, maspcg_handle** out);
MASPCG_API maspcg_status maspcg_destroy(maspcg_handle* h);
/* cudaStream_t; NULL selects the handle's own stream (created non-blocking:
 * it does not wait for work on the legacy default stream, so a caller that
 * produces inputs on another stream orders them before the call). */
MASPCG_API maspcg_status maspcg_set_stream(maspcg_handle* h, void* stream);
/* The cudaStream_t the handle's work runs on (no counterpart in the
 * reference, which runs on the caller's stream): the one set by
 * maspcg_set_stream, else the handle's own. */
MASPCG_API maspcg_status maspcg_get_stream(const maspcg_handle* h, void** stream);

/* Replaces TraditionalMAS32Preconditioner::initPreconditioner_Neighbor +
 * the caller's cudaMemcpy of d_neighborListInit / d_neighborStart /
 * d_neighborNumInit / d_partId_map_real / d_real_map_partId +
 * initPreconditioner_Matrix (TraditionalMAS32Preconditioner.cuh:78-101,
 * TraditionalMAS32Preconditioner.cu:2889-2977, caller gl_main.cu:1502-1536).
 *   vert_num              FEM vertices (totalNodes)
 *   collision_node_offset vertex-number offset of the FEM range in contact pairs
 *   neighbor_*            vertex neighbour CSR (u32), list of neighbor_list_size
 *   part_map_real         part_map_size slots (multiple of bank_size): slot -> vertex or -1
 *   real_map_part         vert_num entries: vertex -> slot
 * Lane 0 of every bank must hold a vertex (the reference leaves the bank's
 * component count undefined otherwise).  CEMAS16 (MASPreconditioner.cu:
 * 2293-2362, the same inputs with 16-slot banks, METIS-sorted in the app)
 * drops an in-bank block whose slots run against its vertex order
 * (prepare_hessian_bcoo_kernel :1822-1914); a partition whose slots follow
 * the vertex order inside every bank loses nothing. */
MASPCG_API maspcg_status maspcg_set_graph(maspcg_handle* h, int vert_num, int collision_node_offset,
                                          const uint32_t* neighbor_start, const uint32_t* neighbor_num,
                                          const uint32_t* neighbor_list, int neighbor_list_size,
                                          const int* part_map_real, int part_map_size, const int* real_map_part);

/* Contact pairs of the current Newton step: the _collisonPairs / cpNum pair of
 * TraditionalMAS32Preconditioner::setPreconditioner_bcoo
 * (TraditionalMAS32Preconditioner.cu:2643-2682).  pairs4 holds 4*n_pairs ints. */
MASPCG_API maspcg_status maspcg_set_contacts(maspcg_handle* h, const int* pairs4, int n_pairs);

/* The assembled system: GIPCTripletMatrix after Converter::convert
 * (global_matrix.h:18-203, converter.cu:137-284).  Upper BCOO in any order;
 * duplicate (row,col) blocks are summed, as the merge sums them.  Every stored
 * block (r, c), r != c, stands for A_rc and its mirror A_cr = A_rc^T, as in the
 * reference's symmetric SpMV (spmv.cu:28-53), which also applies to a block
 * stored below the diagonal.  The caller passes the triplets the reference
 * merges, so FEM-FEM contact triplets must already have gone through
 * maspcg_adjust_contact_triplets (or the reference's own adjust kernel):
 * before it, a barrier's coupling appears as both (a, b) and (b, a) and would
 * be counted twice, exactly as the reference would count it without that
 * step.
 *   block_rows         total block rows of the system
 *   fem_offset_blocks  first block row of the FEM vertices (MAS range)
 *   abd_body_count     affine bodies occupying block rows [0, 4*abd_body_count) */
MASPCG_API maspcg_status maspcg_set_matrix_bcoo(maspcg_handle* h, const double* values9_colmajor, const int* rows,
                                                const int* cols, int n_blocks, int block_rows, int fem_offset_blocks,
                                                int abd_body_count);

/* The same from a sub-range of a larger triplet list, as the reference hands
 * a subsystem's triplets to the MAS preconditioner: setPreconditioner_bcoo's
 * (values, rows, cols, indices, offset, triplet_num)
 * (TraditionalMAS32Preconditioner.cuh:102-108) with the indices of
 * LocalPreconditioner::calculate_subsystem_bcoo_indices
 * (linear_system/preconditioner/i_preconditioner.cu:54-89).  Block t < n_blocks
 * is source triplet s = indices[t] (s = t when indices is NULL) with rows[s] -
 * offset and cols[s] - offset; source_count is the length of the source
 * arrays (9 * source_count values).  The gather runs on the device; host or
 * device pointers.  An index at or past source_count makes the call return
 * MASPCG_ERR_INVALID_ARGUMENT ("matrix block index out of range"). */
MASPCG_API maspcg_status maspcg_set_matrix_bcoo_indexed(maspcg_handle* h, const double* values9_colmajor,
                                                        const int* rows, const int* cols, long long source_count,
                                                        const uint32_t* indices, int n_blocks, int offset,
                                                        int block_rows, int fem_offset_blocks, int abd_body_count);

/* Replaces LocalPreconditioner::assemble of TraditionalMAS32_Preconditioner /
 * MAS_Preconditioner (CEMAS16) / ABDPreconditioner / DiagPreconditioner
 * (traditional_mas32_preconditioner.cu:20-32, fem_mas_preconditioner.cu:18-31,
 * abd_preconditioner.cu:33-36, diag_preconditioner.cu:74-80): hierarchy for
 * the current contacts, domain matrices, inverses. */
MASPCG_API maspcg_status maspcg_build_preconditioner(maspcg_handle* h);

/* Replaces TraditionalMAS32Preconditioner::refresh_fixed_graph_bcoo
 * (TraditionalMAS32Preconditioner.cuh:118-121, .cu:229-234; caller
 * agipc/agipc_galerkin.cu:131): new values for the blocks of the last
 * maspcg_set_matrix_bcoo, i.e. the same n_blocks triplets with the same rows
 * and cols in the same order (values9 holds 9 * n_blocks doubles, host or
 * device).  The BCSR structure, the internal row order and the MAS hierarchy
 * of the last build are kept; the merged values, the domain matrices and
 * their inverses, and the ABD / block-Jacobi inverses are recomputed, the
 * same as maspcg_set_matrix_bcoo + maspcg_build_preconditioner would give for
 * those values (bit for bit).  As in the reference, the caller guarantees
 * that the structure, the graph and the contact set are unchanged; nothing
 * checks it. */
MASPCG_API maspcg_status maspcg_refresh_matrix_values(maspcg_handle* h, const double* values9_colmajor);

/* The same with the values picked by index from a larger list, as the
 * reference passes them (refresh_fixed_graph_bcoo(values, rows, cols,
 * indices, offset, count)): block t takes values9[indices[t]] for the
 * n_blocks triplets of the last set_matrix (the row and column indices are
 * unchanged and not needed).  source_count bounds the indices; the gather
 * runs on the device.  Host or device pointers. */
MASPCG_API maspcg_status maspcg_refresh_matrix_values_indexed(maspcg_handle* h, const double* values9_colmajor,
                                                             long long source_count, const uint32_t* indices);

/* Replaces IterativeSolver::solve(x, b) -> iterations
 * (i_linear_system_solver.h:43-44, pcg_solver.cu:160-326).  b, x: 3*block_rows
 * doubles.  out may be NULL. */
MASPCG_API maspcg_status maspcg_solve(maspcg_handle* h, const double* b, double* x, maspcg_result* out);

/* Replaces GlobalLinearSystem::apply_preconditioner(z, r)
 * (global_linear_system.cu:293-306): z = M^-1 r over the whole system. */
MASPCG_API maspcg_status maspcg_apply_preconditioner(maspcg_handle* h, const double* r, double* z);

/* Replaces GlobalLinearSystem::spmv(a, x, b, y) (global_linear_system.cu:323-364):
 * y = a*A*x + b*y in FP64. */
MASPCG_API maspcg_status maspcg_spmv(maspcg_handle* h, double a, const double* x, double b, double* y);

/* ---- introspection (parity tests, diagnostics) ---- */

/* y = A x formed by the PCG iteration's own SpMV kernel (no counterpart in
 * the reference: it exposes the product the solve computes, for parity
 * checks against the FP64 product of maspcg_spmv).  x is rounded to the
 * working precision: FP32 in MASPCG_PREC_FP32 and MIXED, where the kernel
 * reads the FP32 matrix tiles and sums in FP32 (the affine-body rows from the
 * FP64 matrix in FP64); FP64 in MASPCG_PREC_REFERENCE.  y is that output
 * widened to FP64.  x, y: 3*block_rows doubles, host or device pointers. */
MASPCG_API maspcg_status maspcg_spmv_working(maspcg_handle* h, const double* x, double* y);

typedef struct {
  int levelnum;          /* computeNumLevels */
  int total_clusters;    /* totalNumberClusters */
  int domains;           /* total_clusters / bank_size */
  int vert_num;          /* totalNodes */
  int part_map_size;     /* totalMapNodes */
  long long going_next_capacity;
  int internal_block_rows;
  int bcsr_blocks;       /* stored blocks of the full BCSR */
  int failed_domains;    /* domains whose elimination met a pivot <= 0 */
  long long kernel_launches; /* kernels of this library launched on the handle so far
                                (graph launches count every kernel node) */
  long long graph_captures;  /* solve graphs captured and instantiated so far: a solve
                                re-captures only when buffers, sizes, the hierarchy's
                                level table, the configuration or the stream changed */
} maspcg_info;

MASPCG_API maspcg_status maspcg_get_info(maspcg_handle* h, maspcg_info* info);

/* Integer hierarchy after the last build, reference layouts
 * (TraditionalMAS32Preconditioner.cuh:35-64); any pointer may be NULL; host
 * pointers.  fine_mask[vert_num], coarse_space_tables[levelnum*vert_num],
 * going_next[going_next_capacity], level_size[2*(levelnum+1)],
 * coarse_table[6*vert_num], prefix_original[part_map_size/bank_size]. */
MASPCG_API maspcg_status maspcg_get_hierarchy(maspcg_handle* h, uint32_t* fine_mask, int* coarse_space_tables,
                                              int* going_next, int* level_size, int* coarse_table,
                                              int* prefix_original);

/* Full BCSR (both triangles) in the internal block-row order.  rowptr
 * [internal_block_rows+1], colidx [bcsr_blocks], values [9*bcsr_blocks]
 * row-major FP64 (may be NULL), internal_of_row [block_rows] (may be NULL). */
MASPCG_API maspcg_status maspcg_get_bcsr(maspcg_handle* h, int* rowptr, int* colidx, double* values_rowmajor,
                                         int* internal_of_row);

/* Domain inverses in the reference's packed layout (GPUMas32MatrixSymf;
 * MasMatrixSymf for CEMAS16): P = B(B+1)/2 upper 3x3 blocks per domain for
 * bank B (528 or 136), block (a,b) at Ba - a(a+1)/2 + b, 9 floats
 * column-major; decoded from whatever precision is stored.  out: domains*P*9. */
MASPCG_API maspcg_status maspcg_get_domain_inverses(maspcg_handle* h, float* out);

/* Assembled FP64 domain matrices (GPUMas32MatrixSymT / MasMatrixSymT layout)
 * of the last build, before the zero-diagonal rule: recomputed on demand.
 * out: domains*P*9 (P as above). */
MASPCG_API maspcg_status maspcg_get_domain_matrices(maspcg_handle* h, double* out);

/* Per-domain numerical checks of the MAS preconditioner: the fields of
 * LocalGpuCheck / check_local_matrices (TraditionalMAS32Preconditioner.cu:
 * 76-147).  A = the assembled FP64 domain matrix with zero diagonal entries
 * set to 1, M = the stored inverse decoded to FP32. */
typedef struct {
  int local_finite;                /* every entry of A finite */
  int inverse_finite;              /* every entry of M finite */
  int local_spd;                   /* FP64 Cholesky of A met only positive pivots */
  int inverse_spd;                 /* M SPD: implied by local_spd and residual <= 1e-3, else its own Cholesky */
  double minimum_local_diagonal;
  double minimum_inverse_diagonal;
  double inverse_residual;         /* ||A M - I||_F / sqrt(n), n = 3 * bank (0 unless both are finite) */
} maspcg_domain_check;

/* The summary gpu_local_checks builds from them (:149-180); passed = every
 * domain SPD both ways, finite, and every inverse residual <= 1e-3.  First
 * failures are domain indices, -1 if none. */
typedef struct {
  int matrix_count;
  int local_spd_count;
  int inverse_spd_count;
  int first_local_spd_failure;
  int first_inverse_spd_failure;
  int nonfinite_local_count;
  int nonfinite_inverse_count;
  int passed;
  double minimum_local_diagonal;
  double minimum_inverse_diagonal;
  double maximum_inverse_residual;
} maspcg_diagnostics;

/* The checks on the domains of the last build: local_diagnostics_gpu and the
 * local part of numerical_diagnostics (TraditionalMAS32Preconditioner.cuh:
 * 116-117, .cu:182-183, :2727-2887).  per_domain (host, one entry per domain,
 * maspcg_get_info().domains) may be NULL; summary may be NULL.  The domain
 * matrices are assembled again on the device for the check. */
MASPCG_API maspcg_status maspcg_local_diagnostics(maspcg_handle* h, maspcg_domain_check* per_domain,
                                                  maspcg_diagnostics* summary);

/* The same checks on caller matrices: gpu_local_checks(local, inverse, count)
 * (:149-180).  packed64: count domains of B(B+1)/2 packed upper FP64 3x3
 * blocks (the layout of maspcg_get_domain_matrices), inverse32: the same in
 * FP32 (maspcg_get_domain_inverses); bank 32 or 16.  Host or device
 * pointers; per_domain / summary on the host, may be NULL.  Any handle. */
MASPCG_API maspcg_status maspcg_check_local_matrices(maspcg_handle* h, int count, int bank, const double* packed64,
                                                     const float* inverse32, maspcg_domain_check* per_domain,
                                                     maspcg_diagnostics* summary);

/* Benchmark introspection (no counterpart in the reference): run one stage
 * `repeats` times on the handle's stream, each run after reading a 256 MB
 * buffer that evicts L2 (clean lines only), and return the mean device
 * milliseconds per run: CUDA events around the whole sequence, minus the
 * same sequence of evictions alone (allocates the buffer on first use).
 * Stages:
 *   0  PCG SpMV with the p.Ap reduction, working precision
 *   1  full preconditioner apply z = M^-1 r, working precision
 *   2  MAS level-0 domain apply alone (restriction/coarse levels excluded)
 *   3  MAS domain assembly + inversion (build)
 *   4  MAS level-0 domain apply (tensor-core passes over 16-bit records staged
 *      in shared memory by TMA bulk copies), two slots per warp
 *   5  the same with one slot per warp (more warps per SM; the solve's choice)
 *   6  the same apply with each record staged by per-lane 16-byte loads (no TMA)
 *   7  MASPCG_PREC_MIXED only: the residual replacement, x_hi += x_lo and
 *      r = b - A x_hi with the FP64 matrix (FP64 sums, FP32 copy of r)
 *   (stage 2 times the variant the solve uses; 4-6 exist to compare them)
 * Vector contents are left unspecified afterwards. */
MASPCG_API maspcg_status maspcg_time_stage(maspcg_handle* h, int stage, int repeats, double* mean_ms);

/* The triplet merge in front of the solve: Converter::convert
 * (StiffGIPC/linear_system/utils/converter.cu:137-284).  Sorts n block
 * triplets by the key (row << 32) + col, ascending, and sums the 3x3 blocks
 * of equal keys.  values9 / values9_out are 9 doubles per block in any fixed
 * layout (summed elementwise; the reference's Eigen column-major).  The
 * outputs need room for n blocks; *n_out receives the number of unique
 * blocks.  The blocks of one key are summed in input order, so the result is
 * deterministic (the reference's FP64 atomics are not).  Negative indices
 * return MASPCG_ERR_INVALID_ARGUMENT.  Host or device pointers; any handle
 * (only its stream and scratch are used). */
MASPCG_API maspcg_status maspcg_convert_bcoo(maspcg_handle* h, const double* values9, const int* rows,
                                             const int* cols, int n, double* values9_out, int* rows_out,
                                             int* cols_out, int* n_out);

/* Contact triplets grouped by kind: GIPC::partitionContactHessian
 * (StiffGIPC/GIPC.cu:9952-10128).  type_hash[t] is 0 (FEM-FEM), 1 (ABD-FEM),
 * 2 (FEM-ABD) or 3 (ABD-ABD); the outputs hold the n triplets ordered by
 * type, stable within a type, and counts[k] the number of type k.  A hash
 * above 3 returns MASPCG_ERR_INVALID_ARGUMENT.  Host or device pointers. */
MASPCG_API maspcg_status maspcg_partition_contact_triplets(maspcg_handle* h, const double* values9, const int* rows,
                                                           const int* cols, const unsigned long long* type_hash,
                                                           int n, double* values9_out, int* rows_out,
                                                           int* cols_out, int counts[4]);

/* Contact-pair dedup of the FEM-FEM contact triplets, in place:
 * adjust_fem_fem_contact_indices_kernel (StiffGIPC/GIPC.cu:10130-10160).  A
 * barrier Hessian emits the full block pattern of its pair, so every coupling
 * appears as (a, b) and as (b, a).  For triplet i, (r, c) = (rows[i],
 * cols[i]) in FEM vertex numbering:
 *   r <= c: rows[i] = r + fem_offset, cols[i] = c + fem_offset; the value is
 *           cleared (nine +0.0) when bd_type[r] or bd_type[c] is nonzero;
 *   r >  c: rows[i] = c + fem_offset, cols[i] = r + fem_offset and the value
 *           is cleared: its upper twin carries the block.
 * bd_type holds n_vertices ints (TetMesh.BoundaryType).  fem_offset is the
 * reference's fem_global_hessian_index_offset (4 * ABD bodies - ABD points).
 * A triplet naming a vertex outside [0, n_vertices) is left unchanged and the
 * call returns MASPCG_ERR_INVALID_ARGUMENT (the reference does not check).
 * Host or device pointers. */
MASPCG_API maspcg_status maspcg_adjust_contact_triplets(maspcg_handle* h, int n, int* rows, int* cols,
                                                        double* values9_colmajor, const int* bd_type, int n_vertices,
                                                        int fem_offset);

/* zero_fem_boundary_hessian_kernel (StiffGIPC/GIPC.cu:10162-10181), in
 * place: the value of triplet i is cleared when bd_type[rows[i] -
 * index_offset] or bd_type[cols[i] - index_offset] is nonzero; indices are
 * not changed.  Range rule and pointers as maspcg_adjust_contact_triplets. */
MASPCG_API maspcg_status maspcg_zero_boundary_triplets(maspcg_handle* h, int n, const int* rows, const int* cols,
                                                       double* values9_colmajor, const int* bd_type, int n_vertices,
                                                       int index_offset);

/* The FEM part of A: per-tet gradient and PSD-projected Hessian of the stable
 * Neo-Hookean energy, _calculate_fem_gradient_hessian
 * (StiffGIPC/femEnergy.cu:1720-1856, SNK1 branch; projection
 * :1641-1717).  Inputs per tet: tets (4 vertex ids), dm_inverse (Dm^-1,
 * 9 doubles row-major), volume, len_rate and vol_rate (the Lame rates,
 * gl_main.cu:586-630); x: current positions, 3 doubles per vertex (n_vertices).
 * gradient (3 doubles per vertex) is accumulated with FP64 atomics, as in the
 * reference: clear it first.  rows/cols/values9_colmajor receive 10 triplets
 * per tet at [10t, 10t + 10): the tet's upper 3x3 blocks with vertex ids +
 * hessian_offset, row <= col.  A vertex id >= n_vertices returns
 * MASPCG_ERR_INVALID_ARGUMENT (checked on the device; that tet is skipped and
 * the outputs are unspecified).  Host or device pointers. */
MASPCG_API maspcg_status maspcg_fem_snk1_gradient_hessian(maspcg_handle* h, int n_tets, const unsigned* tets,
                                                          int n_vertices, const double* x, const double* dm_inverse,
                                                          const double* volume, const double* len_rate,
                                                          const double* vol_rate, double dt, int hessian_offset,
                                                          double* gradient, int* rows, int* cols,
                                                          double* values9_colmajor);

/* The AGIPC coarse space (StiffGIPC/agipc/agipc_galerkin.cu, mapping of
 * agipc_criterion.cuh:13-25).  Fine blocks [0, prefix_blocks) pass through;
 * FEM node k (fine block prefix_blocks + k, k < fem_nodes) belongs to coarse
 * node fine_to_coarse[k] (< coarse_nodes), whose blocks start at
 * prefix_blocks + coarse_block_bases[c] and whose basis is the subset
 * basis_masks[c] (bits 0-3, 1..15) of (1, x, y, z) at the node's rest
 * position rest_positions[3k..3k+2]: a translational node has mask 1, an
 * affine node 15.  The coarse system has prefix_blocks + coarse_block_nodes
 * block rows. */
typedef struct maspcg_galerkin_map {
  const int* fine_to_coarse;
  const int* coarse_block_bases;
  const int* basis_masks;
  const double* rest_positions;
  int prefix_blocks;
  int fem_nodes;
  int coarse_nodes;
  int coarse_block_nodes;
} maspcg_galerkin_map;

/* A_c = P^T A P (count_expanded_blocks / emit_expanded_blocks + Converter,
 * agipc_galerkin.cu:221-283, :921-953): every fine upper triplet expands into
 * phi_i[a] phi_j[b] A_ij blocks, which are merged as maspcg_convert_bcoo does.
 * Writes the unique upper coarse blocks (row <= col, ascending keys) and
 * *n_coarse; if capacity is smaller, returns MASPCG_ERR_CAPACITY with the
 * needed count in *n_coarse. */
MASPCG_API maspcg_status maspcg_galerkin_coarse_matrix(maspcg_handle* h, const maspcg_galerkin_map* map,
                                                       const double* values9, const int* rows, const int* cols,
                                                       int n, double* coarse_values9, int* coarse_rows,
                                                       int* coarse_cols, int capacity, int* n_coarse);

/* b_c = P^T b (reduce_mixed_rhs, agipc_galerkin.cu:285-306; FP64 atomics as
 * in the reference).  fine_rhs: 3 (prefix_blocks + fem_nodes) doubles;
 * coarse_rhs: 3 (prefix_blocks + coarse_block_nodes). */
MASPCG_API maspcg_status maspcg_galerkin_restrict(maspcg_handle* h, const maspcg_galerkin_map* map,
                                                  const double* fine_rhs, double* coarse_rhs);

/* x = P x_c (prolongate_mixed, agipc_galerkin.cu:355-369). */
MASPCG_API maspcg_status maspcg_galerkin_prolong(maspcg_handle* h, const maspcg_galerkin_map* map,
                                                 const double* coarse_x, double* fine_x);

/* Matrix adjoint of the solve (no counterpart in the reference; the backward
 * of the differentiable Newton-step solve).  For L(x) with x = A^-1 b and
 * lam = A^-1 dL/dx, writes dL/d(values) for every input block t of an upper
 * BCOO list, (r, c) = (rows[t], cols[t]):
 *   r != c:  grad9[t] = -(lam_r x_c^T + x_r lam_c^T)
 *   r == c:  grad9[t] = -lam_r x_r^T
 * column-major 3x3 like values9_colmajor.  lam and x: 3*block_rows doubles in
 * the caller's order.  Host or device pointers. */
MASPCG_API maspcg_status maspcg_bcoo_gradient(maspcg_handle* h, const int* rows, const int* cols, int n_blocks,
                                              const double* lam, const double* x, double* grad9_colmajor);

/* The matrix adjoint chained to per-tet Young's modulus (no counterpart in
 * the reference; the backward of the differentiable solve): the first
 * n_tets * blocks_per_tet blocks of an upper BCOO list are the element blocks
 * of the tets in tet order (blocks_per_tet each, 10 for a tetrahedron's upper
 * blocks), each linear in its tet's modulus youngs[t].  With lam and x as in
 * maspcg_bcoo_gradient, grad_youngs[t] = sum over tet t's blocks k of
 * <G_k, values9_k> / youngs[t], G_k the block gradient of
 * maspcg_bcoo_gradient, computed without storing G.  Host or device pointers. */
MASPCG_API maspcg_status maspcg_element_modulus_gradient(maspcg_handle* h, int n_tets, int blocks_per_tet,
                                                         const int* rows, const int* cols,
                                                         const double* values9_colmajor, const double* lam,
                                                         const double* x, const double* youngs,
                                                         double* grad_youngs);

/* Test hook for the bounded waits (no counterpart in the reference): the
 * grid barriers of the MASPCG_FLAG_FUSED_HEAD kernel give up after
 * barrier_limit spins (default 2^24, each a 64 ns sleep) and then stop the
 * solve, which returns MASPCG_ERR_CUDA ("a grid barrier of the fused
 * iteration kernel timed out"); barrier_extra > 0 makes every barrier wait
 * for arrivals that never come, so a test can drive that path without a GPU
 * fault.  (0, default) restores normal barriers.  Applies from the next
 * maspcg_solve. */
MASPCG_API maspcg_status maspcg_set_wait_test_hooks(maspcg_handle* h, long long barrier_limit, int barrier_extra);

/* Most vectors one maspcg_residual_norms_noalloc call accepts. */
#define MASPCG_RESIDUAL_MAX_VECTORS 8

/* Allocation-free residual check (no counterpart in the reference): for
 * j < count, residual_norms[j] = ||b_j - A x_j||_2 and, when rhs_norms is not
 * NULL, rhs_norms[j] = ||b_j||_2, in FP64, with A the matrix of the last
 * maspcg_set_matrix_bcoo.  x and b are DEVICE pointers to `count` vectors of
 * 3*block_rows doubles stored one after another, in the caller's row order;
 * the norms go to host memory.  count outside 1..MASPCG_RESIDUAL_MAX_VECTORS
 * returns MASPCG_ERR_CAPACITY; host x or b return MASPCG_ERR_INVALID_ARGUMENT.
 *
 * The call allocates no memory: its scratch (per-block partial sums, results
 * and a completion ticket) is one fixed 65,696-byte device array per device
 * inside the library.  Its device address is looked up on every call; the
 * first call for a device (and the first after that device's context was
 * created again) also clears the array's completion ticket with a small
 * memset and a stream synchronisation: make that first call before any stream
 * capture is active.  Calls for one device are serialised by a lock held until
 * the call's stream has finished; the call synchronises the handle's stream
 * before it returns. */
MASPCG_API maspcg_status maspcg_residual_norms_noalloc(maspcg_handle* h, int count, const double* x, const double* b,
                                                       double* residual_norms, double* rhs_norms);

#ifdef __cplusplus
}
#endif
#endif /* MASPCG_H */
