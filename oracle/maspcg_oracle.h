/*
 * maspcg_oracle.h -- CPU restatement of StiffGIPC's Newton-step linear solve.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the parity checker for the CUDA
 * path in agipc_learning_b200/ and the timed CPU baseline of bench.py.  It is
 * never linked into, called by, or shipped with the product path.  Only
 * tests/, __graft_entry__.smoke() and bench.py (cpu_baseline leg and the
 * --impl reference arm) may load it.
 *
 * Every function restates one piece of the reference (KLBSTL/AGIPC_LEARNING,
 * StiffGIPC) in plain C; the file:line it follows is given beside it.  The
 * reference itself cannot be compiled in this environment (it needs Eigen 3.4
 * inside device code), so parity is pinned against the reference's own
 * known-answer tests and fixtures instead (see tests/golden/).
 *
 * Block layout conventions (shared with the product ABI):
 *   - a 3x3 block is 9 doubles in Eigen::Matrix3d column-major order,
 *     element (r,c) at index r + 3*c  (global_matrix.h:21-25);
 *   - a symmetric matrix is given as upper BCOO: row <= col, block (r,c)
 *     holds A_rc, and A_cr = A_rc^T is implied (spmv.cu:28-53).
 */
#ifndef MASPCG_ORACLE_H
#define MASPCG_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- BCOO --- */

/* Converter::convert (converter.cu:137-284): triplets -> unique blocks sorted
 * by the 64-bit key (row<<32)+col, duplicates summed.  The sort is stable and
 * duplicates are summed in input order.  Returns the unique count; outputs
 * must hold n entries. */
int orc_convert_triplets(int n, const int* rows, const int* cols, const double* vals9,
                         int* out_rows, int* out_cols, double* out_vals9);
int orc_partition_contacts(int n, const int* rows, const int* cols, const double* vals9, const uint64_t* type,
                           int* out_rows, int* out_cols, double* out_vals9, int* counts);

/* adjust_fem_fem_contact_indices_kernel (GIPC.cu:10130-10160), in place:
 * r <= c keeps its order, r > c swaps to the upper slot and is cleared, an
 * upper triplet touching a nonzero bd_type is cleared; offset added to both
 * indices.  Returns the first triplet index naming a vertex outside
 * [0, nv) (that triplet untouched) or -1. */
int orc_adjust_contacts(int n, int* rows, int* cols, double* vals9, const int* bd_type, int nv, int offset);
/* zero_fem_boundary_hessian_kernel (GIPC.cu:10162-10181), in place; same
 * return rule with the vertex index row/col - offset. */
int orc_zero_boundary(int n, const int* rows, const int* cols, double* vals9, const int* bd_type, int nv, int offset);

/* Spmv::*_sym_spmv (spmv.cu:28-53, CPU loop spmv.cu:348-364):
 * y = a*A*x + b*y with A given as upper BCOO.  Sequential, input order. */
void orc_sym_spmv(double a, const double* vals9, const int* rows, const int* cols,
                  int nblocks, int dof, const double* x, double b, double* y);

/* Full block-CSR (both triangles) from upper BCOO.  rowptr has nb+1 entries,
 * colidx/vals9 room for 2*nblocks.  Columns within a row are ascending.
 * Returns the number of stored blocks. */
int orc_upper_to_full_bcsr(int nb, int nblocks, const int* rows, const int* cols,
                           const double* vals9, int* rowptr, int* colidx, double* full_vals9);

/* y = A*x over a full BCSR (OpenMP over rows; deterministic per row). */
void orc_bcsr_spmv(int nb, const int* rowptr, const int* colidx, const double* vals9,
                   const double* x, double* y);

/* ---------------------------------------------------------------- MAS32 -- */

/* MAS bank: 32 (TraditionalMAS32), or 16 for the CEMAS16 build (-DORC_BANK=16,
 * liboracle16.so: MASPreconditioner.cu, the same algorithm with BANKSIZE 16
 * and the differences marked ORC_BANK == 16 in maspcg_oracle.c). */
#ifndef ORC_BANK
#define ORC_BANK 32
#endif
#define ORC_MAX_LEVELS 6

typedef struct orc_mas orc_mas;

/* initPreconditioner_Neighbor + caller uploads (TraditionalMAS32Preconditioner.cu:2889-2926,
 * gl_main.cu:1502-1536).  Arrays are copied. Returns NULL on invalid input. */
orc_mas* orc_mas_create(int vert_num, int collision_node_offset,
                        const uint32_t* neighbor_start, const uint32_t* neighbor_num,
                        const uint32_t* neighbor_list, int neighbor_list_size,
                        const int* part_map_real, int part_map_size,
                        const int* real_map_part);
void orc_mas_free(orc_mas* m);

/* computeNumLevels (TraditionalMAS32Preconditioner.cu:2142-2161). */
int orc_compute_num_levels(int vert_num);
int orc_mas_levelnum(const orc_mas* m);
/* gipc::hierarchy_capacity (gipc/hierarchy_capacity.h:10-22); -1 on overflow. */
long long orc_hierarchy_capacity(long long vertices, long long mapped, long long levels, long long bank);
long long orc_mas_going_next_capacity(const orc_mas* m);

/* ReorderRealtime (TraditionalMAS32Preconditioner.cu:2189-2230) with contact
 * pairs encoded as int4 (x,y,z,w) exactly as _buildCollisionConnection_new
 * (:1550-1962).  Returns totalNumberClusters. */
int orc_mas_reorder(orc_mas* m, const int* pairs4, int cp_num);

/* Export the integer hierarchy.  Any pointer may be NULL.
 *   fine_mask[nv], coarse_space_tables[nv*levelnum], going_next[capacity],
 *   level_size[2*(levelnum+1)] (x,y pairs), coarse_table[nv*6],
 *   prefix_original[C0/32]. */
void orc_mas_get_hierarchy(const orc_mas* m, uint32_t* fine_mask, int* coarse_space_tables,
                           int* going_next, int* level_size, int* coarse_table,
                           int* prefix_original);
int orc_mas_total_clusters(const orc_mas* m);

/* PrepareHessian_bcoo (:2467-2557): scatter the selected upper blocks into the
 * packed FP64 domain matrices (prepare_hessian_bcoo_kernel :2234-2338 and
 * prepare_hessian_bcoo_sum_kernel :2340-2464), expand with the zero-diagonal
 * rule (expand_symmetric_mas32 :1062-1096), invert by Gauss-Jordan without
 * pivoting (__inverse6_P96x96 :1099-1146) and store the FP32 packed upper
 * inverse. */
void orc_mas_prepare_hessian(orc_mas* m, const double* vals9, const int* rows, const int* cols,
                             const uint32_t* indices, int offset, int triplet_num);

/* Domain matrices: packed upper, 528 blocks per domain, block (a,b) a<=b at
 * index 32a - a(a+1)/2 + b, each block 9 values column-major.
 * packed64 gets the FP64 matrices before the zero-diagonal rule,
 * inverse32 the FP32 inverses.  Either may be NULL. */
void orc_mas_get_domains(const orc_mas* m, double* packed64, float* inverse32);

/* Replace the FP32 inverses (the layout of orc_mas_get_domains) with the
 * caller's, after orc_mas_prepare_hessian: the apply then uses exactly those
 * operators (to check another build's inverses through the same apply). */
void orc_mas_set_inverses(orc_mas* m, const float* inverse32);

/* preconditioning (:2684-2725): R,Z are double3 arrays of length vert_num. */
void orc_mas_precondition(const orc_mas* m, const double* R, double* Z);

/* check_local_matrices (:76-147) on given packed matrices.  Per domain the 7
 * results are {local_finite, inverse_finite, local_spd, inverse_spd,
 * min_local_diag, min_inverse_diag, inverse_residual}. */
void orc_local_checks(int count, const double* packed64, const float* inverse32, double* results7);

/* Block-Jacobi inverses.
 * 3x3: DiagPreconditioner (diag_preconditioner.cu:10-39): identity where the
 *      diagonal block is missing. out: nb*9 (column-major).
 * 12x12: ABDPreconditioner (setup_abd_system_gradient_and_hessian.cu:407-441),
 *      gathered from blocks with row/4 == col/4 inside the ABD range.
 *      out: bodies*144 row-major. */
void orc_diag3_inverse(int nb, int nblocks, const int* rows, const int* cols, const double* vals9,
                       double* inv9);
int orc_abd_inverse(int bodies, int nblocks, const int* rows, const int* cols, const double* vals9,
                    double* inv144);

/* ------------------------------------------------------------------ PCG -- */

enum {
  ORC_PRECOND_DIAG3 = 0, /* DiagPreconditioner (global) + ABD local */
  ORC_PRECOND_MAS16 = 1, /* the same with CEMAS16 (liboracle16.so only) */
  ORC_PRECOND_MAS32 = 2, /* identity copy + ABD local + MAS on the FEM range (bank ORC_BANK) */
  ORC_PRECOND_NONE = -1
};
enum {
  ORC_GATE_RZ = 0,     /* PCGSolver::pcg: |rz_prev| <= tol*rz0, checked after the update */
  ORC_GATE_EUCLID = 1  /* ||r||^2 <= tol^2 ||b||^2 after the update (replay harness) */
};
enum {
  ORC_STATUS_CONVERGED = 1,
  ORC_STATUS_ITERATION_CAP = 2,
  ORC_STATUS_NONPOSITIVE_CURVATURE = 3,
  ORC_STATUS_NONFINITE = 4,
  ORC_STATUS_INVALID_RZ = 5
};

typedef struct {
  int precond;
  int gate;
  double tol;
  int max_iter;          /* PCGSolver: loop k=1..max_iter-1; <=0 means 0.3*dof */
  int nb;                /* block rows */
  int fem_offset;        /* first FEM block row */
  int fem_count;         /* FEM vertices (MAS range) */
  int abd_bodies;        /* bodies occupy block rows [0, 4*abd_bodies) */
  int replay_checks;     /* 1: stop on rz<=0 / curvature<=0 like run_replay_pcg */
} orc_pcg_opts;

typedef struct {
  int iterations;
  int status;
  double rz0;
  double rz_last;
  double rel_res_recursive;
  double rel_res_true;
} orc_pcg_result;

/* PCGSolver::solve + PCGSolver::pcg (pcg_solver.cu:160-326) with
 * GlobalLinearSystem::apply_preconditioner (global_linear_system.cu:293-306).
 * A is the unique upper BCOO.  mas must have been prepared when precond is
 * MAS32 and fem_count > 0.  Returns iterations. */
int orc_pcg(const orc_pcg_opts* o, const double* vals9, const int* rows, const int* cols, int nblocks,
            const orc_mas* mas, const double* b, double* x, orc_pcg_result* out);

int orc_num_threads(void);

/* FP64 direct solve of the symmetric positive definite system given by its
 * upper BCOO blocks (Eigen column-major 3x3 values; repeated blocks add):
 * reverse Cuthill-McKee ordering of the block graph, envelope (skyline)
 * Cholesky A = L L^T of the reordered scalar matrix, two triangular solves.
 * The FP64 direct oracle at small sizes (the reference's own scripts use
 * SciPy's sparse LU; Eigen's sparse Cholesky is not available here).
 * Returns 0, -1 if a pivot is not positive, -2 if memory runs out.
 * envelope_out (may be NULL) receives the number of stored entries of L. */
int orc_direct_solve(int nb, int nblocks, const int* rows, const int* cols, const double* vals9, const double* b,
                     double* x, long long* envelope_out);

#ifdef __cplusplus
}
#endif
#endif
