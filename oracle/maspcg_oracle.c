/*
 * maspcg_oracle.c -- CPU restatement of StiffGIPC's MAS32-preconditioned PCG.
 *
 * TEST INFRASTRUCTURE ONLY (see maspcg_oracle.h).  Not part of the product.
 *
 * Integer work (hierarchy, BCOO structure) follows the reference step by step
 * so that its outputs are bit-exact with the reference's definition.  Floating
 * point work follows the reference's precision choices (FP64 PCG and domain
 * matrices, FP64 Gauss-Jordan inverse cast to FP32, FP32 MAS apply) with a
 * fixed summation order where the reference uses atomics.
 *
 * Built twice: liboracle.so (ORC_BANK 32, TraditionalMAS32Preconditioner.cu)
 * and liboracle16.so (ORC_BANK 16, CEMAS16: MASPreconditioner.cu, whose
 * kernels are the MAS32 ones with BANKSIZE 16 apart from the three places
 * marked ORC_BANK == 16 below).
 *
 * Parity pins: the spmv self-test KAT (spmv.cu:301-459), the MAS32 hierarchy
 * self-test KAT (TraditionalMAS32Preconditioner.cu:257-427), the local
 * diagnostics cases (:182-215), hierarchy_capacity asserts
 * (tests/runtime_options_tests.cpp:33-36) and the 257-block coarse replay
 * fixture (reports/agipc_reproduction/make_coarse_replay_fixture.py with the
 * results in AGIPC_COARSE_MAS32_REPLAY.md:35-52).
 */
#include "maspcg_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define BANK ORC_BANK
#define NPACK (BANK * (BANK + 1) / 2) /* 528 packed upper 3x3 blocks */
#define DIM (3 * BANK)                /* 96 scalar rows per domain */

static inline int popc32(uint32_t x) { return __builtin_popcount(x); }
/* CUDA __ffs: 1-based index of the lowest set bit, 0 when none. */
static inline int ffs32(uint32_t x) { return x ? __builtin_ctz(x) + 1 : 0; }
static inline uint32_t lanemask_lt(int lane) { return (1u << lane) - 1u; }
/* packed upper index of block (a,b), a <= b (eigen_data.h GPUMas32MatrixSymT). */
static inline int pk(int a, int b) { return BANK * a - a * (a + 1) / 2 + b; }
static inline int ceil32(int n) { return (n + BANK - 1) / BANK * BANK; }

int orc_num_threads(void)
{
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* ======================================================================= */
/*  BCOO conversion and SpMV                                                */
/* ======================================================================= */

typedef struct {
  uint64_t key;
  int idx;
} keyidx;

static int cmp_keyidx(const void* a, const void* b)
{
  const keyidx* x = (const keyidx*)a;
  const keyidx* y = (const keyidx*)b;
  if (x->key != y->key) return x->key < y->key ? -1 : 1;
  return x->idx < y->idx ? -1 : (x->idx > y->idx);
}

/* converter.cu:8-20 (key), :160-198 (stable radix sort + gather),
 * :237-284 (run heads, exclusive scan, segmented 3x3 sum). */
int orc_convert_triplets(int n, const int* rows, const int* cols, const double* vals9,
                         int* out_rows, int* out_cols, double* out_vals9)
{
  if (n < 1) return 0;
  keyidx* k = (keyidx*)malloc(sizeof(keyidx) * (size_t)n);
  for (int i = 0; i < n; ++i) {
    k[i].key = ((uint64_t)(uint32_t)rows[i] << 32) + (uint64_t)(uint32_t)cols[i];
    k[i].idx = i;
  }
  qsort(k, (size_t)n, sizeof(keyidx), cmp_keyidx);
  int u = -1;
  for (int i = 0; i < n; ++i) {
    if (i == 0 || k[i].key != k[i - 1].key) {
      ++u;
      out_rows[u] = (int)(k[i].key >> 32);
      out_cols[u] = (int)(k[i].key & 0xffffffffu);
      memset(out_vals9 + 9 * (size_t)u, 0, 9 * sizeof(double));
    }
    const double* s = vals9 + 9 * (size_t)k[i].idx;
    double* d = out_vals9 + 9 * (size_t)u;
    for (int e = 0; e < 9; ++e) d[e] += s[e];
  }
  free(k);
  return u + 1;
}

/* GIPC.cu:9952-10128 (partitionContactHessian) with _partition_collision_
 * triplets / _reorder_triplets (GIPC.cu:218-283): a stable sort of contact
 * triplets on their type hash 0..3 (FEM-FEM, ABD-FEM, FEM-ABD, ABD-ABD), here
 * as a counting sort; counts[k] = triplets of type k.  Returns -1 for a hash
 * above 3. */
int orc_partition_contacts(int n, const int* rows, const int* cols, const double* vals9, const uint64_t* type,
                           int* out_rows, int* out_cols, double* out_vals9, int* counts)
{
  int start[4] = {0, 0, 0, 0};
  for (int k = 0; k < 4; ++k) counts[k] = 0;
  for (int i = 0; i < n; ++i) {
    if (type[i] > 3) return -1;
    counts[type[i]]++;
  }
  for (int k = 1; k < 4; ++k) start[k] = start[k - 1] + counts[k - 1];
  for (int i = 0; i < n; ++i) {
    const int d = start[type[i]]++;
    out_rows[d] = rows[i];
    out_cols[d] = cols[i];
    memcpy(out_vals9 + 9 * (size_t)d, vals9 + 9 * (size_t)i, 9 * sizeof(double));
  }
  return 0;
}

/* adjust_fem_fem_contact_indices_kernel (GIPC.cu:10130-10160): one triplet
 * at a time, in input order. */
int orc_adjust_contacts(int n, int* rows, int* cols, double* vals9, const int* bd_type, int nv, int offset)
{
  int first_bad = -1;
  for (int i = 0; i < n; ++i) {
    const int r = rows[i], c = cols[i];
    if (r < 0 || c < 0 || r >= nv || c >= nv) {
      if (first_bad < 0) first_bad = i;
      continue;
    }
    int clear;
    if (r <= c) {
      rows[i] = r + offset;
      cols[i] = c + offset;
      clear = bd_type[r] != 0 || bd_type[c] != 0;
    } else {
      rows[i] = c + offset;
      cols[i] = r + offset;
      clear = 1;
    }
    if (clear)
      for (int e = 0; e < 9; ++e) vals9[9 * (size_t)i + e] = 0.0;
  }
  return first_bad;
}

/* zero_fem_boundary_hessian_kernel (GIPC.cu:10162-10181). */
int orc_zero_boundary(int n, const int* rows, const int* cols, double* vals9, const int* bd_type, int nv, int offset)
{
  int first_bad = -1;
  for (int i = 0; i < n; ++i) {
    const int a = rows[i] - offset, b = cols[i] - offset;
    if (a < 0 || b < 0 || a >= nv || b >= nv) {
      if (first_bad < 0) first_bad = i;
      continue;
    }
    if (bd_type[a] != 0 || bd_type[b] != 0)
      for (int e = 0; e < 9; ++e) vals9[9 * (size_t)i + e] = 0.0;
  }
  return first_bad;
}

/* spmv.cu:14-53 and the self-test CPU loop spmv.cu:348-364. */
void orc_sym_spmv(double a, const double* vals9, const int* rows, const int* cols,
                  int nblocks, int dof, const double* x, double b, double* y)
{
  for (int i = 0; i < dof; ++i) y[i] = (b != 0.0) ? b * y[i] : 0.0;
  for (int k = 0; k < nblocks; ++k) {
    const double* B = vals9 + 9 * (size_t)k;
    const int i = rows[k], j = cols[k];
    for (int r = 0; r < 3; ++r) {
      double s = 0.0;
      for (int c = 0; c < 3; ++c) s += B[r + 3 * c] * x[3 * j + c];
      y[3 * i + r] += a * s;
    }
    if (i != j) {
      for (int r = 0; r < 3; ++r) {
        double s = 0.0;
        for (int c = 0; c < 3; ++c) s += B[c + 3 * r] * x[3 * i + c];
        y[3 * j + r] += a * s;
      }
    }
  }
}

typedef struct {
  int col;
  int src;
  int transpose;
} bcsr_ent;

static int cmp_ent(const void* a, const void* b)
{
  const bcsr_ent* x = (const bcsr_ent*)a;
  const bcsr_ent* y = (const bcsr_ent*)b;
  if (x->col != y->col) return x->col < y->col ? -1 : 1;
  return x->src < y->src ? -1 : (x->src > y->src);
}

int orc_upper_to_full_bcsr(int nb, int nblocks, const int* rows, const int* cols,
                           const double* vals9, int* rowptr, int* colidx, double* full_vals9)
{
  int* cnt = (int*)calloc((size_t)nb + 1, sizeof(int));
  for (int k = 0; k < nblocks; ++k) {
    cnt[rows[k]]++;
    if (rows[k] != cols[k]) cnt[cols[k]]++;
  }
  rowptr[0] = 0;
  for (int i = 0; i < nb; ++i) rowptr[i + 1] = rowptr[i] + cnt[i];
  const int total = rowptr[nb];
  bcsr_ent* ent = (bcsr_ent*)malloc(sizeof(bcsr_ent) * (size_t)(total > 0 ? total : 1));
  int* fill = (int*)calloc((size_t)nb, sizeof(int));
  for (int k = 0; k < nblocks; ++k) {
    const int i = rows[k], j = cols[k];
    bcsr_ent e = {j, k, 0};
    ent[rowptr[i] + fill[i]++] = e;
    if (i != j) {
      bcsr_ent f = {i, k, 1};
      ent[rowptr[j] + fill[j]++] = f;
    }
  }
  for (int i = 0; i < nb; ++i)
    qsort(ent + rowptr[i], (size_t)(rowptr[i + 1] - rowptr[i]), sizeof(bcsr_ent), cmp_ent);
  for (int t = 0; t < total; ++t) {
    colidx[t] = ent[t].col;
    const double* s = vals9 + 9 * (size_t)ent[t].src;
    double* d = full_vals9 + 9 * (size_t)t;
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) d[r + 3 * c] = ent[t].transpose ? s[c + 3 * r] : s[r + 3 * c];
  }
  free(ent);
  free(fill);
  free(cnt);
  return total;
}

void orc_bcsr_spmv(int nb, const int* rowptr, const int* colidx, const double* vals9,
                   const double* x, double* y)
{
#pragma omp parallel for schedule(static)
  for (int i = 0; i < nb; ++i) {
    double s0 = 0, s1 = 0, s2 = 0;
    for (int t = rowptr[i]; t < rowptr[i + 1]; ++t) {
      const double* B = vals9 + 9 * (size_t)t;
      const double* xj = x + 3 * (size_t)colidx[t];
      s0 += B[0] * xj[0] + B[3] * xj[1] + B[6] * xj[2];
      s1 += B[1] * xj[0] + B[4] * xj[1] + B[7] * xj[2];
      s2 += B[2] * xj[0] + B[5] * xj[1] + B[8] * xj[2];
    }
    y[3 * i] = s0;
    y[3 * i + 1] = s1;
    y[3 * i + 2] = s2;
  }
}

/* ======================================================================= */
/*  MAS32 hierarchy (TraditionalMAS32Preconditioner.cu)                      */
/* ======================================================================= */

struct orc_mas {
  int nv;        /* totalNodes */
  int c0;        /* totalMapNodes */
  int levelnum;
  int node_offset;
  int nlist_size;
  uint32_t *nstart, *nnum_init, *nlist_init, *nnum, *nlist;
  int *pmr, *rmp;
  uint32_t* fine_mask;
  int *prefix_orig, *prefix_sum_orig;
  int* cst; /* coarse space tables, nv*levelnum */
  int* going_next;
  long long gn_cap;
  int level_size[2 * (ORC_MAX_LEVELS + 2)];
  int* coarse_table; /* nv*6 */
  uint32_t *next_mask, *next_prefix, *next_prefix_sum;
  int total_clusters;
  int ndom;
  double* packed64; /* ndom*528*9 */
  float* inv32;     /* ndom*528*9 */
};

int orc_compute_num_levels(int vert_num)
{
  /* computeNumLevels, TraditionalMAS32Preconditioner.cu:2142-2161 */
  int n_level = 1;
  int level_sz = ceil32(vert_num);
  while (level_sz > BANK) {
    level_sz /= BANK;
    n_level++;
    level_sz = ceil32(level_sz);
  }
  n_level = n_level + 1;
  return n_level > 6 ? 6 : n_level;
}

long long orc_hierarchy_capacity(long long vertices, long long mapped, long long levels, long long bank)
{
  /* gipc/hierarchy_capacity.h:10-22 */
  const long long base = vertices > mapped ? vertices : mapped;
  if (!base || !levels) return 0;
  const long long maximum = (long long)(((unsigned long long)-1 >> 1) / sizeof(unsigned int));
  if (!bank || base > maximum || bank - 1 > maximum - base) return -1;
  const long long padded = (base + bank - 1) / bank * bank;
  if (padded > maximum / levels) return -1;
  return padded * levels;
}

orc_mas* orc_mas_create(int vert_num, int collision_node_offset, const uint32_t* neighbor_start,
                        const uint32_t* neighbor_num, const uint32_t* neighbor_list,
                        int neighbor_list_size, const int* part_map_real, int part_map_size,
                        const int* real_map_part)
{
  if (vert_num < 1 || part_map_size < vert_num || part_map_size % BANK) return NULL;
  orc_mas* m = (orc_mas*)calloc(1, sizeof(orc_mas));
  m->nv = vert_num;
  m->c0 = part_map_size;
  m->node_offset = collision_node_offset;
  m->levelnum = orc_compute_num_levels(part_map_size > vert_num ? part_map_size : vert_num);
  m->nlist_size = neighbor_list_size;
  const size_t nv = (size_t)vert_num;
  m->nstart = (uint32_t*)malloc(nv * 4);
  m->nnum_init = (uint32_t*)malloc(nv * 4);
  m->nnum = (uint32_t*)malloc(nv * 4);
  m->nlist_init = (uint32_t*)malloc((size_t)(neighbor_list_size > 0 ? neighbor_list_size : 1) * 4);
  m->nlist = (uint32_t*)malloc((size_t)(neighbor_list_size > 0 ? neighbor_list_size : 1) * 4);
  memcpy(m->nstart, neighbor_start, nv * 4);
  memcpy(m->nnum_init, neighbor_num, nv * 4);
  if (neighbor_list_size > 0) memcpy(m->nlist_init, neighbor_list, (size_t)neighbor_list_size * 4);
  m->pmr = (int*)malloc((size_t)part_map_size * 4);
  m->rmp = (int*)malloc(nv * 4);
  memcpy(m->pmr, part_map_real, (size_t)part_map_size * 4);
  memcpy(m->rmp, real_map_part, nv * 4);
  m->fine_mask = (uint32_t*)calloc(nv, 4);
  const size_t banks0 = (size_t)part_map_size / BANK;
  m->prefix_orig = (int*)calloc(banks0 + 1, 4);
  m->prefix_sum_orig = (int*)calloc(banks0 + 1, 4);
  m->cst = (int*)malloc(nv * (size_t)m->levelnum * 4);
  m->gn_cap = orc_hierarchy_capacity(vert_num, part_map_size, m->levelnum, BANK);
  m->going_next = (int*)malloc((size_t)m->gn_cap * 4);
  memset(m->going_next, 0xff, (size_t)m->gn_cap * 4);
  m->coarse_table = (int*)malloc(nv * 6 * 4);
  memset(m->coarse_table, 0xff, nv * 6 * 4);
  m->next_mask = (uint32_t*)calloc(nv, 4);
  m->next_prefix = (uint32_t*)calloc(nv / BANK + 2, 4);
  m->next_prefix_sum = (uint32_t*)calloc(nv / BANK + 2, 4);
  return m;
}

void orc_mas_free(orc_mas* m)
{
  if (!m) return;
  free(m->nstart); free(m->nnum_init); free(m->nnum); free(m->nlist_init); free(m->nlist);
  free(m->pmr); free(m->rmp); free(m->fine_mask); free(m->prefix_orig); free(m->prefix_sum_orig);
  free(m->cst); free(m->going_next); free(m->coarse_table); free(m->next_mask);
  free(m->next_prefix); free(m->next_prefix_sum); free(m->packed64); free(m->inv32);
  free(m);
}

int orc_mas_levelnum(const orc_mas* m) { return m->levelnum; }
long long orc_mas_going_next_capacity(const orc_mas* m) { return m->gn_cap; }
int orc_mas_total_clusters(const orc_mas* m) { return m->total_clusters; }

/* _buildCML0_new (:463-...) */
static void build_cml0(orc_mas* m)
{
  for (int tdx = 0; tdx < m->c0; ++tdx) {
    const int bank = tdx / BANK, lane = tdx % BANK;
    const int idx = m->pmr[tdx];
    if (idx < 0) continue;
    uint32_t mask = 1u << lane;
    uint32_t nk = 0;
    const uint32_t st = m->nstart[idx];
    for (uint32_t i = 0; i < m->nnum[idx]; ++i) {
      const uint32_t v = m->nlist[st + i];
      const int pv = m->rmp[v];
      if (pv / BANK == bank)
        mask |= 1u << (uint32_t)(pv % BANK);
      else
        m->nlist[st + nk++] = v;
    }
    m->nnum[idx] = nk;
    m->fine_mask[idx] = mask;
  }
}

/* int4 contact decoding of _buildCollisionConnection_new (:1550-1962). */
static int decode_pair(const int* p, int* v)
{
  int x = p[0], y = p[1], z = p[2], w = p[3];
  int cnt;
  if (x >= 0) {
    if (w < 0) w = -w - 1;
    cnt = 4;
  } else {
    x = -x - 1;
    if (z < 0) {
      if (y < 0) {
        y = -y - 1;
        z = -z - 1;
        w = -w - 1;
        cnt = 4;
      } else {
        cnt = 2;
      }
    } else if (w < 0) {
      if (y < 0) {
        y = -y - 1;
        w = -w - 1;
        cnt = 4;
      } else {
        cnt = 3;
      }
    } else {
      cnt = 4;
    }
  }
  v[0] = x; v[1] = y; v[2] = z; v[3] = w;
  return cnt;
}

static void collision_connection(orc_mas* m, uint32_t* connect, const int* cst_level_base,
                                 const int* pairs4, int cp_num)
{
  for (int p = 0; p < cp_num; ++p) {
    int v[4];
    const int cnt = decode_pair(pairs4 + 4 * (size_t)p, v);
    int cp[4];
    for (int i = 0; i < cnt; ++i) {
      v[i] -= m->node_offset;
      /* an index past the FEM range is undefined in the reference; treated as absent */
      if (v[i] >= m->nv) v[i] = -1;
      if (v[i] >= 0)
        cp[i] = cst_level_base ? cst_level_base[v[i]] : m->rmp[v[i]];
      else
        cp[i] = -1;
    }
    uint32_t conn[4] = {0, 0, 0, 0};
    for (int i = 0; i < cnt; ++i)
      for (int j = i + 1; j < cnt; ++j) {
        const uint32_t my = (uint32_t)cp[i], ot = (uint32_t)cp[j];
        if (my == ot) continue;
        if (my / BANK == ot / BANK) {
          conn[i] |= 1u << (ot % BANK);
          conn[j] |= 1u << (my % BANK);
        }
      }
    if (cst_level_base) {
      for (int i = 0; i < cnt; ++i)
        if (cp[i] >= 0) connect[cp[i]] |= conn[i];
    } else {
      for (int i = 0; i < cnt; ++i)
        if (v[i] >= 0) connect[v[i]] |= conn[i];
    }
  }
}

/* _preparePrefixSumL0_new (:560-...) */
static void prepare_prefix_sum_l0(orc_mas* m)
{
  const int banks = m->c0 / BANK;
  for (int b = 0; b < banks; ++b) {
    uint32_t cache[BANK];
    int idxs[BANK];
    for (int lane = 0; lane < BANK; ++lane) {
      idxs[lane] = m->pmr[b * BANK + lane];
      cache[lane] = idxs[lane] >= 0 ? m->fine_mask[idxs[lane]] : 0u;
    }
    int count = 0;
    for (int lane = 0; lane < BANK; ++lane) {
      if (idxs[lane] < 0) continue;
      uint32_t mask = cache[lane];
      uint32_t visited = 1u << lane;
      while (mask != 0xffffffffu) {
        const uint32_t todo = visited ^ mask;
        if (!todo) break;
        const int nxt = ffs32(todo) - 1;
        visited |= 1u << nxt;
        mask |= cache[nxt];
      }
      m->fine_mask[idxs[lane]] = mask;
      if (popc32(mask & lanemask_lt(lane)) == 0) count++;
    }
    if (idxs[0] >= 0) m->prefix_orig[b] = count;
  }
}

/* _buildLevel1_new (:681-744) with the thrust exclusive scan of BuildLevel1 */
static void build_level1(orc_mas* m)
{
  const int number = m->c0;
  const int warps = (number + BANK - 1) / BANK;
  int acc = 0;
  for (int b = 0; b < warps; ++b) {
    m->prefix_sum_orig[b] = acc;
    acc += m->prefix_orig[b];
  }
  m->level_size[2] = m->prefix_sum_orig[warps - 1] + m->prefix_orig[warps - 1];
  m->level_size[3] = ceil32(number);
  for (int b = 0; b < warps; ++b) {
    uint32_t elected = 0;
    int idxs[BANK];
    int lane_prefix[BANK];
    for (int lane = 0; lane < BANK; ++lane) {
      const int tdx = b * BANK + lane;
      idxs[lane] = tdx < number ? m->pmr[tdx] : -1;
      if (idxs[lane] >= 0 && popc32(m->fine_mask[idxs[lane]] & lanemask_lt(lane)) == 0)
        elected |= 1u << lane;
    }
    for (int lane = 0; lane < BANK; ++lane)
      if (idxs[lane] >= 0) lane_prefix[lane] = popc32(elected & lanemask_lt(lane)) + m->prefix_sum_orig[b];
    for (int lane = 0; lane < BANK; ++lane) {
      const int idx = idxs[lane];
      if (idx < 0) continue;
      const int el = ffs32(m->fine_mask[idx]) - 1;
      const int coarse = lane_prefix[el];
      m->cst[idx] = coarse;
      m->going_next[idx] = coarse + ceil32(number);
    }
  }
}

/* _buildConnectMaskLx_new (:821-903) */
static void build_connect_mask_lx(orc_mas* m, int level)
{
  const int banks = m->c0 / BANK;
  const int* prev = m->cst + (size_t)(level - 1) * m->nv;
  for (int b = 0; b < banks; ++b) {
    uint32_t cache[BANK], conn[BANK];
    int ci[BANK], idxs[BANK];
    for (int lane = 0; lane < BANK; ++lane) {
      const int idx = m->pmr[b * BANK + lane];
      idxs[lane] = idx;
      if (idx < 0) continue;
      const uint32_t coarse = (uint32_t)prev[idx];
      uint32_t c = 0, nk = 0;
      const uint32_t st = m->nstart[idx];
      for (uint32_t i = 0; i < m->nnum[idx]; ++i) {
        const uint32_t u = m->nlist[st + i];
        const uint32_t cc = (uint32_t)prev[u];
        if (coarse / BANK == cc / BANK)
          c |= 1u << (cc % BANK);
        else
          m->nlist[st + nk++] = u;
      }
      m->nnum[idx] = nk;
      conn[lane] = c;
      cache[lane] = 0;
    }
    for (int lane = 0; lane < BANK; ++lane) {
      const int idx = idxs[lane];
      if (idx < 0) continue;
      const uint32_t prefix = m->fine_mask[idx];
      if (popc32(prefix) == BANK) {
        cache[0] |= conn[lane];
        ci[lane] = 0;
      } else {
        const int e = ffs32(prefix) - 1;
        if (conn[lane]) cache[e] |= conn[lane];
        ci[lane] = e;
      }
    }
    for (int lane = 0; lane < BANK; ++lane) {
      const int idx = idxs[lane];
      if (idx < 0) continue;
      const uint32_t cm = cache[ci[lane]];
      if (cm && popc32(m->fine_mask[idx] & lanemask_lt(lane)) == 0) m->next_mask[prev[idx]] |= cm;
    }
  }
}

/* _nextLevelCluster (:905-956) */
static void next_level_cluster(orc_mas* m, int number)
{
  const int banks = (number + BANK - 1) / BANK;
  for (int b = 0; b < banks; ++b) {
    uint32_t cache[BANK];
    const int lanes = (number - b * BANK) < BANK ? (number - b * BANK) : BANK;
    for (int lane = 0; lane < lanes; ++lane) cache[lane] = (1u << lane) | m->next_mask[b * BANK + lane];
    int count = 0;
    for (int lane = 0; lane < lanes; ++lane) {
      uint32_t mask = cache[lane];
      uint32_t visited = 1u << lane;
      for (;;) {
        const uint32_t todo = visited ^ mask;
        if (!todo) break;
        const int nxt = ffs32(todo) - 1;
        visited |= 1u << nxt;
        mask |= cache[nxt];
      }
      m->next_mask[b * BANK + lane] = mask;
      if (popc32(mask & lanemask_lt(lane)) == 0) count++;
    }
    m->next_prefix[b] = (uint32_t)count;
  }
}

/* _prefixSumLx (:958-1009) with the thrust exclusive scan of PrefixSumLx */
static void prefix_sum_lx(orc_mas* m, int level, int level_begin, int number)
{
  const int banks = (number + BANK - 1) / BANK;
  uint32_t acc = 0;
  for (int b = 0; b < banks; ++b) {
    m->next_prefix_sum[b] = acc;
    acc += m->next_prefix[b];
  }
  m->level_size[2 * (level + 1)] = (int)(m->next_prefix_sum[banks - 1] + m->next_prefix[banks - 1]);
  m->level_size[2 * (level + 1) + 1] = level_begin + ceil32(number);
  for (int b = 0; b < banks; ++b) {
    const int lanes = (number - b * BANK) < BANK ? (number - b * BANK) : BANK;
    uint32_t elected = 0;
    uint32_t lane_prefix[BANK], out[BANK];
    for (int lane = 0; lane < lanes; ++lane)
      if (popc32(m->next_mask[b * BANK + lane] & lanemask_lt(lane)) == 0) elected |= 1u << lane;
    for (int lane = 0; lane < lanes; ++lane)
      lane_prefix[lane] = (uint32_t)popc32(elected & lanemask_lt(lane)) + m->next_prefix_sum[b];
    for (int lane = 0; lane < lanes; ++lane) {
      const int idx = b * BANK + lane;
      const int el = ffs32(m->next_mask[idx]) - 1;
      out[lane] = lane_prefix[el];
      m->going_next[idx + level_begin] = (int)out[lane] + level_begin + ceil32(number);
    }
    for (int lane = 0; lane < lanes; ++lane) m->next_mask[b * BANK + lane] = out[lane];
  }
}

int orc_mas_reorder(orc_mas* m, const int* pairs4, int cp_num)
{
  memcpy(m->nlist, m->nlist_init, (size_t)(m->nlist_size > 0 ? m->nlist_size : 0) * 4);
  memcpy(m->nnum, m->nnum_init, (size_t)m->nv * 4);
  memset(m->level_size, 0, sizeof(int) * 2 * (size_t)m->levelnum);

  build_cml0(m);
  if (cp_num) collision_connection(m, m->fine_mask, NULL, pairs4, cp_num);
  prepare_prefix_sum_l0(m);
  build_level1(m);
  for (int level = 1; level < m->levelnum; ++level) {
    memset(m->next_mask, 0, (size_t)m->nv * 4);
    build_connect_mask_lx(m, level);
    if (cp_num) collision_connection(m, m->next_mask, m->cst + (size_t)(level - 1) * m->nv, pairs4, cp_num);
    const int count = m->level_size[2 * level];
    const int begin = m->level_size[2 * level + 1];
    if (count >= 1) {
      next_level_cluster(m, count);
      prefix_sum_lx(m, level, begin, count);
    }
    /* _computeNextLevel (:1011-1022) */
    for (int idx = 0; idx < m->nv; ++idx)
      m->cst[(size_t)level * m->nv + idx] = (int)m->next_mask[m->cst[(size_t)(level - 1) * m->nv + idx]];
  }
  m->total_clusters = m->level_size[2 * m->levelnum + 1];
  /* _aggregationKernel (:1024-1058) */
  for (int idx = 0; idx < m->nv; ++idx) {
    int cur = idx;
    for (int l = 0; l < m->levelnum - 1; ++l) {
      cur = m->going_next[cur];
      m->coarse_table[(size_t)idx * 6 + l] = cur;
    }
  }
  return m->total_clusters;
}

void orc_mas_get_hierarchy(const orc_mas* m, uint32_t* fine_mask, int* coarse_space_tables,
                           int* going_next, int* level_size, int* coarse_table, int* prefix_original)
{
  const size_t nv = (size_t)m->nv;
  if (fine_mask) memcpy(fine_mask, m->fine_mask, nv * 4);
  if (coarse_space_tables) memcpy(coarse_space_tables, m->cst, nv * (size_t)m->levelnum * 4);
  if (going_next) memcpy(going_next, m->going_next, (size_t)m->gn_cap * 4);
  if (level_size) memcpy(level_size, m->level_size, sizeof(int) * 2 * (size_t)(m->levelnum + 1));
  if (coarse_table) memcpy(coarse_table, m->coarse_table, nv * 6 * 4);
  if (prefix_original) memcpy(prefix_original, m->prefix_orig, (size_t)(m->c0 / BANK) * 4);
}

/* ======================================================================= */
/*  MAS32 domain matrices, Gauss-Jordan inverse, apply                        */
/* ======================================================================= */

static inline double* blk64(orc_mas* m, int dom, int b) { return m->packed64 + ((size_t)dom * NPACK + b) * 9; }

/* full-view block (r,c) of a level-0 packed domain: transpose of (c,r) below the diagonal */
static void full_block(const double* dom_base, int r, int c, double* out)
{
  if (c >= r) {
    memcpy(out, dom_base + (size_t)pk(r, c) * 9, 9 * sizeof(double));
  } else {
    const double* s = dom_base + (size_t)pk(c, r) * 9;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) out[i + 3 * j] = s[j + 3 * i];
  }
}

void orc_mas_prepare_hessian(orc_mas* m, const double* vals9, const int* rows, const int* cols,
                             const uint32_t* indices, int offset, int triplet_num)
{
  const int levels = m->levelnum;
  m->ndom = m->total_clusters / BANK;
  free(m->packed64);
  free(m->inv32);
  m->packed64 = (double*)calloc((size_t)m->ndom * NPACK * 9, sizeof(double));
  m->inv32 = (float*)calloc((size_t)m->ndom * NPACK * 9, sizeof(float));
  const int* gn = m->going_next;

  /* prepare_hessian_bcoo_kernel (:2234-2338) */
  for (int I = 0; I < triplet_num; ++I) {
    const int index = indices ? (int)indices[I] : I;
    const int vr_real = rows[index] - offset;
    const int vc_real = cols[index] - offset;
    const double* H = vals9 + 9 * (size_t)index;
    int vc = m->rmp[vc_real];
    int vr = m->rmp[vr_real];
    int cp = vc / BANK;
    if (vc / BANK == vr / BANK) {
      const int a = vr % BANK, b = vc % BANK;
      if (vc >= vr) {
        memcpy(blk64(m, cp, pk(a, b)), H, 9 * sizeof(double));
      } else {
#if ORC_BANK == 16
        /* CEMAS16 keeps an in-bank block only when its slots follow its
         * vertex order (MASPreconditioner.cu:1846-1857): dropped */
#else
        double* d = blk64(m, cp, pk(b, a));
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j) d[i + 3 * j] = H[j + 3 * i];
#endif
      }
    } else {
      for (int level = 1; level < levels; ++level) {
        if (level == 1) {
          vc = gn[vc_real];
          vr = gn[vr_real];
        } else {
          vc = gn[vc];
          vr = gn[vr];
        }
        cp = vc / BANK;
        if (vc / BANK != vr / BANK) continue;
        if (vc >= vr) {
          double* d = blk64(m, cp, pk(vr % BANK, vc % BANK));
          for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
              d[i + 3 * j] += H[i + 3 * j];
              if (vc == vr) d[i + 3 * j] += H[j + 3 * i];
            }
        } else {
          double* d = blk64(m, cp, pk(vc % BANK, vr % BANK));
          for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) d[i + 3 * j] += H[j + 3 * i];
        }
      }
    }
  }

  /* prepare_hessian_bcoo_sum_kernel (:2340-2464): Galerkin sums of the
   * level-0 domains into the coarse levels. */
  const int banks0 = m->c0 / BANK;
  for (int hid = 0; hid < banks0; ++hid) {
    const double* base = m->packed64 + (size_t)hid * NPACK * 9;
    const int prefix = m->prefix_orig[hid];
    for (int lr = 0; lr < BANK; ++lr) {
      const int rdx0 = m->pmr[hid * BANK + lr];
      if (rdx0 < 0) continue;
      if (prefix == 1) {
        if (m->pmr[hid * BANK] < 0) continue; /* lane 0 carries the row sum */
#if ORC_BANK == 16
        /* CEMAS16: a warp of 32 entries spans rows (2k, 2k+1) and its sum is
         * added by entry (2k, 0) (MASPreconditioner.cu:1955-2005) */
        if (m->pmr[hid * BANK + (lr & ~1)] < 0) continue;
#endif
        double mat[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, b9[9];
        for (int lc = 0; lc < BANK; ++lc) {
          if (m->pmr[hid * BANK + lc] < 0) continue;
          full_block(base, lr, lc, b9);
          for (int e = 0; e < 9; ++e) mat[e] += b9[e];
        }
        int next = gn[rdx0];
        for (int level = 1; level < levels; ++level) {
          double* d = blk64(m, next / BANK, pk(next % BANK, next % BANK));
          for (int e = 0; e < 9; ++e) d[e] += mat[e];
          next = gn[next];
        }
      } else {
        for (int lc = 0; lc < BANK; ++lc) {
          const int cdx0 = m->pmr[hid * BANK + lc];
          if (cdx0 < 0) continue;
          double b9[9];
          full_block(base, lr, lc, b9);
          int rdx = rdx0, cdx = cdx0;
          for (int level = 1; level < levels; ++level) {
            rdx = gn[rdx];
            cdx = gn[cdx];
            if (rdx / BANK == cdx / BANK && cdx >= rdx) {
              double* d = blk64(m, cdx / BANK, pk(rdx % BANK, cdx % BANK));
              for (int e = 0; e < 9; ++e) d[e] += b9[e];
            }
          }
        }
      }
    }
  }

  /* expand_symmetric_mas32 (:1062-1096) + __inverse6_P96x96 (:1099-1146).
   * The update is written as fma() because nvcc contracts the reference's
   * "m[k][i] += rate * m[j][i]" into a fused multiply-add. */
#pragma omp parallel
  {
    double* a = (double*)malloc(sizeof(double) * DIM * DIM);
    double col[DIM];
#pragma omp for schedule(dynamic, 4)
    for (int d = 0; d < m->ndom; ++d) {
      const double* P = m->packed64 + (size_t)d * NPACK * 9;
      for (int r = 0; r < DIM; ++r) {
        for (int c = 0; c < DIM; ++c) {
          const int br = r / 3, bc = c / 3;
          a[r * DIM + c] = (bc >= br) ? P[(size_t)pk(br, bc) * 9 + (r % 3) + 3 * (c % 3)]
                                      : P[(size_t)pk(bc, br) * 9 + (c % 3) + 3 * (r % 3)];
        }
        if (a[r * DIM + r] == 0.0) a[r * DIM + r] = 1.0;
      }
      for (int j = 0; j < DIM; ++j) {
        const double pivot = a[j * DIM + j];
        for (int i = 0; i < DIM; ++i) col[i] = a[i * DIM + j];
        for (int i = 0; i < DIM; ++i) a[i * DIM + j] = (i == j) ? 1.0 : 0.0;
        for (int i = 0; i < DIM; ++i) a[j * DIM + i] /= pivot;
        for (int k = 0; k < DIM; ++k) {
          if (k == j) continue;
          const double rate = -col[k];
          for (int i = 0; i < DIM; ++i) a[k * DIM + i] = fma(rate, a[j * DIM + i], a[k * DIM + i]);
        }
      }
#if ORC_BANK == 16
      /* CEMAS16 copies the upper elements of each diagonal 3x3 block onto
       * the lower ones before the store (MASPreconditioner.cu:705-711) */
      for (int i = 0; i < DIM; ++i) {
        if (i % 3 < 2)
          a[(i + 1) * DIM + i] = a[i * DIM + i + 1];
        else
          a[i * DIM + i - 2] = a[(i - 2) * DIM + i];
      }
#endif
      float* out = m->inv32 + (size_t)d * NPACK * 9;
      for (int r = 0; r < DIM; ++r)
        for (int c = 0; c < DIM; ++c) {
          const int br = r / 3, bc = c / 3;
          if (bc >= br) out[(size_t)pk(br, bc) * 9 + (r % 3) + 3 * (c % 3)] = (float)a[r * DIM + c];
        }
    }
    free(a);
  }
}

void orc_mas_get_domains(const orc_mas* m, double* packed64, float* inverse32)
{
  const size_t n = (size_t)m->ndom * NPACK * 9;
  if (packed64 && m->packed64) memcpy(packed64, m->packed64, n * sizeof(double));
  if (inverse32 && m->inv32) memcpy(inverse32, m->inv32, n * sizeof(float));
}

void orc_mas_set_inverses(orc_mas* m, const float* inverse32)
{
  if (m->inv32 && inverse32) memcpy(m->inv32, inverse32, (size_t)m->ndom * NPACK * 9 * sizeof(float));
}

/* preconditioning (:2684-2725) = __buildMultiLevelR_optimized_new (:1149-1266)
 * + _schwarzLocalXSym6 (:1375-1462) + __collectFinalZ_new (:1268-1299).
 * FP32 inside, FP64 at the edges, fixed summation order. */
void orc_mas_precondition(const orc_mas* m, const double* R, double* Z)
{
  const int total = m->total_clusters;
  float* mr = (float*)calloc((size_t)total * 3, sizeof(float));
  float* mz = (float*)calloc((size_t)total * 3, sizeof(float));
  const int* gn = m->going_next;
  for (int t = 0; t < m->c0; ++t) {
    const int idx = m->pmr[t];
    if (idx < 0) continue;
    const float r0 = (float)R[3 * (size_t)idx], r1 = (float)R[3 * (size_t)idx + 1], r2 = (float)R[3 * (size_t)idx + 2];
    mr[3 * (size_t)t] = r0;
    mr[3 * (size_t)t + 1] = r1;
    mr[3 * (size_t)t + 2] = r2;
    int cur = idx;
    for (int level = 1; level < m->levelnum; ++level) {
      cur = gn[cur];
      mr[3 * (size_t)cur] += r0;
      mr[3 * (size_t)cur + 1] += r1;
      mr[3 * (size_t)cur + 2] += r2;
    }
  }
#pragma omp parallel for schedule(static)
  for (int d = 0; d < m->ndom; ++d) {
    const float* P = m->inv32 + (size_t)d * NPACK * 9;
    for (int lr = 0; lr < BANK; ++lr) {
      float z0 = 0.f, z1 = 0.f, z2 = 0.f;
      for (int lc = 0; lc < BANK; ++lc) {
        const float* x = mr + 3 * ((size_t)d * BANK + lc);
        if (lc >= lr) {
          const float* B = P + (size_t)pk(lr, lc) * 9;
          z0 += B[0] * x[0] + B[3] * x[1] + B[6] * x[2];
          z1 += B[1] * x[0] + B[4] * x[1] + B[7] * x[2];
          z2 += B[2] * x[0] + B[5] * x[1] + B[8] * x[2];
        } else {
          const float* B = P + (size_t)pk(lc, lr) * 9;
          z0 += B[0] * x[0] + B[1] * x[1] + B[2] * x[2];
          z1 += B[3] * x[0] + B[4] * x[1] + B[5] * x[2];
          z2 += B[6] * x[0] + B[7] * x[1] + B[8] * x[2];
        }
      }
      float* z = mz + 3 * ((size_t)d * BANK + lr);
      z[0] = z0;
      z[1] = z1;
      z[2] = z2;
    }
  }
#pragma omp parallel for schedule(static)
  for (int idx = 0; idx < m->nv; ++idx) {
    const int rdx = m->rmp[idx];
    float c0 = mz[3 * (size_t)rdx], c1 = mz[3 * (size_t)rdx + 1], c2 = mz[3 * (size_t)rdx + 2];
    for (int l = 1; l < m->levelnum; ++l) {
      const int now = m->coarse_table[(size_t)idx * 6 + l - 1];
      c0 += mz[3 * (size_t)now];
      c1 += mz[3 * (size_t)now + 1];
      c2 += mz[3 * (size_t)now + 2];
    }
    Z[3 * (size_t)idx] = c0;
    Z[3 * (size_t)idx + 1] = c1;
    Z[3 * (size_t)idx + 2] = c2;
  }
  free(mr);
  free(mz);
}

/* check_local_matrices (:76-147) */
static double packed_scalar64(const double* P, int row, int col)
{
  int br = row / 3, bc = col / 3, rr = row % 3, cc = col % 3;
  if (br > bc) {
    int t = br; br = bc; bc = t;
    t = rr; rr = cc; cc = t;
  }
  return P[(size_t)pk(br, bc) * 9 + rr + 3 * cc];
}
static double packed_scalar32(const float* P, int row, int col)
{
  int br = row / 3, bc = col / 3, rr = row % 3, cc = col % 3;
  if (br > bc) {
    int t = br; br = bc; bc = t;
    t = rr; rr = cc; cc = t;
  }
  return (double)P[(size_t)pk(br, bc) * 9 + rr + 3 * cc];
}
static int cholesky_check(double* w)
{
  for (int k = 0; k < DIM; ++k) {
    const double pivot = w[k * DIM + k];
    if (!isfinite(pivot) || pivot <= 0) return 0;
    w[k * DIM + k] = sqrt(pivot);
    for (int r = k + 1; r < DIM; ++r) w[r * DIM + k] /= w[k * DIM + k];
    for (int r = k + 1; r < DIM; ++r)
      for (int c = k + 1; c <= r; ++c) w[r * DIM + c] -= w[r * DIM + k] * w[c * DIM + k];
  }
  return 1;
}

void orc_local_checks(int count, const double* packed64, const float* inverse32, double* res)
{
#pragma omp parallel
  {
    double* w = (double*)malloc(sizeof(double) * DIM * DIM);
    double* a = (double*)malloc(sizeof(double) * DIM * DIM);
#pragma omp for schedule(dynamic, 1)
    for (int d = 0; d < count; ++d) {
      const double* L = packed64 + (size_t)d * NPACK * 9;
      const float* B = inverse32 + (size_t)d * NPACK * 9;
      int fin0 = 1, fin1 = 1;
      double min_a = INFINITY, min_b = INFINITY;
      for (int i = 0; i < DIM * DIM; ++i) {
        const int r = i / DIM, c = i % DIM;
        double av = packed_scalar64(L, r, c);
        const double bv = packed_scalar32(B, r, c);
        if (r == c && av == 0) av = 1;
        if (!isfinite(av)) fin0 = 0;
        if (!isfinite(bv)) fin1 = 0;
        a[i] = av;
        if (r == c) {
          min_a = fmin(min_a, av);
          min_b = fmin(min_b, bv);
        }
      }
      int pos0 = fin0, pos1 = fin1;
      if (fin0) {
        memcpy(w, a, sizeof(double) * DIM * DIM);
        pos0 = cholesky_check(w);
      }
      double resid = 0;
      if (fin0 && fin1) {
        double s = 0;
        for (int r = 0; r < DIM; ++r)
          for (int c = 0; c < DIM; ++c) {
            double p = 0;
            for (int k = 0; k < DIM; ++k) p += a[r * DIM + k] * packed_scalar32(B, k, c);
            const double e = p - (r == c ? 1.0 : 0.0);
            s += e * e;
          }
        resid = sqrt(s / DIM);
      }
      if (fin1 && !(pos0 && resid <= 1e-3)) {
        for (int i = 0; i < DIM * DIM; ++i) w[i] = packed_scalar32(B, i / DIM, i % DIM);
        pos1 = cholesky_check(w);
      }
      double* o = res + 7 * (size_t)d;
      o[0] = fin0; o[1] = fin1; o[2] = pos0; o[3] = pos1; o[4] = min_a; o[5] = min_b; o[6] = resid;
    }
    free(w);
    free(a);
  }
}

/* ======================================================================= */
/*  Block-Jacobi inverses                                                    */
/* ======================================================================= */

static int invert_dense(int n, const double* A, double* out)
{
  /* Gauss-Jordan with partial pivoting (row-major). */
  double* a = (double*)malloc(sizeof(double) * (size_t)n * 2 * n);
  for (int r = 0; r < n; ++r)
    for (int c = 0; c < 2 * n; ++c) a[r * 2 * n + c] = c < n ? A[r * n + c] : (c - n == r ? 1.0 : 0.0);
  for (int k = 0; k < n; ++k) {
    int piv = k;
    for (int r = k + 1; r < n; ++r)
      if (fabs(a[r * 2 * n + k]) > fabs(a[piv * 2 * n + k])) piv = r;
    if (a[piv * 2 * n + k] == 0.0) {
      free(a);
      return 0;
    }
    if (piv != k)
      for (int c = 0; c < 2 * n; ++c) {
        const double t = a[k * 2 * n + c];
        a[k * 2 * n + c] = a[piv * 2 * n + c];
        a[piv * 2 * n + c] = t;
      }
    const double inv = 1.0 / a[k * 2 * n + k];
    for (int c = 0; c < 2 * n; ++c) a[k * 2 * n + c] *= inv;
    for (int r = 0; r < n; ++r) {
      if (r == k) continue;
      const double f = a[r * 2 * n + k];
      if (f == 0.0) continue;
      for (int c = 0; c < 2 * n; ++c) a[r * 2 * n + c] -= f * a[k * 2 * n + c];
    }
  }
  for (int r = 0; r < n; ++r)
    for (int c = 0; c < n; ++c) out[r * n + c] = a[r * 2 * n + n + c];
  free(a);
  return 1;
}

void orc_diag3_inverse(int nb, int nblocks, const int* rows, const int* cols, const double* vals9,
                       double* inv9)
{
  for (int i = 0; i < nb; ++i)
    for (int e = 0; e < 9; ++e) inv9[9 * (size_t)i + e] = (e % 4 == 0) ? 1.0 : 0.0;
  for (int k = 0; k < nblocks; ++k) {
    if (rows[k] != cols[k]) continue;
    const double* H = vals9 + 9 * (size_t)k;
    /* cofactor inverse of a 3x3 (column-major in and out) */
    const double a = H[0], b = H[3], c = H[6], d = H[1], e = H[4], f = H[7], g = H[2], h = H[5], i = H[8];
    const double A = e * i - f * h, B = -(d * i - f * g), C = d * h - e * g;
    const double det = a * A + b * B + c * C;
    const double inv = 1.0 / det;
    double* o = inv9 + 9 * (size_t)rows[k];
    o[0] = A * inv; o[3] = -(b * i - c * h) * inv; o[6] = (b * f - c * e) * inv;
    o[1] = B * inv; o[4] = (a * i - c * g) * inv;  o[7] = -(a * f - c * d) * inv;
    o[2] = C * inv; o[5] = -(a * h - b * g) * inv; o[8] = (a * e - b * d) * inv;
  }
}

int orc_abd_inverse(int bodies, int nblocks, const int* rows, const int* cols, const double* vals9,
                    double* inv144)
{
  double* P = (double*)calloc((size_t)bodies * 144, sizeof(double));
  for (int k = 0; k < nblocks; ++k) {
    const int r = rows[k], c = cols[k];
    if (r >= 4 * bodies || c >= 4 * bodies || r / 4 != c / 4) continue;
    const double* H = vals9 + 9 * (size_t)k;
    double* B = P + (size_t)(r / 4) * 144;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        B[((r % 4) * 3 + i) * 12 + (c % 4) * 3 + j] = H[i + 3 * j];
        if (r != c) B[((c % 4) * 3 + i) * 12 + (r % 4) * 3 + j] = H[j + 3 * i];
      }
  }
  int ok = 1;
  for (int bdy = 0; bdy < bodies; ++bdy) ok &= invert_dense(12, P + (size_t)bdy * 144, inv144 + (size_t)bdy * 144);
  free(P);
  return ok;
}

/* ======================================================================= */
/*  PCG                                                                      */
/* ======================================================================= */

static double pdot(const double* a, const double* b, int n)
{
  /* fixed chunking, summed in chunk order: deterministic for any thread count */
  enum { CH = 64 };
  double part[CH];
  const int per = (n + CH - 1) / CH;
#pragma omp parallel for schedule(static)
  for (int c = 0; c < CH; ++c) {
    double s = 0;
    const int lo = c * per, hi = (lo + per < n) ? lo + per : n;
    for (int i = lo; i < hi; ++i) s += a[i] * b[i];
    part[c] = s;
  }
  double s = 0;
  for (int c = 0; c < CH; ++c) s += part[c];
  return s;
}

typedef struct {
  const orc_pcg_opts* o;
  const orc_mas* mas;
  double* diag_inv;
  double* abd_inv;
} precond_ctx;

static void apply_precond(const precond_ctx* p, const double* r, double* z, int n)
{
  const orc_pcg_opts* o = p->o;
  if (o->precond == ORC_PRECOND_DIAG3) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < o->nb; ++i) {
      const double* D = p->diag_inv + 9 * (size_t)i;
      const double* x = r + 3 * (size_t)i;
      for (int a = 0; a < 3; ++a) z[3 * (size_t)i + a] = D[a] * x[0] + D[a + 3] * x[1] + D[a + 6] * x[2];
    }
  } else {
    memcpy(z, r, sizeof(double) * (size_t)n);
  }
  if (o->abd_bodies > 0 && o->precond != ORC_PRECOND_NONE) {
#pragma omp parallel for schedule(static)
    for (int bdy = 0; bdy < o->abd_bodies; ++bdy) {
      const double* P = p->abd_inv + 144 * (size_t)bdy;
      for (int a = 0; a < 12; ++a) {
        double s = 0;
        for (int c = 0; c < 12; ++c) s += P[a * 12 + c] * r[12 * (size_t)bdy + c];
        z[12 * (size_t)bdy + a] = s;
      }
    }
  }
  if ((o->precond == ORC_PRECOND_MAS32 || o->precond == ORC_PRECOND_MAS16) && o->fem_count > 0 && p->mas)
    orc_mas_precondition(p->mas, r + 3 * (size_t)o->fem_offset, z + 3 * (size_t)o->fem_offset);
}

int orc_pcg(const orc_pcg_opts* o, const double* vals9, const int* rows, const int* cols, int nblocks,
            const orc_mas* mas, const double* b, double* x, orc_pcg_result* out)
{
  const int nb = o->nb, n = 3 * nb;
  int* rowptr = (int*)malloc(sizeof(int) * ((size_t)nb + 1));
  int* colidx = (int*)malloc(sizeof(int) * (size_t)(2 * nblocks + 1));
  double* fv = (double*)malloc(sizeof(double) * 9 * (size_t)(2 * nblocks + 1));
  orc_upper_to_full_bcsr(nb, nblocks, rows, cols, vals9, rowptr, colidx, fv);
  precond_ctx pc = {o, mas, NULL, NULL};
  if (o->precond == ORC_PRECOND_DIAG3) {
    pc.diag_inv = (double*)malloc(sizeof(double) * 9 * (size_t)nb);
    orc_diag3_inverse(nb, nblocks, rows, cols, vals9, pc.diag_inv);
  }
  if (o->abd_bodies > 0) {
    pc.abd_inv = (double*)malloc(sizeof(double) * 144 * (size_t)o->abd_bodies);
    orc_abd_inverse(o->abd_bodies, nblocks, rows, cols, vals9, pc.abd_inv);
  }
  double* r = (double*)malloc(sizeof(double) * (size_t)n);
  double* z = (double*)malloc(sizeof(double) * (size_t)n);
  double* p = (double*)malloc(sizeof(double) * (size_t)n);
  double* ap = (double*)malloc(sizeof(double) * (size_t)n);
  const int max_iter = o->max_iter > 0 ? o->max_iter : (int)(0.3 * (double)n);
  const int replay = o->replay_checks;

  memset(x, 0, sizeof(double) * (size_t)n);
  memcpy(r, b, sizeof(double) * (size_t)n);
  apply_precond(&pc, r, z, n);
  double rz = pdot(r, z, n);
  memcpy(p, z, sizeof(double) * (size_t)n);
  const double rz0 = rz;
  const double bb = pdot(b, b, n);
  double rr = bb;
  int status = ORC_STATUS_ITERATION_CAP;
  /* PCGSolver: k = 1..max_iter-1 updates, returns max_iter at the cap.
   * Replay harness: at most max_iter updates. */
  const int last = replay ? max_iter : max_iter - 1;
  int k;
  for (k = 1; k <= last; ++k) {
    if (replay && (!isfinite(rz) || rz <= 0)) {
      status = ORC_STATUS_INVALID_RZ;
      k -= 1;
      break;
    }
    orc_bcsr_spmv(nb, rowptr, colidx, fv, p, ap);
    const double pap = pdot(p, ap, n);
    if (replay && (!isfinite(pap) || pap <= 0)) {
      status = ORC_STATUS_NONPOSITIVE_CURVATURE;
      k -= 1;
      break;
    }
    const double alpha = rz / pap;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
      x[i] += alpha * p[i];
      r[i] -= alpha * ap[i];
    }
    rr = pdot(r, r, n);
    if (replay && !isfinite(rr)) {
      status = ORC_STATUS_NONFINITE;
      break;
    }
    if (o->gate == ORC_GATE_RZ) {
      if (fabs(rz) <= o->tol * rz0) {
        status = ORC_STATUS_CONVERGED;
        break;
      }
    } else if (rr <= o->tol * o->tol * bb) {
      status = ORC_STATUS_CONVERGED;
      break;
    }
    apply_precond(&pc, r, z, n);
    const double rz_new = pdot(r, z, n);
    if (replay && (!isfinite(rz_new) || rz_new <= 0 || fabs(rz) < 1e-30)) {
      status = ORC_STATUS_INVALID_RZ;
      break;
    }
    const double beta = rz_new / rz;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
    rz = rz_new;
  }
  if (status == ORC_STATUS_ITERATION_CAP) k = replay ? max_iter : max_iter;
  /* true residual */
  orc_bcsr_spmv(nb, rowptr, colidx, fv, x, ap);
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; ++i) ap[i] = b[i] - ap[i];
  const double tr = pdot(ap, ap, n);
  if (out) {
    out->iterations = k;
    out->status = status;
    out->rz0 = rz0;
    out->rz_last = rz;
    out->rel_res_recursive = bb > 0 ? sqrt(rr / bb) : 0;
    out->rel_res_true = bb > 0 ? sqrt(tr / bb) : sqrt(tr);
  }
  free(r); free(z); free(p); free(ap); free(rowptr); free(colidx); free(fv);
  free(pc.diag_inv); free(pc.abd_inv);
  return k;
}


/* ---- FP64 direct solve: reverse Cuthill-McKee + envelope Cholesky ----
 *
 * Ordering (Cuthill and McKee, 1969, reversed as George, 1971, recommends):
 * per connected component of the block graph, a breadth-first search from a
 * pseudo-peripheral node (George and Liu, 1979: start at a node of minimum
 * degree, move to a minimum-degree node of the last level while the number
 * of levels grows), neighbours visited in increasing degree; the whole order
 * reversed.  The three scalars of a block stay together.
 *
 * Factorisation: row i of L is stored from its first nonzero column f(i) to
 * the diagonal (the envelope of A under the ordering holds all of L's fill),
 * and L_ij = (A_ij - sum_{k >= max(f(i), f(j))} L_ik L_jk) / L_jj row by row.
 */
static int cmp_int(const void* a, const void* b)
{
  const int x = *(const int*)a, y = *(const int*)b;
  return (x > y) - (x < y);
}

/* Breadth-first levels from s over unvisited (mark == 0) nodes; returns the
 * number of levels, fills `order` with the visit order and `last` with the
 * first index of the last level.  Marks are reset before returning. */
static int bfs_levels(int s, const int* ptr, const int* adj, int* mark, int* order, int* count, int* last)
{
  int head = 0, tail = 0, levels = 0;
  order[tail++] = s;
  mark[s] = 1;
  int level_end = tail;
  *last = 0;
  while (head < tail) {
    *last = head;
    for (; head < level_end; ++head) {
      const int u = order[head];
      for (int q = ptr[u]; q < ptr[u + 1]; ++q)
        if (!mark[adj[q]]) {
          mark[adj[q]] = 1;
          order[tail++] = adj[q];
        }
    }
    level_end = tail;
    ++levels;
  }
  for (int q = 0; q < tail; ++q) mark[order[q]] = 0;
  *count = tail;
  return levels;
}

static int rcm_order(int nb, int nblocks, const int* rows, const int* cols, int* perm)
{
  int* deg = (int*)calloc((size_t)nb + 1, sizeof(int));
  int* ptr = (int*)malloc(sizeof(int) * ((size_t)nb + 1));
  if (!deg || !ptr) return -2;
  for (int k = 0; k < nblocks; ++k)
    if (rows[k] != cols[k]) {
      deg[rows[k]]++;
      deg[cols[k]]++;
    }
  ptr[0] = 0;
  for (int i = 0; i < nb; ++i) ptr[i + 1] = ptr[i] + deg[i];
  int* adj = (int*)malloc(sizeof(int) * ((size_t)ptr[nb] + 1));
  int* fill = (int*)calloc((size_t)nb, sizeof(int));
  int* mark = (int*)calloc((size_t)nb, sizeof(int));
  int* order = (int*)malloc(sizeof(int) * ((size_t)nb + 1));
  int* nbr = (int*)malloc(sizeof(int) * ((size_t)nb + 1));
  if (!adj || !fill || !mark || !order || !nbr) return -2;
  for (int k = 0; k < nblocks; ++k)
    if (rows[k] != cols[k]) {
      adj[ptr[rows[k]] + fill[rows[k]]++] = cols[k];
      adj[ptr[cols[k]] + fill[cols[k]]++] = rows[k];
    }
  /* sorted, unique neighbour lists; degree = unique neighbours */
  for (int i = 0; i < nb; ++i) {
    int* a = adj + ptr[i];
    const int n = fill[i];
    qsort(a, (size_t)n, sizeof(int), cmp_int);
    int m = 0;
    for (int q = 0; q < n; ++q)
      if (m == 0 || a[q] != a[m - 1]) a[m++] = a[q];
    deg[i] = m;
  }
  /* compact into ptr/adj with the unique lists */
  {
    int w = 0;
    for (int i = 0; i < nb; ++i) {
      const int s = ptr[i];
      ptr[i] = w;
      for (int q = 0; q < deg[i]; ++q) adj[w++] = adj[s + q];
    }
    ptr[nb] = w;
  }
  int* visited = (int*)calloc((size_t)nb, sizeof(int));
  if (!visited) return -2;
  int out = 0;
  for (;;) {
    /* an unvisited node of minimum degree starts the next component */
    int s = -1;
    for (int i = 0; i < nb; ++i)
      if (!visited[i] && (s < 0 || deg[i] < deg[s])) s = i;
    if (s < 0) break;
    /* pseudo-peripheral node over the component (visited nodes are masked) */
    for (int i = 0; i < nb; ++i) mark[i] = visited[i];
    int count = 0, last = 0;
    int levels = bfs_levels(s, ptr, adj, mark, order, &count, &last);
    for (int it = 0; it < 16; ++it) {
      int best = order[last];
      for (int q = last; q < count; ++q)
        if (deg[order[q]] < deg[best]) best = order[q];
      int c2 = 0, l2 = 0;
      const int lv2 = bfs_levels(best, ptr, adj, mark, order, &c2, &l2);
      if (lv2 <= levels) break;
      s = best;
      levels = lv2;
      count = c2;
      last = l2;
    }
    /* Cuthill-McKee from s: neighbours in increasing degree (then index) */
    int head = out, tail = out;
    perm[tail++] = s;
    visited[s] = 1;
    while (head < tail) {
      const int u = perm[head++];
      int n = 0;
      for (int q = ptr[u]; q < ptr[u + 1]; ++q)
        if (!visited[adj[q]]) {
          visited[adj[q]] = 1;
          nbr[n++] = adj[q];
        }
      for (int a = 1; a < n; ++a) { /* insertion sort by (degree, index) */
        const int v = nbr[a];
        int b = a - 1;
        while (b >= 0 && (deg[nbr[b]] > deg[v] || (deg[nbr[b]] == deg[v] && nbr[b] > v))) {
          nbr[b + 1] = nbr[b];
          --b;
        }
        nbr[b + 1] = v;
      }
      for (int a = 0; a < n; ++a) perm[tail++] = nbr[a];
    }
    out = tail;
  }
  for (int i = 0, j = nb - 1; i < j; ++i, --j) { /* reverse */
    const int t = perm[i];
    perm[i] = perm[j];
    perm[j] = t;
  }
  free(deg);
  free(ptr);
  free(adj);
  free(fill);
  free(mark);
  free(order);
  free(nbr);
  free(visited);
  return 0;
}

int orc_direct_solve(int nb, int nblocks, const int* rows, const int* cols, const double* vals9, const double* b,
                     double* x, long long* envelope_out)
{
  const int n = 3 * nb;
  int* perm = (int*)malloc(sizeof(int) * ((size_t)nb + 1));
  int* inv = (int*)malloc(sizeof(int) * ((size_t)nb + 1));
  int* first = (int*)malloc(sizeof(int) * ((size_t)n + 1));
  long long* off = (long long*)malloc(sizeof(long long) * ((size_t)n + 1));
  if (!perm || !inv || !first || !off) return -2;
  if (rcm_order(nb, nblocks, rows, cols, perm) != 0) return -2;
  for (int k = 0; k < nb; ++k) inv[perm[k]] = k;
  for (int i = 0; i < n; ++i) first[i] = i;
  /* the envelope: first column of every row of the reordered lower triangle */
  for (int k = 0; k < nblocks; ++k) {
    const int pr = inv[rows[k]], pc = inv[cols[k]];
    for (int a = 0; a < 3; ++a)
      for (int c = 0; c < 3; ++c) {
        int i = 3 * pr + a, j = 3 * pc + c;
        if (i < j) {
          const int t = i;
          i = j;
          j = t;
        }
        if (j < first[i]) first[i] = j;
      }
  }
  off[0] = 0;
  for (int i = 0; i < n; ++i) off[i + 1] = off[i] + (i - first[i] + 1);
  double* env = (double*)calloc((size_t)off[n], sizeof(double));
  if (!env) return -2;
  if (envelope_out) *envelope_out = off[n];
  /* scatter A's lower triangle: a diagonal block adds each of its entries
     once at its own position, an off-diagonal block stands for itself and
     its transpose, which meet at one lower position */
  for (int k = 0; k < nblocks; ++k) {
    const int pr = inv[rows[k]], pc = inv[cols[k]];
    const double* v = vals9 + 9 * (size_t)k;
    for (int a = 0; a < 3; ++a)
      for (int c = 0; c < 3; ++c) {
        int i = 3 * pr + a, j = 3 * pc + c;
        if (rows[k] == cols[k] && i < j) continue; /* upper half of a diagonal block */
        if (i < j) {
          const int t = i;
          i = j;
          j = t;
        }
        env[off[i] + (j - first[i])] += v[a + 3 * c];
      }
  }
  /* L L^T, row by row */
  int status = 0;
  for (int i = 0; i < n && status == 0; ++i) {
    const int fi = first[i];
    double* Li = env + off[i] - fi; /* Li[j] = L_ij, j in [fi, i] */
    for (int j = fi; j < i; ++j) {
      const int fj = first[j];
      const double* Lj = env + off[j] - fj;
      const int k0 = fi > fj ? fi : fj;
      double s = Li[j];
      for (int k = k0; k < j; ++k) s -= Li[k] * Lj[k];
      Li[j] = s / Lj[j];
    }
    double d = Li[i];
    for (int k = fi; k < i; ++k) d -= Li[k] * Li[k];
    if (!(d > 0.0)) {
      status = -1;
      break;
    }
    Li[i] = sqrt(d);
  }
  if (status == 0) {
    double* z = (double*)malloc(sizeof(double) * (size_t)n);
    if (!z) {
      free(env);
      return -2;
    }
    for (int k = 0; k < nb; ++k)
      for (int a = 0; a < 3; ++a) z[3 * k + a] = b[3 * (size_t)perm[k] + a];
    for (int i = 0; i < n; ++i) { /* L y = P b */
      const double* Li = env + off[i] - first[i];
      double s = z[i];
      for (int k = first[i]; k < i; ++k) s -= Li[k] * z[k];
      z[i] = s / Li[i];
    }
    for (int i = n - 1; i >= 0; --i) { /* L^T z = y, by columns of L^T = rows of L */
      const double* Li = env + off[i] - first[i];
      z[i] /= Li[i];
      for (int k = first[i]; k < i; ++k) z[k] -= Li[k] * z[i];
    }
    for (int k = 0; k < nb; ++k)
      for (int a = 0; a < 3; ++a) x[3 * (size_t)perm[k] + a] = z[3 * k + a];
    free(z);
  }
  free(env);
  free(perm);
  free(inv);
  free(first);
  free(off);
  return status;
}
