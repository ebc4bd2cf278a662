/*
 * synth.c -- seeded synthetic IPC Newton systems and the caller-side inputs
 * of the MAS32 preconditioner (host C, OpenMP).
 *
 * The reference (KLBSTL/AGIPC_LEARNING, StiffGIPC) assembles its Hessian from
 * scene data on the GPU.  The systems here are generated from the formulas the
 * reference uses, so that the linear solve can be exercised and timed without
 * a scene:
 *   - Freudenthal 6-tetrahedron split of a structured vertex grid;
 *   - stable Neo-Hookean "SNK1" energy (femEnergy.cu:432-459, :1032-1050)
 *     with the Lame rates mu' = 4mu/3, lambda' = lambda + 5mu/6
 *     (gl_main.cu:586-590, :621-630), element Hessian dt^2 * V * G^T H9 G;
 *   - lumped mass rho*V/4 per tet corner entered as m*I (gl_main.cu:611-614,
 *     GIPC.cu:10183-10199), i.e. A = M + dt^2 K (+ barrier Hessians);
 *   - IPC log barrier b(d) = -(d - dhat)^2 log(d/dhat) scaled by kappa;
 *   - affine bodies with q = [p, A(:,0), A(:,1), A(:,2)], J = [I, x1 I, x2 I, x3 I]
 *     and coupling blocks J^T H (setup_abd_system_gradient_and_hessian.cu:348-405).
 * Every 12x12 that is not provably PSD is projected by eigenvalue clamping.
 *
 * Also here: the two caller-side inputs of TraditionalMAS32Preconditioner that
 * the reference computes on the host -- the vertex neighbour CSR
 * (tetrahedra_obj::getVertNeighbors, load_mesh.cpp:934-1040) and the Morton
 * partition maps (set_gpu_mas32_partition, gl_main.cu:1178-1242) -- restated
 * with the same ordering rules.
 *
 * Random numbers: xoshiro256** seeded through splitmix64.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define EXPORT __attribute__((visibility("default")))

/* ------------------------------------------------------------- random --- */
typedef struct {
  uint64_t s[4];
} rng_t;

static uint64_t splitmix64(uint64_t* x)
{
  uint64_t z = (*x += 0x9e3779b97f4a7c15ull);
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}
static void rng_seed(rng_t* r, uint64_t seed)
{
  uint64_t x = seed;
  for (int i = 0; i < 4; ++i) r->s[i] = splitmix64(&x);
}
static inline uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
static uint64_t rng_next(rng_t* r)
{
  uint64_t* s = r->s;
  const uint64_t result = rotl(s[1] * 5, 7) * 9;
  const uint64_t t = s[1] << 17;
  s[2] ^= s[0];
  s[3] ^= s[1];
  s[1] ^= s[2];
  s[0] ^= s[3];
  s[2] ^= t;
  s[3] = rotl(s[3], 45);
  return result;
}
/* uniform in [0,1) with 53 bits */
static double rng_uniform(rng_t* r) { return (double)(rng_next(r) >> 11) * (1.0 / 9007199254740992.0); }
static double rng_normal(rng_t* r)
{
  double u1 = rng_uniform(r), u2 = rng_uniform(r);
  if (u1 < 1e-300) u1 = 1e-300;
  return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
}
/* Per-item stream: independent of thread count. */
static void rng_item(rng_t* r, uint64_t seed, uint64_t item) { rng_seed(r, seed ^ (item * 0xd1342543de82ef95ull + 0x632be59bd9b4e019ull)); }

EXPORT void syn_normal(long long n, uint64_t seed, int round_to_float, double* out)
{
#pragma omp parallel for schedule(static)
  for (long long blk = 0; blk < (n + 1023) / 1024; ++blk) {
    rng_t r;
    rng_item(&r, seed, (uint64_t)blk);
    const long long lo = blk * 1024, hi = lo + 1024 < n ? lo + 1024 : n;
    for (long long i = lo; i < hi; ++i) {
      const double v = rng_normal(&r);
      out[i] = round_to_float ? (double)(float)v : v;
    }
  }
}

/* ---------------------------------------------------------------- mesh --- */

/* Freudenthal split: the 6 tets of a cell share the main diagonal 0-7 and walk
 * the coordinate permutations; neighbouring cells share consistent faces. */
static const int kFreud[6][4] = {
    {0, 1, 3, 7}, {0, 1, 5, 7}, {0, 2, 3, 7}, {0, 2, 6, 7}, {0, 4, 5, 7}, {0, 4, 6, 7}};

EXPORT void syn_box_sizes(int nx, int ny, int nz, long long* nv, long long* ntet)
{
  *nv = (long long)nx * ny * nz;
  *ntet = 6LL * (nx - 1) * (ny - 1) * (nz - 1);
}

EXPORT void syn_box_mesh(int nx, int ny, int nz, double h, double* X, int* tets)
{
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        const long long v = ((long long)k * ny + j) * nx + i;
        X[3 * v] = i * h;
        X[3 * v + 1] = j * h;
        X[3 * v + 2] = k * h;
      }
  long long t = 0;
  for (int k = 0; k < nz - 1; ++k)
    for (int j = 0; j < ny - 1; ++j)
      for (int i = 0; i < nx - 1; ++i) {
        int corner[8];
        for (int c = 0; c < 8; ++c) {
          const int di = c & 1, dj = (c >> 1) & 1, dk = (c >> 2) & 1;
          corner[c] = (int)(((long long)(k + dk) * ny + (j + dj)) * nx + (i + di));
        }
        for (int q = 0; q < 6; ++q, ++t)
          for (int c = 0; c < 4; ++c) tets[4 * t + c] = corner[kFreud[q][c]];
      }
}

EXPORT void syn_perturb(long long nv, const double* X, double amplitude, uint64_t seed, double* x)
{
#pragma omp parallel for schedule(static)
  for (long long v = 0; v < nv; ++v) {
    rng_t r;
    rng_item(&r, seed, (uint64_t)v);
    for (int c = 0; c < 3; ++c) x[3 * v + c] = X[3 * v + c] + amplitude * (2.0 * rng_uniform(&r) - 1.0);
  }
}

/* ---------------------------------------------------- small dense algebra --- */

static int chol_pd(int n, const double* A)
{
  double L[144];
  for (int i = 0; i < n * n; ++i) L[i] = A[i];
  for (int k = 0; k < n; ++k) {
    double d = L[k * n + k];
    for (int p = 0; p < k; ++p) d -= L[k * n + p] * L[k * n + p];
    if (!(d > 0)) return 0;
    d = sqrt(d);
    L[k * n + k] = d;
    for (int i = k + 1; i < n; ++i) {
      double s = L[i * n + k];
      for (int p = 0; p < k; ++p) s -= L[i * n + p] * L[k * n + p];
      L[i * n + k] = s / d;
    }
  }
  return 1;
}

/* Cyclic Jacobi eigen-decomposition of a symmetric n x n (n <= 12) followed by
 * clamping negative eigenvalues to zero: A <- Q max(L,0) Q^T. */
static void psd_project(int n, double* A)
{
  double a[144], q[144];
  memcpy(a, A, sizeof(double) * n * n);
  for (int i = 0; i < n * n; ++i) q[i] = (i % (n + 1) == 0) ? 1.0 : 0.0;
  for (int sweep = 0; sweep < 60; ++sweep) {
    double off = 0, diag = 0;
    for (int i = 0; i < n; ++i) {
      diag += a[i * n + i] * a[i * n + i];
      for (int j = i + 1; j < n; ++j) off += a[i * n + j] * a[i * n + j];
    }
    if (off <= 1e-30 * diag || off == 0) break;
    for (int p = 0; p < n; ++p)
      for (int r = p + 1; r < n; ++r) {
        const double apr = a[p * n + r];
        if (fabs(apr) < 1e-300) continue;
        const double theta = (a[r * n + r] - a[p * n + p]) / (2 * apr);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1));
        const double c = 1 / sqrt(t * t + 1), s = t * c;
        for (int k = 0; k < n; ++k) {
          const double akp = a[k * n + p], akr = a[k * n + r];
          a[k * n + p] = c * akp - s * akr;
          a[k * n + r] = s * akp + c * akr;
        }
        for (int k = 0; k < n; ++k) {
          const double apk = a[p * n + k], ark = a[r * n + k];
          a[p * n + k] = c * apk - s * ark;
          a[r * n + k] = s * apk + c * ark;
        }
        for (int k = 0; k < n; ++k) {
          const double qkp = q[k * n + p], qkr = q[k * n + r];
          q[k * n + p] = c * qkp - s * qkr;
          q[k * n + r] = s * qkp + c * qkr;
        }
      }
  }
  double lam[12];
  for (int i = 0; i < n; ++i) lam[i] = a[i * n + i] > 0 ? a[i * n + i] : 0.0;
  for (int i = 0; i < n; ++i)
    for (int j = i; j < n; ++j) {
      double s = 0;
      for (int k = 0; k < n; ++k) s += q[i * n + k] * lam[k] * q[j * n + k];
      A[i * n + j] = A[j * n + i] = s;
    }
}

static void inv3(const double* m, double* o, double* det)
{
  /* row-major 3x3 */
  const double a = m[0], b = m[1], c = m[2], d = m[3], e = m[4], f = m[5], g = m[6], h = m[7], i = m[8];
  const double A = e * i - f * h, B = -(d * i - f * g), C = d * h - e * g;
  *det = a * A + b * B + c * C;
  const double id = 1.0 / *det;
  o[0] = A * id; o[1] = -(b * i - c * h) * id; o[2] = (b * f - c * e) * id;
  o[3] = B * id; o[4] = (a * i - c * g) * id; o[5] = -(a * f - c * d) * id;
  o[6] = C * id; o[7] = -(a * h - b * g) * id; o[8] = (a * e - b * d) * id;
}

/* Write the 10 upper blocks of a 4-vertex 12x12 (row-major) as triplets. */
static void emit_12x12(const double* H, const int* vid, int row_offset, int* rows, int* cols, double* vals9)
{
  int t = 0;
  for (int a = 0; a < 4; ++a)
    for (int b = a; b < 4; ++b, ++t) {
      int va = vid[a], vb = vid[b];
      int ra = a, rb = b;
      if (va > vb) {
        int tmp = va; va = vb; vb = tmp;
        tmp = ra; ra = rb; rb = tmp;
      }
      rows[t] = va + row_offset;
      cols[t] = vb + row_offset;
      double* o = vals9 + 9 * t;
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) o[i + 3 * j] = H[(3 * ra + i) * 12 + 3 * rb + j];
    }
}

/* ------------------------------------------------------------------ FEM --- */

/* d^2 Psi / dF^2 of SNK1, vec(F) column-major (index i + 3j). */
static void snk1_hessian9(const double* F /*row-major*/, double mu_l, double la_l, double* H9)
{
  double f[3][3]; /* f[c] = column c of F */
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r) f[c][r] = F[3 * r + c];
  double g[3][3];
  /* dJ/df0 = f1 x f2, dJ/df1 = f2 x f0, dJ/df2 = f0 x f1 */
  for (int c = 0; c < 3; ++c) {
    const double* u = f[(c + 1) % 3];
    const double* v = f[(c + 2) % 3];
    g[c][0] = u[1] * v[2] - u[2] * v[1];
    g[c][1] = u[2] * v[0] - u[0] * v[2];
    g[c][2] = u[0] * v[1] - u[1] * v[0];
  }
  const double J = f[0][0] * g[0][0] + f[0][1] * g[0][1] + f[0][2] * g[0][2];
  const double alpha = 1.0 + mu_l / la_l;
  const double s = la_l * (J - alpha);
  for (int i = 0; i < 81; ++i) H9[i] = 0;
  for (int a = 0; a < 9; ++a) {
    H9[a * 9 + a] += mu_l;
    for (int b = 0; b < 9; ++b) H9[a * 9 + b] += la_l * g[a / 3][a % 3] * g[b / 3][b % 3];
  }
  /* s * d^2J/dF^2: block (c, c+1) = -[f_{c+2}]x, block (c, c+2) = [f_{c+1}]x */
  for (int c = 0; c < 3; ++c) {
    const int c1 = (c + 1) % 3, c2 = (c + 2) % 3;
    const double* w = f[c2];
    const double* y = f[c1];
    /* [w]x = [[0,-w2,w1],[w2,0,-w0],[-w1,w0,0]] */
    const double Wx[9] = {0, -w[2], w[1], w[2], 0, -w[0], -w[1], w[0], 0};
    const double Yx[9] = {0, -y[2], y[1], y[2], 0, -y[0], -y[1], y[0], 0};
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        H9[(3 * c + i) * 9 + 3 * c1 + j] += -s * Wx[3 * i + j];
        H9[(3 * c + i) * 9 + 3 * c2 + j] += s * Yx[3 * i + j];
      }
  }
}

/* Element Hessian + triplets for every tet.  E_tet may be NULL (uniform E).
 * Writes 10 triplets per tet at [10t, 10t+10). Returns the number of tets
 * whose 9x9 was not positive definite (projected at 12x12). */
EXPORT long long syn_fem_triplets(long long ntet, const int* tets, const double* X, const double* x,
                                  const double* E_tet, double E, double nu, double dt, int row_offset,
                                  int* rows, int* cols, double* vals9)
{
  long long projected = 0;
#pragma omp parallel for schedule(static) reduction(+ : projected)
  for (long long t = 0; t < ntet; ++t) {
    const int* v = tets + 4 * t;
    double Dm[9], Ds[9], Dinv[9], det;
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) {
        Dm[3 * r + c] = X[3 * (long long)v[c + 1] + r] - X[3 * (long long)v[0] + r];
        Ds[3 * r + c] = x[3 * (long long)v[c + 1] + r] - x[3 * (long long)v[0] + r];
      }
    inv3(Dm, Dinv, &det);
    const double vol = fabs(det) / 6.0;
    double F[9];
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) F[3 * r + c] = Ds[3 * r] * Dinv[c] + Ds[3 * r + 1] * Dinv[3 + c] + Ds[3 * r + 2] * Dinv[6 + c];
    const double Et = E_tet ? E_tet[t] : E;
    const double mu = Et / (2 * (1 + nu)), la = Et * nu / ((1 + nu) * (1 - 2 * nu));
    const double mu_l = 4 * mu / 3, la_l = la + 5 * mu / 6;
    double H9[81];
    snk1_hessian9(F, mu_l, la_l, H9);
    const int pd = chol_pd(9, H9);
    /* coefficients c[a][j] with dF_ij/dx_{a,i} = c[a][j] */
    double cf[4][3];
    for (int j = 0; j < 3; ++j) {
      cf[1][j] = Dinv[0 * 3 + j];
      cf[2][j] = Dinv[1 * 3 + j];
      cf[3][j] = Dinv[2 * 3 + j];
      cf[0][j] = -(cf[1][j] + cf[2][j] + cf[3][j]);
    }
    double H[144];
    const double scale = vol * dt * dt;
    for (int a = 0; a < 4; ++a)
      for (int i = 0; i < 3; ++i)
        for (int b = 0; b < 4; ++b)
          for (int k = 0; k < 3; ++k) {
            double s = 0;
            for (int j = 0; j < 3; ++j)
              for (int l = 0; l < 3; ++l) s += cf[a][j] * cf[b][l] * H9[(i + 3 * j) * 9 + (k + 3 * l)];
            H[(3 * a + i) * 12 + 3 * b + k] = scale * s;
          }
    if (!pd) {
      psd_project(12, H);
      projected++;
    }
    emit_12x12(H, v, row_offset, rows + 10 * t, cols + 10 * t, vals9 + 90 * t);
  }
  return projected;
}

/* Lumped mass m_v = sum rho*V_t/4 (rest volumes). */
EXPORT void syn_lumped_mass(long long nv, long long ntet, const int* tets, const double* X, double rho, double* mass)
{
  memset(mass, 0, sizeof(double) * (size_t)nv);
  for (long long t = 0; t < ntet; ++t) {
    const int* v = tets + 4 * t;
    double Dm[9], Dinv[9], det;
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) Dm[3 * r + c] = X[3 * (long long)v[c + 1] + r] - X[3 * (long long)v[0] + r];
    inv3(Dm, Dinv, &det);
    const double q = fabs(det) / 6.0 * rho / 4.0;
    for (int c = 0; c < 4; ++c) mass[v[c]] += q;
  }
}

EXPORT void syn_mass_triplets(long long nv, const double* mass, int row_offset, int* rows, int* cols, double* vals9)
{
  for (long long v = 0; v < nv; ++v) {
    rows[v] = cols[v] = (int)v + row_offset;
    double* o = vals9 + 9 * v;
    memset(o, 0, 9 * sizeof(double));
    o[0] = o[4] = o[8] = mass[v];
  }
}

/* ------------------------------------------------------------- surface --- */

typedef struct {
  uint64_t key;
  int tri[3];
} face_t;

static int cmp_face(const void* a, const void* b)
{
  const uint64_t x = ((const face_t*)a)->key, y = ((const face_t*)b)->key;
  return x < y ? -1 : (x > y);
}

/* Boundary triangles (faces owned by one tet), oriented as in the tet.
 * tris must hold 4*ntet*3 ints; returns the count. */
EXPORT long long syn_boundary_triangles(long long nv, long long ntet, const int* tets, int* tris)
{
  (void)nv;
  static const int fidx[4][3] = {{1, 2, 3}, {0, 3, 2}, {0, 1, 3}, {0, 2, 1}};
  face_t* f = (face_t*)malloc(sizeof(face_t) * (size_t)(4 * ntet));
  for (long long t = 0; t < ntet; ++t)
    for (int q = 0; q < 4; ++q) {
      int a = tets[4 * t + fidx[q][0]], b = tets[4 * t + fidx[q][1]], c = tets[4 * t + fidx[q][2]];
      face_t* e = f + 4 * t + q;
      e->tri[0] = a; e->tri[1] = b; e->tri[2] = c;
      int s0 = a, s1 = b, s2 = c, tmp;
      if (s0 > s1) { tmp = s0; s0 = s1; s1 = tmp; }
      if (s1 > s2) { tmp = s1; s1 = s2; s2 = tmp; }
      if (s0 > s1) { tmp = s0; s0 = s1; s1 = tmp; }
      e->key = ((uint64_t)s0 << 42) | ((uint64_t)s1 << 21) | (uint64_t)s2;
    }
  qsort(f, (size_t)(4 * ntet), sizeof(face_t), cmp_face);
  long long n = 0;
  for (long long i = 0; i < 4 * ntet;) {
    long long j = i + 1;
    while (j < 4 * ntet && f[j].key == f[i].key) ++j;
    if (j - i == 1) {
      tris[3 * n] = f[i].tri[0];
      tris[3 * n + 1] = f[i].tri[1];
      tris[3 * n + 2] = f[i].tri[2];
      ++n;
    }
    i = j;
  }
  free(f);
  return n;
}

/* ------------------------------------------------------------- contact --- */

static inline double barrier_d1(double d, double dh)
{
  return -(2 * (d - dh) * log(d / dh) + (d - dh) * (d - dh) / d);
}
static inline double barrier_d2(double d, double dh)
{
  return -(2 * log(d / dh) + 4 * (d - dh) / d - (d - dh) * (d - dh) / (d * d));
}

/* kappa*(b'' g g^T + b' S), PSD-projected, where g = t (x) n is the distance
 * gradient for weights t over the 4 vertices and unit normal n, and S is the
 * tangential curvature term (I - n n^T)/h (x) t t^T. */
static void barrier_hessian(const double* n, const double* t, double d, double dhat, double kappa,
                            double h, double* H)
{
  const double b1 = barrier_d1(d, dhat), b2 = barrier_d2(d, dhat);
  for (int a = 0; a < 4; ++a)
    for (int i = 0; i < 3; ++i)
      for (int b = 0; b < 4; ++b)
        for (int k = 0; k < 3; ++k) {
          const double gg = t[a] * n[i] * t[b] * n[k];
          const double P = ((i == k) ? 1.0 : 0.0) - n[i] * n[k];
          H[(3 * a + i) * 12 + 3 * b + k] = kappa * (b2 * gg + b1 * P * t[a] * t[b] / h);
        }
  psd_project(12, H);
}

static int cmp_int(const void* a, const void* b)
{
  const int x = *(const int*)a, y = *(const int*)b;
  return x < y ? -1 : (x > y);
}

typedef struct {
  int nx, ny, nz;
  int* cell_start; /* per grid cell of the primitive's first vertex */
  int* items;
} grid_index_t;

static void grid_coords(const double* X, int v, double h, int* g)
{
  for (int c = 0; c < 3; ++c) g[c] = (int)floor(X[3 * (long long)v + c] / h + 0.5);
}

/* Bucket primitives (triangles or edges of `arity` vertices) by the grid cell
 * of their first vertex. */
static void build_grid_index(grid_index_t* gi, int nx, int ny, int nz, const double* X, double h,
                             const int* prims, long long nprim, int arity)
{
  gi->nx = nx; gi->ny = ny; gi->nz = nz;
  const long long ncell = (long long)nx * ny * nz;
  gi->cell_start = (int*)calloc((size_t)ncell + 1, sizeof(int));
  gi->items = (int*)malloc(sizeof(int) * (size_t)(nprim > 0 ? nprim : 1));
  int* cellof = (int*)malloc(sizeof(int) * (size_t)(nprim > 0 ? nprim : 1));
  for (long long p = 0; p < nprim; ++p) {
    int g[3];
    grid_coords(X, prims[arity * p], h, g);
    if (g[0] < 0) g[0] = 0;
    if (g[0] >= nx) g[0] = nx - 1;
    if (g[1] < 0) g[1] = 0;
    if (g[1] >= ny) g[1] = ny - 1;
    if (g[2] < 0) g[2] = 0;
    if (g[2] >= nz) g[2] = nz - 1;
    cellof[p] = (int)(((long long)g[2] * ny + g[1]) * nx + g[0]);
    gi->cell_start[cellof[p] + 1]++;
  }
  for (long long c = 0; c < ncell; ++c) gi->cell_start[c + 1] += gi->cell_start[c];
  int* fill = (int*)calloc((size_t)ncell, sizeof(int));
  for (long long p = 0; p < nprim; ++p) gi->items[gi->cell_start[cellof[p]] + fill[cellof[p]]++] = (int)p;
  free(fill);
  free(cellof);
}

static void free_grid_index(grid_index_t* gi)
{
  free(gi->cell_start);
  free(gi->items);
}

/* Candidates of the primitive index within +-2 cells of grid point g whose
 * vertices are all within Chebyshev distance 2 and disjoint from excl. */
static int gather_candidates(const grid_index_t* gi, const int* prims, int arity, const double* X, double h,
                             const int* g, const int* excl, int nexcl, int* out, int cap)
{
  int n = 0;
  for (int dz = -2; dz <= 2; ++dz)
    for (int dy = -2; dy <= 2; ++dy)
      for (int dx = -2; dx <= 2; ++dx) {
        const int cx = g[0] + dx, cy = g[1] + dy, cz = g[2] + dz;
        if (cx < 0 || cy < 0 || cz < 0 || cx >= gi->nx || cy >= gi->ny || cz >= gi->nz) continue;
        const long long c = ((long long)cz * gi->ny + cy) * gi->nx + cx;
        for (int s = gi->cell_start[c]; s < gi->cell_start[c + 1]; ++s) {
          const int p = gi->items[s];
          int ok = 1;
          for (int q = 0; q < arity && ok; ++q) {
            const int v = prims[arity * (long long)p + q];
            int gv[3];
            grid_coords(X, v, h, gv);
            if (abs(gv[0] - g[0]) > 2 || abs(gv[1] - g[1]) > 2 || abs(gv[2] - g[2]) > 2) ok = 0;
            for (int e = 0; e < nexcl; ++e)
              if (v == excl[e]) ok = 0;
          }
          if (ok && n < cap) out[n++] = p;
        }
      }
  qsort(out, (size_t)n, sizeof(int), cmp_int);
  return n;
}

static void tri_normal(const double* X, const int* tri, double* n)
{
  double e1[3], e2[3];
  for (int c = 0; c < 3; ++c) {
    e1[c] = X[3 * (long long)tri[1] + c] - X[3 * (long long)tri[0] + c];
    e2[c] = X[3 * (long long)tri[2] + c] - X[3 * (long long)tri[0] + c];
  }
  n[0] = e1[1] * e2[2] - e1[2] * e2[1];
  n[1] = e1[2] * e2[0] - e1[0] * e2[2];
  n[2] = e1[0] * e2[1] - e1[1] * e2[0];
  const double l = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
  for (int c = 0; c < 3; ++c) n[c] = l > 0 ? n[c] / l : (c == 2);
}

/* Point-triangle pairs between surface vertices and surface triangles within
 * 2 grid cells.  Grid dims (nx,ny,nz) with spacing h index the rest positions.
 * Outputs: pairs4 (int4 per pair, IPC point-triangle encoding (-v-1,t0,t1,t2)
 * with the given vertex offset), and 10 triplets per pair.  Returns the
 * number of pairs written. */
EXPORT long long syn_contacts_pt(int nx, int ny, int nz, double h, const double* X, long long ntri, const int* tris,
                                 long long npairs, double dhat, double kappa, uint64_t seed, int row_offset,
                                 int vertex_offset, int* pairs4, int* rows, int* cols, double* vals9)
{
  /* surface vertices = vertices of boundary triangles */
  long long nv = (long long)nx * ny * nz;
  char* on = (char*)calloc((size_t)nv, 1);
  for (long long t = 0; t < 3 * ntri; ++t) on[tris[t]] = 1;
  long long ns = 0;
  for (long long v = 0; v < nv; ++v) ns += on[v];
  int* sv = (int*)malloc(sizeof(int) * (size_t)(ns > 0 ? ns : 1));
  ns = 0;
  for (long long v = 0; v < nv; ++v)
    if (on[v]) sv[ns++] = (int)v;
  free(on);
  grid_index_t gi;
  build_grid_index(&gi, nx, ny, nz, X, h, tris, ntri, 3);
  long long written = 0;
  const int cap = 4096;
  int* cand = (int*)malloc(sizeof(int) * cap);
  rng_t r;
  rng_seed(&r, seed);
  for (long long p = 0; p < npairs; ++p) {
    int ncand = 0, v = -1, tries = 0;
    while (ncand == 0 && tries++ < 64) {
      v = sv[rng_next(&r) % (uint64_t)ns];
      int g[3];
      grid_coords(X, v, h, g);
      ncand = gather_candidates(&gi, tris, 3, X, h, g, &v, 1, cand, cap);
    }
    if (ncand == 0) break;
    const int* tri = tris + 3 * (long long)cand[rng_next(&r) % (uint64_t)ncand];
    const double d = dhat * (0.1 + 0.9 * rng_uniform(&r));
    double w0 = rng_uniform(&r), w1 = rng_uniform(&r);
    if (w0 + w1 > 1) { w0 = 1 - w0; w1 = 1 - w1; }
    const double w2 = 1 - w0 - w1;
    double n[3];
    tri_normal(X, tri, n);
    const double t4[4] = {1.0, -w0, -w1, -w2};
    double H[144];
    barrier_hessian(n, t4, d, dhat, kappa, h, H);
    const int vid[4] = {v, tri[0], tri[1], tri[2]};
    emit_12x12(H, vid, row_offset, rows + 10 * written, cols + 10 * written, vals9 + 90 * written);
    pairs4[4 * written] = -(v + vertex_offset) - 1;
    pairs4[4 * written + 1] = tri[0] + vertex_offset;
    pairs4[4 * written + 2] = tri[1] + vertex_offset;
    pairs4[4 * written + 3] = tri[2] + vertex_offset;
    ++written;
  }
  free(cand);
  free(sv);
  free_grid_index(&gi);
  return written;
}

static int cmp64(const void* x, const void* y)
{
  const uint64_t a = *(const uint64_t*)x, b = *(const uint64_t*)y;
  return a < b ? -1 : (a > b);
}

/* Unique boundary edges (from boundary triangles), sorted. edges: 2*3*ntri. */
EXPORT long long syn_boundary_edges(long long ntri, const int* tris, int* edges)
{
  uint64_t* k = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)(3 * ntri > 0 ? 3 * ntri : 1));
  for (long long t = 0; t < ntri; ++t)
    for (int e = 0; e < 3; ++e) {
      int a = tris[3 * t + e], b = tris[3 * t + (e + 1) % 3];
      if (a > b) { int tmp = a; a = b; b = tmp; }
      k[3 * t + e] = ((uint64_t)a << 32) | (uint32_t)b;
    }
  qsort(k, (size_t)(3 * ntri), sizeof(uint64_t), cmp64);
  long long n = 0;
  for (long long i = 0; i < 3 * ntri; ++i)
    if (i == 0 || k[i] != k[i - 1]) {
      edges[2 * n] = (int)(k[i] >> 32);
      edges[2 * n + 1] = (int)(k[i] & 0xffffffffu);
      ++n;
    }
  free(k);
  return n;
}

/* Edge-edge pairs between surface edges within 2 grid cells, IPC encoding
 * (e0,e1,e2,e3) all non-negative. */
EXPORT long long syn_contacts_ee(int nx, int ny, int nz, double h, const double* X, long long nedge, const int* edges,
                                 long long npairs, double dhat, double kappa, uint64_t seed, int row_offset,
                                 int vertex_offset, int* pairs4, int* rows, int* cols, double* vals9)
{
  grid_index_t gi;
  build_grid_index(&gi, nx, ny, nz, X, h, edges, nedge, 2);
  const int cap = 4096;
  int* cand = (int*)malloc(sizeof(int) * cap);
  rng_t r;
  rng_seed(&r, seed);
  long long written = 0;
  for (long long p = 0; p < npairs; ++p) {
    int ncand = 0, e0 = -1, tries = 0;
    while (ncand == 0 && tries++ < 64) {
      e0 = (int)(rng_next(&r) % (uint64_t)nedge);
      int g[3];
      grid_coords(X, edges[2 * (long long)e0], h, g);
      ncand = gather_candidates(&gi, edges, 2, X, h, g, edges + 2 * (long long)e0, 2, cand, cap);
    }
    if (ncand == 0) break;
    const int* ea = edges + 2 * (long long)e0;
    const int* eb = edges + 2 * (long long)cand[rng_next(&r) % (uint64_t)ncand];
    const double d = dhat * (0.1 + 0.9 * rng_uniform(&r));
    const double s = rng_uniform(&r), q = rng_uniform(&r);
    double da[3], db[3], n[3];
    for (int c = 0; c < 3; ++c) {
      da[c] = X[3 * (long long)ea[1] + c] - X[3 * (long long)ea[0] + c];
      db[c] = X[3 * (long long)eb[1] + c] - X[3 * (long long)eb[0] + c];
    }
    n[0] = da[1] * db[2] - da[2] * db[1];
    n[1] = da[2] * db[0] - da[0] * db[2];
    n[2] = da[0] * db[1] - da[1] * db[0];
    double l = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
    if (l < 1e-12) { /* parallel edges: any normal orthogonal to da */
      const double ax = fabs(da[0]) < 0.5 * sqrt(da[0] * da[0] + da[1] * da[1] + da[2] * da[2]) ? 1.0 : 0.0;
      const double o[3] = {ax, 1.0 - ax, 0.0};
      n[0] = da[1] * o[2] - da[2] * o[1];
      n[1] = da[2] * o[0] - da[0] * o[2];
      n[2] = da[0] * o[1] - da[1] * o[0];
      l = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
    }
    for (int c = 0; c < 3; ++c) n[c] /= l;
    const double t4[4] = {1 - s, s, -(1 - q), -q};
    double H[144];
    barrier_hessian(n, t4, d, dhat, kappa, h, H);
    const int vid[4] = {ea[0], ea[1], eb[0], eb[1]};
    emit_12x12(H, vid, row_offset, rows + 10 * written, cols + 10 * written, vals9 + 90 * written);
    for (int c = 0; c < 4; ++c) pairs4[4 * written + c] = vid[c] + vertex_offset;
    ++written;
  }
  free(cand);
  free_grid_index(&gi);
  return written;
}

/* ----------------------------------------------------------------- ABD --- */

/* Orthogonality energy V(A) = ||A A^T - I||_F^2: Hessian w.r.t. vec(A)
 * column-major (index a + 3b for A_ab). */
static void orth_hessian(const double* A /*row-major*/, double* H9)
{
  double C[9];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double s = 0;
      for (int k = 0; k < 3; ++k) s += A[3 * i + k] * A[3 * j + k];
      C[3 * i + j] = s - (i == j);
    }
  for (int p = 0; p < 9; ++p)
    for (int q = 0; q < 9; ++q) {
      const int a = p % 3, b = p / 3, c = q % 3, d = q / 3;
      double s = 0;
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
          const double dpa = ((i == a) ? A[3 * j + b] : 0.0) + ((j == a) ? A[3 * i + b] : 0.0);
          const double dqc = ((i == c) ? A[3 * j + d] : 0.0) + ((j == c) ? A[3 * i + d] : 0.0);
          const double d2 = (b == d) ? (((i == a && j == c) ? 1.0 : 0.0) + ((j == a && i == c) ? 1.0 : 0.0)) : 0.0;
          s += dpa * dqc + C[3 * i + j] * d2;
        }
      H9[9 * p + q] = 2 * s;
    }
}

/* ABD body Hessians: mass m, cube of side `size` (inertia m s^2/12 per axis),
 * stiffness k on the orthogonality energy at A = I + noise, scaled by dt^2.
 * Writes 10 upper triplets per body (block rows 4b..4b+3). */
EXPORT void syn_abd_bodies(int bodies, double mass, double size, double stiffness, double noise, double dt,
                           uint64_t seed, int* rows, int* cols, double* vals9)
{
#pragma omp parallel for schedule(static)
  for (int bdy = 0; bdy < bodies; ++bdy) {
    rng_t r;
    rng_item(&r, seed, (uint64_t)bdy);
    double A[9];
    for (int i = 0; i < 9; ++i) A[i] = (i % 4 == 0 ? 1.0 : 0.0) + noise * (2 * rng_uniform(&r) - 1);
    double H9[81];
    orth_hessian(A, H9);
    psd_project(9, H9);
    double H[144];
    memset(H, 0, sizeof(H));
    const double inertia = mass * size * size / 12.0;
    for (int i = 0; i < 3; ++i) H[i * 12 + i] = mass;
    for (int i = 3; i < 12; ++i) H[i * 12 + i] = inertia;
    for (int p = 0; p < 9; ++p)
      for (int q = 0; q < 9; ++q) H[(3 + p) * 12 + 3 + q] += dt * dt * stiffness * H9[9 * p + q];
    const int vid[4] = {4 * bdy, 4 * bdy + 1, 4 * bdy + 2, 4 * bdy + 3};
    emit_12x12(H, vid, 0, rows + 10 * bdy, cols + 10 * bdy, vals9 + 90 * bdy);
  }
}

/* ABD-point / FEM-triangle pairs.  Body b's corners are x = c_b + (+-s/2)^3
 * with c_b above the slab; each pair picks a body corner and a top-surface
 * triangle of the slab.  The 4-vertex barrier Hessian H (point, t0, t1, t2)
 * is reduced to DOFs: body-body J^T H_pp J, body-vertex J^T H_pt, vertex-vertex
 * H_tt.  Triplets per pair: 10 (body 4x4 upper) + 12 (3 vertices x 4 body
 * rows) + 6 (triangle upper) = 28.  Pair encoding for the MAS contact graph:
 * (-(abd_vertex)-1, t0+vo, t1+vo, t2+vo) with abd_vertex = 8b+corner and
 * vo = 8*bodies (the FEM vertex offset in vertex numbering). */
EXPORT long long syn_abd_contacts(int bodies, double size, long long ntop, const int* top_tris, const double* X,
                                  long long npairs, double dhat, double kappa, double h, uint64_t seed,
                                  int fem_row_offset, int* pairs4, int* rows, int* cols, double* vals9)
{
  rng_t r;
  rng_seed(&r, seed);
  long long w = 0;
  for (long long p = 0; p < npairs; ++p) {
    const int bdy = (int)(rng_next(&r) % (uint64_t)bodies);
    const int corner = (int)(rng_next(&r) % 8);
    const int* tri = top_tris + 3 * (long long)(rng_next(&r) % (uint64_t)ntop);
    const double xb[3] = {((corner & 1) ? 0.5 : -0.5) * size, ((corner & 2) ? 0.5 : -0.5) * size,
                          ((corner & 4) ? 0.5 : -0.5) * size};
    const double d = dhat * (0.1 + 0.9 * rng_uniform(&r));
    double w0 = rng_uniform(&r), w1 = rng_uniform(&r);
    if (w0 + w1 > 1) { w0 = 1 - w0; w1 = 1 - w1; }
    double n[3];
    tri_normal(X, tri, n);
    const double w2 = 1 - w0 - w1;
    const double t4[4] = {1.0, -w0, -w1, -w2};
    double H[144];
    barrier_hessian(n, t4, d, dhat, kappa, h, H);
    /* J (3x12) = [I, xb0 I, xb1 I, xb2 I] */
    const double jc[4] = {1.0, xb[0], xb[1], xb[2]};
    double Hbb[144];
    for (int a = 0; a < 4; ++a)
      for (int i = 0; i < 3; ++i)
        for (int b = 0; b < 4; ++b)
          for (int k = 0; k < 3; ++k) Hbb[(3 * a + i) * 12 + 3 * b + k] = jc[a] * jc[b] * H[i * 12 + k];
    const int bvid[4] = {4 * bdy, 4 * bdy + 1, 4 * bdy + 2, 4 * bdy + 3};
    emit_12x12(Hbb, bvid, 0, rows + w, cols + w, vals9 + 9 * w);
    w += 10;
    for (int q = 0; q < 3; ++q)
      for (int a = 0; a < 4; ++a) {
        rows[w] = 4 * bdy + a;
        cols[w] = tri[q] + fem_row_offset;
        double* o = vals9 + 9 * w;
        for (int i = 0; i < 3; ++i)
          for (int k = 0; k < 3; ++k) o[i + 3 * k] = jc[a] * H[i * 12 + 3 * (q + 1) + k];
        ++w;
      }
    for (int q = 0; q < 3; ++q)
      for (int s = q; s < 3; ++s) {
        int vq = tri[q], vs = tri[s], rq = q, rs = s;
        if (vq > vs) {
          int tmp = vq; vq = vs; vs = tmp;
          tmp = rq; rq = rs; rs = tmp;
        }
        rows[w] = vq + fem_row_offset;
        cols[w] = vs + fem_row_offset;
        double* o = vals9 + 9 * w;
        for (int i = 0; i < 3; ++i)
          for (int k = 0; k < 3; ++k) o[i + 3 * k] = H[(3 * (rq + 1) + i) * 12 + 3 * (rs + 1) + k];
        ++w;
      }
    pairs4[4 * p] = -(8 * bdy + corner) - 1;
    pairs4[4 * p + 1] = tri[0] + 8 * bodies;
    pairs4[4 * p + 2] = tri[1] + 8 * bodies;
    pairs4[4 * p + 3] = tri[2] + 8 * bodies;
  }
  return w;
}

/* ------------------------------------------------------ triplet assembly --- */

/* LSD radix sort of (key, payload) by the 64-bit key; stable. */
static void radix_sort_kv(long long n, uint64_t* key, long long* val, int key_bits)
{
  uint64_t* k2 = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)(n > 0 ? n : 1));
  long long* v2 = (long long*)malloc(sizeof(long long) * (size_t)(n > 0 ? n : 1));
  const int DIG = 11, R = 1 << DIG;
  long long* cnt = (long long*)malloc(sizeof(long long) * R);
  for (int shift = 0; shift < key_bits; shift += DIG) {
    memset(cnt, 0, sizeof(long long) * R);
    for (long long i = 0; i < n; ++i) cnt[(key[i] >> shift) & (R - 1)]++;
    long long s = 0;
    for (int d = 0; d < R; ++d) {
      const long long c = cnt[d];
      cnt[d] = s;
      s += c;
    }
    for (long long i = 0; i < n; ++i) {
      const long long o = cnt[(key[i] >> shift) & (R - 1)]++;
      k2[o] = key[i];
      v2[o] = val[i];
    }
    memcpy(key, k2, sizeof(uint64_t) * (size_t)n);
    memcpy(val, v2, sizeof(long long) * (size_t)n);
  }
  free(k2);
  free(v2);
  free(cnt);
}

/* Sum duplicate (row,col) triplets; output sorted by (row,col).  In-place
 * safe is NOT required: out arrays must not alias the inputs. Returns count. */
EXPORT long long syn_assemble(long long n, const int* rows, const int* cols, const double* vals9, int* orow,
                              int* ocol, double* ovals9)
{
  if (n <= 0) return 0;
  uint64_t* key = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)n);
  long long* idx = (long long*)malloc(sizeof(long long) * (size_t)n);
  int maxv = 0;
  for (long long i = 0; i < n; ++i) {
    key[i] = ((uint64_t)(uint32_t)rows[i] << 32) | (uint32_t)cols[i];
    idx[i] = i;
    if (rows[i] > maxv) maxv = rows[i];
    if (cols[i] > maxv) maxv = cols[i];
  }
  int bits = 1;
  while ((1LL << bits) <= maxv) ++bits;
  /* compact key: row<<bits | col, then sort on 2*bits */
  for (long long i = 0; i < n; ++i) key[i] = ((uint64_t)(uint32_t)rows[i] << bits) | (uint32_t)cols[i];
  radix_sort_kv(n, key, idx, 2 * bits);
  long long u = -1;
  uint64_t prev = ~0ull;
  for (long long i = 0; i < n; ++i) {
    if (i == 0 || key[i] != prev) {
      ++u;
      orow[u] = rows[idx[i]];
      ocol[u] = cols[idx[i]];
      memset(ovals9 + 9 * u, 0, 9 * sizeof(double));
      prev = key[i];
    }
    const double* s = vals9 + 9 * idx[i];
    double* d = ovals9 + 9 * u;
    for (int e = 0; e < 9; ++e) d[e] += s[e];
  }
  free(key);
  free(idx);
  return u + 1;
}

/* -------------------------------------------------- MAS32 caller inputs --- */

/* tetrahedra_obj::getVertNeighbors (load_mesh.cpp:934-1040): unique tet edges
 * oriented as first met, visited in (first,second) order, pushed to both
 * ends.  list must hold 12*ntet entries.  Returns the list size. */
EXPORT long long syn_vertex_neighbors(long long nv, long long ntet, const int* tets, uint32_t* start, uint32_t* num,
                                      uint32_t* list)
{
  static const int pr[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3}};
  const long long ne = 6 * ntet;
  uint64_t* ukey = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)(ne > 0 ? ne : 1));
  long long* ord = (long long*)malloc(sizeof(long long) * (size_t)(ne > 0 ? ne : 1));
  int bits = 1;
  while ((1LL << bits) <= nv) ++bits;
  for (long long t = 0; t < ntet; ++t)
    for (int e = 0; e < 6; ++e) {
      const uint32_t a = (uint32_t)tets[4 * t + pr[e][0]], b = (uint32_t)tets[4 * t + pr[e][1]];
      const uint32_t lo = a < b ? a : b, hi = a < b ? b : a;
      ukey[6 * t + e] = ((uint64_t)lo << bits) | hi;
      ord[6 * t + e] = 6 * t + e;
    }
  /* stable sort by unordered key: the first occurrence in tet order comes first */
  radix_sort_kv(ne, ukey, ord, 2 * bits);
  uint64_t* ekey = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)(ne > 0 ? ne : 1));
  long long* dummy = (long long*)malloc(sizeof(long long) * (size_t)(ne > 0 ? ne : 1));
  long long m = 0;
  for (long long i = 0; i < ne; ++i) {
    if (i > 0 && ukey[i] == ukey[i - 1]) continue;
    const long long t = ord[i] / 6;
    const int e = (int)(ord[i] % 6);
    const uint32_t a = (uint32_t)tets[4 * t + pr[e][0]], b = (uint32_t)tets[4 * t + pr[e][1]];
    ekey[m] = ((uint64_t)a << bits) | b; /* oriented (first, second) */
    dummy[m] = m;
    ++m;
  }
  radix_sort_kv(m, ekey, dummy, 2 * bits);
  memset(num, 0, sizeof(uint32_t) * (size_t)nv);
  for (long long i = 0; i < m; ++i) {
    num[ekey[i] >> bits]++;
    num[ekey[i] & ((1ull << bits) - 1)]++;
  }
  long long off = 0;
  for (long long v = 0; v < nv; ++v) {
    start[v] = (uint32_t)off;
    off += num[v];
  }
  uint32_t* fill = (uint32_t*)calloc((size_t)nv, sizeof(uint32_t));
  for (long long i = 0; i < m; ++i) {
    const uint32_t a = (uint32_t)(ekey[i] >> bits), b = (uint32_t)(ekey[i] & ((1ull << bits) - 1));
    list[start[a] + fill[a]++] = b;
    list[start[b] + fill[b]++] = a;
  }
  free(fill);
  free(ukey);
  free(ord);
  free(ekey);
  free(dummy);
  return off;
}

static uint32_t expand_morton_10(uint32_t v)
{
  v &= 0x000003ffu;
  v = (v | (v << 16)) & 0x030000FFu;
  v = (v | (v << 8)) & 0x0300F00Fu;
  v = (v | (v << 4)) & 0x030C30C3u;
  v = (v | (v << 2)) & 0x09249249u;
  return v;
}

static uint32_t quantize10(double value, double lo, double hi)
{
  const double extent = hi - lo;
  double t = extent > 0.0 ? (value - lo) / extent : 0.0;
  if (t < 0) t = 0;
  if (t > 1) t = 1;
  return (uint32_t)(t * 1023.0 + 0.5);
}

/* set_gpu_mas32_partition (gl_main.cu:1202-1242): stable sort by 30-bit
 * Morton code of positions quantised to 10 bits per axis over the bounding
 * box, ties by index; part_map_real has ceil32(nv) slots, -1 at the tail. */
EXPORT void syn_morton_partition(long long nv, const double* X, int* part_map_real, int* real_map_part)
{
  double lo[3] = {X[0], X[1], X[2]}, hi[3] = {X[0], X[1], X[2]};
  for (long long v = 1; v < nv; ++v)
    for (int c = 0; c < 3; ++c) {
      if (X[3 * v + c] < lo[c]) lo[c] = X[3 * v + c];
      if (X[3 * v + c] > hi[c]) hi[c] = X[3 * v + c];
    }
  uint64_t* key = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)nv);
  long long* ord = (long long*)malloc(sizeof(long long) * (size_t)nv);
  for (long long v = 0; v < nv; ++v) {
    const uint32_t code = expand_morton_10(quantize10(X[3 * v], lo[0], hi[0])) |
                          (expand_morton_10(quantize10(X[3 * v + 1], lo[1], hi[1])) << 1) |
                          (expand_morton_10(quantize10(X[3 * v + 2], lo[2], hi[2])) << 2);
    key[v] = code;
    ord[v] = v;
  }
  radix_sort_kv(nv, key, ord, 33); /* stable: ties keep index order */
  const long long slots = (nv + 31) / 32 * 32;
  for (long long s = 0; s < slots; ++s) part_map_real[s] = -1;
  for (long long s = 0; s < nv; ++s) {
    part_map_real[s] = (int)ord[s];
    real_map_part[ord[s]] = (int)s;
  }
  free(key);
  free(ord);
}
