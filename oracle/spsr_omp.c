/*
 * CPU restatement of the jspsr sparse screened-Poisson reconstruction path in C with OpenMP.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the cpu_baseline /
 * --impl reference legs of bench.py load this library (through oracle/fast.py), as the checker or
 * as the timed CPU baseline.  The product (neural-galerkin_b200/jspsr) never loads it.
 *
 * It is the same algorithm as oracle/spsr.py, stage for stage, written for the host's cores so that
 * full-size clouds (hundreds of thousands of points) finish in seconds: structure decisions (voxel
 * quantisation, octant signs, neighbour quantisation) in float32 exactly as the reference's torch
 * code makes them, everything numeric in FP64, each level solved by Jacobi-preconditioned CG in
 * FP64 to the requested relative residual.  Reference files followed (inside
 * huangjh-pub/neural-galerkin):
 *   jspsr/__init__.py:8-61                      reconstruct
 *   jspsr/core/_hash_backend.py:13-28           compute_density
 *   jspsr/core/_hash_backend.py:176-290         neighbour queries (incl. the coarse->fine inversion)
 *   jspsr/core/_hash_backend.py:332-356         splat_data
 *   jspsr/core/_hash_backend.py:414-444,457-510 adaptive hierarchy, trilinear weights
 *   jspsr/core/hashtree.py:103-116,157-192      range kernel, interpolated field
 *   jspsr/core/reconstructor.py:59-195          solve_multigrid (RHS, correction, LHS + screening)
 *   jspsr/core/reconstructor.py:197-255         chi, mean-chi level set
 *   jspsr/core/reconstructor.py:296-397         extract_multiscale_mesh
 *   jspsr/bases/bezier_tensor.py:36-121         B-spline basis and its integral tables
 *   csrc/marching_cubes/dual_mc_inds.cu:45-141  dual-cube corner accumulation
 *   csrc/marching_cubes/dual_mc.cu:20-133       dual marching cubes
 * The 1-D integral tables and the marching-cubes triangle table are passed in by the caller
 * (oracle/tables.py, oracle/mc_tables.py).  Parity: tests/test_oracle_fast.py checks this library
 * against oracle/spsr.py, which is pinned by the reference's own golden runs.
 */
#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------- keys and key maps */
#define PACK_OFF (1 << 20)
static inline int64_t pack3(int64_t x, int64_t y, int64_t z) {
  return ((x + PACK_OFF) << 42) | ((y + PACK_OFF) << 21) | (z + PACK_OFF);
}
static inline void unpack3(int64_t k, int32_t* c) {
  const int64_t m = (1 << 21) - 1;
  c[0] = (int32_t)((k >> 42) - PACK_OFF);
  c[1] = (int32_t)(((k >> 21) & m) - PACK_OFF);
  c[2] = (int32_t)((k & m) - PACK_OFF);
}
static inline uint64_t mix64(uint64_t x) {
  x ^= x >> 30;
  x *= 0xbf58476d1ce4e5b9ull;
  x ^= x >> 27;
  x *= 0x94d049bb133111ebull;
  return x ^ (x >> 31);
}

/* Open-addressing map from packed key to row (keys are positive, -1 marks an empty slot); key and
 * value share a 16-byte slot, so a probe touches one cache line. */
typedef struct {
  int64_t k, v;
} Slot;
typedef struct {
  Slot* s;
  int64_t mask;
} Map;

static void map_init(Map* m, int64_t n) {
  int64_t cap = 16;
  while (cap < 2 * n + 16) cap <<= 1;
  m->s = (Slot*)malloc((size_t)cap * sizeof(Slot));
  m->mask = cap - 1;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < cap; i++) m->s[i].k = -1;
}
static void map_free(Map* m) {
  free(m->s);
  m->s = NULL;
}
/* Insert key -> val; returns 1 when the key was new.  Safe to call from several threads. */
static inline int map_put(Map* m, int64_t key, int64_t val) {
  int64_t s = (int64_t)(mix64((uint64_t)key) & (uint64_t)m->mask);
  for (;;) {
    const int64_t prev = __sync_val_compare_and_swap(&m->s[s].k, (int64_t)-1, key);
    if (prev == -1) {
      m->s[s].v = val;
      return 1;
    }
    if (prev == key) return 0;
    s = (s + 1) & m->mask;
  }
}
static inline int64_t map_get(const Map* m, int64_t key) {
  int64_t s = (int64_t)(mix64((uint64_t)key) & (uint64_t)m->mask);
  for (;;) {
    const int64_t k = m->s[s].k;
    if (k == key) return m->s[s].v;
    if (k == -1) return -1;
    s = (s + 1) & m->mask;
  }
}

/* Stable LSD radix sort of non-negative 64-bit keys, 16 bits per pass, threads share each pass. */
static void radix_sort(int64_t* a, int64_t n) {
  if (n < 2) return;
  int64_t* tmp = (int64_t*)malloc((size_t)n * sizeof(int64_t));
  const int nt = omp_get_max_threads();
  int64_t* hist = (int64_t*)malloc((size_t)nt * 65536 * sizeof(int64_t));
  int64_t *src = a, *dst = tmp;
  for (int pass = 0; pass < 4; pass++) {
    const int shift = 16 * pass;
    memset(hist, 0, (size_t)nt * 65536 * sizeof(int64_t));
#pragma omp parallel num_threads(nt)
    {
      const int t = omp_get_thread_num();
      const int64_t lo = n * t / nt, hi = n * (t + 1) / nt;
      int64_t* h = hist + (size_t)t * 65536;
      for (int64_t i = lo; i < hi; i++) h[((uint64_t)src[i] >> shift) & 0xffff]++;
    }
    int64_t run = 0;
    for (int d = 0; d < 65536; d++)
      for (int t = 0; t < nt; t++) {
        const int64_t c = hist[(size_t)t * 65536 + d];
        hist[(size_t)t * 65536 + d] = run;
        run += c;
      }
#pragma omp parallel num_threads(nt)
    {
      const int t = omp_get_thread_num();
      const int64_t lo = n * t / nt, hi = n * (t + 1) / nt;
      int64_t* h = hist + (size_t)t * 65536;
      for (int64_t i = lo; i < hi; i++) dst[h[((uint64_t)src[i] >> shift) & 0xffff]++] = src[i];
    }
    int64_t* sw = src;
    src = dst;
    dst = sw;
  }
  free(hist);
  free(tmp);
}

/* Sorted unique keys of a candidate list (de-duplicated through a key set first, then sorted). */
static int64_t* unique_keys(const int64_t* cand, int64_t n, int64_t* n_out) {
  Map set;
  map_init(&set, n);
  int64_t cnt = 0;
#pragma omp parallel for reduction(+ : cnt) schedule(static)
  for (int64_t i = 0; i < n; i++) cnt += map_put(&set, cand[i], 0);
  int64_t* u = (int64_t*)malloc((size_t)(cnt > 0 ? cnt : 1) * sizeof(int64_t));
  int64_t w = 0;
  for (int64_t s = 0; s <= set.mask; s++)
    if (set.s[s].k != -1) u[w++] = set.s[s].k;
  map_free(&set);
  radix_sort(u, cnt);
  *n_out = cnt;
  return u;
}

/* One level: sorted unique voxel min-corners (finest-voxel units) and a key -> row map. */
typedef struct {
  int64_t n;
  int32_t stride;
  int64_t* keys;
  int32_t* coords;
  Map map;
} Grid;

static void grid_from_keys(Grid* g, int64_t* keys, int64_t n, int stride) {
  g->n = n;
  g->stride = stride;
  g->keys = keys;
  g->coords = (int32_t*)malloc((size_t)(n > 0 ? n : 1) * 3 * sizeof(int32_t));
  map_init(&g->map, n);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; i++) {
    unpack3(keys[i], g->coords + 3 * i);
    map_put(&g->map, keys[i], i);
  }
}
static void grid_free(Grid* g) {
  free(g->keys);
  free(g->coords);
  map_free(&g->map);
}
static inline int64_t grid_row(const Grid* g, int64_t x, int64_t y, int64_t z) {
  return map_get(&g->map, pack3(x, y, z));
}

/* ------------------------------------------------------------------------- basis and tables */
static inline double bspline(double x) {
  if (x >= -1.5 && x < -0.5) return (x + 1.5) * (x + 1.5);
  if (x >= -0.5 && x < 0.5) return -2 * x * x + 1.5;
  if (x >= 0.5 && x < 1.5) return (x - 1.5) * (x - 1.5);
  return 0.0;
}

/* 1-D integral tables per level ratio 2^m (oracle/tables.py): kinds in this order. */
enum { T_SSI, T_SDI, T_DPI, T_PI, T_IDPI, T_IPI, T_KINDS };
typedef struct {
  const double* p[T_KINDS][32];
  int64_t len[T_KINDS][32];
} Tables;

static int ilog2(int64_t v) {
  int m = 0;
  while ((1ll << m) < v) m++;
  return m;
}

/* int grad B_src . grad B_tgt between voxel centres rel (source-stride units), bezier_tensor.py:75-96 */
static inline double deriv_deriv(const Tables* T, const double rel[3], int s_src, int s_tgt) {
  const int M = s_tgt / s_src, m = ilog2(M);
  double c[3], g[3];
  for (int a = 0; a < 3; a++) {
    const int64_t idx = (int64_t)nearbyint(rel[a] + M * 1.5 + 0.5);
    if (idx < 0 || idx >= T->len[T_SSI][m]) return 0.0;
    c[a] = T->p[T_SSI][m][idx] * s_src;
    g[a] = T->p[T_SDI][m][idx] / s_tgt;
  }
  return g[0] * c[1] * c[2] + c[0] * g[1] * c[2] + c[0] * c[1] * g[2];
}

/* int grad B_tgt . data over a data voxel, bezier_tensor.py:98-121 */
static inline double const_deriv(const Tables* T, const double data[3], const double rel[3], int s_data, int s_tgt) {
  const double *dpi, *pi;
  double i_mult, ds;
  int64_t idx[3];
  if (s_tgt >= s_data) {
    const int M = s_tgt / s_data, m = ilog2(M);
    for (int a = 0; a < 3; a++) idx[a] = (int64_t)nearbyint(rel[a] + (3 * M - 1) / 2.0);
    dpi = T->p[T_DPI][m];
    pi = T->p[T_PI][m];
    i_mult = (double)s_data / s_tgt;
    ds = s_data;
  } else {
    const int M = s_data / s_tgt, m = ilog2(M) - 1;
    for (int a = 0; a < 3; a++) idx[a] = (int64_t)nearbyint(rel[a] * M + M / 2.0 + 0.5);
    dpi = T->p[T_IDPI][m];
    pi = T->p[T_IPI][m];
    i_mult = 1.0;
    ds = s_tgt;
  }
  double c[3], g[3];
  for (int a = 0; a < 3; a++) {
    c[a] = dpi[idx[a]] * ds;
    g[a] = pi[idx[a]] * i_mult;
  }
  return data[0] * g[0] * c[1] * c[2] + data[1] * c[0] * g[1] * c[2] + data[2] * c[0] * c[1] * g[2];
}

/* Ordered offsets of an n^3 range: Chebyshev shells outward, lexicographic inside a shell. */
static int range_kernel(int n, int32_t* out) {
  const int r = n / 2;
  int w = 0;
  for (int shell = 0; shell <= r; shell++)
    for (int x = -r; x <= r; x++)
      for (int y = -r; y <= r; y++)
        for (int z = -r; z <= r; z++) {
          const int ax = abs(x), ay = abs(y), az = abs(z);
          const int s = ax > ay ? (ax > az ? ax : az) : (ay > az ? ay : az);
          if (s != shell) continue;
          out[3 * w] = x;
          out[3 * w + 1] = y;
          out[3 * w + 2] = z;
          w++;
        }
  return w;
}

/* ------------------------------------------------------------------------- point geometry */
static const int CONFORM[8][3] = {{0, 0, 0}, {0, 0, 1}, {0, 1, 0}, {0, 1, 1},
                                  {1, 0, 0}, {1, 0, 1}, {1, 1, 0}, {1, 1, 1}};

/* 8 trilinear corner cells and weights of one point (_hash_backend.py:469-510): corner cells from
 * the float32 quantisation, weights in FP64. */
static inline void trilinear(const float* q32, const double* q64, int stride, int32_t corners[8][3], double w[8]) {
  const float s = (float)stride;
  int d[3], sg[3];
  double loc[3];
  for (int a = 0; a < 3; a++) {
    const float d32 = floorf(q32[a] / s) * s;
    const float rel = (q32[a] - d32) - (float)(stride / 2.0);
    sg[a] = rel > 0.f ? 1 : (rel < 0.f ? -1 : 0);
    d[a] = (int)d32;
    loc[a] = fabs(q64[a] - (double)d32 - stride / 2.0) / stride;
  }
  for (int c = 0; c < 8; c++) {
    for (int a = 0; a < 3; a++) corners[c][a] = d[a] + CONFORM[c][a] * sg[a] * stride;
    w[c] = (CONFORM[c][0] ? loc[0] : 1 - loc[0]) * (CONFORM[c][1] ? loc[1] : 1 - loc[1]) *
           (CONFORM[c][2] ? loc[2] : 1 - loc[2]);
  }
}

/* Basis neighbours of a point query at a level (the 27-offset get_neighbours_data of
 * hashtree.py:169-181 with source xyz / vs - 0.5): rows and B-spline values, in kernel order. */
static inline int point_basis(const Grid* g, const int32_t* k27, const float* q32, const double* q64,
                              int64_t rows[27], double phi[27]) {
  const int s = g->stride;
  int quant[3];
  for (int a = 0; a < 3; a++) {
    const float pos = q32[a] - 0.5f;
    quant[a] = (int)(floorf((pos + 0.5f) / (float)s) * (float)s);
  }
  int w = 0;
  for (int k = 0; k < 27; k++) {
    const int64_t r = grid_row(g, quant[0] + (int64_t)k27[3 * k] * s, quant[1] + (int64_t)k27[3 * k + 1] * s,
                               quant[2] + (int64_t)k27[3 * k + 2] * s);
    if (r < 0) continue;
    double b = 1.0;
    for (int a = 0; a < 3; a++) {
      const double nt = (double)k27[3 * k + a] * s + (quant[a] - (q64[a] - 0.5)) + (s - 1) / 2.0;
      b *= bspline(-nt / s);
    }
    rows[w] = r;
    phi[w] = b;
    w++;
  }
  return w;
}

/* Per-point basis data of one level, 27 slots per point (row -1 = absent). */
typedef struct {
  int64_t* rows;
  double* phi;
} PointBasis;

static void point_basis_all(PointBasis* pb, const Grid* g, const int32_t* k27, const float* q32, const double* q64,
                            int64_t n) {
  pb->rows = (int64_t*)malloc((size_t)n * 27 * sizeof(int64_t));
  pb->phi = (double*)malloc((size_t)n * 27 * sizeof(double));
#pragma omp parallel for schedule(static)
  for (int64_t p = 0; p < n; p++) {
    int64_t r[27];
    double f[27];
    const int c = point_basis(g, k27, q32 + 3 * p, q64 + 3 * p, r, f);
    for (int k = 0; k < 27; k++) {
      pb->rows[p * 27 + k] = k < c ? r[k] : -1;
      pb->phi[p * 27 + k] = k < c ? f[k] : 0.0;
    }
  }
}

static inline void atomic_add(double* p, double v) {
#pragma omp atomic
  *p += v;
}

/* ------------------------------------------------------------------------- sparse matrices */
typedef struct {
  int64_t n, nnz;
  int64_t* rowptr;
  int32_t* cols;
  double* vals;
} Csr;

static void csr_free(Csr* a) {
  free(a->rowptr);
  free(a->cols);
  free(a->vals);
}

/* slot of column c in row i (columns sorted), or -1 */
static inline int64_t csr_slot(const Csr* a, int64_t i, int64_t c) {
  int64_t lo = a->rowptr[i], hi = a->rowptr[i + 1];
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if (a->cols[mid] < c) lo = mid + 1;
    else hi = mid;
  }
  return lo < a->rowptr[i + 1] && a->cols[lo] == c ? lo : -1;
}

/* Same-level stiffness over the range-5 stencil (reconstructor.py:170-179), columns sorted. */
static void stiffness_same_level(Csr* A, const Grid* g, const Tables* T, const int32_t* k125) {
  const int64_t n = g->n;
  const int s = g->stride;
  double kval[125];
  for (int k = 0; k < 125; k++) {
    const double rel[3] = {k125[3 * k], k125[3 * k + 1], k125[3 * k + 2]};
    kval[k] = deriv_deriv(T, rel, s, s);
  }
  A->n = n;
  A->rowptr = (int64_t*)malloc((size_t)(n + 1) * sizeof(int64_t));
  int64_t* cnt = (int64_t*)malloc((size_t)(n > 0 ? n : 1) * sizeof(int64_t));
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; i++) {
    const int32_t* c = g->coords + 3 * i;
    int64_t m = 0;
    for (int k = 0; k < 125; k++)
      m += grid_row(g, c[0] + (int64_t)k125[3 * k] * s, c[1] + (int64_t)k125[3 * k + 1] * s,
                    c[2] + (int64_t)k125[3 * k + 2] * s) >= 0;
    cnt[i] = m;
  }
  A->rowptr[0] = 0;
  for (int64_t i = 0; i < n; i++) A->rowptr[i + 1] = A->rowptr[i] + cnt[i];
  free(cnt);
  A->nnz = A->rowptr[n];
  A->cols = (int32_t*)malloc((size_t)(A->nnz > 0 ? A->nnz : 1) * sizeof(int32_t));
  A->vals = (double*)malloc((size_t)(A->nnz > 0 ? A->nnz : 1) * sizeof(double));
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; i++) {
    const int32_t* c = g->coords + 3 * i;
    int32_t cc[125];
    double vv[125];
    int m = 0;
    for (int k = 0; k < 125; k++) {
      const int64_t r = grid_row(g, c[0] + (int64_t)k125[3 * k] * s, c[1] + (int64_t)k125[3 * k + 1] * s,
                                 c[2] + (int64_t)k125[3 * k + 2] * s);
      if (r < 0) continue;
      int j = m++;
      while (j > 0 && cc[j - 1] > r) {       /* insertion sort by column */
        cc[j] = cc[j - 1];
        vv[j] = vv[j - 1];
        j--;
      }
      cc[j] = (int32_t)r;
      vv[j] = kval[k];
    }
    memcpy(A->cols + A->rowptr[i], cc, (size_t)m * sizeof(int32_t));
    memcpy(A->vals + A->rowptr[i], vv, (size_t)m * sizeof(double));
  }
}

/* A += scale * Phi^T W Phi on A's pattern (the screening Gram, reconstructor.py:59-77,180-183). */
static void add_gram(Csr* A, const PointBasis* pb, int64_t npts, double scale) {
#pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t p = 0; p < npts; p++) {
    const int64_t* r = pb->rows + p * 27;
    const double* f = pb->phi + p * 27;
    for (int a = 0; a < 27 && r[a] >= 0; a++)
      for (int b = 0; b < 27 && r[b] >= 0; b++) {
        const int64_t slot = csr_slot(A, r[a], r[b]);
        if (slot >= 0) atomic_add(A->vals + slot, scale * f[a] * f[b]);
      }
  }
}

static void spmv(const Csr* A, const double* x, double* y) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < A->n; i++) {
    double s = 0.0;
    for (int64_t j = A->rowptr[i]; j < A->rowptr[i + 1]; j++) s += A->vals[j] * x[A->cols[j]];
    y[i] = s;
  }
}
static double dot(const double* a, const double* b, int64_t n) {
  double s = 0.0;
#pragma omp parallel for reduction(+ : s) schedule(static)
  for (int64_t i = 0; i < n; i++) s += a[i] * b[i];
  return s;
}

/* Jacobi-preconditioned CG in FP64 from x = 0 to |r| <= tol |b| (scipy.sparse.linalg.cg, rtol). */
static int cg64(const Csr* A, const double* b, double* x, double tol, int maxiter) {
  const int64_t n = A->n;
  double* dinv = (double*)malloc((size_t)n * sizeof(double));
  double* r = (double*)malloc((size_t)n * sizeof(double));
  double* z = (double*)malloc((size_t)n * sizeof(double));
  double* p = (double*)malloc((size_t)n * sizeof(double));
  double* q = (double*)malloc((size_t)n * sizeof(double));
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; i++) {
    const int64_t slot = csr_slot(A, i, i);
    dinv[i] = 1.0 / A->vals[slot];
    x[i] = 0.0;
    r[i] = b[i];
    p[i] = 0.0;
  }
  const double atol = tol * sqrt(dot(b, b, n));
  double rho = 0.0, rho_prev = 0.0;
  int it = 0;
  while (it < maxiter && sqrt(dot(r, r, n)) > atol) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; i++) z[i] = dinv[i] * r[i];
    rho_prev = rho;
    rho = dot(r, z, n);
    const double beta = it == 0 ? 0.0 : rho / rho_prev;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; i++) p[i] = z[i] + beta * p[i];
    spmv(A, p, q);
    const double alpha = rho / dot(p, q, n);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; i++) {
      x[i] += alpha * p[i];
      r[i] -= alpha * q[i];
    }
    it++;
  }
  free(dinv);
  free(r);
  free(z);
  free(p);
  free(q);
  return it;
}

/* ------------------------------------------------------------------------- the reconstruction */
#define MAX_LEVELS 24

typedef struct {
  /* inputs */
  int64_t n;
  int depth;
  double vs;
  /* per point */
  double* density;
  int32_t* level;
  /* per level */
  Grid grid[MAX_LEVELS];
  double* normals[MAX_LEVELS]; /* splatted normal data [V,3] or NULL */
  double* rhs[MAX_LEVELS];
  double* x[MAX_LEVELS];
  Csr lhs[MAX_LEVELS];
  int iters[MAX_LEVELS];
  /* mesh */
  double mean_chi;
  int64_t n_primal, n_dual, n_cubes, n_verts, n_faces;
  double* dual_values; /* [n_primal] */
  double* dual_pos;    /* [n_primal, 3] */
  int32_t* cubes;      /* [n_cubes, 8] complete dual cubes (primal ids) */
  double* verts;       /* [n_verts, 3] */
  int64_t* faces;      /* [n_faces, 3] */
  int64_t* vkeys;      /* [n_verts] (larger id << 32 | smaller id) of each vertex's primal-sample pair */
  double seconds[8];   /* stage times: tree, assembly+solve, mesh; mesh parts: dual centres, accumulation, field, MC */
} Ctx;

static void scale_points(const float* xyz, int64_t n, double vs, float* q32, double* q64) {
  const float inv = 1.0f / (float)vs;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < 3 * n; i++) {
    q32[i] = xyz[i] * inv;
    q64[i] = (double)xyz[i] / vs;
  }
}

/* Unique trilinear corner cells at `stride` of the points selected by `sel` (all when NULL). */
static void corner_grid(Grid* g, const float* q32, const double* q64, int64_t n, const uint8_t* sel, int stride) {
  int64_t* cand = (int64_t*)malloc((size_t)(n > 0 ? n : 1) * 8 * sizeof(int64_t));
  int64_t m = 0;
  int64_t* idx = (int64_t*)malloc((size_t)(n > 0 ? n : 1) * sizeof(int64_t));
  for (int64_t p = 0; p < n; p++)
    if (!sel || sel[p]) idx[m++] = p;
#pragma omp parallel for schedule(static)
  for (int64_t t = 0; t < m; t++) {
    int32_t c[8][3];
    double w[8];
    trilinear(q32 + 3 * idx[t], q64 + 3 * idx[t], stride, c, w);
    for (int k = 0; k < 8; k++) cand[8 * t + k] = pack3(c[k][0], c[k][1], c[k][2]);
  }
  int64_t nu = 0;
  int64_t* keys = unique_keys(cand, 8 * m, &nu);
  free(cand);
  free(idx);
  grid_from_keys(g, keys, nu, stride);
}

static void compute_density(Ctx* C, const float* xyz, const int32_t* k27) {
  const int64_t n = C->n;
  const double vsd = 4 * C->vs;
  float* q32 = (float*)malloc((size_t)n * 3 * sizeof(float));
  double* q64 = (double*)malloc((size_t)n * 3 * sizeof(double));
  scale_points(xyz, n, vsd, q32, q64);
  Grid g;
  corner_grid(&g, q32, q64, n, NULL, 1);
  double* wd = (double*)calloc((size_t)(g.n > 0 ? g.n : 1), sizeof(double));
  /* corner-major accumulation, as np.bincount over the (8 N) corner list */
  int64_t* rows = (int64_t*)malloc((size_t)n * 8 * sizeof(int64_t));
  double* ws = (double*)malloc((size_t)n * 8 * sizeof(double));
#pragma omp parallel for schedule(static)
  for (int64_t p = 0; p < n; p++) {
    int32_t c[8][3];
    double w[8];
    trilinear(q32 + 3 * p, q64 + 3 * p, 1, c, w);
    for (int k = 0; k < 8; k++) {
      rows[k * n + p] = grid_row(&g, c[k][0], c[k][1], c[k][2]);
      ws[k * n + p] = w[k];
    }
  }
  for (int64_t t = 0; t < 8 * n; t++) wd[rows[t]] += ws[t];
  free(rows);
  free(ws);
  C->density = (double*)malloc((size_t)n * sizeof(double));
#pragma omp parallel for schedule(static)
  for (int64_t p = 0; p < n; p++) {
    int64_t r[27];
    double f[27];
    const int c = point_basis(&g, k27, q32 + 3 * p, q64 + 3 * p, r, f);
    double s = 0.0;
    for (int k = 0; k < c; k++) s += f[k] * wd[r[k]];
    C->density[p] = s / 16.0;
  }
  free(wd);
  grid_free(&g);
  free(q32);
  free(q64);
}

/* Pairs between a finer (or equal) source level and a coarser (or equal) target level over a
 * (rng)^3 range (voxel_neighbours of the non-conv query, _hash_backend.py:191-228): calls fn(si,
 * ti, rel) for every pair, rel = (c_tgt - c_src) / s_src between centres, source by source. */
#define FOR_PAIRS_FINE_TO_COARSE(SRC, TGT, KER, NK, ...)                                           \
  do {                                                                                             \
    const int ss_ = (SRC)->stride, st_ = (TGT)->stride;                                            \
    _Pragma("omp parallel for schedule(static)") for (int64_t si = 0; si < (SRC)->n; si++) {       \
      const int32_t* sc_ = (SRC)->coords + 3 * si;                                                 \
      int64_t q_[3];                                                                               \
      double coff_[3];                                                                             \
      for (int a_ = 0; a_ < 3; a_++) {                                                             \
        q_[a_] = (int64_t)(floor((sc_[a_] + 0.5 * ss_) / st_) * st_);                              \
        coff_[a_] = (double)(q_[a_] - sc_[a_]) / ss_ + (st_ / ss_ - 1) / 2.0;                      \
      }                                                                                            \
      for (int k_ = 0; k_ < (NK); k_++) {                                                          \
        const int64_t ti = grid_row((TGT), q_[0] + (int64_t)(KER)[3 * k_] * st_,                   \
                                    q_[1] + (int64_t)(KER)[3 * k_ + 1] * st_,                      \
                                    q_[2] + (int64_t)(KER)[3 * k_ + 2] * st_);                     \
        if (ti < 0) continue;                                                                      \
        double rel[3];                                                                             \
        for (int a_ = 0; a_ < 3; a_++) rel[a_] = (double)(KER)[3 * k_ + a_] * (st_ / ss_) + coff_[a_]; \
        __VA_ARGS__                                                                                \
      }                                                                                            \
    }                                                                                              \
  } while (0)

static void level_rhs(Ctx* C, int d, const Tables* T, const int32_t* k27, const int32_t* k125,
                      const PointBasis* pbs, int64_t npts, double alpha, double delta) {
  const Grid* gd = &C->grid[d];
  const int64_t n = gd->n;
  double* rhs = (double*)calloc((size_t)(n > 0 ? n : 1), sizeof(double));
  const double sf = pow(0.25, d);
  /* divergence of the splatted normals of every data level (reconstructor.py:126-141) */
  for (int dd = 0; dd < C->depth; dd++) {
    if (!C->normals[dd]) continue;
    const Grid* gdd = &C->grid[dd];
    const double* nd = C->normals[dd];
    if (dd <= d) {
      /* data voxel (source, finer) -> target voxels (coarser) */
      FOR_PAIRS_FINE_TO_COARSE(gdd, gd, k27, 27, {
        const double data[3] = {-nd[3 * si], -nd[3 * si + 1], -nd[3 * si + 2]};
        atomic_add(rhs + ti, const_deriv(T, data, rel, gdd->stride, gd->stride));
      });
    } else {
      /* coarser data: query fine target -> coarse data, keep near pairs, offsets in data units
       * (the inversion of _hash_backend.py:270-290) */
      const int s_f = gd->stride, s_c = gdd->stride;
      FOR_PAIRS_FINE_TO_COARSE(gd, gdd, k27, 27, {
        int near = 1;
        for (int a = 0; a < 3; a++) near &= fabs(rel[a]) < 3 / 2.0 + 1.0e-6;
        if (near) {
          double r2[3];
          for (int a = 0; a < 3; a++) r2[a] = -rel[a] / s_c * s_f;
          const double data[3] = {-nd[3 * ti], -nd[3 * ti + 1], -nd[3 * ti + 2]};
          atomic_add(rhs + si, const_deriv(T, data, r2, s_c, s_f));
        }
      });
    }
  }
  /* screening target (reconstructor.py:143-151) */
  if (alpha > 0) {
    const PointBasis* pb = &pbs[d];
#pragma omp parallel for schedule(static)
    for (int64_t p = 0; p < npts; p++)
      for (int k = 0; k < 27 && pb->rows[p * 27 + k] >= 0; k++)
        atomic_add(rhs + pb->rows[p * 27 + k], sf * alpha * delta * pb->phi[p * 27 + k]);
  }
  /* coarser solutions through the cross-level stiffness and screening (reconstructor.py:153-168) */
  for (int dd = C->depth - 1; dd > d; dd--) {
    const Grid* gc = &C->grid[dd];
    const double* xc = C->x[dd];
    FOR_PAIRS_FINE_TO_COARSE(gd, gc, k125, 125, {
      rhs[si] -= deriv_deriv(T, rel, gd->stride, gc->stride) * xc[ti];
    });
    if (alpha > 0) {
      const PointBasis *pf = &pbs[d], *pc = &pbs[dd];
#pragma omp parallel for schedule(static)
      for (int64_t p = 0; p < npts; p++) {
        double f = 0.0;
        for (int k = 0; k < 27 && pc->rows[p * 27 + k] >= 0; k++) f += pc->phi[p * 27 + k] * xc[pc->rows[p * 27 + k]];
        for (int k = 0; k < 27 && pf->rows[p * 27 + k] >= 0; k++)
          atomic_add(rhs + pf->rows[p * 27 + k], -sf * alpha * pf->phi[p * 27 + k] * f);
      }
    }
  }
  C->rhs[d] = rhs;
  (void)k125;
}

/* chi_raw at positions (sum over levels of the interpolated field, reconstructor.py:197-226). */
static void chi_raw(const Ctx* C, const float* pos32, const double* pos64, int64_t m, const int32_t* k27,
                    double* out) {
  const float inv = 1.0f / (float)C->vs;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < m; i++) {
    float q32[3];
    double q64[3];
    for (int a = 0; a < 3; a++) {
      q32[a] = pos32[3 * i + a] * inv;
      q64[a] = pos64[3 * i + a] / C->vs;
    }
    double s = 0.0;
    for (int d = C->depth - 1; d >= 0; d--) {
      int64_t r[27];
      double f[27];
      const int c = point_basis(&C->grid[d], k27, q32, q64, r, f);
      double sd = 0.0;
      for (int k = 0; k < c; k++) sd += f[k] * C->x[d][r[k]];
      s += sd;
    }
    out[i] = s;
  }
}

/* ------------------------------------------------------------------------- mesh */
static const int MC_CORNER[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0},
                                    {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
static const int MC_EDGES[12][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {4, 5}, {5, 6},
                                    {6, 7}, {7, 4}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};

static inline int octant_slot(int ox, int oy, int oz) {
  for (int i = 0; i < 8; i++)
    if (MC_CORNER[i][0] == ox && MC_CORNER[i][1] == oy && MC_CORNER[i][2] == oz) return i;
  return -1;
}

/* Edge vertex with the reference's 1e-5 snapping (dual_mc.cu:20-31). */
static inline void interp(const double* p1, const double* p2, double v1, double v2, double* out) {
  const double w2 = fabs(v2 - v1) > 0 ? -v1 / (v2 - v1) : 0.0;
  for (int a = 0; a < 3; a++) out[a] = p1[a] * (1 - w2) + p2[a] * w2;
  const int snap1 = fabs(v1) < 1e-5 || (fabs(v2) >= 1e-5 && fabs(v1 - v2) < 1e-5);
  const int snap2 = !(fabs(v1) < 1e-5) && fabs(v2) < 1e-5;
  if (snap1)
    for (int a = 0; a < 3; a++) out[a] = p1[a];
  if (snap2)
    for (int a = 0; a < 3; a++) out[a] = p2[a];
}

static int cmp_i64(const void* a, const void* b) {
  const int64_t x = *(const int64_t*)a, y = *(const int64_t*)b;
  return x < y ? -1 : x > y;
}

static void extract_mesh(Ctx* C, const float* xyz, const int32_t* k27, const int32_t* tri_table, int n_up) {
  const int L = C->depth;
  int max_depth = L;
  /* conformal leaves per level (reconstructor.py:319-336) */
  int32_t* base[MAX_LEVELS] = {0};
  int64_t nbase[MAX_LEVELS] = {0};
  uint8_t* keep[MAX_LEVELS] = {0};
  for (int d = 0; d < L; d++) {
    const Grid* g = &C->grid[d];
    const int s = g->stride;
    int32_t* cells;
    int64_t nc;
    if (d < max_depth - 1) {
      int64_t* pk = (int64_t*)malloc((size_t)(g->n > 0 ? g->n : 1) * sizeof(int64_t));
#pragma omp parallel for schedule(static)
      for (int64_t i = 0; i < g->n; i++) {
        int64_t c[3];
        for (int a = 0; a < 3; a++) c[a] = (int64_t)floor(g->coords[3 * i + a] / (double)s / 2.0) * s * 2;
        pk[i] = pack3(c[0], c[1], c[2]);
      }
      int64_t npar = 0;
      int64_t* par = unique_keys(pk, g->n, &npar);
      free(pk);
      nc = npar * 8;
      cells = (int32_t*)malloc((size_t)(nc > 0 ? nc : 1) * 3 * sizeof(int32_t));
#pragma omp parallel for schedule(static)
      for (int64_t i = 0; i < npar; i++) {
        int32_t c[3];
        unpack3(par[i], c);
        for (int k = 0; k < 8; k++)
          for (int a = 0; a < 3; a++) cells[(8 * i + k) * 3 + a] = c[a] + CONFORM[k][a] * s;
      }
      free(par);
    } else {
      nc = g->n;
      cells = (int32_t*)malloc((size_t)(nc > 0 ? nc : 1) * 3 * sizeof(int32_t));
      memcpy(cells, g->coords, (size_t)nc * 3 * sizeof(int32_t));
    }
    if (d > 0) {
      /* cells not present among the finer level's cells */
      Map finer;
      map_init(&finer, nbase[d - 1]);
      const int32_t* fb = base[d - 1];
#pragma omp parallel for schedule(static)
      for (int64_t i = 0; i < nbase[d - 1]; i++) map_put(&finer, pack3(fb[3 * i], fb[3 * i + 1], fb[3 * i + 2]), i);
      uint8_t* ol = (uint8_t*)malloc((size_t)(nc > 0 ? nc : 1));
      int64_t any = 0;
#pragma omp parallel for reduction(+ : any) schedule(static)
      for (int64_t i = 0; i < nc; i++) {
        ol[i] = map_get(&finer, pack3(cells[3 * i], cells[3 * i + 1], cells[3 * i + 2])) < 0;
        any += ol[i];
      }
      map_free(&finer);
      if (!any) {
        free(ol);
        free(cells);
        max_depth = d;
        break;
      }
      keep[d] = ol;
    }
    base[d] = cells;
    nbase[d] = nc;
  }
  for (int d = 1; d < max_depth; d++) {
    int64_t w = 0;
    for (int64_t i = 0; i < nbase[d]; i++)
      if (keep[d][i]) {
        for (int a = 0; a < 3; a++) base[d][3 * w + a] = base[d][3 * i + a];
        w++;
      }
    nbase[d] = w;
    free(keep[d]);
  }
  /* expanded primal samples, their positions, and the dual centres (unique sample corners) */
  const int e3 = n_up * n_up * n_up;
  int64_t start[MAX_LEVELS + 1];
  start[0] = 0;
  for (int d = 0; d < max_depth; d++) start[d + 1] = start[d] + nbase[d] * e3;
  const int64_t np = start[max_depth];
  int32_t* epb = (int32_t*)malloc((size_t)(np > 0 ? np : 1) * 3 * sizeof(int32_t));
  int32_t* lvl_of = (int32_t*)malloc((size_t)(np > 0 ? np : 1) * sizeof(int32_t));
  for (int d = 0; d < max_depth; d++) {
    const int s = C->grid[d].stride;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < nbase[d]; i++)
      for (int e = 0; e < e3; e++) {
        const int ex[3] = {e / (n_up * n_up), (e / n_up) % n_up, e % n_up};
        const int64_t o = start[d] + i * e3 + e;
        for (int a = 0; a < 3; a++) epb[3 * o + a] = base[d][3 * i + a] * n_up + ex[a] * s;
        lvl_of[o] = d;
      }
    free(base[d]);
  }
  int64_t* cand = (int64_t*)malloc((size_t)(np > 0 ? np : 1) * 8 * sizeof(int64_t));
#pragma omp parallel for schedule(static)
  for (int64_t o = 0; o < np; o++) {
    const int s = C->grid[lvl_of[o]].stride;
    for (int k = 0; k < 8; k++)
      cand[8 * o + k] = pack3(epb[3 * o] + CONFORM[k][0] * s, epb[3 * o + 1] + CONFORM[k][1] * s,
                              epb[3 * o + 2] + CONFORM[k][2] * s);
  }
  int64_t nd = 0;
  int64_t* dkeys = unique_keys(cand, 8 * np, &nd);
  free(cand);
  Grid dual;
  grid_from_keys(&dual, dkeys, nd, 1);
  C->seconds[5] = omp_get_wtime();
  /* dual-cube corner accumulation (dual_mc_inds.cu:45-141): corners, edge points, face points */
  int32_t* acc = (int32_t*)malloc((size_t)(nd > 0 ? nd : 1) * 8 * sizeof(int32_t));
  int32_t* cnt = (int32_t*)calloc((size_t)(nd > 0 ? nd : 1), sizeof(int32_t));
#pragma omp parallel for schedule(dynamic, 256)
  for (int64_t o = 0; o < np; o++) {
    const int s = C->grid[lvl_of[o]].stride;
    const int32_t* pbp = epb + 3 * o;
    const int32_t pid = (int32_t)o;
#define ACC_POINT(X, Y, Z, NO, OCTS)                                  \
  do {                                                                \
    const int64_t row_ = grid_row(&dual, (X), (Y), (Z));              \
    if (row_ >= 0) {                                                  \
      __sync_fetch_and_add(cnt + row_, (NO));                         \
      for (int t_ = 0; t_ < (NO); t_++) acc[row_ * 8 + (OCTS)[t_]] = pid; \
    }                                                                 \
  } while (0)
    for (int c = 0; c < 8; c++) {
      const int cx = (c >> 2) & 1, cy = (c >> 1) & 1, cz = c & 1;
      const int oc[1] = {octant_slot(1 - cx, 1 - cy, 1 - cz)};
      ACC_POINT(pbp[0] + cx * s, pbp[1] + cy * s, pbp[2] + cz * s, 1, oc);
    }
    for (int a = 0; a < 3; a++) {
      const int b0 = a == 0 ? 1 : 0, b1 = a == 2 ? 1 : 2;
      for (int v0 = 0; v0 < 2; v0++)
        for (int v1 = 0; v1 < 2; v1++)
          for (int t = 1; t < s; t++) {
            int off[3], oc[2];
            off[b0] = v0 * s;
            off[b1] = v1 * s;
            off[a] = t;
            for (int oa = 0; oa < 2; oa++) {
              int oo[3];
              oo[b0] = 1 - v0;
              oo[b1] = 1 - v1;
              oo[a] = oa;
              oc[oa] = octant_slot(oo[0], oo[1], oo[2]);
            }
            ACC_POINT(pbp[0] + off[0], pbp[1] + off[1], pbp[2] + off[2], 2, oc);
          }
    }
    for (int a = 0; a < 3; a++) {
      const int b0 = a == 0 ? 1 : 0, b1 = a == 2 ? 1 : 2;
      for (int side = 0; side < 2; side++)
        for (int u = 1; u < s; u++)
          for (int v = 1; v < s; v++) {
            int off[3], oc[4], w = 0;
            off[a] = side * s;
            off[b0] = u;
            off[b1] = v;
            for (int o0 = 0; o0 < 2; o0++)
              for (int o1 = 0; o1 < 2; o1++) {
                int oo[3];
                oo[a] = 1 - side;
                oo[b0] = o0;
                oo[b1] = o1;
                oc[w++] = octant_slot(oo[0], oo[1], oo[2]);
              }
            ACC_POINT(pbp[0] + off[0], pbp[1] + off[1], pbp[2] + off[2], 4, oc);
          }
    }
#undef ACC_POINT
  }
  grid_free(&dual);
  C->seconds[3] = omp_get_wtime();
  /* field at the primal samples, minus the mean chi at the input points */
  double* pos64 = (double*)malloc((size_t)(np > 0 ? np : 1) * 3 * sizeof(double));
  float* pos32 = (float*)malloc((size_t)(np > 0 ? np : 1) * 3 * sizeof(float));
  const double evs = C->vs / n_up;
  const float evs32 = (float)evs;
#pragma omp parallel for schedule(static)
  for (int64_t o = 0; o < np; o++) {
    const int s = C->grid[lvl_of[o]].stride;
    for (int a = 0; a < 3; a++) {
      pos64[3 * o + a] = (double)(epb[3 * o + a] + s) * evs;
      pos32[3 * o + a] = (float)(epb[3 * o + a] + s) * evs32;
    }
  }
  {
    double* xyz64 = (double*)malloc((size_t)C->n * 3 * sizeof(double));
    double* chi = (double*)malloc((size_t)C->n * sizeof(double));
    for (int64_t i = 0; i < 3 * C->n; i++) xyz64[i] = xyz[i];
    chi_raw(C, xyz, xyz64, C->n, k27, chi);
    double sw = 0.0, swc = 0.0;
    for (int64_t i = 0; i < C->n; i++) {
      const double w = 1.0 / C->density[i];
      swc += chi[i] * w;
      sw += w;
    }
    C->mean_chi = swc / sw;
    free(xyz64);
    free(chi);
  }
  double* vals = (double*)malloc((size_t)(np > 0 ? np : 1) * sizeof(double));
  chi_raw(C, pos32, pos64, np, k27, vals);
#pragma omp parallel for schedule(static)
  for (int64_t o = 0; o < np; o++) vals[o] -= C->mean_chi;
  free(pos32);
  C->seconds[4] = omp_get_wtime();
  /* complete cubes in dual order, their triangles and vertex ids (dual_mc.cu:33-133) */
  int64_t* tri_off = (int64_t*)malloc((size_t)(nd + 1) * sizeof(int64_t));
  int64_t ncubes = 0;
  for (int64_t r = 0; r < nd; r++) ncubes += cnt[r] == 8;
  int32_t* cubes = (int32_t*)malloc((size_t)(ncubes > 0 ? ncubes : 1) * 8 * sizeof(int32_t));
  int64_t* ctype = (int64_t*)malloc((size_t)(ncubes > 0 ? ncubes : 1) * sizeof(int64_t));
  {
    int64_t w = 0;
    for (int64_t r = 0; r < nd; r++)
      if (cnt[r] == 8) memcpy(cubes + 8 * w++, acc + 8 * r, 8 * sizeof(int32_t));
  }
  free(acc);
  free(cnt);
  tri_off[0] = 0;
  for (int64_t c = 0; c < ncubes; c++) {
    int64_t t = 0;
    for (int i = 0; i < 8; i++) t |= (int64_t)(vals[cubes[8 * c + i]] < 0) << i;
    ctype[c] = t;
    int nv = 0;
    while (nv < 16 && tri_table[t * 16 + nv] != -1) nv++;
    tri_off[c + 1] = tri_off[c] + nv / 3;
  }
  const int64_t ntri = tri_off[ncubes];
  double* tris = (double*)malloc((size_t)(ntri > 0 ? ntri : 1) * 9 * sizeof(double));
  int64_t* vkey = (int64_t*)malloc((size_t)(ntri > 0 ? ntri : 1) * 3 * sizeof(int64_t));
#pragma omp parallel for schedule(static)
  for (int64_t c = 0; c < ncubes; c++) {
    const int32_t* ids = cubes + 8 * c;
    for (int64_t t = tri_off[c]; t < tri_off[c + 1]; t++)
      for (int j = 0; j < 3; j++) {
        const int e = tri_table[ctype[c] * 16 + 3 * (t - tri_off[c]) + j];
        const int a = MC_EDGES[e][0], b = MC_EDGES[e][1];
        const int64_t ia = ids[a], ib = ids[b];
        interp(pos64 + 3 * ia, pos64 + 3 * ib, vals[ia], vals[ib], tris + 9 * t + 3 * j);
        const int64_t hi = ia > ib ? ia : ib, lo = ia > ib ? ib : ia;
        vkey[3 * t + j] = (hi << 32) | lo;
      }
  }
  free(ctype);
  free(tri_off);
  /* vertices: unique (vid0, vid1) keys in sorted order, each at its first occurrence */
  const int64_t nk = 3 * ntri;
  int64_t* sk = (int64_t*)malloc((size_t)(nk > 0 ? nk : 1) * sizeof(int64_t));
  memcpy(sk, vkey, (size_t)nk * sizeof(int64_t));
  radix_sort(sk, nk);
  int64_t nu = 0;
  for (int64_t i = 0; i < nk; i++)
    if (i == 0 || sk[i] != sk[i - 1]) sk[nu++] = sk[i];
  Map vmap;
  map_init(&vmap, nu);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < nu; i++) map_put(&vmap, sk[i], i);
  C->n_verts = nu;
  C->n_faces = ntri;
  C->vkeys = (int64_t*)malloc((size_t)(nu > 0 ? nu : 1) * sizeof(int64_t));
  memcpy(C->vkeys, sk, (size_t)nu * sizeof(int64_t));
  C->verts = (double*)malloc((size_t)(nu > 0 ? nu : 1) * 3 * sizeof(double));
  C->faces = (int64_t*)malloc((size_t)(nk > 0 ? nk : 1) * sizeof(int64_t));
  int64_t* first = (int64_t*)malloc((size_t)(nu > 0 ? nu : 1) * sizeof(int64_t));
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < nu; i++) first[i] = INT64_MAX;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < nk; i++) {
    const int64_t v = map_get(&vmap, vkey[i]);
    C->faces[i] = v;
    int64_t cur = first[v];
    while (i < cur && !__sync_bool_compare_and_swap(first + v, cur, i)) cur = first[v];
  }
#pragma omp parallel for schedule(static)
  for (int64_t v = 0; v < nu; v++)
    for (int a = 0; a < 3; a++) C->verts[3 * v + a] = tris[3 * first[v] + a];
  map_free(&vmap);
  free(first);
  free(sk);
  free(vkey);
  free(tris);
  free(epb);
  free(lvl_of);
  C->n_primal = np;
  C->n_dual = nd;
  C->n_cubes = ncubes;
  C->cubes = cubes;
  C->dual_values = vals;
  C->dual_pos = pos64;
  (void)cmp_i64;
}

/* ------------------------------------------------------------------------- entry points */
/* tables: T_KINDS x n_mult arrays packed back to back; lens[T_KINDS * n_mult] their lengths.
 * tri_table: int32 [256 * 16].  Returns a context (NULL on bad arguments); free with spsr_free. */
void* spsr_reconstruct(const float* xyz, const float* nrm, int64_t n, double vs, int depth, double min_density,
                       double alpha, double delta, double cg_tol, int cg_maxiter, int n_up, const double* tables,
                       const int64_t* lens, int n_mult, const int32_t* tri_table, int threads, int mesh) {
  if (n <= 0 || depth < 1 || depth > MAX_LEVELS || n_mult < depth || n_mult > 32 || !xyz || !nrm) return NULL;
  if (threads > 0) omp_set_num_threads(threads);
  Ctx* C = (Ctx*)calloc(1, sizeof(Ctx));
  C->n = n;
  C->depth = depth;
  C->vs = vs;
  Tables T;
  memset(&T, 0, sizeof(T));
  {
    const double* p = tables;
    for (int k = 0; k < T_KINDS; k++)
      for (int m = 0; m < n_mult; m++) {
        T.p[k][m] = p;
        T.len[k][m] = lens[k * n_mult + m];
        p += T.len[k][m];
      }
  }
  int32_t k27[27 * 3], k125[125 * 3];
  range_kernel(3, k27);
  range_kernel(5, k125);
  double t0 = omp_get_wtime();
  /* density and point levels (_hash_backend.py:13-28,428-429) */
  compute_density(C, xyz, k27);
  C->level = (int32_t*)malloc((size_t)n * sizeof(int32_t));
  for (int64_t p = 0; p < n; p++) {
    const double t = log(C->density[p] / min_density) / log(4.0);
    double l = -(floor(t) < 0 ? floor(t) : 0.0);
    if (l > depth - 1) l = depth - 1;
    C->level[p] = (int32_t)l;
  }
  /* hierarchy (_hash_backend.py:434-444) */
  float* q32 = (float*)malloc((size_t)n * 3 * sizeof(float));
  double* q64 = (double*)malloc((size_t)n * 3 * sizeof(double));
  scale_points(xyz, n, vs, q32, q64);
  uint8_t* sel = (uint8_t*)malloc((size_t)n);
  for (int d = 0; d < depth; d++) {
    int64_t m = 0;
    for (int64_t p = 0; p < n; p++) m += (sel[p] = C->level[p] <= d);
    if (m == 0) {
      for (int dd = 0; dd < d; dd++) grid_free(&C->grid[dd]);
      free(sel);
      free(q32);
      free(q64);
      free(C->density);
      free(C->level);
      free(C);
      return NULL;      /* an empty level: the reference asserts, the caller lowers min_density */
    }
    corner_grid(&C->grid[d], q32, q64, n, sel, 1 << d);
  }
  /* splatted normals of the points of each exact level, / stride^3 (__init__.py:40-48) */
  for (int d = 0; d < depth; d++) {
    const Grid* g = &C->grid[d];
    int64_t m = 0;
    for (int64_t p = 0; p < n; p++) m += C->level[p] == d;
    if (m == 0) continue;
    double* out = (double*)calloc((size_t)g->n * 3, sizeof(double));
    for (int c = 0; c < 8; c++)              /* corner-major, as np.add.at over the corner list */
      for (int64_t p = 0; p < n; p++) {
        if (C->level[p] != d) continue;
        int32_t cc[8][3];
        double w[8];
        trilinear(q32 + 3 * p, q64 + 3 * p, g->stride, cc, w);
        const int64_t r = grid_row(g, cc[c][0], cc[c][1], cc[c][2]);
        if (r < 0) continue;
        const double wp = 1.0 / C->density[p];
        for (int a = 0; a < 3; a++) out[3 * r + a] += w[c] * ((double)nrm[3 * p + a] * wp);
      }
    const double s3 = (double)g->stride * g->stride * g->stride;
    for (int64_t i = 0; i < 3 * g->n; i++) out[i] /= s3;
    C->normals[d] = out;
  }
  /* screening data per level (reconstructor.py:110-120) */
  PointBasis pbs[MAX_LEVELS];
  for (int d = 0; d < depth; d++) point_basis_all(&pbs[d], &C->grid[d], k27, q32, q64, n);
  C->seconds[0] = omp_get_wtime() - t0;
  t0 = omp_get_wtime();
  /* coarse-to-fine solve (reconstructor.py:122-189) */
  for (int d = depth - 1; d >= 0; d--) {
    level_rhs(C, d, &T, k27, k125, pbs, n, alpha, delta);
    stiffness_same_level(&C->lhs[d], &C->grid[d], &T, k125);
    if (alpha > 0) add_gram(&C->lhs[d], &pbs[d], n, pow(0.25, d) * alpha);
    C->x[d] = (double*)malloc((size_t)(C->grid[d].n > 0 ? C->grid[d].n : 1) * sizeof(double));
    C->iters[d] = cg64(&C->lhs[d], C->rhs[d], C->x[d], cg_tol, cg_maxiter);
  }
  C->seconds[1] = omp_get_wtime() - t0;
  for (int d = 0; d < depth; d++) {
    free(pbs[d].rows);
    free(pbs[d].phi);
  }
  free(sel);
  free(q32);
  free(q64);
  t0 = omp_get_wtime();
  if (mesh) extract_mesh(C, xyz, k27, tri_table, n_up);
  const double t1 = omp_get_wtime();
  C->seconds[2] = t1 - t0;
  if (mesh) {
    /* mesh stages: dual centres, dual-cube accumulation, field, marching cubes + vertices */
    const double a = C->seconds[5], b = C->seconds[3], c = C->seconds[4];
    C->seconds[3] = a - t0;
    C->seconds[4] = b - a;
    C->seconds[5] = c - b;
    C->seconds[6] = t1 - c;
  }
  return C;
}

void spsr_free(void* ctx) {
  Ctx* C = (Ctx*)ctx;
  if (!C) return;
  for (int d = 0; d < C->depth; d++) {
    grid_free(&C->grid[d]);
    free(C->normals[d]);
    free(C->rhs[d]);
    free(C->x[d]);
    csr_free(&C->lhs[d]);
  }
  free(C->density);
  free(C->level);
  free(C->dual_values);
  free(C->dual_pos);
  free(C->cubes);
  free(C->verts);
  free(C->faces);
  free(C->vkeys);
  free(C);
}

/* Sizes: out[0..3] = n_primal, n_dual, n_cubes, n_verts; out[4] = n_faces; per level d:
 * out[8 + 4d ..] = voxels, nnz, CG iterations, has splatted normals. */
void spsr_sizes(const void* ctx, int64_t* out) {
  const Ctx* C = (const Ctx*)ctx;
  out[0] = C->n_primal;
  out[1] = C->n_dual;
  out[2] = C->n_cubes;
  out[3] = C->n_verts;
  out[4] = C->n_faces;
  for (int d = 0; d < C->depth; d++) {
    out[8 + 4 * d] = C->grid[d].n;
    out[9 + 4 * d] = C->lhs[d].nnz;
    out[10 + 4 * d] = C->iters[d];
    out[11 + 4 * d] = C->normals[d] != NULL;
  }
}

void spsr_points(const void* ctx, double* density, int32_t* level) {
  const Ctx* C = (const Ctx*)ctx;
  memcpy(density, C->density, (size_t)C->n * sizeof(double));
  memcpy(level, C->level, (size_t)C->n * sizeof(int32_t));
}

/* Level d: coords int32 [V,3], rhs and x double [V], CSR (rowptr [V+1], cols [nnz], vals [nnz]);
 * any output pointer may be NULL. */
void spsr_level(const void* ctx, int d, int32_t* coords, double* rhs, double* x, int64_t* rowptr, int64_t* cols,
                double* vals, double* normals) {
  const Ctx* C = (const Ctx*)ctx;
  const int64_t n = C->grid[d].n, nnz = C->lhs[d].nnz;
  if (coords) memcpy(coords, C->grid[d].coords, (size_t)n * 3 * sizeof(int32_t));
  if (rhs) memcpy(rhs, C->rhs[d], (size_t)n * sizeof(double));
  if (x) memcpy(x, C->x[d], (size_t)n * sizeof(double));
  if (rowptr) memcpy(rowptr, C->lhs[d].rowptr, (size_t)(n + 1) * sizeof(int64_t));
  if (cols)
    for (int64_t j = 0; j < nnz; j++) cols[j] = C->lhs[d].cols[j];
  if (vals) memcpy(vals, C->lhs[d].vals, (size_t)nnz * sizeof(double));
  if (normals && C->normals[d]) memcpy(normals, C->normals[d], (size_t)n * 3 * sizeof(double));
}

/* Mesh: vertices double [nv,3], faces int64 [nf,3], the field at the primal samples minus the mean
 * (double [n_primal]), the samples' positions (double [n_primal,3]), the complete dual cubes
 * (int32 [n_cubes, 8] primal ids), mean chi, the stage times (seconds [7]) and each vertex's
 * primal-sample pair key (int64 [nv]). */
void spsr_mesh(const void* ctx, double* verts, int64_t* faces, double* dual_values, double* dual_pos,
               int32_t* cubes, double* mean_chi, double* seconds, int64_t* vkeys) {
  const Ctx* C = (const Ctx*)ctx;
  if (vkeys) memcpy(vkeys, C->vkeys, (size_t)C->n_verts * sizeof(int64_t));
  if (verts) memcpy(verts, C->verts, (size_t)C->n_verts * 3 * sizeof(double));
  if (faces) memcpy(faces, C->faces, (size_t)C->n_faces * 3 * sizeof(int64_t));
  if (dual_values) memcpy(dual_values, C->dual_values, (size_t)C->n_primal * sizeof(double));
  if (dual_pos) memcpy(dual_pos, C->dual_pos, (size_t)C->n_primal * 3 * sizeof(double));
  if (cubes) memcpy(cubes, C->cubes, (size_t)C->n_cubes * 8 * sizeof(int32_t));
  if (mean_chi) *mean_chi = C->mean_chi;
  if (seconds) memcpy(seconds, C->seconds, 7 * sizeof(double));
}
