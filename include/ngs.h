/*
 * libngs -- B200 (sm_100a) kernels for the sparse screened-Poisson
 * reconstruction path of neural-galerkin ("jspsr").
 *
 * C ABI: plain pointers and sizes, no framework types.  Unless stated
 * otherwise every pointer is DEVICE memory, every call is asynchronous on the
 * given stream, nothing is allocated inside the library, and the return value
 * is an ngs_status.  Where the reference's op returned a freshly allocated
 * tensor, the caller passes the output buffer (and, where needed, a scratch
 * workspace whose size a *_workspace_bytes() query reports).
 *
 * Citations "ref: file:line" name the reference interface an entry point
 * replaces (paths inside huangjh-pub/neural-galerkin).
 */
#ifndef NGS_H_
#define NGS_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* ngs_stream;   /* == cudaStream_t */

typedef enum {
  NGS_OK = 0,
  NGS_ERR_INVALID_ARG = 1,
  NGS_ERR_OOM = 2,               /* caller-provided buffer / workspace too small */
  NGS_ERR_HASH_INSERT = 3,       /* hash table full or probe bound exceeded */
  NGS_ERR_NOT_CONVERGED = 4,     /* iterative solve hit max_iter above tolerance */
  NGS_ERR_TOPOLOGY = 5,          /* dual-grid corner accumulation overflow */
  NGS_ERR_CUDA = 6,              /* CUDA runtime error: see ngs_last_cuda_error() */
  NGS_ERR_TIMEOUT = 7            /* a bounded device-side wait gave up */
} ngs_status;

const char* ngs_status_string(int status);
const char* ngs_last_cuda_error(void);
int ngs_version(void);
/* Number of kernels this library has launched in the process (for launch accounting). */
int64_t ngs_launch_count(void);
void ngs_reset_launch_count(void);

/* ======================================================================= hashing
 * ref: csrc/common/hashmap_cuda.cu:247-305 (hash_cuda), :204-235,307-339
 * (kernel_hash_cuda), :341-379 (build_hash_table), :381-398 (hash_table_query);
 * Python binding jspsr/ext.py:14-84 (CuckooHashTable).
 * Keys: FNV-1a-64 over (uint32) coordinates folded to 60 bits, bit-identical
 * to the reference.  The table is an open-addressing table of 16-byte
 * {key, value} slots probed by 8-lane groups (one 128-byte bucket per probe);
 * query results (value + 1, 0 = absent) are identical to the reference's
 * cuckoo table, the slot layout is not (the reference's is randomised).      */

typedef struct ngs_hash_table {
  void* slots;          /* nslots x {uint64 key, int64 value}, 16-byte aligned */
  int64_t nslots;       /* power of two, >= 8 */
  int64_t inserted;     /* number of keys inserted (HashLookupData.inserted_size) */
} ngs_hash_table;

/* hash_cuda: coords int32 or int64 [n, dim], dim in {2,3,4} -> out int64[n] */
int ngs_hash_coords(const void* coords, int coords_int64, int64_t n, int dim, int64_t* out, ngs_stream s);
/* kernel_hash_cuda: coords [n, 3|4], offsets int32 [k, 3] -> out int64 [k, n] (k-major) */
int ngs_kernel_hash(const void* coords, int coords_int64, int64_t n, int dim, const int32_t* offsets,
                    int64_t k, int64_t* out, ngs_stream s);
/* Slot count the builder needs for n keys (load <= 1/2, or <= 1/4 when enlarge). */
int64_t ngs_hash_table_slots(int64_t n, int enlarge);
/* build_hash_table: vals == NULL means value = row index.  table->slots must hold
 * table->nslots slots; status_dev (int, device) receives NGS_ERR_HASH_INSERT on failure.
 * A repeated key keeps the smallest value. */
int ngs_hash_table_build(ngs_hash_table* table, const int64_t* keys, const int64_t* vals, int64_t n,
                         int* status_dev, ngs_stream s);
/* hash_table_query: out[i] = value + 1 where keys[i] is present, else 0 */
int ngs_hash_table_query(const ngs_hash_table* table, const int64_t* keys, int64_t m, int64_t* out,
                         ngs_stream s);
/* Convenience: out[i] = row of coords[i] (int32 [m,3]) or -1, through FNV keys. */
int ngs_hash_table_query_coords(const ngs_hash_table* table, const int32_t* coords, int64_t m,
                                int64_t* out, ngs_stream s);

/* ======================================================================= scans */
size_t ngs_scan_workspace_bytes(int64_t n);
/* Exclusive prefix sum of int64 values; *total_dev receives the sum.
 * ref: the torch::cumsum calls of csrc/sparse_op/sparse_product.cu:222-223,
 * csrc/marching_cubes/dual_mc.cu:162 and jspsr/core/solver.py:41-48. */
int ngs_exclusive_scan_i64(const int64_t* in, int64_t n, int64_t* out, int64_t* total_dev, void* ws,
                           size_t ws_bytes, ngs_stream s);
int ngs_exclusive_scan_i32(const int32_t* in, int64_t n, int64_t* out, int64_t* total_dev, void* ws,
                           size_t ws_bytes, ngs_stream s);

/* ======================================================================= voxel index (rank bitmap)
 * Replaces torch.unique(dim=0) + one CuckooHashTable per level
 * (ref: jspsr/core/_hash_backend.py:358-378,414-467, jspsr/core/ops.py:103-127).
 * A level's cells live on a lattice of pitch `stride`; the grid holds one bit
 * per cell of its box plus per-word prefix counts, so the row of a voxel is
 * its rank in lexicographic (x, y, z) order.                                  */

typedef struct ngs_grid {
  int32_t origin[3];    /* min corner of the box, finest-voxel units, multiple of stride */
  int32_t dims[3];      /* box size in cells */
  int32_t stride;       /* lattice pitch (power of two) */
  int32_t log2_stride;
  int32_t zwords;       /* 64-bit words per (x, y) row: ceil(dims[2] / 64) */
  int32_t pad_;
  int64_t nwords;       /* dims[0] * dims[1] * zwords */
  void* words;          /* nwords x 16 bytes {uint32 rank, uint32 pad, uint64 bits}, zeroed before marking */
} ngs_grid;

/* Fused neighbour query of one level (ref: jspsr/core/_hash_backend.py:176-228, which builds the
 * [K, N] key matrix of csrc/common/hashmap_cuda.cu:204-235, probes the level's cuckoo table and
 * compacts with torch.where).  Two passes over tiles of 256 sources, no K x N intermediate.
 * src: float [n,3] (src_float = 1; the reference's point queries xyz / vs - 0.5) or int32 [n,3]
 * voxel coordinates at src_stride.  conv = 0 snaps each source to the level's lattice as
 * floor((src + src_stride/2) / g.stride) * g.stride, conv = 1 uses it as is; the probes are
 * origin + offsets[j] * g.stride, j < k <= 128.  row_of_rank (optional, int64 [ranks]) maps a
 * lexicographic rank to the row of a level whose coordinate list is not sorted.
 * transposed = 0 (k-major): tile_counts int64 [k * ngs_grid_neighbours_tiles(n)] (offset-major)
 * and per_offset int64 [k] (the reference's nbsizes); transposed = 1 (source-major): per_source
 * int64 [n].  masks: int32 [n, 4] scratch carried from count to fill.  start = exclusive scan of
 * tile_counts (k-major) or per_source (source-major); fill writes int64 src_ids, int64 tgt_ids and
 * int32 kidx (offset index) of every hit in the chosen order. */
int64_t ngs_grid_neighbours_tiles(int64_t n);
int ngs_grid_neighbours_count(ngs_grid g, const int64_t* row_of_rank, const void* src, int src_float, int64_t n,
                              int src_stride, int conv, const int32_t* offsets, int k, int transposed,
                              uint32_t* masks, int64_t* tile_counts, int64_t* per_offset, int64_t* per_source,
                              ngs_stream s);
int ngs_grid_neighbours_fill(ngs_grid g, const int64_t* row_of_rank, const void* src, int src_float, int64_t n,
                             int src_stride, int conv, const int32_t* offsets, int k, int transposed,
                             const uint32_t* masks, const int64_t* start, int64_t* src_ids, int64_t* tgt_ids,
                             int32_t* kidx, ngs_stream s);

/* ======================================================================= nearest neighbours, signed distance
 * Exact k-nearest-neighbour search on a uniform cell grid and the signed distance from oriented
 * points (ref: ext/sdfgen/sdf_from_points.cu:31-116 with the k-d tree of
 * csrc/common/kdtree_cuda.cu:1071-1279; Python binding ext/__init__.py:11-16).  g: a zeroed grid of
 * stride 1 in cell units (cell side h = 1 / inv_h) over the reference points' cells.
 * mark_cells marks the occupied cells (then ngs_grid_finalize); bucket writes every point's cell row
 * (cell_of) and the counts per cell (cell_count, zeroed); the caller scans the counts into start
 * (int64 [cells + 1]); scatter fills sorted (int32 [n], the points cell by cell; cursor int32
 * [cells], zeroed).  knn_sdf: per query the k <= 32 nearest points (idx_out int32 [q, k], d2_out
 * float [q, k] squared distances, nearest first, ties to the smaller index; either may be NULL) and,
 * when sdf_out is given, the signed distance with the reference's rule (magnitude from the nearest
 * point, |n.(q-p)| within stdv, |q-p| beyond; negative unless more than k/2 normals face the query). */
int ngs_knn_mark_cells(ngs_grid g, const float* xyz, int64_t n, float inv_h, ngs_stream s);
int ngs_knn_bucket(ngs_grid g, const float* xyz, int64_t n, float inv_h, int32_t* cell_of, int32_t* cell_count,
                   ngs_stream s);
int ngs_knn_scatter(const int32_t* cell_of, int64_t n, const int64_t* start, int32_t* cursor, int32_t* sorted,
                    ngs_stream s);
int ngs_knn_sdf(ngs_grid g, const int64_t* start, const int32_t* sorted, const float* ref_xyz, const float* ref_normal,
                const float* queries, int64_t nq, float inv_h, float h, int k, float stdv, int32_t* idx_out,
                float* d2_out, float* sdf_out, ngs_stream s);

/* min/max of a float [n,3] array -> bbox_dev float[6] = (min xyz, max xyz) */
int ngs_points_bbox(const float* xyz, int64_t n, float* bbox_dev, ngs_stream s);
/* Mark the 8 trilinear corner cells of every point with level <= max_level
 * (levels == NULL: all points). ref: _hash_backend.py:457-462,469-510 */
int ngs_grid_mark_points(ngs_grid g, const float* xyz, int64_t n, float inv_vs, const int32_t* levels,
                         int max_level, ngs_stream s);
/* Mark coords[i] + offsets[j] * offset_scale for every i, j (offsets int32 [n_off, 3]; NULL = origin). */
int ngs_grid_mark_coords(ngs_grid g, const int32_t* coords, int64_t n, const int32_t* offsets, int n_off,
                         int offset_scale, ngs_stream s);
/* Mark cells[i] * 2 + {0, stride, 2 stride}^3: the corners of the 2x2x2 expanded samples of each cell
 * (the same cells as ngs_grid_mark_coords on the expanded samples with the 8 unit offsets). */
int ngs_grid_mark_cell_corners(ngs_grid g, const int32_t* cells, int64_t n, int stride, ngs_stream s);
size_t ngs_grid_workspace_bytes(const ngs_grid* g);
/* Prefix counts over the words; *count_dev (int64) receives the number of cells set. */
int ngs_grid_finalize(ngs_grid g, void* ws, size_t ws_bytes, int64_t* count_dev, ngs_stream s);
/* Sorted coordinates of the set cells: coords int32 [count, 3]. */
int ngs_grid_emit_coords(ngs_grid g, int32_t* coords, ngs_stream s);
/* rows[i] = row of coords[i] (int32 [n,3]) or -1. */
int ngs_grid_lookup(ngs_grid g, const int32_t* coords, int64_t n, int64_t* rows, ngs_stream s);
/* *out_dev (int64) = a bound on |column - row| of the 5^3-stencil matrix over the grid's n set cells
 * (rows = ranks in (x, y, z) order), from the first rank of every (x, y) column: the value the PCG
 * takes as ngs_pcg_system.band.  No counterpart in the reference (its solver has no such window). */
int ngs_grid_band_bound(ngs_grid g, int64_t n, int64_t* out_dev, ngs_stream s);

/* ======================================================================= density / splatting
 * ref: jspsr/core/_hash_backend.py:13-28 (compute_density), :332-356 (splat_data),
 * :414-444 (point levels), jspsr/__init__.py:40-48 (normal splatting).
 * inv_vs is fp32(1 / fp32(voxel_size)) (the reference's quantisation), vs is the
 * FP64 voxel size used for the fractional positions.                          */
int ngs_splat_weights(ngs_grid g, const float* xyz, int64_t n, float inv_vs, double vs, float* wd, ngs_stream s);
/* density = (sum_k B(.) wd) / 16; level = clamp(-floor(log4(density / min_density)), 0, depth-1);
 * weight = 1 / density.  Any output pointer may be NULL. */
int ngs_density_eval(ngs_grid g, const float* xyz, int64_t n, float inv_vs, double vs, const float* wd,
                     float min_density, int depth, float* density, int32_t* levels, float* weight, ngs_stream s);
/* out[row] += trilinear weight * data[p] * scale for points with levels[p] == level
 * (levels == NULL: all points); data is float [n, dim] or NULL (= 1). */
int ngs_splat_data(ngs_grid g, const float* xyz, int64_t n, float inv_vs, double vs, const float* data, int dim,
                   const float* point_scale, const int32_t* levels, int level, float scale, float* out, ngs_stream s);

/* ======================================================================= basis at points
 * Screening data / evaluate_interpolated support (ref: jspsr/core/reconstructor.py:110-120,
 * jspsr/core/hashtree.py:157-192).  For every point, its 27 neighbour voxels
 * (lexicographic k in [-1,1]^3): rows int32 [n, 27] (-1 absent), phi float [n, 27]. */
int ngs_point_basis(ngs_grid g, const float* xyz, int64_t n, float inv_vs, double vs, int32_t* rows, float* phi,
                    ngs_stream s);
/* out[p] (+)= sum_k phi[p,k] * x[rows[p,k]]  (accumulate != 0: add to out) */
int ngs_point_field(const int32_t* rows, const float* phi, int64_t n, const float* x, float* out, int accumulate,
                    ngs_stream s);
/* Field value (grad == 0) or gradient (grad != 0, out float [n,3]) of sum_k B(.) x_k at arbitrary
 * positions, accumulated into out. ref: jspsr/core/hashtree.py:157-192 */
int ngs_eval_field(ngs_grid g, const float* pos, int64_t n, float inv_vs, double vs, const float* x, int grad,
                   float* out, ngs_stream s);
/* The field of all levels (the sum of ngs_eval_field over them, added in level order) in one pass:
 * grids[l] and x[l] of n_levels <= NGS_MAX_FIELD_LEVELS levels; accumulates into out like
 * ngs_eval_field.  (evaluate_raw_chi, reconstructor.py:197-226, as one launch.) */
#define NGS_MAX_FIELD_LEVELS 16
int ngs_eval_field_levels(const ngs_grid* grids, const float* const* x, int n_levels, const float* pos, int64_t n,
                          float inv_vs, double vs, int grad, float* out, ngs_stream s);
/* The field (grad 0) at the 2x2x2 mesh samples of n_cells leaf cells (pos and out: 8 samples per cell,
 * (ex, ey, ez) lexicographic, as ngs_expand_cells writes them with n_up = 2).  On every level whose
 * cells are at least half the leaf cell's size, the samples of a cell share one 4x4x4 neighbourhood,
 * read once.  Same sums as ngs_eval_field_levels on those positions (contracted axis by axis),
 * accumulated into out. */
int ngs_eval_field_cells(const ngs_grid* grids, const float* const* x, int n_levels, int64_t n_cells,
                         const float* pos, float inv_vs, double vs, float* out, ngs_stream s);
/* sum_p w[p] * v[p] and sum_p w[p] into sums_dev double[2] (mean-chi level set). */
int ngs_weighted_sum(const float* v, const float* w, int64_t n, double* sums_dev, ngs_stream s);

/* ======================================================================= Galerkin assembly
 * ref: jspsr/core/reconstructor.py:122-189, jspsr/bases/bezier_tensor.py:75-121,
 * csrc/sparse_op/sparse_product.cu:100-137 (screening product).
 * Same-level matrix A_d: CSR over the 5x5x5 stencil of present voxels, columns
 * sorted; masks[i] (uint32 x4) flags which of the 125 lexicographic offsets are
 * present, so the slot of offset o in row i is rowptr[i] + popc(mask below o). */
int ngs_stencil_count(ngs_grid g, const int32_t* coords, int64_t V, uint32_t* masks, int64_t* counts, ngs_stream s);
/* cols / stiffness values: stencil125 (double[125]) holds the stiffness of each offset;
 * diag_slot (int64 [V]) receives the slot of the diagonal entry. */
int ngs_stencil_fill(ngs_grid g, const int32_t* coords, int64_t V, const uint32_t* masks, const int64_t* rowptr,
                     const double* stencil125, int32_t* cols, double* vals, int64_t* diag_slot, ngs_stream s);
/* vals[slot(a, b)] += scale * w[p] * phi[p,a] * phi[p,b] over all point pairs (w NULL = 1). */
int ngs_screen_gram(const int32_t* rows, const float* phi, int64_t n, const float* w, const uint32_t* masks,
                    const int64_t* rowptr, double scale, double* vals, ngs_stream s);
/* ngs_screen_gram with the points grouped by cell: order = the point ids sorted by keys (keys[i] is
 * the key of point order[i]: first present row of the point's 27 * 27 + that row's position, or -1
 * for a point with no voxel at this level).  One atomic per (cell chunk of at most 128 points, row,
 * column) instead of per point; the same sums up to the order of FP64 additions.  No counterpart in
 * the reference. */
/* keys[p] = first present row of rows[p, 0..26] * 27 + its position, or -1 (the cell key of
 * ngs_screen_gram_grouped). */
int ngs_point_cell_keys(const int32_t* rows, int64_t n, int64_t* keys, ngs_stream s);
int ngs_screen_gram_grouped(const int32_t* rows, const float* phi, int64_t n, const float* w, const int64_t* order,
                            const int64_t* keys, const uint32_t* masks, const int64_t* rowptr, double scale,
                            double* vals, ngs_stream s);
/* rhs[row] += scale * sum_p w[p] * phi[p,k]  (screening target term). */
int ngs_screen_rhs(const int32_t* rows, const float* phi, int64_t n, const float* w, double scale, double* rhs,
                   ngs_stream s);
/* rhs[row] += scale * sum_p w[p] * phi[p,k] * field[p] (field nullable: 1) with the points grouped
 * by cell as for ngs_screen_gram_grouped (order / keys): one atomic per (run of a cell's points
 * within 32 sorted positions, row).  Covers ngs_screen_rhs (field NULL) and ngs_correction_screen
 * (field given, scale negated). */
int ngs_screen_rhs_grouped(const int32_t* rows, const float* phi, int64_t n, const float* w, const float* field,
                           const int64_t* order, const int64_t* keys, double scale, double* rhs, ngs_stream s);
/* Divergence RHS from splatted normals of a data level (ref: reconstructor.py:126-141):
 * rhs[t] -= int grad B_t . n_data over the pairs of get_neighbours(data, target, 3).
 * tab_f / tab_g: per-axis 1-D tables (FP64) of the level ratio (see jspsr/bases/tables.py). */
int ngs_rhs_normals(ngs_grid data_grid, const int32_t* data_coords, int64_t n_data, const float* normals,
                    ngs_grid tgt_grid, const int32_t* tgt_coords, int64_t n_tgt, const double* tab_c, const double* tab_g,
                    int tab_len, double* rhs, ngs_stream s);
/* rhs_fine[i] -= sum_j K(i, j) x_coarse[j] over the range-5 pairs (i fine, j coarse);
 * tab_c / tab_g are the shifted-integral tables of the ratio, already scaled. ref: reconstructor.py:153-168 */
int ngs_correction_stiffness(const int32_t* fine_coords, int64_t n_fine, int fine_stride, ngs_grid coarse_grid,
                             const float* x_coarse, const double* tab_c, const double* tab_g, int tab_len,
                             double* rhs, ngs_stream s);
/* rhs[row] -= scale * w[p] * phi[p,k] * field[p]  (screening part of the correction). */
int ngs_correction_screen(const int32_t* rows, const float* phi, int64_t n, const float* w, const float* field,
                          double scale, double* rhs, ngs_stream s);
/* vals32[i] = (float) vals64[i]; inv_diag[i] = 1 / vals64[diag_slot[i]]; b32 = (float) b64 */
int ngs_finish_system(const double* vals64, int64_t nnz, const int64_t* diag_slot, int64_t V, float* vals32,
                      float* inv_diag, ngs_stream s);

/* ======================================================================= solver
 * ref: csrc/sparse_solve/solve_pcg.cu:15-136 (solve_pcg_diag), jspsr/core/solver.py:101-202.
 * One persistent cooperative kernel per solve: SpMV + both dot products fused,
 * FP64 reductions in fixed order, bounded grid barriers, convergence decided on
 * the device.  mode:
 *   NGS_PCG_REFERENCE  FP32 Jacobi-PCG with the reference's stopping rule
 *                      (recursive residual <= tol * |b|), optional residual
 *                      replacement every ceil(sqrt(n)) iterations (res_fix).
 *   NGS_PCG_MIXED      FP32 SpMV / vectors, FP64 dots, FP64 solution, true FP64
 *                      residual (vals64, b64) every `replace_every` iterations;
 *                      stops on the true residual.
 *   NGS_PCG_FP64       all-FP64 Jacobi-PCG (vals64, b64), device-side loop.        */
enum { NGS_PCG_REFERENCE = 0, NGS_PCG_MIXED = 1, NGS_PCG_FP64 = 2 };

/* Matrix-free operator of one level of the B-spline system (no counterpart in the reference, whose
 * solve multiplies an assembled CSR: csrc/sparse_solve/solve_pcg.cu:67-73, assembled at
 * jspsr/core/reconstructor.py:176-185):
 *     A = K (*) v  +  alpha * Phi^T (Phi v)
 * K: the level's 5x5x5 stiffness stencil (125 FP64 values, offsets (dx, dy, dz) in [-2, 2]^3 in
 * lexicographic order), applied over the level's rank bitmap; Phi: the point basis, [N, 27] rows
 * (-1: absent) and values, and the same pairs transposed per row (t_ptr [n+1], t_point / t_phi [E],
 * ascending point index within a row).  scratch32 / scratch64: [N] per-point products (MIXED uses
 * both, FP64 the second).  Used by ngs_pcg_solve / ngs_pcg_solve_batch (MIXED and FP64 modes) when
 * ngs_pcg_system.op is set; the solver then reads no CSR (rowptr, cols, vals32/64 may be NULL) and
 * `nnz` carries the operator's work per application (60 * n + 2 * E) for the block count. */
typedef struct ngs_pcg_operator {
  ngs_grid grid;
  const int32_t* coords;     /* [n, 3] voxel coordinates (finest-voxel units) */
  const double* stencil;     /* [125] */
  double alpha;              /* screening weight of the level */
  int64_t n_points;
  const int32_t* point_rows; /* [N, 27] */
  const float* point_phi;    /* [N, 27] */
  const int64_t* t_ptr;      /* [n + 1] */
  const int32_t* t_point;    /* [E] */
  const float* t_phi;        /* [E] */
  float* scratch32;          /* [N] */
  double* scratch64;         /* [N] */
} ngs_pcg_operator;

typedef struct ngs_pcg_system {
  int64_t n;
  int64_t nnz;
  const int64_t* rowptr;     /* [n+1] */
  const int32_t* cols;       /* [nnz] */
  const float* vals32;       /* [nnz] (REFERENCE, MIXED) */
  const double* vals64;      /* [nnz] (MIXED, FP64) */
  const float* b32;          /* [n]   (REFERENCE) */
  const double* b64;         /* [n]   (MIXED, FP64) */
  const float* inv_diag;     /* [n] */
  float* x32;                /* [n] out (REFERENCE, MIXED: FP32 copy of x) */
  double* x64;               /* [n] out (MIXED, FP64) */
  const int16_t* col_delta;  /* [nnz] optional: column - row of every entry; when given the solver
                                reads these 2-byte deltas instead of the 4-byte columns in the
                                launches that use its shared-memory window (see band), and the
                                4-byte columns, if given too, in the others (NULL: cols) */
  const ngs_pcg_operator* op;/* optional: matrix-free operator instead of the CSR (NULL: CSR) */
  int64_t band;              /* optional: a bound on |column - row| over the matrix, for a CSR whose
                                columns increase within every row (0: unknown, or unsorted rows).
                                When a block's rows plus 2 band fit the solver's shared-memory
                                window, each block stages its slice of the search vector there;
                                otherwise the launch reserves no shared memory for it and the space
                                stays with the L1 cache that the gathers hit */
} ngs_pcg_system;

typedef struct ngs_pcg_config {
  int mode;
  int max_iter;              /* < 0: unbounded (the reference's default) */
  double tol;                /* relative to |b| */
  int res_fix;               /* REFERENCE mode: replace every ceil(sqrt(n)) */
  int replace_every;         /* MIXED mode */
  int blocks;                /* 0: as many co-resident blocks as fit */
  double timeout_s;          /* bound of every device-side wait */
} ngs_pcg_config;

/* col_delta[j] = cols[j] - row(j) for a CSR whose every |column - row| fits int16 (the caller
 * checks the bound; ref: no counterpart, the reference's SpMV reads int32 columns,
 * csrc/sparse_solve/solve_pcg.cu:67-73). */
int ngs_csr_col_delta(const int64_t* rowptr, const int32_t* cols, int64_t n, int16_t* col_delta, ngs_stream s);
size_t ngs_pcg_workspace_bytes(int64_t n, int mode);
/* info_dev: int64[4] = {iterations, status, replacements, reserved};
 * resid_dev: double[2] = {final |r|, |b|}.  Iterations and status are also valid
 * when the call returns NGS_ERR_NOT_CONVERGED / NGS_ERR_TIMEOUT (read them after sync). */
int ngs_pcg_solve(const ngs_pcg_system* sys, const ngs_pcg_config* cfg, void* ws, size_t ws_bytes,
                  int64_t* info_dev, double* resid_dev, ngs_stream s);

/* Several independent systems in ONE cooperative launch (the serving path's batched solve; no
 * counterpart in the reference).  Every system keeps the block count a single ngs_pcg_solve of it
 * would use (ngs_pcg_blocks), so its tile plan and reduction order -- and therefore its result,
 * bit for bit -- are those of solving it alone; its status, iterations and residual land in its own
 * info_dev / resid_dev.  All items share one mode; at most NGS_PCG_BATCH_MAX items; the blocks of
 * all non-empty items must fit ngs_pcg_block_capacity(mode) (co-residency of a cooperative launch),
 * otherwise NGS_ERR_INVALID_ARG and nothing is launched -- split the batch.  Each item needs its own
 * workspace of ngs_pcg_workspace_bytes(n, mode) bytes. */
#define NGS_PCG_BATCH_MAX 64
typedef struct ngs_pcg_batch_item {
  ngs_pcg_system sys;
  ngs_pcg_config cfg;
  void* ws;
  size_t ws_bytes;
  int64_t* info_dev;         /* int64[4], as ngs_pcg_solve */
  double* resid_dev;         /* double[2] */
} ngs_pcg_batch_item;
/* Co-resident blocks of the cooperative launch; blocks a system takes in it (0: the system is small
 * enough for one thread-block cluster and is solved by its own cluster launch, alone or in a batch --
 * ngs_pcg_cluster_size gives the CTAs of that cluster, 0 for the cooperative path). */
int ngs_pcg_block_capacity(int mode);
/* 1 if a solve of a system of n rows, nnz non-zeros and bandwidth bound band (as
 * ngs_pcg_system.band) stages its search vector in shared memory -- the launches in which the solver
 * reads 2-byte column deltas -- else 0.  No counterpart in the reference. */
int ngs_pcg_window(int64_t n, int64_t nnz, int64_t band, int mode);
int ngs_pcg_blocks(int64_t n, int64_t nnz, int mode);
int ngs_pcg_cluster_size(int64_t n, int64_t nnz, int mode);
int ngs_pcg_solve_batch(const ngs_pcg_batch_item* items, int n_items, ngs_stream s);

/* ngs_pcg_solve without any workspace from the caller, for callers that cannot allocate device
 * memory when they solve (no counterpart in the reference).  Scratch lives in a static device
 * array inside the library, sized for n <= ngs_pcg_noalloc_max_rows() (131072) rows; larger
 * systems return NGS_ERR_OOM before anything is launched, a negative n NGS_ERR_INVALID_ARG.  Every
 * call looks up the array's device address in the CUDA context current at the call
 * (cudaGetSymbolAddress; it allocates nothing), so primary and driver-created contexts alike get
 * their own copy; the first call in each context loads the library's device code there -- make
 * that first call before any stream capture.  All calls in the process share the one array: calls that may overlap on the GPU
 * (different streams, or concurrent host threads) race and must be serialised by the caller.
 * Nothing is allocated: no cudaMalloc / cudaFree, no allocating library routine.  Assembled (CSR)
 * systems only: a system with a matrix-free operator (sys->op) returns NGS_ERR_INVALID_ARG. */
int64_t ngs_pcg_noalloc_max_rows(void);
int ngs_pcg_solve_noalloc(const ngs_pcg_system* sys, const ngs_pcg_config* cfg, int64_t* info_dev,
                          double* resid_dev, ngs_stream s);

/* Builders of the matrix-free operator (ngs_pcg_operator; no counterpart in the reference, which
 * assembles the screening Gram into its LHS: jspsr/core/reconstructor.py:181-185 over
 * csrc/sparse_op/sparse_product.cu:100-137).
 * ngs_mf_count: counts[V] (zeroed by the caller) += present (point, slot) pairs per row, max_dev[0]
 *   (zeroed) = the largest count.
 * ngs_mf_fill: the transposed pairs, ascending point index within each row (t_ptr = exclusive scan
 *   of the counts, cursor[V] zeroed scratch, tmp_point / tmp_phi [E] scratch).
 * ngs_mf_diag: inv_diag[i] = 1 / (stencil_center + alpha * sum phi^2) (FP64 sum, FP32 result).
 * ngs_mf_screen_rhs: rhs[i] += scale * sum over the row's pairs of phi * (val ? val[point] : 1).
 * ngs_mf_apply64: y = A x in FP64 (t64: [N] scratch); two launches. */
int ngs_mf_count(const int32_t* point_rows, int64_t n_points, int64_t V, int32_t* counts, int32_t* max_dev,
                 ngs_stream s);
int ngs_mf_fill(const int32_t* point_rows, const float* point_phi, int64_t n_points, const int64_t* t_ptr, int64_t V,
                int32_t* cursor, int32_t* tmp_point, float* tmp_phi, int32_t* t_point, float* t_phi, ngs_stream s);
int ngs_mf_diag(const int64_t* t_ptr, const float* t_phi, int64_t V, double stencil_center, double alpha,
                float* inv_diag, ngs_stream s);
int ngs_mf_screen_rhs(const int64_t* t_ptr, const int32_t* t_point, const float* t_phi, int64_t V, const float* val,
                      double scale, double* rhs, ngs_stream s);
int ngs_mf_apply64(const ngs_pcg_operator* op, int64_t n, const double* x, double* y, ngs_stream s);
/* The screening Gram scale * sum_p phi_p phi_p^T added into an assembled stencil CSR (rowptr, the
 * 128-bit offset masks of ngs_stencil_count, vals FP64) from the transposed pairs; no atomics, fixed
 * summation order (ref: csrc/sparse_op/sparse_product.cu:100-137 + jspsr/core/reconstructor.py:181-185). */
int ngs_mf_gram(const int64_t* t_ptr, const int32_t* t_point, const float* t_phi, int64_t V, const int32_t* point_rows,
                const float* point_phi, const uint32_t* masks, const int64_t* rowptr, double scale, double* vals,
                ngs_stream s);

/* ======================================================================= sparse convolution
 * ref: csrc/sparse_op/convolution_cuda.cu:52-174 (convolution_forward_cuda), :176-282
 * (convolution_backward_cuda), called by models/ascn/utils.py:108-190 (ConvolutionFunction).
 * Feature types: NGS_F16 / NGS_BF16 run on the tensor cores (tcgen05.mma, FP32 accumulation),
 * NGS_F32 on the CUDA cores in FP32 (as the reference's FP32 cuBLAS path).
 * ngs_conv_table: table[row, k] (int32 [n_rows, K], filled here) = the row paired with `row` at offset
 *   k in nbmaps (int32 [P, 2], the pairs of offset k at starts[k] .. starts[k+1], starts int64 [K+1] on
 *   the device), -1 for none; key_col is the column of nbmaps that indexes the table; mid >= 0 sets
 *   table[row, mid] = row (the reference's forward takes the centre offset as the identity when the
 *   input and output sets are the same).
 * ngs_conv_gather_gemm: out[r, n] = sum_k sum_c x[table[r, k], c] * bt[k, n, c] (bt = the weights of
 *   every offset with the reduction index innermost), one kernel, every output row written once
 *   (FP32 out when out_f32, else the input type).  Forward: x = input, bt = W^T per offset
 *   (ngs_conv_transpose_weight); input gradient: x = output gradient, table of the other column,
 *   bt = W as stored.
 * ngs_conv_weight_grad: grad_w[k, i, o] = sum over the pairs (in, out) of offset k of x[in, i] * gy[out, o]
 *   (in_col: the nbmaps column of the input rows); splits of the pairs summed in a fixed order through
 *   ws (ngs_conv_weight_grad_ws_bytes; max_pairs = the largest per-offset pair count).
 * error_dev (int, zeroed by the caller): NGS_ERR_TIMEOUT if a bounded device wait ran out. */
enum { NGS_F16 = 0, NGS_BF16 = 1, NGS_F32 = 2 };
int ngs_conv_table(const int32_t* nbmaps, const int64_t* starts_dev, int K, int key_col, int64_t n_rows, int mid,
                   int32_t* table, ngs_stream s);
int ngs_conv_transpose_weight(const void* w, int K, int a, int b, int dtype, void* wt, ngs_stream s);
int ngs_conv_tensor_core_ok(int kdim, int ncols, int dtype);
int ngs_conv_gather_gemm(const void* x, int64_t n_src, int kdim, const int32_t* table, int64_t n_rows, int K,
                         const void* bt, int ncols, int dtype, void* out, int out_f32, int* error_dev, ngs_stream s);
size_t ngs_conv_weight_grad_ws_bytes(int K, int cin, int cout, int64_t max_pairs);
int ngs_conv_weight_grad(const void* x, int64_t n_in, int cin, const void* gy, int64_t n_out, int cout,
                         const int32_t* nbmaps, const int64_t* starts_dev, int K, int64_t max_pairs, int in_col,
                         int dtype, void* grad_w, int out_f32, void* ws, size_t ws_bytes, int* error_dev, ngs_stream s);

/* Plain building blocks for the host-driven FP64 comparator (one launch each). */
int ngs_spmv64(int64_t n, const int64_t* rowptr, const int32_t* cols, const double* vals, const double* x,
               double* y, ngs_stream s);
int ngs_dot64(const double* a, const double* b, int64_t n, double* out_dev, ngs_stream s);
int ngs_axpby64(int64_t n, double alpha, const double* x, double beta, double* y, ngs_stream s);
int ngs_mul64(int64_t n, const double* a, const double* b, double* out, ngs_stream s);

/* ======================================================================= reference sparse ops
 * ref: csrc/sparse_op/sparse_product.cu:52-82 (sparse_meshgrid), :202-258 (screened_multiplication),
 * :260-322 (screened_multiplication_backward).  a_start / b_start are exclusive prefix sums of the
 * per-point lengths; val_dim is 1 (float [A]) or 3 (float [A,3]).                              */
int ngs_sparse_meshgrid(const int64_t* a_start, const int64_t* a_len, const int64_t* b_start, const int64_t* b_len,
                        const int64_t* ab_start, int64_t n_points, int64_t* a_inds, int64_t* b_inds, ngs_stream s);
int ngs_screened_multiplication(const ngs_hash_table* pairs, const float* a_val, const float* b_val, int val_dim,
                                const int64_t* a_inds, const int64_t* b_inds, const int64_t* a_start,
                                const int64_t* a_len, const int64_t* b_start, const int64_t* b_len,
                                const float* weight, int64_t n_points, float* res, ngs_stream s);
int ngs_screened_multiplication_backward(const ngs_hash_table* pairs, const float* a_val, const float* b_val,
                                         int val_dim, const int64_t* a_inds, const int64_t* b_inds,
                                         const int64_t* a_start, const int64_t* a_len, const int64_t* b_start,
                                         const int64_t* b_len, const float* weight, int64_t n_points,
                                         const float* grad_res, float* grad_a, float* grad_b, float* grad_w,
                                         ngs_stream s);

/* ref: csrc/integration/ddi.cu:51-76 (ddi_forward), :113-141 (ddi_backward).
 * src / tgt float [P, 3C] (component-major, axis-minor), rel_pos int64 [P, 3],
 * ff / dfdf float [C, C, R]; p, q float [P, 3] (overwritten). */
int ngs_ddi_forward(const float* src, const float* tgt, const int64_t* rel_pos, const float* ff, const float* dfdf,
                    int64_t n_pairs, int C, int R, float* p, float* q, ngs_stream s);
int ngs_ddi_backward(const float* src, const float* tgt, const int64_t* rel_pos, const float* ff,
                     const float* dfdf, const float* grad_p, const float* grad_q, int64_t n_pairs, int C, int R,
                     float* grad_src, float* grad_tgt, ngs_stream s);

/* ======================================================================= marching cubes
 * ref: csrc/marching_cubes/primal_mc.cu:170-235 (marching_cubes_sparse), dual_mc.cu:135-189
 * (dual_marching_cubes_sparse), dual_mc_inds.cu:143-182 (dual_marching_cubes_indices).
 * Two phases: *_count writes per-cell vertex counts; the caller scans them
 * (ngs_exclusive_scan_i32) and *_emit writes triangles at the scanned offsets.   */
int ngs_primal_mc_count(const float* sdf, int64_t n_cubes, int r, int32_t* vcount, ngs_stream s);
int ngs_primal_mc_emit(const float* base, const float* sdf, int64_t n_cubes, int r, const int64_t* voffset,
                       float* tris, int32_t* vert_ids, int32_t* src_ids, float* src_w, ngs_stream s);
/* Dual-cube corner accumulation for one level of primal cells (expanded units):
 * probes corners / edge / face points of each cell of size `stride` in the dual-centre index and
 * writes, per dual cube and slot, slot_words int32: 2 = (primal id, depth) as the reference's
 * acc int32 [D, 8, 2]; 1 = the primal id alone, acc int32 [D, 8] (all the dual MC passes read).
 * cnt int32 [D] counts the slot writes; acc must be 8-byte aligned. */
int ngs_dual_mc_indices_grid(ngs_grid dual, const int32_t* primal_base, int64_t n_primal, int stride, int depth,
                             int64_t idx_base, int32_t* acc, int slot_words, int32_t* cnt, ngs_stream s);
int ngs_dual_mc_indices_hash(const ngs_hash_table* dual, const int32_t* primal_base, int64_t n_primal, int stride,
                             int depth, int64_t idx_base, int32_t* acc, int slot_words, int32_t* cnt, ngs_stream s);
/* The same accumulation for level-0 leaf cells (cell stride 1, n_up = 2) given as cells, not as
 * expanded samples: the 8 samples of cell i have ids idx_base + 8 i + e (ngs_expand_cells order);
 * each of a cell's 27 sample corners is looked up once.  dual must have stride 1. */
int ngs_dual_mc_indices_cells(ngs_grid dual, const int32_t* cells, int64_t n_cells, int depth, int64_t idx_base,
                              int32_t* acc, int slot_words, int32_t* cnt, ngs_stream s);
/* Keep cubes with cnt == 8: keep_dev int32 flags for a scan, then compaction of the rows of
 * 8 * slot_words int32 (acc and acc_out 16-byte aligned). */
int ngs_dual_mc_select(const int32_t* cnt, int64_t n, int32_t* keep, ngs_stream s);
int ngs_dual_mc_compact(const int32_t* acc, int slot_words, const int32_t* keep, const int64_t* keep_offset,
                        int64_t n, int32_t* acc_out, ngs_stream s);
/* Dual MC over n_cubes cubes of acc (slot_words as above).  cnt (nullable): the accumulation counts
 * of an uncompacted acc; cubes whose count is not 8 emit nothing, so the triangles come out as from
 * the compacted acc and the select / compact pass can be skipped.  NULL: every cube is complete
 * (the reference's op). */
int ngs_dual_mc_count(const int32_t* acc, int slot_words, const int32_t* cnt, int64_t n_cubes, const float* values,
                      int32_t* vcount, ngs_stream s);
int ngs_dual_mc_emit(const int32_t* acc, int slot_words, const int32_t* cnt, int64_t n_cubes, const float* pos,
                     const float* values, const int64_t* voffset, float* tris, int32_t* vert_ids, ngs_stream s);
/* Vertex de-duplication of (vid0, vid1) edge keys (replaces torch.unique(dim=0, return_inverse),
 * ref: jspsr/core/reconstructor.py:380-383): bucket sort by vid0 over n_primal buckets.
 * Phase 1 counts per bucket; the caller scans counts into bucket_start; phase 2 scatters and
 * sorts each bucket, marks first occurrences; the caller scans `first` into vertex ids;
 * phase 3 writes faces (int64 [n_keys]) and vertex positions. */
int ngs_vdedup_count(const int32_t* vert_ids, int64_t n_keys, int32_t* bucket_count, ngs_stream s);
int ngs_vdedup_sort(const int32_t* vert_ids, int64_t n_keys, const int64_t* bucket_start, int64_t n_buckets,
                    int32_t* bucket_fill, int64_t* sorted_keys, int32_t* first, ngs_stream s);
int ngs_vdedup_emit(const int32_t* vert_ids, const float* tris, int64_t n_keys, const int64_t* bucket_start,
                    const int32_t* bucket_count, const int64_t* sorted_keys, const int64_t* vertex_id,
                    int64_t* faces, float* vertices, ngs_stream s);

/* ======================================================================= multi-level mesh helpers
 * ref: jspsr/core/reconstructor.py:319-376.  Conformal children: for every parent
 * (coords at 2*stride) its 8 children at stride, in (0,0,0),(0,0,1),... order;
 * leaf[i] = 1 when child i has no cell in `finer_parents` (NULL grid words: all leaves). */
int ngs_conformal_children(const int32_t* parents, int64_t n_parents, int stride, int32_t* children, ngs_stream s);
int ngs_leaf_flags(const int32_t* cells, int64_t n, ngs_grid finer_parents, int32_t* leaf, ngs_stream s);
int ngs_compact_coords(const int32_t* coords, const int32_t* keep, const int64_t* keep_offset, int64_t n,
                       int32_t* out, ngs_stream s);
/* Expanded primal cells: cell * n_up + (i,j,k) * stride for i,j,k < n_up -> int32 [n * n_up^3, 3];
 * positions (cell_exp + stride) * evs as float [n * n_up^3, 3] (may be NULL). */
int ngs_expand_cells(const int32_t* cells, int64_t n, int n_up, int stride, float evs, int32_t* out,
                     float* pos, ngs_stream s);

#ifdef __cplusplus
}
#endif
#endif  /* NGS_H_ */
