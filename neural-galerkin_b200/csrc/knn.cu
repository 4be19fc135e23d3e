// Exact k-nearest-neighbour search and signed distance from oriented points, on a uniform cell grid.
//
// Replaces the FLANN-derived CUDA k-d tree of the reference (csrc/common/kdtree_cuda.cu:1071-1279,
// built and queried by ext/sdfgen/sdf_from_points.cu:70-116) and its voting kernel
// (ext/sdfgen/sdf_from_points.cu:31-68): the ground-truth occupancy of the training loop
// (models/full_net.py:135-142 calls it with k = 8, stdv = 0.02).
//
// Layout: the reference points are bucketed by a cubic cell of side h.  The occupied cells form a
// rank bitmap (ngs_grid, stride 1 in cell units), so a cell's bucket is found with one 128-bit load;
// a counting sort (counts by atomics, an exclusive scan, a scatter) lays the points out cell by cell.
// A query walks Chebyshev rings of cells around its own cell, keeping the k best (squared distance,
// point index) pairs in registers -- ties broken by the smaller index, so the result does not depend
// on the order of points inside a bucket -- and stops once k are held and the k-th distance is at
// most r h: every point of ring r + 1 or beyond is farther than r h from a query inside the centre
// cell.  The ring walk is clipped to the grid's box, and ends when the box is covered.
//
// The signed distance then follows the reference exactly: magnitude from the nearest neighbour p0,
// |n0 . (q - p0)| when |q - p0| < stdv, else |q - p0|; sign negative unless more than k / 2 of the
// k neighbours see the query on the positive side of their normal (n . (q - p) > 0).
#include "ngs_common.cuh"

constexpr int KNN_MAX_K = 32;

__global__ void knn_mark_cells_kernel(ngs_grid g, const float* __restrict__ xyz, int64_t n, float inv_h) {
  unsigned long long* words = reinterpret_cast<unsigned long long*>(g.words);
  for (int64_t i = ngs_gtid(); i < n; i += ngs_gstride()) {
    int bit;
    const int64_t w = grid_word_index(g, (int)floorf(xyz[3 * i] * inv_h), (int)floorf(xyz[3 * i + 1] * inv_h),
                                      (int)floorf(xyz[3 * i + 2] * inv_h), &bit);
    if (w >= 0) atomicOr(words + 2 * w + 1, 1ull << bit);
  }
}

__global__ void knn_bucket_kernel(ngs_grid g, const float* __restrict__ xyz, int64_t n, float inv_h,
                                  int32_t* __restrict__ cell_of, int32_t* __restrict__ cell_count) {
  for (int64_t i = ngs_gtid(); i < n; i += ngs_gstride()) {
    const int64_t r = grid_row(g, (int)floorf(xyz[3 * i] * inv_h), (int)floorf(xyz[3 * i + 1] * inv_h),
                               (int)floorf(xyz[3 * i + 2] * inv_h));
    cell_of[i] = (int32_t)r;
    if (r >= 0) atomicAdd(cell_count + r, 1);
  }
}

__global__ void knn_scatter_kernel(const int32_t* __restrict__ cell_of, int64_t n, const int64_t* __restrict__ start,
                                   int32_t* __restrict__ cursor, int32_t* __restrict__ sorted) {
  for (int64_t i = ngs_gtid(); i < n; i += ngs_gstride()) {
    const int32_t c = cell_of[i];
    if (c >= 0) sorted[start[c] + atomicAdd(cursor + c, 1)] = (int32_t)i;
  }
}

// (d2, idx) ordering: smaller distance first, then smaller index
NGS_DEV bool knn_less(float da, int ia, float db, int ib) { return da < db || (da == db && ia < ib); }

__global__ void knn_sdf_kernel(ngs_grid g, const int64_t* __restrict__ start, const int32_t* __restrict__ sorted,
                               const float* __restrict__ ref, const float* __restrict__ nrm,
                               const float* __restrict__ q, int64_t nq, float inv_h, float h, int k, float stdv,
                               int32_t* __restrict__ idx_out, float* __restrict__ d2_out, float* __restrict__ sdf_out) {
  for (int64_t i = ngs_gtid(); i < nq; i += ngs_gstride()) {
    const float px = q[3 * i], py = q[3 * i + 1], pz = q[3 * i + 2];
    const int cx = (int)floorf(px * inv_h), cy = (int)floorf(py * inv_h), cz = (int)floorf(pz * inv_h);
    const int lo[3] = {g.origin[0], g.origin[1], g.origin[2]};
    const int hi[3] = {g.origin[0] + g.dims[0] - 1, g.origin[1] + g.dims[1] - 1, g.origin[2] + g.dims[2] - 1};
    const int c[3] = {cx, cy, cz};
    int rmax = 0;
#pragma unroll
    for (int a = 0; a < 3; a++) rmax = max(rmax, max(c[a] - lo[a], hi[a] - c[a]));
    float bd[KNN_MAX_K];
    int bi[KNN_MAX_K];
    int cnt = 0;
    for (int r = 0; r <= rmax; r++) {
      const int x0 = max(cx - r, lo[0]), x1 = min(cx + r, hi[0]);
      const int y0 = max(cy - r, lo[1]), y1 = min(cy + r, hi[1]);
      for (int x = x0; x <= x1; x++) {
        for (int y = y0; y <= y1; y++) {
          const bool side = abs(x - cx) == r || abs(y - cy) == r;
          // on the ring: every z of the column when x or y is at distance r, else only cz -+ r
          for (int z = side ? cz - r : cz - r; z <= cz + r; z += (side || r == 0) ? 1 : 2 * r) {
            if (z < lo[2] || z > hi[2]) continue;
            const int64_t cell = grid_row(g, x, y, z);
            if (cell < 0) continue;
            for (int64_t t = start[cell]; t < start[cell + 1]; t++) {
              const int pid = sorted[t];
              const float dx = ref[3 * pid] - px, dy = ref[3 * pid + 1] - py, dz = ref[3 * pid + 2] - pz;
              const float d2 = dx * dx + dy * dy + dz * dz;
              if (cnt == k && !knn_less(d2, pid, bd[k - 1], bi[k - 1])) continue;
              int s = cnt < k ? cnt++ : k - 1;     // insertion into the sorted list
              while (s > 0 && knn_less(d2, pid, bd[s - 1], bi[s - 1])) {
                bd[s] = bd[s - 1];
                bi[s] = bi[s - 1];
                s--;
              }
              bd[s] = d2;
              bi[s] = pid;
            }
          }
        }
      }
      const float reach = (float)r * h;
      if (cnt == k && bd[k - 1] <= reach * reach) break;
    }
    if (idx_out)
      for (int j = 0; j < k; j++) idx_out[i * k + j] = j < cnt ? bi[j] : -1;
    if (d2_out)
      for (int j = 0; j < k; j++) d2_out[i * k + j] = j < cnt ? bd[j] : INFINITY;
    if (sdf_out) {
      float sdf = 0.f;
      int pos = 0;
      for (int j = 0; j < cnt; j++) {
        const int pid = bi[j];
        const float rx = px - ref[3 * pid], ry = py - ref[3 * pid + 1], rz = pz - ref[3 * pid + 2];
        const float d = nrm[3 * pid] * rx + nrm[3 * pid + 1] * ry + nrm[3 * pid + 2] * rz;
        if (j == 0) {
          const float len = sqrtf(rx * rx + ry * ry + rz * rz);
          sdf = len < stdv ? fabsf(d) : len;
        }
        if (d > 0.f) pos++;
      }
      sdf_out[i] = pos <= k / 2 ? -sdf : sdf;
    }
  }
}

extern "C" int ngs_knn_mark_cells(ngs_grid g, const float* xyz, int64_t n, float inv_h, ngs_stream s) {
  if (!g.words || g.stride != 1 || n < 0 || (n > 0 && !xyz) || !(inv_h > 0.f)) return NGS_ERR_INVALID_ARG;
  if (n == 0) return NGS_OK;
  { ngs_count_launch(); knn_mark_cells_kernel<<<ngs_blocks(n, 256), 256, 0, (cudaStream_t)s>>>(g, xyz, n, inv_h); }
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}

extern "C" int ngs_knn_bucket(ngs_grid g, const float* xyz, int64_t n, float inv_h, int32_t* cell_of,
                              int32_t* cell_count, ngs_stream s) {
  if (!g.words || g.stride != 1 || n < 0 || (n > 0 && (!xyz || !cell_of || !cell_count)) || !(inv_h > 0.f))
    return NGS_ERR_INVALID_ARG;
  if (n == 0) return NGS_OK;
  { ngs_count_launch(); knn_bucket_kernel<<<ngs_blocks(n, 256), 256, 0, (cudaStream_t)s>>>(g, xyz, n, inv_h, cell_of, cell_count); }
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}

extern "C" int ngs_knn_scatter(const int32_t* cell_of, int64_t n, const int64_t* start, int32_t* cursor, int32_t* sorted,
                               ngs_stream s) {
  if (n < 0 || (n > 0 && (!cell_of || !start || !cursor || !sorted))) return NGS_ERR_INVALID_ARG;
  if (n == 0) return NGS_OK;
  { ngs_count_launch(); knn_scatter_kernel<<<ngs_blocks(n, 256), 256, 0, (cudaStream_t)s>>>(cell_of, n, start, cursor, sorted); }
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}

extern "C" int ngs_knn_sdf(ngs_grid g, const int64_t* start, const int32_t* sorted, const float* ref_xyz,
                           const float* ref_normal, const float* queries, int64_t nq, float inv_h, float h, int k,
                           float stdv, int32_t* idx_out, float* d2_out, float* sdf_out, ngs_stream s) {
  if (!g.words || g.stride != 1 || nq < 0 || k < 1 || k > KNN_MAX_K || !(inv_h > 0.f) || !start || !sorted ||
      !ref_xyz || (nq > 0 && !queries) || (sdf_out && !ref_normal))
    return NGS_ERR_INVALID_ARG;
  if (nq == 0) return NGS_OK;
  { ngs_count_launch(); knn_sdf_kernel<<<ngs_blocks(nq, 128), 128, 0, (cudaStream_t)s>>>(
      g, start, sorted, ref_xyz, ref_normal, queries, nq, inv_h, h, k, stdv, idx_out, d2_out, sdf_out); }
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}
