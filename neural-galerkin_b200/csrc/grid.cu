// Rank-bitmap voxel index, density estimation, splatting and basis evaluation at points.
#include "ngs_common.cuh"
#include "scan.cuh"

// ----------------------------------------------------------------------------- index build
NGS_DEV void grid_set(const ngs_grid& g, int x, int y, int z) {
  int bit;
  const int64_t w = grid_word_index(g, x, y, z, &bit);
  if (w < 0) return;
  unsigned long long* bits = reinterpret_cast<unsigned long long*>(static_cast<char*>(g.words) + w * 16 + 8);
  const unsigned long long m = 1ull << bit;
  if (!(*reinterpret_cast<volatile unsigned long long*>(bits) & m)) atomicOr(bits, m);
}

// 8 trilinear corners of each point at the grid's stride (_hash_backend.py:469-510).
__global__ void mark_points_kernel(ngs_grid g, const float* __restrict__ xyz, int64_t n, float inv_vs,
                                   const int32_t* __restrict__ levels, int max_level) {
  const float inv_s = 1.0f / (float)g.stride;
  for (int64_t p = ngs_gtid(); p < n; p += ngs_gstride()) {
    if (levels && levels[p] > max_level) continue;
    int d[3], sg[3];
#pragma unroll
    for (int a = 0; a < 3; a++) tri_axis(q32(xyz[p * 3 + a], inv_vs), g.stride, inv_s, &d[a], &sg[a]);
#pragma unroll
    for (int c = 0; c < 8; c++) {
      const int nx = (c >> 2) & 1, ny = (c >> 1) & 1, nz = c & 1;
      grid_set(g, d[0] + nx * sg[0] * g.stride, d[1] + ny * sg[1] * g.stride, d[2] + nz * sg[2] * g.stride);
    }
  }
}

__global__ void mark_coords_kernel(ngs_grid g, const int32_t* __restrict__ c, int64_t n,
                                   const int32_t* __restrict__ off, int n_off, int scale) {
  const int64_t total = n * n_off;
  for (int64_t t = ngs_gtid(); t < total; t += ngs_gstride()) {
    const int64_t i = t / n_off;
    const int o = (int)(t - i * n_off);
    int ox = 0, oy = 0, oz = 0;
    if (off) {
      ox = off[o * 3] * scale;
      oy = off[o * 3 + 1] * scale;
      oz = off[o * 3 + 2] * scale;
    }
    grid_set(g, c[i * 3] + ox, c[i * 3 + 1] + oy, c[i * 3 + 2] + oz);
  }
}

// The 27 lattice points c * 2 + {0, s, 2s}^3 of each cell: the corners of the cell's 2 x 2 x 2
// expanded samples (n_up = 2), what marking every sample's 8 corners sets.  One thread per (cell,
// x, y) column: the column's three z points usually share a bitmap word and take one atomic.
__global__ void mark_cell_corners_kernel(ngs_grid g, const int32_t* __restrict__ c, int64_t n, int s) {
  const int64_t total = n * 9;
  for (int64_t t = ngs_gtid(); t < total; t += ngs_gstride()) {
    const int64_t i = t / 9;
    const int col = (int)(t - i * 9);
    const int x = c[i * 3] * 2 + (col / 3) * s, y = c[i * 3 + 1] * 2 + (col % 3) * s, z0 = c[i * 3 + 2] * 2;
    int64_t have = -1;
    unsigned long long m = 0ull;
#pragma unroll
    for (int k = 0; k < 3; k++) {
      int bit;
      const int64_t w = grid_word_index(g, x, y, z0 + k * s, &bit);
      if (w != have) {
        if (have >= 0) {
          unsigned long long* bits = reinterpret_cast<unsigned long long*>(static_cast<char*>(g.words) + have * 16 + 8);
          if ((*reinterpret_cast<volatile unsigned long long*>(bits) & m) != m) atomicOr(bits, m);
        }
        have = w;
        m = 0ull;
      }
      if (w >= 0) m |= 1ull << bit;
    }
    if (have >= 0) {
      unsigned long long* bits = reinterpret_cast<unsigned long long*>(static_cast<char*>(g.words) + have * 16 + 8);
      if ((*reinterpret_cast<volatile unsigned long long*>(bits) & m) != m) atomicOr(bits, m);
    }
  }
}

struct WordPopc {
  const GridWord* w;
  NGS_DEV int64_t operator()(int64_t i) const { return __popcll(w[i].bits); }
};
struct WordRank {
  GridWord* w;
  NGS_DEV void operator()(int64_t i, int64_t v) const { w[i].rank = (uint32_t)v; }
};

__global__ void emit_coords_kernel(ngs_grid g, int32_t* __restrict__ out) {
  const GridWord* words = static_cast<const GridWord*>(g.words);
  const int64_t per_x = (int64_t)g.dims[1] * g.zwords;
  for (int64_t w = ngs_gtid(); w < g.nwords; w += ngs_gstride()) {
    unsigned long long bits = words[w].bits;
    if (!bits) continue;
    int64_t r = words[w].rank;
    const int i = (int)(w / per_x);
    const int64_t rem = w - (int64_t)i * per_x;
    const int j = (int)(rem / g.zwords);
    const int kw = (int)(rem - (int64_t)j * g.zwords);
    while (bits) {
      const int b = __ffsll((long long)bits) - 1;
      bits &= bits - 1;
      const int k = kw * 64 + b;
      out[r * 3] = g.origin[0] + i * g.stride;
      out[r * 3 + 1] = g.origin[1] + j * g.stride;
      out[r * 3 + 2] = g.origin[2] + k * g.stride;
      r++;
    }
  }
}

__global__ void lookup_kernel(ngs_grid g, const int32_t* __restrict__ c, int64_t n, int64_t* __restrict__ rows) {
  for (int64_t i = ngs_gtid(); i < n; i += ngs_gstride()) rows[i] = grid_row(g, c[i * 3], c[i * 3 + 1], c[i * 3 + 2]);
}

static bool grid_ok(const ngs_grid& g) {
  return g.words && g.stride > 0 && (1 << g.log2_stride) == g.stride && g.dims[0] > 0 && g.dims[1] > 0 &&
         g.dims[2] > 0 && g.zwords == (g.dims[2] + 63) / 64 &&
         g.nwords == (int64_t)g.dims[0] * g.dims[1] * g.zwords &&
         (reinterpret_cast<uintptr_t>(g.words) & 15u) == 0;
}

extern "C" int ngs_grid_mark_points(ngs_grid g, const float* xyz, int64_t n, float inv_vs, const int32_t* levels,
                                    int max_level, ngs_stream s) {
  if (!grid_ok(g) || n < 0 || (n > 0 && !xyz)) return NGS_ERR_INVALID_ARG;
  if (n == 0) return NGS_OK;
  { ngs_count_launch(); mark_points_kernel<<<ngs_blocks(n, 256), 256, 0, (cudaStream_t)s>>>(g, xyz, n, inv_vs, levels, max_level); }
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}

extern "C" int ngs_grid_mark_coords(ngs_grid g, const int32_t* coords, int64_t n, const int32_t* offsets, int n_off,
                                    int offset_scale, ngs_stream s) {
  if (!grid_ok(g) || n < 0 || (n > 0 && !coords)) return NGS_ERR_INVALID_ARG;
  if (!offsets) n_off = 1;
  if (n == 0 || n_off <= 0) return NGS_OK;
  { ngs_count_launch(); mark_coords_kernel<<<ngs_blocks(n * n_off, 256), 256, 0, (cudaStream_t)s>>>(g, coords, n, offsets, n_off,
                                                                             offset_scale); }
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}

extern "C" int ngs_grid_mark_cell_corners(ngs_grid g, const int32_t* cells, int64_t n, int stride, ngs_stream s) {
  if (!grid_ok(g) || n < 0 || stride < 1 || (n > 0 && !cells)) return NGS_ERR_INVALID_ARG;
  if (n == 0) return NGS_OK;
  { ngs_count_launch(); mark_cell_corners_kernel<<<ngs_blocks(n * 9, 256), 256, 0, (cudaStream_t)s>>>(g, cells, n, stride); }
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}

extern "C" size_t ngs_grid_workspace_bytes(const ngs_grid* g) { return g ? ngs_scan_ws_bytes(g->nwords) : 0; }

extern "C" int ngs_grid_finalize(ngs_grid g, void* ws, size_t ws_bytes, int64_t* count_dev, ngs_stream s) {
  if (!grid_ok(g)) return NGS_ERR_INVALID_ARG;
  GridWord* w = static_cast<GridWord*>(g.words);
  return ngs_scan(WordPopc{w}, WordRank{w}, g.nwords, count_dev, ws, ws_bytes, (cudaStream_t)s);
}

extern "C" int ngs_grid_emit_coords(ngs_grid g, int32_t* coords, ngs_stream s) {
  if (!grid_ok(g) || !coords) return NGS_ERR_INVALID_ARG;
  { ngs_count_launch(); emit_coords_kernel<<<ngs_blocks(g.nwords, 256), 256, 0, (cudaStream_t)s>>>(g, coords); }
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}

// A bound on |column - row| of the level's 5^3-stencil matrix from the rank bitmap alone.  Rows are
// ranks in (x, y, z) order, so the stencil of a voxel of column (x, y) reaches from the first rank of
// column (x-2, y-2) to the last rank of column (x+2, y+2), while the voxel's own rank lies within
// column (x, y): per column the larger of the two one-sided spans, then the maximum over columns.
// The first rank of a column is the scanned rank of its first word.
__global__ void band_bound_kernel(ngs_grid g, int64_t n, unsigned long long* __restrict__ out) {
  const GridWord* w = static_cast<const GridWord*>(g.words);
  const int64_t d0 = g.dims[0], d1 = g.dims[1], zw = g.zwords, ncol = d0 * d1;
  unsigned long long best = 0;
  for (int64_t c = ngs_gtid(); c < ncol; c += ngs_gstride()) {
    const int64_t x = c / d1, y = c - x * d1;
    const int64_t lo = (x >= 2 ? x - 2 : 0) * d1 + (y >= 2 ? y - 2 : 0);
    const int64_t hi = (x + 2 < d0 ? x + 2 : d0 - 1) * d1 + (y + 2 < d1 ? y + 2 : d1 - 1) + 1;
    const int64_t s_c = w[c * zw].rank, s_lo = w[lo * zw].rank;
    const int64_t s_next = c + 1 < ncol ? (int64_t)w[(c + 1) * zw].rank : n;
    const int64_t s_hi = hi < ncol ? (int64_t)w[hi * zw].rank : n;
    const int64_t span = max(s_hi - s_c, s_next - s_lo);
    if (span > 0 && (unsigned long long)span > best) best = (unsigned long long)span;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long t = __shfl_xor_sync(0xffffffffu, best, o);
    best = t > best ? t : best;
  }
  if ((threadIdx.x & 31) == 0 && best > 0) atomicMax(out, best);
}

extern "C" int ngs_grid_band_bound(ngs_grid g, int64_t n, int64_t* out_dev, ngs_stream s) {
  if (!grid_ok(g) || n < 0 || !out_dev) return NGS_ERR_INVALID_ARG;
  cudaStream_t st = (cudaStream_t)s;
  cudaMemsetAsync(out_dev, 0, sizeof(int64_t), st);
  const int64_t ncol = (int64_t)g.dims[0] * g.dims[1];
  { ngs_count_launch(); band_bound_kernel<<<ngs_blocks(ncol, 256), 256, 0, st>>>(g, n, reinterpret_cast<unsigned long long*>(out_dev)); }
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}

extern "C" int ngs_grid_lookup(ngs_grid g, const int32_t* coords, int64_t n, int64_t* rows, ngs_stream s) {
  if (!grid_ok(g) || n < 0 || (n > 0 && (!coords || !rows))) return NGS_ERR_INVALID_ARG;
  if (n == 0) return NGS_OK;
  { ngs_count_launch(); lookup_kernel<<<ngs_blocks(n, 256), 256, 0, (cudaStream_t)s>>>(g, coords, n, rows); }
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}

// ----------------------------------------------------------------------------- trilinear splat
// Corner cells from the fp32 quantisation; weights from the FP64 fractional position.
struct Trilinear {
  int d[3], sg[3];
  float loc[3];
};

NGS_DEV Trilinear trilinear(const float* p, float inv_vs, double vs, int stride) {
  Trilinear t;
  const float inv_s = 1.0f / (float)stride;
#pragma unroll
  for (int a = 0; a < 3; a++) {
    tri_axis(q32(p[a], inv_vs), stride, inv_s, &t.d[a], &t.sg[a]);
    const double rel = (double)p[a] / vs - (double)t.d[a] - 0.5 * stride;
    t.loc[a] = (float)(fabs(rel) / stride);
  }
  return t;
}

NGS_DEV float tri_weight(const Trilinear& t, int c) {
  const int nx = (c >> 2) & 1, ny = (c >> 1) & 1, nz = c & 1;
  return (nx ? t.loc[0] : 1.f - t.loc[0]) * (ny ? t.loc[1] : 1.f - t.loc[1]) * (nz ? t.loc[2] : 1.f - t.loc[2]);
}

__global__ void splat_kernel(ngs_grid g, const float* __restrict__ xyz, int64_t n, float inv_vs, double vs,
                             const float* __restrict__ data, int dim, const float* __restrict__ pscale,
                             const int32_t* __restrict__ levels, int level, float scale, float* __restrict__ out) {
  for (int64_t p = ngs_gtid(); p < n; p += ngs_gstride()) {
    if (levels && levels[p] != level) continue;
    const Trilinear t = trilinear(xyz + p * 3, inv_vs, vs, g.stride);
    const float ps = (pscale ? pscale[p] : 1.f) * scale;
#pragma unroll
    for (int c = 0; c < 8; c++) {
      const int nx = (c >> 2) & 1, ny = (c >> 1) & 1, nz = c & 1;
      const int64_t r = grid_row(g, t.d[0] + nx * t.sg[0] * g.stride, t.d[1] + ny * t.sg[1] * g.stride,
                                 t.d[2] + nz * t.sg[2] * g.stride);
      if (r < 0) continue;
      const float w = tri_weight(t, c) * ps;
      if (!data) {
        atomicAdd(out + r, w);
      } else {
        for (int k = 0; k < dim; k++) atomicAdd(out + r * dim + k, w * data[p * dim + k]);
      }
    }
  }
}

extern "C" int ngs_splat_weights(ngs_grid g, const float* xyz, int64_t n, float inv_vs, double vs, float* wd,
                                 ngs_stream s) {
  if (!grid_ok(g) || n < 0 || (n > 0 && (!xyz || !wd))) return NGS_ERR_INVALID_ARG;
  if (n == 0) return NGS_OK;
  { ngs_count_launch(); splat_kernel<<<ngs_blocks(n, 256), 256, 0, (cudaStream_t)s>>>(g, xyz, n, inv_vs, vs, nullptr, 1, nullptr,
                                                                 nullptr, 0, 1.f, wd); }
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}

extern "C" int ngs_splat_data(ngs_grid g, const float* xyz, int64_t n, float inv_vs, double vs, const float* data,
                              int dim, const float* point_scale, const int32_t* levels, int level, float scale,
                              float* out, ngs_stream s) {
  if (!grid_ok(g) || n < 0 || dim < 1 || (n > 0 && (!xyz || !out))) return NGS_ERR_INVALID_ARG;
  if (n == 0) return NGS_OK;
  { ngs_count_launch(); splat_kernel<<<ngs_blocks(n, 256), 256, 0, (cudaStream_t)s>>>(g, xyz, n, inv_vs, vs, data, dim, point_scale,
                                                                 levels, level, scale, out); }
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}

// ----------------------------------------------------------------------------- basis at points
// Neighbourhood of a point at stride s (hashtree.py:168-181): quantised cell q and, per axis,
// the position relative to the centre of cell q + k*s, in units of s, for k = -1, 0, 1.
struct PointNbr {
  int q[3];
  float rel[3][3];
};

// One axis of a point's neighbourhood: the cell q the point falls in and the basis arguments of the
// cells q - stride, q, q + stride.
NGS_DEV void axis_nbr(float p, float inv_vs, double vs, int stride, float inv_s, int& q, float (&rel)[3]) {
  q = point_quant(q32(p, inv_vs), stride, inv_s);
  const double pos = (double)p / vs - 0.5;
  // strides are powers of two: scaling by the reciprocal is exact, the same bits as the division
  const double is = 1.0 / (double)stride;
#pragma unroll
  for (int k = 0; k < 3; k++)
    rel[k] = (float)((pos - (double)q - (double)((k - 1) * stride) - 0.5 * (stride - 1)) * is);
}

NGS_DEV PointNbr point_nbr(const float* p, float inv_vs, double vs, int stride) {
  PointNbr r;
  const float inv_s = 1.0f / (float)stride;
#pragma unroll
  for (int a = 0; a < 3; a++) axis_nbr(p[a], inv_vs, vs, stride, inv_s, r.q[a], r.rel[a]);
  return r;
}

__global__ void density_kernel(ngs_grid g, const float* __restrict__ xyz, int64_t n, float inv_vs, double vs,
                               const float* __restrict__ wd, float inv_min_density, float inv_ln4, int depth,
                               float* __restrict__ density, int32_t* __restrict__ levels, float* __restrict__ weight) {
  for (int64_t p = ngs_gtid(); p < n; p += ngs_gstride()) {
    const PointNbr nb = point_nbr(xyz + p * 3, inv_vs, vs, 1);
    float bx[3], by[3], bz[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
      bx[k] = bspline(nb.rel[0][k]);
      by[k] = bspline(nb.rel[1][k]);
      bz[k] = bspline(nb.rel[2][k]);
    }
    float acc = 0.f;
    for (int kx = 0; kx < 3; kx++)
      for (int ky = 0; ky < 3; ky++)
        for (int kz = 0; kz < 3; kz++) {
          const int64_t r = grid_row(g, nb.q[0] + kx - 1, nb.q[1] + ky - 1, nb.q[2] + kz - 1);
          if (r >= 0) acc += bx[kx] * by[ky] * bz[kz] * wd[r];
        }
    const float rho = __fmul_rn(acc, 0.0625f);
    if (density) density[p] = rho;
    if (weight) weight[p] = __fdiv_rn(1.0f, rho);
    if (levels) {
      // -floor(log(rho / min_density) / ln 4), clamped (_hash_backend.py:428-429);
      // both divisions by scalars run as products with fp32 reciprocals, as torch does on CUDA.
      const float t = floorf(__fmul_rn(logf(__fmul_rn(rho, inv_min_density)), inv_ln4));
      int lv = -(int)fminf(t, 0.f);
      levels[p] = min(lv, depth - 1);
    }
  }
}

extern "C" int ngs_density_eval(ngs_grid g, const float* xyz, int64_t n, float inv_vs, double vs, const float* wd,
                                float min_density, int depth, float* density, int32_t* levels, float* weight,
                                ngs_stream s) {
  if (!grid_ok(g) || g.stride != 1 || n < 0 || (n > 0 && (!xyz || !wd)) || min_density <= 0.f || depth < 1)
    return NGS_ERR_INVALID_ARG;
  if (n == 0) return NGS_OK;
  const float inv_md = 1.0f / min_density;
  const float inv_ln4 = 1.0f / (float)1.3862943611198906;
  { ngs_count_launch(); density_kernel<<<ngs_blocks(n, 256), 256, 0, (cudaStream_t)s>>>(g, xyz, n, inv_vs, vs, wd, inv_md, inv_ln4, depth,
                                                                   density, levels, weight); }
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}

__global__ void point_basis_kernel(ngs_grid g, const float* __restrict__ xyz, int64_t n, float inv_vs, double vs,
                                   int32_t* __restrict__ rows, float* __restrict__ phi) {
  for (int64_t p = ngs_gtid(); p < n; p += ngs_gstride()) {
    const PointNbr nb = point_nbr(xyz + p * 3, inv_vs, vs, g.stride);
    float bx[3], by[3], bz[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
      bx[k] = bspline(nb.rel[0][k]);
      by[k] = bspline(nb.rel[1][k]);
      bz[k] = bspline(nb.rel[2][k]);
    }
    for (int kx = 0; kx < 3; kx++)
      for (int ky = 0; ky < 3; ky++)
        for (int kz = 0; kz < 3; kz++) {
          const int o = kx * 9 + ky * 3 + kz;
          const int64_t r = grid_row(g, nb.q[0] + (kx - 1) * g.stride, nb.q[1] + (ky - 1) * g.stride,
                                     nb.q[2] + (kz - 1) * g.stride);
          rows[p * 27 + o] = (int32_t)r;
          phi[p * 27 + o] = r >= 0 ? bx[kx] * by[ky] * bz[kz] : 0.f;
        }
  }
}

extern "C" int ngs_point_basis(ngs_grid g, const float* xyz, int64_t n, float inv_vs, double vs, int32_t* rows,
                               float* phi, ngs_stream s) {
  if (!grid_ok(g) || n < 0 || (n > 0 && (!xyz || !rows || !phi))) return NGS_ERR_INVALID_ARG;
  if (n == 0) return NGS_OK;
  { ngs_count_launch(); point_basis_kernel<<<ngs_blocks(n, 128), 128, 0, (cudaStream_t)s>>>(g, xyz, n, inv_vs, vs, rows, phi); }
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}

__global__ void point_field_kernel(const int32_t* __restrict__ rows, const float* __restrict__ phi, int64_t n,
                                   const float* __restrict__ x, float* __restrict__ out, int accumulate) {
  for (int64_t p = ngs_gtid(); p < n; p += ngs_gstride()) {
    float acc = 0.f;
#pragma unroll 9
    for (int k = 0; k < 27; k++) {
      const int32_t r = rows[p * 27 + k];
      if (r >= 0) acc += phi[p * 27 + k] * x[r];
    }
    out[p] = accumulate ? out[p] + acc : acc;
  }
}

extern "C" int ngs_point_field(const int32_t* rows, const float* phi, int64_t n, const float* x, float* out,
                               int accumulate, ngs_stream s) {
  if (n < 0 || (n > 0 && (!rows || !phi || !x || !out))) return NGS_ERR_INVALID_ARG;
  if (n == 0) return NGS_OK;
  { ngs_count_launch(); point_field_kernel<<<ngs_blocks(n, 256), 256, 0, (cudaStream_t)s>>>(rows, phi, n, x, out, accumulate); }
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}

// One level's field (or gradient) at a point: 27 basis functions around it (hashtree.py:157-192,
// bezier_tensor.py:56-73: the gradient is per finest-voxel unit / stride).  All nine bitmap probes
// are issued before the coefficient gathers.
NGS_DEV void level_field(const ngs_grid& g, const float* p, float inv_vs, double vs, const float* __restrict__ x,
                         int grad, float& v, float& gx, float& gy, float& gz) {
  const float inv_s = 1.0f / (float)g.stride;
  const PointNbr nb = point_nbr(p, inv_vs, vs, g.stride);
  float b[3][3], db[3][3];
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int k = 0; k < 3; k++) {
      b[a][k] = bspline(nb.rel[a][k]);
      db[a][k] = bspline_d(nb.rel[a][k]) * inv_s;
    }
  int32_t rows[3][3][3];
#pragma unroll
  for (int kx = 0; kx < 3; kx++)
#pragma unroll
    for (int ky = 0; ky < 3; ky++)
      grid_rows_zrun<3>(g, nb.q[0] + (kx - 1) * g.stride, nb.q[1] + (ky - 1) * g.stride, nb.q[2] - g.stride, rows[kx][ky]);
  float lv = 0.f, lx = 0.f, ly = 0.f, lz = 0.f;
#pragma unroll
  for (int kx = 0; kx < 3; kx++)
#pragma unroll
    for (int ky = 0; ky < 3; ky++)
#pragma unroll
      for (int kz = 0; kz < 3; kz++) {
        const int32_t r = rows[kx][ky][kz];
        if (r < 0) continue;
        const float xr = x[r];
        if (!grad) {
          lv += b[0][kx] * b[1][ky] * b[2][kz] * xr;
        } else {
          lx += db[0][kx] * b[1][ky] * b[2][kz] * xr;
          ly += b[0][kx] * db[1][ky] * b[2][kz] * xr;
          lz += b[0][kx] * b[1][ky] * db[2][kz] * xr;
        }
      }
  v = lv;
  gx = lx;
  gy = ly;
  gz = lz;
}

// Field value / gradient at arbitrary positions, accumulated into out
__global__ void __launch_bounds__(128, 6) eval_field_kernel(ngs_grid g, const float* __restrict__ pos, int64_t n, float inv_vs, double vs,
                                  const float* __restrict__ x, int grad, float* __restrict__ out) {
  for (int64_t p = ngs_gtid(); p < n; p += ngs_gstride()) {
    float v, gx, gy, gz;
    level_field(g, pos + p * 3, inv_vs, vs, x, grad, v, gx, gy, gz);
    if (!grad) {
      out[p] += v;
    } else {
      out[p * 3] += gx;
      out[p * 3 + 1] += gy;
      out[p * 3 + 2] += gz;
    }
  }
}

// All levels in one pass: the point is read once and out written once; the per-level terms are
// added in level order, as the per-level launches would add them.
struct FieldLevels {
  ngs_grid g[NGS_MAX_FIELD_LEVELS];
  const float* x[NGS_MAX_FIELD_LEVELS];
  int n;
};

__global__ void __launch_bounds__(128, 6) eval_field_levels_kernel(const __grid_constant__ FieldLevels fl, const float* __restrict__ pos,
                                         int64_t n, float inv_vs, double vs, int grad, float* __restrict__ out) {
  for (int64_t p = ngs_gtid(); p < n; p += ngs_gstride()) {
    const float q[3] = {pos[p * 3], pos[p * 3 + 1], pos[p * 3 + 2]};
    float sv = grad ? 0.f : out[p];
    float sx = 0.f, sy = 0.f, sz = 0.f;
    if (grad) {
      sx = out[p * 3];
      sy = out[p * 3 + 1];
      sz = out[p * 3 + 2];
    }
    for (int l = 0; l < fl.n; l++) {
      float v, gx, gy, gz;
      level_field(fl.g[l], q, inv_vs, vs, fl.x[l], grad, v, gx, gy, gz);
      sv += v;
      sx += gx;
      sy += gy;
      sz += gz;
    }
    if (!grad) {
      out[p] = sv;
    } else {
      out[p * 3] = sx;
      out[p * 3 + 1] = sy;
      out[p * 3 + 2] = sz;
    }
  }
}

// The field at the 2 x 2 x 2 mesh samples of leaf cells (the primal samples of the dual marching
// cubes, n_upsample = 2): pos holds the 8 samples of cell c at 8c .. 8c+7, (ex, ey, ez) in
// lexicographic order, and along each axis they take two positions.  On a field level whose cells
// are at least half the leaf cell's size, the two positions of an axis fall in the same or in
// adjacent field cells, so the 8 samples' 27-cell neighbourhoods lie in one 4 x 4 x 4 box.  The box
// is looked up once (16 runs of 4 cells along z) and the tensor-product sums are contracted axis by
// axis in registers -- z while the box is read, y per x slab of the box, then x (8 samples) --
// with each sample's three basis values placed at its offset in a 4-wide weight vector.  That is
// 224 multiply-adds per cell and level instead of 8 x 27 triple products.  Levels whose cells are
// smaller take the per-sample path.  Levels are added in level order.
// One sample's value on one level, out of line: the per-cell kernel calls it only for field levels
// finer than half its cell.
__device__ __noinline__ float sample_field(const ngs_grid& g, const float* p, float inv_vs, double vs,
                                           const float* __restrict__ x) {
  float v, gx, gy, gz;
  level_field(g, p, inv_vs, vs, x, 0, v, gx, gy, gz);
  return v;
}

// w[i] for a thread-dependent i, by selects (an indexed register array would go to local memory).
NGS_DEV float sel4(const float (&w)[4], int i) { return i == 0 ? w[0] : i == 1 ? w[1] : i == 2 ? w[2] : w[3]; }

// Eight 128-thread blocks per SM (64 registers, a few spilled to L1): the kernel waits on its bitmap
// runs and gathers, and twice the resident warps hide more of that than the spills cost (2.1 -> 1.6
// ms for the 300k cloud's mesh samples).
__global__ void __launch_bounds__(128, 8) field_cells_kernel(const __grid_constant__ FieldLevels fl,
                                                          int64_t n_cells, const float* __restrict__ pos,
                                                          float inv_vs, double vs, float* __restrict__ out) {
  for (int64_t c = ngs_gtid(); c < n_cells; c += ngs_gstride()) {
    const float* P = pos + c * 24;
    float acc[8];
#pragma unroll
    for (int e = 0; e < 8; e++) acc[e] = out[c * 8 + e];
    for (int l = 0; l < fl.n; l++) {
      const ngs_grid& g = fl.g[l];
      const float* __restrict__ x = fl.x[l];
      const int S = g.stride;
      const float inv_s = 1.0f / (float)S;
      // per axis a and side t (sample (t,0,0) carries x, (0,t,0) y, (0,0,t) z): the field cell and
      // the 4-wide weights over the box cells q0 - S .. q0 + 2S
      int q0[3];
      float w[3][2][4];
      bool boxed = true;
#pragma unroll
      for (int a = 0; a < 3; a++) {
        int q[2];
        float bs[2][3];
#pragma unroll
        for (int t = 0; t < 2; t++) {
          float rel[3];
          axis_nbr(P[(t << (2 - a)) * 3 + a], inv_vs, vs, S, inv_s, q[t], rel);
#pragma unroll
          for (int k = 0; k < 3; k++) bs[t][k] = bspline(rel[k]);
        }
        q0[a] = q[0];
        const int d = q[1] - q[0];
        boxed = boxed && (d == 0 || d == S);
        const bool sh = d != 0;
#pragma unroll
        for (int t = 0; t < 2; t++) {
          const bool st = t == 1 && sh;
          w[a][t][0] = st ? 0.f : bs[t][0];
          w[a][t][1] = st ? bs[t][0] : bs[t][1];
          w[a][t][2] = st ? bs[t][1] : bs[t][2];
          w[a][t][3] = st ? bs[t][2] : 0.f;
        }
      }
      if (!boxed) {
#pragma unroll
        for (int e = 0; e < 8; e++) acc[e] += sample_field(g, P + e * 3, inv_vs, vs, x);
        continue;
      }
      // one x slab of the box at a time (its 4 runs of 4 cells along z in flight together): z sums
      // while the runs are read, folded into the slab's y sums, which go into the x sums -- each sum
      // in the same order as a contraction of the whole box axis by axis
      float xs[8];
#pragma unroll
      for (int e = 0; e < 8; e++) xs[e] = 0.f;
#pragma unroll 1
      for (int ix = 0; ix < 4; ix++) {
        float cy[2][2] = {{0.f, 0.f}, {0.f, 0.f}};             // [tz][ty]
#pragma unroll
        for (int iy = 0; iy < 4; iy++) {
          int32_t r[4];
          grid_rows_zrun<4>(g, q0[0] + (ix - 1) * S, q0[1] + (iy - 1) * S, q0[2] - S, r);
          float xv[4];
#pragma unroll
          for (int iz = 0; iz < 4; iz++) xv[iz] = r[iz] >= 0 ? x[r[iz]] : 0.f;
#pragma unroll
          for (int tz = 0; tz < 2; tz++) {
            float sum = 0.f;
#pragma unroll
            for (int iz = 0; iz < 4; iz++) sum += w[2][tz][iz] * xv[iz];
#pragma unroll
            for (int ty = 0; ty < 2; ty++) cy[tz][ty] += w[1][ty][iy] * sum;
          }
        }
#pragma unroll
        for (int tx = 0; tx < 2; tx++) {
          const float wx = sel4(w[0][tx], ix);
#pragma unroll
          for (int ty = 0; ty < 2; ty++)
#pragma unroll
            for (int tz = 0; tz < 2; tz++) xs[tx * 4 + ty * 2 + tz] += wx * cy[tz][ty];
        }
      }
#pragma unroll
      for (int e = 0; e < 8; e++) acc[e] += xs[e];
    }
#pragma unroll
    for (int e = 0; e < 8; e++) out[c * 8 + e] = acc[e];
  }
}

extern "C" int ngs_eval_field_cells(const ngs_grid* grids, const float* const* x, int n_levels, int64_t n_cells,
                                    const float* pos, float inv_vs, double vs, float* out, ngs_stream s) {
  if (!grids || !x || n_levels < 1 || n_levels > NGS_MAX_FIELD_LEVELS || n_cells < 0 ||
      (n_cells > 0 && (!pos || !out)))
    return NGS_ERR_INVALID_ARG;
  FieldLevels fl;
  fl.n = n_levels;
  for (int l = 0; l < n_levels; l++) {
    if (!grid_ok(grids[l]) || !x[l]) return NGS_ERR_INVALID_ARG;
    fl.g[l] = grids[l];
    fl.x[l] = x[l];
  }
  if (n_cells == 0) return NGS_OK;
  { ngs_count_launch(); field_cells_kernel<<<ngs_blocks(n_cells, 128), 128, 0, (cudaStream_t)s>>>(fl, n_cells, pos, inv_vs, vs, out); }
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}

extern "C" int ngs_eval_field_levels(const ngs_grid* grids, const float* const* x, int n_levels, const float* pos,
                                     int64_t n, float inv_vs, double vs, int grad, float* out, ngs_stream s) {
  if (!grids || !x || n_levels < 1 || n_levels > NGS_MAX_FIELD_LEVELS || n < 0 || (n > 0 && (!pos || !out)))
    return NGS_ERR_INVALID_ARG;
  FieldLevels fl;
  fl.n = n_levels;
  for (int l = 0; l < n_levels; l++) {
    if (!grid_ok(grids[l]) || !x[l]) return NGS_ERR_INVALID_ARG;
    fl.g[l] = grids[l];
    fl.x[l] = x[l];
  }
  if (n == 0) return NGS_OK;
  { ngs_count_launch(); eval_field_levels_kernel<<<ngs_blocks(n, 128), 128, 0, (cudaStream_t)s>>>(fl, pos, n, inv_vs, vs, grad, out); }
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}

extern "C" int ngs_eval_field(ngs_grid g, const float* pos, int64_t n, float inv_vs, double vs, const float* x,
                              int grad, float* out, ngs_stream s) {
  if (!grid_ok(g) || n < 0 || (n > 0 && (!pos || !x || !out))) return NGS_ERR_INVALID_ARG;
  if (n == 0) return NGS_OK;
  { ngs_count_launch(); eval_field_kernel<<<ngs_blocks(n, 128), 128, 0, (cudaStream_t)s>>>(g, pos, n, inv_vs, vs, x, grad, out); }
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}
