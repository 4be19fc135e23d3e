// Galerkin assembly of the screened-Poisson system on one level
// (jspsr/core/reconstructor.py:122-189, jspsr/bases/bezier_tensor.py:75-121).
//
// Layout: CSR over the lexicographically sorted voxels of the level; the
// columns of a row are its present neighbours in the 5x5x5 stencil, in
// lexicographic offset order, hence sorted.  A 128-bit mask per row records
// which of the 125 offsets are present, so the CSR slot of any (row, offset)
// pair is rowptr + popc(mask below offset) -- the screening Gram product
// therefore adds straight into the matrix instead of going through the
// reference's second hash table keyed by (row, col) pairs.
#include "ngs_common.cuh"


// ----------------------------------------------------------------------------- structure
// One warp per row: lane l < 25 owns the stencil column (dx, dy) = (l / 5 - 2, l % 5 - 2) and its
// five cells along z (offsets o = 5 l .. 5 l + 4 in lexicographic order), found with one or two
// bitmap words; a warp scan of the lanes' counts gives every lane its first CSR slot, so the row's
// entries are written by consecutive lanes.
NGS_DEV void stencil_column(const ngs_grid& g, const int32_t* __restrict__ coords, int64_t i, int lane,
                            int32_t (&r)[5]) {
  const int cx = coords[i * 3], cy = coords[i * 3 + 1], cz = coords[i * 3 + 2];
  if (lane < 25)
    grid_rows_zrun<5>(g, cx + (lane / 5 - 2) * g.stride, cy + (lane % 5 - 2) * g.stride, cz - 2 * g.stride, r);
  else
    for (int t = 0; t < 5; t++) r[t] = -1;
}

__global__ void stencil_count_kernel(ngs_grid g, const int32_t* __restrict__ coords, int64_t V,
                                     uint4* __restrict__ masks, int64_t* __restrict__ counts) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t i = ngs_gtid() >> 5; i < V; i += warps) {
    int32_t r[5];
    stencil_column(g, coords, i, lane, r);
    // lane l's column fills mask bits 5l .. 5l+4 (cell t of the column at bit 5l + t); each of the
    // four 32-bit words is the OR of the lanes' shifted patterns
    unsigned pat = 0u;
#pragma unroll
    for (int t = 0; t < 5; t++) pat |= (r[t] >= 0 ? 1u : 0u) << t;
    const int lo = 5 * lane;
    unsigned w[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const int sh = lo - 32 * k;             // position of the pattern's bit 0 in word k
      const unsigned part = sh >= 32 || sh <= -5 ? 0u : (sh >= 0 ? pat << sh : pat >> -sh);
      w[k] = __reduce_or_sync(0xffffffffu, part);
    }
    const unsigned total = __reduce_add_sync(0xffffffffu, (unsigned)__popc(pat));
    if (lane == 0) {
      masks[i] = make_uint4(w[0], w[1], w[2], w[3]);
      counts[i] = (int64_t)total;
    }
  }
}

__global__ void stencil_fill_kernel(ngs_grid g, const int32_t* __restrict__ coords, int64_t V,
                                    const uint4* __restrict__ masks, const int64_t* __restrict__ rowptr,
                                    const double* __restrict__ stencil, int32_t* __restrict__ cols,
                                    double* __restrict__ vals, int64_t* __restrict__ diag_slot) {
  __shared__ double st[125];
  for (int t = threadIdx.x; t < 125; t += blockDim.x) st[t] = stencil[t];
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t i = ngs_gtid() >> 5; i < V; i += warps) {
    int32_t r[5];
    stencil_column(g, coords, i, lane, r);
    int c = 0;
#pragma unroll
    for (int t = 0; t < 5; t++) c += r[t] >= 0 ? 1 : 0;
    int pre = c;                                      // inclusive warp scan of the counts
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, pre, d);
      if (lane >= d) pre += y;
    }
    int64_t slot = rowptr[i] + (pre - c);
#pragma unroll
    for (int t = 0; t < 5; t++) {
      if (r[t] < 0) continue;
      const int o = 5 * lane + t;
      cols[slot] = r[t];
      vals[slot] = st[o];
      if (o == 62) diag_slot[i] = slot;
      slot++;
    }
  }
}

extern "C" int ngs_stencil_count(ngs_grid g, const int32_t* coords, int64_t V, uint32_t* masks, int64_t* counts,
                                 ngs_stream s) {
  if (!g.words || V < 0 || (V > 0 && (!coords || !masks || !counts))) return NGS_ERR_INVALID_ARG;
  if (V == 0) return NGS_OK;
  { ngs_count_launch(); stencil_count_kernel<<<ngs_blocks(V * 32, 256), 256, 0, (cudaStream_t)s>>>(g, coords, V, reinterpret_cast<uint4*>(masks),
                                                                       counts); }
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}

extern "C" int ngs_stencil_fill(ngs_grid g, const int32_t* coords, int64_t V, const uint32_t* masks,
                                const int64_t* rowptr, const double* stencil125, int32_t* cols, double* vals,
                                int64_t* diag_slot, ngs_stream s) {
  if (!g.words || V < 0 || (V > 0 && (!coords || !masks || !rowptr || !stencil125 || !cols || !vals || !diag_slot)))
    return NGS_ERR_INVALID_ARG;
  if (V == 0) return NGS_OK;
  { ngs_count_launch(); stencil_fill_kernel<<<ngs_blocks(V * 32, 256), 256, 0, (cudaStream_t)s>>>(
      g, coords, V, reinterpret_cast<const uint4*>(masks), rowptr, stencil125, cols, vals, diag_slot); }
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}

// ----------------------------------------------------------------------------- screening
// One warp per point; lane a (< 27) owns the point's neighbour a and adds
// w * phi_a * phi_b into row a for every present neighbour b.
__global__ void screen_gram_kernel(const int32_t* __restrict__ rows, const float* __restrict__ phi, int64_t n,
                                   const float* __restrict__ w, const uint4* __restrict__ masks,
                                   const int64_t* __restrict__ rowptr, double scale, double* __restrict__ vals) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t p = ngs_gtid() >> 5; p < n; p += warps) {
    const int32_t ra = lane < 27 ? rows[p * 27 + lane] : -1;
    const float pa = lane < 27 ? phi[p * 27 + lane] : 0.f;
    const double sa = scale * (double)(w ? w[p] : 1.f) * (double)pa;
    uint4 m = make_uint4(0, 0, 0, 0);
    int64_t base = 0;
    if (ra >= 0) {
      m = masks[ra];
      base = rowptr[ra];
    }
    const int ax = lane / 9, ay = (lane / 3) % 3, az = lane % 3;
#pragma unroll 3
    for (int b = 0; b < 27; b++) {
      const int32_t rb = __shfl_sync(0xffffffffu, ra, b);
      const float pb = __shfl_sync(0xffffffffu, pa, b);
      if (ra < 0 || rb < 0) continue;
      const int bx = b / 9, by = (b / 3) % 3, bz = b % 3;
      const int o = (bx - ax + 2) * 25 + (by - ay + 2) * 5 + (bz - az + 2);
      atomicAdd(vals + base + popc_below(m, o), sa * (double)pb);
    }
  }
}

extern "C" int ngs_screen_gram(const int32_t* rows, const float* phi, int64_t n, const float* w, const uint32_t* masks,
                               const int64_t* rowptr, double scale, double* vals, ngs_stream s) {
  if (n < 0 || (n > 0 && (!rows || !phi || !masks || !rowptr || !vals))) return NGS_ERR_INVALID_ARG;
  if (n == 0) return NGS_OK;
  { ngs_count_launch(); screen_gram_kernel<<<ngs_blocks(n * 32, 256), 256, 0, (cudaStream_t)s>>>(
      rows, phi, n, w, reinterpret_cast<const uint4*>(masks), rowptr, scale, vals); }
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}

// The cell key of each point: its first present neighbour row * 27 + that neighbour's position, or
// -1 when none of the 27 is present.  Points in one cell share all 27 rows, so the key identifies
// the cell (the cell is the first present neighbour's voxel minus that position's offset).
__global__ void point_cell_keys_kernel(const int32_t* __restrict__ rows, int64_t n, int64_t* __restrict__ keys) {
  for (int64_t p = ngs_gtid(); p < n; p += ngs_gstride()) {
    int64_t key = -1;
    for (int a = 0; a < 27; a++) {
      const int32_t r = rows[p * 27 + a];
      if (r >= 0) {
        key = (int64_t)r * 27 + a;
        break;
      }
    }
    keys[p] = key;
  }
}

extern "C" int ngs_point_cell_keys(const int32_t* rows, int64_t n, int64_t* keys, ngs_stream s) {
  if (n < 0 || (n > 0 && (!rows || !keys))) return NGS_ERR_INVALID_ARG;
  if (n == 0) return NGS_OK;
  { ngs_count_launch(); point_cell_keys_kernel<<<ngs_blocks(n, 256), 256, 0, (cudaStream_t)s>>>(rows, n, keys); }
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}

// Points sorted by cell key are taken in chunks: a run of equal keys is cut at every multiple of
// NGS_GROUP_CHUNK positions, so that one warp never walks more than that many points (on a coarse
// level of a large scene, millions of points share one cell).  A chunk starts where the key changes
// or at a cut; keys < 0 (no voxel) start nothing.
constexpr int64_t NGS_GROUP_CHUNK = 128;
NGS_DEV bool group_chunk_start(const int64_t* __restrict__ keys, int64_t i) {
  const int64_t key = keys[i];
  if (key < 0) return false;
  return i == 0 || keys[i - 1] != key || i % NGS_GROUP_CHUNK == 0;
}

// The same sum with the points grouped by their 27-voxel neighbourhood: points in one cell share all
// 27 rows, so their outer products are summed in registers (lane a keeps row a's 27 sums) and each
// (row, column) slot takes one atomic per cell chunk instead of one per point.  order / keys: the
// points sorted by key = first present row * 27 + its position (-1: no voxel), a key that fixes the
// cell.  One warp per sorted position; the warp at a chunk start does the chunk.
__global__ void screen_gram_grouped_kernel(const int32_t* __restrict__ rows, const float* __restrict__ phi,
                                           int64_t n, const float* __restrict__ w, const int64_t* __restrict__ order,
                                           const int64_t* __restrict__ keys, const uint4* __restrict__ masks,
                                           const int64_t* __restrict__ rowptr, double scale,
                                           double* __restrict__ vals) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t i = ngs_gtid() >> 5; i < n; i += warps) {
    const int64_t key = keys[i];
    if (!group_chunk_start(keys, i)) continue;                    // warp-uniform
    const int64_t p0 = order[i];
    const int32_t ra = lane < 27 ? rows[p0 * 27 + lane] : -1;
    double acc[27];
#pragma unroll
    for (int b = 0; b < 27; b++) acc[b] = 0.0;
    for (int64_t j = i; j < n && keys[j] == key && (j == i || j % NGS_GROUP_CHUNK != 0); j++) {
      const int64_t p = order[j];
      const float pa = lane < 27 ? phi[p * 27 + lane] : 0.f;
      const double sa = (double)(w ? w[p] : 1.f) * (double)pa;
#pragma unroll
      for (int b = 0; b < 27; b++) acc[b] += sa * (double)__shfl_sync(0xffffffffu, pa, b);
    }
    const uint4 m = ra >= 0 ? masks[ra] : make_uint4(0, 0, 0, 0);
    const int64_t base = ra >= 0 ? rowptr[ra] : 0;
    const int ax = lane / 9, ay = (lane / 3) % 3, az = lane % 3;
#pragma unroll
    for (int b = 0; b < 27; b++) {
      const int32_t rb = __shfl_sync(0xffffffffu, ra, b);      // all 32 lanes take part in the shuffle
      if (ra < 0 || rb < 0) continue;
      const int bx = b / 9, by = (b / 3) % 3, bz = b % 3;
      const int o = (bx - ax + 2) * 25 + (by - ay + 2) * 5 + (bz - az + 2);
      atomicAdd(vals + base + popc_below(m, o), scale * acc[b]);
    }
  }
}

extern "C" int ngs_screen_gram_grouped(const int32_t* rows, const float* phi, int64_t n, const float* w,
                                       const int64_t* order, const int64_t* keys, const uint32_t* masks,
                                       const int64_t* rowptr, double scale, double* vals, ngs_stream s) {
  if (n < 0 || (n > 0 && (!rows || !phi || !order || !keys || !masks || !rowptr || !vals))) return NGS_ERR_INVALID_ARG;
  if (n == 0) return NGS_OK;
  { ngs_count_launch(); screen_gram_grouped_kernel<<<ngs_blocks(n * 32, 256), 256, 0, (cudaStream_t)s>>>(
      rows, phi, n, w, order, keys, reinterpret_cast<const uint4*>(masks), rowptr, scale, vals); }
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}

__global__ void screen_rhs_kernel(const int32_t* __restrict__ rows, const float* __restrict__ phi, int64_t n,
                                  const float* __restrict__ w, const float* __restrict__ field, double scale,
                                  double* __restrict__ rhs) {
  const int64_t total = n * 27;
  for (int64_t t = ngs_gtid(); t < total; t += ngs_gstride()) {
    const int32_t r = rows[t];
    if (r < 0) continue;
    const int64_t p = t / 27;
    double v = scale * (double)phi[t];
    if (w) v *= (double)w[p];
    if (field) v *= (double)field[p];
    atomicAdd(rhs + r, v);
  }
}

// Screening RHS terms over the points sorted by cell key (the Gram's order / keys): one point per
// lane, 32 sorted points per warp step.  For each of the 27 neighbours, the lanes of a run of equal
// keys (points of one cell, which share their 27 rows) are summed by a segmented warp scan and the
// run's last lane adds the sum -- one atomic per (run, row) instead of one per point.  On coarse
// levels most points share few rows, and per-point atomics serialise there.
__global__ void screen_rhs_grouped_kernel(const int32_t* __restrict__ rows, const float* __restrict__ phi, int64_t n,
                                          const float* __restrict__ w, const float* __restrict__ field,
                                          const int64_t* __restrict__ order, const int64_t* __restrict__ keys,
                                          double scale, double* __restrict__ rhs) {
  const int lane = threadIdx.x & 31;
  const int64_t n_round = (n + 31) & ~(int64_t)31;
  for (int64_t i = ngs_gtid(); i < n_round; i += ngs_gstride()) {
    const int64_t key = i < n ? keys[i] : -1;
    const bool valid = key >= 0;
    const int64_t p = valid ? order[i] : 0;
    double sp = valid ? scale : 0.0;
    if (valid && w) sp *= (double)w[p];
    if (valid && field) sp *= (double)field[p];
    const int64_t prev = __shfl_up_sync(0xffffffffu, key, 1), next = __shfl_down_sync(0xffffffffu, key, 1);
    const unsigned heads = __ballot_sync(0xffffffffu, lane == 0 || prev != key);
    const int start = 31 - __clz(heads & (0xffffffffu >> (31 - lane)));
    const bool tail = lane == 31 || next != key;
    for (int a = 0; a < 27; a++) {
      double v = valid ? sp * (double)phi[p * 27 + a] : 0.0;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const double y = __shfl_up_sync(0xffffffffu, v, o);
        if (lane - o >= start) v += y;
      }
      if (tail && valid) {
        const int32_t r = rows[p * 27 + a];
        if (r >= 0) atomicAdd(rhs + r, v);
      }
    }
  }
}

extern "C" int ngs_screen_rhs_grouped(const int32_t* rows, const float* phi, int64_t n, const float* w,
                                      const float* field, const int64_t* order, const int64_t* keys, double scale,
                                      double* rhs, ngs_stream s) {
  if (n < 0 || (n > 0 && (!rows || !phi || !order || !keys || !rhs))) return NGS_ERR_INVALID_ARG;
  if (n == 0) return NGS_OK;
  { ngs_count_launch(); screen_rhs_grouped_kernel<<<ngs_blocks(n, 256), 256, 0, (cudaStream_t)s>>>(
      rows, phi, n, w, field, order, keys, scale, rhs); }
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}

extern "C" int ngs_screen_rhs(const int32_t* rows, const float* phi, int64_t n, const float* w, double scale,
                              double* rhs, ngs_stream s) {
  if (n < 0 || (n > 0 && (!rows || !phi || !rhs))) return NGS_ERR_INVALID_ARG;
  if (n == 0) return NGS_OK;
  { ngs_count_launch(); screen_rhs_kernel<<<ngs_blocks(n * 27, 256), 256, 0, (cudaStream_t)s>>>(rows, phi, n, w, nullptr, scale, rhs); }
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}

extern "C" int ngs_correction_screen(const int32_t* rows, const float* phi, int64_t n, const float* w,
                                     const float* field, double scale, double* rhs, ngs_stream s) {
  if (n < 0 || (n > 0 && (!rows || !phi || !field || !rhs))) return NGS_ERR_INVALID_ARG;
  if (n == 0) return NGS_OK;
  { ngs_count_launch(); screen_rhs_kernel<<<ngs_blocks(n * 27, 256), 256, 0, (cudaStream_t)s>>>(rows, phi, n, w, field, -scale, rhs); }
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}

// ----------------------------------------------------------------------------- RHS from normals
// target stride >= data stride: scatter from every data voxel to the 27 target voxels around the
// target cell that holds the data voxel's centre (get_coords_neighbours, _hash_backend.py:194-228).
__global__ void rhs_scatter_kernel(const int32_t* __restrict__ dc, int64_t nd, int sd, const float* __restrict__ nrm,
                                   ngs_grid tg, const double* __restrict__ tc, const double* __restrict__ tgv,
                                   int tab_len, double* __restrict__ rhs) {
  const int st = tg.stride, M = st / sd;
  const int lane = threadIdx.x & 31;
  // whole warps run the loop (the warp collectives below): lanes past the end contribute nothing
  const int64_t nd_round = (nd + 31) & ~(int64_t)31;
  for (int64_t i = ngs_gtid(); i < nd_round; i += ngs_gstride()) {
    const bool valid = i < nd;
    const int64_t ii = valid ? i : nd - 1;
    int q[3], c[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
      c[a] = dc[ii * 3 + a];
      q[a] = (int)floorf(((float)c[a] + 0.5f * (float)sd) / (float)st) * st;
    }
    const double n0 = valid ? nrm[ii * 3] : 0.0, n1 = valid ? nrm[ii * 3 + 1] : 0.0, n2 = valid ? nrm[ii * 3 + 2] : 0.0;
    // data voxels in lexicographic order: neighbouring lanes often share the target cell q (always,
    // for a coarse target level).  Lanes of one run of equal q are summed by a segmented scan and
    // the run's last lane adds the sum -- one atomic per run and target instead of one per voxel.
    bool same_prev = true, same_next = true;
#pragma unroll
    for (int a = 0; a < 3; a++) {
      same_prev &= __shfl_up_sync(0xffffffffu, q[a], 1) == q[a];
      same_next &= __shfl_down_sync(0xffffffffu, q[a], 1) == q[a];
    }
    const unsigned heads = __ballot_sync(0xffffffffu, lane == 0 || !same_prev);
    const int start = 31 - __clz(heads & (0xffffffffu >> (31 - lane)));      // first lane of my run
    const bool tail = lane == 31 || !same_next;
    for (int kx = -1; kx <= 1; kx++)
      for (int ky = -1; ky <= 1; ky++)
        for (int kz = -1; kz <= 1; kz++) {
          const int k[3] = {kx, ky, kz};
          double cv[3], gv[3];
          bool ok = true;
#pragma unroll
          for (int a = 0; a < 3; a++) {
            // rel = k*M + (q - c)/sd + (M-1)/2 ; idx = rel + (3M-1)/2  (integer)
            const int idx = k[a] * M + (q[a] - c[a]) / sd + 2 * M - 1;
            ok &= (idx >= 0 && idx < tab_len);
            cv[a] = ok ? tc[idx] : 0.0;
            gv[a] = ok ? tgv[idx] : 0.0;
          }
          double v = ok ? n0 * gv[0] * cv[1] * cv[2] + n1 * cv[0] * gv[1] * cv[2] + n2 * cv[0] * cv[1] * gv[2] : 0.0;
#pragma unroll
          for (int o = 1; o < 32; o <<= 1) {
            const double y = __shfl_up_sync(0xffffffffu, v, o);
            if (lane - o >= start) v += y;
          }
          if (!tail) continue;
          const int64_t t = grid_row(tg, q[0] + kx * st, q[1] + ky * st, q[2] + kz * st);
          if (t >= 0 && v != 0.0) atomicAdd(rhs + t, -v);
        }
  }
}

// target stride < data stride (coarse data, fine target): gather per target voxel over the coarse
// data voxels whose centre lies within 1.5 fine voxels (the inverted map, _hash_backend.py:254-262).
__global__ void rhs_gather_kernel(ngs_grid dg, const float* __restrict__ nrm, const int32_t* __restrict__ tcoords,
                                  int64_t nt, int st, const double* __restrict__ tc, const double* __restrict__ tgv,
                                  int tab_len, double* __restrict__ rhs) {
  const int sd = dg.stride, M = sd / st;
  for (int64_t i = ngs_gtid(); i < nt; i += ngs_gstride()) {
    int q[3], c[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
      c[a] = tcoords[i * 3 + a];
      q[a] = (int)floorf(((float)c[a] + 0.5f * (float)st) / (float)sd) * sd;
    }
    double acc = 0.0;
    for (int kx = -1; kx <= 1; kx++)
      for (int ky = -1; ky <= 1; ky++)
        for (int kz = -1; kz <= 1; kz++) {
          const int k[3] = {kx, ky, kz};
          double cv[3], gv[3];
          bool ok = true;
#pragma unroll
          for (int a = 0; a < 3; a++) {
            // nt = k*M + (q - c)/st + (M-1)/2 (fine units), keep |nt| < 1.5;
            // rel = -nt * st / sd ; idx = rel * M + M/2 + 0.5 = -nt + M/2 + 0.5 (integer)
            const int two_nt = 2 * (k[a] * M + (q[a] - c[a]) / st) + (M - 1);
            ok &= (two_nt > -3 - 1 && two_nt < 3 + 1) && (abs(two_nt) <= 3);
            const int idx = (-two_nt + M + 1) / 2;
            ok &= (idx >= 0 && idx < tab_len);
            cv[a] = ok ? tc[idx] : 0.0;
            gv[a] = ok ? tgv[idx] : 0.0;
          }
          if (!ok) continue;
          const int64_t d = grid_row(dg, q[0] + kx * sd, q[1] + ky * sd, q[2] + kz * sd);
          if (d < 0) continue;
          const double n0 = nrm[d * 3], n1 = nrm[d * 3 + 1], n2 = nrm[d * 3 + 2];
          acc += n0 * gv[0] * cv[1] * cv[2] + n1 * cv[0] * gv[1] * cv[2] + n2 * cv[0] * cv[1] * gv[2];
        }
    rhs[i] -= acc;
  }
}

// target stride == data stride: every data voxel D scatters to the targets D + k stride, k in
// {-1, 0, 1}^3, so each target T gathers from the data voxels T - k stride instead -- 9 runs of 3
// cells along z, no atomics, a fixed summation order.  The table index of offset k is k + 1.
__global__ void rhs_same_level_kernel(ngs_grid dg, const float* __restrict__ nrm, const int32_t* __restrict__ tcoords,
                                      int64_t nt, const double* __restrict__ tc, const double* __restrict__ tgv,
                                      double* __restrict__ rhs) {
  const int s = dg.stride;
  for (int64_t i = ngs_gtid(); i < nt; i += ngs_gstride()) {
    const int c0 = tcoords[i * 3], c1 = tcoords[i * 3 + 1], c2 = tcoords[i * 3 + 2];
    double acc = 0.0;
#pragma unroll
    for (int jx = -1; jx <= 1; jx++)
#pragma unroll
      for (int jy = -1; jy <= 1; jy++) {
        int32_t r[3];
        grid_rows_zrun<3>(dg, c0 + jx * s, c1 + jy * s, c2 - s, r);
#pragma unroll
        for (int jz = -1; jz <= 1; jz++) {
          const int32_t d = r[jz + 1];
          if (d < 0) continue;
          // data voxel D = T + j s sees the target at offset k = -j: table index 1 - j
          const double cx = tc[1 - jx], cy = tc[1 - jy], cz = tc[1 - jz];
          const double gx = tgv[1 - jx], gy = tgv[1 - jy], gz = tgv[1 - jz];
          const double n0 = nrm[(int64_t)d * 3], n1 = nrm[(int64_t)d * 3 + 1], n2 = nrm[(int64_t)d * 3 + 2];
          acc += n0 * gx * cy * cz + n1 * cx * gy * cz + n2 * cx * cy * gz;
        }
      }
    rhs[i] -= acc;
  }
}

extern "C" int ngs_rhs_normals(ngs_grid data_grid, const int32_t* data_coords, int64_t n_data, const float* normals,
                               ngs_grid tgt_grid, const int32_t* tgt_coords, int64_t n_tgt, const double* tab_c,
                               const double* tab_g, int tab_len, double* rhs, ngs_stream s) {
  if (!normals || !tab_c || !tab_g || !rhs || tab_len <= 0) return NGS_ERR_INVALID_ARG;
  cudaStream_t st = (cudaStream_t)s;
  if (tgt_grid.stride == data_grid.stride && tgt_coords && data_grid.words && tab_len == 3) {
    if (n_tgt <= 0 || n_data <= 0) return NGS_OK;
    { ngs_count_launch(); rhs_same_level_kernel<<<ngs_blocks(n_tgt, 128), 128, 0, st>>>(data_grid, normals, tgt_coords, n_tgt,
                                                                                       tab_c, tab_g, rhs); }
  } else if (tgt_grid.stride >= data_grid.stride) {
    if (n_data <= 0) return NGS_OK;
    if (!data_coords || !tgt_grid.words) return NGS_ERR_INVALID_ARG;
    { ngs_count_launch(); rhs_scatter_kernel<<<ngs_blocks(n_data, 128), 128, 0, st>>>(data_coords, n_data, data_grid.stride, normals,
                                                               tgt_grid, tab_c, tab_g, tab_len, rhs); }
  } else {
    if (n_tgt <= 0) return NGS_OK;
    if (!tgt_coords || !data_grid.words) return NGS_ERR_INVALID_ARG;
    { ngs_count_launch(); rhs_gather_kernel<<<ngs_blocks(n_tgt, 128), 128, 0, st>>>(data_grid, normals, tgt_coords, n_tgt, tgt_grid.stride,
                                                              tab_c, tab_g, tab_len, rhs); }
  }
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}

// ----------------------------------------------------------------------------- cross-level correction
// rhs_fine[i] -= sum over the 125 coarse neighbours j of K(i, j) * x_coarse[j]
// (reconstructor.py:153-168, stiffness part; computed matrix-free).
// 64 registers (eight 128-thread blocks per SM, no spills): more resident warps to wait on the bitmap
// runs and gathers (0.89 -> 0.82 ms for the 300k cloud).
__global__ void __launch_bounds__(128, 8) correction_kernel(const int32_t* __restrict__ fc, int64_t nf, int sf, ngs_grid cg,
                                  const float* __restrict__ x, const double* __restrict__ tc,
                                  const double* __restrict__ tg, int tab_len, double* __restrict__ rhs) {
  extern __shared__ double tabs[];
  for (int t = threadIdx.x; t < tab_len; t += blockDim.x) {
    tabs[t] = tc[t];
    tabs[tab_len + t] = tg[t];
  }
  __syncthreads();
  const int sc = cg.stride, M = sc / sf;
  for (int64_t i = ngs_gtid(); i < nf; i += ngs_gstride()) {
    int q[3], base[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
      const int c = fc[i * 3 + a];
      q[a] = (int)floorf(((float)c + 0.5f * (float)sf) / (float)sc) * sc;
      // idx = rel + 1.5M + 0.5 with rel = k*M + (q - c)/sf + (M-1)/2  ->  k*M + (q - c)/sf + 2M
      base[a] = (q[a] - c) / sf + 2 * M;
    }
    double acc = 0.0;
    for (int kx = -2; kx <= 2; kx++) {
      const int ix = kx * M + base[0];
      if (ix < 0 || ix >= tab_len) continue;
      for (int ky = -2; ky <= 2; ky++) {
        const int iy = ky * M + base[1];
        if (iy < 0 || iy >= tab_len) continue;
        int32_t rz[5];                       // the 5 coarse cells along z, one or two bitmap words
        grid_rows_zrun<5>(cg, q[0] + kx * sc, q[1] + ky * sc, q[2] - 2 * sc, rz);
        // K = g_x c_y c_z + c_x g_y c_z + c_x c_y g_z = A c_z + B g_z for the column (kx, ky)
        const double A = tabs[tab_len + ix] * tabs[iy] + tabs[ix] * tabs[tab_len + iy];
        const double B = tabs[ix] * tabs[iy];
#pragma unroll
        for (int kz = -2; kz <= 2; kz++) {
          const int iz = kz * M + base[2];
          if (iz < 0 || iz >= tab_len) continue;
          const int64_t j = rz[kz + 2];
          if (j < 0) continue;
          acc += (A * tabs[iz] + B * tabs[tab_len + iz]) * (double)x[j];
        }
      }
    }
    rhs[i] -= acc;
  }
}

extern "C" int ngs_correction_stiffness(const int32_t* fine_coords, int64_t n_fine, int fine_stride, ngs_grid cg,
                                        const float* x_coarse, const double* tab_c, const double* tab_g, int tab_len,
                                        double* rhs, ngs_stream s) {
  // tables of 3M + 2 entries each: level ratios M up to 2^12 (13 levels) fit one block's shared memory
  if (n_fine < 0 || fine_stride <= 0 || cg.stride <= fine_stride || tab_len <= 0 || tab_len > 12290)
    return NGS_ERR_INVALID_ARG;
  if (n_fine == 0) return NGS_OK;
  if (!fine_coords || !cg.words || !x_coarse || !tab_c || !tab_g || !rhs) return NGS_ERR_INVALID_ARG;
  const size_t smem = 2 * (size_t)tab_len * sizeof(double);
  if (smem > 48 * 1024) {
    const cudaError_t e = cudaFuncSetAttribute(correction_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return ngs_set_cuda_error(e);
  }
  { ngs_count_launch(); correction_kernel<<<ngs_blocks(n_fine, 128), 128, smem, (cudaStream_t)s>>>(
      fine_coords, n_fine, fine_stride, cg, x_coarse, tab_c, tab_g, tab_len, rhs); }
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}

// ----------------------------------------------------------------------------- finish
__global__ void finish_kernel(const double* __restrict__ v64, int64_t nnz, const int64_t* __restrict__ diag_slot,
                              int64_t V, float* __restrict__ v32, float* __restrict__ inv_diag) {
  for (int64_t i = ngs_gtid(); i < nnz; i += ngs_gstride()) v32[i] = (float)v64[i];
  for (int64_t i = ngs_gtid(); i < V; i += ngs_gstride()) inv_diag[i] = (float)(1.0 / v64[diag_slot[i]]);
}

extern "C" int ngs_finish_system(const double* vals64, int64_t nnz, const int64_t* diag_slot, int64_t V, float* vals32,
                                 float* inv_diag, ngs_stream s) {
  if (nnz < 0 || V < 0 || (nnz > 0 && (!vals64 || !vals32)) || (V > 0 && (!diag_slot || !inv_diag)))
    return NGS_ERR_INVALID_ARG;
  if (nnz == 0 && V == 0) return NGS_OK;
  { ngs_count_launch(); finish_kernel<<<ngs_blocks(nnz > V ? nnz : V, 256), 256, 0, (cudaStream_t)s>>>(vals64, nnz, diag_slot, V, vals32,
                                                                                inv_diag); }
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}
