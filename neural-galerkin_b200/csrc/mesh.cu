// Multi-level dual marching cubes (jspsr/core/reconstructor.py:296-397,
// csrc/marching_cubes/dual_mc_inds.cu:45-182, dual_mc.cu:20-189).
#include <algorithm>
#include "ngs_common.cuh"
#include "hash_table.cuh"

// Triangle table (Lorensen / Bourke, data file) -- 256 cases x 16 edges, -1 terminated.
__constant__ signed char c_tri[256][16] = {
#include "mc_tables.inc"
};
// Edge endpoints in interpolation order (p1, p2); corner i of the MC cube sits at
// (0,0,0),(1,0,0),(1,1,0),(0,1,0),(0,0,1),(1,0,1),(1,1,1),(0,1,1).
__constant__ int c_edge[12][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {4, 5}, {5, 6},
                                  {6, 7}, {7, 4}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};
__constant__ int c_corner[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0},
                                   {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
// MC corner holding the octant (ox, oy, oz), indexed by ox + 2 oy + 4 oz.
__constant__ int c_octant_slot[8] = {0, 1, 3, 2, 4, 5, 7, 6};

NGS_DEV int num_verts(int t) {
  int n = 0;
  while (n < 16 && c_tri[t][n] >= 0) n++;
  return n;
}

NGS_DEV int cube_type(const float* v) {
  int t = 0;
#pragma unroll
  for (int i = 0; i < 8; i++) t |= (v[i] < 0.f ? 1 : 0) << i;
  return t;
}

// Edge vertex with the reference's 1e-5 snapping rules; returns the weight of p1.
NGS_DEV float sdf_interp(const float* p1, const float* p2, float v1, float v2, float* out) {
  if (fabsf(v1) < 1.0e-5f) { out[0] = p1[0]; out[1] = p1[1]; out[2] = p1[2]; return 1.f; }
  if (fabsf(v2) < 1.0e-5f) { out[0] = p2[0]; out[1] = p2[1]; out[2] = p2[2]; return 0.f; }
  if (fabsf(v1 - v2) < 1.0e-5f) { out[0] = p1[0]; out[1] = p1[1]; out[2] = p1[2]; return 1.f; }
  const float w2 = (0.0f - v1) / (v2 - v1);
  const float w1 = 1.f - w2;
#pragma unroll
  for (int a = 0; a < 3; a++) out[a] = p1[a] * w1 + p2[a] * w2;
  return w1;
}

// ----------------------------------------------------------------------------- dual corner accumulation
// The probes of one primal cell of stride s: its 8 corners (one dual-cube slot each), the 12 (s - 1)
// interior points of its edges (two slots) and the 6 (s - 1)^2 interior points of its faces (four
// slots).  The index space is laid out kind by kind -- all corner probes, then all edge probes,
// then all face probes -- so that the threads of a warp take the same branch, and it is indexed in
// 32 bits whenever it fits.
//
// More than 8 slot writes into one dual cube is the reference's "Topology Error"
// (dual_mc_inds.cu:86,115,135): such a cube's count ends above 8 and the cube is dropped by
// ngs_dual_mc_select, which keeps the cubes with exactly 8 writes; every probe therefore writes its
// slots unconditionally and adds to the count without reading it back.
template <typename Lookup, typename Idx, int W>
__global__ void dual_inds_kernel(Lookup lk, const int32_t* __restrict__ pb, Idx n_primal, int stride, int depth,
                                 int64_t idx_base, int32_t* __restrict__ acc, int32_t* __restrict__ cnt) {
  const Idx sm1 = (Idx)stride - 1;
  const Idx n_corner = n_primal * 8, n_edge = n_primal * 12 * sm1;
  const Idx total = n_corner + n_edge + n_primal * 6 * sm1 * sm1;
  for (Idx t = (Idx)ngs_gtid(); t < total; t += (Idx)ngs_gstride()) {
    Idx pid;
    // the probe's offset from the cell's base corner and its slots, kept in registers (axes are
    // chosen with selects, not by indexing)
    int off[3] = {0, 0, 0};
    auto put = [&](int axis, int v) {
#pragma unroll
      for (int k = 0; k < 3; k++) off[k] = axis == k ? v : off[k];
    };
    int slots[4] = {0, 0, 0, 0}, ns;
    if (t < n_corner) {
      pid = t >> 3;
      const int q = (int)(t & 7);
      // corner (cx, cy, cz) = bits of q (x most significant): primal in the opposite octant
      const int cx = (q >> 2) & 1, cy = (q >> 1) & 1, cz = q & 1;
      off[0] = cx * stride;
      off[1] = cy * stride;
      off[2] = cz * stride;
      slots[0] = c_octant_slot[(1 - cx) + 2 * (1 - cy) + 4 * (1 - cz)];
      ns = 1;
    } else if (t < n_corner + n_edge) {
      const Idx q = t - n_corner, per = 12 * sm1;
      pid = q / per;
      const Idx in = q - pid * per;
      const int e = (int)(in / sm1), tt = (int)(in - (Idx)e * sm1) + 1;
      const int ax = e >> 2, v0 = (e >> 1) & 1, v1 = e & 1;
      const int b0 = ax == 0 ? 1 : 0, b1 = ax == 2 ? 1 : 2;
      put(ax, tt);
      put(b0, v0 * stride);
      put(b1, v1 * stride);
      // octant (oc[ax] = o, oc[b0] = 1 - v0, oc[b1] = 1 - v1) as ox + 2 oy + 4 oz
      const int rest = ((1 - v0) << b0) + ((1 - v1) << b1);
      slots[0] = c_octant_slot[rest];
      slots[1] = c_octant_slot[rest + (1 << ax)];
      ns = 2;
    } else {
      const Idx q = t - n_corner - n_edge, fc = sm1 * sm1, per = 6 * fc;
      pid = q / per;
      const Idx in = q - pid * per;
      const int f = (int)(in / fc);
      const int uv = (int)(in - (Idx)f * fc);
      const int ax = f >> 1, side = f & 1;
      const int b0 = ax == 0 ? 1 : 0, b1 = ax == 2 ? 1 : 2;
      put(ax, side * stride);
      put(b0, uv % (int)sm1 + 1);
      put(b1, uv / (int)sm1 + 1);
      // octant (oc[ax] = 1 - side, oc[b0] = o & 1, oc[b1] = o >> 1)
      const int base = (1 - side) << ax;
#pragma unroll
      for (int o = 0; o < 4; o++) slots[o] = c_octant_slot[base + ((o & 1) << b0) + ((o >> 1) << b1)];
      ns = 4;
    }
    const int64_t row = lk(pb[(int64_t)pid * 3] + off[0], pb[(int64_t)pid * 3 + 1] + off[1],
                           pb[(int64_t)pid * 3 + 2] + off[2]);
    if (row < 0) continue;
    atomicAdd(cnt + row, ns);
    const int32_t id = (int32_t)((int64_t)pid + idx_base);
    if constexpr (W == 2) {
      const int2 v = make_int2(id, depth);
      int2* dst = reinterpret_cast<int2*>(acc) + row * 8;
      dst[slots[0]] = v;
      if (ns > 1) dst[slots[1]] = v;
      if (ns > 2) {
        dst[slots[2]] = v;
        dst[slots[3]] = v;
      }
    } else {
      int32_t* dst = acc + row * 8;
      dst[slots[0]] = id;
      if (ns > 1) dst[slots[1]] = id;
      if (ns > 2) {
        dst[slots[2]] = id;
        dst[slots[3]] = id;
      }
    }
  }
}

// Probes of n_primal cells of stride s: launch over 32-bit indices when they fit.
template <typename Lookup, int W>
void launch_dual_inds_w(Lookup lk, const int32_t* pb, int64_t n_primal, int stride, int depth, int64_t idx_base,
                        int32_t* acc, int32_t* cnt, cudaStream_t s) {
  const int64_t per = 8 + 12 * (int64_t)(stride - 1) + 6 * (int64_t)(stride - 1) * (stride - 1);
  const int64_t total = n_primal * per;
  const unsigned grid = ngs_blocks(total, 256);
  ngs_count_launch();
  // 32-bit indexing needs the whole index space plus one grid stride below 2^32
  if (total + (int64_t)grid * 256 < (int64_t)UINT32_MAX)
    dual_inds_kernel<Lookup, uint32_t, W><<<grid, 256, 0, s>>>(lk, pb, (uint32_t)n_primal, stride, depth, idx_base, acc,
                                                               cnt);
  else
    dual_inds_kernel<Lookup, int64_t, W><<<grid, 256, 0, s>>>(lk, pb, n_primal, stride, depth, idx_base, acc, cnt);
}

// slot_words 2: the reference's (primal id, depth) pairs; 1: primal ids alone (the dual MC passes
// read nothing else)
template <typename Lookup>
void launch_dual_inds(Lookup lk, const int32_t* pb, int64_t n_primal, int stride, int depth, int64_t idx_base,
                      int32_t* acc, int slot_words, int32_t* cnt, cudaStream_t s) {
  if (slot_words == 2) launch_dual_inds_w<Lookup, 2>(lk, pb, n_primal, stride, depth, idx_base, acc, cnt, s);
  else launch_dual_inds_w<Lookup, 1>(lk, pb, n_primal, stride, depth, idx_base, acc, cnt, s);
}

struct GridLookup {
  ngs_grid g;
  NGS_DEV int64_t operator()(int x, int y, int z) const { return grid_row(g, x, y, z); }
};
struct KeyLookup {
  const Slot* slots;
  int64_t mask;
  NGS_DEV int64_t operator()(int x, int y, int z) const {
    unsigned long long h = NGS_FNV_BASIS;
    h = fnv_step(h, (unsigned)x);
    h = fnv_step(h, (unsigned)y);
    h = fnv_step(h, (unsigned)z);
    return table_find_single(slots, mask, fnv_fold(h));
  }
};

// Level-0 cells (stride 1: every probe is a sample corner) taken a cell at a time: the 8 expanded
// samples of cell i (ids idx_base + 8 i + e, e = ex*4 + ey*2 + ez) have their corners on the
// lattice c * 2 + p, p in {0,1,2}^3.  Each of the 27 lattice points is looked up once (9 runs of 3
// along z) and takes one count update for all the samples that touch it; sample e reaches point p
// through its corner q = p - e, which fills the slot of the octant opposite q -- the same slots and
// counts as the per-sample probes of dual_inds_kernel.
template <int W>
__global__ void dual_inds_cells_kernel(ngs_grid dual, const int32_t* __restrict__ cells, int64_t n, int depth,
                                       int64_t idx_base, int32_t* __restrict__ acc, int32_t* __restrict__ cnt) {
  for (int64_t i = ngs_gtid(); i < n; i += ngs_gstride()) {
    const int x0 = cells[i * 3] * 2, y0 = cells[i * 3 + 1] * 2, z0 = cells[i * 3 + 2] * 2;
    const int64_t id0 = idx_base + i * 8;
    // the 9 runs looked up first, all their bitmap loads in flight together, then the updates
    int32_t r[9][3];
#pragma unroll
    for (int pxy = 0; pxy < 9; pxy++) grid_rows_zrun<3>(dual, x0 + pxy / 3, y0 + pxy % 3, z0, r[pxy]);
#pragma unroll
    for (int pxy = 0; pxy < 9; pxy++) {
      const int px = pxy / 3, py = pxy % 3;
#pragma unroll
      for (int pz = 0; pz < 3; pz++) {
        const int64_t row = r[pxy][pz];
        if (row < 0) continue;
        const int nx = px == 1 ? 2 : 1, ny = py == 1 ? 2 : 1, nz = pz == 1 ? 2 : 1;
        atomicAdd(cnt + row, nx * ny * nz);
        for (int ex = px == 2 ? 1 : 0; ex <= (px == 0 ? 0 : 1); ex++)
          for (int ey = py == 2 ? 1 : 0; ey <= (py == 0 ? 0 : 1); ey++)
            for (int ez = pz == 2 ? 1 : 0; ez <= (pz == 0 ? 0 : 1); ez++) {
              const int qx = px - ex, qy = py - ey, qz = pz - ez;
              const int slot = c_octant_slot[(1 - qx) + 2 * (1 - qy) + 4 * (1 - qz)];
              const int32_t id = (int32_t)(id0 + ex * 4 + ey * 2 + ez);
              if constexpr (W == 2) reinterpret_cast<int2*>(acc)[row * 8 + slot] = make_int2(id, depth);
              else acc[row * 8 + slot] = id;
            }
      }
    }
  }
}

extern "C" int ngs_dual_mc_indices_cells(ngs_grid dual, const int32_t* cells, int64_t n_cells, int depth,
                                         int64_t idx_base, int32_t* acc, int slot_words, int32_t* cnt, ngs_stream s) {
  if (!dual.words || dual.stride != 1 || n_cells < 0 || (n_cells > 0 && (!cells || !acc || !cnt)))
    return NGS_ERR_INVALID_ARG;
  if ((slot_words != 1 && slot_words != 2) || (reinterpret_cast<uintptr_t>(acc) & 7u)) return NGS_ERR_INVALID_ARG;
  if (n_cells == 0) return NGS_OK;
  ngs_count_launch();
  if (slot_words == 2)
    dual_inds_cells_kernel<2><<<ngs_blocks(n_cells, 128), 128, 0, (cudaStream_t)s>>>(dual, cells, n_cells, depth,
                                                                                     idx_base, acc, cnt);
  else
    dual_inds_cells_kernel<1><<<ngs_blocks(n_cells, 128), 128, 0, (cudaStream_t)s>>>(dual, cells, n_cells, depth,
                                                                                     idx_base, acc, cnt);
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}

extern "C" int ngs_dual_mc_indices_grid(ngs_grid dual, const int32_t* primal_base, int64_t n_primal, int stride,
                                        int depth, int64_t idx_base, int32_t* acc, int slot_words, int32_t* cnt,
                                        ngs_stream s) {
  if (!dual.words || stride < 1 || n_primal < 0 || (n_primal > 0 && (!primal_base || !acc || !cnt)))
    return NGS_ERR_INVALID_ARG;
  if ((slot_words != 1 && slot_words != 2) || (reinterpret_cast<uintptr_t>(acc) & 7u)) return NGS_ERR_INVALID_ARG;
  if (n_primal == 0) return NGS_OK;
  launch_dual_inds(GridLookup{dual}, primal_base, n_primal, stride, depth, idx_base, acc, slot_words, cnt,
                   (cudaStream_t)s);
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}

extern "C" int ngs_dual_mc_indices_hash(const ngs_hash_table* dual, const int32_t* primal_base, int64_t n_primal,
                                        int stride, int depth, int64_t idx_base, int32_t* acc, int slot_words,
                                        int32_t* cnt, ngs_stream s) {
  if (!dual || !dual->slots || stride < 1 || n_primal < 0 || (n_primal > 0 && (!primal_base || !acc || !cnt)))
    return NGS_ERR_INVALID_ARG;
  if ((slot_words != 1 && slot_words != 2) || (reinterpret_cast<uintptr_t>(acc) & 7u)) return NGS_ERR_INVALID_ARG;
  if (n_primal == 0) return NGS_OK;
  launch_dual_inds(KeyLookup{static_cast<const Slot*>(dual->slots), dual->nslots - 1}, primal_base, n_primal, stride,
                   depth, idx_base, acc, slot_words, cnt, (cudaStream_t)s);
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}

__global__ void select_kernel(const int32_t* __restrict__ cnt, int64_t n, int32_t* __restrict__ keep) {
  for (int64_t i = ngs_gtid(); i < n; i += ngs_gstride()) keep[i] = cnt[i] == 8 ? 1 : 0;
}

// rows of 8 * slot_words int32 (32 or 64 bytes), copied as int4
__global__ void compact_acc_kernel(const int32_t* __restrict__ acc, int quads, const int32_t* __restrict__ keep,
                                   const int64_t* __restrict__ off, int64_t n, int32_t* __restrict__ out) {
  for (int64_t i = ngs_gtid(); i < n; i += ngs_gstride()) {
    if (!keep[i]) continue;
    const int4* src = reinterpret_cast<const int4*>(acc) + i * quads;
    int4* dst = reinterpret_cast<int4*>(out) + off[i] * quads;
    for (int k = 0; k < quads; k++) dst[k] = src[k];
  }
}

extern "C" int ngs_dual_mc_select(const int32_t* cnt, int64_t n, int32_t* keep, ngs_stream s) {
  if (n < 0 || (n > 0 && (!cnt || !keep))) return NGS_ERR_INVALID_ARG;
  if (n == 0) return NGS_OK;
  { ngs_count_launch(); select_kernel<<<ngs_blocks(n, 256), 256, 0, (cudaStream_t)s>>>(cnt, n, keep); }
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}

extern "C" int ngs_dual_mc_compact(const int32_t* acc, int slot_words, const int32_t* keep, const int64_t* keep_offset,
                                   int64_t n, int32_t* acc_out, ngs_stream s) {
  if (n < 0 || (n > 0 && (!acc || !keep || !keep_offset || !acc_out))) return NGS_ERR_INVALID_ARG;
  if (slot_words != 1 && slot_words != 2) return NGS_ERR_INVALID_ARG;
  if ((reinterpret_cast<uintptr_t>(acc) | reinterpret_cast<uintptr_t>(acc_out)) & 15u) return NGS_ERR_INVALID_ARG;
  if (n == 0) return NGS_OK;
  { ngs_count_launch(); compact_acc_kernel<<<ngs_blocks(n, 256), 256, 0, (cudaStream_t)s>>>(acc, 2 * slot_words, keep, keep_offset, n,
                                                                                     acc_out); }
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}

// ----------------------------------------------------------------------------- dual MC
// cnt (optional): the accumulation counts of an uncompacted acc; cubes whose count is not 8 emit
// nothing, which leaves the triangles of the others in the order a compacted acc gives them.
__global__ void dual_count_kernel(const int32_t* __restrict__ acc, int W, const int32_t* __restrict__ cnt, int64_t m,
                                  const float* __restrict__ values, int32_t* __restrict__ vcount) {
  for (int64_t c = ngs_gtid(); c < m; c += ngs_gstride()) {
    if (cnt && cnt[c] != 8) {
      vcount[c] = 0;
      continue;
    }
    float v[8];
#pragma unroll
    for (int i = 0; i < 8; i++) v[i] = values[acc[(c * 8 + i) * W]];
    vcount[c] = num_verts(cube_type(v));
  }
}

// A warp per 32 consecutive cubes.  A thread per cube would leave most lanes idle (most cubes have
// no vertices: 6 of 32 lanes active on average).  Here each lane stages the corner ids, values and
// case of its own cube, if it emits, in shared memory; then the warp takes its cubes' vertices --
// contiguous in the output, since voff is the exclusive scan of the count pass -- 32 at a time:
// vertex j belongs to the last lane whose start offset is at most j (a binary search over the
// lanes' offsets by shuffles), as its k-th vertex, edge c_tri[case][k].
constexpr int EMIT_WARPS = 4;

__global__ void __launch_bounds__(EMIT_WARPS * 32) dual_emit_kernel(
    const int32_t* __restrict__ acc, int W, const int32_t* __restrict__ cnt, int64_t m, const float* __restrict__ pos,
    const float* __restrict__ values, const int64_t* __restrict__ voff, float* __restrict__ tris,
    int32_t* __restrict__ vids) {
  __shared__ int s_id[EMIT_WARPS][32][8];
  __shared__ float s_v[EMIT_WARPS][32][8];
  __shared__ int s_t[EMIT_WARPS][32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t chunks = (m + 31) / 32, step = (int64_t)gridDim.x * EMIT_WARPS;
  for (int64_t ch = (int64_t)blockIdx.x * EMIT_WARPS + w; ch < chunks; ch += step) {
    const int64_t c = ch * 32 + lane;
    const bool in = c < m;
    const int64_t start = in ? voff[c] : 0;
    // a cube emits if its count-pass range is not empty (the last cube: always looked at)
    bool active = in && !(c + 1 < m && voff[c + 1] == start) && !(cnt && cnt[c] != 8);
    int nv = 0;
    if (active) {
      float v[8];
#pragma unroll
      for (int i = 0; i < 8; i++) {
        const int id = acc[(c * 8 + i) * W];
        v[i] = values[id];
        s_id[w][lane][i] = id;
        s_v[w][lane][i] = v[i];
      }
      const int t = cube_type(v);
      s_t[w][lane] = t;
      nv = num_verts(t);
    }
    const int64_t first = __shfl_sync(0xffffffffu, start, 0);
    const int rel = in ? (int)(start - first) : 0x7fffffff;      // this lane's first vertex in the warp's range
    int total = nv;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) total += __shfl_xor_sync(0xffffffffu, total, o);
    __syncwarp();
    for (int j0 = 0; j0 < total; j0 += 32) {                   // warp-uniform trip count
      const int j = j0 + lane;
      int L = 0;
#pragma unroll
      for (int sstep = 16; sstep > 0; sstep >>= 1) {
        const int r = __shfl_sync(0xffffffffu, rel, L + sstep);
        if (r <= j) L += sstep;
      }
      const int rL = __shfl_sync(0xffffffffu, rel, L);
      if (j < total) {
        const int k = j - rL;
        const int e = c_tri[s_t[w][L]][k];
        const int a = c_edge[e][0], b = c_edge[e][1];
        const int ia = s_id[w][L][a], ib = s_id[w][L][b];
        const float p1[3] = {pos[(int64_t)ia * 3], pos[(int64_t)ia * 3 + 1], pos[(int64_t)ia * 3 + 2]};
        const float p2[3] = {pos[(int64_t)ib * 3], pos[(int64_t)ib * 3 + 1], pos[(int64_t)ib * 3 + 2]};
        float out[3];
        sdf_interp(p1, p2, s_v[w][L][a], s_v[w][L][b], out);
        const int64_t o = first + j;
        tris[o * 3] = out[0];
        tris[o * 3 + 1] = out[1];
        tris[o * 3 + 2] = out[2];
        vids[o * 2] = max(ia, ib);
        vids[o * 2 + 1] = min(ia, ib);
      }
    }
    __syncwarp();                                                // the next chunk overwrites the stage
  }
}

extern "C" int ngs_dual_mc_count(const int32_t* acc, int slot_words, const int32_t* cnt, int64_t n_cubes,
                                 const float* values, int32_t* vcount, ngs_stream s) {
  if (n_cubes < 0 || (n_cubes > 0 && (!acc || !values || !vcount))) return NGS_ERR_INVALID_ARG;
  if (slot_words != 1 && slot_words != 2) return NGS_ERR_INVALID_ARG;
  if (n_cubes == 0) return NGS_OK;
  { ngs_count_launch(); dual_count_kernel<<<ngs_blocks(n_cubes, 256), 256, 0, (cudaStream_t)s>>>(acc, slot_words, cnt, n_cubes, values,
                                                                                    vcount); }
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}

extern "C" int ngs_dual_mc_emit(const int32_t* acc, int slot_words, const int32_t* cnt, int64_t n_cubes,
                                const float* pos, const float* values, const int64_t* voffset, float* tris,
                                int32_t* vert_ids, ngs_stream s) {
  if (n_cubes < 0 || (n_cubes > 0 && (!acc || !pos || !values || !voffset || !tris || !vert_ids)))
    return NGS_ERR_INVALID_ARG;
  if (slot_words != 1 && slot_words != 2) return NGS_ERR_INVALID_ARG;
  if (n_cubes == 0) return NGS_OK;
  { ngs_count_launch(); dual_emit_kernel<<<ngs_blocks(n_cubes, EMIT_WARPS * 32), EMIT_WARPS * 32, 0, (cudaStream_t)s>>>(acc, slot_words, cnt, n_cubes, pos, values,
                                                                                             voffset, tris, vert_ids); }
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}

// ----------------------------------------------------------------------------- vertex de-duplication
__global__ void vd_count_kernel(const int32_t* __restrict__ vids, int64_t n, int32_t* __restrict__ cnt) {
  for (int64_t i = ngs_gtid(); i < n; i += ngs_gstride()) atomicAdd(cnt + vids[i * 2], 1);
}

__global__ void vd_scatter_kernel(const int32_t* __restrict__ vids, int64_t n, const int64_t* __restrict__ start,
                                  int32_t* __restrict__ fill, int64_t* __restrict__ sorted) {
  for (int64_t i = ngs_gtid(); i < n; i += ngs_gstride()) {
    const int32_t b = vids[i * 2];
    const int32_t pos = atomicAdd(fill + b, 1);
    sorted[start[b] + pos] = ((int64_t)vids[i * 2 + 1] << 32) | (int64_t)i;
  }
}

// Sort each bucket by (vid1, key index) and flag the first key of every distinct vid1.  One warp
// per bucket: the keys of a bucket are distinct (the low half is the key's index), so each key's
// position is the number of keys below it, counted by broadcasting the bucket through the warp
// 32 keys at a time; then every lane writes its keys straight to their positions.  K keys per lane
// live in registers, so the warp sorts buckets of up to 32 K keys; K is picked per bucket.
template <int K>
NGS_DEV void vd_rank_sort(int64_t s0, int c, int lane, int64_t* __restrict__ sorted, int32_t* __restrict__ first) {
  int64_t mine[K];
  int rank[K];
#pragma unroll
  for (int k = 0; k < K; k++) {
    const int idx = lane + 32 * k;
    mine[k] = idx < c ? sorted[s0 + idx] : INT64_MAX;
    rank[k] = 0;
  }
  const int nchunks = (c + 31) / 32;
  for (int chunk = 0; chunk < nchunks; chunk++) {
    const int64_t other = chunk * 32 + lane < c ? sorted[s0 + chunk * 32 + lane] : INT64_MAX;
    const int lim = min(32, c - chunk * 32);
    for (int j = 0; j < lim; j++) {
      const int64_t o = __shfl_sync(0xffffffffu, other, j);
#pragma unroll
      for (int k = 0; k < K; k++) rank[k] += o < mine[k] ? 1 : 0;
    }
  }
  __syncwarp();
#pragma unroll
  for (int k = 0; k < K; k++)
    if (lane + 32 * k < c) sorted[s0 + rank[k]] = mine[k];
  __syncwarp();
  for (int i = lane; i < c; i += 32)
    first[s0 + i] = (i == 0 || (sorted[s0 + i] >> 32) != (sorted[s0 + i - 1] >> 32)) ? 1 : 0;
  __syncwarp();
}

// A bucket of at most 8 keys sorted by the lane that owns it: the keys in registers, Batcher's
// 19-comparator odd-even merge network (empty slots hold INT64_MAX and stay at the end), then the
// sorted keys and the first-of-vid1 flags written back.
constexpr int VD_LANE_MAX = 8;
NGS_DEV void vd_lane_sort(int64_t s0, int c, int64_t* __restrict__ sorted, int32_t* __restrict__ first) {
  int64_t k[VD_LANE_MAX];
#pragma unroll
  for (int i = 0; i < VD_LANE_MAX; i++) k[i] = i < c ? sorted[s0 + i] : INT64_MAX;
  constexpr int net[19][2] = {{0, 1}, {2, 3}, {4, 5}, {6, 7}, {0, 2}, {1, 3}, {4, 6}, {5, 7}, {1, 2}, {5, 6},
                              {0, 4}, {1, 5}, {2, 6}, {3, 7}, {2, 4}, {3, 5}, {1, 2}, {3, 4}, {5, 6}};
#pragma unroll
  for (int q = 0; q < 19; q++) {
    const int64_t a = k[net[q][0]], b = k[net[q][1]];
    k[net[q][0]] = a < b ? a : b;
    k[net[q][1]] = a < b ? b : a;
  }
#pragma unroll
  for (int i = 0; i < VD_LANE_MAX; i++) {
    if (i < c) {
      sorted[s0 + i] = k[i];
      first[s0 + i] = (i == 0 || (k[i] >> 32) != (k[i - 1 > 0 ? i - 1 : 0] >> 32)) ? 1 : 0;
    }
  }
}

__global__ void __launch_bounds__(256, 4) vd_sort_kernel(const int64_t* __restrict__ start, const int32_t* __restrict__ count, int64_t nb,
                               int64_t* __restrict__ sorted, int32_t* __restrict__ first) {
  const int lane = threadIdx.x & 31;
  const int64_t warp0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  // a warp reads 32 bucket counts at once (most buckets are empty or hold a few keys); the buckets of
  // 2..8 keys are sorted by their own lanes at once, those of 9..512 keys by the whole warp one after
  // the other
  for (int64_t base = warp0 * 32; base < nb; base += nwarps * 32) {
    const int64_t b = base + lane;
    const int c = b < nb ? count[b] : 0;
    if (c == 1) first[start[b]] = 1;
    else if (c >= 2 && c <= VD_LANE_MAX) vd_lane_sort(start[b], c, sorted, first);
    unsigned todo = __ballot_sync(0xffffffffu, c > VD_LANE_MAX && c <= 512);
    while (todo) {
      const int src = __ffs(todo) - 1;
      todo &= todo - 1;
      const int cb = __shfl_sync(0xffffffffu, c, src);
      const int64_t s0 = start[base + src];
      if (cb <= 32) vd_rank_sort<1>(s0, cb, lane, sorted, first);
      else if (cb <= 128) vd_rank_sort<4>(s0, cb, lane, sorted, first);
      else vd_rank_sort<16>(s0, cb, lane, sorted, first);
    }
    // larger buckets (the corners of coarse cells shared by many fine dual cubes): vd_sort_big_kernel
  }
}

// Buckets of more than 512 keys: one block per bucket, bitonic sort in shared memory (up to
// VD_BIG_MAX keys); beyond that one thread sorts by insertion (not produced by these dual grids).
// Each block scans a contiguous stretch of the bucket counts, 256 at a time, collects the large
// ones and sorts them one after the other.
constexpr int VD_BIG_MAX = 4096;

__global__ void __launch_bounds__(256) vd_sort_big_kernel(const int64_t* __restrict__ start,
                                                          const int32_t* __restrict__ count, int64_t nb,
                                                          int64_t* __restrict__ sorted, int32_t* __restrict__ first) {
  __shared__ int64_t keys[VD_BIG_MAX];
  __shared__ int64_t found[256];
  __shared__ int nfound;
  const int64_t per = (nb + gridDim.x - 1) / gridDim.x;
  const int64_t b0 = (int64_t)blockIdx.x * per, b1 = min(nb, b0 + per);
  for (int64_t base = b0; base < b1; base += blockDim.x) {
    if (threadIdx.x == 0) nfound = 0;
    __syncthreads();
    const int64_t b = base + threadIdx.x;
    if (b < b1 && count[b] > 512) found[atomicAdd(&nfound, 1)] = b;
    __syncthreads();
    const int nf = nfound;
    for (int f = 0; f < nf; f++) {
      const int64_t bk = found[f];
      const int64_t s0 = start[bk];
      const int c = count[bk];
      if (c <= VD_BIG_MAX) {
        int P = 1;
        while (P < c) P <<= 1;
        for (int i = threadIdx.x; i < P; i += blockDim.x) keys[i] = i < c ? sorted[s0 + i] : INT64_MAX;
        __syncthreads();
        for (int k = 2; k <= P; k <<= 1) {
          for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < P; i += blockDim.x) {
              const int l = i ^ j;
              if (l > i) {
                const int64_t a = keys[i], bb = keys[l];
                const bool up = (i & k) == 0;
                if ((a > bb) == up) {
                  keys[i] = bb;
                  keys[l] = a;
                }
              }
            }
            __syncthreads();
          }
        }
        for (int i = threadIdx.x; i < c; i += blockDim.x) {
          sorted[s0 + i] = keys[i];
          first[s0 + i] = (i == 0 || (keys[i] >> 32) != (keys[i - 1] >> 32)) ? 1 : 0;
        }
        __syncthreads();
      } else if (threadIdx.x == 0) {
        for (int i = 1; i < c; i++) {
          const int64_t key = sorted[s0 + i];
          int j = i - 1;
          while (j >= 0 && sorted[s0 + j] > key) {
            sorted[s0 + j + 1] = sorted[s0 + j];
            j--;
          }
          sorted[s0 + j + 1] = key;
        }
        for (int i = 0; i < c; i++)
          first[s0 + i] = (i == 0 || (sorted[s0 + i] >> 32) != (sorted[s0 + i - 1] >> 32)) ? 1 : 0;
      }
      __syncthreads();
    }
  }
}

__global__ void vd_emit_kernel(const int32_t* __restrict__ vids, const float* __restrict__ tris, int64_t n,
                               const int64_t* __restrict__ start, const int32_t* __restrict__ count,
                               const int64_t* __restrict__ sorted, const int64_t* __restrict__ vertex_id,
                               int64_t* __restrict__ faces, float* __restrict__ verts) {
  for (int64_t i = ngs_gtid(); i < n; i += ngs_gstride()) {
    const int32_t b = vids[i * 2];
    const int64_t v1 = vids[i * 2 + 1];
    int64_t lo = start[b], hi = start[b] + count[b] - 1;
    // first position whose vid1 >= v1
    while (lo < hi) {
      const int64_t mid = (lo + hi) >> 1;
      if ((sorted[mid] >> 32) < v1) lo = mid + 1; else hi = mid;
    }
    const int64_t vid = vertex_id[lo];
    faces[i] = vid;
    if ((sorted[lo] & 0xffffffffll) == i) {
      verts[vid * 3] = tris[i * 3];
      verts[vid * 3 + 1] = tris[i * 3 + 1];
      verts[vid * 3 + 2] = tris[i * 3 + 2];
    }
  }
}

extern "C" int ngs_vdedup_count(const int32_t* vert_ids, int64_t n_keys, int32_t* bucket_count, ngs_stream s) {
  if (n_keys < 0 || (n_keys > 0 && (!vert_ids || !bucket_count))) return NGS_ERR_INVALID_ARG;
  if (n_keys == 0) return NGS_OK;
  if (n_keys > 0x7fffffffLL) return NGS_ERR_INVALID_ARG;
  { ngs_count_launch(); vd_count_kernel<<<ngs_blocks(n_keys, 256), 256, 0, (cudaStream_t)s>>>(vert_ids, n_keys, bucket_count); }
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}

extern "C" int ngs_vdedup_sort(const int32_t* vert_ids, int64_t n_keys, const int64_t* bucket_start, int64_t n_buckets,
                               int32_t* bucket_fill, int64_t* sorted_keys, int32_t* first, ngs_stream s) {
  if (n_keys < 0 || n_buckets < 0 || (n_keys > 0 && (!vert_ids || !bucket_start || !bucket_fill || !sorted_keys || !first)))
    return NGS_ERR_INVALID_ARG;
  if (n_keys == 0) return NGS_OK;
  cudaStream_t st = (cudaStream_t)s;
  { ngs_count_launch(); vd_scatter_kernel<<<ngs_blocks(n_keys, 256), 256, 0, st>>>(vert_ids, n_keys, bucket_start, bucket_fill, sorted_keys); }
  { ngs_count_launch(); vd_sort_kernel<<<ngs_blocks(n_buckets, 256), 256, 0, st>>>(bucket_start, bucket_fill, n_buckets, sorted_keys, first); }
  { ngs_count_launch(); vd_sort_big_kernel<<<(unsigned)std::min<int64_t>((int64_t)ngs_num_sms() * 8, (n_buckets + 255) / 256), 256, 0, st>>>(bucket_start, bucket_fill, n_buckets, sorted_keys, first); }
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}

extern "C" int ngs_vdedup_emit(const int32_t* vert_ids, const float* tris, int64_t n_keys, const int64_t* bucket_start,
                               const int32_t* bucket_count, const int64_t* sorted_keys, const int64_t* vertex_id,
                               int64_t* faces, float* vertices, ngs_stream s) {
  if (n_keys < 0 || (n_keys > 0 && (!vert_ids || !tris || !bucket_start || !bucket_count || !sorted_keys ||
                                    !vertex_id || !faces || !vertices)))
    return NGS_ERR_INVALID_ARG;
  if (n_keys == 0) return NGS_OK;
  { ngs_count_launch(); vd_emit_kernel<<<ngs_blocks(n_keys, 256), 256, 0, (cudaStream_t)s>>>(vert_ids, tris, n_keys, bucket_start,
                                                                     bucket_count, sorted_keys, vertex_id, faces,
                                                                     vertices); }
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}

// ----------------------------------------------------------------------------- conformal tree helpers
__global__ void children_kernel(const int32_t* __restrict__ par, int64_t n, int stride, int32_t* __restrict__ out) {
  const int64_t total = n * 8;
  for (int64_t t = ngs_gtid(); t < total; t += ngs_gstride()) {
    const int64_t p = t >> 3;
    const int c = (int)(t & 7);
    out[t * 3] = par[p * 3] + ((c >> 2) & 1) * stride;
    out[t * 3 + 1] = par[p * 3 + 1] + ((c >> 1) & 1) * stride;
    out[t * 3 + 2] = par[p * 3 + 2] + (c & 1) * stride;
  }
}

__global__ void leaf_kernel(const int32_t* __restrict__ cells, int64_t n, ngs_grid g, int32_t* __restrict__ leaf) {
  for (int64_t i = ngs_gtid(); i < n; i += ngs_gstride())
    leaf[i] = g.words ? (grid_row(g, cells[i * 3], cells[i * 3 + 1], cells[i * 3 + 2]) < 0 ? 1 : 0) : 1;
}

__global__ void compact_coords_kernel(const int32_t* __restrict__ c, const int32_t* __restrict__ keep,
                                      const int64_t* __restrict__ off, int64_t n, int32_t* __restrict__ out) {
  for (int64_t i = ngs_gtid(); i < n; i += ngs_gstride()) {
    if (!keep[i]) continue;
    const int64_t o = off[i];
    out[o * 3] = c[i * 3];
    out[o * 3 + 1] = c[i * 3 + 1];
    out[o * 3 + 2] = c[i * 3 + 2];
  }
}

__global__ void expand_kernel(const int32_t* __restrict__ c, int64_t n, int n_up, int stride, float evs,
                              int32_t* __restrict__ out, float* __restrict__ pos) {
  const int e3 = n_up * n_up * n_up;
  const int64_t total = n * e3;
  for (int64_t t = ngs_gtid(); t < total; t += ngs_gstride()) {
    const int64_t i = t / e3;
    const int e = (int)(t - i * e3);
    const int ex = e / (n_up * n_up), ey = (e / n_up) % n_up, ez = e % n_up;
    const int v[3] = {c[i * 3] * n_up + ex * stride, c[i * 3 + 1] * n_up + ey * stride, c[i * 3 + 2] * n_up + ez * stride};
#pragma unroll
    for (int a = 0; a < 3; a++) {
      out[t * 3 + a] = v[a];
      if (pos) pos[t * 3 + a] = __fmul_rn((float)(v[a] + stride), evs);
    }
  }
}

extern "C" int ngs_conformal_children(const int32_t* parents, int64_t n_parents, int stride, int32_t* children,
                                      ngs_stream s) {
  if (n_parents < 0 || (n_parents > 0 && (!parents || !children))) return NGS_ERR_INVALID_ARG;
  if (n_parents == 0) return NGS_OK;
  { ngs_count_launch(); children_kernel<<<ngs_blocks(n_parents * 8, 256), 256, 0, (cudaStream_t)s>>>(parents, n_parents, stride, children); }
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}

extern "C" int ngs_leaf_flags(const int32_t* cells, int64_t n, ngs_grid finer_parents, int32_t* leaf, ngs_stream s) {
  if (n < 0 || (n > 0 && (!cells || !leaf))) return NGS_ERR_INVALID_ARG;
  if (n == 0) return NGS_OK;
  { ngs_count_launch(); leaf_kernel<<<ngs_blocks(n, 256), 256, 0, (cudaStream_t)s>>>(cells, n, finer_parents, leaf); }
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}

extern "C" int ngs_compact_coords(const int32_t* coords, const int32_t* keep, const int64_t* keep_offset, int64_t n,
                                  int32_t* out, ngs_stream s) {
  if (n < 0 || (n > 0 && (!coords || !keep || !keep_offset || !out))) return NGS_ERR_INVALID_ARG;
  if (n == 0) return NGS_OK;
  { ngs_count_launch(); compact_coords_kernel<<<ngs_blocks(n, 256), 256, 0, (cudaStream_t)s>>>(coords, keep, keep_offset, n, out); }
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}

extern "C" int ngs_expand_cells(const int32_t* cells, int64_t n, int n_up, int stride, float evs, int32_t* out,
                                float* pos, ngs_stream s) {
  if (n < 0 || n_up < 1 || (n > 0 && (!cells || !out))) return NGS_ERR_INVALID_ARG;
  if (n == 0) return NGS_OK;
  { ngs_count_launch(); expand_kernel<<<ngs_blocks(n * n_up * n_up * n_up, 256), 256, 0, (cudaStream_t)s>>>(cells, n, n_up, stride, evs, out,
                                                                                     pos); }
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}
