// Fused neighbour queries of a voxel level: source (point or voxel) + offset -> rank-bitmap probe ->
// compaction, in two passes over tiles of 256 sources, with no [K, N] intermediate.
//
// Replaces the reference's query chain (jspsr/core/_hash_backend.py:176-228): kernel_hash_cuda builds
// a [K, N] int64 key matrix (csrc/common/hashmap_cuda.cu:204-235), hash_table_query probes it, and
// torch.where compacts the hits -- three full passes over K x N.  Here pass 1 probes each (source,
// offset) once in the L2-resident bitmap and keeps one bit per pair (16 bytes per source for up to
// 128 offsets) plus the counts; a scan of the counts gives every pair its output slot; pass 2 probes
// the hits again and writes (source, target, offset index) straight to their slots, in either of the
// reference's two orders:
//   k-major ("not transposed"): all hits of offset 0 by ascending source, then offset 1, ...;
//                               counts per offset (the reference's nbsizes over K)
//   source-major (transposed):  all hits of source 0 by ascending offset, then source 1, ...;
//                               counts per source (nbsizes over N)
// Source quantisation follows the reference in fp32: a non-conv query snaps the source to the target
// lattice as floor((src + src_stride / 2) / stride) * stride (_hash_backend.py:196-198); a
// conv-based query uses the source coordinates as they are.  A probe hits only a cell of the level's
// lattice that holds a voxel: an off-lattice probe misses, as an absent key would in the hash table.
#include "ngs_common.cuh"
#include "scan.cuh"

constexpr int NB_TILE = 256;          // sources per block
constexpr int NB_MAX_K = 128;         // offsets per query (a 5x5x5 range is 125)
constexpr int NB_WORDS = NB_MAX_K / 32;

struct NbQuery {
  ngs_grid g;
  const int64_t* row_of_rank;   // optional: row of each lexicographic rank (levels with unsorted coords)
  const void* src;              // float [n, 3] or int32 [n, 3]
  int src_float;
  int64_t n;
  int src_stride;
  int conv;
  const int32_t* offsets;       // int32 [k, 3], in units of the target stride
  int k;
};

// Row of the lattice cell at (x, y, z), or -1 when the cell is off the lattice, outside the box or empty.
NGS_DEV int64_t nb_row(const NbQuery& q, int x, int y, int z) {
  const ngs_grid& g = q.g;
  const int dx = x - g.origin[0], dy = y - g.origin[1], dz = z - g.origin[2];
  if ((dx | dy | dz) < 0 || ((dx | dy | dz) & (g.stride - 1))) return -1;
  const int64_t r = grid_row(g, x, y, z);
  if (r < 0 || !q.row_of_rank) return r;
  return q.row_of_rank[r];
}

// The source's lattice cell on the target level (the probe origin).
NGS_DEV void nb_origin(const NbQuery& q, int64_t i, int (&c)[3]) {
  const int st = q.g.stride;
  if (q.src_float) {
    const float* p = static_cast<const float*>(q.src) + i * 3;
    const float half = 0.5f * (float)q.src_stride, inv = 1.0f / (float)st;
#pragma unroll
    for (int a = 0; a < 3; a++)
      c[a] = q.conv ? (int)p[a] : (int)__fmul_rn(floorf(__fmul_rn(__fadd_rn(p[a], half), inv)), (float)st);
  } else {
    const int32_t* p = static_cast<const int32_t*>(q.src) + i * 3;
    const float half = 0.5f * (float)q.src_stride, inv = 1.0f / (float)st;
#pragma unroll
    for (int a = 0; a < 3; a++)
      c[a] = q.conv ? p[a] : (int)__fmul_rn(floorf(__fmul_rn(__fadd_rn((float)p[a], half), inv)), (float)st);
  }
}

// Pass 1: hit bits of every (source, offset) and the counts.  k-major: tile_counts[j * ntiles + tile]
// (hits of offset j in the tile) and per_offset[j]; source-major: per_source[i].
__global__ void __launch_bounds__(NB_TILE) nb_count_kernel(NbQuery q, uint32_t* __restrict__ masks, int transposed,
                                                           int64_t* __restrict__ tile_counts,
                                                           unsigned long long* __restrict__ per_offset,
                                                           int64_t* __restrict__ per_source) {
  __shared__ int s_cnt[NB_MAX_K];
  const int64_t ntiles = (q.n + NB_TILE - 1) / NB_TILE;
  const int lane = threadIdx.x & 31;
  for (int j = threadIdx.x; j < q.k; j += blockDim.x) s_cnt[j] = 0;
  __syncthreads();
  const int64_t i = (int64_t)blockIdx.x * NB_TILE + threadIdx.x;
  const bool live = i < q.n;
  int c[3] = {0, 0, 0};
  if (live) nb_origin(q, i, c);
  const int st = q.g.stride;
  uint32_t m[NB_WORDS] = {0u, 0u, 0u, 0u};
  for (int j = 0; j < q.k; j++) {
    bool hit = false;
    if (live) {
      const int32_t* o = q.offsets + 3 * j;
      hit = nb_row(q, c[0] + o[0] * st, c[1] + o[1] * st, c[2] + o[2] * st) >= 0;
    }
    if (hit) m[j >> 5] |= 1u << (j & 31);
    if (!transposed) {
      const unsigned b = __ballot_sync(0xffffffffu, hit);
      if (lane == 0 && b) atomicAdd(&s_cnt[j], __popc(b));
    }
  }
  if (live) {
    reinterpret_cast<uint4*>(masks)[i] = make_uint4(m[0], m[1], m[2], m[3]);
    if (transposed) per_source[i] = __popc(m[0]) + __popc(m[1]) + __popc(m[2]) + __popc(m[3]);
  }
  if (!transposed) {
    __syncthreads();
    for (int j = threadIdx.x; j < q.k; j += blockDim.x) {
      tile_counts[(int64_t)j * ntiles + blockIdx.x] = s_cnt[j];
      if (s_cnt[j]) atomicAdd(per_offset + j, (unsigned long long)s_cnt[j]);
    }
  }
}

// Pass 2: every hit written to its slot.  start: k-major, the exclusive scan of tile_counts
// (slot of the first hit of offset j in tile t); source-major, the exclusive scan of per_source.
__global__ void __launch_bounds__(NB_TILE) nb_fill_kernel(NbQuery q, const uint32_t* __restrict__ masks,
                                                          int transposed, const int64_t* __restrict__ start,
                                                          int64_t* __restrict__ src_ids, int64_t* __restrict__ tgt_ids,
                                                          int32_t* __restrict__ kidx) {
  constexpr int NW = NB_TILE / 32;
  __shared__ int s_wcnt[NB_MAX_K][NW];     // hits of offset j in warp w, then its exclusive prefix over warps
  const int64_t ntiles = (q.n + NB_TILE - 1) / NB_TILE;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int64_t i = (int64_t)blockIdx.x * NB_TILE + threadIdx.x;
  const bool live = i < q.n;
  uint4 mv = make_uint4(0u, 0u, 0u, 0u);
  if (live) mv = reinterpret_cast<const uint4*>(masks)[i];
  const uint32_t m[NB_WORDS] = {mv.x, mv.y, mv.z, mv.w};
  int c[3] = {0, 0, 0};
  if (live) nb_origin(q, i, c);
  const int st = q.g.stride;
  if (transposed) {
    if (!live) return;
    int64_t pos = start[i];
    for (int w = 0; w < NB_WORDS; w++) {
      uint32_t bits = m[w];
      while (bits) {
        const int j = w * 32 + __ffs(bits) - 1;
        bits &= bits - 1;
        const int32_t* o = q.offsets + 3 * j;
        src_ids[pos] = i;
        tgt_ids[pos] = nb_row(q, c[0] + o[0] * st, c[1] + o[1] * st, c[2] + o[2] * st);
        kidx[pos] = j;
        pos++;
      }
    }
    return;
  }
  for (int j = 0; j < q.k; j++) {
    const unsigned b = __ballot_sync(0xffffffffu, (m[j >> 5] >> (j & 31)) & 1u);
    if (lane == 0) s_wcnt[j][wid] = __popc(b);
  }
  __syncthreads();
  for (int j = threadIdx.x; j < q.k; j += blockDim.x) {
    int run = 0;
    for (int w = 0; w < NW; w++) {
      const int t = s_wcnt[j][w];
      s_wcnt[j][w] = run;
      run += t;
    }
  }
  __syncthreads();
  const unsigned lt = (1u << lane) - 1u;
  for (int j = 0; j < q.k; j++) {
    const bool hit = (m[j >> 5] >> (j & 31)) & 1u;
    const unsigned b = __ballot_sync(0xffffffffu, hit);
    if (!hit) continue;
    const int64_t pos = start[(int64_t)j * ntiles + blockIdx.x] + s_wcnt[j][wid] + __popc(b & lt);
    const int32_t* o = q.offsets + 3 * j;
    src_ids[pos] = i;
    tgt_ids[pos] = nb_row(q, c[0] + o[0] * st, c[1] + o[1] * st, c[2] + o[2] * st);
    kidx[pos] = j;
  }
}

static bool nb_args_ok(const ngs_grid& g, const void* src, int64_t n, int src_stride, const int32_t* offsets, int k) {
  if (!g.words || g.stride < 1 || (g.stride & (g.stride - 1)) || n < 0 || k < 1 || k > NB_MAX_K || !offsets)
    return false;
  if (n > 0 && !src) return false;
  return src_stride >= 1;
}

extern "C" int64_t ngs_grid_neighbours_tiles(int64_t n) { return (n + NB_TILE - 1) / NB_TILE; }

extern "C" int ngs_grid_neighbours_count(ngs_grid g, const int64_t* row_of_rank, const void* src, int src_float,
                                         int64_t n, int src_stride, int conv, const int32_t* offsets, int k,
                                         int transposed, uint32_t* masks, int64_t* tile_counts, int64_t* per_offset,
                                         int64_t* per_source, ngs_stream s) {
  if (!nb_args_ok(g, src, n, src_stride, offsets, k)) return NGS_ERR_INVALID_ARG;
  if (transposed ? (n > 0 && (!masks || !per_source)) : (!per_offset || (n > 0 && (!masks || !tile_counts))))
    return NGS_ERR_INVALID_ARG;
  cudaStream_t st = (cudaStream_t)s;
  if (!transposed) cudaMemsetAsync(per_offset, 0, (size_t)k * sizeof(int64_t), st);
  if (n == 0) return NGS_OK;
  const NbQuery q{g, row_of_rank, src, src_float, n, src_stride, conv, offsets, k};
  { ngs_count_launch(); nb_count_kernel<<<(unsigned)ngs_grid_neighbours_tiles(n), NB_TILE, 0, st>>>(
      q, masks, transposed, tile_counts, reinterpret_cast<unsigned long long*>(per_offset), per_source); }
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}

extern "C" int ngs_grid_neighbours_fill(ngs_grid g, const int64_t* row_of_rank, const void* src, int src_float,
                                        int64_t n, int src_stride, int conv, const int32_t* offsets, int k,
                                        int transposed, const uint32_t* masks, const int64_t* start, int64_t* src_ids,
                                        int64_t* tgt_ids, int32_t* kidx, ngs_stream s) {
  if (!nb_args_ok(g, src, n, src_stride, offsets, k)) return NGS_ERR_INVALID_ARG;
  if (n == 0) return NGS_OK;
  if (!masks || !start || !src_ids || !tgt_ids || !kidx) return NGS_ERR_INVALID_ARG;
  const NbQuery q{g, row_of_rank, src, src_float, n, src_stride, conv, offsets, k};
  { ngs_count_launch(); nb_fill_kernel<<<(unsigned)ngs_grid_neighbours_tiles(n), NB_TILE, 0, (cudaStream_t)s>>>(
      q, masks, transposed, start, src_ids, tgt_ids, kidx); }
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}
