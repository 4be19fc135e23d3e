// Device-wide exclusive scan (reduce-then-scan, three launches) over int64
// values produced by a Load functor and consumed by a Store functor.  Used for
// CSR row pointers, triangle offsets, voxel ranks and compaction offsets.
#pragma once
#include "ngs_common.cuh"

constexpr int NGS_SCAN_THREADS = 512;
constexpr int NGS_SCAN_ITEMS = 8;
constexpr int64_t NGS_SCAN_TILE = (int64_t)NGS_SCAN_THREADS * NGS_SCAN_ITEMS;

inline int64_t ngs_scan_tiles(int64_t n) { return (n + NGS_SCAN_TILE - 1) / NGS_SCAN_TILE; }
inline size_t ngs_scan_ws_bytes(int64_t n) { return (size_t)(ngs_scan_tiles(n) + 1) * sizeof(int64_t); }

// Inclusive block scan of one value per thread; returns the inclusive prefix and
// writes the block total to *total.
NGS_DEV int64_t block_inclusive_scan(int64_t v, int64_t* total) {
  __shared__ int64_t warp_tot[32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int64_t t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += t;
  }
  if (lane == 31) warp_tot[wid] = v;
  __syncthreads();
  if (wid == 0) {
    const int nw = (blockDim.x + 31) >> 5;
    int64_t t = lane < nw ? warp_tot[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int64_t u = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= o) t += u;
    }
    warp_tot[lane] = t;
  }
  __syncthreads();
  if (wid > 0) v += warp_tot[wid - 1];
  *total = warp_tot[((blockDim.x + 31) >> 5) - 1];
  __syncthreads();
  return v;
}

template <class Load>
__global__ void __launch_bounds__(NGS_SCAN_THREADS) scan_reduce_kernel(Load ld, int64_t n, int64_t* tile_sums) {
  const int64_t base = (int64_t)blockIdx.x * NGS_SCAN_TILE;
  int64_t s = 0;
#pragma unroll
  for (int i = 0; i < NGS_SCAN_ITEMS; i++) {
    const int64_t idx = base + (int64_t)i * NGS_SCAN_THREADS + threadIdx.x;
    if (idx < n) s += ld(idx);
  }
  s = warp_sum(s);
  __shared__ int64_t ws[NGS_SCAN_THREADS / 32];
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    int64_t t = threadIdx.x < NGS_SCAN_THREADS / 32 ? ws[threadIdx.x] : 0;
    t = warp_sum(t);
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = t;
  }
}

// Single block: exclusive scan of the tile sums in place, total to tile_sums[ntiles] and *total.
static __global__ void __launch_bounds__(1024) scan_tiles_kernel(int64_t* tile_sums, int64_t ntiles, int64_t* total) {
  int64_t carry = 0;
  for (int64_t base = 0; base < ntiles; base += blockDim.x) {
    const int64_t i = base + threadIdx.x;
    const int64_t v = i < ntiles ? tile_sums[i] : 0;
    int64_t tot;
    const int64_t inc = block_inclusive_scan(v, &tot);
    if (i < ntiles) tile_sums[i] = carry + inc - v;
    carry += tot;
  }
  if (threadIdx.x == 0) {
    tile_sums[ntiles] = carry;
    if (total) *total = carry;
  }
}

template <class Load, class Store>
__global__ void __launch_bounds__(NGS_SCAN_THREADS) scan_apply_kernel(Load ld, Store st, int64_t n,
                                                                     const int64_t* tile_sums) {
  const int64_t base = (int64_t)blockIdx.x * NGS_SCAN_TILE + (int64_t)threadIdx.x * NGS_SCAN_ITEMS;
  int64_t v[NGS_SCAN_ITEMS];
  int64_t s = 0;
#pragma unroll
  for (int i = 0; i < NGS_SCAN_ITEMS; i++) {
    v[i] = (base + i < n) ? ld(base + i) : 0;
    s += v[i];
  }
  int64_t tot;
  const int64_t inc = block_inclusive_scan(s, &tot);
  int64_t run = tile_sums[blockIdx.x] + inc - s;
#pragma unroll
  for (int i = 0; i < NGS_SCAN_ITEMS; i++) {
    if (base + i < n) st(base + i, run);
    run += v[i];
  }
}

template <class Load, class Store>
int ngs_scan(Load ld, Store st, int64_t n, int64_t* total, void* ws, size_t ws_bytes, cudaStream_t s) {
  if (n == 0) {
    if (total) cudaMemsetAsync(total, 0, sizeof(int64_t), s);
    return NGS_OK;
  }
  if (!ws || ws_bytes < ngs_scan_ws_bytes(n)) return NGS_ERR_OOM;
  const int64_t tiles = ngs_scan_tiles(n);
  if (tiles > 0x7fffffffLL) return NGS_ERR_INVALID_ARG;
  int64_t* tile_sums = static_cast<int64_t*>(ws);
  { ngs_count_launch(); scan_reduce_kernel<<<(unsigned)tiles, NGS_SCAN_THREADS, 0, s>>>(ld, n, tile_sums); }
  { ngs_count_launch(); scan_tiles_kernel<<<1, 1024, 0, s>>>(tile_sums, tiles, total); }
  { ngs_count_launch(); scan_apply_kernel<<<(unsigned)tiles, NGS_SCAN_THREADS, 0, s>>>(ld, st, n, tile_sums); }
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}
