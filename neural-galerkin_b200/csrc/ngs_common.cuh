// Shared device helpers of the B200 screened-Poisson library (libngs).
//
// Voxel index ("rank bitmap"): a level's voxels live on a regular lattice of
// pitch `stride` (finest-voxel units).  Over the level's bounding box we keep
// one bit per lattice cell, 64 cells per 16-byte word together with the
// exclusive count of set bits before the word.  A voxel's row index is then
//     rank(word) + popc(bits & below(bit))
// which is exactly its position in the lexicographically sorted (x, y, z)
// coordinate list -- the order `torch.unique(dim=0)` gives the reference
// (jspsr/core/ops.py:103-127).  A lookup is one 128-bit load; the 5x5x5
// neighbourhood of a voxel touches at most 50 consecutive-in-z words.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "../../include/ngs.h"

#define NGS_DEV __device__ __forceinline__

struct __align__(16) GridWord {
  uint32_t rank;
  uint32_t pad;
  unsigned long long bits;
};

// Cell (i, j, k) of the box -> word ((i * dims1 + j) * zwords + k / 64), bit k % 64.
NGS_DEV int64_t grid_row(const ngs_grid& g, int x, int y, int z) {
  const int dx = x - g.origin[0], dy = y - g.origin[1], dz = z - g.origin[2];
  if ((dx | dy | dz) < 0) return -1;
  const int i = dx >> g.log2_stride, j = dy >> g.log2_stride, k = dz >> g.log2_stride;
  if (i >= g.dims[0] || j >= g.dims[1] || k >= g.dims[2]) return -1;
  const int64_t w = ((int64_t)i * g.dims[1] + j) * g.zwords + (k >> 6);
  const uint4 v = __ldg(reinterpret_cast<const uint4*>(g.words) + w);
  const unsigned long long bits = (unsigned long long)v.z | ((unsigned long long)v.w << 32);
  const int b = k & 63;
  if (!((bits >> b) & 1ull)) return -1;
  return (int64_t)v.x + __popcll(bits & ((1ull << b) - 1ull));
}

// Rows of K consecutive cells along z, (x, y, z + t * stride) for t = 0 .. K-1, or -1 where absent.
// The run covers at most two bitmap words; each is loaded once.
template <int K>
NGS_DEV void grid_rows_zrun(const ngs_grid& g, int x, int y, int z, int32_t (&r)[K]) {
#pragma unroll
  for (int t = 0; t < K; t++) r[t] = -1;
  const int dx = x - g.origin[0], dy = y - g.origin[1], dz = z - g.origin[2];
  if ((dx | dy) < 0) return;
  const int i = dx >> g.log2_stride, j = dy >> g.log2_stride;
  if (i >= g.dims[0] || j >= g.dims[1]) return;
  const uint4* row = reinterpret_cast<const uint4*>(g.words) + ((int64_t)i * g.dims[1] + j) * g.zwords;
  const int k0 = dz >> g.log2_stride;               // arithmetic shift: floor for cells below the box
  int have = -1;
  uint4 v = make_uint4(0, 0, 0, 0);
#pragma unroll
  for (int t = 0; t < K; t++) {
    const int k = k0 + t;
    if (k < 0 || k >= g.dims[2]) continue;
    const int w = k >> 6;
    if (w != have) {
      v = __ldg(row + w);
      have = w;
    }
    const unsigned long long bits = (unsigned long long)v.z | ((unsigned long long)v.w << 32);
    const int b = k & 63;
    if ((bits >> b) & 1ull) r[t] = (int32_t)(v.x + (unsigned)__popcll(bits & ((1ull << b) - 1ull)));
  }
}

NGS_DEV int64_t grid_word_index(const ngs_grid& g, int x, int y, int z, int* bit) {
  const int dx = x - g.origin[0], dy = y - g.origin[1], dz = z - g.origin[2];
  if ((dx | dy | dz) < 0) return -1;
  const int i = dx >> g.log2_stride, j = dy >> g.log2_stride, k = dz >> g.log2_stride;
  if (i >= g.dims[0] || j >= g.dims[1] || k >= g.dims[2]) return -1;
  *bit = k & 63;
  return ((int64_t)i * g.dims[1] + j) * g.zwords + (k >> 6);
}

// A row's slot of stencil offset o (0..124) under its 128-bit offset mask: the set bits below o.
NGS_DEV int popc_below(const uint4 m, int o) {
  // number of set bits of the 128-bit mask m strictly below bit o
  const unsigned w[4] = {m.x, m.y, m.z, m.w};
  int c = 0;
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const int lo = i * 32;
    if (o >= lo + 32) c += __popc(w[i]);
    else if (o > lo) c += __popc(w[i] & ((1u << (o - lo)) - 1u));
  }
  return c;
}

// ----------------------------------------------------------------------------- B-spline
// Quadratic B-spline scaled by 2 (jspsr/bases/bezier_tensor.py:17-22,36-54).
NGS_DEV float bspline(float x) {
  if (x >= -1.5f && x < -0.5f) return (x + 1.5f) * (x + 1.5f);
  if (x >= -0.5f && x < 0.5f) return -2.f * x * x + 1.5f;
  if (x >= 0.5f && x < 1.5f) return (x - 1.5f) * (x - 1.5f);
  return 0.f;
}
NGS_DEV float bspline_d(float x) {
  if (x >= -1.5f && x < -0.5f) return 2.f * x + 3.f;
  if (x >= -0.5f && x < 0.5f) return -4.f * x;
  if (x >= 0.5f && x < 1.5f) return 2.f * x - 3.f;
  return 0.f;
}
NGS_DEV double bspline64(double x) {
  if (x >= -1.5 && x < -0.5) return (x + 1.5) * (x + 1.5);
  if (x >= -0.5 && x < 0.5) return -2.0 * x * x + 1.5;
  if (x >= 0.5 && x < 1.5) return (x - 1.5) * (x - 1.5);
  return 0.0;
}

// ----------------------------------------------------------------------------- point quantisation
// The reference quantises `xyz / voxel_size` in fp32; torch evaluates a tensor
// divided by a Python float on CUDA as a product with the fp32 reciprocal.  The
// structure decisions below use exactly that value, with rounding-exact
// intrinsics so that nvcc cannot contract them into FMAs.
NGS_DEV float q32(float x, float inv_vs) { return __fmul_rn(x, inv_vs); }

// Trilinear corner cell and octant sign along one axis at `stride`
// (jspsr/core/_hash_backend.py:472-476): d = floor(q / s) * s, sign(q - d - s/2).
NGS_DEV void tri_axis(float q, int stride, float inv_stride, int* d_out, int* sgn_out) {
  const float d = __fmul_rn(floorf(__fmul_rn(q, inv_stride)), (float)stride);
  const float rel = __fsub_rn(__fsub_rn(q, d), 0.5f * (float)stride);
  *d_out = (int)d;
  *sgn_out = rel > 0.f ? 1 : (rel < 0.f ? -1 : 0);
}

// Neighbour quantisation of a point query (jspsr/core/_hash_backend.py:196-198 with
// source = xyz / vs - 0.5, source stride 1): floor((q - 0.5 + 0.5) / s) * s.
NGS_DEV int point_quant(float q, int stride, float inv_stride) {
  const float pos = __fsub_rn(q, 0.5f);
  return (int)__fmul_rn(floorf(__fmul_rn(__fadd_rn(pos, 0.5f), inv_stride)), (float)stride);
}

// ----------------------------------------------------------------------------- FNV key
NGS_DEV unsigned long long fnv_fold(unsigned long long h) {
  return (h >> 60) ^ (h & 0x0FFFFFFFFFFFFFFFull);
}
NGS_DEV unsigned long long fnv_step(unsigned long long h, unsigned int v) {
  return (h ^ (unsigned long long)v) * 1099511628211ull;
}
#define NGS_FNV_BASIS 14695981039346656037ull

// ----------------------------------------------------------------------------- reductions
template <typename T>
NGS_DEV T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

#define NGS_CHECK_LAUNCH()                                  \
  do {                                                      \
    cudaError_t _e = cudaGetLastError();                    \
    if (_e != cudaSuccess) return ngs_set_cuda_error(_e);   \
  } while (0)

int ngs_set_cuda_error(cudaError_t e);
// Host-side count of kernel launches issued by the library (every <<<>>> and cooperative launch).
void ngs_count_launch();

NGS_DEV int64_t ngs_gtid() { return (int64_t)blockIdx.x * blockDim.x + threadIdx.x; }
NGS_DEV int64_t ngs_gstride() { return (int64_t)gridDim.x * blockDim.x; }

// Streaming multiprocessors of the current device (queried once per device and cached).
int ngs_num_sms();

// Grid of a grid-stride kernel: enough blocks for n items, at most per_sm blocks per SM.
inline unsigned int ngs_blocks(int64_t n, int threads, int per_sm = 64) {
  int64_t b = (n + threads - 1) / threads;
  const int64_t cap = (int64_t)ngs_num_sms() * per_sm;
  if (b < 1) b = 1;
  if (b > cap) b = cap;
  return (unsigned int)b;
}
