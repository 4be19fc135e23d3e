// Sparse convolution over voxel neighbour maps (ref: csrc/sparse_op/convolution_cuda.cu:52-282 and
// its caller models/ascn/utils.py:108-190): out[o] = sum_k in[i_k(o)] @ W[k] over the (input, output)
// pairs of every kernel offset k.
//
// The reference runs, per offset, a gather kernel into a dense buffer, a cuBLAS GEMM and a scatter-add
// kernel (27 x 3 launches and two buffers through HBM per layer).  Here the map is first turned into
// an output-major table (row o, offset k) -> input row or -1, and ONE kernel computes a 128-row tile
// of the output: for every offset the tile's 128 input rows are gathered straight into shared memory
// in the tensor core's K-major 128-byte-swizzled layout, the offset's weights beside them, and
// tcgen05.mma accumulates all offsets into the same TMEM accumulator (FP32); the epilogue reads TMEM
// once and writes each output row once -- no scatter, no atomics, no intermediate buffers.  The input
// gradient is the same kernel over the transposed table with W[k]^T; the weight gradient is a GEMM
// over the pairs of one offset (split over CTAs, partials reduced in a fixed order).
//
// Warp roles in the tile kernel (288 threads): warps 0-7 gather tiles into a ring of shared-memory
// stages (two threads per tile row) and run the epilogue (warp w reads TMEM lanes 32(w%4).. = tile
// rows, column half w/4); warp 8 allocates TMEM and one of its lanes issues the MMAs.  Stages are
// handed over through mbarriers: "full" (256 producer arrivals after their stores and a proxy
// fence) and "empty" (tcgen05.commit of the MMAs that read the stage).  Every wait is bounded; on timeout the kernel records NGS_ERR_TIMEOUT,
// stops issuing, waits (bounded) for its MMAs and releases its TMEM before returning.
#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include "ngs_common.cuh"

namespace conv {

constexpr int BM = 128;              // tile rows (UMMA M)
constexpr int BK = 64;               // reduction elements per stage (128 bytes of 16-bit values)
constexpr int UK = 16;               // UMMA K of kind::f16
constexpr int PRODUCERS = 256;       // warps 0-7
constexpr int THREADS = PRODUCERS + 32;
constexpr int KMAX = 128;            // kernel offsets (5^3 = 125 at most)
constexpr unsigned long long WAIT_NS = 2000000000ull;   // bound of one mbarrier wait (2 s)

NGS_DEV uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

NGS_DEV unsigned long long now_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

NGS_DEV void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
NGS_DEV void mbar_arrive(uint64_t* bar) {
  asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(smem_u32(bar)) : "memory");
}
NGS_DEV bool mbar_try(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait for the phase of the given parity to complete; false when the bound ran out or another
// thread of the CTA already gave up (abort flag in shared memory).
NGS_DEV bool mbar_wait(uint64_t* bar, uint32_t parity, volatile int* abort) {
  if (mbar_try(bar, parity)) return true;
  const unsigned long long t0 = now_ns();
  while (!mbar_try(bar, parity)) {
    if (*abort) return false;
    if (now_ns() - t0 > WAIT_NS) {
      *abort = 1;
      return false;
    }
  }
  return true;
}

// Shared-memory matrix descriptor of a K-major tile with 128-byte swizzle: rows of 128 bytes, 8-row
// groups 1024 bytes apart (stride byte offset), leading byte offset 16 (unused by this layout but set
// as the canonical form has it), descriptor version 1, swizzle mode 2 (128 B).  The tile must start on
// a 1024-byte boundary; a K step inside the 128-byte row advances the start address.
NGS_DEV uint64_t kmajor_sw128_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

// Shared-memory matrix descriptor of an MN-major tile with 128-byte swizzle: each 128-byte row holds 64
// consecutive M (or N) elements at one K index, 8 K rows form a 1024-byte swizzle atom (stride byte
// offset 1024 between the atoms along K), and the 64-element atoms along M sit 8 KB apart (leading
// byte offset: 64 K rows per stage).  A K step of 16 advances the start address by two atoms.
constexpr uint32_t MN_ATOM_BYTES = 64 * 128;
NGS_DEV uint64_t mnmajor_sw128_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(MN_ATOM_BYTES >> 4) << 16) |
         ((uint64_t)(1024 >> 4) << 32) | ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

// Instruction descriptor of kind::f16 with FP32 accumulation, both operands K-major.
// bf16: 1 = BF16 inputs, 0 = FP16 inputs (A and B always share the type).
NGS_DEV uint32_t f16_idesc(int m, int n, int bf16) {
  const uint32_t fmt = bf16 ? 1u : 0u;
  return (1u << 4) | (fmt << 7) | (fmt << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}
// The same with both operands MN-major (bits 15 and 16).
NGS_DEV uint32_t f16_idesc_mn(int m, int n, int bf16) { return f16_idesc(m, n, bf16) | (1u << 15) | (1u << 16); }

NGS_DEV void umma_f16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(accumulate)
      : "memory");
}
// Arrives on the mbarrier once every MMA issued so far by this thread has completed.
NGS_DEV void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}
NGS_DEV void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
NGS_DEV void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// Generic-proxy stores to shared memory become visible to the tensor core (async proxy).
NGS_DEV void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// TMEM allocation by one whole warp; the column base lands in *dst (shared memory).
NGS_DEV void tmem_alloc(uint32_t* dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)), "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
NGS_DEV void tmem_free(uint32_t base, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base), "r"(ncols) : "memory");
}
// 16 consecutive FP32 columns of this thread's TMEM lane (warp w reads lanes 32w..32w+31).
NGS_DEV void tmem_ld16(uint32_t addr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(addr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int j = 0; j < 16; j++) v[j] = __uint_as_float(r[j]);
}

// Byte offset of 16-byte chunk c of row r in a K-major 128-byte-swizzled tile (1024-byte aligned).
NGS_DEV uint32_t sw128(int r, int c) { return (uint32_t)(r * 128 + ((c ^ (r & 7)) << 4)); }

}  // namespace conv

// ----------------------------------------------------------------------------- gather tables
// table[row, k] = the source row paired with `row` at offset k (-1: none).  Pairs of offset k are
// nbmaps[starts[k] .. starts[k+1]) as (c0, c1) int32 pairs; key_col picks the column that indexes the
// table rows, the other column is the source.  mid >= 0: table[row, mid] = row for every row (the
// reference's forward computes that offset as one dense product over all rows).
__global__ void conv_table_kernel(const int32_t* __restrict__ nbmaps, const int64_t* __restrict__ starts, int K,
                                  int key_col, int64_t n_rows, int mid, int32_t* __restrict__ table) {
  const int64_t total = starts[K];
  for (int64_t p = ngs_gtid(); p < total; p += ngs_gstride()) {
    int lo = 0, hi = K - 1;                    // offset of pair p: last k with starts[k] <= p
    while (lo < hi) {
      const int m = (lo + hi + 1) >> 1;
      if (starts[m] <= p) lo = m; else hi = m - 1;
    }
    if (lo == mid) continue;
    const int32_t key = nbmaps[2 * p + key_col], src = nbmaps[2 * p + 1 - key_col];
    if (key < 0 || key >= n_rows) continue;    // the reference's scatter skips negative targets
    table[(int64_t)key * K + lo] = src < 0 ? -1 : src;
  }
  if (mid >= 0)
    for (int64_t r = ngs_gtid(); r < n_rows; r += ngs_gstride()) table[r * K + mid] = (int32_t)r;
}

extern "C" int ngs_conv_table(const int32_t* nbmaps, const int64_t* starts_dev, int K, int key_col, int64_t n_rows,
                              int mid, int32_t* table, ngs_stream s) {
  if (K < 1 || K > 128 || (key_col != 0 && key_col != 1) || n_rows < 0 || mid >= K || !starts_dev ||
      (n_rows > 0 && !table))
    return NGS_ERR_INVALID_ARG;
  cudaStream_t st = (cudaStream_t)s;
  if (n_rows > 0 && cudaMemsetAsync(table, 0xFF, (size_t)n_rows * K * sizeof(int32_t), st) != cudaSuccess)
    return ngs_set_cuda_error(cudaGetLastError());
  ngs_count_launch();
  conv_table_kernel<<<ngs_blocks(n_rows > 0 ? n_rows * 4 : 1, 256, 16), 256, 0, st>>>(nbmaps, starts_dev, K, key_col,
                                                                                      n_rows, mid, table);
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}

// ----------------------------------------------------------------------------- the tile kernel
// One CTA computes a 128 x N tile (N <= 256, a multiple of 16) of D = sum over `steps` of A_s B_s^T,
// every A_s (128 x 64) and B_s (N x 64) filled by the producers straight into a shared-memory stage
// (K-major, 128-byte swizzle), accumulated in TMEM by tcgen05.mma, and handed to the epilogue.
// Fill: the source of the tiles -- fill(step, a, b, tid) stores the stage's A and B rows (zeros where
// there is no data) and returns the number of valid reduction elements of the step (<= 64).
// Store: store(row, col, v[16]) takes 16 consecutive accumulator columns of one tile row.
namespace conv {

struct TileShape {
  int steps;          // reduction steps of this tile (0: the tile is all zeros)
  int n;              // N of the MMA
  int stages;
  uint32_t stage_bytes;
};

constexpr uint32_t A_BYTES = BM * 128;   // 16 KB

template <typename Fill, typename Store>
NGS_DEV void run_tile(const TileShape& t, uint8_t* smem, Fill& fill, Store& store, int bf16, int* error,
                      bool mn_major = false) {
  __shared__ uint64_t full_bar[8], empty_bar[8], done_bar;
  __shared__ uint32_t tmem_slot;
  __shared__ int abort_flag;
  __shared__ int ksteps_of[8];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int S = t.stages;
  const uint32_t ncols_alloc = t.n <= 32 ? 32u : t.n <= 64 ? 64u : t.n <= 128 ? 128u : 256u;
  if (tid == 0) {
    for (int s = 0; s < S; s++) {
      mbar_init(&full_bar[s], PRODUCERS);
      mbar_init(&empty_bar[s], 1);
    }
    mbar_init(&done_bar, 1);
    abort_flag = 0;
  }
  if (warp == PRODUCERS / 32) tmem_alloc(&tmem_slot, ncols_alloc);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_slot;

  if (tid < PRODUCERS) {
    // producers: fill the ring of stages
    for (int s = 0; s < t.steps; s++) {
      const int st = s % S;
      if (s >= S && !mbar_wait(&empty_bar[st], (uint32_t)((s / S) - 1) & 1u, &abort_flag)) break;
      uint8_t* a = smem + (size_t)st * t.stage_bytes;
      const int valid = fill(s, a, a + A_BYTES, tid);
      if (tid == 0) ksteps_of[st] = (valid + UK - 1) / UK;
      fence_async_smem();
      mbar_arrive(&full_bar[st]);
    }
  } else if (lane == 0) {
    // one thread issues the MMAs of every stage, then commits the stage back to the producers
    const uint32_t idesc = mn_major ? f16_idesc_mn(BM, t.n, bf16) : f16_idesc(BM, t.n, bf16);
    for (int s = 0; s < t.steps; s++) {
      const int st = s % S;
      if (!mbar_wait(&full_bar[st], (uint32_t)(s / S) & 1u, &abort_flag)) break;
      tc_fence_after();
      const uint32_t a = smem_u32(smem + (size_t)st * t.stage_bytes), b = a + A_BYTES;
      const int ks = ksteps_of[st];
      for (int kk = 0; kk < ks; kk++)
        umma_f16(tmem,
                 mn_major ? mnmajor_sw128_desc(a + kk * 2048) : kmajor_sw128_desc(a + kk * 32),
                 mn_major ? mnmajor_sw128_desc(b + kk * 2048) : kmajor_sw128_desc(b + kk * 32), idesc,
                 (s > 0 || kk > 0) ? 1u : 0u);
      umma_commit(&empty_bar[st]);
    }
    umma_commit(&done_bar);        // arrives once everything issued above has completed
  }

  if (tid < PRODUCERS) {
    // epilogue: warp w reads TMEM lanes 32 (w % 4) .. (its tile rows), every other 16-column chunk
    bool ok = mbar_wait(&done_bar, 0u, &abort_flag);
    ok = __all_sync(0xffffffffu, ok) && !abort_flag;
    tc_fence_after();
    const int w = warp & 3, half = warp >> 2;
    const int row = 32 * w + lane;
    for (int cc = half; cc < t.n / 16; cc += 2) {
      float v[16];
      if (ok && t.steps > 0) {
        tmem_ld16(tmem + ((uint32_t)(32 * w) << 16) + (uint32_t)(cc * 16), v);
      } else {
#pragma unroll
        for (int j = 0; j < 16; j++) v[j] = 0.f;
      }
      if (ok) store(row, cc * 16, v);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == PRODUCERS / 32) {
    tc_fence_after();
    tmem_free(tmem, ncols_alloc);
  }
  if (tid == 0 && abort_flag) atomicExch(error, NGS_ERR_TIMEOUT);
}

NGS_DEV uint4 ldg16(const uint16_t* p) { return __ldg(reinterpret_cast<const uint4*>(p)); }

NGS_DEV void st16_row(void* out, bool f32, int bf16, int64_t off, const float (&v)[16]) {
  if (f32) {
    float4* o = reinterpret_cast<float4*>(static_cast<float*>(out) + off);
#pragma unroll
    for (int j = 0; j < 4; j++) o[j] = make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
  } else {
    uint32_t p[8];
#pragma unroll
    for (int j = 0; j < 8; j++) {
      if (bf16) {
        const __nv_bfloat162 h = __floats2bfloat162_rn(v[2 * j], v[2 * j + 1]);
        p[j] = *reinterpret_cast<const uint32_t*>(&h);
      } else {
        const __half2 h = __floats2half2_rn(v[2 * j], v[2 * j + 1]);
        p[j] = *reinterpret_cast<const uint32_t*>(&h);
      }
    }
    uint4* o = reinterpret_cast<uint4*>(static_cast<uint16_t*>(out) + off);
    o[0] = make_uint4(p[0], p[1], p[2], p[3]);
    o[1] = make_uint4(p[4], p[5], p[6], p[7]);
  }
}

}  // namespace conv

// ----------------------------------------------------------------------------- gather GEMM (forward, input grad)
// out[r, n] = sum over offsets k with table[r, k] = i >= 0 of sum_c x[i, c] * bt[k, n, c]
// (forward: x = input features, bt = W[k]^T; input gradient: x = output gradient, table transposed,
// bt = W[k] as stored).  Grid: (row tiles, column tiles of 256).
struct GatherGemm {
  const uint16_t* x;
  int64_t n_src;
  int kdim;
  const int32_t* table;
  int64_t n_rows;
  int K;
  const uint16_t* bt;
  int ncols;
  void* out;
  int out_f32;
  int bf16;
  int stages;
  uint32_t stage_bytes;
  int* error;
};

__global__ void __launch_bounds__(conv::THREADS, 1) conv_gather_gemm_kernel(const __grid_constant__ GatherGemm g) {
  using namespace conv;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
  __shared__ uint32_t act_mask[KMAX / 32];
  __shared__ int act_list[KMAX];
  __shared__ int n_act;
  const int tid = threadIdx.x;
  const int64_t r0 = (int64_t)blockIdx.x * BM;
  const int n0 = blockIdx.y * 256;
  const int N = min(256, g.ncols - n0);
  // the offsets with at least one pair in this tile (empty offsets cost nothing)
  if (tid < KMAX / 32) act_mask[tid] = 0u;
  __syncthreads();
  if (tid < BM && r0 + tid < g.n_rows)
    for (int k = 0; k < g.K; k++)
      if (__ldg(g.table + (r0 + tid) * g.K + k) >= 0) atomicOr(&act_mask[k >> 5], 1u << (k & 31));
  __syncthreads();
  if (tid == 0) {
    int c = 0;
    for (int k = 0; k < g.K; k++)
      if (act_mask[k >> 5] >> (k & 31) & 1u) act_list[c++] = k;
    n_act = c;
  }
  __syncthreads();
  const int nchunks = (g.kdim + BK - 1) / BK;
  TileShape t{n_act * nchunks, N, g.stages, g.stage_bytes};

  // two producers per tile row, four 16-byte chunks each; B rows spread over all producers
  auto fill = [&](int s, uint8_t* a, uint8_t* b, int p) -> int {
    const int k = act_list[s / nchunks];
    const int c0 = (s % nchunks) * BK;
    const int row = p >> 1, half = p & 1;
    int32_t src = -1;
    if (r0 + row < g.n_rows) src = __ldg(g.table + (r0 + row) * g.K + k);
    const bool have = src >= 0 && src < g.n_src;
    uint4 v[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int e = c0 + (half * 4 + j) * 8;
      v[j] = (have && e < g.kdim) ? ldg16(g.x + (int64_t)src * g.kdim + e) : make_uint4(0, 0, 0, 0);
    }
#pragma unroll
    for (int j = 0; j < 4; j++) *reinterpret_cast<uint4*>(a + sw128(row, half * 4 + j)) = v[j];
    for (int idx = p; idx < N * 8; idx += PRODUCERS) {
      const int n = idx >> 3, c = idx & 7, e = c0 + c * 8;
      const uint4 w = e < g.kdim ? ldg16(g.bt + ((int64_t)k * g.ncols + n0 + n) * g.kdim + e) : make_uint4(0, 0, 0, 0);
      *reinterpret_cast<uint4*>(b + sw128(n, c)) = w;
    }
    return min(BK, g.kdim - c0);
  };
  auto store = [&](int row, int col, const float (&v)[16]) {
    if (r0 + row < g.n_rows) st16_row(g.out, g.out_f32 != 0, g.bf16, (r0 + row) * g.ncols + n0 + col, v);
  };
  run_tile(t, smem, fill, store, g.bf16, g.error);
}

// ----------------------------------------------------------------------------- weight gradient
// part[k, split, m, n] = sum over the pairs p of offset k in the split's range of
// x[in(p), m0 + m] * gy[out(p), n0 + n]: A = the pairs' input rows transposed (rows m = input
// channels, reduction over pairs), B = their output-gradient rows transposed.  Grid: (splits,
// offsets, channel tiles).  The splits are summed in order by conv_wgrad_reduce_kernel.
struct WeightGrad {
  const uint16_t* x;         // [n_in, cin]
  const uint16_t* gy;        // [n_out, cout]
  int64_t n_in, n_out;
  int cin, cout;
  const int32_t* nbmaps;     // [P, 2]
  const int64_t* starts;     // [K + 1]
  int in_col;                // column of the input row in a pair (the other is the output row)
  int K;
  int splits;
  int m_tiles;               // ceil(cin / 128)
  float* part;               // [K, splits, cin, cout]
  int mn;                    // channels in multiples of 64: rows copied as they are into MN-major stages
  int bf16;
  int stages;
  uint32_t stage_bytes;
  int* error;
};

__global__ void __launch_bounds__(conv::THREADS, 1) conv_wgrad_kernel(const __grid_constant__ WeightGrad g) {
  using namespace conv;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
  const int split = blockIdx.x, k = blockIdx.y;
  const int m0 = (blockIdx.z % g.m_tiles) * BM, n0 = (blockIdx.z / g.m_tiles) * 256;
  const int N = min(256, g.cout - n0);
  const int64_t p_begin = __ldg(g.starts + k), p_count = __ldg(g.starts + k + 1) - p_begin;
  // this split's pairs, in whole chunks of 64
  const int64_t chunks = (p_count + BK - 1) / BK;
  const int64_t per = (chunks + g.splits - 1) / g.splits;
  const int64_t c_begin = min(chunks, (int64_t)split * per), c_end = min(chunks, c_begin + per);
  TileShape t{(int)(c_end - c_begin), N, g.stages, g.stage_bytes};

  // producer p: pair column kk = p % 64 of the stage, channel quarter q = p / 64 of the A rows (32
  // input channels) and of the B rows (N / 4 output channels); 16-bit values stored transposed
  auto fill = [&](int s, uint8_t* a, uint8_t* b, int p) -> int {
    const int64_t pc = (c_begin + s) * BK;              // first pair of the step (relative to p_begin)
    const int kk = p & 63, q = p >> 6;
    const int64_t pair = pc + kk;
    int32_t xi = -1, yo = -1;
    if (pair < p_count) {
      xi = __ldg(g.nbmaps + 2 * (p_begin + pair) + g.in_col);
      yo = __ldg(g.nbmaps + 2 * (p_begin + pair) + 1 - g.in_col);
    }
    const bool hx = xi >= 0 && xi < g.n_in, hy = yo >= 0 && yo < g.n_out;
    uint16_t* a16 = reinterpret_cast<uint16_t*>(a);
    uint16_t* b16 = reinterpret_cast<uint16_t*>(b);
    const int chunk = kk >> 3, within = kk & 7;
    for (int m = q * 32; m < q * 32 + 32; m++) {
      const int c = m0 + m;
      const uint16_t v = (hx && c < g.cin) ? __ldg(g.x + (int64_t)xi * g.cin + c) : (uint16_t)0;
      a16[(sw128(m, chunk) >> 1) + within] = v;
    }
    const int nq = N / 4;
    for (int n = q * nq; n < q * nq + nq; n++) {
      const int c = n0 + n;
      const uint16_t v = hy ? __ldg(g.gy + (int64_t)yo * g.cout + c) : (uint16_t)0;
      b16[(sw128(n, chunk) >> 1) + within] = v;
    }
    return (int)min((int64_t)BK, p_count - pc);
  };
  // MN-major form: the stage's K index is the pair, each 128-byte row 64 consecutive channels of one
  // pair, so a producer copies 16-byte pieces of its pair's rows as they are (no transposition)
  auto fill_mn = [&](int s, uint8_t* a, uint8_t* b, int p) -> int {
    const int64_t pc = (c_begin + s) * BK;
    const int kk = p & 63, q = p >> 6;
    const int64_t pair = pc + kk;
    int32_t xi = -1, yo = -1;
    if (pair < p_count) {
      xi = __ldg(g.nbmaps + 2 * (p_begin + pair) + g.in_col);
      yo = __ldg(g.nbmaps + 2 * (p_begin + pair) + 1 - g.in_col);
    }
    const bool hx = xi >= 0 && xi < g.n_in, hy = yo >= 0 && yo < g.n_out;
#pragma unroll
    for (int j = 0; j < 4; j++) {                    // A: 16 chunks of 8 channels, 4 per quarter
      const int c = q * 4 + j, ch = m0 + c * 8;
      const uint4 v = (hx && ch < g.cin) ? ldg16(g.x + (int64_t)xi * g.cin + ch) : make_uint4(0, 0, 0, 0);
      *reinterpret_cast<uint4*>(a + (c >> 3) * MN_ATOM_BYTES + sw128(kk, c & 7)) = v;
    }
    const int per = N / 32;                          // B: N / 8 chunks, a quarter each
    for (int j = 0; j < per; j++) {
      const int c = q * per + j, ch = n0 + c * 8;
      const uint4 v = hy ? ldg16(g.gy + (int64_t)yo * g.cout + ch) : make_uint4(0, 0, 0, 0);
      *reinterpret_cast<uint4*>(b + (c >> 3) * MN_ATOM_BYTES + sw128(kk, c & 7)) = v;
    }
    return (int)min((int64_t)BK, p_count - pc);
  };
  float* part = g.part + ((int64_t)k * g.splits + split) * g.cin * g.cout;
  auto store = [&](int row, int col, const float (&v)[16]) {
    if (m0 + row < g.cin) {
      float4* o = reinterpret_cast<float4*>(part + (int64_t)(m0 + row) * g.cout + n0 + col);
#pragma unroll
      for (int j = 0; j < 4; j++) o[j] = make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
    }
  };
  if (g.mn) run_tile(t, smem, fill_mn, store, g.bf16, g.error, true);
  else run_tile(t, smem, fill, store, g.bf16, g.error);
}

// grad_w[k, c, n] = sum over splits (in order) of part[k, split, c, n]; FP32 or 16-bit out.
__global__ void conv_wgrad_reduce_kernel(const float* __restrict__ part, int K, int splits, int64_t cc, void* out,
                                         int out_f32, int bf16) {
  const int64_t total = (int64_t)K * cc;
  for (int64_t e = ngs_gtid(); e < total; e += ngs_gstride()) {
    const int64_t k = e / cc, j = e % cc;
    float acc = 0.f;
    for (int s = 0; s < splits; s++) acc += part[(k * splits + s) * cc + j];
    if (out_f32) static_cast<float*>(out)[e] = acc;
    else if (bf16) static_cast<__nv_bfloat16*>(out)[e] = __float2bfloat16_rn(acc);
    else static_cast<__half*>(out)[e] = __float2half_rn(acc);
  }
}

// ----------------------------------------------------------------------------- CUDA-core path
// FP32 inputs (the reference's path outside autocast is an FP32 cuBLAS GEMM, so FP32 stays FP32 here)
// and 16-bit shapes the tensor-core tiles do not take (kdim not a multiple of 8, ncols not a multiple
// of 16): one thread per output element, FP32 accumulation.
template <typename T>
NGS_DEV float to_f(T v) { return (float)v; }
template <>
NGS_DEV float to_f<__half>(__half v) { return __half2float(v); }
template <>
NGS_DEV float to_f<__nv_bfloat16>(__nv_bfloat16 v) { return __bfloat162float(v); }

template <typename T>
NGS_DEV void put(void* out, int64_t i, float v, bool f32) {
  if (f32) static_cast<float*>(out)[i] = v;
  else if constexpr (sizeof(T) == 2) static_cast<T*>(out)[i] = (T)v;
  else static_cast<float*>(out)[i] = v;
}

template <typename T>
__global__ void conv_gather_gemm_simt_kernel(const T* __restrict__ x, int64_t n_src, int kdim,
                                             const int32_t* __restrict__ table, int64_t n_rows, int K,
                                             const T* __restrict__ bt, int ncols, void* out, int out_f32) {
  const int64_t total = n_rows * ncols;
  for (int64_t e = ngs_gtid(); e < total; e += ngs_gstride()) {
    const int64_t r = e / ncols;
    const int n = (int)(e % ncols);
    float acc = 0.f;
    for (int k = 0; k < K; k++) {
      const int32_t src = table[r * K + k];
      if (src < 0 || src >= n_src) continue;
      const T* xr = x + (int64_t)src * kdim;
      const T* br = bt + ((int64_t)k * ncols + n) * kdim;
      for (int c = 0; c < kdim; c++) acc += to_f(xr[c]) * to_f(br[c]);
    }
    put<T>(out, e, acc, out_f32 != 0);
  }
}

template <typename T>
__global__ void conv_wgrad_simt_kernel(const T* __restrict__ x, const T* __restrict__ gy, int64_t n_in, int64_t n_out,
                                       int cin, int cout, const int32_t* __restrict__ nbmaps,
                                       const int64_t* __restrict__ starts, int in_col, int K, void* out, int out_f32) {
  const int64_t total = (int64_t)K * cin * cout;
  for (int64_t e = ngs_gtid(); e < total; e += ngs_gstride()) {
    const int k = (int)(e / ((int64_t)cin * cout));
    const int ci = (int)((e / cout) % cin), co = (int)(e % cout);
    float acc = 0.f;
    for (int64_t p = starts[k]; p < starts[k + 1]; p++) {
      const int32_t i = nbmaps[2 * p + in_col], o = nbmaps[2 * p + 1 - in_col];
      if (i < 0 || i >= n_in || o < 0 || o >= n_out) continue;
      acc += to_f(x[(int64_t)i * cin + ci]) * to_f(gy[(int64_t)o * cout + co]);
    }
    put<T>(out, e, acc, out_f32 != 0);
  }
}

template <typename T>
__global__ void conv_transpose_kernel(const T* __restrict__ w, int K, int a, int b, T* __restrict__ wt) {
  const int64_t total = (int64_t)K * a * b;
  for (int64_t e = ngs_gtid(); e < total; e += ngs_gstride()) {
    const int64_t k = e / ((int64_t)a * b), i = (e / b) % a, j = e % b;
    wt[(k * b + j) * a + i] = w[e];
  }
}

// ----------------------------------------------------------------------------- host entry points
namespace {

bool aligned16(const void* p) { return ((uintptr_t)p & 15u) == 0; }

// Stages of the ring for an N-column tile, and the dynamic shared memory of the launch.
void tile_plan(int n, int& stages, uint32_t& stage_bytes, size_t& smem) {
  const uint32_t nb = (uint32_t)((n + 7) / 8 * 8) * 128u;
  stage_bytes = (conv::A_BYTES + nb + 1023u) & ~1023u;
  stages = (int)((200u * 1024u) / stage_bytes);
  if (stages > 4) stages = 4;
  if (stages < 2) stages = 2;
  smem = (size_t)stages * stage_bytes + 1024;        // + alignment of the first stage to 1024 bytes
}

template <typename T>
int simt_gemm(const void* x, int64_t n_src, int kdim, const int32_t* table, int64_t n_rows, int K, const void* bt,
              int ncols, void* out, int out_f32, cudaStream_t st) {
  ngs_count_launch();
  conv_gather_gemm_simt_kernel<T><<<ngs_blocks(n_rows * ncols, 256), 256, 0, st>>>(
      static_cast<const T*>(x), n_src, kdim, table, n_rows, K, static_cast<const T*>(bt), ncols, out, out_f32);
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}

}  // namespace

extern "C" int ngs_conv_transpose_weight(const void* w, int K, int a, int b, int dtype, void* wt, ngs_stream s) {
  if (!w || !wt || K < 1 || a < 1 || b < 1 || dtype < NGS_F16 || dtype > NGS_F32) return NGS_ERR_INVALID_ARG;
  cudaStream_t st = (cudaStream_t)s;
  const int64_t total = (int64_t)K * a * b;
  ngs_count_launch();
  if (dtype == NGS_F32)
    conv_transpose_kernel<float><<<ngs_blocks(total, 256), 256, 0, st>>>(static_cast<const float*>(w), K, a, b,
                                                                        static_cast<float*>(wt));
  else
    conv_transpose_kernel<uint16_t><<<ngs_blocks(total, 256), 256, 0, st>>>(static_cast<const uint16_t*>(w), K, a, b,
                                                                           static_cast<uint16_t*>(wt));
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}

extern "C" int ngs_conv_tensor_core_ok(int kdim, int ncols, int dtype) {
  return (dtype == NGS_F16 || dtype == NGS_BF16) && kdim >= 8 && kdim % 8 == 0 && ncols >= 16 && ncols % 16 == 0;
}

extern "C" int ngs_conv_gather_gemm(const void* x, int64_t n_src, int kdim, const int32_t* table, int64_t n_rows, int K,
                                    const void* bt, int ncols, int dtype, void* out, int out_f32, int* error_dev,
                                    ngs_stream s) {
  if (n_src < 0 || n_rows < 0 || kdim < 1 || ncols < 1 || K < 1 || K > conv::KMAX || dtype < NGS_F16 ||
      dtype > NGS_F32 || (n_rows > 0 && (!table || !out || !bt)) || (n_src > 0 && !x) || !error_dev)
    return NGS_ERR_INVALID_ARG;
  if (n_rows == 0) return NGS_OK;
  cudaStream_t st = (cudaStream_t)s;
  if (!ngs_conv_tensor_core_ok(kdim, ncols, dtype) || !aligned16(x) || !aligned16(bt) || !aligned16(out)) {
    if (dtype == NGS_F32) return simt_gemm<float>(x, n_src, kdim, table, n_rows, K, bt, ncols, out, 1, st);
    if (dtype == NGS_BF16) return simt_gemm<__nv_bfloat16>(x, n_src, kdim, table, n_rows, K, bt, ncols, out, out_f32, st);
    return simt_gemm<__half>(x, n_src, kdim, table, n_rows, K, bt, ncols, out, out_f32, st);
  }
  GatherGemm g{};
  g.x = static_cast<const uint16_t*>(x);
  g.n_src = n_src;
  g.kdim = kdim;
  g.table = table;
  g.n_rows = n_rows;
  g.K = K;
  g.bt = static_cast<const uint16_t*>(bt);
  g.ncols = ncols;
  g.out = out;
  g.out_f32 = out_f32;
  g.bf16 = dtype == NGS_BF16;
  g.error = error_dev;
  size_t smem = 0;
  tile_plan(ncols < 256 ? ncols : 256, g.stages, g.stage_bytes, smem);
  if (cudaFuncSetAttribute(conv_gather_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
      cudaSuccess)
    return ngs_set_cuda_error(cudaGetLastError());
  const dim3 grid((unsigned)((n_rows + conv::BM - 1) / conv::BM), (unsigned)((ncols + 255) / 256));
  ngs_count_launch();
  conv_gather_gemm_kernel<<<grid, conv::THREADS, smem, st>>>(g);
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}

extern "C" size_t ngs_conv_weight_grad_ws_bytes(int K, int cin, int cout, int64_t max_pairs) {
  int64_t splits = (max_pairs + 2047) / 2048;
  if (splits < 1) splits = 1;
  if (splits > 64) splits = 64;
  return (size_t)K * splits * cin * cout * sizeof(float);
}

extern "C" int ngs_conv_weight_grad(const void* x, int64_t n_in, int cin, const void* gy, int64_t n_out, int cout,
                                    const int32_t* nbmaps, const int64_t* starts_dev, int K, int64_t max_pairs,
                                    int in_col, int dtype, void* grad_w, int out_f32, void* ws, size_t ws_bytes,
                                    int* error_dev, ngs_stream s) {
  if (n_in < 0 || n_out < 0 || cin < 1 || cout < 1 || K < 1 || K > conv::KMAX || max_pairs < 0 ||
      (in_col != 0 && in_col != 1) || dtype < NGS_F16 || dtype > NGS_F32 || !starts_dev || !grad_w || !error_dev ||
      (max_pairs > 0 && !nbmaps) || (n_in > 0 && !x) || (n_out > 0 && !gy))
    return NGS_ERR_INVALID_ARG;
  cudaStream_t st = (cudaStream_t)s;
  const int64_t total = (int64_t)K * cin * cout;
  const bool tc = (dtype == NGS_F16 || dtype == NGS_BF16) && cout % 16 == 0 && aligned16(grad_w);
  if (!tc) {
    ngs_count_launch();
    if (dtype == NGS_F32)
      conv_wgrad_simt_kernel<float><<<ngs_blocks(total, 256), 256, 0, st>>>(
          static_cast<const float*>(x), static_cast<const float*>(gy), n_in, n_out, cin, cout, nbmaps, starts_dev,
          in_col, K, grad_w, 1);
    else if (dtype == NGS_BF16)
      conv_wgrad_simt_kernel<__nv_bfloat16><<<ngs_blocks(total, 256), 256, 0, st>>>(
          static_cast<const __nv_bfloat16*>(x), static_cast<const __nv_bfloat16*>(gy), n_in, n_out, cin, cout, nbmaps,
          starts_dev, in_col, K, grad_w, out_f32);
    else
      conv_wgrad_simt_kernel<__half><<<ngs_blocks(total, 256), 256, 0, st>>>(
          static_cast<const __half*>(x), static_cast<const __half*>(gy), n_in, n_out, cin, cout, nbmaps, starts_dev,
          in_col, K, grad_w, out_f32);
    NGS_CHECK_LAUNCH();
    return NGS_OK;
  }
  const size_t need = ngs_conv_weight_grad_ws_bytes(K, cin, cout, max_pairs);
  if (!ws || ws_bytes < need) return NGS_ERR_OOM;
  WeightGrad g{};
  g.x = static_cast<const uint16_t*>(x);
  g.gy = static_cast<const uint16_t*>(gy);
  g.n_in = n_in;
  g.n_out = n_out;
  g.cin = cin;
  g.cout = cout;
  g.nbmaps = nbmaps;
  g.starts = starts_dev;
  g.in_col = in_col;
  g.K = K;
  g.splits = (int)(need / ((size_t)K * cin * cout * sizeof(float)));
  g.m_tiles = (cin + conv::BM - 1) / conv::BM;
  g.part = static_cast<float*>(ws);
  g.mn = cin % 64 == 0 && cout % 64 == 0 && aligned16(x) && aligned16(gy);
  g.bf16 = dtype == NGS_BF16;
  g.error = error_dev;
  size_t smem = 0;
  tile_plan(cout < 256 ? cout : 256, g.stages, g.stage_bytes, smem);
  if (cudaFuncSetAttribute(conv_wgrad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return ngs_set_cuda_error(cudaGetLastError());
  const dim3 grid((unsigned)g.splits, (unsigned)K, (unsigned)(g.m_tiles * ((cout + 255) / 256)));
  ngs_count_launch();
  conv_wgrad_kernel<<<grid, conv::THREADS, smem, st>>>(g);
  NGS_CHECK_LAUNCH();
  ngs_count_launch();
  conv_wgrad_reduce_kernel<<<ngs_blocks(total, 256), 256, 0, st>>>(g.part, K, g.splits, (int64_t)cin * cout, grad_w,
                                                                  out_f32, g.bf16);
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}
