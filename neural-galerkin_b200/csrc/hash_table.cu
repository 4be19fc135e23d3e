// Coordinate keys and the general key -> value table behind jspsr.ext.CuckooHashTable.
//
// Keys are the reference's FNV-1a-64 folded to 60 bits (hashmap_cuda.cu:247-261)
// so every key a caller computes is bit-identical.  The table itself is new:
// open addressing with linear probing over 16-byte {key, value} slots; a query
// is served by an 8-lane group that loads one 128-byte bucket per step with
// coalesced 128-bit loads and decides hit / miss with two ballots.
#include "hash_table.cuh"

template <typename T, int D>
__global__ void hash_rows_kernel(const T* __restrict__ c, int64_t n, int64_t* __restrict__ out) {
  for (int64_t i = ngs_gtid(); i < n; i += ngs_gstride()) {
    unsigned long long h = NGS_FNV_BASIS;
#pragma unroll
    for (int j = 0; j < D; j++) h = fnv_step(h, (unsigned int)c[i * D + j]);
    out[i] = (int64_t)fnv_fold(h);
  }
}

template <typename T, int D>
__global__ void kernel_hash_kernel(const T* __restrict__ c, int64_t n, const int32_t* __restrict__ off, int64_t k,
                                   int64_t* __restrict__ out) {
  const int64_t total = n * k;
  for (int64_t t = ngs_gtid(); t < total; t += ngs_gstride()) {
    const int64_t kk = t / n, i = t - kk * n;
    unsigned long long h = NGS_FNV_BASIS;
#pragma unroll
    for (int j = 0; j < 3; j++) h = fnv_step(h, (unsigned int)(c[i * D + j] + (T)off[kk * 3 + j]));
    if (D == 4) h = fnv_step(h, (unsigned int)c[i * D + 3]);
    out[t] = (int64_t)fnv_fold(h);
  }
}

extern "C" int ngs_hash_coords(const void* coords, int coords_int64, int64_t n, int dim, int64_t* out, ngs_stream s) {
  if (n < 0 || dim < 2 || dim > 4 || (n > 0 && (!coords || !out))) return NGS_ERR_INVALID_ARG;
  if (n == 0) return NGS_OK;
  cudaStream_t st = (cudaStream_t)s;
  const unsigned b = ngs_blocks(n, 256);
  const int key = (coords_int64 ? 10 : 0) + dim;
  switch (key) {
    case 2: { ngs_count_launch(); hash_rows_kernel<int32_t, 2><<<b, 256, 0, st>>>((const int32_t*)coords, n, out); } break;
    case 3: { ngs_count_launch(); hash_rows_kernel<int32_t, 3><<<b, 256, 0, st>>>((const int32_t*)coords, n, out); } break;
    case 4: { ngs_count_launch(); hash_rows_kernel<int32_t, 4><<<b, 256, 0, st>>>((const int32_t*)coords, n, out); } break;
    case 12: { ngs_count_launch(); hash_rows_kernel<int64_t, 2><<<b, 256, 0, st>>>((const int64_t*)coords, n, out); } break;
    case 13: { ngs_count_launch(); hash_rows_kernel<int64_t, 3><<<b, 256, 0, st>>>((const int64_t*)coords, n, out); } break;
    default: { ngs_count_launch(); hash_rows_kernel<int64_t, 4><<<b, 256, 0, st>>>((const int64_t*)coords, n, out); } break;
  }
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}

extern "C" int ngs_kernel_hash(const void* coords, int coords_int64, int64_t n, int dim, const int32_t* offsets,
                               int64_t k, int64_t* out, ngs_stream s) {
  if (n < 0 || k < 0 || (dim != 3 && dim != 4)) return NGS_ERR_INVALID_ARG;
  if (n == 0 || k == 0) return NGS_OK;
  if (!coords || !offsets || !out) return NGS_ERR_INVALID_ARG;
  cudaStream_t st = (cudaStream_t)s;
  const unsigned b = ngs_blocks(n * k, 256);
  if (coords_int64) {
    if (dim == 3) { ngs_count_launch(); kernel_hash_kernel<int64_t, 3><<<b, 256, 0, st>>>((const int64_t*)coords, n, offsets, k, out); }
    else { ngs_count_launch(); kernel_hash_kernel<int64_t, 4><<<b, 256, 0, st>>>((const int64_t*)coords, n, offsets, k, out); }
  } else {
    if (dim == 3) { ngs_count_launch(); kernel_hash_kernel<int32_t, 3><<<b, 256, 0, st>>>((const int32_t*)coords, n, offsets, k, out); }
    else { ngs_count_launch(); kernel_hash_kernel<int32_t, 4><<<b, 256, 0, st>>>((const int32_t*)coords, n, offsets, k, out); }
  }
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}

// ----------------------------------------------------------------------------- table
extern "C" int64_t ngs_hash_table_slots(int64_t n, int enlarge) {
  int64_t want = (enlarge ? 4 : 2) * (n > 0 ? n : 1);
  int64_t s = 8;
  while (s < want) s <<= 1;
  return s;
}

__global__ void table_init_kernel(Slot* slots, int64_t n) {
  for (int64_t i = ngs_gtid(); i < n; i += ngs_gstride()) {
    slots[i].key = kEmpty;
    slots[i].val = 0x7FFFFFFFFFFFFFFFll;
  }
}

__global__ void table_insert_kernel(Slot* __restrict__ slots, int64_t mask, const int64_t* __restrict__ keys,
                                    const int64_t* __restrict__ vals, int64_t n, int* status) {
  for (int64_t i = ngs_gtid(); i < n; i += ngs_gstride()) {
    const unsigned long long key = (unsigned long long)keys[i];
    const long long val = vals ? (long long)vals[i] : (long long)i;
    int64_t slot = (int64_t)(mix64(key) & (unsigned long long)mask);
    bool done = false;
    for (int64_t probe = 0; probe <= mask; probe++) {
      const unsigned long long prev = atomicCAS(&slots[slot].key, kEmpty, key);
      if (prev == kEmpty || prev == key) {
        atomicMin(&slots[slot].val, val);
        done = true;
        break;
      }
      slot = (slot + 1) & mask;
    }
    if (!done && status) atomicExch(status, NGS_ERR_HASH_INSERT);
  }
}

// 8 lanes per query: one 128-byte bucket per step.
NGS_DEV long long table_find(const Slot* __restrict__ slots, int64_t mask, unsigned long long key, int lane8,
                             unsigned group_mask) {
  const int64_t h = (int64_t)(mix64(key) & (unsigned long long)mask);
  int64_t bucket = h & ~7ll;
  int first = (int)(h & 7);
  const int64_t nb = (mask + 1) >> 3;
  for (int64_t step = 0; step <= nb; step++) {
    const uint4 v = __ldg(reinterpret_cast<const uint4*>(slots + bucket + lane8));
    const unsigned long long k = (unsigned long long)v.x | ((unsigned long long)v.y << 32);
    const long long val = (long long)((unsigned long long)v.z | ((unsigned long long)v.w << 32));
    const unsigned hit = __ballot_sync(group_mask, k == key);
    const unsigned empty = __ballot_sync(group_mask, k == kEmpty && lane8 >= first);
    if (hit) {
      const int src = __ffs(hit) - 1;
      return __shfl_sync(group_mask, val, src);
    }
    if (empty) return -1;
    bucket = (bucket + 8) & mask;
    first = 0;
  }
  return -1;
}

__global__ void table_query_kernel(const Slot* __restrict__ slots, int64_t mask, const int64_t* __restrict__ q,
                                   int64_t m, int64_t* __restrict__ out) {
  const int lane = threadIdx.x & 31, lane8 = lane & 7;
  const unsigned group_mask = 0xFFu << (lane & 24);
  const int64_t groups = (int64_t)gridDim.x * (blockDim.x >> 3);
  // All lanes of a warp iterate together; groups past the end skip the work.
  for (int64_t base = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 3;; base += groups) {
    const bool active = base < m;
    if (!__ballot_sync(0xffffffffu, active)) break;
    if (active) {
      const long long r = table_find(slots, mask, (unsigned long long)q[base], lane8, group_mask);
      if (lane8 == 0) out[base] = r + 1;
    }
  }
}

__global__ void table_query_coords_kernel(const Slot* __restrict__ slots, int64_t mask, const int32_t* __restrict__ c,
                                          int64_t m, int64_t* __restrict__ out) {
  const int lane = threadIdx.x & 31, lane8 = lane & 7;
  const unsigned group_mask = 0xFFu << (lane & 24);
  const int64_t groups = (int64_t)gridDim.x * (blockDim.x >> 3);
  for (int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 3;; i += groups) {
    const bool active = i < m;
    if (!__ballot_sync(0xffffffffu, active)) break;
    if (active) {
      unsigned long long h = NGS_FNV_BASIS;
      h = fnv_step(h, (unsigned)c[i * 3]);
      h = fnv_step(h, (unsigned)c[i * 3 + 1]);
      h = fnv_step(h, (unsigned)c[i * 3 + 2]);
      const long long r = table_find(slots, mask, fnv_fold(h), lane8, group_mask);
      if (lane8 == 0) out[i] = r;
    }
  }
}

extern "C" int ngs_hash_table_build(ngs_hash_table* t, const int64_t* keys, const int64_t* vals, int64_t n,
                                    int* status_dev, ngs_stream s) {
  if (!t || !t->slots || t->nslots < 8 || (t->nslots & (t->nslots - 1)) || n < 0 || (n > 0 && !keys))
    return NGS_ERR_INVALID_ARG;
  if (n > t->nslots) return NGS_ERR_OOM;
  if ((reinterpret_cast<uintptr_t>(t->slots) & 15u) != 0) return NGS_ERR_INVALID_ARG;
  cudaStream_t st = (cudaStream_t)s;
  Slot* slots = static_cast<Slot*>(t->slots);
  { ngs_count_launch(); table_init_kernel<<<ngs_blocks(t->nslots, 256), 256, 0, st>>>(slots, t->nslots); }
  if (n > 0) { ngs_count_launch(); table_insert_kernel<<<ngs_blocks(n, 256), 256, 0, st>>>(slots, t->nslots - 1, keys, vals, n, status_dev); }
  t->inserted = n;
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}

extern "C" int ngs_hash_table_query(const ngs_hash_table* t, const int64_t* keys, int64_t m, int64_t* out,
                                    ngs_stream s) {
  if (!t || !t->slots || m < 0 || (m > 0 && (!keys || !out))) return NGS_ERR_INVALID_ARG;
  if (m == 0) return NGS_OK;
  { ngs_count_launch(); table_query_kernel<<<ngs_blocks(m * 8, 256), 256, 0, (cudaStream_t)s>>>(
      static_cast<const Slot*>(t->slots), t->nslots - 1, keys, m, out); }
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}

extern "C" int ngs_hash_table_query_coords(const ngs_hash_table* t, const int32_t* coords, int64_t m, int64_t* out,
                                           ngs_stream s) {
  if (!t || !t->slots || m < 0 || (m > 0 && (!coords || !out))) return NGS_ERR_INVALID_ARG;
  if (m == 0) return NGS_OK;
  { ngs_count_launch(); table_query_coords_kernel<<<ngs_blocks(m * 8, 256), 256, 0, (cudaStream_t)s>>>(
      static_cast<const Slot*>(t->slots), t->nslots - 1, coords, m, out); }
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}

