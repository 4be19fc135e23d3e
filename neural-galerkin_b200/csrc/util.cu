// Status strings, CUDA error capture, device-wide scans and small reductions.
#include <atomic>
#include <cstdio>
#include <cstring>
#include "ngs_common.cuh"
#include "scan.cuh"

static thread_local char g_cuda_error[256] = "";

int ngs_set_cuda_error(cudaError_t e) {
  snprintf(g_cuda_error, sizeof(g_cuda_error), "%s: %s", cudaGetErrorName(e), cudaGetErrorString(e));
  return NGS_ERR_CUDA;
}

extern "C" const char* ngs_last_cuda_error(void) { return g_cuda_error; }

static std::atomic<long long> g_launches{0};
void ngs_count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
extern "C" int64_t ngs_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }
extern "C" void ngs_reset_launch_count(void) { g_launches.store(0, std::memory_order_relaxed); }

extern "C" int ngs_version(void) { return 10000; }

int ngs_num_sms() {
  static std::atomic<int> cached[64];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) dev = 0;
  if (dev >= 0 && dev < 64) {
    const int c = cached[dev].load(std::memory_order_relaxed);
    if (c > 0) return c;
  }
  int sms = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 1) {
    cudaGetLastError();
    sms = 1;
  }
  if (dev >= 0 && dev < 64) cached[dev].store(sms, std::memory_order_relaxed);
  return sms;
}

extern "C" const char* ngs_status_string(int status) {
  switch (status) {
    case NGS_OK: return "ok";
    case NGS_ERR_INVALID_ARG: return "invalid argument";
    case NGS_ERR_OOM: return "buffer or workspace too small";
    case NGS_ERR_HASH_INSERT: return "hash table insert failed (table full or probe bound exceeded)";
    case NGS_ERR_NOT_CONVERGED: return "iterative solve did not reach the tolerance within max_iter";
    case NGS_ERR_TOPOLOGY: return "dual grid corner accumulation overflow (topology error)";
    case NGS_ERR_CUDA: return "CUDA runtime error";
    case NGS_ERR_TIMEOUT: return "device-side wait timed out";
    default: return "unknown status";
  }
}

// ----------------------------------------------------------------------------- scans
struct LoadI64 {
  const int64_t* p;
  NGS_DEV int64_t operator()(int64_t i) const { return p[i]; }
};
struct LoadI32 {
  const int32_t* p;
  NGS_DEV int64_t operator()(int64_t i) const { return (int64_t)p[i]; }
};
struct StoreI64 {
  int64_t* p;
  NGS_DEV void operator()(int64_t i, int64_t v) const { p[i] = v; }
};

extern "C" size_t ngs_scan_workspace_bytes(int64_t n) { return ngs_scan_ws_bytes(n); }

extern "C" int ngs_exclusive_scan_i64(const int64_t* in, int64_t n, int64_t* out, int64_t* total_dev, void* ws,
                                      size_t ws_bytes, ngs_stream s) {
  if (n < 0 || (n > 0 && (!in || !out))) return NGS_ERR_INVALID_ARG;
  return ngs_scan(LoadI64{in}, StoreI64{out}, n, total_dev, ws, ws_bytes, (cudaStream_t)s);
}

extern "C" int ngs_exclusive_scan_i32(const int32_t* in, int64_t n, int64_t* out, int64_t* total_dev, void* ws,
                                      size_t ws_bytes, ngs_stream s) {
  if (n < 0 || (n > 0 && (!in || !out))) return NGS_ERR_INVALID_ARG;
  return ngs_scan(LoadI32{in}, StoreI64{out}, n, total_dev, ws, ws_bytes, (cudaStream_t)s);
}

// ----------------------------------------------------------------------------- bbox
NGS_DEV unsigned int f2ord(float f) {
  unsigned int u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

__global__ void bbox_init_kernel(unsigned int* b) {
  if (threadIdx.x < 3) b[threadIdx.x] = 0xffffffffu;
  else if (threadIdx.x < 6) b[threadIdx.x] = 0u;
}

__global__ void bbox_kernel(const float* __restrict__ xyz, int64_t n, unsigned int* b) {
  unsigned int mn[3] = {0xffffffffu, 0xffffffffu, 0xffffffffu}, mx[3] = {0u, 0u, 0u};
  for (int64_t i = ngs_gtid(); i < n; i += ngs_gstride()) {
#pragma unroll
    for (int a = 0; a < 3; a++) {
      const unsigned int o = f2ord(xyz[i * 3 + a]);
      mn[a] = min(mn[a], o);
      mx[a] = max(mx[a], o);
    }
  }
#pragma unroll
  for (int a = 0; a < 3; a++) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      mn[a] = min(mn[a], __shfl_xor_sync(0xffffffffu, mn[a], o));
      mx[a] = max(mx[a], __shfl_xor_sync(0xffffffffu, mx[a], o));
    }
  }
  if ((threadIdx.x & 31) == 0) {
    for (int a = 0; a < 3; a++) {
      atomicMin(b + a, mn[a]);
      atomicMax(b + 3 + a, mx[a]);
    }
  }
}

__global__ void bbox_decode_kernel(unsigned int* b) {
  if (threadIdx.x < 6) {
    const unsigned int o = b[threadIdx.x];
    const unsigned int u = (o & 0x80000000u) ? (o & 0x7fffffffu) : ~o;
    b[threadIdx.x] = u;   // reinterpreted as float by the caller
  }
}

extern "C" int ngs_points_bbox(const float* xyz, int64_t n, float* bbox_dev, ngs_stream s) {
  if (n <= 0 || !xyz || !bbox_dev) return NGS_ERR_INVALID_ARG;
  cudaStream_t st = (cudaStream_t)s;
  unsigned int* b = reinterpret_cast<unsigned int*>(bbox_dev);
  { ngs_count_launch(); bbox_init_kernel<<<1, 32, 0, st>>>(b); }
  { ngs_count_launch(); bbox_kernel<<<ngs_blocks(n, 256, 8), 256, 0, st>>>(xyz, n, b); }
  { ngs_count_launch(); bbox_decode_kernel<<<1, 32, 0, st>>>(b); }
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}

// ----------------------------------------------------------------------------- weighted sum
__global__ void weighted_sum_kernel(const float* __restrict__ v, const float* __restrict__ w, int64_t n,
                                    double* sums) {
  double a = 0.0, b = 0.0;
  for (int64_t i = ngs_gtid(); i < n; i += ngs_gstride()) {
    const double wi = w ? (double)w[i] : 1.0;
    a += wi * (double)v[i];
    b += wi;
  }
  a = warp_sum(a);
  b = warp_sum(b);
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(sums, a);
    atomicAdd(sums + 1, b);
  }
}

extern "C" int ngs_weighted_sum(const float* v, const float* w, int64_t n, double* sums_dev, ngs_stream s) {
  if (n < 0 || !v || !sums_dev) return NGS_ERR_INVALID_ARG;
  cudaStream_t st = (cudaStream_t)s;
  cudaMemsetAsync(sums_dev, 0, 2 * sizeof(double), st);
  if (n > 0) { ngs_count_launch(); weighted_sum_kernel<<<ngs_blocks(n, 256, 4), 256, 0, st>>>(v, w, n, sums_dev); }
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}
