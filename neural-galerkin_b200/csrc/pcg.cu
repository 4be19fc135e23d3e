// Persistent Jacobi-PCG for the per-level Galerkin systems
// (replaces csrc/sparse_solve/solve_pcg.cu:15-136 and jspsr/core/solver.py:189-202).
//
// The reference drives cuSPARSE SpMV + cuBLAS level-1 from the host with three
// device->host reads per iteration.  Here one cooperative kernel runs the whole
// solve: the Chronopoulos-Gear form of PCG needs a single reduction per
// iteration, so an iteration is
//     phase A  (own rows)  p = u + b p;  s = w + b s;  x += a p;  r -= a s;  u = M r
//     barrier              u visible to every block
//     phase B  (own rows)  w = A u, partial dots (r,u), (w,u), (r,r)
//     barrier + reduce     the last block to arrive sums the per-block partials in
//                          block order (deterministic) and releases the others.
// Every wait is bounded by the global nanosecond timer; on timeout the kernel
// records NGS_ERR_TIMEOUT and returns.  Every solve is bounded too: at most
// NGS_PCG_ITER_CAP iterations, and a deadline that the last block of each
// reduction checks, so that all blocks stop at the same iteration.  Dots are
// FP64 in every mode.
//
// Mixed precision (NGS_PCG_MIXED) is iterative refinement: the inner PCG runs on
// the FP32 matrix values with FP64 vectors and FP64 accumulation, until its
// residual has dropped by `inner_rtol`; then the true residual b - A x is formed
// with the FP64 matrix and the inner solve restarts from it.  The FP32 matrix is
// a fixed SPD perturbation of the FP64 one, so each outer step contracts the
// error by about |A32 - A64| |A64^-1| and the solve converges to the FP64 system.
#include <cmath>
#include "ngs_common.cuh"

constexpr int PCG_THREADS = 256;
constexpr int PCG_ROW_LANES = 16;   // lanes per row in the SpMV

struct PcgArgs {
  int64_t n;
  const int64_t* rowptr;
  const int32_t* cols;
  const void* vals;          // recurrence matrix (float or double)
  const double* vals64;      // replacement matrix (MIXED)
  const void* b;             // float (REFERENCE) or double
  const float* inv_diag;
  void* x;                   // float (REFERENCE) or double
  float* x32_out;            // optional FP32 copy of x
  void* r;                   // residual, RT
  void* p;
  void* s;
  void* u;
  void* w;
  double* partials;          // [nblocks][4]
  double* result;            // [4]
  unsigned int* count;
  unsigned int* gen;
  int* error;
  int64_t* info;             // {iters, status, replacements, -}
  double* resid;             // {|r|, |b|}
  double tol;
  int max_iter;
  int replace_every;         // <= 0: never
  double inner_rtol;          // MIXED: relative reduction of an inner solve
  unsigned long long wait_ns;     // bound of one barrier wait
  unsigned long long* deadline;   // absolute global-timer deadline, set at the first reduction
  unsigned long long budget_ns;   // time budget of the whole solve
  unsigned int nblocks;
};

constexpr int NGS_PCG_ITER_CAP = 20000;

NGS_DEV unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

template <typename T>
NGS_DEV T ld_cg(const T* p) { return *reinterpret_cast<const volatile T*>(p); }

// Block sums of NV doubles -> per-block partials -> fixed-order grid reduction.
template <int NV>
NGS_DEV bool reduce_barrier(const PcgArgs& a, const double (&v)[NV], double (&out)[NV]) {
  __shared__ double red[NV > 0 ? NV : 1][PCG_THREADS / 32];
  __shared__ int last, ok;
  __shared__ unsigned int gen0;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < NV; k++) {
    const double t = warp_sum(v[k]);
    if (lane == 0) red[k][wid] = t;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    ok = 1;
#pragma unroll
    for (int k = 0; k < NV; k++) {
      double t = 0.0;
      for (int i = 0; i < PCG_THREADS / 32; i++) t += red[k][i];
      a.partials[(size_t)blockIdx.x * 4 + k] = t;
    }
    gen0 = *reinterpret_cast<volatile unsigned int*>(a.gen);
    __threadfence();
    const unsigned int arrived = atomicAdd(a.count, 1u);
    last = (arrived == a.nblocks - 1);
  }
  __syncthreads();
  if (last) {
    __threadfence();
#pragma unroll
    for (int k = 0; k < NV; k++) {
      double t = 0.0;
      for (unsigned int i = threadIdx.x; i < a.nblocks; i += PCG_THREADS) t += ld_cg(a.partials + (size_t)i * 4 + k);
      t = warp_sum(t);
      if (lane == 0) red[k][wid] = t;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
      for (int k = 0; k < NV; k++) {
        double t = 0.0;
        for (int i = 0; i < PCG_THREADS / 32; i++) t += red[k][i];
        a.result[k] = t;
      }
      const unsigned long long now = global_ns();
      if (*a.deadline == 0ull) *a.deadline = now + a.budget_ns;
      a.result[3] = now > *a.deadline ? 1.0 : 0.0;   // one decision for every block
      *a.count = 0;
      __threadfence();
      atomicExch(a.gen, gen0 + 1u);
    }
  } else if (threadIdx.x == 0) {
    const unsigned long long t0 = global_ns();
    while (*reinterpret_cast<volatile unsigned int*>(a.gen) == gen0) {
      if (*reinterpret_cast<volatile int*>(a.error)) { ok = 0; break; }
      if (global_ns() - t0 > a.wait_ns) {
        atomicExch(a.error, NGS_ERR_TIMEOUT);
        ok = 0;
        break;
      }
      __nanosleep(32);
    }
    __threadfence();
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < NV; k++) out[k] = ld_cg(a.result + k);
  return ok != 0;
}

NGS_DEV bool past_deadline(const PcgArgs& a) { return ld_cg(a.result + 3) != 0.0; }

NGS_DEV bool plain_barrier(const PcgArgs& a) {
  double v[1] = {0.0}, o[1];
  return reduce_barrier<1>(a, v, o);
}

// Row-parallel SpMV, PCG_ROW_LANES lanes per row; the group leader hands the row's
// product to `epi(row, acc)`, which writes whatever the row owns and returns a
// contribution to the block's partial sum.  Outputs of an SpMV are only ever
// consumed by its own epilogue or after a grid barrier.
template <typename MT, typename VT, typename ACC, typename Epi>
NGS_DEV double spmv_rows(const PcgArgs& a, const MT* __restrict__ vals, const VT* __restrict__ v, Epi epi) {
  const int sub = threadIdx.x & (PCG_ROW_LANES - 1);
  const unsigned gmask = ((1u << PCG_ROW_LANES) - 1u) << ((threadIdx.x & 31) & ~(PCG_ROW_LANES - 1));
  const int64_t groups = (int64_t)gridDim.x * (PCG_THREADS / PCG_ROW_LANES);
  double dsum = 0.0;
  for (int64_t row = ((int64_t)blockIdx.x * PCG_THREADS + threadIdx.x) / PCG_ROW_LANES;; row += groups) {
    if (!__any_sync(0xffffffffu, row < a.n)) break;
    if (row < a.n) {
      const int64_t beg = a.rowptr[row], end = a.rowptr[row + 1];
      ACC acc = (ACC)0;
      for (int64_t j = beg + sub; j < end; j += PCG_ROW_LANES)
        acc += (ACC)__ldg(vals + j) * (ACC)v[__ldg(a.cols + j)];
#pragma unroll
      for (int o = PCG_ROW_LANES / 2; o > 0; o >>= 1) acc += __shfl_xor_sync(gmask, acc, o);
      if (sub == 0) dsum += epi(row, (double)acc);
    }
  }
  return dsum;
}

template <int MODE>
struct PcgTypes;
template <> struct PcgTypes<NGS_PCG_REFERENCE> { using MT = float; using VT = float; using RT = float; };
template <> struct PcgTypes<NGS_PCG_MIXED> { using MT = float; using VT = double; using RT = double; };
template <> struct PcgTypes<NGS_PCG_FP64> { using MT = double; using VT = double; using RT = double; };

// Recurrence SpMV of a mode: REFERENCE is all FP32 (as cuSPARSE SpMV in the reference);
// MIXED reads FP32 matrix values and accumulates in FP64; FP64 is all FP64.
template <int MODE, typename VT, typename Epi>
NGS_DEV double spmv_mode(const PcgArgs& a, const VT* v, Epi epi) {
  if constexpr (MODE == NGS_PCG_FP64) return spmv_rows<double, VT, double>(a, static_cast<const double*>(a.vals), v, epi);
  else if constexpr (MODE == NGS_PCG_MIXED) return spmv_rows<float, VT, double>(a, static_cast<const float*>(a.vals), v, epi);
  else return spmv_rows<float, VT, float>(a, static_cast<const float*>(a.vals), v, epi);
}

template <int MODE>
__global__ void __launch_bounds__(PCG_THREADS) pcg_kernel(PcgArgs a) {
  using VT = typename PcgTypes<MODE>::VT;
  using RT = typename PcgTypes<MODE>::RT;
  const RT* b = static_cast<const RT*>(a.b);
  RT* x = static_cast<RT*>(a.x);
  RT* r = static_cast<RT*>(a.r);
  VT* p = static_cast<VT*>(a.p);
  VT* s = static_cast<VT*>(a.s);
  VT* u = static_cast<VT*>(a.u);
  VT* w = static_cast<VT*>(a.w);
  const int64_t n = a.n;
  const int64_t t0 = ngs_gtid(), ts = ngs_gstride();
  const int sqrt_n = (int)ceil(sqrt((double)n));

  // w = A u; returns (w, u)
  auto w_epi = [&](int64_t row, double acc) -> double {
    w[row] = (VT)acc;
    return acc * (double)u[row];
  };
  // r = b - A x, u = M r; returns (r, r)
  auto true_res_epi = [&](int64_t row, double acc) -> double {
    const RT ri = (RT)((double)b[row] - acc);
    r[row] = ri;
    u[row] = (VT)((double)a.inv_diag[row] * (double)ri);
    return (double)ri * (double)ri;
  };

  // init: x = 0, r = b, u = M r, p = s = 0; partial (b, b)
  double part[3] = {0.0, 0.0, 0.0}, res[3];
  for (int64_t i = t0; i < n; i += ts) {
    const RT bi = b[i];
    x[i] = (RT)0;
    r[i] = bi;
    u[i] = (VT)((double)a.inv_diag[i] * (double)bi);
    p[i] = (VT)0;
    s[i] = (VT)0;
    part[0] += (double)bi * (double)bi;
  }
  if (!reduce_barrier<3>(a, part, res)) return;
  const double bnorm = sqrt(res[0]);
  const double atol = a.tol * bnorm;
  part[0] = part[1] = part[2] = 0.0;
  part[1] = spmv_mode<MODE>(a, u, w_epi);
  for (int64_t i = t0; i < n; i += ts) {
    part[0] += (double)r[i] * (double)u[i];
    part[2] += (double)r[i] * (double)r[i];
  }
  if (!reduce_barrier<3>(a, part, res)) return;
  double gamma = res[0], delta = res[1], rho = res[2];
  double alpha = delta != 0.0 ? gamma / delta : 0.0, beta = 0.0;
  int it = 0, replacements = 0;
  const double rtol_inner = MODE == NGS_PCG_MIXED ? a.inner_rtol : 0.0;
  double target = fmax(atol, rtol_inner * sqrt(rho));
  bool converged = sqrt(rho) <= atol || bnorm == 0.0, timed_out = false;
  const int cap = (a.max_iter >= 0 && a.max_iter < NGS_PCG_ITER_CAP) ? a.max_iter : NGS_PCG_ITER_CAP;
  while (!converged && it < cap) {
    if (past_deadline(a)) { timed_out = true; break; }
    const bool replace =
        (MODE == NGS_PCG_MIXED && a.replace_every > 0 && (it + 1) % a.replace_every == 0) ||
        (MODE == NGS_PCG_REFERENCE && a.replace_every > 0 && (it + 1) % sqrt_n == 0);
    // phase A (own rows)
    for (int64_t i = t0; i < n; i += ts) {
      const VT pi = (VT)((double)u[i] + beta * (double)p[i]);
      const VT si = (VT)((double)w[i] + beta * (double)s[i]);
      p[i] = pi;
      s[i] = si;
      x[i] = (RT)((double)x[i] + alpha * (double)pi);
      if (!replace) {
        const RT ri = (RT)((double)r[i] - alpha * (double)si);
        r[i] = ri;
        u[i] = (VT)((double)a.inv_diag[i] * (double)ri);
      }
    }
    if (replace) {
      // residual replacement: r = b - A x (FP64 matrix in MIXED mode, the FP32 one in REFERENCE mode)
      if (!plain_barrier(a)) return;
      if constexpr (MODE == NGS_PCG_MIXED) spmv_rows<double, RT, double>(a, a.vals64, x, true_res_epi);
      else spmv_rows<float, RT, float>(a, static_cast<const float*>(a.vals), x, true_res_epi);
      replacements++;
    }
    if (!plain_barrier(a)) return;
    // phase B
    part[0] = part[1] = part[2] = 0.0;
    part[1] = spmv_mode<MODE>(a, u, w_epi);
    for (int64_t i = t0; i < n; i += ts) {
      part[0] += (double)r[i] * (double)u[i];
      part[2] += (double)r[i] * (double)r[i];
    }
    if (!reduce_barrier<3>(a, part, res)) return;
    it++;
    const double gamma_new = res[0];
    delta = res[1];
    rho = res[2];
    if (sqrt(rho) <= target) {
      if (MODE != NGS_PCG_MIXED) { converged = true; break; }
      // end of an inner solve: true FP64 residual, stop or restart the recurrences from it
      if (!plain_barrier(a)) return;
      part[0] = part[1] = part[2] = 0.0;
      part[2] = spmv_rows<double, RT, double>(a, a.vals64, x, true_res_epi);
      replacements++;
      if (!plain_barrier(a)) return;
      part[1] = spmv_mode<MODE>(a, u, w_epi);
      for (int64_t i = t0; i < n; i += ts) part[0] += (double)r[i] * (double)u[i];
      if (!reduce_barrier<3>(a, part, res)) return;
      rho = res[2];
      if (sqrt(rho) <= atol) { converged = true; break; }
      gamma = res[0];
      delta = res[1];
      alpha = delta != 0.0 ? gamma / delta : 0.0;
      beta = 0.0;
      target = fmax(atol, rtol_inner * sqrt(rho));
      continue;
    }
    beta = gamma != 0.0 ? gamma_new / gamma : 0.0;
    const double den = delta - beta * gamma_new / alpha;
    alpha = den != 0.0 ? gamma_new / den : 0.0;
    gamma = gamma_new;
  }
  if (a.x32_out)
    for (int64_t i = t0; i < n; i += ts) a.x32_out[i] = (float)x[i];
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    a.info[0] = it;
    a.info[1] = converged ? NGS_OK : (timed_out ? NGS_ERR_TIMEOUT : NGS_ERR_NOT_CONVERGED);
    a.info[2] = replacements;
    a.resid[0] = sqrt(rho);
    a.resid[1] = bnorm;
  }
}

static size_t align_up(size_t v) { return (v + 255) & ~(size_t)255; }

extern "C" size_t ngs_pcg_workspace_bytes(int64_t n, int mode) {
  const size_t vt = mode == NGS_PCG_REFERENCE ? 4 : 8;
  const size_t rt = mode == NGS_PCG_REFERENCE ? 4 : 8;
  size_t bytes = align_up(n * rt) + 4 * align_up(n * vt);     // r, p, s, u, w
  bytes += align_up((size_t)148 * 32 * 4 * sizeof(double));    // partials (upper bound of blocks)
  bytes += align_up(4 * sizeof(double)) + align_up(8 * sizeof(unsigned int));
  return bytes;
}

template <int MODE>
static int launch_pcg(PcgArgs& a, int blocks_req, cudaStream_t st) {
  int dev = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pcg_kernel<MODE>, PCG_THREADS, 0);
  if (per_sm < 1) return NGS_ERR_CUDA;
  int64_t blocks = (int64_t)sms * per_sm;
  const int64_t need = (a.n * PCG_ROW_LANES + PCG_THREADS - 1) / PCG_THREADS;
  if (blocks > need) blocks = need > 0 ? need : 1;
  if (blocks_req > 0 && blocks_req < blocks) blocks = blocks_req;
  if (blocks > 148 * 32) blocks = 148 * 32;
  a.nblocks = (unsigned int)blocks;
  void* args[] = {&a};
  ngs_count_launch();
  cudaError_t e = cudaLaunchCooperativeKernel((const void*)pcg_kernel<MODE>, dim3((unsigned)blocks), dim3(PCG_THREADS),
                                              args, 0, st);
  if (e != cudaSuccess) return ngs_set_cuda_error(e);
  return NGS_OK;
}

extern "C" int ngs_pcg_solve(const ngs_pcg_system* sys, const ngs_pcg_config* cfg, void* ws, size_t ws_bytes,
                             int64_t* info_dev, double* resid_dev, ngs_stream s) {
  if (!sys || !cfg || !info_dev || !resid_dev || sys->n < 0 || !sys->rowptr || (sys->nnz > 0 && !sys->cols) ||
      !sys->inv_diag)
    return NGS_ERR_INVALID_ARG;
  const int mode = cfg->mode;
  if (mode < NGS_PCG_REFERENCE || mode > NGS_PCG_FP64) return NGS_ERR_INVALID_ARG;
  if (mode == NGS_PCG_REFERENCE && (!sys->vals32 || !sys->b32 || !sys->x32)) return NGS_ERR_INVALID_ARG;
  if (mode == NGS_PCG_MIXED && (!sys->vals32 || !sys->vals64 || !sys->b64 || !sys->x64)) return NGS_ERR_INVALID_ARG;
  if (mode == NGS_PCG_FP64 && (!sys->vals64 || !sys->b64 || !sys->x64)) return NGS_ERR_INVALID_ARG;
  if (!ws || ws_bytes < ngs_pcg_workspace_bytes(sys->n, mode)) return NGS_ERR_OOM;
  cudaStream_t st = (cudaStream_t)s;
  const int64_t n = sys->n;
  if (n == 0) {
    cudaMemsetAsync(info_dev, 0, 4 * sizeof(int64_t), st);
    cudaMemsetAsync(resid_dev, 0, 2 * sizeof(double), st);
    return NGS_OK;
  }
  const size_t vt = mode == NGS_PCG_REFERENCE ? 4 : 8;
  const size_t rt = mode == NGS_PCG_REFERENCE ? 4 : 8;
  char* base = static_cast<char*>(ws);
  PcgArgs a{};
  a.n = n;
  a.rowptr = sys->rowptr;
  a.cols = sys->cols;
  a.vals = mode == NGS_PCG_FP64 ? (const void*)sys->vals64 : (const void*)sys->vals32;
  a.vals64 = sys->vals64;
  a.b = mode == NGS_PCG_REFERENCE ? (const void*)sys->b32 : (const void*)sys->b64;
  a.inv_diag = sys->inv_diag;
  a.x = mode == NGS_PCG_REFERENCE ? (void*)sys->x32 : (void*)sys->x64;
  a.x32_out = mode == NGS_PCG_REFERENCE ? nullptr : sys->x32;
  a.r = base; base += align_up(n * rt);
  a.p = base; base += align_up(n * vt);
  a.s = base; base += align_up(n * vt);
  a.u = base; base += align_up(n * vt);
  a.w = base; base += align_up(n * vt);
  a.partials = reinterpret_cast<double*>(base); base += align_up((size_t)148 * 32 * 4 * sizeof(double));
  a.result = reinterpret_cast<double*>(base); base += align_up(4 * sizeof(double));
  unsigned int* ctl = reinterpret_cast<unsigned int*>(base);
  a.count = ctl;
  a.gen = ctl + 1;
  a.error = reinterpret_cast<int*>(ctl + 2);
  a.deadline = reinterpret_cast<unsigned long long*>(ctl + 4);
  cudaMemsetAsync(ctl, 0, 8 * sizeof(unsigned int), st);
  a.info = info_dev;
  a.resid = resid_dev;
  a.tol = cfg->tol;
  a.max_iter = cfg->max_iter;
  a.replace_every = mode == NGS_PCG_REFERENCE ? (cfg->res_fix ? 1 : 0) : cfg->replace_every;
  const double timeout = cfg->timeout_s > 0 ? cfg->timeout_s : 10.0;
  a.wait_ns = (unsigned long long)(timeout * 1e9);
  a.budget_ns = a.wait_ns;
  a.inner_rtol = 1.0e-4;
  int rc;
  if (mode == NGS_PCG_REFERENCE) rc = launch_pcg<NGS_PCG_REFERENCE>(a, cfg->blocks, st);
  else if (mode == NGS_PCG_MIXED) rc = launch_pcg<NGS_PCG_MIXED>(a, cfg->blocks, st);
  else rc = launch_pcg<NGS_PCG_FP64>(a, cfg->blocks, st);
  return rc;
}

// ----------------------------------------------------------------------------- FP64 building blocks
__global__ void spmv64_kernel(int64_t n, const int64_t* __restrict__ rp, const int32_t* __restrict__ cols,
                              const double* __restrict__ vals, const double* __restrict__ x, double* __restrict__ y) {
  const int sub = threadIdx.x & 15;
  const unsigned gmask = 0xFFFFu << ((threadIdx.x & 31) & 16);
  const int64_t groups = (int64_t)gridDim.x * (blockDim.x / 16);
  for (int64_t row = ngs_gtid() / 16;; row += groups) {
    if (!__any_sync(0xffffffffu, row < n)) break;
    if (row < n) {
      double acc = 0.0;
      for (int64_t j = rp[row] + sub; j < rp[row + 1]; j += 16) acc += vals[j] * x[cols[j]];
#pragma unroll
      for (int o = 8; o > 0; o >>= 1) acc += __shfl_xor_sync(gmask, acc, o);
      if (sub == 0) y[row] = acc;
    }
  }
}

__global__ void dot64_kernel(const double* __restrict__ a, const double* __restrict__ b, int64_t n, double* out) {
  double t = 0.0;
  for (int64_t i = ngs_gtid(); i < n; i += ngs_gstride()) t += a[i] * b[i];
  t = warp_sum(t);
  if ((threadIdx.x & 31) == 0) atomicAdd(out, t);
}

__global__ void axpby64_kernel(int64_t n, double alpha, const double* __restrict__ x, double beta, double* y) {
  for (int64_t i = ngs_gtid(); i < n; i += ngs_gstride()) y[i] = alpha * x[i] + beta * y[i];
}

__global__ void mul64_kernel(int64_t n, const double* __restrict__ a, const double* __restrict__ b, double* out) {
  for (int64_t i = ngs_gtid(); i < n; i += ngs_gstride()) out[i] = a[i] * b[i];
}

extern "C" int ngs_spmv64(int64_t n, const int64_t* rowptr, const int32_t* cols, const double* vals, const double* x,
                          double* y, ngs_stream s) {
  if (n < 0 || (n > 0 && (!rowptr || !cols || !vals || !x || !y))) return NGS_ERR_INVALID_ARG;
  if (n == 0) return NGS_OK;
  { ngs_count_launch(); spmv64_kernel<<<ngs_blocks(n * 16, 256), 256, 0, (cudaStream_t)s>>>(n, rowptr, cols, vals, x, y); }
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}

extern "C" int ngs_dot64(const double* a, const double* b, int64_t n, double* out_dev, ngs_stream s) {
  if (n < 0 || !out_dev || (n > 0 && (!a || !b))) return NGS_ERR_INVALID_ARG;
  cudaMemsetAsync(out_dev, 0, sizeof(double), (cudaStream_t)s);
  if (n > 0) { ngs_count_launch(); dot64_kernel<<<ngs_blocks(n, 256, 148 * 4), 256, 0, (cudaStream_t)s>>>(a, b, n, out_dev); }
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}

extern "C" int ngs_axpby64(int64_t n, double alpha, const double* x, double beta, double* y, ngs_stream s) {
  if (n < 0 || (n > 0 && (!x || !y))) return NGS_ERR_INVALID_ARG;
  if (n == 0) return NGS_OK;
  { ngs_count_launch(); axpby64_kernel<<<ngs_blocks(n, 256), 256, 0, (cudaStream_t)s>>>(n, alpha, x, beta, y); }
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}

extern "C" int ngs_mul64(int64_t n, const double* a, const double* b, double* out, ngs_stream s) {
  if (n < 0 || (n > 0 && (!a || !b || !out))) return NGS_ERR_INVALID_ARG;
  if (n == 0) return NGS_OK;
  { ngs_count_launch(); mul64_kernel<<<ngs_blocks(n, 256), 256, 0, (cudaStream_t)s>>>(n, a, b, out); }
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}
