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
//     barrier + reduce     every block publishes its partials, arrives, and once all
//                          have arrived sums all partials itself in block order
//                          (deterministic, the same bits in every block).
// The SpMV streams the CSR arrays straight from HBM: eight lanes per row at two blocks per SM,
// in one of two forms -- 4-byte columns, a row at a time with up to eight (column, value) pairs
// and their vector gathers in flight per lane, or 2-byte column deltas in a software-pipelined
// loop that gathers from a shared-memory window of the vector -- each with its own kernel for the
// single-system and cluster solves.  (Staging CSR tiles through shared memory with bulk copies ran
// at less than half this rate: the product and row-sum passes over shared memory, not the copies,
// bounded it.)
// Every wait is bounded by the global nanosecond timer; on timeout the kernel
// records NGS_ERR_TIMEOUT and returns.  Every solve is bounded too: at most
// NGS_PCG_ITER_CAP iterations, and a deadline that block 0 checks at each
// reduction and publishes with it, so that all blocks stop at the same iteration.  Dots are
// FP64 in every mode.
//
// Mixed precision (NGS_PCG_MIXED) is iterative refinement: the inner PCG runs on
// the FP32 matrix with FP32 search vectors (SpMV products summed in FP32 over rounds
// of four or eight, the rounds in FP64), FP64 dots, and FP64 x and r, until its residual
// has dropped by `inner_rtol`; then
// the true residual b - A x is formed with the FP64 matrix and the inner solve
// restarts from it.  The FP32 matrix is a fixed SPD perturbation of the FP64 one,
// so each outer step contracts the error by about |A32 - A64| |A64^-1| and the
// solve converges to the FP64 system.
//
// This file is compiled without multiply-add contraction (build.py): the solver body is inlined
// into the single-system, cluster and batched kernels, and only uncontracted arithmetic is
// guaranteed to round the same way in all of them, which makes a batched solve bit-identical to
// the solo one.
#include <algorithm>
#include <cmath>
#include "mf.cuh"

constexpr int PCG_THREADS = 512;
constexpr int PCG_MIN_BLOCKS = 2;      // blocks per SM the register budget is sized for
constexpr int PCG_ROW_LANES = 8;       // lanes per row in the SpMV
constexpr int PCG_ROW_COST = 8;        // work of a row on top of its non-zeros (vector traffic)
constexpr int PCG_BLOCK_WORK = 16384;  // work (non-zeros + row cost) that justifies one more block
constexpr int PCG_CLUSTER_MAX = 16;    // CTAs of the largest thread-block cluster a small system gets
constexpr int PCG_CLUSTER_NEED = 64;   // systems of at most this many blocks' work are solved by a cluster
// Most blocks one cooperative solve may use (B200: 148 SMs x 2 = 296).  The capacity query clamps to
// it, and the per-block partials area of the workspace is sized from it: reductions double-buffer the
// partials by barrier parity, 2 x PCG_MAX_BLOCKS x 4 doubles.
constexpr int PCG_MAX_BLOCKS = 1024;
constexpr size_t PCG_PARTIALS_BYTES = (size_t)2 * PCG_MAX_BLOCKS * 4 * sizeof(double);

struct PcgArgs {
  int64_t n;
  int64_t nnz;
  const int64_t* rowptr;
  const int32_t* cols;
  const int16_t* cols16;     // column - row per entry (2 bytes instead of 4), or NULL
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
  double* partials;          // [2][nblocks][4]: per-block partial sums, by barrier parity
  unsigned int* count;       // arrival counter of the grid barriers
  int* error;
  int64_t* info;             // {iters, status, replacements, -}
  double* resid;             // {|r|, |b|}
  double tol;
  int max_iter;
  int replace_every;         // <= 0: never
  double inner_rtol;         // MIXED: relative reduction of an inner solve
  unsigned long long wait_ns;     // bound of one barrier wait
  unsigned long long* deadline;   // absolute global-timer deadline, set by block 0 at the first reduction
  unsigned long long budget_ns;   // time budget of the whole solve
  unsigned int nblocks;
  int evict_first;                // stream the matrix past the caches (it does not fit L2)
  int mf;                         // the matrix-free operator below replaces the CSR
  ngs_pcg_operator op;
  int win_cap;                    // elements of the search vector a block can stage in shared memory
};

// Shared memory (dynamic) of every PCG block for its window of the search vector: the SpMV of a
// block's rows gathers from the contiguous range of rows that its columns span (rows are ranks in
// (x, y, z) order, so a block's 5x5x5 stencils reach a band of neighbouring x slabs), loaded once per
// iteration with coalesced loads.  Gathers from L1 cost one wavefront per distinct cache line of the
// warp (the ~60 columns of a row lie in 25 different z columns); from shared memory a few at most.
constexpr int PCG_WIN_BYTES = 96 * 1024;

constexpr int NGS_PCG_ITER_CAP = 20000;

NGS_DEV unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

template <typename T>
NGS_DEV T ld_cg(const T* p) { return *reinterpret_cast<const volatile T*>(p); }

// Block b owns the rows whose first non-zero lies in [b * nnz / B, (b + 1) * nnz / B).
NGS_DEV int64_t first_row_at(const int64_t* __restrict__ rp, int64_t n, int64_t e) {
  int64_t lo = 0, hi = n;
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if (rp[mid] < e) lo = mid + 1; else hi = mid;
  }
  return lo;
}

// Rows [row0, row1) of block bid, and whether every one of them holds at least one entry
// (an SPD row holds its diagonal); the check is block-uniform.
NGS_DEV bool block_rows(const PcgArgs& a, unsigned bid, int64_t& row0, int64_t& row1) {
  __shared__ int64_t bounds[2];
  __shared__ int bad;
  if (a.mf) {                   // matrix-free: every row costs about the same; equal row ranges
    row0 = (a.n * (int64_t)bid) / a.nblocks;
    row1 = (a.n * ((int64_t)bid + 1)) / a.nblocks;
    return true;
  }
  if (threadIdx.x == 0) {
    const int64_t B = a.nblocks;
    bounds[0] = first_row_at(a.rowptr, a.n, (a.nnz * (int64_t)bid) / B);
    bounds[1] = bid + 1 == a.nblocks ? a.n : first_row_at(a.rowptr, a.n, (a.nnz * ((int64_t)bid + 1)) / B);
    bad = 0;
  }
  __syncthreads();
  row0 = bounds[0];
  row1 = bounds[1];
  for (int64_t r = row0 + threadIdx.x; r < row1; r += blockDim.x)
    if (a.rowptr[r + 1] <= a.rowptr[r]) bad = 1;
  return __syncthreads_or(bad) == 0;
}

// Loads of the (immutable) matrix.  A matrix larger than L2 is streamed evict-first, so that the
// gathered vector keeps its place in the caches; a smaller one stays cached for the next iteration.
template <bool STREAM, typename T>
NGS_DEV T ld_mat(const T* p) {
  if constexpr (STREAM) return __ldcs(p);
  else return __ldg(p);
}

// One round of a row's entries for lane sub: entries j0, j0 + L, ...; entries past the row's end
// gather the row's own element (the diagonal's, cached) and weigh it by zero, so that the gathers
// need no predicate.
template <bool STREAM, bool DELTA, int L, int U, typename MT>
NGS_DEV void spmv_load_round(const PcgArgs& a, const MT* __restrict__ vals, int64_t row, int64_t j0, int64_t e1,
                             int32_t (&c)[U], MT (&m)[U]) {
#pragma unroll
  for (int k = 0; k < U; k++) {
    const int64_t j = j0 + (int64_t)k * L;
    if constexpr (DELTA) c[k] = (int32_t)row + (j < e1 ? (int32_t)ld_mat<STREAM>(a.cols16 + j) : 0);
    else c[k] = j < e1 ? ld_mat<STREAM>(a.cols + j) : (int32_t)row;
    m[k] = j < e1 ? ld_mat<STREAM>(vals + j) : (MT)0;
  }
}

// The round's products summed in the matrix type (two chains), returned in ACC: one conversion per
// round instead of two per product; the FP64 refinement of the mixed mode works from the true
// residual, so this rounding only shapes the inner iterations.
template <typename MT, typename VT, typename ACC, int U>
NGS_DEV ACC spmv_round_sum(const VT* v, int64_t voff, const int32_t (&c)[U], const MT (&m)[U]) {
  VT xv[U];
#pragma unroll
  for (int k = 0; k < U; k++) xv[k] = v[c[k] - voff];
  MT r0 = (MT)0, r1 = (MT)0;
#pragma unroll
  for (int k = 0; k < U; k += 2) {
    r0 += m[k] * (MT)xv[k];
    r1 += m[k + 1] * (MT)xv[k + 1];
  }
  return (ACC)r0 + (ACC)r1;
}

// y = A v over rows [row0, row1): eight lanes per row, a warp on four consecutive rows (their entries
// are contiguous: coalesced matrix loads).  epi(row, acc, pre(row)) consumes each row's product (lane
// 0 of its group) and returns a contribution to the thread's partial sum.  The gathered vector is
// read with plain loads: it was written earlier in this launch.  Both forms end with a block barrier,
// after which every thread may read the rows written by the epilogue.
//
// Software-pipelined form (2-byte column deltas): the next row's pointers and first round of entries
// are loaded before this row's gathers are consumed (a row otherwise waits on three dependent round
// trips: row pointer, matrix entries, gathered vector).  Rounds of four entries per lane keep the
// loop at 64 registers (two 512-thread blocks per SM); the prefetch is unconditional -- past the
// group's last row it reads an empty range -- so that the arrays stay in registers.
template <bool STREAM, bool DELTA, typename MT, typename VT, typename ACC, typename Pre, typename Epi>
NGS_DEV void spmv_rows_piped(const PcgArgs& a, const MT* __restrict__ vals, const VT* v, int64_t voff, int64_t row0,
                             int64_t row1, Pre pre, Epi epi, double& dsum) {
  constexpr int L = PCG_ROW_LANES;
  constexpr int U = 4;
  const int sub = threadIdx.x & (L - 1);
  const unsigned gmask = ((1u << L) - 1u) << ((threadIdx.x & 31) & ~(L - 1));
  const int64_t step = blockDim.x / L;
  int64_t row = row0 + threadIdx.x / L;
  int64_t e0 = 0, e1 = 0;
  if (row < row1) {
    e0 = a.rowptr[row];
    e1 = a.rowptr[row + 1];
  }
  int32_t c[U];
  MT m[U];
  spmv_load_round<STREAM, DELTA, L, U>(a, vals, row, e0 + sub, e1, c, m);
  for (; row < row1; row += step) {
    const int64_t ce0 = e0, ce1 = e1, nrow = row + step;
    const bool more = nrow < row1;
    e0 = more ? a.rowptr[nrow] : 0;
    e1 = more ? a.rowptr[nrow + 1] : 0;
    const double2 ax = pre(row);
    ACC acc = spmv_round_sum<MT, VT, ACC, U>(v, voff, c, m);
    for (int64_t j0 = ce0 + sub + U * L; j0 < ce1; j0 += U * L) {     // the row's further rounds
      spmv_load_round<STREAM, DELTA, L, U>(a, vals, row, j0, ce1, c, m);
      acc += spmv_round_sum<MT, VT, ACC, U>(v, voff, c, m);
    }
    spmv_load_round<STREAM, DELTA, L, U>(a, vals, more ? nrow : row, e0 + sub, e1, c, m);
#pragma unroll
    for (int o = L / 2; o > 0; o >>= 1) acc += __shfl_xor_sync(gmask, acc, o);
    if (sub == 0) dsum += epi(row, (double)acc, ax);
  }
  // the epilogue wrote rows that other threads of the block read next (their rows in phase A)
  __syncthreads();
}

// Row-at-a-time form (4-byte columns): rounds of eight entries per lane, all of a round's loads and
// gathers in flight; a 5x5x5 stencil row (<= 125 entries, ~60 on a surface) takes one or two
// rounds.  With 4-byte columns this form is the faster one on large matrices (the level 0 of a
// 5M-point room: 94 against 98 ms), with 2-byte deltas the pipelined one (the level 0 of a
// 300k-point cloud: 9.3 against 9.7 ms).
template <bool STREAM, bool DELTA, typename MT, typename VT, typename ACC, typename Pre, typename Epi>
NGS_DEV void spmv_rows_plain(const PcgArgs& a, const MT* __restrict__ vals, const VT* v, int64_t voff, int64_t row0,
                             int64_t row1, Pre pre, Epi epi, double& dsum) {
  constexpr int L = PCG_ROW_LANES;
  constexpr int U = 8;
  const int sub = threadIdx.x & (L - 1);
  const unsigned gmask = ((1u << L) - 1u) << ((threadIdx.x & 31) & ~(L - 1));
  const int64_t step = blockDim.x / L;
  for (int64_t row = row0 + threadIdx.x / L; row < row1; row += step) {
    const int64_t e0 = a.rowptr[row], e1 = a.rowptr[row + 1];
    const double2 ax = pre(row);
    ACC acc = (ACC)0;
    for (int64_t j0 = e0 + sub; j0 < e1; j0 += U * L) {
      int32_t c[U];
      MT m[U];
      spmv_load_round<STREAM, DELTA, L, U>(a, vals, row, j0, e1, c, m);
      acc += spmv_round_sum<MT, VT, ACC, U>(v, voff, c, m);
    }
#pragma unroll
    for (int o = L / 2; o > 0; o >>= 1) acc += __shfl_xor_sync(gmask, acc, o);
    if (sub == 0) dsum += epi(row, (double)acc, ax);
  }
  __syncthreads();
}
// The streaming choice is a template argument: one load form per instantiation (a runtime choice
// per load cost 7 % of the level-0 solve and forced register spills).  FORM picks the SpMV form at
// compile time (kernels specialised per form, so that one form's register allocation is not shaped
// by the others') or, with PCG_FORM_ANY, at run time from the system (one kernel for every system of
// a batch or a cluster launch).  Each form runs the same uncontracted arithmetic in every kernel, so
// a system's result does not depend on which kernel solved it.
constexpr int PCG_FORM_ANY = 0, PCG_FORM_DELTA_STREAM = 1, PCG_FORM_DELTA = 2, PCG_FORM_COLS_STREAM = 3,
              PCG_FORM_COLS = 4;

template <int FORM, typename MT, typename VT, typename ACC, typename Pre, typename Epi>
NGS_DEV void spmv_rows(const PcgArgs& a, const MT* __restrict__ vals, const VT* v, int64_t voff, int64_t row0,
                       int64_t row1, Pre pre, Epi epi, double& dsum) {
  if constexpr (FORM == PCG_FORM_DELTA_STREAM) {
    spmv_rows_piped<true, true, MT, VT, ACC>(a, vals, v, voff, row0, row1, pre, epi, dsum);
  } else if constexpr (FORM == PCG_FORM_DELTA) {
    spmv_rows_piped<false, true, MT, VT, ACC>(a, vals, v, voff, row0, row1, pre, epi, dsum);
  } else if constexpr (FORM == PCG_FORM_COLS_STREAM) {
    spmv_rows_plain<true, false, MT, VT, ACC>(a, vals, v, voff, row0, row1, pre, epi, dsum);
  } else if constexpr (FORM == PCG_FORM_COLS) {
    spmv_rows_plain<false, false, MT, VT, ACC>(a, vals, v, voff, row0, row1, pre, epi, dsum);
  } else if (a.cols16) {
    // the column encoding too: 2-byte deltas when the caller supplied them, 4-byte columns otherwise
    if (a.evict_first) spmv_rows_piped<true, true, MT, VT, ACC>(a, vals, v, voff, row0, row1, pre, epi, dsum);
    else spmv_rows_piped<false, true, MT, VT, ACC>(a, vals, v, voff, row0, row1, pre, epi, dsum);
  } else {
    if (a.evict_first) spmv_rows_plain<true, false, MT, VT, ACC>(a, vals, v, voff, row0, row1, pre, epi, dsum);
    else spmv_rows_plain<false, false, MT, VT, ACC>(a, vals, v, voff, row0, row1, pre, epi, dsum);
  }
}

// The range of columns [wlo, whi) that the rows [row0, row1) reach (columns are sorted within a row:
// its first and last entries bound it), into shared memory.  Block-wide.
NGS_DEV void csr_window(const PcgArgs& a, int64_t row0, int64_t row1, unsigned long long& wlo,
                        unsigned long long& whi) {
  if (threadIdx.x == 0) {
    wlo = ~0ull;
    whi = 0ull;
  }
  __syncthreads();
  unsigned long long mlo = ~0ull, mhi = 0ull;
  for (int64_t r = row0 + threadIdx.x; r < row1; r += blockDim.x) {
    const int64_t e0 = a.rowptr[r], e1 = a.rowptr[r + 1];
    if (e1 <= e0) continue;
    const int64_t c0 = a.cols16 ? r + a.cols16[e0] : a.cols[e0];
    const int64_t c1 = a.cols16 ? r + a.cols16[e1 - 1] : a.cols[e1 - 1];
    mlo = min(mlo, (unsigned long long)c0);
    mhi = max(mhi, (unsigned long long)(c1 + 1));
  }
  if (mlo != ~0ull) atomicMin(&wlo, mlo);
  if (mhi != 0ull) atomicMax(&whi, mhi);
  __syncthreads();
  if (threadIdx.x == 0 && wlo == ~0ull) wlo = whi = 0ull;
  __syncthreads();
}

// Grid synchronisation of a cooperative launch through one arrival counter in global memory (zeroed
// before the launch, never reset inside it): barrier k of the launch (k = 1, 2, ... -- every block
// takes the same sequence) is passed once the counter reaches k * nblocks.  Thread 0 of the block
// arrives and waits; the wait is bounded by the global timer and ends early if another block
// recorded an error.
NGS_DEV bool grid_arrive_wait(const PcgArgs& a, unsigned int target) {
  __threadfence();
  atomicAdd(a.count, 1u);
  const unsigned long long t0 = global_ns();
  while (*reinterpret_cast<volatile unsigned int*>(a.count) < target) {
    if (*reinterpret_cast<volatile int*>(a.error)) return false;
    if (global_ns() - t0 > a.wait_ns) {
      atomicExch(a.error, NGS_ERR_TIMEOUT);
      return false;
    }
    __nanosleep(32);
  }
  __threadfence();
  return true;
}

// Synchronisation of the blocks that solve one system.  GridSync: the blocks of a cooperative
// launch, through the arrival counter (bounded waits).  A reduction publishes the block's partial
// sums before arriving, and after the barrier EVERY block sums all blocks' partials itself, in block
// order with the same code -- the same bits in every block, and no second round trip through a
// last block that sums and releases the others.  The partials are double-buffered by barrier
// parity: a block can only write the buffer of reduction k + 2 after every block has arrived at
// reduction k + 1, that is, after every block has read reduction k.  The solve deadline is decided
// by block 0 and travels in its partial slot 3, so every block takes the same decision.
// ClusterSync: the CTAs of one thread-block cluster, through the hardware cluster barrier and
// distributed shared memory -- no spinning, no co-residency requirement beyond the cluster, which
// the hardware schedules as a unit.
struct GridSync {
  const PcgArgs& a;
  unsigned bid;
  unsigned int epoch;
  bool is_late;
  NGS_DEV GridSync(const PcgArgs& args, unsigned b) : a(args), bid(b), epoch(0), is_late(false) {}

  NGS_DEV bool barrier() {
    __shared__ int ok;
    epoch++;
    __syncthreads();
    if (threadIdx.x == 0) ok = grid_arrive_wait(a, epoch * a.nblocks);
    __syncthreads();
    return ok != 0;
  }

  template <int NV>
  NGS_DEV bool reduce(const double (&v)[NV], double (&out)[NV]) {
    static_assert(NV <= 3, "slot 3 carries the deadline flag");
    __shared__ double red[NV][PCG_THREADS / 32];
    __shared__ int ok;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    epoch++;
    double* part = a.partials + (size_t)(epoch & 1u) * a.nblocks * 4;
#pragma unroll
    for (int k = 0; k < NV; k++) {
      const double t = warp_sum(v[k]);
      if (lane == 0) red[k][wid] = t;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
      for (int k = 0; k < NV; k++) {
        double t = 0.0;
        for (int i = 0; i < PCG_THREADS / 32; i++) t += red[k][i];
        part[(size_t)bid * 4 + k] = t;
      }
      if (bid == 0) {
        const unsigned long long now = global_ns();
        if (*a.deadline == 0ull) *a.deadline = now + a.budget_ns;
        part[3] = now > *a.deadline ? 1.0 : 0.0;
      }
      ok = grid_arrive_wait(a, epoch * a.nblocks);
    }
    __syncthreads();
    if (!ok) return false;
#pragma unroll
    for (int k = 0; k < NV; k++) {
      double t = 0.0;
      for (unsigned int i = threadIdx.x; i < a.nblocks; i += PCG_THREADS) t += ld_cg(part + (size_t)i * 4 + k);
      t = warp_sum(t);
      __syncwarp();
      if (lane == 0) red[k][wid] = t;
    }
    is_late = ld_cg(part + 3) != 0.0;
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NV; k++) {
      double t = 0.0;
      for (int i = 0; i < PCG_THREADS / 32; i++) t += red[k][i];
      out[k] = t;
    }
    __syncthreads();            // red is rewritten by the next reduction
    return true;
  }
  NGS_DEV bool late() const { return is_late; }
};

NGS_DEV void cluster_sync_all() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
NGS_DEV double ld_dsmem(const double* p, unsigned rank) {
  uint32_t la = (uint32_t)__cvta_generic_to_shared(p), ra;
  double v;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(ra) : "r"(la), "r"(rank));
  asm volatile("ld.shared::cluster.f64 %0, [%1];" : "=d"(v) : "r"(ra) : "memory");
  return v;
}
NGS_DEV unsigned cluster_rank() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
NGS_DEV unsigned cluster_size() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(r));
  return r;
}

struct ClusterSync {
  unsigned rank, size;
  double* cred;                    // shared [2][4]: this CTA's partial sums, double-buffered
  double* bcast;                   // shared [4]: the cluster sums, for the CTA's threads
  int parity;
  unsigned long long deadline, budget;   // rank 0, thread 0 decides the deadline for everyone
  bool is_late;
  template <int NV>
  NGS_DEV bool reduce(const double (&v)[NV], double (&out)[NV]) {
    __shared__ double red[NV > 0 ? NV : 1][PCG_THREADS / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; k++) {
      const double t = warp_sum(v[k]);
      if (lane == 0) red[k][wid] = t;
    }
    __syncthreads();
    double* mine = cred + parity * 4;
    if (threadIdx.x == 0) {
#pragma unroll
      for (int k = 0; k < NV; k++) {
        double t = 0.0;
        for (int i = 0; i < PCG_THREADS / 32; i++) t += red[k][i];
        mine[k] = t;
      }
      if (rank == 0) {
        const unsigned long long now = global_ns();
        if (deadline == 0ull) deadline = now + budget;
        mine[3] = now > deadline ? 1.0 : 0.0;
      }
    }
    cluster_sync_all();          // every CTA's partials are written
    if (threadIdx.x == 0) {
      // the same fixed rank order in every CTA: every CTA gets the same sums, bit for bit
#pragma unroll
      for (int k = 0; k < NV; k++) {
        double t = 0.0;
        for (unsigned r = 0; r < size; r++) t += ld_dsmem(mine + k, r);
        bcast[k] = t;
      }
      bcast[3] = ld_dsmem(mine + 3, 0);
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NV; k++) out[k] = bcast[k];
    is_late = bcast[3] != 0.0;
    __syncthreads();             // bcast is rewritten by the next reduction
    parity ^= 1;                 // the other buffer: a CTA may write it while others still read this one
    return true;
  }
  NGS_DEV bool barrier() {
    cluster_sync_all();
    return true;
  }
  NGS_DEV bool late() const { return is_late; }
};

template <int MODE>
struct PcgTypes;
template <> struct PcgTypes<NGS_PCG_REFERENCE> { using MT = float; using VT = float; using RT = float; using ACC = float; };
template <> struct PcgTypes<NGS_PCG_MIXED> { using MT = float; using VT = float; using RT = double; using ACC = double; };
template <> struct PcgTypes<NGS_PCG_FP64> { using MT = double; using VT = double; using RT = double; using ACC = double; };

// Status of a solve.  The launcher zeroes info; every write is a maximum, and the codes grow with
// severity (OK < INVALID_ARG < NOT_CONVERGED < TIMEOUT), so that a block that gave up at a barrier
// and block 0 finishing its own rows can both write without one hiding the other.
NGS_DEV void pcg_record(const PcgArgs& a, int status, int it) {
  atomicMax(reinterpret_cast<unsigned long long*>(a.info + 1), (unsigned long long)status);
  atomicMax(reinterpret_cast<unsigned long long*>(a.info), (unsigned long long)it);
}

// A barrier or reduction gave up (its bounded wait ran out, or another block recorded an error):
// the block leaves the solve and says why.
NGS_DEV void pcg_abandon(const PcgArgs& a, int it) {
  if (threadIdx.x == 0) {
    const int e = *reinterpret_cast<volatile int*>(a.error);
    pcg_record(a, e != 0 ? e : NGS_ERR_TIMEOUT, it);
  }
}

// The solve of one system by the blocks bid = 0 .. a.nblocks-1 of a launch (all of them for a
// single solve, a contiguous range for one system of a batch, the CTAs of one cluster).
// OPS: which operators the instantiation carries -- PCG_OPS_CSR, PCG_OPS_MF, or both (chosen per system
// at run time; the batched kernel when a batch mixes them).  Single-operator instantiations keep the
// register budget of the other operator's code out of the kernel.
constexpr int PCG_OPS_CSR = 1, PCG_OPS_MF = 2, PCG_OPS_BOTH = 3;

template <int MODE, int OPS, int FORM, typename Sync>
NGS_DEV void pcg_body(const PcgArgs& a, const unsigned bid, Sync& sy) {
  using MT = typename PcgTypes<MODE>::MT;
  using VT = typename PcgTypes<MODE>::VT;
  using RT = typename PcgTypes<MODE>::RT;
  using ACC = typename PcgTypes<MODE>::ACC;
  const RT* b = static_cast<const RT*>(a.b);
  RT* x = static_cast<RT*>(a.x);
  RT* r = static_cast<RT*>(a.r);
  VT* p = static_cast<VT*>(a.p);
  VT* s = static_cast<VT*>(a.s);
  VT* u = static_cast<VT*>(a.u);
  VT* w = static_cast<VT*>(a.w);
  const MT* vals = static_cast<const MT*>(a.vals);
  const int sqrt_n = (int)ceil(sqrt((double)a.n));

  int64_t row0, row1;
  const bool rows_ok = block_rows(a, bid, row0, row1);
  const int64_t i0 = row0 + threadIdx.x, i1 = row1, is = PCG_THREADS;

  // w = A u; returns (w, u).
  auto w_pre = [&](int64_t row) -> double2 { return make_double2((double)u[row], 0.0); };
  auto w_epi = [&](int64_t row, double acc, double2 ax) -> double {
    w[row] = (VT)acc;
    return acc * ax.x;
  };
  // r = b - A x, u = M r; returns (r, r).
  auto res_pre = [&](int64_t row) -> double2 { return make_double2((double)b[row], (double)a.inv_diag[row]); };
  auto true_res_epi = [&](int64_t row, double acc, double2 ax) -> double {
    const RT ri = (RT)(ax.x - acc);
    r[row] = ri;
    u[row] = (VT)(ax.y * (double)ri);
    return (double)ri * (double)ri;
  };
  // the true residual uses the FP64 matrix in MIXED mode, the recurrence matrix otherwise
  auto spmv_true = [&](double& sum) {
    if constexpr (MODE == NGS_PCG_MIXED) spmv_rows<FORM, double, RT, double>(a, a.vals64, x, 0, row0, row1, res_pre, true_res_epi, sum);
    else spmv_rows<FORM, MT, RT, ACC>(a, vals, x, 0, row0, row1, res_pre, true_res_epi, sum);
  };
  // w = A u: the block's window of u staged in shared memory when it fits (refreshed every product;
  // the grid barrier before the product made every block's u rows visible)
  // (the window bounds stay in shared memory, not in registers across the solve)
  extern __shared__ __align__(16) unsigned char pcg_win_raw[];
  __shared__ unsigned long long win_bounds[2];
  if (threadIdx.x == 0) win_bounds[0] = win_bounds[1] = 0ull;
  __syncthreads();
  if constexpr (OPS & PCG_OPS_CSR) {
    if (!a.mf && rows_ok && a.win_cap > 0) csr_window(a, row0, row1, win_bounds[0], win_bounds[1]);
  }
  auto spmv_w = [&](double& sum) {
    const int64_t wlo = (int64_t)win_bounds[0], wn = (int64_t)win_bounds[1] - wlo;
    if (wn > 0 && wn <= a.win_cap) {
      VT* win = reinterpret_cast<VT*>(pcg_win_raw);
      for (int64_t i = threadIdx.x; i < wn; i += PCG_THREADS) win[i] = u[wlo + i];
      __syncthreads();
      spmv_rows<FORM, MT, VT, ACC>(a, vals, win, wlo, row0, row1, w_pre, w_epi, sum);
    } else {
      spmv_rows<FORM, MT, VT, ACC>(a, vals, u, 0, row0, row1, w_pre, w_epi, sum);
    }
  };

  // Matrix-free operator (mf.cuh): the stencil in shared memory (FP32 for the inner products of the
  // mixed mode, FP64 for its true residual and for the FP64 mode), the points split evenly over the
  // blocks.  An application is two passes with a barrier between them: t = Phi v over the block's
  // points, then the block's rows.  Returns false if the barrier gave up.
  __shared__ float ks32[125];
  __shared__ double ks64[125];
  int64_t pt0 = 0, pt1 = 0;
  if ((OPS & PCG_OPS_MF) && a.mf) {
    for (int k = threadIdx.x; k < 125; k += PCG_THREADS) {
      ks64[k] = a.op.stencil[k];
      ks32[k] = (float)a.op.stencil[k];
    }
    pt0 = (a.op.n_points * (int64_t)bid) / a.nblocks;
    pt1 = (a.op.n_points * ((int64_t)bid + 1)) / a.nblocks;
    __syncthreads();
  }
  auto mf_w = [&](double& sum) -> bool {
    if constexpr (MODE == NGS_PCG_REFERENCE) {
      return false;                                   // not offered in this mode (rejected on the host)
    } else {
      using TT = VT;
      TT* t = MODE == NGS_PCG_FP64 ? reinterpret_cast<TT*>(a.op.scratch64) : reinterpret_cast<TT*>(a.op.scratch32);
      mf_points<VT, TT>(a.op, u, t, pt0 + threadIdx.x, pt1, PCG_THREADS);
      if (!sy.barrier()) return false;
      const MT* ks = MODE == NGS_PCG_FP64 ? reinterpret_cast<const MT*>(ks64) : reinterpret_cast<const MT*>(ks32);
      for (int64_t i = i0; i < i1; i += is) sum += w_epi(i, (double)mf_row<MT, VT, TT, ACC>(a.op, ks, u, t, i), w_pre(i));
      __syncthreads();
      return true;
    }
  };
  auto mf_true = [&](double& sum) -> bool {
    if constexpr (MODE == NGS_PCG_REFERENCE) {
      return false;
    } else {
      mf_points<RT, double>(a.op, x, a.op.scratch64, pt0 + threadIdx.x, pt1, PCG_THREADS);
      if (!sy.barrier()) return false;
      for (int64_t i = i0; i < i1; i += is)
        sum += true_res_epi(i, mf_row<double, RT, double, double>(a.op, ks64, x, a.op.scratch64, i), res_pre(i));
      __syncthreads();
      return true;
    }
  };
  // w = A u / r = b - A x through whichever operator the system has; false: a barrier gave up
  auto apply_w = [&](double& sum) -> bool {
    if constexpr (OPS & PCG_OPS_MF) {
      if (OPS == PCG_OPS_MF || a.mf) return mf_w(sum);
    }
    if constexpr (OPS & PCG_OPS_CSR) spmv_w(sum);
    return true;
  };
  auto apply_true = [&](double& sum) -> bool {
    if constexpr (OPS & PCG_OPS_MF) {
      if (OPS == PCG_OPS_MF || a.mf) return mf_true(sum);
    }
    if constexpr (OPS & PCG_OPS_CSR) spmv_true(sum);
    return true;
  };

  // init: x = 0, r = b, u = M r, p = s = 0; partial (b, b); part[1] flags empty rows
  double part[3] = {0.0, rows_ok ? 0.0 : 1.0, 0.0}, res[3];
  int it = 0, replacements = 0;
  for (int64_t i = i0; i < i1; i += is) {
    const RT bi = b[i];
    x[i] = (RT)0;
    r[i] = bi;
    u[i] = (VT)((double)a.inv_diag[i] * (double)bi);
    p[i] = (VT)0;
    s[i] = (VT)0;
    part[0] += (double)bi * (double)bi;
  }
  if (!sy.template reduce<3>(part, res)) return pcg_abandon(a, it);
  if (res[1] > 0.0) {                                    // every block sees the same flag: no copy was issued
    if (bid == 0 && threadIdx.x == 0) pcg_record(a, NGS_ERR_INVALID_ARG, 0);
    return;
  }
  const double bnorm = sqrt(res[0]);
  const double atol = a.tol * bnorm;
  part[0] = part[1] = part[2] = 0.0;
  if (!apply_w(part[1])) return pcg_abandon(a, it);
  for (int64_t i = i0; i < i1; i += is) {
    part[0] += (double)r[i] * (double)u[i];
    part[2] += (double)r[i] * (double)r[i];
  }
  if (!sy.template reduce<3>(part, res)) return pcg_abandon(a, it);
  double gamma = res[0], delta = res[1], rho = res[2];
  double alpha = delta != 0.0 ? gamma / delta : 0.0, beta = 0.0;
  const double rtol_inner = MODE == NGS_PCG_MIXED ? a.inner_rtol : 0.0;
  double target = fmax(atol, rtol_inner * sqrt(rho));
  bool converged = sqrt(rho) <= atol || bnorm == 0.0, timed_out = false;
  const int cap = (a.max_iter >= 0 && a.max_iter < NGS_PCG_ITER_CAP) ? a.max_iter : NGS_PCG_ITER_CAP;
  while (!converged && it < cap) {
    if (sy.late()) { timed_out = true; break; }
    const bool replace =
        (MODE == NGS_PCG_MIXED && a.replace_every > 0 && (it + 1) % a.replace_every == 0) ||
        (MODE == NGS_PCG_REFERENCE && a.replace_every > 0 && (it + 1) % sqrt_n == 0);
    // phase A (own rows); the dots (r,u), (r,r) of the new residual are taken here
    part[0] = part[1] = part[2] = 0.0;
#pragma unroll 4
    for (int64_t i = i0; i < i1; i += is) {
      const VT pi = (VT)((double)u[i] + beta * (double)p[i]);
      const VT si = (VT)((double)w[i] + beta * (double)s[i]);
      p[i] = pi;
      s[i] = si;
      x[i] = (RT)((double)x[i] + alpha * (double)pi);
      if (!replace) {
        const RT ri = (RT)((double)r[i] - alpha * (double)si);
        const VT ui = (VT)((double)a.inv_diag[i] * (double)ri);
        r[i] = ri;
        u[i] = ui;
        part[0] += (double)ri * (double)ui;
        part[2] += (double)ri * (double)ri;
      }
    }
    if (replace) {
      // residual replacement: r = b - A x (FP64 matrix in MIXED mode, the FP32 one in REFERENCE mode)
      if (!sy.barrier()) return pcg_abandon(a, it);
      double rr = 0.0;
      if (!apply_true(rr)) return pcg_abandon(a, it);
      part[2] = rr;
      for (int64_t i = i0; i < i1; i += is) part[0] += (double)r[i] * (double)u[i];
      replacements++;
    }
    if (!sy.barrier()) return pcg_abandon(a, it);
    // phase B: w = A u and (w, u)
    if (!apply_w(part[1])) return pcg_abandon(a, it);
    if (!sy.template reduce<3>(part, res)) return pcg_abandon(a, it);
    it++;
    const double gamma_new = res[0];
    delta = res[1];
    rho = res[2];
    if (sqrt(rho) <= target) {
      if (MODE != NGS_PCG_MIXED) { converged = true; break; }
      // end of an inner solve: true FP64 residual, stop or restart the recurrences from it
      if (!sy.barrier()) return pcg_abandon(a, it);
      part[0] = part[1] = part[2] = 0.0;
      if (!apply_true(part[2])) return pcg_abandon(a, it);
      replacements++;
      for (int64_t i = i0; i < i1; i += is) part[0] += (double)r[i] * (double)u[i];
      if (!sy.barrier()) return pcg_abandon(a, it);
      if (!apply_w(part[1])) return pcg_abandon(a, it);
      if (!sy.template reduce<3>(part, res)) return pcg_abandon(a, it);
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
    for (int64_t i = i0; i < i1; i += is) a.x32_out[i] = (float)x[i];
  if (bid == 0 && threadIdx.x == 0) {
    pcg_record(a, converged ? NGS_OK : (timed_out ? NGS_ERR_TIMEOUT : NGS_ERR_NOT_CONVERGED), it);
    a.info[2] = replacements;
    a.resid[0] = sqrt(rho);
    a.resid[1] = bnorm;
  }
}

template <int MODE, int OPS>
__global__ void __launch_bounds__(PCG_THREADS, PCG_MIN_BLOCKS) pcg_kernel(const __grid_constant__ PcgArgs a) {
  GridSync sy(a, blockIdx.x);
  pcg_body<MODE, OPS, PCG_FORM_ANY>(a, blockIdx.x, sy);
}

// The single-system solve of an assembled matrix with its SpMV form fixed at compile time.
template <int MODE, int FORM>
__global__ void __launch_bounds__(PCG_THREADS, PCG_MIN_BLOCKS) pcg_form_kernel(const __grid_constant__ PcgArgs a) {
  GridSync sy(a, blockIdx.x);
  pcg_body<MODE, PCG_OPS_CSR, FORM>(a, blockIdx.x, sy);
}

// A small system solved by one thread-block cluster (a.nblocks CTAs, the whole grid).
template <int MODE, int OPS>
__global__ void __launch_bounds__(PCG_THREADS, PCG_MIN_BLOCKS) pcg_cluster_kernel(const __grid_constant__ PcgArgs a) {
  __shared__ double cred[8], bcast[4];
  ClusterSync sy{cluster_rank(), cluster_size(), cred, bcast, 0, 0ull, a.budget_ns, false};
  pcg_body<MODE, OPS, PCG_FORM_ANY>(a, sy.rank, sy);
  cluster_sync_all();            // no CTA exits while another may still read its shared memory
}

// The cluster solve of an assembled matrix with its SpMV form fixed at compile time (the matrices
// of cluster-sized systems are far below the streaming threshold: the unstreamed forms only).
template <int MODE, int FORM>
__global__ void __launch_bounds__(PCG_THREADS, PCG_MIN_BLOCKS) pcg_cluster_form_kernel(const __grid_constant__ PcgArgs a) {
  __shared__ double cred[8], bcast[4];
  ClusterSync sy{cluster_rank(), cluster_size(), cred, bcast, 0, 0ull, a.budget_ns, false};
  pcg_body<MODE, PCG_OPS_CSR, FORM>(a, sy.rank, sy);
  cluster_sync_all();
}

// A batch of independent systems in one cooperative launch: system k owns the blocks
// [start[k], start[k+1]), with the block count its single solve would use, so that its tile plan,
// its reductions and therefore its result are bit-identical to solving it alone.  Every system has
// its own workspace, barrier counters, deadline and status.
struct PcgBatch {
  PcgArgs sys[NGS_PCG_BATCH_MAX];
  unsigned int start[NGS_PCG_BATCH_MAX + 1];
  int nsys;
};
static_assert(sizeof(PcgBatch) <= 32000, "batch arguments must fit the kernel parameter space");

template <int MODE, int OPS>
__global__ void __launch_bounds__(PCG_THREADS, PCG_MIN_BLOCKS) pcg_batch_kernel(const __grid_constant__ PcgBatch b) {
  int lo = 0, hi = b.nsys - 1;              // last system whose first block is <= blockIdx.x
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (b.start[mid] <= blockIdx.x) lo = mid; else hi = mid - 1;
  }
  GridSync sy(b.sys[lo], blockIdx.x - b.start[lo]);
  pcg_body<MODE, OPS, PCG_FORM_ANY>(b.sys[lo], blockIdx.x - b.start[lo], sy);
}

static size_t align_up(size_t v) { return (v + 255) & ~(size_t)255; }

// Element sizes of a mode's workspace vectors: search vectors (p, s, u, w) and residual r.  The one
// definition that both the size query and the carve-up use.
static size_t pcg_vec_bytes(int mode) { return mode == NGS_PCG_FP64 ? 8 : 4; }
static size_t pcg_res_bytes(int mode) { return mode == NGS_PCG_REFERENCE ? 4 : 8; }

extern "C" size_t ngs_pcg_workspace_bytes(int64_t n, int mode) {
  const size_t vt = pcg_vec_bytes(mode);
  const size_t rt = pcg_res_bytes(mode);
  size_t bytes = align_up(n * rt) + 4 * align_up(n * vt);     // r, p, s, u, w
  bytes += align_up(PCG_PARTIALS_BYTES);                        // partials, double-buffered
  bytes += align_up(4 * sizeof(double)) + align_up(8 * sizeof(unsigned int));
  return bytes;
}

// Co-resident blocks of the cooperative kernels on the current device: the fewest over every
// instantiation a solve of this mode may launch (single, batched; CSR, matrix-free, both).
// A PCG kernel runs with PCG_WIN_BYTES of dynamic shared memory (the vector window) or none; the
// occupancy queries assume the window, so that the capacity holds for either launch.  The attribute
// is set by those queries (the capacity of the cooperative kernels, the cluster limit of the cluster
// kernels), which are cached per device and which every launch path calls before it launches.
static void pcg_smem_attr(const void* f) {
  cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, PCG_WIN_BYTES);
}

static int pcg_occupancy(const void* f) {
  int v = 0;
  pcg_smem_attr(f);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, f, PCG_THREADS, PCG_WIN_BYTES) != cudaSuccess) v = 0;
  return v;
}

// Cached per device (the occupancy queries and attribute settings behind it cost tens of
// microseconds of host time, and every solve asks).
template <int MODE>
static int pcg_capacity() {
  static int cached[64];
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  if (dev >= 0 && dev < 64 && cached[dev] > 0) return cached[dev];
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  int per_sm = pcg_occupancy((const void*)pcg_kernel<MODE, PCG_OPS_CSR>);
  per_sm = std::min(per_sm, pcg_occupancy((const void*)pcg_batch_kernel<MODE, PCG_OPS_CSR>));
  if constexpr (MODE != NGS_PCG_REFERENCE) {
    per_sm = std::min(per_sm, pcg_occupancy((const void*)pcg_form_kernel<MODE, PCG_FORM_DELTA_STREAM>));
    per_sm = std::min(per_sm, pcg_occupancy((const void*)pcg_form_kernel<MODE, PCG_FORM_DELTA>));
    per_sm = std::min(per_sm, pcg_occupancy((const void*)pcg_form_kernel<MODE, PCG_FORM_COLS_STREAM>));
    per_sm = std::min(per_sm, pcg_occupancy((const void*)pcg_form_kernel<MODE, PCG_FORM_COLS>));
    per_sm = std::min(per_sm, pcg_occupancy((const void*)pcg_kernel<MODE, PCG_OPS_MF>));
    per_sm = std::min(per_sm, pcg_occupancy((const void*)pcg_batch_kernel<MODE, PCG_OPS_MF>));
    per_sm = std::min(per_sm, pcg_occupancy((const void*)pcg_batch_kernel<MODE, PCG_OPS_BOTH>));
  }
  const int64_t cap = (int64_t)sms * per_sm;
  const int out = (int)(cap < PCG_MAX_BLOCKS ? cap : PCG_MAX_BLOCKS);   // the partials area holds this many
  if (dev >= 0 && dev < 64 && out > 0) cached[dev] = out;
  return out;
}

// Blocks one solve uses: as many co-resident blocks as fit, fewer for small systems (about
// PCG_BLOCK_WORK non-zeros each, so that an iteration's critical path stays short).
static int64_t pcg_blocks_for(int64_t n, int64_t nnz, int blocks_req, int capacity) {
  int64_t blocks = capacity;
  const int64_t need = (nnz + (int64_t)PCG_ROW_COST * n + PCG_BLOCK_WORK - 1) / PCG_BLOCK_WORK;
  if (blocks > need) blocks = need > 0 ? need : 1;
  if (blocks_req > 0 && blocks_req < blocks) blocks = blocks_req;
  return blocks < 1 ? 0 : blocks;
}

static int capacity_of(int mode) {
  if (mode == NGS_PCG_REFERENCE) return pcg_capacity<NGS_PCG_REFERENCE>();
  if (mode == NGS_PCG_MIXED) return pcg_capacity<NGS_PCG_MIXED>();
  return pcg_capacity<NGS_PCG_FP64>();
}

extern "C" int ngs_pcg_block_capacity(int mode) {
  if (mode < NGS_PCG_REFERENCE || mode > NGS_PCG_FP64) return 0;
  return capacity_of(mode);
}

// Largest cluster of pcg_cluster_kernel<MODE, *> the current device can run (cached per device): the
// smaller of the CSR and the matrix-free instantiation.
static int pcg_cluster_limit_of_kernel(const void* f) {
  int limit = 0;
  pcg_smem_attr(f);
  if (cudaFuncSetAttribute(f, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) == cudaSuccess) {
    cudaLaunchConfig_t lc = {};
    lc.gridDim = dim3(PCG_CLUSTER_MAX);
    lc.blockDim = dim3(PCG_THREADS);
    lc.dynamicSmemBytes = PCG_WIN_BYTES;
    cudaLaunchAttribute attr;
    attr.id = cudaLaunchAttributeClusterDimension;
    attr.val.clusterDim.x = PCG_CLUSTER_MAX;
    attr.val.clusterDim.y = 1;
    attr.val.clusterDim.z = 1;
    lc.attrs = &attr;
    lc.numAttrs = 1;
    if (cudaOccupancyMaxPotentialClusterSize(&limit, f, &lc) != cudaSuccess) limit = 0;
  }
  cudaGetLastError();   // a refused query leaves no sticky error: the cooperative path is used instead
  return limit;
}

template <int MODE>
static int pcg_cluster_limit() {
  static int cached[64];
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 0 && dev < 64 && cached[dev] != 0) return cached[dev] > 0 ? cached[dev] : 0;
  int limit = pcg_cluster_limit_of_kernel((const void*)pcg_cluster_kernel<MODE, PCG_OPS_CSR>);
  if constexpr (MODE != NGS_PCG_REFERENCE) {
    limit = std::min(limit, pcg_cluster_limit_of_kernel((const void*)pcg_cluster_kernel<MODE, PCG_OPS_MF>));
    limit = std::min(limit, pcg_cluster_limit_of_kernel((const void*)pcg_cluster_form_kernel<MODE, PCG_FORM_DELTA>));
    limit = std::min(limit, pcg_cluster_limit_of_kernel((const void*)pcg_cluster_form_kernel<MODE, PCG_FORM_COLS>));
  }
  if (limit > PCG_CLUSTER_MAX) limit = PCG_CLUSTER_MAX;
  if (dev >= 0 && dev < 64) cached[dev] = limit > 0 ? limit : -1;
  return limit;
}

static int cluster_limit_of(int mode) {
  if (mode == NGS_PCG_REFERENCE) return pcg_cluster_limit<NGS_PCG_REFERENCE>();
  if (mode == NGS_PCG_MIXED) return pcg_cluster_limit<NGS_PCG_MIXED>();
  return pcg_cluster_limit<NGS_PCG_FP64>();
}

// CTAs of the cluster that solves a system of this size, or 0 for the cooperative grid path: a
// system of at most PCG_CLUSTER_NEED blocks' work goes to one cluster of up to PCG_CLUSTER_MAX CTAs
// (unless the caller asked for a block count).
static int pcg_cluster_for(int64_t n, int64_t nnz, int blocks_req, int limit) {
  if (blocks_req > 0 || limit < 1) return 0;
  const int64_t need = (nnz + (int64_t)PCG_ROW_COST * n + PCG_BLOCK_WORK - 1) / PCG_BLOCK_WORK;
  if (need > PCG_CLUSTER_NEED) return 0;
  return (int)(need < 1 ? 1 : (need < limit ? need : limit));
}

extern "C" int ngs_pcg_cluster_size(int64_t n, int64_t nnz, int mode) {
  if (mode < NGS_PCG_REFERENCE || mode > NGS_PCG_FP64 || n <= 0) return 0;
  return pcg_cluster_for(n, nnz, 0, cluster_limit_of(mode));
}

static void pcg_set_window(PcgArgs& a, int mode, int64_t band, int64_t nblocks);

// Whether a solo solve of such a system stages its search vector in shared memory (the same decision
// as ngs_pcg_solve), so that a caller builds 2-byte column deltas only where they are read.
extern "C" int ngs_pcg_window(int64_t n, int64_t nnz, int64_t band, int mode) {
  if (mode < NGS_PCG_REFERENCE || mode > NGS_PCG_FP64 || n <= 0 || nnz < 0 || band <= 0) return 0;
  const int csize = ngs_pcg_cluster_size(n, nnz, mode);
  const int64_t blocks = csize > 0 ? csize : pcg_blocks_for(n, nnz, 0, capacity_of(mode));
  if (blocks < 1) return 0;
  PcgArgs a{};
  a.n = n;
  a.nnz = nnz;
  pcg_set_window(a, mode, band, blocks);
  return a.win_cap > 0 ? 1 : 0;
}

extern "C" int ngs_pcg_blocks(int64_t n, int64_t nnz, int mode) {
  if (mode < NGS_PCG_REFERENCE || mode > NGS_PCG_FP64 || n <= 0) return 0;
  if (ngs_pcg_cluster_size(n, nnz, mode) > 0) return 0;      // solved by a cluster, outside the grid
  return (int)pcg_blocks_for(n, nnz, 0, capacity_of(mode));
}

static void* pcg_cluster_kernel_of(int mode, bool mf) {
  if (mode == NGS_PCG_REFERENCE) return (void*)pcg_cluster_kernel<NGS_PCG_REFERENCE, PCG_OPS_CSR>;
  if (mode == NGS_PCG_MIXED)
    return mf ? (void*)pcg_cluster_kernel<NGS_PCG_MIXED, PCG_OPS_MF> : (void*)pcg_cluster_kernel<NGS_PCG_MIXED, PCG_OPS_CSR>;
  return mf ? (void*)pcg_cluster_kernel<NGS_PCG_FP64, PCG_OPS_MF> : (void*)pcg_cluster_kernel<NGS_PCG_FP64, PCG_OPS_CSR>;
}

// Whether the blocks of a system stage their slice of the search vector in shared memory (the
// window): only when the caller bounded the bandwidth and every block's column range fits, rows per
// block + 2 band.  A launch whose systems take no window reserves no shared memory for it, so that
// the space stays with the L1 cache the gathers hit: a window reserved for blocks that cannot use it
// cost 7 % of the level-0 solve of a 300k-point cloud (half of its blocks do not fit) and 9 % on a
// 5M-point room.
// The column encoding follows: with the window, the 2-byte deltas in the software-pipelined row loop
// (level 1 of a 300k-point cloud: 3.51 against 3.76 ms with 4-byte columns); without it, the 4-byte
// columns in the row-at-a-time loop when the caller supplied both (its level 0: 9.22 against 9.34
// ms).  Solo and batched solves of a system take the same decision, so their results stay identical.
static void pcg_set_window(PcgArgs& a, int mode, int64_t band, int64_t nblocks) {
  const int64_t cap = PCG_WIN_BYTES / (int64_t)pcg_vec_bytes(mode);
  const int64_t rows = nblocks > 0 ? (a.n + nblocks - 1) / nblocks : a.n;
  a.win_cap = (!a.mf && band > 0 && rows + 2 * band <= cap) ? (int)cap : 0;
  if (a.win_cap == 0 && a.cols && a.cols16) {
    a.cols16 = nullptr;
    a.evict_first = (size_t)a.nnz * (4 + (mode == NGS_PCG_FP64 ? 8 : 4)) > (size_t)96 << 20;
  }
}

static size_t pcg_win_smem(const PcgArgs& a) { return a.win_cap > 0 ? PCG_WIN_BYTES : 0; }

// One cluster of `csize` CTAs solves the system (an ordinary launch: the hardware places the whole
// cluster at once, so the cluster barrier needs no cooperative launch).
static int launch_cluster(PcgArgs& a, int mode, int csize, cudaStream_t st) {
  a.nblocks = (unsigned int)csize;
  cudaMemsetAsync(a.count, 0, 8 * sizeof(unsigned int), st);
  cudaLaunchConfig_t lc = {};
  lc.gridDim = dim3((unsigned)csize);
  lc.blockDim = dim3(PCG_THREADS);
  lc.dynamicSmemBytes = pcg_win_smem(a);
  lc.stream = st;
  cudaLaunchAttribute attr;
  attr.id = cudaLaunchAttributeClusterDimension;
  attr.val.clusterDim.x = (unsigned)csize;
  attr.val.clusterDim.y = 1;
  attr.val.clusterDim.z = 1;
  lc.attrs = &attr;
  lc.numAttrs = 1;
  void* args[] = {&a};
  ngs_count_launch();
  const void* f = pcg_cluster_kernel_of(mode, a.mf != 0);
  if (!a.mf && !a.evict_first && (mode == NGS_PCG_MIXED || mode == NGS_PCG_FP64)) {
    if (mode == NGS_PCG_MIXED)
      f = a.cols16 ? (const void*)pcg_cluster_form_kernel<NGS_PCG_MIXED, PCG_FORM_DELTA>
                   : (const void*)pcg_cluster_form_kernel<NGS_PCG_MIXED, PCG_FORM_COLS>;
    else
      f = a.cols16 ? (const void*)pcg_cluster_form_kernel<NGS_PCG_FP64, PCG_FORM_DELTA>
                   : (const void*)pcg_cluster_form_kernel<NGS_PCG_FP64, PCG_FORM_COLS>;
  }
  const cudaError_t e = cudaLaunchKernelExC(&lc, f, args);
  if (e != cudaSuccess) return ngs_set_cuda_error(e);
  return NGS_OK;
}

// Zero a system's status record: the kernel's status writes are maxima over it, and an empty system
// (nothing to launch) reports 0 iterations, NGS_OK.
static void pcg_clear_status(int64_t* info_dev, double* resid_dev, cudaStream_t st) {
  cudaMemsetAsync(info_dev, 0, 4 * sizeof(int64_t), st);
  cudaMemsetAsync(resid_dev, 0, 2 * sizeof(double), st);
}

// Validate one system, carve its workspace and fill the kernel arguments (nblocks left 0).
// Returns NGS_OK, an error, or 1 for an empty system (nothing to launch).  Touches no device memory.
static int prepare_pcg(const ngs_pcg_system* sys, const ngs_pcg_config* cfg, void* ws, size_t ws_bytes,
                       int64_t* info_dev, double* resid_dev, cudaStream_t st, PcgArgs& a) {
  if (!sys || !cfg || !info_dev || !resid_dev || sys->n < 0 || !sys->inv_diag) return NGS_ERR_INVALID_ARG;
  const int mode = cfg->mode;
  if (mode < NGS_PCG_REFERENCE || mode > NGS_PCG_FP64) return NGS_ERR_INVALID_ARG;
  const ngs_pcg_operator* op = sys->op;
  if (op) {
    // matrix-free: MIXED and FP64 modes; no CSR is read
    if (mode == NGS_PCG_REFERENCE || op->n_points < 0 || op->n_points > (int64_t)0x7fffffff || sys->nnz < 0 ||
        (sys->n > 0 && (!op->coords || !op->stencil || !op->t_ptr || !op->grid.words)) ||
        (op->n_points > 0 && (!op->point_rows || !op->point_phi || !op->t_point || !op->t_phi || !op->scratch64 ||
                              (mode == NGS_PCG_MIXED && !op->scratch32))) ||
        !sys->b64 || !sys->x64)
      return NGS_ERR_INVALID_ARG;
  } else {
    if (!sys->rowptr || (sys->nnz > 0 && !sys->cols && !sys->col_delta)) return NGS_ERR_INVALID_ARG;
    if (mode == NGS_PCG_REFERENCE && (!sys->vals32 || !sys->b32 || !sys->x32)) return NGS_ERR_INVALID_ARG;
    if (mode == NGS_PCG_MIXED && (!sys->vals32 || !sys->vals64 || !sys->b64 || !sys->x64)) return NGS_ERR_INVALID_ARG;
    if (mode == NGS_PCG_FP64 && (!sys->vals64 || !sys->b64 || !sys->x64)) return NGS_ERR_INVALID_ARG;
  }
  if (!ws || ws_bytes < ngs_pcg_workspace_bytes(sys->n, mode)) return NGS_ERR_OOM;
  const int64_t n = sys->n;
  if (n == 0) return 1;
  const size_t vt = pcg_vec_bytes(mode);
  const size_t rt = pcg_res_bytes(mode);
  char* base = static_cast<char*>(ws);
  a = PcgArgs{};
  a.n = n;
  a.nnz = sys->nnz;
  a.rowptr = sys->rowptr;
  a.cols = sys->cols;
  a.cols16 = sys->col_delta;
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
  a.partials = reinterpret_cast<double*>(base); base += align_up(PCG_PARTIALS_BYTES);
  unsigned int* ctl = reinterpret_cast<unsigned int*>(base);
  a.count = ctl;
  a.error = reinterpret_cast<int*>(ctl + 2);
  a.deadline = reinterpret_cast<unsigned long long*>(ctl + 4);
  a.info = info_dev;
  a.resid = resid_dev;
  a.tol = cfg->tol;
  a.max_iter = cfg->max_iter;
  a.replace_every = mode == NGS_PCG_REFERENCE ? (cfg->res_fix ? 1 : 0) : cfg->replace_every;
  const double timeout = cfg->timeout_s > 0 ? cfg->timeout_s : 10.0;
  a.wait_ns = (unsigned long long)(timeout * 1e9);
  a.budget_ns = a.wait_ns;
  a.inner_rtol = 1.0e-4;
  a.win_cap = 0;                       // decided with the block count (pcg_set_window)
  const size_t mat_bytes = (size_t)sys->nnz * ((sys->col_delta ? 2 : 4) + (mode == NGS_PCG_FP64 ? 8 : 4));
  a.evict_first = mat_bytes > (size_t)96 << 20;
  if (op) {
    a.mf = 1;
    a.op = *op;
    a.rowptr = nullptr;
    a.cols = nullptr;
    a.cols16 = nullptr;
    a.evict_first = 0;
  }
  return NGS_OK;
}

// The single-system kernel of an assembled matrix in the MIXED and FP64 modes: the one specialised
// for its SpMV form.
template <int MODE>
static void* pcg_form_kernel_for(const PcgArgs& a) {
  if (a.cols16) return a.evict_first ? (void*)pcg_form_kernel<MODE, PCG_FORM_DELTA_STREAM> : (void*)pcg_form_kernel<MODE, PCG_FORM_DELTA>;
  return a.evict_first ? (void*)pcg_form_kernel<MODE, PCG_FORM_COLS_STREAM> : (void*)pcg_form_kernel<MODE, PCG_FORM_COLS>;
}

static void* pcg_kernel_of(int mode, bool mf) {
  if (mode == NGS_PCG_REFERENCE) return (void*)pcg_kernel<NGS_PCG_REFERENCE, PCG_OPS_CSR>;
  if (mode == NGS_PCG_MIXED)
    return mf ? (void*)pcg_kernel<NGS_PCG_MIXED, PCG_OPS_MF> : (void*)pcg_kernel<NGS_PCG_MIXED, PCG_OPS_CSR>;
  return mf ? (void*)pcg_kernel<NGS_PCG_FP64, PCG_OPS_MF> : (void*)pcg_kernel<NGS_PCG_FP64, PCG_OPS_CSR>;
}

// ops: PCG_OPS_CSR / _MF / _BOTH, from the systems of the batch.
template <int MODE>
static void* pcg_batch_kernel_ops(int ops) {
  if constexpr (MODE == NGS_PCG_REFERENCE) {
    return (void*)pcg_batch_kernel<MODE, PCG_OPS_CSR>;
  } else {
    if (ops == PCG_OPS_MF) return (void*)pcg_batch_kernel<MODE, PCG_OPS_MF>;
    if (ops == PCG_OPS_BOTH) return (void*)pcg_batch_kernel<MODE, PCG_OPS_BOTH>;
    return (void*)pcg_batch_kernel<MODE, PCG_OPS_CSR>;
  }
}

static void* pcg_batch_kernel_of(int mode, int ops) {
  if (mode == NGS_PCG_REFERENCE) return pcg_batch_kernel_ops<NGS_PCG_REFERENCE>(ops);
  if (mode == NGS_PCG_MIXED) return pcg_batch_kernel_ops<NGS_PCG_MIXED>(ops);
  return pcg_batch_kernel_ops<NGS_PCG_FP64>(ops);
}

extern "C" int ngs_pcg_solve(const ngs_pcg_system* sys, const ngs_pcg_config* cfg, void* ws, size_t ws_bytes,
                             int64_t* info_dev, double* resid_dev, ngs_stream s) {
  cudaStream_t st = (cudaStream_t)s;
  PcgArgs a;
  const int rc = prepare_pcg(sys, cfg, ws, ws_bytes, info_dev, resid_dev, st, a);
  if (rc != NGS_OK && rc != 1) return rc;
  pcg_clear_status(info_dev, resid_dev, st);
  if (rc == 1) return NGS_OK;
  const int csize = pcg_cluster_for(a.n, a.nnz, cfg->blocks, cluster_limit_of(cfg->mode));
  if (csize > 0) {
    pcg_set_window(a, cfg->mode, sys->band, csize);
    return launch_cluster(a, cfg->mode, csize, st);
  }
  const int cap = capacity_of(cfg->mode);
  if (cap < 1) return NGS_ERR_CUDA;
  const int64_t blocks = pcg_blocks_for(a.n, a.nnz, cfg->blocks, cap);
  if (blocks < 1) return NGS_ERR_INVALID_ARG;
  a.nblocks = (unsigned int)blocks;
  pcg_set_window(a, cfg->mode, sys->band, blocks);
  cudaMemsetAsync(a.count, 0, 8 * sizeof(unsigned int), st);
  void* args[] = {&a};
  ngs_count_launch();
  void* f = a.mf ? pcg_kernel_of(cfg->mode, true)
             : cfg->mode == NGS_PCG_MIXED ? pcg_form_kernel_for<NGS_PCG_MIXED>(a)
             : cfg->mode == NGS_PCG_FP64 ? pcg_form_kernel_for<NGS_PCG_FP64>(a)
             : pcg_kernel_of(cfg->mode, false);
  const cudaError_t e = cudaLaunchCooperativeKernel(f, dim3((unsigned)blocks), dim3(PCG_THREADS), args, pcg_win_smem(a),
                                                    st);
  if (e != cudaSuccess) return ngs_set_cuda_error(e);
  return NGS_OK;
}

extern "C" int ngs_pcg_solve_batch(const ngs_pcg_batch_item* items, int n_items, ngs_stream s) {
  if (!items || n_items < 0 || n_items > NGS_PCG_BATCH_MAX) return NGS_ERR_INVALID_ARG;
  if (n_items == 0) return NGS_OK;
  cudaStream_t st = (cudaStream_t)s;
  const int mode = items[0].cfg.mode;
  for (int k = 0; k < n_items; k++)
    if (items[k].cfg.mode != mode) return NGS_ERR_INVALID_ARG;
  if (mode < NGS_PCG_REFERENCE || mode > NGS_PCG_FP64) return NGS_ERR_INVALID_ARG;
  const int cap = capacity_of(mode);
  if (cap < 1) return NGS_ERR_CUDA;
  static thread_local PcgBatch b;          // 15 KB: kept off the stack
  static thread_local PcgArgs small[NGS_PCG_BATCH_MAX];
  static thread_local int small_size[NGS_PCG_BATCH_MAX];
  static thread_local int empty[NGS_PCG_BATCH_MAX];
  b.nsys = 0;
  int nsmall = 0, nempty = 0;
  unsigned int total = 0;
  const int climit = cluster_limit_of(mode);
  // validate and size everything before the first memset, so that a rejected batch touches nothing
  for (int k = 0; k < n_items; k++) {
    const ngs_pcg_batch_item& it = items[k];
    PcgArgs a;
    const int rc = prepare_pcg(&it.sys, &it.cfg, it.ws, it.ws_bytes, it.info_dev, it.resid_dev, st, a);
    if (rc == 1) {
      empty[nempty++] = k;
      continue;
    }
    if (rc != NGS_OK) return rc;
    const int csize = pcg_cluster_for(a.n, a.nnz, it.cfg.blocks, climit);
    if (csize > 0) {                         // solved by its own cluster, as it would be alone
      pcg_set_window(a, mode, it.sys.band, csize);
      small[nsmall] = a;
      small_size[nsmall++] = csize;
      continue;
    }
    const int64_t blocks = pcg_blocks_for(a.n, a.nnz, it.cfg.blocks, cap);
    if (blocks < 1) return NGS_ERR_INVALID_ARG;
    if (total + blocks > (unsigned)cap) return NGS_ERR_INVALID_ARG;   // not co-resident: split the batch
    a.nblocks = (unsigned int)blocks;
    pcg_set_window(a, mode, it.sys.band, blocks);       // as it would be alone: the same bits
    b.start[b.nsys] = total;
    b.sys[b.nsys++] = a;
    total += (unsigned)blocks;
  }
  for (int k = 0; k < nempty; k++) pcg_clear_status(items[empty[k]].info_dev, items[empty[k]].resid_dev, st);
  for (int k = 0; k < nsmall; k++) {
    pcg_clear_status(small[k].info, small[k].resid, st);
    const int rc = launch_cluster(small[k], mode, small_size[k], st);
    if (rc != NGS_OK) return rc;
  }
  if (b.nsys == 0) return NGS_OK;
  b.start[b.nsys] = total;
  for (int k = 0; k < b.nsys; k++) {
    pcg_clear_status(b.sys[k].info, b.sys[k].resid, st);
    cudaMemsetAsync(b.sys[k].count, 0, 8 * sizeof(unsigned int), st);
  }
  int ops = 0;
  size_t smem = 0;
  for (int k = 0; k < b.nsys; k++) {
    ops |= b.sys[k].mf ? PCG_OPS_MF : PCG_OPS_CSR;
    smem = std::max(smem, pcg_win_smem(b.sys[k]));
  }
  void* args[] = {&b};
  ngs_count_launch();
  void* f = pcg_batch_kernel_of(mode, ops);
  const cudaError_t e = cudaLaunchCooperativeKernel(f, dim3(total), dim3(PCG_THREADS), args, smem, st);
  if (e != cudaSuccess) return ngs_set_cuda_error(e);
  return NGS_OK;
}

// ----------------------------------------------------------------------------- solve without allocating
// Some callers cannot allocate device memory at the moment they need a solve: code that runs
// inside a host callback or a driver-managed context where cudaMalloc is not permitted, allocators
// that must not be re-entered, or embedded runtimes that hand this library only the buffers they
// own.  For them ngs_pcg_solve_noalloc uses a fixed scratch area that is part of the library image
// itself (a static device array), so the call allocates nothing.  The array is sized for systems of
// up to kNoallocMaxRows rows in the widest (8-byte vector) mode; larger systems are rejected.  Every
// GPU that loads the library keeps this array until the process exits.
static constexpr int64_t kNoallocMaxRows = 131072;
static constexpr size_t noalloc_align(size_t v) { return (v + 255) & ~(size_t)255; }
static constexpr size_t kNoallocScratchBytes =
    noalloc_align(kNoallocMaxRows * 8) + 4 * noalloc_align(kNoallocMaxRows * 8) + noalloc_align(PCG_PARTIALS_BYTES) +
    noalloc_align(4 * sizeof(double)) + noalloc_align(8 * sizeof(unsigned int));
static __device__ __align__(256) unsigned char g_pcg_noalloc_scratch[kNoallocScratchBytes];

// The host cannot use g_pcg_noalloc_scratch as a device address.  Its address belongs to the CUDA
// context that is current, so it is looked up on every call, with that context current (the lookup
// allocates nothing; the first one in a context loads this library's device code into it, which is
// why the first call in each context should come before any stream capture).
static int noalloc_scratch(void** out) {
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_pcg_noalloc_scratch);
  if (e != cudaSuccess) return ngs_set_cuda_error(e);
  *out = p;
  return NGS_OK;
}

extern "C" int64_t ngs_pcg_noalloc_max_rows(void) { return kNoallocMaxRows; }

extern "C" int ngs_pcg_solve_noalloc(const ngs_pcg_system* sys, const ngs_pcg_config* cfg, int64_t* info_dev,
                                     double* resid_dev, ngs_stream s) {
  if (!sys || !cfg || sys->n < 0) return NGS_ERR_INVALID_ARG;
  if (sys->op) return NGS_ERR_INVALID_ARG;                     // assembled (CSR) systems only
  if (sys->n > kNoallocMaxRows) return NGS_ERR_OOM;            // too large for the built-in scratch
  if (ngs_pcg_workspace_bytes(sys->n, cfg->mode) > kNoallocScratchBytes) return NGS_ERR_OOM;
  void* ws = nullptr;
  const int rc = noalloc_scratch(&ws);
  if (rc != NGS_OK) return rc;
  // ngs_pcg_solve clears the control words it needs zeroed (arrival counter, error word, deadline)
  // and the kernel initialises every vector and writes each partial before reading it, so what the
  // previous call left in the shared scratch does not matter.
  return ngs_pcg_solve(sys, cfg, ws, kNoallocScratchBytes, info_dev, resid_dev, s);
}

// ----------------------------------------------------------------------------- 2-byte column deltas
__global__ void col_delta_kernel(const int64_t* __restrict__ rp, const int32_t* __restrict__ cols, int64_t n,
                                 int16_t* __restrict__ out) {
  const int sub = threadIdx.x & 7;
  const int64_t groups = (int64_t)gridDim.x * (blockDim.x / 8);
  for (int64_t row = ngs_gtid() / 8; row < n; row += groups)
    for (int64_t j = rp[row] + sub; j < rp[row + 1]; j += 8) out[j] = (int16_t)(cols[j] - (int32_t)row);
}

extern "C" int ngs_csr_col_delta(const int64_t* rowptr, const int32_t* cols, int64_t n, int16_t* col_delta,
                                 ngs_stream s) {
  if (n < 0 || (n > 0 && (!rowptr || !cols || !col_delta))) return NGS_ERR_INVALID_ARG;
  if (n == 0) return NGS_OK;
  { ngs_count_launch(); col_delta_kernel<<<ngs_blocks(n * 8, 256), 256, 0, (cudaStream_t)s>>>(rowptr, cols, n, col_delta); }
  NGS_CHECK_LAUNCH();
  return NGS_OK;
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
  if (n > 0) { ngs_count_launch(); dot64_kernel<<<ngs_blocks(n, 256, 4), 256, 0, (cudaStream_t)s>>>(a, b, n, out_dev); }
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
