// Builders of the matrix-free level operator (mf.cuh): the point basis transposed per row, the
// Jacobi diagonal, the screening right-hand side from the transposed pairs, and an FP64 product.
//
// The transposed pairs replace the screening Gram that the reference assembles into its LHS
// (jspsr/core/reconstructor.py:181-185, csrc/sparse_op/sparse_product.cu:100-137): a level's Gram
// has as many entries as its stiffness pattern (~60 per row), its point form only 27 per point.
#include "mf.cuh"

__global__ void mf_count_kernel(const int32_t* __restrict__ rows, int64_t total, int32_t* __restrict__ counts) {
  for (int64_t e = ngs_gtid(); e < total; e += ngs_gstride()) {
    const int32_t r = rows[e];
    if (r >= 0) atomicAdd(counts + r, 1);
  }
}

__global__ void mf_max_kernel(const int32_t* __restrict__ counts, int64_t V, int32_t* __restrict__ max_dev) {
  int32_t m = 0;
  for (int64_t i = ngs_gtid(); i < V; i += ngs_gstride()) m = max(m, counts[i]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0 && m > 0) atomicMax(max_dev, m);
}

extern "C" int ngs_mf_count(const int32_t* point_rows, int64_t n_points, int64_t V, int32_t* counts, int32_t* max_dev,
                            ngs_stream s) {
  if (n_points < 0 || V < 0 || (n_points > 0 && !point_rows) || (V > 0 && (!counts || !max_dev)))
    return NGS_ERR_INVALID_ARG;
  if (n_points > 0 && V > 0) {
    ngs_count_launch();
    mf_count_kernel<<<ngs_blocks(n_points * 27, 256), 256, 0, (cudaStream_t)s>>>(point_rows, n_points * 27, counts);
    NGS_CHECK_LAUNCH();
  }
  if (V > 0) {
    ngs_count_launch();
    mf_max_kernel<<<ngs_blocks(V, 256, 8), 256, 0, (cudaStream_t)s>>>(counts, V, max_dev);
    NGS_CHECK_LAUNCH();
  }
  return NGS_OK;
}

// Pairs into their row's range in arrival order (atomic cursor) ...
__global__ void mf_scatter_kernel(const int32_t* __restrict__ rows, const float* __restrict__ phi, int64_t total,
                                  const int64_t* __restrict__ t_ptr, int32_t* __restrict__ cursor,
                                  int32_t* __restrict__ tmp_point, float* __restrict__ tmp_phi) {
  for (int64_t e = ngs_gtid(); e < total; e += ngs_gstride()) {
    const int32_t r = rows[e];
    if (r < 0) continue;
    const int64_t pos = t_ptr[r] + atomicAdd(cursor + r, 1);
    tmp_point[pos] = (int32_t)(e / 27);
    tmp_phi[pos] = phi[e];
  }
}

// ... then each row's pairs ranked by point index (a point occurs at most once per row): eight lanes
// per row (rows hold ~7 pairs on a fine level), every lane counts the smaller indices of its entries.
// The order, and with it every sum over the pairs, is then independent of the atomic arrival order.
__global__ void mf_rank_kernel(const int64_t* __restrict__ t_ptr, int64_t V, const int32_t* __restrict__ tmp_point,
                               const float* __restrict__ tmp_phi, int32_t* __restrict__ t_point,
                               float* __restrict__ t_phi) {
  constexpr int G = 8;
  const int sub = threadIdx.x & (G - 1);
  const int64_t groups = ngs_gstride() / G;
  for (int64_t row = ngs_gtid() / G; row < V; row += groups) {
    const int64_t e0 = t_ptr[row], len = t_ptr[row + 1] - e0;
    for (int64_t j = sub; j < len; j += G) {
      const int32_t pj = tmp_point[e0 + j];
      int64_t rank = 0;
      for (int64_t k = 0; k < len; k++) rank += tmp_point[e0 + k] < pj;
      t_point[e0 + rank] = pj;
      t_phi[e0 + rank] = tmp_phi[e0 + j];
    }
  }
}

extern "C" int ngs_mf_fill(const int32_t* point_rows, const float* point_phi, int64_t n_points, const int64_t* t_ptr,
                           int64_t V, int32_t* cursor, int32_t* tmp_point, float* tmp_phi, int32_t* t_point,
                           float* t_phi, ngs_stream s) {
  if (n_points < 0 || V < 0 || n_points > (int64_t)0x7fffffff ||
      (n_points > 0 && (!point_rows || !point_phi)) ||
      (V > 0 && (!t_ptr || !cursor || !tmp_point || !tmp_phi || !t_point || !t_phi)))
    return NGS_ERR_INVALID_ARG;
  if (n_points == 0 || V == 0) return NGS_OK;
  ngs_count_launch();
  mf_scatter_kernel<<<ngs_blocks(n_points * 27, 256), 256, 0, (cudaStream_t)s>>>(point_rows, point_phi, n_points * 27,
                                                                                t_ptr, cursor, tmp_point, tmp_phi);
  NGS_CHECK_LAUNCH();
  ngs_count_launch();
  mf_rank_kernel<<<ngs_blocks(V * 8, 256), 256, 0, (cudaStream_t)s>>>(t_ptr, V, tmp_point, tmp_phi, t_point, t_phi);
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}

__global__ void mf_diag_kernel(const int64_t* __restrict__ t_ptr, const float* __restrict__ t_phi, int64_t V,
                               double center, double alpha, float* __restrict__ inv_diag) {
  for (int64_t i = ngs_gtid(); i < V; i += ngs_gstride()) {
    double sq = 0.0;
    for (int64_t e = t_ptr[i]; e < t_ptr[i + 1]; e++) {
      const double ph = (double)t_phi[e];
      sq += ph * ph;
    }
    inv_diag[i] = (float)(1.0 / (center + alpha * sq));
  }
}

extern "C" int ngs_mf_diag(const int64_t* t_ptr, const float* t_phi, int64_t V, double stencil_center, double alpha,
                           float* inv_diag, ngs_stream s) {
  if (V < 0 || (V > 0 && (!t_ptr || !t_phi || !inv_diag))) return NGS_ERR_INVALID_ARG;
  if (V == 0) return NGS_OK;
  ngs_count_launch();
  mf_diag_kernel<<<ngs_blocks(V, 256), 256, 0, (cudaStream_t)s>>>(t_ptr, t_phi, V, stencil_center, alpha, inv_diag);
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}

// Screening right-hand side terms (reconstructor.py:142-149 and the screening part of the
// correction, :163-169) in gather form: every row sums its own pairs, no atomics.
__global__ void mf_screen_rhs_kernel(const int64_t* __restrict__ t_ptr, const int32_t* __restrict__ t_point,
                                     const float* __restrict__ t_phi, int64_t V, const float* __restrict__ val,
                                     double scale, double* __restrict__ rhs) {
  for (int64_t i = ngs_gtid(); i < V; i += ngs_gstride()) {
    double acc = 0.0;
    for (int64_t e = t_ptr[i]; e < t_ptr[i + 1]; e++)
      acc += (double)t_phi[e] * (val ? (double)val[t_point[e]] : 1.0);
    rhs[i] += scale * acc;
  }
}

extern "C" int ngs_mf_screen_rhs(const int64_t* t_ptr, const int32_t* t_point, const float* t_phi, int64_t V,
                                 const float* val, double scale, double* rhs, ngs_stream s) {
  if (V < 0 || (V > 0 && (!t_ptr || !t_point || !t_phi || !rhs))) return NGS_ERR_INVALID_ARG;
  if (V == 0) return NGS_OK;
  ngs_count_launch();
  mf_screen_rhs_kernel<<<ngs_blocks(V, 256), 256, 0, (cudaStream_t)s>>>(t_ptr, t_point, t_phi, V, val, scale, rhs);
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}

// y = A x in FP64, outside the solver (tests compare it with the assembled CSR).
__global__ void mf_points64_kernel(const ngs_pcg_operator op, const double* __restrict__ x) {
  mf_points<double, double>(op, x, op.scratch64, ngs_gtid(), op.n_points, ngs_gstride());
}

__global__ void mf_rows64_kernel(const ngs_pcg_operator op, int64_t n, const double* __restrict__ x,
                                 double* __restrict__ y) {
  __shared__ double ks[125];
  for (int k = threadIdx.x; k < 125; k += blockDim.x) ks[k] = op.stencil[k];
  __syncthreads();
  for (int64_t i = ngs_gtid(); i < n; i += ngs_gstride())
    y[i] = mf_row<double, double, double, double>(op, ks, x, op.scratch64, i);
}

extern "C" int ngs_mf_apply64(const ngs_pcg_operator* op, int64_t n, const double* x, double* y, ngs_stream s) {
  if (!op || n < 0 || op->n_points < 0 || (n > 0 && (!x || !y || !op->coords || !op->stencil || !op->t_ptr ||
                                                    !op->grid.words)) ||
      (op->n_points > 0 && (!op->point_rows || !op->point_phi || !op->scratch64)))
    return NGS_ERR_INVALID_ARG;
  if (n == 0) return NGS_OK;
  cudaStream_t st = (cudaStream_t)s;
  if (op->n_points > 0) {
    ngs_count_launch();
    mf_points64_kernel<<<ngs_blocks(op->n_points, 256), 256, 0, st>>>(*op, x);
    NGS_CHECK_LAUNCH();
  }
  ngs_count_launch();
  mf_rows64_kernel<<<ngs_blocks(n, 256), 256, 0, st>>>(*op, n, x, y);
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}

// ----------------------------------------------------------------------------- screening Gram
// The level's screening Gram alpha * sum_p phi_p phi_p^T added into the assembled CSR (ref: the pair
// products of csrc/sparse_op/sparse_product.cu:100-137 summed into the LHS at
// jspsr/core/reconstructor.py:181-185), from the transposed pairs: row i owns its slots, so one warp
// per row adds, for each point p among the row's pairs (in pair order), phi_p(i) * phi_p(j) for the
// point's 27 rows j -- lanes 0..26 hold the point's rows and values; within one point the 27 rows sit
// at 27 distinct stencil offsets from i, so the per-offset sums of the row (shared memory) take no
// atomics, and the order of the sums is fixed.  One add per present slot at the end.
constexpr int MF_GRAM_THREADS = 256;

__global__ void __launch_bounds__(MF_GRAM_THREADS) mf_gram_kernel(
    const int64_t* __restrict__ t_ptr, const int32_t* __restrict__ t_point, const float* __restrict__ t_phi,
    int64_t V, const int32_t* __restrict__ prow, const float* __restrict__ pphi, const uint4* __restrict__ masks,
    const int64_t* __restrict__ rowptr, double scale, double* __restrict__ vals) {
  __shared__ double acc[MF_GRAM_THREADS / 32][125];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t warps = ngs_gstride() >> 5;
  const int ax = lane / 9, ay = (lane / 3) % 3, az = lane % 3;
  for (int64_t i = ngs_gtid() >> 5; i < V; i += warps) {
    for (int o = lane; o < 125; o += 32) acc[w][o] = 0.0;
    __syncwarp();
    const int64_t e0 = t_ptr[i], e1 = t_ptr[i + 1];
    // the row's pairs 32 at a time on the lanes, then two points per step with both points' rows and
    // values in flight together
    for (int64_t base = e0; base < e1; base += 32) {
      const int cnt = (int)min((int64_t)32, e1 - base);
      const int32_t my_p = lane < cnt ? t_point[base + lane] : 0;
      const float my_f = lane < cnt ? t_phi[base + lane] : 0.f;
      for (int q = 0; q < cnt; q += 2) {
        const bool two = q + 1 < cnt;
        const int64_t pa = __shfl_sync(0xffffffffu, my_p, q), pb = __shfl_sync(0xffffffffu, my_p, two ? q + 1 : q);
        const double fa = (double)__shfl_sync(0xffffffffu, my_f, q);
        const double fb = (double)__shfl_sync(0xffffffffu, my_f, two ? q + 1 : q);
        const int32_t ra = lane < 27 ? __ldg(prow + pa * 27 + lane) : -1;
        const float va = lane < 27 ? __ldg(pphi + pa * 27 + lane) : 0.f;
        const int32_t rb = (lane < 27 && two) ? __ldg(prow + pb * 27 + lane) : -1;
        const float vb = (lane < 27 && two) ? __ldg(pphi + pb * 27 + lane) : 0.f;
        const int aa = __ffs((int)__ballot_sync(0xffffffffu, ra == (int32_t)i)) - 1;
        const int ab = __ffs((int)__ballot_sync(0xffffffffu, rb == (int32_t)i)) - 1;
        if (ra >= 0 && aa >= 0) {
          const int o = (ax - aa / 9 + 2) * 25 + (ay - (aa / 3) % 3 + 2) * 5 + (az - aa % 3 + 2);
          acc[w][o] += fa * (double)va;
        }
        __syncwarp();
        if (rb >= 0 && ab >= 0) {
          const int o = (ax - ab / 9 + 2) * 25 + (ay - (ab / 3) % 3 + 2) * 5 + (az - ab % 3 + 2);
          acc[w][o] += fb * (double)vb;
        }
        __syncwarp();
      }
    }
    const uint4 m = masks[i];
    const int64_t base = rowptr[i];
    for (int o = lane; o < 125; o += 32) {
      const unsigned word = o < 32 ? m.x : o < 64 ? m.y : o < 96 ? m.z : m.w;
      if ((word >> (o & 31)) & 1u) vals[base + popc_below(m, o)] += scale * acc[w][o];
    }
    __syncwarp();
  }
}

extern "C" int ngs_mf_gram(const int64_t* t_ptr, const int32_t* t_point, const float* t_phi, int64_t V,
                           const int32_t* point_rows, const float* point_phi, const uint32_t* masks,
                           const int64_t* rowptr, double scale, double* vals, ngs_stream s) {
  if (V < 0 || (V > 0 && (!t_ptr || !t_point || !t_phi || !point_rows || !point_phi || !masks || !rowptr || !vals)))
    return NGS_ERR_INVALID_ARG;
  if (V == 0) return NGS_OK;
  ngs_count_launch();
  mf_gram_kernel<<<ngs_blocks(V * 32, MF_GRAM_THREADS), MF_GRAM_THREADS, 0, (cudaStream_t)s>>>(
      t_ptr, t_point, t_phi, V, point_rows, point_phi, reinterpret_cast<const uint4*>(masks), rowptr, scale, vals);
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}
