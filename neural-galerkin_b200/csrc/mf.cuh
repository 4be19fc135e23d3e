// Matrix-free application of one level's B-spline Galerkin operator
//     A v = K (*) v + alpha * Phi^T (Phi v)
// (the reference assembles A as a CSR: jspsr/core/reconstructor.py:176-185 with the screening Gram of
// csrc/sparse_op/sparse_product.cu:100-137, and multiplies it in csrc/sparse_solve/solve_pcg.cu).
//
// Why: the same-level stiffness of the B-spline basis depends on the offset between two voxels only
// (125 values), and the screening Gram is a sum of rank-one terms, one per point over its 27
// neighbours.  Per row, the CSR stores ~60 (column, value) pairs and its product gathers ~60 vector
// elements from scattered rows; here the stencil's columns come from the level's rank bitmap (a
// z-run of five cells is one or two 16-byte words, and its present voxels have consecutive rows,
// so a warp of consecutive rows reads contiguous vector elements), and the screening term is two
// passes over the 27 (point, row) pairs of each point: t = Phi v per point, then per row the sum of
// phi * t over the row's own pairs (kept transposed, ascending point index).
#pragma once
#include "ngs_common.cuh"

// t[p] = sum_a phi[p, a] * v[rows[p, a]] for the points p = first, first + step, ... < last, one
// thread per point: its 27 row loads, then its 27 gathers, are independent (all in flight at once);
// the products are summed in TT in slot order.
template <typename VT, typename TT>
NGS_DEV void mf_points(const ngs_pcg_operator& op, const VT* v, TT* t, int64_t first, int64_t last, int64_t step) {
  for (int64_t p = first; p < last; p += step) {
    const int32_t* __restrict__ pr = op.point_rows + p * 27;
    const float* __restrict__ pf = op.point_phi + p * 27;
    int32_t r[27];
#pragma unroll
    for (int a = 0; a < 27; a++) r[a] = __ldg(pr + a);
    TT acc = (TT)0;
#pragma unroll
    for (int a = 0; a < 27; a++)
      if (r[a] >= 0) acc += (TT)__ldg(pf + a) * (TT)v[r[a]];
    t[p] = acc;
  }
}

// (A v)[row] given t = Phi v: the stencil over the 25 (x, y) columns of the row's 5x5x5
// neighbourhood (five z cells each; products in KT, one KT sum per column, columns summed in ACC),
// plus alpha times the row's screening pairs (summed in ACC).
template <typename KT, typename VT, typename TT, typename ACC>
NGS_DEV ACC mf_row(const ngs_pcg_operator& op, const KT* __restrict__ ks, const VT* v, const TT* t, int64_t row) {
  const int s = op.grid.stride;
  const int x = __ldg(op.coords + row * 3), y = __ldg(op.coords + row * 3 + 1), z = __ldg(op.coords + row * 3 + 2);
  ACC acc = (ACC)0;
#pragma unroll 1
  for (int dx = -2; dx <= 2; dx++) {
#pragma unroll
    for (int dy = -2; dy <= 2; dy++) {
      int32_t r[5];
      grid_rows_zrun<5>(op.grid, x + dx * s, y + dy * s, z - 2 * s, r);
      const KT* kk = ks + (dx + 2) * 25 + (dy + 2) * 5;
      KT part = (KT)0;
#pragma unroll
      for (int k = 0; k < 5; k++)
        if (r[k] >= 0) part += kk[k] * (KT)v[r[k]];
      acc += (ACC)part;
    }
  }
  const int64_t e0 = __ldg(op.t_ptr + row), e1 = __ldg(op.t_ptr + row + 1);
  ACC sc = (ACC)0;
  for (int64_t e = e0; e < e1; e++) sc += (ACC)__ldg(op.t_phi + e) * (ACC)t[__ldg(op.t_point + e)];
  return acc + (ACC)op.alpha * sc;
}
