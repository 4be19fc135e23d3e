// The reference's generic sparse ops, kept for callers of jspsr.ext
// (csrc/sparse_op/sparse_product.cu, csrc/integration/ddi.cu, csrc/marching_cubes/primal_mc.cu).
#include "ngs_common.cuh"
#include "hash_table.cuh"

// ----------------------------------------------------------------------------- sparse meshgrid
__global__ void meshgrid_kernel(const int64_t* __restrict__ a0, const int64_t* __restrict__ al,
                                const int64_t* __restrict__ b0, const int64_t* __restrict__ bl,
                                const int64_t* __restrict__ ab0, int64_t np, int64_t* __restrict__ ai,
                                int64_t* __restrict__ bi) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t p = ngs_gtid() >> 5; p < np; p += warps) {
    const int64_t na = al[p], nb = bl[p], tot = na * nb, base = ab0[p];
    for (int64_t t = lane; t < tot; t += 32) {
      const int64_t a = t / nb;
      ai[base + t] = a0[p] + a;
      bi[base + t] = b0[p] + (t - a * nb);
    }
  }
}

extern "C" int ngs_sparse_meshgrid(const int64_t* a_start, const int64_t* a_len, const int64_t* b_start,
                                   const int64_t* b_len, const int64_t* ab_start, int64_t n_points, int64_t* a_inds,
                                   int64_t* b_inds, ngs_stream s) {
  if (n_points < 0 || (n_points > 0 && (!a_start || !a_len || !b_start || !b_len || !ab_start || !a_inds || !b_inds)))
    return NGS_ERR_INVALID_ARG;
  if (n_points == 0) return NGS_OK;
  { ngs_count_launch(); meshgrid_kernel<<<ngs_blocks(n_points * 32, 256), 256, 0, (cudaStream_t)s>>>(a_start, a_len, b_start, b_len,
                                                                              ab_start, n_points, a_inds, b_inds); }
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}

// ----------------------------------------------------------------------------- screened multiplication
NGS_DEV unsigned long long pair_key(int64_t a, int64_t b) {
  unsigned long long h = NGS_FNV_BASIS;
  h = fnv_step(h, (unsigned int)a);
  h = fnv_step(h, (unsigned int)b);
  return fnv_fold(h);
}

NGS_DEV float vmul(const float* av, const float* bv, int dim, int64_t a, int64_t b) {
  if (dim == 1) return av[a] * bv[b];
  return av[a * 3] * bv[b * 3] + av[a * 3 + 1] * bv[b * 3 + 1] + av[a * 3 + 2] * bv[b * 3 + 2];
}

// One warp per point; lanes stride over the point's `a` entries.
__global__ void smult_kernel(const Slot* __restrict__ slots, int64_t mask, const float* __restrict__ av,
                             const float* __restrict__ bv, int dim, const int64_t* __restrict__ ai,
                             const int64_t* __restrict__ bi, const int64_t* __restrict__ a0,
                             const int64_t* __restrict__ al, const int64_t* __restrict__ b0,
                             const int64_t* __restrict__ bl, const float* __restrict__ w, int64_t np,
                             float* __restrict__ res) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t p = ngs_gtid() >> 5; p < np; p += warps) {
    const float wp = w[p];
    for (int64_t a = a0[p] + lane; a < a0[p] + al[p]; a += 32) {
      for (int64_t b = b0[p]; b < b0[p] + bl[p]; b++) {
        const long long pos = table_find_single(slots, mask, pair_key(ai[a], bi[b]));
        if (pos < 0) continue;
        atomicAdd(res + pos, vmul(av, bv, dim, a, b) * wp);
      }
    }
  }
}

__global__ void smult_back_kernel(const Slot* __restrict__ slots, int64_t mask, const float* __restrict__ av,
                                  const float* __restrict__ bv, int dim, const int64_t* __restrict__ ai,
                                  const int64_t* __restrict__ bi, const int64_t* __restrict__ a0,
                                  const int64_t* __restrict__ al, const int64_t* __restrict__ b0,
                                  const int64_t* __restrict__ bl, const float* __restrict__ w, int64_t np,
                                  const float* __restrict__ g, float* __restrict__ ga, float* __restrict__ gb,
                                  float* __restrict__ gw) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t p = ngs_gtid() >> 5; p < np; p += warps) {
    const float wp = w[p];
    float gwp = 0.f;
    for (int64_t a = a0[p] + lane; a < a0[p] + al[p]; a += 32) {
      for (int64_t b = b0[p]; b < b0[p] + bl[p]; b++) {
        const long long pos = table_find_single(slots, mask, pair_key(ai[a], bi[b]));
        if (pos < 0) continue;
        const float gr = g[pos];
        for (int k = 0; k < dim; k++) {
          atomicAdd(ga + a * dim + k, gr * wp * bv[b * dim + k]);
          atomicAdd(gb + b * dim + k, gr * wp * av[a * dim + k]);
        }
        gwp += gr * vmul(av, bv, dim, a, b);
      }
    }
    gwp = warp_sum(gwp);
    if (lane == 0) gw[p] += gwp;
  }
}

extern "C" int ngs_screened_multiplication(const ngs_hash_table* pairs, const float* a_val, const float* b_val,
                                           int val_dim, const int64_t* a_inds, const int64_t* b_inds,
                                           const int64_t* a_start, const int64_t* a_len, const int64_t* b_start,
                                           const int64_t* b_len, const float* weight, int64_t n_points, float* res,
                                           ngs_stream s) {
  if (!pairs || !pairs->slots || (val_dim != 1 && val_dim != 3) || n_points < 0) return NGS_ERR_INVALID_ARG;
  if (n_points == 0) return NGS_OK;
  if (!a_val || !b_val || !a_inds || !b_inds || !a_start || !a_len || !b_start || !b_len || !weight || !res)
    return NGS_ERR_INVALID_ARG;
  { ngs_count_launch(); smult_kernel<<<ngs_blocks(n_points * 32, 256), 256, 0, (cudaStream_t)s>>>(
      static_cast<const Slot*>(pairs->slots), pairs->nslots - 1, a_val, b_val, val_dim, a_inds, b_inds, a_start, a_len,
      b_start, b_len, weight, n_points, res); }
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}

extern "C" int ngs_screened_multiplication_backward(const ngs_hash_table* pairs, const float* a_val, const float* b_val,
                                                    int val_dim, const int64_t* a_inds, const int64_t* b_inds,
                                                    const int64_t* a_start, const int64_t* a_len,
                                                    const int64_t* b_start, const int64_t* b_len, const float* weight,
                                                    int64_t n_points, const float* grad_res, float* grad_a,
                                                    float* grad_b, float* grad_w, ngs_stream s) {
  if (!pairs || !pairs->slots || (val_dim != 1 && val_dim != 3) || n_points < 0) return NGS_ERR_INVALID_ARG;
  if (n_points == 0) return NGS_OK;
  if (!a_val || !b_val || !a_inds || !b_inds || !a_start || !a_len || !b_start || !b_len || !weight || !grad_res ||
      !grad_a || !grad_b || !grad_w)
    return NGS_ERR_INVALID_ARG;
  { ngs_count_launch(); smult_back_kernel<<<ngs_blocks(n_points * 32, 256), 256, 0, (cudaStream_t)s>>>(
      static_cast<const Slot*>(pairs->slots), pairs->nslots - 1, a_val, b_val, val_dim, a_inds, b_inds, a_start, a_len,
      b_start, b_len, weight, n_points, grad_res, grad_a, grad_b, grad_w); }
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}

// ----------------------------------------------------------------------------- learned-basis integrals
// p[P,v] = sum_{s,t} src[P, 3s+v] tgt[P, 3t+v] ff[s, t, r_v]; q likewise with dfdf.
// One thread per (pair, axis); the C x C tables of the axis' offset are read from L1/L2.
template <int CMAX>
__global__ void ddi_fwd_kernel(const float* __restrict__ src, const float* __restrict__ tgt,
                               const int64_t* __restrict__ rel, const float* __restrict__ ff,
                               const float* __restrict__ dd, int64_t np, int C, int R, float* __restrict__ p,
                               float* __restrict__ q) {
  const int64_t total = np * 3;
  for (int64_t t = ngs_gtid(); t < total; t += ngs_gstride()) {
    const int64_t pr = t / 3;
    const int v = (int)(t - pr * 3);
    const int r = (int)rel[pr * 3 + v];
    float cs[CMAX], ct[CMAX];
    for (int k = 0; k < C; k++) {
      cs[k] = src[pr * 3 * C + 3 * k + v];
      ct[k] = tgt[pr * 3 * C + 3 * k + v];
    }
    float pv = 0.f, qv = 0.f;
    for (int si = 0; si < C; si++) {
      float fp = 0.f, fq = 0.f;
      for (int ti = 0; ti < C; ti++) {
        const int64_t o = ((int64_t)si * C + ti) * R + r;
        fp += __ldg(ff + o) * ct[ti];
        fq += __ldg(dd + o) * ct[ti];
      }
      pv += cs[si] * fp;
      qv += cs[si] * fq;
    }
    p[t] = pv;
    q[t] = qv;
  }
}

template <int CMAX>
__global__ void ddi_bwd_kernel(const float* __restrict__ src, const float* __restrict__ tgt,
                               const int64_t* __restrict__ rel, const float* __restrict__ ff,
                               const float* __restrict__ dd, const float* __restrict__ gp,
                               const float* __restrict__ gq, int64_t np, int C, int R, float* __restrict__ gs,
                               float* __restrict__ gt) {
  const int64_t total = np * 3;
  for (int64_t t = ngs_gtid(); t < total; t += ngs_gstride()) {
    const int64_t pr = t / 3;
    const int v = (int)(t - pr * 3);
    const int r = (int)rel[pr * 3 + v];
    const float a = gp[t], b = gq[t];
    float cs[CMAX], ct[CMAX], acc_t[CMAX];
    for (int k = 0; k < C; k++) {
      cs[k] = src[pr * 3 * C + 3 * k + v];
      ct[k] = tgt[pr * 3 * C + 3 * k + v];
      acc_t[k] = 0.f;
    }
    for (int si = 0; si < C; si++) {
      float accs = 0.f;
      for (int ti = 0; ti < C; ti++) {
        const int64_t o = ((int64_t)si * C + ti) * R + r;
        const float m = a * __ldg(ff + o) + b * __ldg(dd + o);
        accs += m * ct[ti];
        acc_t[ti] += m * cs[si];
      }
      gs[pr * 3 * C + 3 * si + v] = accs;
    }
    for (int k = 0; k < C; k++) gt[pr * 3 * C + 3 * k + v] = acc_t[k];
  }
}

extern "C" int ngs_ddi_forward(const float* src, const float* tgt, const int64_t* rel_pos, const float* ff,
                               const float* dfdf, int64_t n_pairs, int C, int R, float* p, float* q, ngs_stream s) {
  if (n_pairs < 0 || C < 1 || C > 32 || R < 1) return NGS_ERR_INVALID_ARG;
  if (n_pairs == 0) return NGS_OK;
  if (!src || !tgt || !rel_pos || !ff || !dfdf || !p || !q) return NGS_ERR_INVALID_ARG;
  { ngs_count_launch(); ddi_fwd_kernel<32><<<ngs_blocks(n_pairs * 3, 128), 128, 0, (cudaStream_t)s>>>(src, tgt, rel_pos, ff, dfdf, n_pairs,
                                                                              C, R, p, q); }
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}

extern "C" int ngs_ddi_backward(const float* src, const float* tgt, const int64_t* rel_pos, const float* ff,
                                const float* dfdf, const float* grad_p, const float* grad_q, int64_t n_pairs, int C,
                                int R, float* grad_src, float* grad_tgt, ngs_stream s) {
  if (n_pairs < 0 || C < 1 || C > 32 || R < 1) return NGS_ERR_INVALID_ARG;
  if (n_pairs == 0) return NGS_OK;
  if (!src || !tgt || !rel_pos || !ff || !dfdf || !grad_p || !grad_q || !grad_src || !grad_tgt)
    return NGS_ERR_INVALID_ARG;
  { ngs_count_launch(); ddi_bwd_kernel<32><<<ngs_blocks(n_pairs * 3, 128), 128, 0, (cudaStream_t)s>>>(src, tgt, rel_pos, ff, dfdf, grad_p,
                                                                              grad_q, n_pairs, C, R, grad_src, grad_tgt); }
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}

// ----------------------------------------------------------------------------- primal sparse MC
// (primal_mc.cu:20-235): cubes of r^3 sub-cells with (r+1)^3 samples each.
__constant__ signed char p_tri[256][16] = {
#include "mc_tables.inc"
};
__constant__ int p_edge[12][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {4, 5}, {5, 6},
                                  {6, 7}, {7, 4}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};
__constant__ int p_corner[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0},
                                   {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};

NGS_DEV float p_interp(const float* p1, const float* p2, float v1, float v2, float* out) {
  if (fabsf(v1) < 1.0e-5f) { out[0] = p1[0]; out[1] = p1[1]; out[2] = p1[2]; return 1.f; }
  if (fabsf(v2) < 1.0e-5f) { out[0] = p2[0]; out[1] = p2[1]; out[2] = p2[2]; return 0.f; }
  if (fabsf(v1 - v2) < 1.0e-5f) { out[0] = p1[0]; out[1] = p1[1]; out[2] = p1[2]; return 1.f; }
  const float w2 = (0.0f - v1) / (v2 - v1);
  const float w1 = 1.f - w2;
#pragma unroll
  for (int a = 0; a < 3; a++) out[a] = p1[a] * w1 + p2[a] * w2;
  return w1;
}

NGS_DEV void primal_corners(const float* sdf, int64_t cube, int r, int rx, int ry, int rz, float* v) {
  const int r1 = r + 1;
#pragma unroll
  for (int i = 0; i < 8; i++)
    v[i] = sdf[((cube * r1 + rx + p_corner[i][0]) * r1 + ry + p_corner[i][1]) * r1 + rz + p_corner[i][2]];
}

__global__ void primal_count_kernel(const float* __restrict__ sdf, int64_t n, int r, int32_t* __restrict__ vcount) {
  const int64_t r3 = (int64_t)r * r * r, total = n * r3;
  for (int64_t t = ngs_gtid(); t < total; t += ngs_gstride()) {
    const int64_t c = t / r3;
    const int sub = (int)(t - c * r3);
    float v[8];
    primal_corners(sdf, c, r, sub / (r * r), (sub / r) % r, sub % r, v);
    int type = 0;
    for (int i = 0; i < 8; i++) type |= (v[i] < 0.f ? 1 : 0) << i;
    int nv = 0;
    while (nv < 16 && p_tri[type][nv] >= 0) nv++;
    vcount[t] = nv;
  }
}

__global__ void primal_emit_kernel(const float* __restrict__ base, const float* __restrict__ sdf, int64_t n, int r,
                                   const int64_t* __restrict__ voff, float* __restrict__ tris,
                                   int32_t* __restrict__ vids, int32_t* __restrict__ sids, float* __restrict__ sw) {
  const int64_t r3 = (int64_t)r * r * r, total = n * r3;
  const int r1 = r + 1;
  const float sbs = 1.0f / (float)r;
  for (int64_t t = ngs_gtid(); t < total; t += ngs_gstride()) {
    const int64_t c = t / r3;
    const int sub = (int)(t - c * r3);
    const int rx = sub / (r * r), ry = (sub / r) % r, rz = sub % r;
    float v[8];
    primal_corners(sdf, c, r, rx, ry, rz, v);
    int type = 0;
    for (int i = 0; i < 8; i++) type |= (v[i] < 0.f ? 1 : 0) << i;
    const float bx = base[c * 3], by = base[c * 3 + 1], bz = base[c * 3 + 2];
    const int64_t o0 = voff[t];
    for (int k = 0; k < 16 && p_tri[type][k] >= 0; k++) {
      const int e = p_tri[type][k];
      const int a = p_edge[e][0], b = p_edge[e][1];
      const float p1[3] = {bx + (float)(rx + p_corner[a][0]) * sbs, by + (float)(ry + p_corner[a][1]) * sbs,
                           bz + (float)(rz + p_corner[a][2]) * sbs};
      const float p2[3] = {bx + (float)(rx + p_corner[b][0]) * sbs, by + (float)(ry + p_corner[b][1]) * sbs,
                           bz + (float)(rz + p_corner[b][2]) * sbs};
      float out[3];
      const float w1 = p_interp(p1, p2, v[a], v[b], out);
      const int64_t o = o0 + k;
      tris[o * 3] = out[0];
      tris[o * 3 + 1] = out[1];
      tris[o * 3 + 2] = out[2];
      int mn[3], axis = 0;
      for (int ax = 0; ax < 3; ax++) {
        mn[ax] = min(p_corner[a][ax], p_corner[b][ax]);
        if (p_corner[a][ax] != p_corner[b][ax]) axis = ax;
      }
      vids[o * 4] = (int)bx * r + rx + mn[0];
      vids[o * 4 + 1] = (int)by * r + ry + mn[1];
      vids[o * 4 + 2] = (int)bz * r + rz + mn[2];
      vids[o * 4 + 3] = axis;
      sids[o * 2] = (int32_t)(c * r1 * r1 * r1 + ((rx + p_corner[a][0]) * r1 + ry + p_corner[a][1]) * r1 + rz +
                              p_corner[a][2]);
      sids[o * 2 + 1] = (int32_t)(c * r1 * r1 * r1 + ((rx + p_corner[b][0]) * r1 + ry + p_corner[b][1]) * r1 + rz +
                                  p_corner[b][2]);
      sw[o] = w1;
    }
  }
}

extern "C" int ngs_primal_mc_count(const float* sdf, int64_t n_cubes, int r, int32_t* vcount, ngs_stream s) {
  if (n_cubes < 0 || r < 1 || (n_cubes > 0 && (!sdf || !vcount))) return NGS_ERR_INVALID_ARG;
  if (n_cubes == 0) return NGS_OK;
  { ngs_count_launch(); primal_count_kernel<<<ngs_blocks(n_cubes * r * r * r, 256), 256, 0, (cudaStream_t)s>>>(sdf, n_cubes, r, vcount); }
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}

extern "C" int ngs_primal_mc_emit(const float* base, const float* sdf, int64_t n_cubes, int r, const int64_t* voffset,
                                  float* tris, int32_t* vert_ids, int32_t* src_ids, float* src_w, ngs_stream s) {
  if (n_cubes < 0 || r < 1) return NGS_ERR_INVALID_ARG;
  if (n_cubes == 0) return NGS_OK;
  if (!base || !sdf || !voffset || !tris || !vert_ids || !src_ids || !src_w) return NGS_ERR_INVALID_ARG;
  { ngs_count_launch(); primal_emit_kernel<<<ngs_blocks(n_cubes * r * r * r, 128), 128, 0, (cudaStream_t)s>>>(base, sdf, n_cubes, r, voffset,
                                                                                       tris, vert_ids, src_ids, src_w); }
  NGS_CHECK_LAUNCH();
  return NGS_OK;
}
