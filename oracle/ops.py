"""CPU restatements of the reference's CUDA ops (op-level oracle).

TEST INFRASTRUCTURE ONLY.  These functions follow the semantics of the
pybind11 ops the reference's Python layer calls, on numpy arrays:

* ``hash_cuda`` / ``kernel_hash_cuda``  -- ``csrc/common/hashmap_cuda.cu:204-235,247-339``
* ``build_hash_table`` / ``hash_table_query`` -- ``hashmap_cuda.cu:341-398`` (results, not slots)
* ``screened_multiplication(_backward)`` / ``sparse_meshgrid`` -- ``csrc/sparse_op/sparse_product.cu:19-322``
* ``ddi_forward`` / ``ddi_backward``     -- ``csrc/integration/ddi.cu:21-141``
* ``solve_pcg_diag``                      -- ``csrc/sparse_solve/solve_pcg.cu:15-136``
* ``marching_cubes_sparse``               -- ``csrc/marching_cubes/primal_mc.cu:7-235``
* ``dual_marching_cubes_indices``         -- ``csrc/marching_cubes/dual_mc_inds.cu:45-182``
* ``dual_marching_cubes_sparse``          -- ``csrc/marching_cubes/dual_mc.cu:20-189``
"""
from __future__ import annotations

import numpy as np

from .spsr import fnv60, _octant_slot, _CORNER_AXIS, MC_EDGES, _interp
from .mc_tables import TRI_TABLE, NUM_VERTS_TABLE


def hash_cuda(idx: np.ndarray) -> np.ndarray:
    """FNV-1a-60 over each row of an int[N, D] array, D in {2, 3, 4}."""
    idx = np.asarray(idx)
    return fnv60([idx[:, j] for j in range(idx.shape[1])]).astype(np.int64)


def kernel_hash_cuda(idx: np.ndarray, offsets: np.ndarray) -> np.ndarray:
    """int64[K, N]: hash of (coord + offset_k) (4th column, if any, passed through)."""
    idx = np.asarray(idx).astype(np.int64)
    off = np.asarray(offsets).astype(np.int64)
    cols = [idx[None, :, j] + off[:, None, j] for j in range(3)]
    if idx.shape[1] == 4:
        cols.append(np.broadcast_to(idx[None, :, 3], cols[0].shape))
    return fnv60(cols).astype(np.int64)


class HashTable:
    """Key -> value map standing in for ``HashLookupData``; first inserted key wins."""

    def __init__(self, keys: np.ndarray, vals: np.ndarray | None = None):
        keys = np.asarray(keys).astype(np.int64)
        vals = np.arange(keys.shape[0]) if vals is None or len(vals) == 0 else np.asarray(vals).astype(np.int64)
        self.inserted_size = keys.shape[0]
        u, first = np.unique(keys, return_index=True)
        self.keys, self.vals = u, vals[first]

    def query(self, q: np.ndarray) -> np.ndarray:
        """value + 1 where found, 0 where absent (``hashtable_lookup``, ``hashmap_cuda.cuh:190-204``)."""
        q = np.asarray(q).astype(np.int64)
        if self.keys.shape[0] == 0:
            return np.zeros(q.shape, dtype=np.int64)
        pos = np.clip(np.searchsorted(self.keys, q), 0, self.keys.shape[0] - 1)
        return np.where(self.keys[pos] == q, self.vals[pos] + 1, 0)


def build_hash_table(keys, vals=None, enlarge=False) -> HashTable:
    return HashTable(keys, vals)


def hash_table_query(table: HashTable, q) -> np.ndarray:
    return table.query(q)


def hash2(a, b):
    """Pair key (``hashmap_cuda.cuh:206-214``)."""
    return fnv60([np.asarray(a), np.asarray(b)]).astype(np.int64)


def _segments(lengths):
    lengths = np.asarray(lengths).astype(np.int64)
    start = np.cumsum(lengths) - lengths
    return start, lengths


def _pairs(a_lengths, b_lengths):
    """All (point, a, b) index triples of the per-point meshgrid."""
    a0, al = _segments(a_lengths)
    b0, bl = _segments(b_lengths)
    npair = al * bl
    pt = np.repeat(np.arange(al.shape[0]), npair)
    local = np.arange(pt.shape[0]) - np.repeat(np.cumsum(npair) - npair, npair)
    a = a0[pt] + local // np.maximum(bl[pt], 1)
    b = b0[pt] + local % np.maximum(bl[pt], 1)
    return pt, a, b


def sparse_meshgrid(a_lengths, b_lengths):
    """(a_inds, b_inds) of every per-point pair, point-major then a-major (``sparse_product.cu:52-82``)."""
    _, a, b = _pairs(a_lengths, b_lengths)
    return a, b


def _vmul(a_val, b_val, a, b):
    if a_val.ndim == 1:
        return a_val[a].astype(np.float64) * b_val[b]
    return np.sum(a_val[a].astype(np.float64) * b_val[b], axis=1)


def screened_multiplication(table: HashTable, a_val, b_val, a_inds, b_inds, a_lengths, b_lengths, weight):
    """res[pair] += a_val[a] * b_val[b] * w[p] over per-point pairs (``sparse_product.cu:100-137,202-258``)."""
    pt, a, b = _pairs(a_lengths, b_lengths)
    pos = table.query(hash2(np.asarray(a_inds)[a], np.asarray(b_inds)[b]))
    ok = pos > 0
    val = _vmul(np.asarray(a_val), np.asarray(b_val), a, b) * np.asarray(weight, dtype=np.float64)[pt]
    return np.bincount(pos[ok] - 1, weights=val[ok], minlength=table.inserted_size)


def screened_multiplication_backward(table, a_val, b_val, a_inds, b_inds, a_lengths, b_lengths, weight, grad_res):
    """Gradients w.r.t. a_val, b_val, weight (``sparse_product.cu:159-198,260-322``)."""
    a_val, b_val = np.asarray(a_val, dtype=np.float64), np.asarray(b_val, dtype=np.float64)
    pt, a, b = _pairs(a_lengths, b_lengths)
    pos = table.query(hash2(np.asarray(a_inds)[a], np.asarray(b_inds)[b]))
    ok = pos > 0
    pt, a, b, g = pt[ok], a[ok], b[ok], np.asarray(grad_res, dtype=np.float64)[pos[ok] - 1]
    w = np.asarray(weight, dtype=np.float64)[pt]
    ga, gb = np.zeros_like(a_val), np.zeros_like(b_val)
    if a_val.ndim == 1:
        np.add.at(ga, a, g * w * b_val[b])
        np.add.at(gb, b, g * w * a_val[a])
    else:
        np.add.at(ga, a, (g * w)[:, None] * b_val[b])
        np.add.at(gb, b, (g * w)[:, None] * a_val[a])
    gw = np.bincount(pt, weights=g * _vmul(a_val, b_val, a, b), minlength=np.asarray(weight).shape[0])
    return ga, gb, gw


def ddi_forward(src, tgt, rel_pos, ff, dfdf):
    """Per pair and axis: p = sum_{s,t} c^src_{s,v} c^tgt_{t,v} FF[s,t,r_v] (``ddi.cu:21-76``)."""
    src = np.asarray(src, dtype=np.float64)
    tgt = np.asarray(tgt, dtype=np.float64)
    rel_pos = np.asarray(rel_pos).astype(np.int64)
    C = ff.shape[0]
    p = np.zeros((src.shape[0], 3))
    q = np.zeros((src.shape[0], 3))
    for v in range(3):
        cs = src[:, v::3][:, :C]       # [P, C] coefficient of component s on axis v
        ct = tgt[:, v::3][:, :C]
        tf = np.transpose(ff[:, :, rel_pos[:, v]], (2, 0, 1))    # [P, C, C]
        td = np.transpose(dfdf[:, :, rel_pos[:, v]], (2, 0, 1))
        p[:, v] = np.einsum("ps,pst,pt->p", cs, tf, ct)
        q[:, v] = np.einsum("ps,pst,pt->p", cs, td, ct)
    return p, q


def ddi_backward(src, tgt, rel_pos, ff, dfdf, grad_p, grad_q):
    """Gradients of ``ddi_forward`` w.r.t. both coefficient arrays (``ddi.cu:78-141``)."""
    src = np.asarray(src, dtype=np.float64)
    tgt = np.asarray(tgt, dtype=np.float64)
    rel_pos = np.asarray(rel_pos).astype(np.int64)
    C = ff.shape[0]
    gs = np.zeros_like(src)
    gt = np.zeros_like(tgt)
    for v in range(3):
        cs = src[:, v::3][:, :C]
        ct = tgt[:, v::3][:, :C]
        m = np.transpose(ff[:, :, rel_pos[:, v]], (2, 0, 1)) * np.asarray(grad_p)[:, v, None, None] + \
            np.transpose(dfdf[:, :, rel_pos[:, v]], (2, 0, 1)) * np.asarray(grad_q)[:, v, None, None]
        gs[:, v::3] = np.einsum("pst,pt->ps", m, ct)
        gt[:, v::3] = np.einsum("pst,ps->pt", m, cs)
    return gs, gt


def solve_pcg_diag(ap, aj, ax, b, inv_diag, tol, max_iter, res_fix, dtype=np.float32):
    """Jacobi-PCG exactly as the reference loop (``solve_pcg.cu:15-136``); returns (x, iters)."""
    ap, aj = np.asarray(ap).astype(np.int64), np.asarray(aj).astype(np.int64)
    n = b.shape[0]
    import scipy.sparse as sp
    A = sp.csr_matrix((np.asarray(ax, dtype=dtype), aj, ap), shape=(n, n))
    b = np.asarray(b, dtype=dtype)
    dinv = np.asarray(inv_diag, dtype=dtype)
    sqrt_n = int(np.ceil(np.sqrt(n)))
    atol = tol * np.linalg.norm(b)
    x = np.zeros(n, dtype=dtype)
    r = b - A @ x
    p = np.zeros(n, dtype=dtype)
    rho = dtype(0)
    it = 0
    while max_iter < 0 or it < max_iter:
        z = dinv * r
        rho1 = rho
        rho = dtype(np.dot(r, z))
        p = z.copy() if it == 0 else z + dtype(rho / rho1) * p
        q = (A @ p).astype(dtype)
        alpha = dtype(rho / np.dot(p, q))
        x = x + alpha * p
        if res_fix and (it + 1) % sqrt_n == 0:
            r = b - (A @ x).astype(dtype)
        else:
            r = r - alpha * q
        it += 1
        if np.linalg.norm(r) <= atol:
            break
    return x, it


# ----------------------------------------------------------------------------- marching cubes
_PRIMAL_CORNER = np.array([(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0),
                           (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)], dtype=np.int64)


def marching_cubes_sparse(cube_base, cube_sdf):
    """Primal sparse MC on r^3 sub-cubes (``primal_mc.cu:20-235``).

    Returns tris f32[T,3,3], vert_ids int32[T,3,4], src_ids int32[T,3,2], src_w f32[T,3,1].
    """
    base = np.asarray(cube_base, dtype=np.float32)
    sdf = np.asarray(cube_sdf, dtype=np.float32)
    M, r1 = sdf.shape[0], sdf.shape[1]
    r = r1 - 1
    g = np.stack(np.meshgrid(np.arange(r), np.arange(r), np.arange(r), indexing="ij"), -1).reshape(-1, 3)
    lif = np.repeat(np.arange(M), r ** 3)
    sub = np.tile(g, (M, 1))
    corner = sub[:, None, :] + _PRIMAL_CORNER[None]              # [C, 8, 3]
    vals = sdf[lif[:, None], corner[..., 0], corner[..., 1], corner[..., 2]]
    ctype = np.zeros(vals.shape[0], dtype=np.int64)
    for i in range(8):
        ctype |= (vals[:, i] < 0).astype(np.int64) << i
    sbs = np.float32(1.0) / np.float32(r)
    pts = base[lif][:, None, :] + corner.astype(np.float32) * sbs   # float32 like the kernel
    ntri = NUM_VERTS_TABLE[ctype] // 3
    cube = np.repeat(np.arange(ctype.shape[0]), ntri)
    local = np.arange(cube.shape[0]) - np.repeat(np.cumsum(ntri) - ntri, ntri)
    T = cube.shape[0]
    tris = np.zeros((T, 3, 3), dtype=np.float32)
    vids = np.zeros((T, 3, 4), dtype=np.int32)
    sids = np.zeros((T, 3, 2), dtype=np.int32)
    sw = np.zeros((T, 3, 1), dtype=np.float32)
    sid0, sid1, sid2 = r1 ** 3, r1 ** 2, r1
    for j in range(3):
        e = TRI_TABLE[ctype[cube], 3 * local + j]
        a, b = MC_EDGES[e, 0], MC_EDGES[e, 1]
        p1, p2 = pts[cube, a], pts[cube, b]
        v1, v2 = vals[cube, a].astype(np.float64), vals[cube, b].astype(np.float64)
        pos = _interp(p1.astype(np.float64), p2.astype(np.float64), v1, v2)
        w1 = np.where(np.abs(v1) < 1e-5, 1.0, np.where(np.abs(v2) < 1e-5, 0.0,
                      np.where(np.abs(v1 - v2) < 1e-5, 1.0, 1 - (-v1 / np.where(v2 == v1, 1, v2 - v1)))))
        tris[:, j] = pos
        ca, cb = _PRIMAL_CORNER[a], _PRIMAL_CORNER[b]
        mn = np.minimum(ca, cb)
        axis = np.argmax(np.abs(ca - cb), axis=1)
        s = sub[cube]
        ib = base[lif[cube]].astype(np.int64)          # int(bx): truncation, as the kernel
        vids[:, j, :3] = ib * r + s + mn
        vids[:, j, 3] = axis
        sids[:, j, 0] = sid0 * lif[cube] + sid1 * (s[:, 0] + ca[:, 0]) + sid2 * (s[:, 1] + ca[:, 1]) + (s[:, 2] + ca[:, 2])
        sids[:, j, 1] = sid0 * lif[cube] + sid1 * (s[:, 0] + cb[:, 0]) + sid2 * (s[:, 1] + cb[:, 1]) + (s[:, 2] + cb[:, 2])
        sw[:, j, 0] = w1
    return tris, vids, sids, sw


def dual_marching_cubes_indices(table: HashTable, expand_primal_base: dict, strides: dict, bases: dict):
    """Dual-cube corner accumulation through key lookups (``dual_mc_inds.cu:45-182``)."""
    nd = table.inserted_size
    acc = np.zeros((nd, 8, 2), dtype=np.int32)
    cnt = np.zeros(nd, dtype=np.int64)
    for d, pb in expand_primal_base.items():
        s = int(strides[d])
        pb = np.asarray(pb).astype(np.int64)
        ids = np.arange(pb.shape[0]) + int(bases[d])
        probes = []
        for c in range(8):
            probes.append((_CORNER_AXIS[c] * s, [_octant_slot(1 - _CORNER_AXIS[c])[0]]))
        for a in range(3):
            b0, b1 = [x for x in range(3) if x != a]
            for v0 in (0, 1):
                for v1 in (0, 1):
                    for t in range(1, s):
                        off = np.zeros(3, dtype=np.int64)
                        off[b0], off[b1], off[a] = v0 * s, v1 * s, t
                        sl = []
                        for oa in (0, 1):
                            o = np.zeros(3, dtype=np.int64)
                            o[b0], o[b1], o[a] = 1 - v0, 1 - v1, oa
                            sl.append(_octant_slot(o)[0])
                        probes.append((off, sl))
        for a in range(3):
            b0, b1 = [x for x in range(3) if x != a]
            for side in (0, 1):
                for u in range(1, s):
                    for v in range(1, s):
                        off = np.zeros(3, dtype=np.int64)
                        off[a], off[b0], off[b1] = side * s, u, v
                        sl = []
                        for o0 in (0, 1):
                            for o1 in (0, 1):
                                o = np.zeros(3, dtype=np.int64)
                                o[a], o[b0], o[b1] = 1 - side, o0, o1
                                sl.append(_octant_slot(o)[0])
                        probes.append((off, sl))
        for off, sl in probes:
            p = pb + off
            pos = table.query(fnv60([p[:, 0], p[:, 1], p[:, 2]]).astype(np.int64))
            ok = pos > 0
            r = pos[ok] - 1
            np.add.at(cnt, r, len(sl))
            for o in sl:
                acc[r, o, 0] = ids[ok]
                acc[r, o, 1] = d
    return acc, cnt.astype(np.int32)


def dual_marching_cubes_sparse(acc, corner_pos, corner_val):
    """Dual MC (``dual_mc.cu:33-189``): tris f32[T,3,3], vert ids int32[T,3,2]."""
    from .spsr import dual_marching_cubes
    tris, vids = dual_marching_cubes(np.asarray(acc), np.asarray(corner_pos, dtype=np.float64),
                                     np.asarray(corner_val, dtype=np.float64))
    return tris.astype(np.float32), vids


# ----------------------------------------------------------------------------- signed distance from points
def knn(queries, ref_xyz, k):
    """Exact k nearest reference points (FP64 distances), nearest first: (indices, squared distances).
    The reference's k-d tree search (``csrc/common/kdtree_cuda.cu:1071-1279``) in scipy's cKDTree."""
    from scipy.spatial import cKDTree
    d, idx = cKDTree(np.asarray(ref_xyz, np.float64)).query(np.asarray(queries, np.float64), k=k)
    return idx.reshape(-1, k), (d ** 2).reshape(-1, k)


def sdf_from_points(queries, ref_xyz, ref_normal, nb_points, stdv):
    """``ext/sdfgen/sdf_from_points.cu:31-68``: magnitude from the nearest point (the distance to its
    tangent plane when closer than ``stdv``, else the distance to it), sign negative unless more than
    ``nb_points // 2`` of the nearest normals see the query on their positive side."""
    q = np.asarray(queries, np.float64)
    idx, _ = knn(q, ref_xyz, nb_points)
    ray = q[:, None, :] - np.asarray(ref_xyz, np.float64)[idx]
    dots = np.sum(np.asarray(ref_normal, np.float64)[idx] * ray, -1)
    length0 = np.linalg.norm(ray[:, 0], axis=1)
    mag = np.where(length0 < stdv, np.abs(dots[:, 0]), length0)
    pos = np.count_nonzero(dots > 0, axis=1)
    return np.where(pos <= nb_points // 2, -mag, mag), idx
