"""The reference's op surface (jspsr.ext) on libngs vs the oracle's CPU restatements.

Integer results (keys, query results, meshgrid, MC topology, dual-cube corners) bit-exact;
float results within the stated tolerance.
"""
import numpy as np
import pytest
import torch

from oracle import ops as O
from oracle import spsr as S

pytestmark = pytest.mark.gpu
DEV = "cuda"


def t(a, dtype=None):
    x = torch.from_numpy(np.ascontiguousarray(a)).to(DEV)
    return x if dtype is None else x.to(dtype)


@pytest.mark.parametrize("dim,dtype", [(2, np.int32), (3, np.int32), (4, np.int32), (3, np.int64), (4, np.int64)])
def test_hash_cuda_bit_exact(dim, dtype):
    from jspsr import ext
    rng = np.random.default_rng(dim)
    c = rng.integers(-2 ** 20, 2 ** 20, size=(5000, dim)).astype(dtype)
    np.testing.assert_array_equal(ext.hash_cuda(t(c)).cpu().numpy(), O.hash_cuda(c))


def test_fnv_golden_keys(golden):
    from jspsr import ext
    g = golden("fnv_keys")
    np.testing.assert_array_equal(ext.hash_cuda(t(g["coords"])).cpu().numpy(), g["keys"])


def test_kernel_hash_bit_exact():
    from jspsr import ext
    rng = np.random.default_rng(1)
    c = rng.integers(-500, 500, size=(1000, 3)).astype(np.int32)
    k = S.range_kernel(5)
    np.testing.assert_array_equal(ext.kernel_hash_cuda(t(c), t(k)).cpu().numpy(), O.kernel_hash_cuda(c, k))


@pytest.mark.parametrize("n,enlarge", [(1, False), (100, False), (50000, False), (50000, True)])
def test_table_build_and_query(n, enlarge):
    from jspsr import ext
    rng = np.random.default_rng(n)
    coords = np.unique(rng.integers(-300, 300, size=(n, 3)), axis=0).astype(np.int32)
    table = ext.CuckooHashTable(t(coords), enlarged=enlarge)
    # present keys map to their rows
    np.testing.assert_array_equal(table.query(t(coords)).cpu().numpy(), np.arange(coords.shape[0]))
    # absent keys miss; neighbour queries agree with the oracle table
    probe = rng.integers(-310, 310, size=(20000, 3)).astype(np.int32)
    ref = S.Grid(coords, 1).lookup(probe)
    np.testing.assert_array_equal(table.query(t(probe)).cpu().numpy(), ref)
    k = S.range_kernel(3)
    res = table.query(t(coords[:200]), t(k)).cpu().numpy()
    ref = S.Grid(coords, 1).lookup(coords[None, :200] + k[:, None])
    np.testing.assert_array_equal(res, ref)


def test_table_duplicates_keep_smallest_value():
    from jspsr import ext
    keys = t(np.array([7, 9, 7, 11, 9], dtype=np.int64))
    data = ext.build_hash_table(keys, t(np.array([5, 3, 2, 8, 4], dtype=np.int64)), False)
    out = ext.hash_table_query(data, t(np.array([7, 9, 11, 12], dtype=np.int64))).cpu().numpy()
    np.testing.assert_array_equal(out, [3, 4, 9, 0])      # value + 1, 0 = absent


def test_empty_queries():
    from jspsr import ext
    table = ext.CuckooHashTable(t(np.zeros((1, 3), np.int32)))
    assert table.query(t(np.zeros((0, 3), np.int32))).numel() == 0
    assert table.query(t(np.zeros((0, 3), np.int32)), t(S.range_kernel(3))).shape == (27, 0)


def _screening_case(seed=0, n_pts=500, dim=1):
    rng = np.random.default_rng(seed)
    al = rng.integers(0, 28, n_pts)
    bl = rng.integers(0, 28, n_pts)
    a_inds = rng.integers(0, 300, al.sum())
    b_inds = rng.integers(0, 300, bl.sum())
    pairs = np.unique(np.stack([rng.integers(0, 300, 20000), rng.integers(0, 300, 20000)], 1), axis=0)
    shape_a = (al.sum(),) if dim == 1 else (al.sum(), 3)
    shape_b = (bl.sum(),) if dim == 1 else (bl.sum(), 3)
    return (pairs, rng.normal(size=shape_a).astype(np.float32), rng.normal(size=shape_b).astype(np.float32),
            a_inds, b_inds, al, bl, rng.uniform(0.5, 2, n_pts).astype(np.float32))


@pytest.mark.parametrize("dim", [1, 3])
def test_screened_multiplication(dim):
    from jspsr import ext
    pairs, av, bv, ai, bi, al, bl, w = _screening_case(dim=dim)
    keys = O.hash2(pairs[:, 0], pairs[:, 1])
    ref_table = O.HashTable(keys)
    table = ext.build_hash_table(t(keys), torch.tensor([], device=DEV), True)
    res = ext.screened_multiplication(table, t(av), t(bv), t(ai), t(bi), t(al), t(bl), t(w)).cpu().numpy()
    ref = O.screened_multiplication(ref_table, av, bv, ai, bi, al, bl, w)
    np.testing.assert_allclose(res, ref, rtol=1e-5, atol=1e-5)
    g = np.random.default_rng(5).normal(size=res.shape).astype(np.float32)
    ga, gb, gw = [x.cpu().numpy() for x in ext.screened_multiplication_backward(
        table, t(av), t(bv), t(ai), t(bi), t(al), t(bl), t(w), t(g))]
    ra, rb, rw = O.screened_multiplication_backward(ref_table, av, bv, ai, bi, al, bl, w, g)
    for x, y in [(ga, ra), (gb, rb), (gw, rw)]:
        np.testing.assert_allclose(x, y, rtol=1e-4, atol=1e-4)


def test_sparse_meshgrid():
    from jspsr import ext
    al = np.array([2, 0, 3, 1], np.int64)
    bl = np.array([1, 4, 2, 0], np.int64)
    a, b = ext.sparse_meshgrid(t(al), t(bl))
    ra, rb = O.sparse_meshgrid(al, bl)
    np.testing.assert_array_equal(a.cpu().numpy(), ra)
    np.testing.assert_array_equal(b.cpu().numpy(), rb)


def test_ddi_forward_backward():
    from jspsr import ext
    rng = np.random.default_rng(3)
    C, R, P = 10, 14, 4000
    src = rng.normal(size=(P, 3 * C)).astype(np.float32)
    tgt = rng.normal(size=(P, 3 * C)).astype(np.float32)
    rel = rng.integers(0, R, size=(P, 3))
    ff = rng.normal(size=(C, C, R)).astype(np.float32)
    dd = rng.normal(size=(C, C, R)).astype(np.float32)
    p, q = ext.ddi_forward(t(src), t(tgt), t(rel), t(ff), t(dd))
    rp, rq = O.ddi_forward(src, tgt, rel, ff, dd)
    np.testing.assert_allclose(p.cpu().numpy(), rp, rtol=1e-4, atol=1e-3)
    np.testing.assert_allclose(q.cpu().numpy(), rq, rtol=1e-4, atol=1e-3)
    gp = rng.normal(size=(P, 3)).astype(np.float32)
    gq = rng.normal(size=(P, 3)).astype(np.float32)
    gs, gt = ext.ddi_backward(t(src), t(tgt), t(rel), t(ff), t(dd), t(gp), t(gq))
    rs, rt = O.ddi_backward(src, tgt, rel, ff, dd, gp, gq)
    np.testing.assert_allclose(gs.cpu().numpy(), rs, rtol=1e-4, atol=1e-3)
    np.testing.assert_allclose(gt.cpu().numpy(), rt, rtol=1e-4, atol=1e-3)


def _spd_csr(n_side=20, shift=0.5):
    import scipy.sparse as sp
    n = n_side ** 3
    e = np.ones(n_side)
    l1 = sp.diags([-e[:-1], 2 * e, -e[:-1]], [-1, 0, 1])
    eye = sp.identity(n_side)
    A = (sp.kron(sp.kron(l1, eye), eye) + sp.kron(sp.kron(eye, l1), eye) + sp.kron(sp.kron(eye, eye), l1)
         + shift * sp.identity(n)).tocsr()
    A.sort_indices()
    return A


def test_solve_pcg_diag_reference_semantics():
    from jspsr import ext
    A = _spd_csr()
    b = np.random.default_rng(0).normal(size=A.shape[0]).astype(np.float32)
    dinv = (1.0 / A.diagonal()).astype(np.float32)
    x, it = ext.solve_pcg_diag(t(A.indptr.astype(np.int32)), t(A.indices.astype(np.int32)),
                               t(A.data.astype(np.float32)), t(b), t(dinv), 1e-5, 300, False)
    x = x.cpu().numpy()
    r = b - A @ x
    assert np.linalg.norm(r) <= 1.5e-5 * np.linalg.norm(b)
    xr, itr = O.solve_pcg_diag(A.indptr, A.indices, A.data, b, dinv, 1e-5, 300, False)
    assert abs(it - itr) <= 2                       # same recurrence in exact arithmetic
    xs = ext.solve_cusparse(t(A.indptr.astype(np.int32)), t(A.indices.astype(np.int32)),
                            t(A.data.astype(np.float32)), t(b), 1e-6).cpu().numpy()
    import scipy.sparse.linalg as spla
    ex = spla.spsolve(A.tocsc(), b.astype(np.float64))
    assert np.linalg.norm(xs - ex) <= 1e-6 * np.linalg.norm(ex)


def test_primal_marching_cubes():
    from jspsr import ext
    rng = np.random.default_rng(7)
    M, r = 50, 4
    base = rng.integers(-10, 10, size=(M, 3)).astype(np.float32)
    sdf = rng.normal(size=(M, r + 1, r + 1, r + 1)).astype(np.float32)
    tris, vids, sids, sw = [x.cpu().numpy() for x in ext.marching_cubes_sparse(t(base), t(sdf))]
    rt, rv, rs, rw = O.marching_cubes_sparse(base, sdf)
    np.testing.assert_array_equal(vids, rv)
    np.testing.assert_array_equal(sids, rs)
    np.testing.assert_allclose(tris, rt, atol=1e-5)
    np.testing.assert_allclose(sw, rw, atol=1e-5)


def _mc_autograd_oracle(base, sdf, grad_vert, bandwidth):
    """numpy restatement of the differentiable primal MC (``ops.py:9-58``): vertices deduplicated by
    their edge ids, area-weighted normals, and the backward that hands each vertex's normal
    component of grad_vert to the two grid values of its edge."""
    tris, vids, sids, sw = O.marching_cubes_sparse(base, sdf)
    unq, inv = np.unique(vids.reshape(-1, 4), axis=0, return_inverse=True)
    inv = inv.reshape(-1)
    verts = np.zeros((unq.shape[0], 3), np.float64)
    verts[inv] = tris.reshape(-1, 3)
    vsrc = np.zeros((unq.shape[0], 2), np.int64)
    vsrc[inv] = sids.reshape(-1, 2)
    vw = np.zeros(unq.shape[0], np.float64)
    vw[inv] = sw.reshape(-1)
    faces = inv.reshape(-1, 3)
    e1 = verts[faces[:, 1]] - verts[faces[:, 0]]
    e2 = verts[faces[:, 2]] - verts[faces[:, 0]]
    fn = np.cross(e1, e2)
    vn = np.zeros_like(verts)
    for k in range(3):
        np.add.at(vn, faces[:, k], fn)
    vn /= np.linalg.norm(vn, axis=1, keepdims=True) + 1e-6
    g = bandwidth * (grad_vert[: verts.shape[0]] * vn).sum(1)
    grid = np.zeros(sdf.size)
    np.add.at(grid, vsrc[:, 0], vw * g)
    np.add.at(grid, vsrc[:, 1], (1 - vw) * g)
    return verts, faces, vn, grid.reshape(sdf.shape)


def test_marching_cubes_autograd():
    """``MarchingCubes`` (vertices, triangles, normals, and the backward to the grid values) against
    its numpy restatement over the oracle's primal MC."""
    from jspsr.core.ops import marching_cubes_op
    M, r = 30, 4
    g = np.stack(np.meshgrid(*[np.arange(r + 1)] * 3, indexing="ij"), -1).astype(np.float32)
    base = np.array([[i, j, k] for i in range(-2, 1) for j in range(-2, 1) for k in range(-2, 1)][:M], np.float32)
    base = base[: min(M, base.shape[0])]
    pts = base[:, None, None, None, :] + g[None] / r
    sdf = (np.linalg.norm(pts + 0.1, axis=-1) - 1.3).astype(np.float32)       # a sphere through the blocks
    sdf_t = t(sdf).requires_grad_(True)
    v, f, n, _ = marching_cubes_op(t(base), sdf_t, 1.0)
    rng = np.random.default_rng(3)
    gv = rng.normal(size=(v.shape[0], 3)).astype(np.float32)
    (v * t(gv)).sum().backward()
    rv, rf, rn, rg = _mc_autograd_oracle(base, sdf, gv, 1.0)
    np.testing.assert_array_equal(f.cpu().numpy(), rf)
    np.testing.assert_allclose(v.detach().cpu().numpy(), rv, atol=1e-5)
    np.testing.assert_allclose(n.detach().cpu().numpy(), rn, atol=1e-4)
    # an edge on a block boundary is seen from both blocks, each with its own copy of the boundary
    # samples, and which copy its vertex draws from is arbitrary (the reference's "randomly pick one
    # solution for overlapping edges"): compare the gradients summed per lattice position
    loc = np.stack(np.meshgrid(*[np.arange(r + 1)] * 3, indexing="ij"), -1).reshape(-1, 3)
    lattice = (base.astype(np.int64)[:, None, :] * r + loc[None]).reshape(-1, 3)
    keys, inv = np.unique(lattice, axis=0, return_inverse=True)

    def per_position(gr):
        out = np.zeros(keys.shape[0])
        np.add.at(out, inv.reshape(-1), gr.reshape(-1))
        return out
    got = per_position(sdf_t.grad.cpu().numpy().astype(np.float64))
    ref = per_position(rg)
    assert np.linalg.norm(got - ref) <= 1e-4 * np.linalg.norm(ref)


def test_dual_marching_cubes_ops(golden):
    """Dual-grid accumulation and dual MC on the oracle's structures and values (sign pattern given)."""
    from jspsr import ext
    g = golden("torus_small")
    vs, depth, md, alpha = g["params"]
    sol = S.solve_multigrid(g["xyz"], g["nrm"], vs, int(depth), md, alpha)
    base, max_depth = S.conformal_leaves(sol.grids, int(depth))
    ex = np.stack(np.meshgrid(*[np.arange(2)] * 3, indexing="ij"), -1).reshape(-1, 3)
    epb = {d: ((base[d] * 2)[:, None] + (ex * sol.grids[d].stride)[None]).reshape(-1, 3).astype(np.int32)
           for d in range(max_depth)}
    cand = np.concatenate([epb[d] + o * sol.grids[d].stride for d in range(max_depth) for o in S.CONFORM_OFFSETS])
    dual = S.unique_rows(cand)
    strides = {d: sol.grids[d].stride for d in range(max_depth)}
    bases = {d: sum(epb[dd].shape[0] for dd in range(d)) for d in range(max_depth)}
    table = ext.CuckooHashTable(t(dual))
    acc, cnt = ext.dual_marching_cubes_indices(table.object, {d: t(v) for d, v in epb.items()}, strides, bases)
    racc, rcnt = S.dual_corner_indices(S.Grid(dual, 1), epb, strides, bases)
    np.testing.assert_array_equal(cnt.cpu().numpy(), rcnt)
    full = rcnt == 8
    np.testing.assert_array_equal(acc.cpu().numpy()[full], racc[full])
    mesh = S.extract_multiscale_mesh(sol, g["xyz"])
    pos = mesh.dual_pos.astype(np.float32)
    vals = mesh.dual_values.astype(np.float32)
    tris, vids = ext.dual_marching_cubes_sparse(t(racc[full]), t(pos), t(vals))
    rt, rv = O.dual_marching_cubes_sparse(racc[full], pos, vals)
    np.testing.assert_array_equal(vids.cpu().numpy(), rv)
    np.testing.assert_allclose(tris.cpu().numpy(), rt, atol=1e-5)
