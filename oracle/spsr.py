"""FP64 CPU oracle of the jspsr sparse screened-Poisson reconstruction path.

TEST INFRASTRUCTURE ONLY.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` may import this
module, and only as the checker or the timed CPU baseline.  The product
(``neural-galerkin_b200/jspsr``) never imports it.

It restates, in numpy / scipy, the algorithm of the reference's Python layer
and of the CUDA ops that layer calls.  Decisions that fix the *structure*
(voxel quantisation, octant signs, neighbour quantisation) are made in float32
exactly as the reference's torch code makes them, so that integer outputs can
be compared bit for bit; everything numeric (weights, integrals, Galerkin
matrices, the per-level solves, the field and the mesh vertices) is FP64 and
each level is solved to machine precision with a direct sparse solver.

Reference files followed (paths inside huangjh-pub/neural-galerkin):

* ``jspsr/__init__.py:8-61``                    -- ``reconstruct``
* ``jspsr/core/_hash_backend.py:13-28``          -- ``compute_density``
* ``jspsr/core/_hash_backend.py:176-228``        -- ``get_coords_neighbours``
* ``jspsr/core/_hash_backend.py:230-290``        -- ``get_self_neighbours`` (incl. inversion)
* ``jspsr/core/_hash_backend.py:332-356``        -- ``splat_data``
* ``jspsr/core/_hash_backend.py:414-444,457-510``-- adaptive hierarchy, trilinear weights
* ``jspsr/core/hashtree.py:103-116,157-192,209-229,266-287``
* ``jspsr/core/reconstructor.py:59-195``         -- ``solve_multigrid`` (RHS, correction, LHS)
* ``jspsr/core/reconstructor.py:197-255``        -- chi evaluation, mean-chi level set
* ``jspsr/core/reconstructor.py:296-397``        -- ``extract_multiscale_mesh``
* ``jspsr/bases/bezier_tensor.py:36-121``        -- B-spline basis and its integrals
* ``csrc/common/hashmap_cuda.cu:247-261``        -- FNV-1a key hash
* ``csrc/marching_cubes/dual_mc_inds.cu:45-141`` -- dual-cube corner accumulation
* ``csrc/marching_cubes/dual_mc.cu:20-133``      -- dual marching cubes

Parity status: the integral tables and the neighbour-offset order are
re-derived (the reference's ``jspsr/data`` files were never published); the
restatement is pinned against the reference's own Python code run on CPU with
these tables (``tests/golden/make_golden.py``).  The CUDA ops of the reference
(hash table, screened product, PCG, marching cubes) cannot run here and are
pinned by known-answer and property tests only.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from . import tables as _tables
from .mc_tables import TRI_TABLE, EDGE_TABLE, NUM_VERTS_TABLE

F32 = np.float32
CONFORM_OFFSETS = np.array([(0, 0, 0), (0, 0, 1), (0, 1, 0), (0, 1, 1),
                            (1, 0, 0), (1, 0, 1), (1, 1, 0), (1, 1, 1)], dtype=np.int32)
_PACK_OFF = 1 << 20


# ----------------------------------------------------------------------------- keys / kernels
def fnv60(columns) -> np.ndarray:
    """FNV-1a 64 over ``(uint32)`` columns folded to 60 bits (``hashmap_cuda.cu:247-261``)."""
    h = np.full(np.asarray(columns[0]).shape, 14695981039346656037, dtype=np.uint64)
    prime = np.uint64(1099511628211)
    with np.errstate(over="ignore"):
        for c in columns:
            h ^= np.asarray(c).astype(np.int64).astype(np.uint32).astype(np.uint64)
            h *= prime
    return (h >> np.uint64(60)) ^ (h & np.uint64(0x0FFFFFFFFFFFFFFF))


def range_kernel(n: int) -> np.ndarray:
    """Ordered neighbour offsets ``int32[n**3, 3]`` (``hashtree.py:103-116``).

    The reference loads the order from the unpublished ``kernel.npz``; the
    incremental neighbour cache (``_hash_backend.py:56-63,270-274``) requires the
    prefix property (first 1 = origin, first 27 = [-1,1]^3, first 125 = [-2,2]^3).
    Chosen order: Chebyshev shells outward, lexicographic (x, y, z) inside a shell.
    """
    assert n % 2 == 1
    r = n // 2
    g = np.stack(np.meshgrid(*[np.arange(-r, r + 1)] * 3, indexing="ij"), -1).reshape(-1, 3)
    shell = np.abs(g).max(1)
    order = np.lexsort((g[:, 2], g[:, 1], g[:, 0], shell))
    return g[order].astype(np.int32)


def pack(c: np.ndarray) -> np.ndarray:
    c = np.asarray(c).astype(np.int64)
    return ((c[..., 0] + _PACK_OFF) << 42) | ((c[..., 1] + _PACK_OFF) << 21) | (c[..., 2] + _PACK_OFF)


def unpack(k: np.ndarray) -> np.ndarray:
    m = (1 << 21) - 1
    return np.stack([(k >> 42) - _PACK_OFF, ((k >> 21) & m) - _PACK_OFF, (k & m) - _PACK_OFF], -1).astype(np.int32)


def unique_rows(c: np.ndarray, return_inverse=False):
    """Lexicographically sorted unique rows, as ``torch.unique(dim=0)`` (``ops.py:103-127``)."""
    keys = pack(c.reshape(-1, 3))
    u, inv = np.unique(keys, return_inverse=True)
    out = unpack(u).reshape(-1, 3)
    return (out, inv.reshape(-1)) if return_inverse else out


class Grid:
    """One level: sorted unique voxel min-corners (finest-voxel units) and a row lookup."""

    def __init__(self, coords: np.ndarray, stride: int):
        self.coords = np.ascontiguousarray(coords, dtype=np.int32).reshape(-1, 3)
        self.stride = int(stride)
        self.keys = pack(self.coords)

    def __len__(self):
        return self.coords.shape[0]

    def lookup(self, c: np.ndarray) -> np.ndarray:
        k = pack(c)
        if len(self.keys) == 0:
            return np.full(k.shape, -1, dtype=np.int64)
        pos = np.clip(np.searchsorted(self.keys, k), 0, len(self.keys) - 1)
        return np.where(self.keys[pos] == k, pos, -1).astype(np.int64)


# ----------------------------------------------------------------------------- basis
def bspline(x):
    """Quadratic B-spline x2 (``bezier_tensor.py:36-44``)."""
    x = np.asarray(x, dtype=np.float64)
    return np.where((x >= -1.5) & (x < -0.5), (x + 1.5) ** 2,
           np.where((x >= -0.5) & (x < 0.5), -2 * x * x + 1.5,
           np.where((x >= 0.5) & (x < 1.5), (x - 1.5) ** 2, 0.0)))


def bspline_d(x):
    """Derivative of the B-spline (``bezier_tensor.py:46-54``)."""
    x = np.asarray(x, dtype=np.float64)
    return np.where((x >= -1.5) & (x < -0.5), 2 * x + 3,
           np.where((x >= -0.5) & (x < 0.5), -4 * x,
           np.where((x >= 0.5) & (x < 1.5), 2 * x - 3, 0.0)))


class BezierTables:
    """FP64 integral tables for level ratios 2**m, m < n_mult (extended analytically past 16)."""

    def __init__(self, n_mult: int):
        t = _tables.bezier_tables(max(n_mult, 1))
        self.ssi, self.sdi = t["SHIFTED_SELF_INTEGRAL"], t["SHIFTED_DERIVATIVE_INTEGRAL"]
        self.dpi, self.pi = t["DERIVATIVE_PARTIAL_INTEGRAL"], t["PARTIAL_INTEGRAL"]
        self.idpi, self.ipi = t["INV_DERIVATIVE_PARTIAL_INTEGRAL"], t["INV_PARTIAL_INTEGRAL"]

    def deriv_deriv(self, rel, s_src, s_tgt):
        """int grad B_src . grad B_tgt (``bezier_tensor.py:75-96``); rel in source-stride units."""
        M = s_tgt // s_src
        m = int(round(math.log2(M)))
        idx = np.round(rel + M * 1.5 + 0.5).astype(np.int64)
        n = len(self.ssi[m])
        bad = ~((idx >= 0) & (idx < n))
        idx = np.clip(idx, 0, n - 1)
        c = self.ssi[m][idx] * s_src
        g = self.sdi[m][idx] / s_tgt
        c[bad] = 0.0
        g[bad] = 0.0
        return g[:, 0] * c[:, 1] * c[:, 2] + c[:, 0] * g[:, 1] * c[:, 2] + c[:, 0] * c[:, 1] * g[:, 2]

    def const_deriv(self, data, rel, s_data, s_tgt):
        """int grad B_tgt . data over a data voxel (``bezier_tensor.py:98-121``)."""
        if s_tgt >= s_data:
            M = s_tgt // s_data
            idx = np.round(rel + (3 * M - 1) / 2.0).astype(np.int64)
            m = int(round(math.log2(M)))
            dpi, pi, i_mult, ds = self.dpi[m], self.pi[m], s_data / s_tgt, s_data
        else:
            M = s_data // s_tgt
            idx = np.round(rel * M + M / 2 + 0.5).astype(np.int64)
            m = int(round(math.log2(M))) - 1
            dpi, pi, i_mult, ds = self.idpi[m], self.ipi[m], 1.0, s_tgt
        c = dpi[idx] * ds
        g = pi[idx] * i_mult
        return (data[:, 0] * g[:, 0] * c[:, 1] * c[:, 2] + data[:, 1] * c[:, 0] * g[:, 1] * c[:, 2]
                + data[:, 2] * c[:, 0] * c[:, 1] * g[:, 2])


# ----------------------------------------------------------------------------- point geometry
def q_f32(xyz32: np.ndarray, vs: float) -> np.ndarray:
    """``xyz / voxel_size`` as torch evaluates it on CUDA: times the fp32 reciprocal."""
    inv = F32(1.0) / F32(vs)
    return (xyz32.astype(F32) * inv).astype(F32)


def trilinear(q32, q64, stride: int, data=None):
    """8 trilinear corners and weights, corner-major (``_hash_backend.py:469-510``).

    Structure (corner cells, octant signs) in float32 as the reference; weights in FP64.
    """
    s = F32(stride)
    d32 = (np.floor(q32 / s) * s).astype(F32)
    rel32 = (q32 - d32 - F32(stride / 2.0)).astype(F32)
    sgn = np.sign(rel32).astype(F32)
    loc = np.abs(q64 - d32.astype(np.float64) - stride / 2.0) / stride
    coords, w = [], []
    for nx, ny, nz in CONFORM_OFFSETS:
        off = np.stack([nx * sgn[:, 0], ny * sgn[:, 1], nz * sgn[:, 2]], 1) * s
        coords.append((d32 + off).astype(np.int32))
        a = (loc[:, 0] if nx else 1 - loc[:, 0]) * (loc[:, 1] if ny else 1 - loc[:, 1]) * \
            (loc[:, 2] if nz else 1 - loc[:, 2])
        w.append(a if data is None else a[:, None] * data)
    return np.concatenate(coords, 0), np.concatenate(w, 0)


def point_neighbours(grid: Grid, q32, q64, kernel, transposed=True):
    """``get_neighbours_data(xyz/vs - 0.5, 1, d, kernel)`` for point queries.

    Returns (pts_ids, vx_ids, rel[P,3]) where rel = position of the point
    relative to the voxel centre in voxel units (``-tgt_offsets / stride``,
    ``hashtree.py:169-181``, ``reconstructor.py:113-119``).
    """
    s = grid.stride
    xyz_pos32 = (q32 - F32(0.5)).astype(F32)
    quant = (np.floor((xyz_pos32 + F32(0.5)) / F32(s)) * F32(s)).astype(np.int32)
    probes = quant[None, :, :] + kernel[:, None, :] * s          # [K, N, 3]
    res = grid.lookup(probes)                                       # [K, N]
    if transposed:
        pts, kk = np.nonzero(res.T != -1)
    else:
        kk, pts = np.nonzero(res != -1)
    vx = res[kk, pts]
    # nt = k*s + (quant - xyz_pos) + (s-1)/2 ; rel = -nt / s  (FP64 from the exact position)
    nt = kernel[kk].astype(np.float64) * s + (quant[pts] - (q64[pts] - 0.5)) + (s - 1) / 2.0
    return pts, vx, -nt / s


def voxel_neighbours(src: Grid, tgt: Grid, kernel, transposed=False):
    """``get_coords_neighbours`` for voxel sources, non-conv mode (``_hash_backend.py:191-228``).

    Returns (src_ids, tgt_ids, rel[P,3]) with rel = (c_tgt - c_src) / s_src between centres.
    """
    ss, st = src.stride, tgt.stride
    assert ss <= st
    quant = (np.floor((src.coords + 0.5 * ss) / st) * st).astype(np.int32)
    c_off = (quant - src.coords) / ss + (st // ss - 1) / 2.0
    res = tgt.lookup(quant[None] + kernel[:, None, :] * st)
    if transposed:
        si, kk = np.nonzero(res.T != -1)
    else:
        kk, si = np.nonzero(res != -1)
    ti = res[kk, si]
    rel = kernel[kk] * (st / ss) + c_off[si]
    return si, ti, rel


def level_pairs(grids, src_d, tgt_d, rng):
    """``get_self_neighbours(src_d, tgt_d, rng)`` incl. the coarse->fine inversion (``_hash_backend.py:230-290``)."""
    kernel = range_kernel(rng)
    if src_d <= tgt_d:
        return voxel_neighbours(grids[src_d], grids[tgt_d], kernel)
    # Inverted: query fine -> coarse, keep near pairs, convert offsets to coarse units.
    si, ti, nt = voxel_neighbours(grids[tgt_d], grids[src_d], kernel)
    near = np.all(np.abs(nt) < rng / 2.0 + 1.0e-6, axis=1)
    nt = -nt / grids[src_d].stride * grids[tgt_d].stride
    return ti[near], si[near], nt[near]


# ----------------------------------------------------------------------------- density / hierarchy
def compute_density(xyz32: np.ndarray, vs: float) -> np.ndarray:
    """B-spline KDE at voxel ``4*vs`` divided by 16 (``_hash_backend.py:13-28``, ``hashtree.py:283-285``)."""
    vsd = 4 * vs
    q32 = q_f32(xyz32, vsd)
    q64 = xyz32.astype(np.float64) / vsd
    corners, _ = trilinear(q32, q64, 1)
    g = Grid(unique_rows(corners), 1)
    corners, w = trilinear(q32, q64, 1)
    rows = g.lookup(corners)
    wd = np.bincount(rows, weights=w, minlength=len(g))
    pts, vx, rel = point_neighbours(g, q32, q64, range_kernel(3))
    phi = bspline(rel[:, 0]) * bspline(rel[:, 1]) * bspline(rel[:, 2])
    dens = np.bincount(pts, weights=phi * wd[vx], minlength=xyz32.shape[0])
    return dens / 16.0


def point_levels(density: np.ndarray, min_density: float, depth: int):
    """``-floor(log4(rho / min_density))`` clamped to [0, depth-1] (``_hash_backend.py:428-429``).

    Also returns the unfloored log4 value so callers can spot boundary cases.
    """
    t = np.log(density / min_density) / np.log(4.0)
    lvl = -np.minimum(np.floor(t), 0)
    return np.minimum(lvl, depth - 1).astype(np.int32), t


def build_hierarchy(xyz32, vs, depth, levels) -> list:
    """Per level: unique trilinear corners of points with level <= d (``_hash_backend.py:434-444``)."""
    q32 = q_f32(xyz32, vs)
    q64 = xyz32.astype(np.float64) / vs
    grids = []
    for d in range(depth):
        m = levels <= d
        if not np.any(m):
            raise ValueError(f"level {d} of the hierarchy is empty; lower min_density")
        c, _ = trilinear(q32[m], q64[m], 2 ** d)
        grids.append(Grid(unique_rows(c), 2 ** d))
    return grids


def splat(grid: Grid, xyz32, vs, data):
    """Trilinear splat of per-point data onto existing voxels (``_hash_backend.py:332-356``)."""
    q32 = q_f32(xyz32, vs)
    q64 = xyz32.astype(np.float64) / vs
    corners, w = trilinear(q32, q64, grid.stride, data)
    rows = grid.lookup(corners)
    ok = rows >= 0
    out = np.zeros((len(grid),) + w.shape[1:])
    np.add.at(out, rows[ok], w[ok])
    return out


# ----------------------------------------------------------------------------- solve
@dataclass
class Solution:
    grids: list
    density: np.ndarray
    levels: np.ndarray
    log4: np.ndarray
    normal_data: dict
    rhs: dict = field(default_factory=dict)
    x: dict = field(default_factory=dict)
    lhs: dict = field(default_factory=dict)
    vs: float = 0.0


def phi_matrix(grid: Grid, q32, q64):
    """Point x voxel B-spline matrix Phi_d (the screening data of ``reconstructor.py:110-120``)."""
    pts, vx, rel = point_neighbours(grid, q32, q64, range_kernel(3))
    phi = bspline(rel[:, 0]) * bspline(rel[:, 1]) * bspline(rel[:, 2])
    return sp.csr_matrix((phi, (pts, vx)), shape=(q32.shape[0], len(grid)))


def stiffness(grids, tabs, d, dd):
    """Stiffness block K_{d,dd} over the range-5 pair list (``reconstructor.py:154-179``)."""
    si, ti, rel = level_pairs(grids, d, dd, 5)
    val = tabs.deriv_deriv(rel, grids[d].stride, grids[dd].stride)
    return sp.csr_matrix((val, (si, ti)), shape=(len(grids[d]), len(grids[dd])))


def solve_multigrid(xyz32, nrm32, vs, depth=4, min_density=32.0, screen_alpha=4.0,
                    screen_delta=0.1, levels=None, keep_lhs=False, cg_tol=None) -> Solution:
    """Tree build + splat + coarse-to-fine Galerkin solve (``__init__.py:34-54``, ``reconstructor.py:79-195``)."""
    xyz32 = np.ascontiguousarray(xyz32, dtype=F32)
    nrm32 = np.ascontiguousarray(nrm32, dtype=F32)
    dens = compute_density(xyz32, vs)
    lv, t = point_levels(dens, min_density, depth)
    if levels is not None:
        lv = levels
    grids = build_hierarchy(xyz32, vs, depth, lv)
    w = 1.0 / dens
    normal_data = {}
    for d in range(depth):
        m = lv == d
        if not np.any(m):
            continue
        normal_data[d] = splat(grids[d], xyz32[m], vs, nrm32[m].astype(np.float64) * w[m, None]) / \
            (grids[d].stride ** 3)

    tabs = BezierTables(depth)
    q32 = q_f32(xyz32, vs)
    q64 = xyz32.astype(np.float64) / vs
    phis = {d: phi_matrix(grids[d], q32, q64) for d in range(depth)}
    sol = Solution(grids, dens, lv, t, normal_data, vs=vs)
    alpha = float(screen_alpha)
    for d in range(depth - 1, -1, -1):
        sf = 0.25 ** d
        n = len(grids[d])
        rhs = np.zeros(n)
        for dd, nd in normal_data.items():
            si, ti, rel = level_pairs(grids, dd, d, 3)
            part = tabs.const_deriv(-nd[si], rel, grids[dd].stride, grids[d].stride)
            rhs += np.bincount(ti, weights=part, minlength=n)
        if alpha > 0:
            rhs += sf * alpha * screen_delta * np.asarray(phis[d].sum(0)).ravel()
        for dd in range(depth - 1, d, -1):
            k = stiffness(grids, tabs, d, dd)
            corr = k @ sol.x[dd]
            if alpha > 0:
                corr += sf * alpha * (phis[d].T @ (phis[dd] @ sol.x[dd]))
            rhs -= corr
        a = stiffness(grids, tabs, d, d)
        if alpha > 0:
            a = a + sf * alpha * (phis[d].T @ phis[d])
        a = a.tocsc()
        if cg_tol is not None:
            sol.x[d] = _cg64(a, rhs, tol=cg_tol)        # the CPU baseline: FP64 CSR + Jacobi CG
        else:
            sol.x[d] = spla.spsolve(a, rhs) if n < 3000 else _cg64(a, rhs)
        sol.rhs[d] = rhs
        if keep_lhs:
            sol.lhs[d] = a.tocsr()
    sol.phis = phis
    return sol


def _cg64(a, b, tol=1e-13, maxiter=50000):
    x, info = spla.cg(a, b, rtol=tol, maxiter=maxiter, M=sp.diags(1.0 / a.diagonal()))
    return x


# ----------------------------------------------------------------------------- field
def evaluate_chi_raw(sol: Solution, pos32: np.ndarray, pos64=None, grad=False):
    """Sum over levels of the interpolated field (``reconstructor.py:197-226``, ``hashtree.py:157-192``)."""
    pos32 = np.ascontiguousarray(pos32, dtype=F32)
    if pos64 is None:
        pos64 = pos32.astype(np.float64)
    q32 = q_f32(pos32, sol.vs)
    q64 = pos64 / sol.vs
    out = np.zeros((pos32.shape[0], 3) if grad else pos32.shape[0])
    for d, xd in sol.x.items():
        g = sol.grids[d]
        pts, vx, rel = point_neighbours(g, q32, q64, range_kernel(3))
        if grad:
            b = [bspline(rel[:, i]) for i in range(3)]
            db = [bspline_d(rel[:, i]) / g.stride for i in range(3)]   # bezier_tensor.py:70-72
            val = np.stack([db[0] * b[1] * b[2], b[0] * db[1] * b[2], b[0] * b[1] * db[2]], 1) * xd[vx, None]
            np.add.at(out, pts, val)
        else:
            phi = bspline(rel[:, 0]) * bspline(rel[:, 1]) * bspline(rel[:, 2])
            out += np.bincount(pts, weights=phi * xd[vx], minlength=pos32.shape[0])
    return out


def mean_chi(sol: Solution, xyz32: np.ndarray):
    """Density-weighted mean of chi at the input points (``reconstructor.py:228-236``)."""
    w = 1.0 / sol.density
    return float(np.sum(evaluate_chi_raw(sol, xyz32) * w) / np.sum(w))


# ----------------------------------------------------------------------------- mesh
_CORNER_AXIS = np.array([(x, y, z) for x in (0, 1) for y in (0, 1) for z in (0, 1)], dtype=np.int64)
_MC_CORNER = np.array([(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0),
                       (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)], dtype=np.int64)
# Edge endpoints in the order the reference interpolates them (``dual_mc.cu:100-111``).
MC_EDGES = np.array([(0, 1), (1, 2), (2, 3), (3, 0), (4, 5), (5, 6), (6, 7), (7, 4),
                     (0, 4), (1, 5), (2, 6), (3, 7)], dtype=np.int64)


def _octant_slot(octant):
    """Dual-cube corner slot holding the primal that lies in ``octant`` (0/1 per axis) of the dual centre."""
    o = np.asarray(octant)
    hit = np.all(_MC_CORNER[None, :, :] == o.reshape(-1, 1, 3), axis=2)
    return np.argmax(hit, axis=1)


def conformal_leaves(grids, max_depth):
    """Conformal leaf cells per level (``reconstructor.py:319-336``)."""
    base, mask = {}, {}
    for d in range(max_depth):
        s = grids[d].stride
        c = grids[d].coords
        if d < max_depth - 1:
            par = unique_rows((np.floor(c / s / 2.0).astype(np.int64) * s * 2).astype(np.int32))
            c = (par[:, None, :] + CONFORM_OFFSETS[None] * s).reshape(-1, 3)
        if d > 0:
            children = Grid(unique_rows(base[d - 1]), 1)
            ol = children.lookup(c) == -1
            if not np.any(ol):
                max_depth = d
                break
            mask[d] = ol
        base[d] = c
    for d in range(1, max_depth):
        base[d] = base[d][mask[d]]
    return base, max_depth


def dual_corner_indices(dual: Grid, epb: dict, strides: dict, bases: dict):
    """Dual-cube corner accumulation (``dual_mc_inds.cu:45-141``).

    Returns acc int32[D, 8, 2] (primal id, depth) and count int32[D].
    """
    nd = len(dual)
    acc = np.zeros((nd, 8, 2), dtype=np.int32)
    cnt = np.zeros(nd, dtype=np.int64)
    writes = np.zeros((nd, 8), dtype=np.int64)
    for d, pb in epb.items():
        s = strides[d]
        ids = np.arange(pb.shape[0]) + bases[d]
        pts, slots = [], []
        for c in range(8):                                   # corners: 1 slot
            off = _CORNER_AXIS[c] * s
            pts.append((pb + off, ids, [_octant_slot(1 - _CORNER_AXIS[c])[0]]))
        for a in range(3):                                   # edges: 2 slots
            b0, b1 = [x for x in range(3) if x != a]
            for v0 in (0, 1):
                for v1 in (0, 1):
                    for t in range(1, s):
                        off = np.zeros(3, dtype=np.int64)
                        off[b0], off[b1], off[a] = v0 * s, v1 * s, t
                        octs = []
                        for oa in (0, 1):
                            o = np.zeros(3, dtype=np.int64)
                            o[b0], o[b1], o[a] = 1 - v0, 1 - v1, oa
                            octs.append(_octant_slot(o)[0])
                        pts.append((pb + off, ids, octs))
        for a in range(3):                                   # faces: 4 slots
            b0, b1 = [x for x in range(3) if x != a]
            for side in (0, 1):
                for u in range(1, s):
                    for v in range(1, s):
                        off = np.zeros(3, dtype=np.int64)
                        off[a], off[b0], off[b1] = side * s, u, v
                        octs = []
                        for o0 in (0, 1):
                            for o1 in (0, 1):
                                o = np.zeros(3, dtype=np.int64)
                                o[a], o[b0], o[b1] = 1 - side, o0, o1
                                octs.append(_octant_slot(o)[0])
                        pts.append((pb + off, ids, octs))
        for p, pid, octs in pts:
            row = dual.lookup(p)
            ok = row >= 0
            r, q = row[ok], pid[ok]
            np.add.at(cnt, r, len(octs))
            for o in octs:
                acc[r, o, 0] = q
                acc[r, o, 1] = d
                np.add.at(writes, (r, np.full_like(r, o)), 1)
    complete = cnt == 8
    assert np.all(writes[complete] == 1), "topology conflict inside a complete dual cube"
    return acc, cnt.astype(np.int32)


def _interp(p1, p2, v1, v2):
    """Edge vertex with the reference's 1e-5 snapping (``dual_mc.cu:20-31``)."""
    w2 = np.where(np.abs(v2 - v1) > 0, -v1 / np.where(v2 - v1 == 0, 1, v2 - v1), 0.0)
    out = p1 * (1 - w2)[:, None] + p2 * w2[:, None]
    snap1 = (np.abs(v1) < 1e-5) | ((np.abs(v2) >= 1e-5) & (np.abs(v1 - v2) < 1e-5))
    snap2 = (~(np.abs(v1) < 1e-5)) & (np.abs(v2) < 1e-5)
    out[snap1] = p1[snap1]
    out[snap2] = p2[snap2]
    return out


def dual_marching_cubes(acc: np.ndarray, corner_pos: np.ndarray, corner_val: np.ndarray):
    """Dual MC over complete cubes (``dual_mc.cu:33-189``): tris f64[T,3,3], vert ids int32[T,3,2].

    Triangles come out cube by cube in cube order, and in table order inside a
    cube, which is the order the reference's prefix-sum layout produces.
    """
    ids = acc[:, :, 0].astype(np.int64)
    vals = corner_val[ids]
    ctype = np.zeros(ids.shape[0], dtype=np.int64)
    for i in range(8):
        ctype |= (vals[:, i] < 0).astype(np.int64) << i
    ntri = NUM_VERTS_TABLE[ctype] // 3
    cube = np.repeat(np.arange(ids.shape[0]), ntri)
    local = np.arange(cube.shape[0]) - np.repeat(np.cumsum(ntri) - ntri, ntri)
    if cube.shape[0] == 0:
        return np.zeros((0, 3, 3)), np.zeros((0, 3, 2), dtype=np.int32)
    tris = np.zeros((cube.shape[0], 3, 3))
    vids = np.zeros((cube.shape[0], 3, 2), dtype=np.int64)
    for j in range(3):
        e = TRI_TABLE[ctype[cube], 3 * local + j]
        a, b = MC_EDGES[e, 0], MC_EDGES[e, 1]
        ia, ib = ids[cube, a], ids[cube, b]
        tris[:, j] = _interp(corner_pos[ia], corner_pos[ib], vals[cube, a], vals[cube, b])
        vids[:, j, 0] = np.maximum(ia, ib)
        vids[:, j, 1] = np.minimum(ia, ib)
    return tris, vids.astype(np.int32)


@dataclass
class Mesh:
    vertices: np.ndarray
    faces: np.ndarray
    acc: np.ndarray = None
    dual_values: np.ndarray = None
    dual_pos: np.ndarray = None
    n_primal: dict = None
    mean_chi: float = 0.0


def extract_multiscale_mesh(sol: Solution, xyz32, n_upsample=2, max_depth=100) -> Mesh:
    """``Reconstructor.extract_multiscale_mesh`` (``reconstructor.py:296-397``), FP64 field."""
    grids = sol.grids
    max_depth = min(max_depth, len(grids))
    base, max_depth = conformal_leaves(grids, max_depth)
    ex = np.stack(np.meshgrid(*[np.arange(n_upsample)] * 3, indexing="ij"), -1).reshape(-1, 3)
    epb = {}
    for d in range(max_depth):
        s = grids[d].stride
        epb[d] = ((base[d] * n_upsample)[:, None, :] + (ex * s)[None]).reshape(-1, 3).astype(np.int32)
    cand = np.concatenate([epb[d] + off * grids[d].stride for d in range(max_depth) for off in CONFORM_OFFSETS], 0)
    dual = Grid(unique_rows(cand), 1)
    strides = {d: grids[d].stride for d in range(max_depth)}
    bases = {d: sum(epb[dd].shape[0] for dd in range(d)) for d in range(max_depth)}
    acc, cnt = dual_corner_indices(dual, epb, strides, bases)
    acc = acc[cnt == 8]
    evs = sol.vs / n_upsample
    pos64 = np.concatenate([(epb[d] + grids[d].stride).astype(np.float64) * evs for d in range(max_depth)], 0)
    pos32 = np.concatenate([((epb[d] + grids[d].stride).astype(F32) * F32(evs)).astype(F32)
                            for d in range(max_depth)], 0)
    mc = mean_chi(sol, xyz32)
    vals = evaluate_chi_raw(sol, pos32, pos64) - mc
    tris, vids = dual_marching_cubes(acc, pos64, vals)
    keys = vids.reshape(-1, 2).astype(np.int64)
    uk, inv = np.unique(keys[:, 0] << 32 | keys[:, 1], return_inverse=True)
    verts = np.zeros((uk.shape[0], 3))
    flat = tris.reshape(-1, 3)
    first = np.full(uk.shape[0], -1)
    order = np.arange(inv.shape[0])[::-1]
    first[inv[order]] = order
    verts = flat[first]
    return Mesh(verts, inv.reshape(-1, 3).astype(np.int64), acc=acc, dual_values=vals, dual_pos=pos64,
                n_primal={d: epb[d].shape[0] for d in epb}, mean_chi=mc)


def reconstruct(xyz, normal, voxel_size, depth=4, min_density=32.0, screen_alpha=4.0, cg_tol=None):
    """End-to-end oracle of ``jspsr.reconstruct`` (``jspsr/__init__.py:8-61``)."""
    xyz32 = np.asarray(xyz, dtype=F32)
    sol = solve_multigrid(xyz32, np.asarray(normal, dtype=F32), voxel_size, depth, min_density, screen_alpha,
                          cg_tol=cg_tol)
    mesh = extract_multiscale_mesh(sol, xyz32, n_upsample=2)
    return mesh, sol
