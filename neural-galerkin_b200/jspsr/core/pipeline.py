"""Device-resident screened-Poisson reconstruction on libngs kernels.

This is the B200 path behind ``jspsr.reconstruct`` (``jspsr/__init__.py:8-61`` of
the reference).  It keeps the reference's formulation step for step --
density-adaptive octree (``_hash_backend.py:414-444``), splatted normals
(``__init__.py:40-48``), coarse-to-fine Galerkin solve with cross-level
correction and screening (``reconstructor.py:79-195``), mean-chi level set and
multi-level dual marching cubes (``reconstructor.py:296-397``) -- but the data
structures are new:

* each level is a rank bitmap (``ngs_grid``): voxel rows are lexicographic ranks,
  so sorted coordinates, inverse maps and neighbour lookups need no sort and no hash;
* the level matrix is a CSR over the 5x5x5 stencil with a per-row offset mask; the
  screening Gram is added in place from the points (no pair hash table);
* the cross-level correction is matrix-free (stiffness by stencil lookups,
  screening through the coarse field at the points);
* each level is solved by one persistent PCG kernel (FP32 SpMV, FP64 dots,
  FP64 residual replacement / refinement).
"""
from __future__ import annotations

import math
import warnings
from dataclasses import dataclass, field

import numpy as np
import torch

from .. import _lib as L
from ..bases import tables as TB

CONFORM_OFFSETS = torch.tensor([(0, 0, 0), (0, 0, 1), (0, 1, 0), (0, 1, 1),
                                (1, 0, 0), (1, 0, 1), (1, 1, 0), (1, 1, 1)], dtype=torch.int32)


# ----------------------------------------------------------------------------- solver spec
@dataclass
class SolverSpec:
    """Parsed solver string, e.g. ``"pcg@tol=1e-7@maxiter=300"`` (grammar of ``solver.py:180-186``)."""
    name: str = "pcg-mixed"
    tol: float = 1.0e-7
    maxiter: int = -1
    res_fix: bool = False
    replace: int = 50
    timeout: float = 20.0

    @property
    def mode(self):
        return {"pcg": L.PCG_REFERENCE, "pcg-mixed": L.PCG_MIXED, "pcg-fp64": L.PCG_FP64,
                "plain-fp64": None}[self.name]


def parse_solver(spec: str) -> SolverSpec:
    """Parse ``name@key=value@...`` without ``eval``; ``cholmod`` / ``mixed`` map to an FP64 solve."""
    parts = spec.split("@")
    name = parts[0]
    out = SolverSpec(name=name)
    if name == "pcg":
        out.tol, out.maxiter = 1.0e-5, -1          # solver.py:192-196 defaults
    elif name in ("cholmod", "mixed"):
        out.name, out.tol, out.maxiter = "pcg-fp64", 1.0e-12, -1
    elif name not in ("pcg-mixed", "pcg-fp64", "plain-fp64"):
        raise NotImplementedError(f"unknown solver {name!r}")
    for kv in parts[1:]:
        k, v = kv.split("=", 1)
        k = k.strip()
        if k == "tol":
            out.tol = float(v)
        elif k == "maxiter":
            out.maxiter = int(float(v))
        elif k == "res_fix":
            out.res_fix = v.strip().lower() in ("1", "true", "yes")
        elif k == "replace":
            out.replace = int(v)
        elif k == "timeout":
            out.timeout = float(v)
        elif k == "verbose":
            pass
        else:
            raise ValueError(f"unknown solver option {k!r}")
    return out


# ----------------------------------------------------------------------------- levels
@dataclass
class Level:
    stride: int
    grid: L.Grid
    words: torch.Tensor
    coords: torch.Tensor = None
    n: int = 0
    # system
    masks: torch.Tensor = None
    rowptr: torch.Tensor = None
    cols: torch.Tensor = None
    vals64: torch.Tensor = None
    vals32: torch.Tensor = None
    diag_slot: torch.Tensor = None
    inv_diag: torch.Tensor = None
    nnz: int = 0
    rows: torch.Tensor = None      # point basis [N, 27]
    phi: torch.Tensor = None
    normals: torch.Tensor = None   # splatted normal data (points with this exact level)
    rhs: torch.Tensor = None
    x64: torch.Tensor = None
    x32: torch.Tensor = None
    info: torch.Tensor = None
    resid: torch.Tensor = None
    col_delta: torch.Tensor = None   # int16 column - row per non-zero (when every delta fits)
    delta_ok: bool = False
    band: int = 0                    # bound on |column - row| (decides the solver's shared-memory window)
    # matrix-free operator (solver reads no CSR): the point basis transposed per row
    group: tuple = None            # (sorted cell keys, point order): screening terms of long-pair levels
    pair_form: bool = False        # screening terms gathered per row from the transposed pairs
    mf: bool = False
    t_ptr: torch.Tensor = None      # [n + 1] int64
    t_point: torch.Tensor = None    # [E] int32
    t_phi: torch.Tensor = None      # [E] float32
    n_pairs: int = 0                # E
    max_pairs: int = 0              # longest row list
    stencil: torch.Tensor = None    # [125] FP64 same-level stiffness


def _box(qmin, qmax, stride, pad=1):
    """Cell box [lo, hi] (multiples of stride) covering the trilinear corners of points in [qmin, qmax]."""
    s = np.float32(stride)
    lo = (np.floor(qmin / s) * s).astype(np.int64) - pad * stride
    hi = (np.floor(qmax / s) * s).astype(np.int64) + pad * stride
    dims = (hi - lo) // stride + 1
    return lo, dims


@dataclass
class Timings:
    events: list = field(default_factory=list)

    def mark(self, name):
        e = torch.cuda.Event(enable_timing=True)
        e.record()
        self.events.append((name, e))

    def summary(self):
        torch.cuda.synchronize()
        out = {}
        for (n0, e0), (n1, e1) in zip(self.events[:-1], self.events[1:]):
            out[n1] = out.get(n1, 0.0) + e0.elapsed_time(e1)
        return out


class DualMesher:
    """The mesh stage shared by the device pipeline and the reference-API ``Reconstructor``: needs
    ``levels`` (objects with a ``stride``), ``vs``, ``dev`` and ``dual_grid_max_words``."""
    dual_grid_max_words = 1 << 27
    t = None

    def _mark(self, name):
        if self.t is not None:
            self.t.mark(name)

    def mesh_from_leaves(self, base: dict, max_depth: int, n_upsample: int, field):
        """Dual marching cubes over the conformal leaf cells ``base[d]`` (int32 [M_d, 3] per level):
        each cell expanded into n_upsample^3 samples, dual centres = the samples' unique corners, the 8
        primal samples of every dual cube accumulated through the dual grid, the field evaluated at
        the samples by ``field(positions)`` (values relative to the iso level), then the cubes'
        triangles and the vertex de-duplication (reconstructor.py:338-397)."""
        st = L.stream()
        dev = self.dev
        # expanded primal cells and their sample positions
        evs = np.float32(self.vs / n_upsample)
        e3 = n_upsample ** 3
        counts = [base[d].shape[0] * e3 for d in range(max_depth)]
        total = sum(counts)
        epb = torch.empty((total, 3), dtype=torch.int32, device=dev)
        pos = torch.empty((total, 3), dtype=torch.float32, device=dev)
        starts = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
        for d in range(max_depth):
            L.call("ngs_expand_cells", L.ptr(base[d]), base[d].shape[0], n_upsample, self.levels[d].stride, evs,
                   L.ptr(epb[starts[d]:]), L.ptr(pos[starts[d]:]), st)
        # dual centres: unique corners of all expanded cells
        # box of the corners actually present (the cells' extent, not the levels' padded boxes: with
        # many levels the coarse boxes would make the bitmap far larger than the surface needs)
        ext = []
        for d in range(max_depth):
            if counts[d] == 0:
                continue
            # the expanded cells of level d span base * n_up .. base * n_up + (n_up - 1) * stride, and
            # their corners one stride further: the extent follows from the (n_up^3 times fewer) cells
            c = base[d]
            s = self.levels[d].stride
            ext.append(torch.cat([c.min(0).values.long() * n_upsample, c.max(0).values.long() * n_upsample + n_upsample * s]))
        ext = torch.stack(ext).cpu().numpy()
        lo = ext[:, :3].min(0)
        hi = ext[:, 3:].max(0)
        dims = (hi - lo) + 1
        offs = L.device_table("conform_offsets", lambda: CONFORM_OFFSETS, dev)
        box_words = int(dims[0]) * int(dims[1]) * ((int(dims[2]) + 63) // 64)
        if box_words <= self.dual_grid_max_words:
            # rank bitmap over the box: dual centres ranked without a sort
            dg, dw = L.make_grid(lo, dims, 1, dev)
            for d in range(max_depth):
                if n_upsample == 2:
                    L.call("ngs_grid_mark_cell_corners", dg, L.ptr(base[d]), base[d].shape[0], self.levels[d].stride, st)
                else:
                    L.call("ngs_grid_mark_coords", dg, L.ptr(epb[starts[d]:]), counts[d], L.ptr(offs), 8,
                           self.levels[d].stride, st)
            dcount = torch.empty(1, dtype=torch.int64, device=dev)
            self._dual_ws = L.grid_finalize(dg, dw, dcount)
            nd = int(dcount.item())
            acc = torch.zeros((nd, 8), dtype=torch.int32, device=dev)
            cnt = torch.zeros(nd, dtype=torch.int32, device=dev)
            for d in range(max_depth):
                if n_upsample == 2 and self.levels[d].stride == 1:
                    L.call("ngs_dual_mc_indices_cells", dg, L.ptr(base[d]), base[d].shape[0], d, int(starts[d]),
                           L.ptr(acc), 1, L.ptr(cnt), st)
                else:
                    L.call("ngs_dual_mc_indices_grid", dg, L.ptr(epb[starts[d]:]), counts[d], self.levels[d].stride,
                           d, int(starts[d]), L.ptr(acc), 1, L.ptr(cnt), st)
        else:
            # deep hierarchies: the coarse cells stretch the box far beyond the surface, so the
            # dual centres are de-duplicated by a sort of packed corner keys and found through the
            # key table instead (the reference's own route, reconstructor.py:347-357)
            if np.any(dims >= (1 << 21)):
                raise ValueError(f"mesh domain of {dims.tolist()} cells exceeds 2^21 cells per axis")
            nd, table = self._dual_centres_by_sort(epb, starts, counts, max_depth, lo, offs)
            acc = torch.zeros((nd, 8), dtype=torch.int32, device=dev)
            cnt = torch.zeros(nd, dtype=torch.int32, device=dev)
            for d in range(max_depth):
                L.call("ngs_dual_mc_indices_hash", L.C.byref(table.table), L.ptr(epb[starts[d]:]), counts[d],
                       self.levels[d].stride, d, int(starts[d]), L.ptr(acc), 1, L.ptr(cnt), st)
            self._dual_ws = table
        # the cubes with all 8 corners (cnt == 8) are the reference's compacted list; nearly every
        # centre is one, so the count and emit passes skip the others in place instead of
        # compacting acc first (same triangles, same order); dual_cubes() compacts on request
        self.topology_overflow = cnt  # counts above 8 mark the reference's "Topology Error"
        self._mark("dual grid")
        # field at the primal samples
        vals = field(pos)
        self._mark("chi")
        verts, faces = self.marching_cubes(acc, cnt, pos, vals, total)
        self._mark("mesh")
        self.mesh_info = dict(n_primal=total, n_dual=nd, max_depth=max_depth, acc_ids=acc, cnt=cnt, values=vals,
                              positions=pos, counts=counts, starts=starts)
        return verts, faces

    def marching_cubes(self, acc, cnt, pos, vals, n_primal=None):
        """Dual marching cubes over the complete dual cubes (count 8) and vertex de-duplication by
        corner-id pair (dual_mc.cu:33-189, reconstructor.py:379-383): vertices [V, 3], faces [F, 3].
        ``vals`` are the field values at the primal samples ``pos`` (any source: the mesh of a field
        computed elsewhere goes through the same kernels)."""
        st, dev = L.stream(), self.dev
        nd = cnt.shape[0]
        total = pos.shape[0] if n_primal is None else n_primal
        vals = vals.contiguous().float()
        # marching cubes
        vcount = torch.empty(nd, dtype=torch.int32, device=dev)
        L.call("ngs_dual_mc_count", L.ptr(acc), 1, L.ptr(cnt), nd, L.ptr(vals), L.ptr(vcount), st)
        voff, vtot = L.scan(vcount)
        nv = int(vtot.item())
        tris = torch.empty((nv, 3), dtype=torch.float32, device=dev)
        vids = torch.empty((nv, 2), dtype=torch.int32, device=dev)
        L.call("ngs_dual_mc_emit", L.ptr(acc), 1, L.ptr(cnt), nd, L.ptr(pos), L.ptr(vals), L.ptr(voff), L.ptr(tris),
               L.ptr(vids), st)
        # vertex de-duplication by (vid0, vid1) (reconstructor.py:380-383)
        bcount = torch.zeros(total, dtype=torch.int32, device=dev)
        L.call("ngs_vdedup_count", L.ptr(vids), nv, L.ptr(bcount), st)
        bstart, _ = L.scan(bcount)
        fill = torch.zeros(total, dtype=torch.int32, device=dev)
        sorted_keys = torch.empty(nv, dtype=torch.int64, device=dev)
        first = torch.empty(nv, dtype=torch.int32, device=dev)
        L.call("ngs_vdedup_sort", L.ptr(vids), nv, L.ptr(bstart), total, L.ptr(fill), L.ptr(sorted_keys),
               L.ptr(first), st)
        vid_of, nvert_t = L.scan(first)
        nvert = int(nvert_t.item())
        faces = torch.empty(nv, dtype=torch.int64, device=dev)
        verts = torch.empty((nvert, 3), dtype=torch.float32, device=dev)
        L.call("ngs_vdedup_emit", L.ptr(vids), L.ptr(tris), nv, L.ptr(bstart), L.ptr(fill), L.ptr(sorted_keys),
               L.ptr(vid_of), L.ptr(faces), L.ptr(verts), st)
        self.mesh_vids = vids          # (larger, smaller) primal-sample pair of every triangle corner
        return verts, faces.view(-1, 3)

    def dual_cubes(self) -> torch.Tensor:
        """The complete dual cubes of the last extract_mesh (count 8), in dual-centre order: the
        reference's compacted [M, 8, 2] (primal id, depth) list (reconstructor.py:366)."""
        acc, cnt = self.mesh_info["acc_ids"], self.mesh_info["cnt"]
        nd = cnt.shape[0]
        st = L.stream()
        keep = torch.empty(nd, dtype=torch.int32, device=self.dev)
        L.call("ngs_dual_mc_select", L.ptr(cnt), nd, L.ptr(keep), st)
        koff, ktot = L.scan(keep)
        m = int(ktot.item())
        ids = torch.empty((m, 8), dtype=torch.int32, device=self.dev)
        L.call("ngs_dual_mc_compact", L.ptr(acc), 1, L.ptr(keep), L.ptr(koff), nd, L.ptr(ids), st)
        # the depth of a primal sample is the level whose segment holds its id
        bounds = torch.as_tensor(np.asarray(self.mesh_info["starts"][1:], dtype=np.int64), device=self.dev)
        depth = torch.bucketize(ids.long(), bounds, right=True).int()
        return torch.stack([ids, depth], dim=2)

    def _dual_centres_by_sort(self, epb, starts, counts, max_depth, lo, offs):
        """Unique corners of the expanded cells, in lexicographic order, and a key table over them."""
        from ..ext import HashLookupData, hash_cuda
        lo_t = torch.as_tensor(lo, dtype=torch.int64, device=self.dev)
        keys = []
        for d in range(max_depth):
            c = epb[starts[d]:starts[d] + counts[d]]
            if c.shape[0] == 0:
                continue
            corners = (c[:, None, :].long() + offs.long()[None] * self.levels[d].stride).reshape(-1, 3) - lo_t
            keys.append((corners[:, 0] << 42) | (corners[:, 1] << 21) | corners[:, 2])
        uk = torch.unique(torch.cat(keys))           # sorted: packed keys order like (x, y, z)
        mask = (1 << 21) - 1
        dual = (torch.stack([uk >> 42, (uk >> 21) & mask, uk & mask], 1) + lo_t).int()
        return int(uk.numel()), HashLookupData(hash_cuda(dual), None, False)



class Reconstruction(DualMesher):
    """One reconstruction, every buffer device-resident."""

    def __init__(self, xyz: torch.Tensor, normal: torch.Tensor, voxel_size: float, depth: int = 4,
                 min_density: float = 32.0, screen_alpha: float = 4.0, screen_delta: float = 0.1,
                 solver: str = "pcg-mixed@tol=1e-7", timings: Timings | None = None, operator: str = "csr"):
        L.require_cuda(xyz, "xyz")
        L.require_cuda(normal, "normal")
        self.xyz = xyz.contiguous().float()
        self.nrm = normal.contiguous().float()
        self.n = self.xyz.shape[0]
        if self.n == 0:
            raise ValueError("empty point cloud")
        self.vs = float(voxel_size)
        self.depth = int(depth)
        self.min_density = None if min_density is None else float(min_density)
        self.alpha = float(screen_alpha)
        self.delta = float(screen_delta)
        self.solver = parse_solver(solver)
        self.dev = self.xyz.device
        self.inv_vs = L.f32_inv(self.vs)
        self.levels: list[Level] = []
        self.t = timings
        self.solve_stats = {}
        self.profile_pcg = False
        self._pcg_events = {}
        self.solve_hook = None     # callable(rec, level, d, item): hands the level's PCG to a batcher
        # largest dual-grid rank bitmap (16-byte words) before the mesh switches to sorted keys
        self.dual_grid_max_words = 1 << 27
        # level operator of the solver: "csr" = the assembled matrix (the faster one on B200: one
        # streamed pass over stored entries per product); "matrix-free" = the stencil over the
        # bitmap plus the point form of the screening, on the levels where the point pairs are fewer
        # than the stiffness non-zeros (FP32-mixed and FP64 solvers)
        if operator not in ("csr", "matrix-free"):
            raise ValueError(f"operator must be 'csr' or 'matrix-free', not {operator!r}")
        self.operator = operator
        self.keep_csr = False      # also assemble the CSR of matrix-free levels (tests compare it)
        # longest pair list of a level whose screening terms go by rows from the transposed pairs (no
        # atomics, no sort); 0: every CSR level groups its points by cell (sort + FP64 atomics per cell
        # chunk), which measured faster on the 300k benchmark (30.5 ms per reconstruction, against 33.0
        # with the pair form on levels 0-2 and 49.0 on every level)
        self.pair_row_limit = 0

    def _mark(self, name):
        if self.t is not None:
            self.t.mark(name)

    # ------------------------------------------------------------------ tree
    def build_tree(self):
        """Density, point levels and the per-level rank bitmaps (_hash_backend.py:13-28,414-444)."""
        st = L.stream()
        self._mark("start")
        bbox = torch.empty(6, dtype=torch.float32, device=self.dev)
        L.call("ngs_points_bbox", L.ptr(self.xyz), self.n, L.ptr(bbox), st)
        b = bbox.cpu().numpy()
        self.bbox = b
        # density at voxel 4 * vs (hashtree.py:283-285): stride-1 grid of that voxel size
        vsd = 4.0 * self.vs
        inv_d = L.f32_inv(vsd)
        qd = [np.float32(b[:3]) * np.float32(inv_d), np.float32(b[3:]) * np.float32(inv_d)]
        lo, dims = _box(qd[0], qd[1], 1)
        gd, wd_words = L.make_grid(lo, dims, 1, self.dev)
        L.call("ngs_grid_mark_points", gd, L.ptr(self.xyz), self.n, np.float32(inv_d), None, 0, st)
        cnt = torch.empty(1, dtype=torch.int64, device=self.dev)
        L.grid_finalize(gd, wd_words, cnt)
        wd = torch.zeros(8 * self.n, dtype=torch.float32, device=self.dev)
        L.call("ngs_splat_weights", gd, L.ptr(self.xyz), self.n, np.float32(inv_d), vsd, L.ptr(wd), st)
        self.density = torch.empty(self.n, dtype=torch.float32, device=self.dev)
        self.point_level = torch.empty(self.n, dtype=torch.int32, device=self.dev)
        self.weight = torch.empty(self.n, dtype=torch.float32, device=self.dev)
        md = self.min_density if self.min_density is not None else 1.0
        L.call("ngs_density_eval", gd, L.ptr(self.xyz), self.n, np.float32(inv_d), vsd, L.ptr(wd),
               np.float32(md), self.depth, L.ptr(self.density), L.ptr(self.point_level), L.ptr(self.weight), st)
        if self.min_density is None:
            # data-dependent layering (no reference counterpart): the median density, so that the
            # denser half of the points sits on the finest level and no level is left empty.  It is
            # rounded down to a quarter power of two: the median itself is a point's density, and the
            # last bits of a density depend on the order of the splat's atomics, so an unrounded
            # threshold would put that point on either side from run to run.
            med = float(torch.median(self.density))
            md = 2.0 ** (math.floor(4.0 * math.log2(med)) / 4.0) if med > 0 else 1.0
            L.call("ngs_density_eval", gd, L.ptr(self.xyz), self.n, np.float32(inv_d), vsd, L.ptr(wd),
                   np.float32(md), self.depth, L.ptr(self.density), L.ptr(self.point_level), L.ptr(self.weight), st)
        self.min_density_used = md
        self._mark("density")
        # level grids
        q = [np.float32(b[:3]) * np.float32(self.inv_vs), np.float32(b[3:]) * np.float32(self.inv_vs)]
        counts = torch.empty(self.depth, dtype=torch.int64, device=self.dev)
        self._ws = []
        for d in range(self.depth):
            s = 2 ** d
            lo, dims = _box(q[0], q[1], s)
            g, words = L.make_grid(lo, dims, s, self.dev)
            L.call("ngs_grid_mark_points", g, L.ptr(self.xyz), self.n, np.float32(self.inv_vs),
                   L.ptr(self.point_level), d, st)
            self._ws.append(L.grid_finalize(g, words, counts[d:d + 1]))
            self.levels.append(Level(stride=s, grid=g, words=words))
        hist = torch.bincount(self.point_level.long(), minlength=self.depth)
        host = torch.cat([counts, hist]).cpu().numpy()
        self.level_hist = host[self.depth:]
        for d, lv in enumerate(self.levels):
            lv.n = int(host[d])
            if lv.n == 0:
                raise ValueError(f"level {d} of the hierarchy is empty; lower min_density")
            lv.coords = torch.empty((lv.n, 3), dtype=torch.int32, device=self.dev)
            L.call("ngs_grid_emit_coords", lv.grid, L.ptr(lv.coords), st)
        self._mark("tree")
        return self

    # ------------------------------------------------------------------ assembly
    def assemble(self):
        """Splat normals, point basis, and each level's operator: the CSR (stiffness + screening Gram)
        or the matrix-free form (stencil table + the point basis transposed per row)."""
        st = L.stream()
        inv = np.float32(self.inv_vs)
        mf_candidate = (self.operator == "matrix-free" and self.alpha > 0 and
                        self.solver.mode in (L.PCG_MIXED, L.PCG_FP64))
        pair_max = torch.zeros(self.depth, dtype=torch.int32, device=self.dev)
        for d, lv in enumerate(self.levels):
            if self.level_hist[d] > 0:
                lv.normals = torch.zeros((lv.n, 3), dtype=torch.float32, device=self.dev)
                L.call("ngs_splat_data", lv.grid, L.ptr(self.xyz), self.n, inv, self.vs, L.ptr(self.nrm), 3,
                       L.ptr(self.weight), L.ptr(self.point_level), d, np.float32(1.0 / lv.stride ** 3),
                       L.ptr(lv.normals), st)
            lv.rows = torch.empty((self.n, 27), dtype=torch.int32, device=self.dev)
            lv.phi = torch.empty((self.n, 27), dtype=torch.float32, device=self.dev)
            L.call("ngs_point_basis", lv.grid, L.ptr(self.xyz), self.n, inv, self.vs, L.ptr(lv.rows), L.ptr(lv.phi), st)
            lv.masks = torch.empty((lv.n, 4), dtype=torch.int32, device=self.dev)
            counts = torch.empty(lv.n, dtype=torch.int64, device=self.dev)
            L.call("ngs_stencil_count", lv.grid, L.ptr(lv.coords), lv.n, L.ptr(lv.masks), L.ptr(counts), st)
            lv.rowptr = torch.empty(lv.n + 1, dtype=torch.int64, device=self.dev)
            L.scan(counts, out=lv.rowptr[:lv.n], total=lv.rowptr[lv.n:])
            if self.alpha > 0 and (mf_candidate or self.pair_row_limit > 0):
                # (point, slot) pairs per row (the screening terms in gather form; their counts also
                # decide the matrix-free operator), the scan places the lists
                pc = torch.zeros(lv.n, dtype=torch.int32, device=self.dev)
                L.call("ngs_mf_count", L.ptr(lv.rows), self.n, lv.n, L.ptr(pc), L.ptr(pair_max[d:d + 1]), st)
                lv.t_ptr = torch.empty(lv.n + 1, dtype=torch.int64, device=self.dev)
                L.scan(pc, out=lv.t_ptr[:lv.n], total=lv.t_ptr[lv.n:])
        self._mark("structure")
        # with the non-zero counts, a bound on |column - row| per level (decides the 2-byte columns), and
        # the pair counts (decide the matrix-free operator): one synchronisation for all levels
        span = [self._row_span_bound(lv) for lv in self.levels]
        pairs = [lv.t_ptr[lv.n] if lv.t_ptr is not None else torch.zeros((), dtype=torch.int64, device=self.dev)
                 for lv in self.levels]
        host = torch.cat([torch.stack([lv.rowptr[lv.n] for lv in self.levels] + span + pairs),
                          pair_max.long()]).cpu().numpy()
        D = self.depth
        nnz, span, npairs, pmax = host[:D], host[D:2 * D], host[2 * D:3 * D], host[3 * D:]
        for d, lv in enumerate(self.levels):
            lv.nnz = int(nnz[d])
            lv.band = int(span[d])
            lv.n_pairs, lv.max_pairs = int(npairs[d]), int(pmax[d])
            # the point form costs 2 gathers per pair against one per stored non-zero; long lists
            # (millions of points per cell on coarse levels of large scenes) stay with the Gram
            lv.mf = bool(mf_candidate and 2 * lv.n_pairs <= lv.nnz and lv.max_pairs <= 4096)
            lv.stencil = L.device_table(("stencil125", lv.stride), lambda s=lv.stride: TB.stencil125(s), self.dev)
            # screening terms per row from the pairs, unless some row has so many (coarse levels of large
            # scenes: millions of points in one cell) that a row's serial walk would dominate -- those
            # levels group the points by cell instead (one sort, FP64 atomics per cell chunk)
            lv.pair_form = bool(self.alpha > 0 and lv.t_ptr is not None and
                                (lv.max_pairs <= self.pair_row_limit or lv.mf))
            if lv.pair_form:
                self._fill_pairs(lv)
            if lv.mf:
                self._assemble_mf(lv, d)
            if not lv.mf or self.keep_csr:
                # 2-byte column deltas where every |column - row| fits and the solver reads them
                # (the launches that stage the vector in shared memory)
                mode = self.solver.mode
                delta_ok = bool(span[d] <= 32767 and mode is not None and
                                L.load().ngs_pcg_window(lv.n, lv.nnz, lv.band, mode) == 1)
                self._assemble_csr(lv, d, delta_ok)
        self._mark("assembly")
        return self

    def _fill_pairs(self, lv: Level):
        """The point basis transposed per row: for every row, its (point, phi) pairs in point order."""
        st = L.stream()
        E = lv.n_pairs
        cursor = torch.zeros(lv.n, dtype=torch.int32, device=self.dev)
        tmp_point = torch.empty(E, dtype=torch.int32, device=self.dev)
        tmp_phi = torch.empty(E, dtype=torch.float32, device=self.dev)
        lv.t_point = torch.empty(E, dtype=torch.int32, device=self.dev)
        lv.t_phi = torch.empty(E, dtype=torch.float32, device=self.dev)
        L.call("ngs_mf_fill", L.ptr(lv.rows), L.ptr(lv.phi), self.n, L.ptr(lv.t_ptr), lv.n, L.ptr(cursor),
               L.ptr(tmp_point), L.ptr(tmp_phi), L.ptr(lv.t_point), L.ptr(lv.t_phi), st)

    def _assemble_mf(self, lv: Level, d: int):
        st = L.stream()
        lv.inv_diag = torch.empty(lv.n, dtype=torch.float32, device=self.dev)
        L.call("ngs_mf_diag", L.ptr(lv.t_ptr), L.ptr(lv.t_phi), lv.n, float(TB.stencil125(lv.stride)[62]),
               self._screen_scale(d), L.ptr(lv.inv_diag), st)

    def _screen_scale(self, d: int) -> float:
        """Screening weight of level d (reconstructor.py:122: alpha * (1/4)^d)."""
        return 0.25 ** d * self.alpha

    def _assemble_csr(self, lv: Level, d: int, delta_ok: bool):
        st = L.stream()
        lv.delta_ok = delta_ok
        lv.cols = torch.empty(lv.nnz, dtype=torch.int32, device=self.dev)
        lv.vals64 = torch.empty(lv.nnz, dtype=torch.float64, device=self.dev)
        lv.diag_slot = torch.empty(lv.n, dtype=torch.int64, device=self.dev)
        L.call("ngs_stencil_fill", lv.grid, L.ptr(lv.coords), lv.n, L.ptr(lv.masks), L.ptr(lv.rowptr),
               L.ptr(lv.stencil), L.ptr(lv.cols), L.ptr(lv.vals64), L.ptr(lv.diag_slot), st)
        if self.alpha > 0 and lv.pair_form:
            # the screening Gram by rows from the transposed pairs: no atomics, fixed summation order
            L.call("ngs_mf_gram", L.ptr(lv.t_ptr), L.ptr(lv.t_point), L.ptr(lv.t_phi), lv.n, L.ptr(lv.rows),
                   L.ptr(lv.phi), L.ptr(lv.masks), L.ptr(lv.rowptr), self._screen_scale(d), L.ptr(lv.vals64), st)
        elif self.alpha > 0:
            # group the points by cell: one FP64 atomic per (cell chunk, slot) instead of per point
            key = torch.empty(self.n, dtype=torch.int64, device=self.dev)
            L.call("ngs_point_cell_keys", L.ptr(lv.rows), self.n, L.ptr(key), st)
            keys, order = torch.sort(key)
            lv.group = (keys, order)          # reused by the screening RHS terms of this level
            L.call("ngs_screen_gram_grouped", L.ptr(lv.rows), L.ptr(lv.phi), self.n, None, L.ptr(order),
                   L.ptr(keys), L.ptr(lv.masks), L.ptr(lv.rowptr), self._screen_scale(d), L.ptr(lv.vals64), st)
        if lv.delta_ok:
            # 2-byte column deltas for the solver's SpMV (6 instead of 8 bytes per non-zero)
            lv.col_delta = torch.empty(lv.nnz, dtype=torch.int16, device=self.dev)
            L.call("ngs_csr_col_delta", L.ptr(lv.rowptr), L.ptr(lv.cols), lv.n, L.ptr(lv.col_delta), st)
        lv.vals32 = torch.empty(lv.nnz, dtype=torch.float32, device=self.dev)
        inv_diag = torch.empty(lv.n, dtype=torch.float32, device=self.dev)
        L.call("ngs_finish_system", L.ptr(lv.vals64), lv.nnz, L.ptr(lv.diag_slot), lv.n, L.ptr(lv.vals32),
               L.ptr(inv_diag), st)
        if not lv.mf:
            lv.inv_diag = inv_diag

    def mf_operator(self, lv: Level, d: int) -> "L.PcgOperator":
        """The C-ABI description of a matrix-free level (scratch for the per-point products included)."""
        op = L.PcgOperator()
        op.grid = lv.grid
        op.coords, op.stencil, op.alpha, op.n_points = lv.coords.data_ptr(), lv.stencil.data_ptr(), \
            self._screen_scale(d), self.n
        op.point_rows, op.point_phi = lv.rows.data_ptr(), lv.phi.data_ptr()
        op.t_ptr, op.t_point, op.t_phi = lv.t_ptr.data_ptr(), lv.t_point.data_ptr(), lv.t_phi.data_ptr()
        s32 = torch.empty(self.n, dtype=torch.float32, device=self.dev)
        s64 = torch.empty(self.n, dtype=torch.float64, device=self.dev)
        op.scratch32, op.scratch64 = s32.data_ptr(), s64.data_ptr()
        return op, (s32, s64)

    @staticmethod
    def _row_span_bound(lv: Level) -> torch.Tensor:
        """Device scalar (int64) >= max |column - row| of the level's 5^3-stencil matrix, from the rank
        bitmap alone (``ngs_grid_band_bound``: rows are ranks in (x, y, z) order, so the stencil of a
        voxel in column (x, y) reaches from the first row of column (x-2, y-2) to the last row of
        column (x+2, y+2)).  It decides the 2-byte column deltas and the solver's vector window."""
        out = torch.zeros((), dtype=torch.int64, device=lv.words.device)
        if lv.n > 0:
            L.call("ngs_grid_band_bound", lv.grid, lv.n, L.ptr(out), L.stream())
        return out

    # ------------------------------------------------------------------ RHS + solve
    def _rhs(self, d):
        st = L.stream()
        lv = self.levels[d]
        rhs = torch.zeros(lv.n, dtype=torch.float64, device=self.dev)
        for dd, ld in enumerate(self.levels):
            if ld.normals is None:
                continue
            tc = L.device_table(("rhs_c", ld.stride, lv.stride), lambda a=ld.stride, b=lv.stride: TB.rhs_tables(a, b)[0],
                                self.dev)
            tg = L.device_table(("rhs_g", ld.stride, lv.stride), lambda a=ld.stride, b=lv.stride: TB.rhs_tables(a, b)[1],
                                self.dev)
            L.call("ngs_rhs_normals", ld.grid, L.ptr(ld.coords), ld.n, L.ptr(ld.normals), lv.grid, L.ptr(lv.coords),
                   lv.n, L.ptr(tc), L.ptr(tg), tc.numel(), L.ptr(rhs), st)
        sf = 0.25 ** d
        if self.alpha > 0:
            self._screen_rhs(lv, None, sf * self.alpha * self.delta, rhs)
        coarser = list(range(self.depth - 1, d, -1))
        if coarser:
            if self.alpha > 0:
                fieldp = torch.zeros(self.n, dtype=torch.float32, device=self.dev)
                for dd in coarser:
                    lc = self.levels[dd]
                    L.call("ngs_point_field", L.ptr(lc.rows), L.ptr(lc.phi), self.n, L.ptr(lc.x32), L.ptr(fieldp), 1, st)
                self._screen_rhs(lv, fieldp, -sf * self.alpha, rhs)
            for dd in coarser:
                lc = self.levels[dd]
                tc = L.device_table(("corr_c", lv.stride, lc.stride),
                                    lambda a=lv.stride, b=lc.stride: TB.correction_tables(a, b)[0], self.dev)
                tg = L.device_table(("corr_g", lv.stride, lc.stride),
                                    lambda a=lv.stride, b=lc.stride: TB.correction_tables(a, b)[1], self.dev)
                L.call("ngs_correction_stiffness", L.ptr(lv.coords), lv.n, lv.stride, lc.grid, L.ptr(lc.x32),
                       L.ptr(tc), L.ptr(tg), tc.numel(), L.ptr(rhs), st)
        lv.rhs = rhs
        return rhs

    def _screen_rhs(self, lv: Level, val, scale: float, rhs: torch.Tensor):
        """rhs += scale * sum over the level's points of phi * (val[point] or 1): gathered per row from the
        transposed pairs (no atomics), or through the cell-grouped points on long-pair levels."""
        st = L.stream()
        if lv.pair_form:
            L.call("ngs_mf_screen_rhs", L.ptr(lv.t_ptr), L.ptr(lv.t_point), L.ptr(lv.t_phi), lv.n,
                   L.ptr(val) if val is not None else None, scale, L.ptr(rhs), st)
        else:
            keys, order = lv.group
            L.call("ngs_screen_rhs_grouped", L.ptr(lv.rows), L.ptr(lv.phi), self.n, None,
                   L.ptr(val) if val is not None else None, L.ptr(order), L.ptr(keys), scale, L.ptr(rhs), st)

    def pcg_item(self, lv: Level) -> "L.PcgBatchItem":
        """Output buffers, workspace and the C-ABI description of one level's PCG solve."""
        spec = self.solver
        lv.x32 = torch.empty(lv.n, dtype=torch.float32, device=self.dev)
        lv.x64 = torch.empty(lv.n, dtype=torch.float64, device=self.dev)
        lv.info = torch.zeros(4, dtype=torch.int64, device=self.dev)
        lv.resid = torch.zeros(2, dtype=torch.float64, device=self.dev)
        item = L.PcgBatchItem()
        sysd = item.sys
        sysd.n, sysd.inv_diag = lv.n, lv.inv_diag.data_ptr()
        keep = []
        if lv.mf:
            op, scratch = self.mf_operator(lv, next(d for d, l in enumerate(self.levels) if l is lv))
            sysd.op = L.C.pointer(op)
            sysd.nnz = 60 * lv.n + 2 * lv.n_pairs          # work of one application (block count)
            b32 = None
            keep += [op, scratch]
        else:
            sysd.nnz = lv.nnz
            sysd.rowptr, sysd.cols = lv.rowptr.data_ptr(), lv.cols.data_ptr()
            sysd.vals32, sysd.vals64 = lv.vals32.data_ptr(), lv.vals64.data_ptr()
            b32 = lv.rhs.float()
            sysd.b32 = b32.data_ptr()
            sysd.col_delta = lv.col_delta.data_ptr() if lv.col_delta is not None else None
            sysd.band = lv.band
        sysd.b64 = lv.rhs.data_ptr()
        sysd.x32, sysd.x64 = lv.x32.data_ptr(), lv.x64.data_ptr()
        cfg = item.cfg
        cfg.mode, cfg.max_iter, cfg.tol = spec.mode, spec.maxiter, spec.tol
        cfg.res_fix, cfg.replace_every, cfg.blocks, cfg.timeout_s = int(spec.res_fix), spec.replace, 0, spec.timeout
        ws_bytes = L.load().ngs_pcg_workspace_bytes(lv.n, spec.mode)
        ws = torch.empty(ws_bytes, dtype=torch.uint8, device=self.dev)
        item.ws, item.ws_bytes = ws.data_ptr(), ws_bytes
        item.info_dev, item.resid_dev = lv.info.data_ptr(), lv.resid.data_ptr()
        lv._keep = (ws, b32, *keep)
        return item

    def _solve_level(self, lv: Level, d: int = 0):
        spec = self.solver
        if spec.mode is None:
            lv.x32 = torch.empty(lv.n, dtype=torch.float32, device=self.dev)
            lv.info = torch.zeros(4, dtype=torch.int64, device=self.dev)
            lv.resid = torch.zeros(2, dtype=torch.float64, device=self.dev)
            if self.profile_pcg:
                ev = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                ev[0].record()
            self._solve_plain_fp64(lv)
            if self.profile_pcg:
                ev[1].record()
                self._pcg_events[d] = ev
            return
        item = self.pcg_item(lv)
        if self.solve_hook is not None:
            # batched solve: returns once the solve is enqueued and this stream waits for it
            self.solve_hook(self, lv, d, item)
        else:
            if self.profile_pcg:
                ev = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                ev[0].record()
            L.call("ngs_pcg_solve", L.C.byref(item.sys), L.C.byref(item.cfg), item.ws, item.ws_bytes, item.info_dev,
                   item.resid_dev, L.stream())
            if self.profile_pcg:
                ev[1].record()
                self._pcg_events[d] = ev
        if spec.mode == L.PCG_REFERENCE:
            lv.x64 = lv.x32.double()

    def _solve_plain_fp64(self, lv: Level):
        """Host-driven FP64 Jacobi-PCG, one launch per vector op and a host check per iteration --
        the 'plain GPU' comparator following the reference loop (solve_pcg.cu:80-128)."""
        spec, st, n = self.solver, L.stream(), lv.n
        A = (lv.rowptr, lv.cols, lv.vals64)
        dinv = (1.0 / lv.vals64[lv.diag_slot])
        b = lv.rhs
        x = torch.zeros(n, dtype=torch.float64, device=self.dev)
        r = b.clone()
        p = torch.zeros_like(x)
        q = torch.empty_like(x)
        z = torch.empty_like(x)
        dot = torch.empty(1, dtype=torch.float64, device=self.dev)

        def dotv(a, c):
            L.call("ngs_dot64", L.ptr(a), L.ptr(c), n, L.ptr(dot), st)
            return float(dot.item())
        atol = spec.tol * math.sqrt(dotv(b, b))
        rho, it = 0.0, 0
        cap = 20000 if spec.maxiter < 0 else min(spec.maxiter, 20000)
        while it < cap:
            L.call("ngs_mul64", n, L.ptr(dinv), L.ptr(r), L.ptr(z), st)
            rho1, rho = rho, dotv(r, z)
            if it == 0:
                p.copy_(z)
            else:
                L.call("ngs_axpby64", n, 1.0, L.ptr(z), rho / rho1, L.ptr(p), st)
            L.call("ngs_spmv64", n, L.ptr(A[0]), L.ptr(A[1]), L.ptr(A[2]), L.ptr(p), L.ptr(q), st)
            alpha = rho / dotv(p, q)
            L.call("ngs_axpby64", n, alpha, L.ptr(p), 1.0, L.ptr(x), st)
            L.call("ngs_axpby64", n, -alpha, L.ptr(q), 1.0, L.ptr(r), st)
            it += 1
            if math.sqrt(dotv(r, r)) <= atol:
                break
        lv.x64 = x
        lv.x32.copy_(x)
        res = math.sqrt(dotv(r, r))
        lv.info[0] = it
        lv.info[1] = L.NGS_OK if res <= atol else L.NGS_ERR_NOT_CONVERGED
        lv.resid[0] = res
        lv.resid[1] = atol / spec.tol if spec.tol > 0 else 0.0

    def solve(self):
        """Coarse-to-fine solve (reconstructor.py:122-189)."""
        for d in range(self.depth - 1, -1, -1):
            self._rhs(d)
            self._mark(f"rhs{d}")
            self._solve_level(self.levels[d], d)
            self._mark(f"pcg{d}")
        self._queue_status()
        return self

    _status_checked = False

    def _queue_status(self):
        """Copy every level's solve record to pinned host memory behind the solves, without waiting:
        the mesh extraction synchronises with the device anyway, after which the copy has landed."""
        self._status_checked = False
        rec = torch.cat([torch.cat([lv.info.double(), lv.resid]) for lv in self.levels])
        self._status_host = torch.empty(rec.shape, dtype=torch.float64, pin_memory=True)
        self._status_host.copy_(rec, non_blocking=True)
        self._status_event = torch.cuda.Event()
        self._status_event.record()

    def check_solves(self):
        """Iteration counts and status of every level; raises ``NgsError`` when a solve failed.

        A solve that gave up (a bounded device wait ran out: NGS_ERR_TIMEOUT), was handed an invalid
        system, or stopped at the library's own iteration cap without reaching the tolerance raises.
        A solve that stopped at a ``maxiter`` the caller asked for keeps the reference's behaviour
        (``solver.py:138-143``: the result is returned and the residual reported) with a warning."""
        if getattr(self, "_status_host", None) is None:
            self._queue_status()
        self._status_event.synchronize()
        self._status_checked = True
        rec = self._status_host.numpy().reshape(self.depth, 6)
        self.solve_stats = {d: dict(iters=int(rec[d, 0]), status=int(rec[d, 1]), replacements=int(rec[d, 2]),
                                    resid=float(rec[d, 4]), bnorm=float(rec[d, 5])) for d in range(self.depth)}
        for d, s in self.solve_stats.items():
            if s["status"] == L.NGS_OK:
                continue
            if s["status"] == L.NGS_ERR_NOT_CONVERGED and self.solver.maxiter >= 0:
                warnings.warn(f"PCG level {d} stopped at maxiter={self.solver.maxiter} with residual "
                              f"{s['resid']:.3e} (|b| = {s['bnorm']:.3e})", RuntimeWarning, stacklevel=3)
                continue
            raise L.NgsError(s["status"], f"PCG level {d}")
        return self.solve_stats

    @property
    def pcg_ms(self):
        """Device time of each level's PCG launch (needs profile_pcg = True before solve)."""
        torch.cuda.synchronize()
        return {d: e[0].elapsed_time(e[1]) for d, e in self._pcg_events.items()}

    # ------------------------------------------------------------------ field
    def chi_raw(self, pos: torch.Tensor, grad: bool = False) -> torch.Tensor:
        """Sum over levels of the interpolated field at positions (reconstructor.py:197-226)."""
        pos = pos.contiguous().float()
        out = torch.zeros((pos.shape[0], 3) if grad else pos.shape[0], dtype=torch.float32, device=self.dev)
        for l0 in range(0, len(self.levels), L.MAX_FIELD_LEVELS):
            lvs = self.levels[l0:l0 + L.MAX_FIELD_LEVELS]
            grids = (L.Grid * len(lvs))(*[lv.grid for lv in lvs])
            xs = (L.C.c_void_p * len(lvs))(*[lv.x32.data_ptr() for lv in lvs])
            L.call("ngs_eval_field_levels", grids, xs, len(lvs), L.ptr(pos), pos.shape[0], np.float32(self.inv_vs),
                   self.vs, int(grad), L.ptr(out), L.stream())
        return out

    def chi_cells(self, pos: torch.Tensor) -> torch.Tensor:
        """chi_raw at the 2x2x2 samples of leaf cells, 8 per cell in expansion order (what
        ngs_expand_cells writes with n_upsample = 2).  The samples of one cell share the
        neighbourhood of every field level at least half as fine as the cell, read once per cell."""
        out = torch.zeros(pos.shape[0], dtype=torch.float32, device=self.dev)
        for l0 in range(0, len(self.levels), L.MAX_FIELD_LEVELS):
            lvs = self.levels[l0:l0 + L.MAX_FIELD_LEVELS]
            grids = (L.Grid * len(lvs))(*[lv.grid for lv in lvs])
            xs = (L.C.c_void_p * len(lvs))(*[lv.x32.data_ptr() for lv in lvs])
            L.call("ngs_eval_field_cells", grids, xs, len(lvs), pos.shape[0] // 8, L.ptr(pos),
                   np.float32(self.inv_vs), self.vs, L.ptr(out), L.stream())
        return out

    def mean_chi(self) -> torch.Tensor:
        """Density-weighted mean of chi at the input points (reconstructor.py:228-236), as a device scalar."""
        chi = torch.zeros(self.n, dtype=torch.float32, device=self.dev)
        for lv in self.levels:
            L.call("ngs_point_field", L.ptr(lv.rows), L.ptr(lv.phi), self.n, L.ptr(lv.x32), L.ptr(chi), 1, L.stream())
        sums = torch.empty(2, dtype=torch.float64, device=self.dev)
        L.call("ngs_weighted_sum", L.ptr(chi), L.ptr(self.weight), self.n, L.ptr(sums), L.stream())
        self.chi_points = chi
        return (sums[0] / sums[1]).float()

    # ------------------------------------------------------------------ mesh
    def extract_mesh(self, n_upsample: int = 2):
        """Multi-level dual marching cubes (reconstructor.py:296-397)."""
        st = L.stream()
        dev = self.dev
        mean = self.mean_chi()
        max_depth = self.depth
        q = [np.float32(self.bbox[:3]) * np.float32(self.inv_vs), np.float32(self.bbox[3:]) * np.float32(self.inv_vs)]
        base, leaf_flags, parent_grids = {}, {}, {}
        # parents at 2s of every level's voxels (but the coarsest), their counts read in one go
        pcount = torch.empty(max(max_depth - 1, 1), dtype=torch.int64, device=dev)
        for d in range(max_depth - 1):
            lv = self.levels[d]
            lo, dims = _box(q[0], q[1], 2 * lv.stride, pad=2)
            pg, pw = L.make_grid(lo, dims, 2 * lv.stride, dev)
            L.call("ngs_grid_mark_coords", pg, L.ptr(lv.coords), lv.n, None, 1, 0, st)
            parent_grids[d] = (pg, pw, L.grid_finalize(pg, pw, pcount[d:d + 1]))
        npar = pcount.cpu().numpy()
        if not self._status_checked:
            # first synchronisation after the solves: their status copy has landed; a failed solve
            # raises here, before any mesh is built from its result
            self.check_solves()
        # each level's cells: all 8 children of its parents (the coarsest level: its voxels), and on
        # levels above 0 the flags of the leaves among them; the leaf counts read in one go
        ltot = []
        for d in range(max_depth):
            if d < max_depth - 1:
                pg = parent_grids[d][0]
                parents = torch.empty((int(npar[d]), 3), dtype=torch.int32, device=dev)
                L.call("ngs_grid_emit_coords", pg, L.ptr(parents), st)
                cells = torch.empty((int(npar[d]) * 8, 3), dtype=torch.int32, device=dev)
                L.call("ngs_conformal_children", L.ptr(parents), int(npar[d]), self.levels[d].stride, L.ptr(cells), st)
            else:
                cells = self.levels[d].coords
            if d > 0:
                leaf = torch.empty(cells.shape[0], dtype=torch.int32, device=dev)
                L.call("ngs_leaf_flags", L.ptr(cells), cells.shape[0], parent_grids[d - 1][0], L.ptr(leaf), st)
                off, tot = L.scan(leaf)
                leaf_flags[d] = (leaf, off)
                ltot.append(tot)
            base[d] = cells
        nleaf = torch.cat(ltot).cpu().numpy() if ltot else np.zeros(0, np.int64)
        for d in range(1, max_depth):
            if int(nleaf[d - 1]) == 0:          # no leaves from level d on: the mesh stops at d - 1
                max_depth = d
                break
        for d in range(1, max_depth):
            leaf, off = leaf_flags[d]
            out = torch.empty((int(nleaf[d - 1]), 3), dtype=torch.int32, device=dev)
            L.call("ngs_compact_coords", L.ptr(base[d]), L.ptr(leaf), L.ptr(off), base[d].shape[0], L.ptr(out), st)
            base[d] = out
        self._mark("leaves")
        field = (lambda pos: self.chi_cells(pos) - mean) if n_upsample == 2 else (lambda pos: self.chi_raw(pos) - mean)
        return self.mesh_from_leaves(base, max_depth, n_upsample, field)

    def run(self, n_upsample: int = 2):
        self.build_tree().assemble().solve()
        mesh = self.extract_mesh(n_upsample)
        if not self._status_checked:
            self.check_solves()        # the mesh extraction has synchronised: no extra wait
        return mesh
