"""Multi-level sparse voxel hierarchy on libngs rank bitmaps (reference API: ``jspsr/core/_hash_backend.py``).

The reference keeps, per level, a coordinate list and a GPU cuckoo table, and answers every
neighbour query by materialising a [K, N] key matrix, probing the table and compacting with
``torch.where``.  Here each level is a :class:`VoxelLevel`: its coordinates in lexicographic order
and a rank bitmap over its lattice (one bit per cell, per-word prefix counts), so that

* a voxel's row is its rank -- sorted coordinates come out of the bitmap, not out of a sort;
* a neighbour query is one fused kernel pair (``ngs_grid_neighbours_count / _fill``): probe each
  (source, offset) in the L2-resident bitmap, keep one bit per pair, scan the counts, write every
  hit to its slot in the reference's order (offset-major, or source-major when transposed);
* lookups of explicit coordinates (splat corners, children, voxel status) are single probes.

Public names and signatures are the reference's; ``SparseFeatureHierarchy`` keeps its semantics
(per-level strides 2^d, coordinates in finest-voxel units, the prefix property of the range
kernel, the coarse-to-fine inversion of region queries) on this storage.
"""
from __future__ import annotations

from typing import Callable, Dict, List, Optional, Tuple

import numpy as np
import torch

from .. import _lib as L

# the 8 trilinear corners, x-major (the corner order of the reference's splat weights)
CORNERS = torch.tensor([(x, y, z) for x in (0, 1) for y in (0, 1) for z in (0, 1)], dtype=torch.int32)
CONFORM = tuple(tuple(int(v) for v in r) for r in CORNERS.tolist())


def range_kernel(n: int, device=None) -> torch.Tensor:
    """Neighbour offsets int32 [n^3, 3] ordered by Chebyshev shell, lexicographic inside a shell.

    Stands in for the unpublished ``data/kernel.npz`` of ``hashtree.py:103-116``; the order within a
    shell only changes summation order, while the prefix property (the first 1 / 27 / 125 offsets are
    radius 0 / 1 / 2) is what lets a pair list of a larger range be cut down to a smaller one."""
    assert n % 2 == 1, "target_range must be odd."
    r = n // 2
    ax = torch.arange(-r, r + 1)
    g = torch.cartesian_prod(ax, ax, ax)
    shell = g.abs().max(1).values
    key = ((shell * (n + 1) + (g[:, 0] + r)) * (n + 1) + (g[:, 1] + r)) * (n + 1) + (g[:, 2] + r)
    return g[torch.argsort(key)].to(dtype=torch.int32, device=device)


# ----------------------------------------------------------------------------- one level
class VoxelLevel:
    """Voxels of one lattice (pitch ``stride``) with a rank bitmap over their bounding box."""

    def __init__(self, coords: torch.Tensor, stride: int):
        self.stride = int(stride)
        self.coords = coords.to(torch.int32).contiguous()
        self.device = self.coords.device
        self.row_of_rank = None
        n = self.coords.shape[0]
        if n == 0:
            self.grid, self.words = L.null_grid(), None
            return
        lo = (self.coords.min(0).values // self.stride * self.stride).cpu().numpy().astype(np.int64)
        hi = self.coords.max(0).values.cpu().numpy().astype(np.int64)
        self.grid, self.words = L.make_grid(lo, (hi - lo) // self.stride + 1, self.stride, self.device)
        st = L.stream()
        L.call("ngs_grid_mark_coords", self.grid, L.ptr(self.coords), n, None, 1, 0, st)
        count = torch.empty(1, dtype=torch.int64, device=self.device)
        self._ws = L.grid_finalize(self.grid, self.words, count)
        # rows of the given list: identical to the ranks when the list is sorted and unique (every
        # builder here produces that); otherwise a rank -> row table, the first row of a repeated
        # coordinate winning (what a hash table keyed by coordinate would return)
        rank = torch.empty(n, dtype=torch.int64, device=self.device)
        L.call("ngs_grid_lookup", self.grid, L.ptr(self.coords), n, L.ptr(rank), st)
        ident = torch.arange(n, device=self.device)
        if int(count.item()) != n or not bool(torch.equal(rank, ident)):
            table = torch.full((int(count.item()),), n, dtype=torch.int64, device=self.device)
            table.scatter_reduce_(0, rank, ident, reduce="amin")
            self.row_of_rank = table

    def __len__(self):
        return self.coords.shape[0]

    # ------------------------------------------------------------------ queries
    def probe(self, coords: torch.Tensor) -> torch.Tensor:
        """Row of each coordinate (int32 [M, 3]), -1 where absent or off this level's lattice."""
        m = coords.shape[0]
        if m == 0 or len(self) == 0:
            return torch.full((m,), -1, dtype=torch.int64, device=self.device)
        c = coords.to(torch.int32).contiguous()
        rank = torch.empty(m, dtype=torch.int64, device=self.device)
        L.call("ngs_grid_lookup", self.grid, L.ptr(c), m, L.ptr(rank), L.stream())
        origin = torch.tensor(list(self.grid.origin), dtype=torch.int32, device=self.device)
        on_lattice = ((c - origin) % self.stride == 0).all(1)
        rank = torch.where(on_lattice, rank, torch.full_like(rank, -1))
        if self.row_of_rank is None:
            return rank
        return torch.where(rank >= 0, self.row_of_rank[rank.clamp(min=0)], rank)

    def neighbours(self, src: torch.Tensor, src_stride: int, offsets: torch.Tensor, conv: bool, transposed: bool):
        """Fused query: every (source, offset) whose probe hits a voxel of this level.

        Returns ``(src_ids, tgt_ids, kidx, counts)``: int64 source and target rows, int32 offset
        indices, and counts per offset (offset-major order) or per source (source-major order)."""
        n, k = src.shape[0], offsets.shape[0]
        dev = self.device
        counts_len = n if transposed else k
        empty = (torch.zeros(0, dtype=torch.int64, device=dev), torch.zeros(0, dtype=torch.int64, device=dev),
                 torch.zeros(0, dtype=torch.int32, device=dev), torch.zeros(counts_len, dtype=torch.int64, device=dev))
        if n == 0 or len(self) == 0:
            return empty
        lib = L.load()
        src = src.contiguous()
        is_float = src.dtype != torch.int32
        if is_float:
            src = src.float().contiguous()
        off = offsets.to(torch.int32).contiguous()
        tiles = lib.ngs_grid_neighbours_tiles(n)
        masks = torch.empty((n, 4), dtype=torch.int32, device=dev)
        st = L.stream()
        args = (self.grid, L.ptr(self.row_of_rank), L.ptr(src), int(is_float), n, int(src_stride), int(conv),
                L.ptr(off), k, int(transposed))
        if transposed:
            counts = torch.empty(n, dtype=torch.int64, device=dev)
            L.call("ngs_grid_neighbours_count", *args, L.ptr(masks), None, None, L.ptr(counts), st)
            start, total = L.scan(counts)
        else:
            tile_counts = torch.empty(k * tiles, dtype=torch.int64, device=dev)
            counts = torch.empty(k, dtype=torch.int64, device=dev)
            L.call("ngs_grid_neighbours_count", *args, L.ptr(masks), L.ptr(tile_counts), L.ptr(counts), None, st)
            start, total = L.scan(tile_counts)
        p = int(total.item())
        src_ids = torch.empty(p, dtype=torch.int64, device=dev)
        tgt_ids = torch.empty(p, dtype=torch.int64, device=dev)
        kidx = torch.empty(p, dtype=torch.int32, device=dev)
        if p:
            L.call("ngs_grid_neighbours_fill", *args, L.ptr(masks), L.ptr(start), L.ptr(src_ids), L.ptr(tgt_ids),
                   L.ptr(kidx), st)
        return src_ids, tgt_ids, kidx, counts


# ----------------------------------------------------------------------------- builders
def corner_cells(xyz: torch.Tensor, voxel_size: float, stride: int, select: Optional[torch.Tensor] = None):
    """Sorted unique trilinear corner cells (stride ``stride``) of the points, or of those with
    ``select`` true: the voxel set of a level (``_hash_backend.py:457-462``).  Marked straight into a
    rank bitmap by ``ngs_grid_mark_points`` (the reference's fp32 quantisation of xyz / vs)."""
    dev = xyz.device
    if select is not None:
        xyz = xyz[select]
    if xyz.shape[0] == 0:
        return torch.zeros((0, 3), dtype=torch.int32, device=dev)
    xyz = xyz.float().contiguous()
    inv = L.f32_inv(voxel_size)
    q = xyz.detach() * np.float32(inv)
    s = int(stride)
    lo = (torch.floor(q.min(0).values / s) * s).cpu().numpy().astype(np.int64) - s
    hi = (torch.floor(q.max(0).values / s) * s).cpu().numpy().astype(np.int64) + s
    g, words = L.make_grid(lo, (hi - lo) // s + 1, s, dev)
    st = L.stream()
    L.call("ngs_grid_mark_points", g, L.ptr(xyz), xyz.shape[0], np.float32(inv), None, 0, st)
    cnt = torch.empty(1, dtype=torch.int64, device=dev)
    ws = L.grid_finalize(g, words, cnt)
    out = torch.empty((int(cnt.item()), 3), dtype=torch.int32, device=dev)
    L.call("ngs_grid_emit_coords", g, L.ptr(out), st)
    del ws
    return out


def unique_cells(coords: torch.Tensor) -> torch.Tensor:
    """Sorted unique rows of int32 [N, 3] cell coordinates (through a rank bitmap, no sort)."""
    from .ops import torch_unique
    if coords.shape[0] == 0:
        return coords.reshape(0, 3).to(torch.int32)
    return torch_unique(coords.to(torch.int32).contiguous(), dim=0)


def trilinear(xyz: torch.Tensor, voxel_size: float, stride: int, data=1, compute_grad: bool = False):
    """Corner cells and weights of trilinear interpolation at stride ``stride``
    (``_hash_backend.py:469-510``): corner-major [8 N, 3] cells, [8 N] or [8 N, C] weights and, with
    ``compute_grad``, [8 N, 3] weight gradients w.r.t. the position.  Evaluated for all eight corners
    at once: per axis the point's cell d, the side sign of the point within it, and the distance
    ``loc`` to the cell centre in cells; corner c takes (1 - loc) or loc per axis by its bit."""
    q = xyz / voxel_size
    d = torch.floor(q / stride) * stride
    off = q - d - stride / 2.0
    sign = torch.sign(off)
    loc = off.abs() / stride                                       # [N, 3]
    bits = CORNERS.to(xyz.device)                                  # [8, 3]
    cells = (d[None] + bits[:, None, :] * sign[None] * stride).int().reshape(-1, 3)
    f = torch.where(bits[:, None, :].bool(), loc[None], 1 - loc[None])          # [8, N, 3]
    w = f[..., 0] * f[..., 1] * f[..., 2]                          # [8, N]
    if isinstance(data, torch.Tensor):
        w = w[..., None] * data[None] if data.dim() > 1 else w * data[None]
        w = w.reshape((-1,) + tuple(w.shape[2:]))
    else:
        w = (w * data).reshape(-1)
    if not compute_grad:
        return cells, w
    assert not isinstance(data, torch.Tensor) and data == 1, "Not supported!"
    df = torch.where(bits[:, None, :].bool(), sign[None], -sign[None]) / (voxel_size * stride)   # d f / d x
    grad = torch.stack([df[..., 0] * f[..., 1] * f[..., 2], f[..., 0] * df[..., 1] * f[..., 2],
                        f[..., 0] * f[..., 1] * df[..., 2]], -1).reshape(-1, 3)
    return cells, w, grad


def compute_density(xyz: torch.Tensor, voxel_size: float) -> torch.Tensor:
    """Kernel density of the points: trilinear splat of ones onto the stride-1 lattice of
    ``voxel_size`` (all 8 corners of every point exist there), then the B-spline interpolation of
    those weights at the points (``_hash_backend.py:13-28``).  Runs the libngs density kernels
    (``ngs_splat_weights``, ``ngs_density_eval``) on the points' own bitmap; returns the KDE value
    (the reference divides by 16 at ``hashtree.py:283-285``, as its caller here does)."""
    xyz = xyz.detach().float().contiguous()
    dev, n = xyz.device, xyz.shape[0]
    if n == 0:
        return torch.zeros(0, device=dev)
    inv = L.f32_inv(voxel_size)
    q = xyz * np.float32(inv)
    lo = torch.floor(q.min(0).values).cpu().numpy().astype(np.int64) - 1
    hi = torch.floor(q.max(0).values).cpu().numpy().astype(np.int64) + 1
    g, words = L.make_grid(lo, hi - lo + 1, 1, dev)
    st = L.stream()
    L.call("ngs_grid_mark_points", g, L.ptr(xyz), n, np.float32(inv), None, 0, st)
    cnt = torch.empty(1, dtype=torch.int64, device=dev)
    ws = L.grid_finalize(g, words, cnt)
    wd = torch.zeros(8 * n, dtype=torch.float32, device=dev)
    L.call("ngs_splat_weights", g, L.ptr(xyz), n, np.float32(inv), float(voxel_size), L.ptr(wd), st)
    dens = torch.empty(n, dtype=torch.float32, device=dev)
    L.call("ngs_density_eval", g, L.ptr(xyz), n, np.float32(inv), float(voxel_size), L.ptr(wd), np.float32(1.0), 1,
           L.ptr(dens), None, None, st)
    del ws
    return dens * 16.0


# ----------------------------------------------------------------------------- pair-list cache
class NeighbourMaps:
    """Pair lists between two levels, kept per (source, target, kind) at the largest range asked so
    far.  Lists are offset-major with counts per offset, and the range kernel has the prefix
    property, so the list of a smaller range is the prefix that its first r^3 offsets cover; a larger
    range is queried afresh (one fused query) and replaces the entry."""

    def __init__(self, device):
        self.device = device
        self.cache: Dict[tuple, tuple] = {}

    def get(self, key, target_range: int, compute: Callable[[int], tuple]):
        have = self.cache.get(key)
        if have is None or have[0] < target_range:
            have = (target_range,) + tuple(compute(target_range))
            self.cache[key] = have
        r, src, tgt, nt, nbs = have
        if r == target_range:
            return src, tgt, nt, nbs
        m = int(nbs[:target_range ** 3].sum())
        return src[:m], tgt[:m], nt[:m], nbs[:target_range ** 3]


# ----------------------------------------------------------------------------- hierarchy
class SparseFeatureHierarchy:
    """Per-level voxel sets of strides 1, 2, 4, ... (finest-voxel units) with neighbour queries."""
    CONFORM_OFFSETS = [list(o) for o in CONFORM]

    def __init__(self, depth: int, voxel_size: float, device, range_kernel):
        self._depth = int(depth)
        self._voxel_size = float(voxel_size)
        self._device = device
        self._range_kernel = range_kernel
        self._strides = [1 << d for d in range(self._depth)]
        self._levels: List[Optional[VoxelLevel]] = [None] * self._depth
        self._maps = NeighbourMaps(device)

    # ------------------------------------------------------------------ properties
    @property
    def depth(self) -> int:
        return self._depth

    @property
    def voxel_size(self) -> float:
        return self._voxel_size

    def get_stride(self, depth: int) -> int:
        return self._strides[depth]

    def level(self, depth: int) -> VoxelLevel:
        lv = self._levels[depth]
        if lv is None:
            lv = self._levels[depth] = VoxelLevel(torch.zeros((0, 3), dtype=torch.int32, device=self._device),
                                                  self._strides[depth])
        return lv

    def get_coords(self, depth: int, expand: int = 0, conforming: bool = False) -> torch.Tensor:
        s = self._strides[depth]
        c = self.level(depth).coords
        if expand >= 3:
            off = self._range_kernel()(expand) * s
            c = unique_cells((c[:, None, :] + off[None]).reshape(-1, 3))
        if conforming:
            parents = unique_cells(torch.div(c, 2 * s, rounding_mode="floor") * (2 * s))
            c = (parents[:, None, :] + CORNERS.to(c.device)[None] * s).reshape(-1, 3)
        return c

    def get_num_voxels(self, depth: int) -> int:
        return len(self._levels[depth]) if self._levels[depth] is not None else 0

    def get_voxel_centers(self, depth: int, normalized: bool = False):
        c = self.get_coords(depth) + self._strides[depth] / 2.0
        return c if normalized else c * self._voxel_size

    def __repr__(self) -> str:
        rows = [f"Depth={self.depth}:"]
        for d in range(self._depth):
            lv = self._levels[d]
            if lv is None or len(lv) == 0:
                rows.append(f" + [{self._strides[d]}] Empty")
                continue
            lo, hi = lv.coords.min(0).values.tolist(), lv.coords.max(0).values.tolist()
            rows.append(f" + [{self._strides[d]}] #Voxels={len(lv)} "
                        f"Bound=[{lo[0]},{hi[0]}]x[{lo[1]},{hi[1]}]x[{lo[2]},{hi[2]}]")
        return "\n".join(rows) + "\n"

    # ------------------------------------------------------------------ neighbour queries
    def get_coords_neighbours(self, source_coords, source_stride: int, target_depth: int, nn_kernel,
                              conv_based: bool = False, transposed: bool = False):
        """(source ids, target ids, neighbour types, counts) of every source and kernel offset whose
        probe on level ``target_depth`` hits a voxel (``_hash_backend.py:176-228``).

        Non-conv: the source snaps to the target lattice and the types are the offsets from the
        source centre to the target centre in source-stride units (float); conv: probes around the
        source as is, types are the kernel offsets (int).  Counts per kernel offset, or per source
        when ``transposed`` (then the pairs are grouped by source)."""
        assert 0 <= target_depth < self._depth
        st = self._strides[target_depth]
        if conv_based:
            assert not source_coords.requires_grad
            assert source_stride >= st, "the target level must be at least as fine as the source stride"
        else:
            assert source_stride <= st, "the target level must be at least as coarse as the source stride"
        src = source_coords.detach()[:, :3]
        src = src.contiguous() if src.dtype == torch.int32 else src.float().contiguous()
        src_ids, tgt_ids, kidx, counts = self.level(target_depth).neighbours(src, source_stride, nn_kernel, conv_based,
                                                                             transposed)
        types = nn_kernel[kidx.long()]
        if not conv_based:
            # centre offset of the snapped target cell, in source strides: snapped - source + half-cell shift
            snapped = torch.div(src[src_ids] + 0.5 * source_stride, st, rounding_mode="floor") * st
            centre = (snapped - src[src_ids]) / source_stride + (st // source_stride - 1) / 2.0
            types = types.float() * (st // source_stride) + centre
        return src_ids, tgt_ids, types, counts

    def get_self_neighbours(self, source_depth: int, target_depth: int, target_range: int,
                            conv_based: bool = False):
        """Cached voxel-to-voxel pair lists between two levels (``_hash_backend.py:230-290``).

        A query from a coarse level to a finer one runs the other way (fine sources, coarse
        targets), keeps the pairs within half the range and swaps them, with the offsets converted
        to coarse units."""
        assert 0 <= source_depth < self._depth and 0 <= target_depth < self._depth
        invert = not conv_based and source_depth > target_depth
        a, b = (target_depth, source_depth) if invert else (source_depth, target_depth)
        kind = "conv" if (conv_based or source_depth == target_depth) else "region"

        def compute(r):
            return self.get_coords_neighbours(self.level(a).coords, self._strides[a], b, self._range_kernel()(r),
                                              conv_based)
        src, tgt, nt, nbs = self._maps.get((a, b, kind), target_range, compute)
        if not invert:
            return src, tgt, nt, nbs
        keep = (nt.abs() < target_range / 2.0 + 1.0e-6).all(1)
        return tgt[keep], src[keep], (nt * (-self._strides[a] / self._strides[b]))[keep], None

    def evaluate_voxel_status(self, coords, depth: int):
        """0 where the voxel does not exist, 1 for a voxel without children, 2 for a voxel with at
        least one child on the next finer level (``_hash_backend.py:292-318``)."""
        rows = self.level(depth).probe(coords)
        status = (rows >= 0).long()
        if depth > 0 and coords.shape[0]:
            kids = (coords[:, None, :] + CORNERS.to(coords.device)[None] * self._strides[depth - 1]).reshape(-1, 3)
            has_kid = (self.level(depth - 1).probe(kids) >= 0).view(-1, 8).any(1)
            status[(rows >= 0) & has_kid] = 2
        return status

    # ------------------------------------------------------------------ data transfer
    def _corner_rows(self, xyz, data_depth: int, data=1):
        cells, w = trilinear(xyz, self._voxel_size, self._strides[data_depth], data)
        return self.level(data_depth).probe(cells), w

    def split_data(self, xyz, data_depth: int, data):
        """Voxel data interpolated trilinearly at the points (``_hash_backend.py:320-330``)."""
        assert data.size(0) == self.get_num_voxels(data_depth), "level data and voxel count differ"
        rows, w = self._corner_rows(xyz, data_depth)
        hit = rows >= 0
        n = xyz.size(0)
        vals = data[rows.clamp(min=0)] * torch.where(hit, w, torch.zeros_like(w)).view((-1,) + (1,) * (data.dim() - 1))
        return vals.view((8, n) + tuple(data.shape[1:])).sum(0)

    def splat_data(self, xyz, data_depth: int, data=None, check_corr: bool = True, return_nf_mask: bool = False):
        """Trilinear splat of per-point data (ones when None) onto the level's voxels
        (``_hash_backend.py:332-356``); corners without a voxel drop their share."""
        if data is not None:
            assert data.size(0) == xyz.size(0), "Input data must agree with xyz in size."
        rows, w = self._corner_rows(xyz, data_depth, 1 if data is None else data)
        hit = rows >= 0
        found = int(hit.sum())
        if found < rows.numel() and check_corr:
            print(f"Warning: {rows.numel() - found} of {rows.numel()} splat corners have no voxel on level "
                  f"{data_depth}; their share is dropped.")
        out = torch.zeros((self.get_num_voxels(data_depth),) + tuple(w.shape[1:]), dtype=w.dtype, device=w.device)
        out.index_add_(0, rows[hit], w[hit])
        if return_nf_mask:
            return out, hit.view(8, -1).sum(0) < 4
        return out

    # ------------------------------------------------------------------ builders
    def _set_levels(self, coords: List[torch.Tensor]):
        self._levels = [VoxelLevel(c, s) for c, s in zip(coords, self._strides)]
        self._maps = NeighbourMaps(self._device)

    def build_hierarchy_dense(self, xyz, expand_range: int = 0):
        """Every level from the finest: trilinear corners (expand_range 2) or the points' own cells
        (expanded by the range kernel), then each coarser level the parents of the finer one."""
        if expand_range == 2:
            finest = corner_cells(xyz, self._voxel_size, 1)
        else:
            finest = unique_cells(torch.floor(xyz / self._voxel_size).int())
            if expand_range > 0:
                off = self._range_kernel()(expand_range)
                finest = unique_cells((finest[:, None, :] + off[None]).reshape(-1, 3))
        coords = [finest]
        for s in self._strides[1:]:
            coords.append(unique_cells(torch.div(coords[-1], s, rounding_mode="floor") * s))
        self._set_levels(coords)

    def build_hierarchy_subdivide(self, xyz, subdivide_policy, expand: bool = False, limit_adaptive_depth: int = 100,
                                  **policy_kwargs):
        """Top-down: a point descends one level while ``subdivide_policy(points, inverse, **kwargs)``
        keeps it; the level of a point is where it stopped (``_hash_backend.py:380-412``)."""
        pts = xyz / self._voxel_size
        point_depth = torch.full((xyz.size(0),), self._depth - 1, dtype=torch.int, device=self._device)
        ids = torch.arange(xyz.size(0), device=self._device)
        coords: List[torch.Tensor] = [None] * self._depth
        inverse = None
        for d in reversed(range(self._depth)):
            if d != self._depth - 1:
                keep = subdivide_policy(pts, inverse, **policy_kwargs)
                pts, ids = pts[keep], ids[keep]
                policy_kwargs = {k: v[keep] if isinstance(v, torch.Tensor) else v for k, v in policy_kwargs.items()}
                point_depth[ids] -= 1
            s = self._strides[d]
            from .ops import torch_unique
            coords[d], inverse = torch_unique((torch.div(pts, s, rounding_mode="floor") * s).int(), dim=0,
                                              return_inverse=True)
        point_depth.clamp_(max=limit_adaptive_depth - 1)
        if expand:
            coords = []
            for d in range(self._depth):
                sel = point_depth <= d
                if not bool(sel.any()):
                    print(f"-- level {d} has no points of its own depth or finer; it stays empty")
                coords.append(corner_cells(xyz, self._voxel_size, self._strides[d], sel))
        self._set_levels(coords)
        return point_depth

    def build_hierarchy_adaptive(self, xyz, xyz_density, log_base: float = 4.0, min_density: float = 8.0,
                                 limit_adaptive_depth: int = 100):
        """Level of a point = how many factors of ``log_base`` its density lies below ``min_density``
        (0 when above), clamped; level d holds the trilinear corners of the points of level <= d
        (``_hash_backend.py:414-444``)."""
        depth = -torch.floor(torch.log(xyz_density / min_density) / np.log(log_base)).int()
        depth = depth.clamp(min=0, max=min(self._depth, limit_adaptive_depth) - 1)
        self._set_levels([corner_cells(xyz, self._voxel_size, s, depth <= d) for d, s in enumerate(self._strides)])
        return depth

    def update_coords(self, depth: int, coords):
        if coords is None:
            coords = torch.zeros((0, 3), dtype=torch.int32, device=self._device)
        assert coords.ndim == 2 and coords.size(1) == 3, coords.size()
        self._levels[depth] = VoxelLevel(coords, self._strides[depth])
        self._maps = NeighbourMaps(self._device)

    # kept for callers of the reference's private helpers
    def _quantize_coords(self, xyz, data_depth: int):
        return corner_cells(xyz, self._voxel_size, self._strides[data_depth])

    def _trilinear_weights(self, xyz, tree_stride: int, xyz_data=1, compute_grad: bool = False):
        return trilinear(xyz, self._voxel_size, tree_stride, xyz_data, compute_grad)
