"""Sparse multi-level voxel hierarchy with neighbour queries (reference: ``jspsr/core/_hash_backend.py``).

Level d holds voxel min-corners (finest-voxel units, multiples of 2^d) in lexicographic order and a
key table over them (``jspsr.ext.CuckooHashTable``).  Same API and semantics as the reference's
``SparseFeatureHierarchy``; sums go through ``index_add_`` instead of torch_scatter, and unique
voxel sets through the libngs rank bitmap (``ops.torch_unique``).
"""
from __future__ import annotations

from typing import List, Union

import numpy as np
import torch

from ..ext import CuckooHashTable
from .ops import torch_unique

CONFORM = ((0, 0, 0), (0, 0, 1), (0, 1, 0), (0, 1, 1), (1, 0, 0), (1, 0, 1), (1, 1, 0), (1, 1, 1))


def _scatter_sum(src, index, n):
    return torch.zeros((n,) + src.shape[1:], dtype=src.dtype, device=src.device).index_add_(0, index.long(), src)


def range_kernel(n: int, device=None) -> torch.Tensor:
    """Ordered neighbour offsets int32 [n^3, 3]: Chebyshev shells outward, lexicographic inside a
    shell.  Replaces the unpublished ``kernel.npz`` (``hashtree.py:103-116``); the prefix property
    (first 1 / 27 / 125 entries = radius 0 / 1 / 2) is what the incremental caches rely on."""
    assert n % 2 == 1, "target_range must be odd."
    r = n // 2
    g = np.stack(np.meshgrid(*[np.arange(-r, r + 1)] * 3, indexing="ij"), -1).reshape(-1, 3)
    order = np.lexsort((g[:, 2], g[:, 1], g[:, 0], np.abs(g).max(1)))
    return torch.tensor(g[order], dtype=torch.int32, device=device)


def compute_density(xyz: torch.Tensor, voxel_size: float) -> torch.Tensor:
    """B-spline kernel density of the points at the given smoothing voxel (``_hash_backend.py:13-28``)."""
    from .hashtree import HashTree
    from ..bases.bezier_tensor import BezierTensorBasis
    tree = HashTree(xyz, voxel_size, 1)
    tree.build_encoder_hierarchy_dense(expand_range=2, uniform_density=True)
    wd = tree.splat_data(xyz, tree.ENCODER, 0, check_corr=False)
    tree.reflect_decoder_coords()
    return tree.evaluate_interpolated(xyz, BezierTensorBasis(), None, 0, wd)


class NeighbourMaps:
    """Cache of level-pair neighbour lists that grows incrementally with the query range."""

    def __init__(self, device):
        self.cache = {}
        self.device = device

    def get_map(self, source_depth: int, target_depth: int, target_range: int, force_recompute: bool = False):
        key = (source_depth, target_depth)
        if force_recompute:
            self.cache.pop(key, None)
        have, src, tgt, nt, nbs = self.cache.get(key, (-1, None, None, None, None))
        if target_range == have:
            return src, tgt, nt, nbs, None
        if target_range < have:
            n = int(torch.sum(nbs[:target_range ** 3]))
            return src[:n], tgt[:n], nt[:n], nbs[:target_range ** 3], None
        return src, tgt, nt, nbs, [have + 2, target_range]

    def update_map(self, source_depth: int, target_depth: int, target_range: int, res: list):
        self.cache[(source_depth, target_depth)] = [target_range] + list(res)


class SparseFeatureHierarchy:
    CONFORM_OFFSETS = [list(o) for o in CONFORM]

    def __init__(self, depth: int, voxel_size: float, device, range_kernel):
        self._depth = depth
        self._voxel_size = voxel_size
        self._device = device
        self._range_kernel = range_kernel
        self._conv_nmap = NeighbourMaps(device)
        self._region_nmap = NeighbourMaps(device)
        self._strides = [2 ** d for d in range(depth)]
        self._coords: List[torch.Tensor] = [None] * depth
        self._hash_table: List[CuckooHashTable] = [None] * depth

    @property
    def depth(self) -> int:
        return self._depth

    @property
    def voxel_size(self) -> float:
        return self._voxel_size

    def get_stride(self, depth: int) -> int:
        return self._strides[depth]

    def get_coords(self, depth: int, expand: int = 0, conforming: bool = False) -> torch.Tensor:
        s = self._strides[depth]
        c = self._coords[depth]
        if expand >= 3:
            off = self._range_kernel()(expand) * s
            c = torch_unique((c[:, None, :] + off[None]).reshape(-1, 3), dim=0)
        if conforming:
            c = torch_unique(((c / s / 2.0).floor().int() * s * 2).int(), dim=0)
            off = torch.tensor(CONFORM, dtype=torch.int32, device=c.device) * s
            c = (c[:, None, :] + off[None]).reshape(-1, 3)
        return c

    def get_num_voxels(self, depth: int) -> int:
        return 0 if self._coords[depth] is None else self._coords[depth].size(0)

    def get_voxel_centers(self, depth: int, normalized: bool = False):
        return (self.get_coords(depth) + self._strides[depth] / 2.0) * (1.0 if normalized else self._voxel_size)

    def __repr__(self) -> str:
        out = f"Depth={self.depth}:\n"
        for s, c in zip(self._strides, self._coords):
            if c is None:
                out += f" + [{s}] Empty\n"
                continue
            lo, hi = c.min(0).values.tolist(), c.max(0).values.tolist()
            out += f" + [{s}] #Voxels={c.size(0)} Bound=[{lo[0]},{hi[0]}]x[{lo[1]},{hi[1]}]x[{lo[2]},{hi[2]}]\n"
        return out

    # ------------------------------------------------------------------ neighbours
    def get_coords_neighbours(self, source_coords, source_stride: int, target_depth: int, nn_kernel,
                              conv_based: bool = False, transposed: bool = False):
        """For each source (point or voxel) the target voxels around it: (src ids, tgt ids, offsets,
        counts).  Offsets are target-centre minus source-centre in source-stride units."""
        assert 0 <= target_depth < self._depth
        st = self._strides[target_depth]
        if not conv_based:
            assert source_stride <= st, "Data must be deeper and has more nodes."
            q = torch.div(source_coords.detach() + 0.5 * source_stride, st, rounding_mode="floor").int() * st
            c_off = (q - source_coords) / source_stride + (st // source_stride - 1) / 2.0
        else:
            assert not source_coords.requires_grad
            assert source_stride >= st, "Data must be sparser and shallower."
            q = source_coords
        hits = self._hash_table[target_depth].query(q, nn_kernel * st)          # [K, N]
        if transposed:
            hits = hits.T
        nbsizes = torch.sum(hits != -1, dim=1)
        if transposed:
            src, kk = torch.where(hits != -1)
            tgt = hits[src, kk]
        else:
            kk, src = torch.where(hits != -1)
            tgt = hits[kk, src]
        nt = nn_kernel[kk]
        if not conv_based:
            nt = nt.float() * (st / source_stride) + c_off[src, :3]
        return src, tgt, nt, nbsizes

    def get_self_neighbours(self, source_depth: int, target_depth: int, target_range: int,
                            conv_based: bool = False):
        """Cached voxel-to-voxel neighbour lists between two levels (``_hash_backend.py:230-290``)."""
        assert 0 <= source_depth < self.depth and 0 <= target_depth < self.depth
        inverted = False
        if not conv_based and source_depth != target_depth:
            maps = self._region_nmap
            if source_depth > target_depth:
                source_depth, target_depth, inverted = target_depth, source_depth, True
        else:
            maps = self._conv_nmap
        fine_s, coarse_s = self._strides[source_depth], self._strides[target_depth]

        def finish(src, tgt, nt, nbs):
            if not inverted:
                return src, tgt, nt, nbs
            near = torch.all(nt.abs() < target_range / 2.0 + 1.0e-6, dim=1)
            return tgt[near], src[near], (-nt / coarse_s * fine_s)[near], None

        src, tgt, nt, nbs, lack = maps.get_map(source_depth, target_depth, target_range)
        if lack is None:
            return finish(src, tgt, nt, nbs)
        kernel = self._range_kernel()(target_range)[max(0, lack[0] - 2) ** 3:]
        s2, t2, n2, b2 = self.get_coords_neighbours(self._coords[source_depth], fine_s, target_depth, kernel,
                                                    conv_based)
        if src is not None:
            s2, t2, n2, b2 = (torch.cat([src, s2]), torch.cat([tgt, t2]), torch.cat([nt, n2]), torch.cat([nbs, b2]))
        maps.update_map(source_depth, target_depth, target_range, [s2, t2, n2, b2])
        return finish(s2, t2, n2, b2)

    def evaluate_voxel_status(self, coords, depth: int):
        """0: no such voxel, 1: leaf voxel, 2: voxel with children (``_hash_backend.py:292-318``)."""
        status = torch.zeros(coords.size(0), dtype=torch.long, device=coords.device)
        sidx, _, _, _ = self.get_coords_neighbours(coords, self._strides[depth], depth, self._identity_kernel(),
                                                   conv_based=True)
        status[sidx] = 1
        if depth > 0:
            off = torch.tensor(CONFORM, dtype=torch.int32, device=self._device) * self._strides[depth - 1]
            kids = (coords[sidx][:, None, :] + off[None]).reshape(-1, 3)
            qidx, _, _, _ = self.get_coords_neighbours(kids, self._strides[depth - 1], depth - 1,
                                                       self._identity_kernel(), conv_based=True)
            status[sidx[torch.div(qidx, 8, rounding_mode="floor")]] = 2
        return status

    # ------------------------------------------------------------------ data transfer
    def split_data(self, xyz, data_depth: int, data):
        """Trilinear interpolation of voxel data at points (``_hash_backend.py:320-330``)."""
        s = self._strides[data_depth]
        assert data.size(0) == self._coords[data_depth].size(0), "Tree data does not agree on size."
        corners, w = self._trilinear_weights(xyz, s)
        src, tgt, _, _ = self.get_coords_neighbours(corners, s, data_depth, self._identity_kernel())
        return _scatter_sum(data[tgt] * w[src, None], src % xyz.size(0), xyz.size(0))

    def splat_data(self, xyz, data_depth: int, data=None, check_corr: bool = True, return_nf_mask: bool = False):
        """Trilinear splat of per-point data onto the level's voxels (``_hash_backend.py:332-356``)."""
        if data is not None:
            assert data.size(0) == xyz.size(0), "Input data must agree with xyz in size."
        s = self._strides[data_depth]
        corners, w = self._trilinear_weights(xyz, s, 1 if data is None else data)
        src, tgt, _, nbs = self.get_coords_neighbours(corners, s, data_depth, self._identity_kernel(), transposed=True)
        if src.size(0) < corners.size(0) and check_corr:
            print("Warning: Some grids that normal should be splatted onto is missing because expansion is too "
                  f"small. # Should = {corners.size(0)}, Actual = {src.size(0)}.")
        out = _scatter_sum(w[src], tgt, self._coords[data_depth].size(0))
        if return_nf_mask:
            return out, nbs.reshape(8, -1).sum(0) < 4
        return out

    # ------------------------------------------------------------------ builders
    def build_hierarchy_dense(self, xyz, expand_range: int = 0):
        if expand_range == 2:
            c = self._quantize_coords(xyz, 0)
        else:
            c = torch_unique(torch.div(xyz, self._voxel_size).floor().int(), dim=0)
            if expand_range > 0:
                off = self._range_kernel()(expand_range)
                c = torch_unique((c[:, None, :] + off[None]).reshape(-1, 3), dim=0)
        self._coords = [c]
        for d in range(1, self.depth):
            self._coords.append(torch_unique((torch.div(self._coords[-1], self._strides[d], rounding_mode="floor")
                                              * self._strides[d]).int(), dim=0))
        self._update_hash_table()

    def build_hierarchy_subdivide(self, xyz, subdivide_policy, expand: bool = False, limit_adaptive_depth: int = 100,
                                  **policy_kwargs):
        pts = xyz / self._voxel_size
        inv = None
        xyz_depth = torch.full((xyz.size(0),), self._depth - 1, device=self._device, dtype=torch.int)
        ids = torch.arange(xyz.size(0), device=self._device)
        for d in range(self._depth - 1, -1, -1):
            if d != self._depth - 1:
                keep = subdivide_policy(pts, inv, **policy_kwargs)
                pts, ids = pts[keep], ids[keep]
                policy_kwargs = {k: v[keep] if isinstance(v, torch.Tensor) else v for k, v in policy_kwargs.items()}
                xyz_depth[ids] -= 1
            c = torch.div(pts, self._strides[d], rounding_mode="floor").int() * self._strides[d]
            self._coords[d], inv = torch_unique(c.int(), dim=0, return_inverse=True)
        xyz_depth.clamp_(max=limit_adaptive_depth - 1)
        if expand:
            self._coords = []
            for d in range(self.depth):
                sel = xyz[xyz_depth <= d]
                if sel.size(0) == 0:
                    print(f"-- disregard level {d} due to insufficient samples!")
                self._coords.append(self._quantize_coords(sel, d))
        self._update_hash_table()
        return xyz_depth

    def build_hierarchy_adaptive(self, xyz, xyz_density, log_base: float = 4.0, min_density: float = 8.0,
                                 limit_adaptive_depth: int = 100):
        """Per-point level from the density, voxels of level d from points of level <= d
        (``_hash_backend.py:414-444``)."""
        level = -(torch.log(xyz_density / min_density) / np.log(log_base)).floor().int().clamp_(max=0)
        level.clamp_(max=min(self.depth - 1, limit_adaptive_depth - 1))
        self._coords = [self._quantize_coords(xyz[level <= d], d) for d in range(self.depth)]
        self._update_hash_table()
        return level

    def update_coords(self, depth: int, coords):
        if coords is None:
            coords = torch.zeros((0, 3), dtype=torch.int32, device=self._device)
        assert coords.ndim == 2 and coords.size(1) == 3, coords.size()
        self._coords[depth] = coords
        self._hash_table[depth] = CuckooHashTable(data=coords)

    def _identity_kernel(self):
        return torch.zeros((1, 3), dtype=torch.int32, device=self._device)

    def _quantize_coords(self, xyz, data_depth: int):
        corners, _ = self._trilinear_weights(xyz, self._strides[data_depth])
        return torch_unique(corners, dim=0)

    def _update_hash_table(self):
        for d in range(self.depth):
            self._hash_table[d] = CuckooHashTable(data=self._coords[d])
            assert self._hash_table[d].dim == 3

    def _trilinear_weights(self, xyz, tree_stride: int, xyz_data=1, compute_grad: bool = False):
        """8 corner cells (corner-major) and trilinear weights (``_hash_backend.py:469-510``)."""
        q = xyz / self._voxel_size
        d = (q / tree_stride).floor() * tree_stride
        rel = q - d - tree_stride / 2.0
        sgn = torch.sign(rel)
        loc = torch.abs(rel) / tree_stride
        corners, w, dw = [], [], []
        for nx, ny, nz in CONFORM:
            corners.append((d + torch.stack([nx * sgn[:, 0], ny * sgn[:, 1], nz * sgn[:, 2]], 1) * tree_stride).int())
            ax = loc[:, 0] if nx else 1 - loc[:, 0]
            ay = loc[:, 1] if ny else 1 - loc[:, 1]
            az = loc[:, 2] if nz else 1 - loc[:, 2]
            a = ax * ay * az
            if compute_grad:
                assert xyz_data == 1, "Not supported!"
                k = self._voxel_size * tree_stride
                gx = (sgn[:, 0] if nx else -sgn[:, 0]) / k
                gy = (sgn[:, 1] if ny else -sgn[:, 1]) / k
                gz = (sgn[:, 2] if nz else -sgn[:, 2]) / k
                dw.append(torch.stack([gx * ay * az, ax * gy * az, ax * ay * gz], 1))
            w.append(a * xyz_data if isinstance(xyz_data, int) or xyz_data.ndim == 1 else a[:, None] * xyz_data)
        if compute_grad:
            return torch.cat(corners), torch.cat(w), torch.cat(dw)
        return torch.cat(corners), torch.cat(w)
