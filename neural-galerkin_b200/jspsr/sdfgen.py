"""Signed distance from oriented points and exact k-nearest neighbours on the GPU.

Drop-in for the reference's ``ext.sdf_from_points(queries, ref_xyz, ref_normal, nb_points, stdv)``
(``ext/__init__.py:11-16``, ``ext/sdfgen/sdf_from_points.cu:70-116``), the ground truth of the
training loop (``models/full_net.py:135-142``).  The reference builds a CUDA k-d tree per call; here
the reference points are bucketed on a uniform cell grid (a libngs rank bitmap of the occupied cells
and a counting sort) and one kernel per query walks rings of cells until its k nearest points are
final, then votes the sign (``csrc/knn.cu``).
"""
from __future__ import annotations

import math

import numpy as np
import torch

from . import _lib as L


class PointIndex:
    """Reference points bucketed by cell for repeated nearest-neighbour queries."""

    def __init__(self, ref_xyz: torch.Tensor, ref_normal: torch.Tensor = None, cell: float = None):
        L.require_cuda(ref_xyz, "ref_xyz")
        self.xyz = ref_xyz.detach().float().contiguous()
        self.normal = None if ref_normal is None else ref_normal.detach().float().contiguous()
        n = self.xyz.shape[0]
        if n == 0:
            raise ValueError("no reference points")
        dev = self.xyz.device
        lo, hi = self.xyz.min(0).values, self.xyz.max(0).values
        ext = float((hi - lo).max().clamp(min=1e-6))
        if cell is None:
            # about 16 points per occupied cell for points on a surface (occupied cells ~ area / h^2)
            cell = 4.0 * ext / math.sqrt(n)
        cell = max(cell, ext / 1024.0)
        self.h = float(cell)
        self.inv_h = np.float32(1.0 / self.h)
        clo = torch.floor(lo * self.inv_h).cpu().numpy().astype(np.int64)
        chi = torch.floor(hi * self.inv_h).cpu().numpy().astype(np.int64)
        self.grid, self.words = L.make_grid(clo, chi - clo + 1, 1, dev)
        st = L.stream()
        L.call("ngs_knn_mark_cells", self.grid, L.ptr(self.xyz), n, self.inv_h, st)
        ncell = torch.empty(1, dtype=torch.int64, device=dev)
        self._ws = L.grid_finalize(self.grid, self.words, ncell)
        nc = int(ncell.item())
        cell_of = torch.empty(n, dtype=torch.int32, device=dev)
        count = torch.zeros(nc, dtype=torch.int32, device=dev)
        L.call("ngs_knn_bucket", self.grid, L.ptr(self.xyz), n, self.inv_h, L.ptr(cell_of), L.ptr(count), st)
        self.start = torch.empty(nc + 1, dtype=torch.int64, device=dev)
        L.scan(count, out=self.start[:nc], total=self.start[nc:])
        cursor = torch.zeros(nc, dtype=torch.int32, device=dev)
        self.sorted = torch.empty(n, dtype=torch.int32, device=dev)
        L.call("ngs_knn_scatter", L.ptr(cell_of), n, L.ptr(self.start), L.ptr(cursor), L.ptr(self.sorted), st)

    def query(self, queries: torch.Tensor, k: int, stdv: float = None, want_knn: bool = True):
        """(indices int32 [Q, k], squared distances [Q, k], signed distance [Q] or None)."""
        L.require_cuda(queries, "queries")
        q = queries.detach().float().contiguous()
        nq, dev = q.shape[0], q.device
        idx = torch.empty((nq, k), dtype=torch.int32, device=dev) if want_knn else None
        d2 = torch.empty((nq, k), dtype=torch.float32, device=dev) if want_knn else None
        sdf = None
        if stdv is not None:
            if self.normal is None:
                raise ValueError("signed distances need the reference normals")
            sdf = torch.empty(nq, dtype=torch.float32, device=dev)
        L.call("ngs_knn_sdf", self.grid, L.ptr(self.start), L.ptr(self.sorted), L.ptr(self.xyz), L.ptr(self.normal),
               L.ptr(q), nq, self.inv_h, self.h, int(k), float(stdv if stdv is not None else 0.0), L.ptr(idx), L.ptr(d2),
               L.ptr(sdf), L.stream())
        return idx, d2, sdf


def knn(queries: torch.Tensor, ref_xyz: torch.Tensor, k: int):
    """Exact k nearest reference points of every query: (indices [Q, k], squared distances [Q, k]),
    nearest first, ties broken by the smaller index."""
    idx, d2, _ = PointIndex(ref_xyz).query(queries, k)
    return idx, d2


def sdf_from_points(queries: torch.Tensor, ref_xyz: torch.Tensor, ref_normal: torch.Tensor, nb_points: int,
                    stdv: float) -> torch.Tensor:
    """Signed distance of every query from the oriented reference points: magnitude from the nearest
    point (distance to its tangent plane within ``stdv``, Euclidean beyond), sign by the majority of
    the ``nb_points`` nearest normals (``ext/sdfgen/sdf_from_points.cu:31-68``)."""
    _, _, sdf = PointIndex(ref_xyz, ref_normal).query(queries, nb_points, stdv=stdv, want_knn=False)
    return sdf
