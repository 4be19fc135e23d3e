"""Screened-Poisson reconstructor for any basis (reference API: ``jspsr/core/reconstructor.py``).

The reference's class and method signatures on this package's machinery:

* ``solve_multigrid`` builds the geometry of every level once (stencil CSR from the level's rank
  bitmap, point basis of the screening points, cross-level and data pair lists from the fused
  neighbour query) and hands the whole coarse-to-fine chain to ``galerkin.GalerkinSolve``: basis
  integrals written straight into the CSR values, the screening Gram added in place from the
  points, every level solved by the persistent PCG, and a hand-written adjoint (second PCG per level
  on the same CSR) for gradients w.r.t. the normal data and the per-voxel basis features;
* the field is evaluated through ``HashTree.evaluate_interpolated`` (differentiable);
* ``extract_multiscale_mesh`` selects the conformal leaf cells with bitmap probes and then runs the
  device pipeline's dual marching cubes (``pipeline.DualMesher``);
* ``extract_mesh`` is the differentiable primal marching cubes of ``ops.marching_cubes_op``.
"""
from __future__ import annotations

from types import SimpleNamespace
from typing import Union

import numpy as np
import torch

from ..bases.abc import BaseBasis
from . import galerkin as G
from ._hash_backend import CORNERS, VoxelLevel
from .hashtree import HashTree, VoxelStatus
from .ops import marching_cubes_op
from .pipeline import DualMesher


class Reconstructor:
    def __init__(self, hash_tree: HashTree, basis: BaseBasis, feat: dict = None):
        self.hash_tree = hash_tree
        self.fixed_level_set = None
        self.branch = hash_tree.DECODER
        self.basis = basis
        self.solutions = {}
        self.sample_weight = None
        if feat is None:
            feat = {}
            for d in range(hash_tree.depth):
                f = torch.zeros((hash_tree.get_coords_size(self.branch, d), basis.get_feature_size()),
                                device=hash_tree.device)
                basis.initialize_feature_value(f)
                feat[d] = f
        self.grid_features = feat

    def set_fixed_level_set(self, value):
        self.fixed_level_set = value

    def _features(self):
        """Per-level features handed to the solve (None for a fixed basis)."""
        if self.basis.get_feature_size() == 0:
            return {d: None for d in self.grid_features}
        return dict(self.grid_features)

    def solve_multigrid(self, start_depth: int, end_depth: int, normal_data: dict,
                        screen_alpha: Union[float, torch.Tensor] = 0.0, screen_xyz: torch.Tensor = None,
                        screen_delta: Union[float, torch.Tensor] = 0.1, solver: str = "pcg", verbose: bool = True):
        """Solve levels ``start_depth`` (coarse) down to ``end_depth`` (fine); ``normal_data[d]`` are
        the splatted normals of level d.  Screening (weight ``screen_alpha``, scalar or per point,
        target ``screen_delta``) needs the screened points.  ``solver``: ``pcg`` / ``pcg-mixed`` /
        ``pcg-fp64`` / ``cholmod`` / ``mixed`` with ``@tol=..@maxiter=..`` options."""
        if isinstance(screen_alpha, torch.Tensor):
            if screen_xyz is None:
                raise ValueError("screening with per-point weights needs the screened points (screen_xyz)")
            assert screen_alpha.size(0) == screen_xyz.size(0)
        elif screen_alpha > 0.0 and screen_xyz is None:
            raise ValueError("screening needs the screened points (screen_xyz)")
        if solver == "mixed":
            solver = "cholmod"            # the reference's mixed mode: exact solves (FP64 PCG here)
        shape = G.ShapeGeometry.build(self.hash_tree, self.branch, start_depth, end_depth, sorted(normal_data),
                                      screen_xyz, screen_alpha, screen_delta, self.basis.get_domain_range())
        sol = G.galerkin_solve(self.basis, [shape], [self._features()], [dict(normal_data)], solver)[0]
        self.solutions = sol
        self.solve_stats = shape.stats
        if verbose:
            for d in shape.order:
                st = self.solve_stats.get(d)
                if st is not None:
                    print(f"level {d}: PCG status {st['status']} after {st['iters']} iterations, |r| = {st['resid']:.3e}")

    def evaluate_raw_chi(self, xyz: torch.Tensor, compute_mask: bool = False, compute_grad: bool = False,
                         depths: list = None):
        """Sum over the solved levels of the interpolated field (or its gradient) at positions."""
        if not self.solutions:
            raise RuntimeError("solve_multigrid has not run: there is no field to evaluate")
        total, mask = 0, None
        for d, x in self.solutions.items():
            if depths is not None and d not in depths:
                continue
            v = self.hash_tree.evaluate_interpolated(xyz, self.basis, self._features().get(d), d, x, compute_mask,
                                                     compute_grad=compute_grad)
            if compute_mask:
                v, m = v
                mask = m if mask is None else mask | m
            total = total + v
        if compute_mask:
            if mask is None:
                mask = torch.zeros(xyz.size(0), dtype=torch.bool, device=xyz.device)
            return total, mask
        return total

    def get_mean_chi(self):
        """Iso level: the fixed one if set, else the sample-weighted mean of chi at the input points."""
        if self.fixed_level_set is not None:
            return self.fixed_level_set
        chi = self.evaluate_raw_chi(self.hash_tree.xyz)
        if self.sample_weight is None:
            print("no sample weights given: the iso level is the plain mean of chi at the points")
            return chi.mean()
        return (chi * self.sample_weight).sum() / self.sample_weight.sum()

    def evaluate_chi(self, xyz: torch.Tensor, compute_mask: bool = False, max_points: int = -1, depths: list = None):
        """chi minus the iso level, in chunks of ``max_points`` queries."""
        iso = self.get_mean_chi()
        chunks = [xyz] if max_points <= 0 else list(torch.split(xyz, max_points))
        parts = [self.evaluate_raw_chi(c, compute_mask=compute_mask, depths=depths) for c in chunks]
        if compute_mask:
            return torch.cat([p[0] for p in parts]) - iso, torch.cat([p[1] for p in parts])
        return torch.cat(parts) - iso

    def extract_mesh(self, base_coords, chi_field, chi_depth: int, build_o3d_mesh: bool = False):
        """Primal sparse marching cubes over r^3 sample blocks per voxel (``reconstructor.py:257-294``):
        (vertices, triangles, vertex normals).  No Open3D mesh is built (Open3D is not a dependency)."""
        if build_o3d_mesh:
            raise NotImplementedError("Open3D meshes are not built; pass build_o3d_mesh=False")
        scale = self.hash_tree.get_stride(self.branch, chi_depth)
        res = int(round((chi_field.size(0) // base_coords.size(0)) ** (1.0 / 3.0)))
        v, t, n, _ = marching_cubes_op(base_coords.float() / scale, chi_field.reshape(-1, res, res, res))
        return v * (scale * self.hash_tree.voxel_size), t, n

    def _leaves(self, max_depth: int, expand: int, trim: bool):
        """Conformal leaf cells per level: a level's cells (the 8 children of its voxels' parents,
        except on the coarsest level) that the next finer level does not cover; with ``trim``, the
        voxels without children instead (``reconstructor.py:310-336``)."""
        ht, br = self.hash_tree, self.branch
        cells = {}
        if trim:
            for d in range(max_depth):
                c = ht.get_coords(br, d)
                cells[d] = c[ht.evaluate_voxel_status(br, c, d) == VoxelStatus.VS_EXIST_STOP.value]
            return cells, max_depth
        keep = {}
        for d in range(max_depth):
            _, c = ht.get_test_grid(0, d, expand, conforming=d < max_depth - 1)
            if d > 0:
                finer = VoxelLevel(cells[d - 1], ht.get_stride(br, d - 1))
                uncovered = finer.probe(c) < 0
                if not bool(uncovered.any()):
                    max_depth = d
                    break
                keep[d] = uncovered
            cells[d] = c
        for d in range(1, max_depth):
            cells[d] = cells[d][keep[d]]
        return {d: cells[d] for d in range(max_depth)}, max_depth

    def extract_multiscale_mesh(self, n_upsample: int = 1, max_depth: int = 100, expand: int = 0, trim: bool = False,
                                build_o3d_mesh: bool = False, max_points: int = -1):
        """Dual marching cubes over the conformal multi-level leaf cells (``reconstructor.py:296-397``):
        (vertices, triangles)."""
        if build_o3d_mesh:
            raise NotImplementedError("Open3D meshes are not built; pass build_o3d_mesh=False")
        ht, br = self.hash_tree, self.branch
        cells, max_depth = self._leaves(min(max_depth, ht.depth), expand, trim)
        mesher = DualMesher()
        mesher.levels = [SimpleNamespace(stride=ht.get_stride(br, d)) for d in range(max_depth)]
        mesher.vs, mesher.dev = ht.voxel_size, ht.device
        base = {d: cells[d].to(torch.int32).contiguous() for d in range(max_depth)}
        with torch.no_grad():
            v, f = mesher.mesh_from_leaves(base, max_depth, n_upsample,
                                           lambda pos: self.evaluate_chi(pos, max_points=max_points).float())
        self.mesher = mesher
        return v, f
