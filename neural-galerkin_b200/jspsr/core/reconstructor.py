"""Screened-Poisson reconstructor with learnable bases (reference: ``jspsr/core/reconstructor.py``).

The general, differentiable form of the solve: any ``BaseBasis`` (Bezier or the learned additive
bases), per-voxel basis features, point-wise screening weights, torch autograd through the
assembly (basis integrals), the screening products and the linear solves.  Integrals, hashing,
screening and the PCG solve run on libngs through ``jspsr.ext``; the coordinate bookkeeping is
torch.  The fixed-basis production path (``jspsr.reconstruct``) is ``core.pipeline``.
"""
from __future__ import annotations

from typing import Union

import numpy as np
import torch

from ..bases.abc import BaseBasis
from ..ext import CuckooHashTable, dual_marching_cubes_indices, dual_marching_cubes_sparse
from .hashtree import HashTree, VoxelStatus
from .ops import marching_cubes_op, screened_multiplication, torch_unique
from .solver import solve_sparse


def _scatter_sum(src, index, n):
    return torch.zeros((n,) + src.shape[1:], dtype=src.dtype, device=src.device).index_add_(0, index.long(), src)


class ScreeningData:
    """Point-by-voxel basis values (sparse, rows grouped by point)."""

    def __init__(self, pts_ids, vx_ids, values, nb_sizes):
        self.pts_ids = pts_ids
        self.vx_ids = vx_ids
        self.values = values
        self.nb_sizes = nb_sizes


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
                feat[d] = torch.zeros((hash_tree.get_coords_size(self.branch, d), basis.get_feature_size()),
                                      device=hash_tree.device)
                basis.initialize_feature_value(feat[d])
        self.grid_features = feat

    def set_fixed_level_set(self, value):
        self.fixed_level_set = value

    @classmethod
    def _evaluate_screening_term(cls, data_a: ScreeningData, data_b: ScreeningData, domain_a, domain_b,
                                 pts_weight=None):
        """sum_p w_p B_a(p) B_b(p) for each (a, b) pair of the domain (``reconstructor.py:55-71``)."""
        if domain_a.size(0) == 0 or domain_b.size(0) == 0:
            return torch.zeros((0,), device=domain_a.device)
        if pts_weight is None:
            pts_weight = torch.ones((data_a.nb_sizes.size(0),), device=domain_a.device)
        elif isinstance(pts_weight, float):
            pts_weight = torch.full((data_a.nb_sizes.size(0),), pts_weight, dtype=torch.float32,
                                    device=domain_a.device)
        table = CuckooHashTable(torch.stack([domain_a, domain_b], dim=1), enlarged=True)
        return screened_multiplication(table.object, data_a.values, data_b.values, data_a.vx_ids, data_b.vx_ids,
                                       data_a.nb_sizes, data_b.nb_sizes, pts_weight)

    def solve_multigrid(self, start_depth: int, end_depth: int, normal_data: dict,
                        screen_alpha: Union[float, torch.Tensor] = 0.0, screen_xyz: torch.Tensor = None,
                        screen_delta: Union[float, torch.Tensor] = 0.1, solver: str = "pcg", verbose: bool = True):
        """Coarse-to-fine cascadic solve, one sparse system per level (``reconstructor.py:73-196``):
        RHS = divergence of the splatted normals + screening target - coarser solutions pushed through
        the cross-level stiffness; LHS = same-level stiffness + screening Gram."""
        if isinstance(screen_alpha, torch.Tensor):
            assert screen_xyz is not None, "Must provide points to be screened."
            assert screen_alpha.size(0) == screen_xyz.size(0)
            should_screen = True
        else:
            should_screen = screen_alpha > 0.0
        ht, br = self.hash_tree, self.branch
        self.solutions = {}
        nb_range = 2 * self.basis.get_domain_range() - 1

        screen_data = {}
        if should_screen:
            base = screen_xyz / ht.voxel_size - 0.5
            for d in range(end_depth, start_depth + 1):
                p_ids, v_ids, off, nbs = ht.get_neighbours_data(
                    base, 1, d, ht.get_range_kernel(self.basis.get_domain_range()), br, transposed=True)
                val = self.basis.evaluate(feat=self.grid_features[d], xyz=-off / ht.get_stride(br, d),
                                          feat_ids=v_ids)
                screen_data[d] = ScreeningData(p_ids, v_ids, val, nbs)

        for d in range(start_depth, end_depth - 1, -1):
            screen_factor = (1 / 4.) ** d
            n_d = ht.get_coords_size(br, d)
            rhs = 0
            for data_depth, nd in normal_data.items():
                n_ids, t_ids, off, _ = ht.get_neighbours(data_depth, d, self.basis.get_domain_range(), br)
                part = self.basis.integrate_const_deriv_product(
                    data=-nd[n_ids], target_feat=self.grid_features[d], rel_pos=off,
                    data_stride=ht.get_stride(br, data_depth), target_stride=ht.get_stride(br, d), target_ids=t_ids)
                rhs = rhs + _scatter_sum(part, t_ids, n_d)
            if should_screen:
                if isinstance(screen_alpha, torch.Tensor) or isinstance(screen_delta, torch.Tensor):
                    mult = (screen_delta * screen_alpha)[screen_data[d].pts_ids]
                else:
                    mult = screen_alpha * screen_delta
                rhs = rhs + screen_factor * _scatter_sum(screen_data[d].values * mult, screen_data[d].vx_ids, n_d)

            for dd in range(start_depth, d, -1):
                s_ids, t_ids, rel, _ = ht.get_neighbours(d, dd, target_range=nb_range, branch=br)
                a_val = self.basis.integrate_deriv_deriv_product(
                    source_feat=self.grid_features[d], target_feat=self.grid_features[dd], rel_pos=rel,
                    source_stride=ht.get_stride(br, d), target_stride=ht.get_stride(br, dd),
                    source_ids=s_ids, target_ids=t_ids)
                if should_screen:
                    a_val = a_val + screen_factor * self._evaluate_screening_term(
                        screen_data[d], screen_data[dd], s_ids, t_ids, screen_alpha)
                rhs = rhs - _scatter_sum(self.solutions[dd][t_ids] * a_val, s_ids, rhs.size(0))

            s_ids, t_ids, rel, _ = ht.get_neighbours(d, d, target_range=nb_range, branch=br)
            lhs = self.basis.integrate_deriv_deriv_product(
                source_feat=self.grid_features[d], target_feat=self.grid_features[d], rel_pos=rel,
                source_stride=ht.get_stride(br, d), target_stride=ht.get_stride(br, d),
                source_ids=s_ids, target_ids=t_ids)
            if should_screen:
                lhs = lhs + screen_factor * self._evaluate_screening_term(
                    screen_data[d], screen_data[d], s_ids, t_ids, screen_alpha)
            cur = ("mixed" if d == end_depth else "cholmod") if solver == "mixed" else solver
            self.solutions[d] = solve_sparse(s_ids, t_ids, lhs, rhs, cur)
            if verbose:
                res = _scatter_sum(self.solutions[d][t_ids] * lhs, s_ids, rhs.size(0)) - rhs
                print(f"Solving complete at level {d}, residual = {torch.linalg.norm(res).item()}.")

    def evaluate_raw_chi(self, xyz: torch.Tensor, compute_mask: bool = False, compute_grad: bool = False,
                         depths: list = None):
        assert len(self.solutions) > 0, "Please run solver before evaluation."
        vals = 0
        mask = torch.zeros((xyz.size(0),), dtype=torch.bool, device=xyz.device) if compute_mask else None
        for d, sol in self.solutions.items():
            if depths is not None and d not in depths:
                continue
            v = self.hash_tree.evaluate_interpolated(xyz, self.basis, self.grid_features[d], d, sol, compute_mask,
                                                     compute_grad=compute_grad)
            if compute_mask:
                vals = vals + v[0]
                mask = torch.logical_or(mask, v[1])
            else:
                vals = vals + v
        return (vals, mask) if compute_mask else vals

    def get_mean_chi(self):
        if self.fixed_level_set is not None:
            return self.fixed_level_set
        chi = self.evaluate_raw_chi(self.hash_tree.xyz)
        if self.sample_weight is None:
            print("Warning: Sample weight not set.")
            return torch.mean(chi)
        return torch.sum(chi * self.sample_weight) / torch.sum(self.sample_weight)

    def evaluate_chi(self, xyz: torch.Tensor, compute_mask: bool = False, max_points: int = -1, depths: list = None):
        mean_chi = self.get_mean_chi()
        n_chunks = int(np.ceil(xyz.size(0) / max_points)) if max_points > 0 else 1
        parts = [self.evaluate_raw_chi(c, compute_mask=compute_mask, depths=depths) for c in torch.chunk(xyz, n_chunks)]
        if compute_mask:
            return torch.cat([p[0] for p in parts]) - mean_chi, torch.cat([p[1] for p in parts])
        return torch.cat(parts) - mean_chi

    def extract_mesh(self, base_coords, chi_field, chi_depth: int, build_o3d_mesh: bool = False):
        """Primal sparse marching cubes on densely sampled blocks (``reconstructor.py:245-283``).
        Returns (vertices, triangles, normals); an Open3D mesh is not built (no Open3D here)."""
        if build_o3d_mesh:
            raise NotImplementedError("Open3D meshes are not built; pass build_o3d_mesh=False")
        scale = self.hash_tree.get_stride(self.branch, chi_depth)
        res = round((chi_field.size(0) // base_coords.size(0)) ** (1 / 3.))
        chi_field = chi_field.reshape(-1, res, res, res)
        v, t, n, _ = marching_cubes_op(base_coords.float() / scale, chi_field)
        return v * (scale * self.hash_tree.voxel_size), t, n

    def extract_multiscale_mesh(self, n_upsample: int = 1, max_depth: int = 100, expand: int = 0, trim: bool = False,
                                build_o3d_mesh: bool = False, max_points: int = -1):
        """Dual marching cubes over the conformal multi-level leaves (``reconstructor.py:285-397``)."""
        if build_o3d_mesh:
            raise NotImplementedError("Open3D meshes are not built; pass build_o3d_mesh=False")
        ht, br = self.hash_tree, self.branch
        max_depth = min(max_depth, ht.depth)
        prim = {}
        if trim:
            for d in range(max_depth):
                c = ht.get_coords(br, d)
                st = ht.evaluate_voxel_status(br, c, d)
                prim[d] = c[st == VoxelStatus.VS_EXIST_STOP.value]
        else:
            masks = {}
            for d in range(max_depth):
                _, c = ht.get_test_grid(0, d, expand, conforming=d < max_depth - 1)
                if d > 0:
                    keep = CuckooHashTable(data=prim[d - 1]).query(c) == -1
                    if not torch.any(keep):
                        max_depth = d
                        break
                    masks[d] = keep
                prim[d] = c
            for d in range(1, max_depth):
                prim[d] = prim[d][masks[d]]

        ev = ht.voxel_size / n_upsample
        e = torch.arange(0, n_upsample, dtype=torch.int, device=ht.device)
        e = torch.stack(torch.meshgrid(e, e, e, indexing="ij"), dim=3).view(-1, 3)
        base = {}
        for d in range(max_depth):
            s = ht.get_stride(br, d)
            base[d] = ((prim[d] * n_upsample).unsqueeze(1) + (e * s).unsqueeze(0)).view(-1, 3)

        corners = torch.tensor([(0, 0, 0), (0, 0, 1), (0, 1, 0), (0, 1, 1), (1, 0, 0), (1, 0, 1), (1, 1, 0), (1, 1, 1)],
                               dtype=torch.int32, device=ht.device)
        centers = torch.cat([(base[d].unsqueeze(1) + corners.unsqueeze(0) * ht.get_stride(br, d)).reshape(-1, 3)
                             for d in range(max_depth)])
        centers = torch_unique(centers, dim=0)
        table = CuckooHashTable(data=centers)
        acc, cnt = dual_marching_cubes_indices(
            table.object, base, {d: ht.get_stride(br, d) for d in range(max_depth)},
            {d: sum(base[k].size(0) for k in range(d)) for d in range(max_depth)})
        acc = acc[cnt == 8]

        dpos, dval = [], []
        for d in range(max_depth):
            p = (base[d] + ht.get_stride(br, d)) * ev
            dpos.append(p)
            dval.append(self.evaluate_chi(p, max_points=max_points))
        tris, vids = dual_marching_cubes_sparse(acc, torch.cat(dpos), torch.cat(dval))
        unq, tri = torch_unique(vids.view(-1, 2), dim=0, return_inverse=True)
        verts = torch.empty((unq.size(0), 3), device=vids.device, dtype=tris.dtype)
        verts[tri] = tris.view(-1, 3)
        return verts, tri.view(-1, 3)
