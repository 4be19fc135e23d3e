"""Multi-branch sparse voxel tree (reference: ``jspsr/core/hashtree.py``).

Three branches (encoder, decoder, decoder-tmp) of ``SparseFeatureHierarchy``; the reconstruction path
reflects the decoder onto the encoder.  The neighbour-offset kernel is generated (Chebyshev shells,
lexicographic inside a shell) instead of loaded from the unpublished ``data/kernel.npz``.
"""
from __future__ import annotations

import weakref
from enum import Enum
from typing import Union

import torch

from ._hash_backend import SparseFeatureHierarchy, compute_density, range_kernel, _scatter_sum


class VoxelStatus(Enum):
    VS_NON_EXIST = 0
    VS_EXIST_STOP = 1
    VS_EXIST_CONTINUE = 2


class HashTree:
    ENCODER = 0
    DECODER = 1
    DECODER_TMP = 2

    def __init__(self, xyz: torch.Tensor, voxel_size: float, depth: int):
        self.xyz = xyz
        self.xyz_depth = None
        self.xyz_density = None
        self.device = xyz.device
        self.is_reflected = False
        self._kernels = {}
        rk = weakref.WeakMethod(self.get_range_kernel)
        self._enc_branch = SparseFeatureHierarchy(depth, voxel_size, self.device, rk)
        self._dec_branch = SparseFeatureHierarchy(depth, voxel_size, self.device, rk)
        self._dec_tmp_branch = SparseFeatureHierarchy(depth, voxel_size, self.device, rk)

    def reflect_decoder_coords(self):
        self._dec_tmp_branch = self._dec_branch = self._enc_branch
        self.is_reflected = True

    @property
    def voxel_size(self) -> float:
        return self._enc_branch.voxel_size

    @property
    def depth(self) -> int:
        return self._enc_branch.depth

    def get_coords(self, branch: int, depth: int):
        return self._get_branch(branch).get_coords(depth)

    def get_stride(self, branch: int, depth: int) -> int:
        return self._get_branch(branch).get_stride(depth)

    def get_coords_size(self, branch: int, depth: int):
        return self._get_branch(branch).get_num_voxels(depth)

    def update_coords(self, branch: int, depth: int, coords: Union[torch.Tensor, None]):
        return self._get_branch(branch).update_coords(depth, coords)

    def get_range_kernel(self, n_range: int) -> torch.Tensor:
        """First n_range^3 offsets of the shell-ordered kernel (``hashtree.py:103-116``)."""
        if n_range not in self._kernels:
            self._kernels[n_range] = range_kernel(n_range, self.device)
        return self._kernels[n_range]

    def _get_branch(self, branch: int) -> SparseFeatureHierarchy:
        if branch == self.ENCODER:
            return self._enc_branch
        if branch == self.DECODER:
            return self._dec_branch
        if branch == self.DECODER_TMP:
            return self._dec_tmp_branch
        raise NotImplementedError

    def evaluate_voxel_status(self, branch: int, coords, depth: int):
        return self._get_branch(branch).evaluate_voxel_status(coords, depth)

    def get_neighbours_data(self, source_coords, source_stride: int, target_depth: int, nn_kernel, branch: int,
                            conv_based: bool = False, transposed: bool = False):
        return self._get_branch(branch).get_coords_neighbours(source_coords, source_stride, target_depth, nn_kernel,
                                                              conv_based, transposed)

    def get_neighbours(self, source_depth: int, target_depth: int, target_range: int, branch: int,
                       conv_based: bool = False):
        return self._get_branch(branch).get_self_neighbours(source_depth, target_depth, target_range, conv_based)

    def evaluate_interpolated(self, query_pos, basis, basis_feat, feat_depth: int, feat, compute_mask: bool = False,
                              compute_grad: bool = False):
        """sum_v feat[v] * B_v(query) over the level's voxels (``hashtree.py:155-190``)."""
        coords = self._dec_branch.get_coords(feat_depth)
        stride = self._dec_branch.get_stride(feat_depth)
        assert feat.size(0) == coords.size(0), "Feature size not compatible."
        if basis_feat is not None:
            assert basis_feat.size(0) == coords.size(0), "Feature size not compatible."
        pos = query_pos / self.voxel_size - 0.5
        base_ids, tgt_ids, tgt_off, _ = self.get_neighbours_data(
            pos, 1, feat_depth, self.get_range_kernel(basis.get_domain_range()), self.DECODER)
        q = -tgt_off / stride
        if compute_grad:
            val = basis.evaluate_derivative(feat=basis_feat, xyz=q, feat_ids=tgt_ids, stride=stride)
            val = val * feat[tgt_ids, None]
        else:
            val = basis.evaluate(feat=basis_feat, xyz=q, feat_ids=tgt_ids) * feat[tgt_ids]
        val = _scatter_sum(val, base_ids, pos.size(0))
        if compute_mask:
            mask = torch.zeros((val.size(0),), device=val.device, dtype=torch.bool)
            mask[base_ids] = True
            return val, mask
        return val

    def get_random_samples(self, sample_per_voxel: int, depth: int, expand: int = 0):
        s = self._dec_branch.get_stride(depth)
        base = self._dec_branch.get_coords(depth, expand=expand)
        local = torch.rand((base.size(0), sample_per_voxel, 3), device=self.device) * s
        return (base.unsqueeze(1) + local.unsqueeze(0)).view(-1, 3) * self.voxel_size

    def get_test_grid(self, resolution: int, depth: int, expand: int = 0, conforming: bool = False):
        s = self._dec_branch.get_stride(depth)
        base = self._dec_branch.get_coords(depth, expand=expand, conforming=conforming)
        if resolution == 0:
            return None, base
        t = torch.linspace(0.0, s, resolution, device=self.device)
        box = torch.stack(torch.meshgrid(t, t, t, indexing="ij"), dim=3).view(-1, 3)
        return (base.unsqueeze(1) + box.unsqueeze(0)).view(-1, 3) * self.voxel_size, base

    def get_voxel_centers(self, depth: int, branch: int = DECODER, normalized: bool = False):
        return self._get_branch(branch).get_voxel_centers(depth, normalized)

    def __repr__(self):
        return "HashTree:\n" + repr(self._enc_branch) + repr(self._dec_branch)

    def _density(self, density_depth: int):
        s = self._enc_branch.get_stride(density_depth)
        return compute_density(self.xyz, s * self.voxel_size) / (s ** 2)

    def build_encoder_hierarchy_dense(self, expand_range: int = 0, density_depth: int = 2,
                                      uniform_density: bool = False):
        self.xyz_density = (torch.ones((self.xyz.size(0),), device=self.device) if uniform_density
                            else self._density(density_depth))
        self._enc_branch.build_hierarchy_dense(self.xyz, expand_range=expand_range)
        self.xyz_depth = torch.zeros((self.xyz.size(0),), device=self.device, dtype=torch.int)

    def build_hierarchy_subdivide(self, subdivide_policy, expand: bool = False, density_depth: int = 2,
                                  limit_adaptive_depth: int = 100, **policy_kwargs):
        self.xyz_density = self._density(density_depth)
        self.xyz_depth = self._enc_branch.build_hierarchy_subdivide(self.xyz, subdivide_policy, expand,
                                                                    limit_adaptive_depth, **policy_kwargs)

    def build_encoder_hierarchy_adaptive(self, density_depth: int = 2, log_base: float = 4.0,
                                         min_density: float = 8.0, uniform_density: bool = False,
                                         limit_adaptive_depth: int = 100):
        """Density-adaptive levels (``hashtree.py:261-285``)."""
        if uniform_density:
            assert log_base == 4.0 and min_density == 8.0 and limit_adaptive_depth == 100
            self.xyz_density = torch.ones((self.xyz.size(0),), device=self.device) * 1e6
        else:
            self.xyz_density = self._density(density_depth)
        self.xyz_depth = self._enc_branch.build_hierarchy_adaptive(self.xyz, self.xyz_density, log_base, min_density,
                                                                   limit_adaptive_depth)

    def split_data(self, xyz, branch: int, data_depth: int, data):
        return self._get_branch(branch).split_data(xyz, data_depth, data)

    def splat_data(self, xyz, branch: int, data_depth: int, data=None, check_corr: bool = True,
                   return_nf_mask: bool = False):
        return self._get_branch(branch).splat_data(xyz, data_depth, data, check_corr, return_nf_mask)
