"""Multi-branch sparse voxel tree (reference API: ``jspsr/core/hashtree.py``).

``HashTree`` keeps the reference's three branches (encoder, decoder, decoder-tmp) of
``SparseFeatureHierarchy``, its branch accessors and its builders; the reconstruction path reflects
the decoder onto the encoder.  Storage and queries are the rank-bitmap levels of ``_hash_backend``;
the neighbour-offset kernel is generated (``range_kernel``) instead of loaded from the unpublished
``data/kernel.npz``.
"""
from __future__ import annotations

import weakref
from enum import Enum
from typing import Union

import torch

from ._hash_backend import SparseFeatureHierarchy, compute_density, range_kernel


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
        kernels = weakref.WeakMethod(self.get_range_kernel)
        self._branches = [SparseFeatureHierarchy(depth, voxel_size, self.device, kernels) for _ in range(3)]

    def reflect_decoder_coords(self):
        """Decoder (and decoder-tmp) share the encoder's levels."""
        enc = self._branches[self.ENCODER]
        self._branches[self.DECODER] = self._branches[self.DECODER_TMP] = enc
        self.is_reflected = True

    @property
    def voxel_size(self) -> float:
        return self._branches[self.ENCODER].voxel_size

    @property
    def depth(self) -> int:
        return self._branches[self.ENCODER].depth

    def _get_branch(self, branch: int) -> SparseFeatureHierarchy:
        if branch not in (self.ENCODER, self.DECODER, self.DECODER_TMP):
            raise NotImplementedError(f"no branch {branch}")
        return self._branches[branch]

    def get_coords(self, branch: int, depth: int):
        return self._get_branch(branch).get_coords(depth)

    def get_stride(self, branch: int, depth: int) -> int:
        return self._get_branch(branch).get_stride(depth)

    def get_coords_size(self, branch: int, depth: int):
        return self._get_branch(branch).get_num_voxels(depth)

    def update_coords(self, branch: int, depth: int, coords: Union[torch.Tensor, None]):
        return self._get_branch(branch).update_coords(depth, coords)

    def get_range_kernel(self, n_range: int) -> torch.Tensor:
        """The first n_range^3 offsets of the shell-ordered kernel, cached per range."""
        k = self._kernels.get(n_range)
        if k is None:
            k = self._kernels[n_range] = range_kernel(n_range, self.device)
        return k

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
        """f(q) = sum over the level's voxels v of feat[v] B_v(q) (or its gradient), where B_v is the
        basis centred on v (``hashtree.py:155-190``); differentiable in ``feat`` and ``basis_feat``.

        The voxels around each query come from one source-major fused query of the level (the
        query snapped to the lattice, the basis' domain range around it); the basis is evaluated at
        the query's position relative to each voxel centre, in voxel units."""
        level = self._branches[self.DECODER]
        stride = level.get_stride(feat_depth)
        n_vox = level.get_num_voxels(feat_depth)
        assert feat.size(0) == n_vox, f"{feat.size(0)} values for the {n_vox} voxels of level {feat_depth}"
        if basis_feat is not None:
            assert basis_feat.size(0) == n_vox, f"{basis_feat.size(0)} basis features for {n_vox} voxels"
        pos = query_pos / self.voxel_size - 0.5
        q_ids, v_ids, types, _ = level.get_coords_neighbours(pos, 1, feat_depth,
                                                             self.get_range_kernel(basis.get_domain_range()),
                                                             transposed=True)
        local = types / (-stride)
        if compute_grad:
            contrib = basis.evaluate_derivative(feat=basis_feat, xyz=local, feat_ids=v_ids, stride=stride) * \
                feat[v_ids, None]
        else:
            contrib = basis.evaluate(feat=basis_feat, xyz=local, feat_ids=v_ids) * feat[v_ids]
        out = torch.zeros((pos.size(0),) + tuple(contrib.shape[1:]), dtype=contrib.dtype, device=contrib.device)
        out = out.index_add(0, q_ids, contrib)
        if not compute_mask:
            return out
        mask = torch.zeros(pos.size(0), dtype=torch.bool, device=pos.device)
        mask[q_ids] = True
        return out, mask

    def get_random_samples(self, sample_per_voxel: int, depth: int, expand: int = 0):
        level = self._branches[self.DECODER]
        s = level.get_stride(depth)
        base = level.get_coords(depth, expand=expand).float()
        jitter = torch.rand((base.size(0), sample_per_voxel, 3), device=self.device) * s
        return (base[:, None, :] + jitter).reshape(-1, 3) * self.voxel_size

    def get_test_grid(self, resolution: int, depth: int, expand: int = 0, conforming: bool = False):
        """Voxel min-corners of a level (optionally expanded / conforming) and, for resolution r > 0,
        r^3 regularly spaced samples spanning each voxel (``hashtree.py:209-229``)."""
        level = self._branches[self.DECODER]
        s = level.get_stride(depth)
        base = level.get_coords(depth, expand=expand, conforming=conforming)
        if resolution == 0:
            return None, base
        t = torch.linspace(0.0, s, resolution, device=self.device)
        lattice = torch.cartesian_prod(t, t, t)
        return (base[:, None, :] + lattice[None]).reshape(-1, 3) * self.voxel_size, base

    def get_voxel_centers(self, depth: int, branch: int = DECODER, normalized: bool = False):
        return self._get_branch(branch).get_voxel_centers(depth, normalized)

    def __repr__(self):
        return "HashTree:\n" + repr(self._branches[self.ENCODER]) + repr(self._branches[self.DECODER])

    # ------------------------------------------------------------------ builders
    def _density(self, density_depth: int):
        """KDE at the stride of ``density_depth``, normalised by stride^2 (``hashtree.py:283-285``)."""
        s = self._branches[self.ENCODER].get_stride(density_depth)
        return compute_density(self.xyz, s * self.voxel_size) / float(s * s)

    def build_encoder_hierarchy_dense(self, expand_range: int = 0, density_depth: int = 2,
                                      uniform_density: bool = False):
        self.xyz_density = torch.ones(self.xyz.size(0), device=self.device) if uniform_density else \
            self._density(density_depth)
        self._branches[self.ENCODER].build_hierarchy_dense(self.xyz, expand_range=expand_range)
        self.xyz_depth = torch.zeros(self.xyz.size(0), dtype=torch.int, device=self.device)

    def build_hierarchy_subdivide(self, subdivide_policy, expand: bool = False, density_depth: int = 2,
                                  limit_adaptive_depth: int = 100, **policy_kwargs):
        self.xyz_density = self._density(density_depth)
        self.xyz_depth = self._branches[self.ENCODER].build_hierarchy_subdivide(
            self.xyz, subdivide_policy, expand, limit_adaptive_depth, **policy_kwargs)

    def build_encoder_hierarchy_adaptive(self, density_depth: int = 2, log_base: float = 4.0,
                                         min_density: float = 8.0, uniform_density: bool = False,
                                         limit_adaptive_depth: int = 100):
        """Density-adaptive levels (``hashtree.py:261-285``); ``uniform_density`` puts every point on
        the finest level."""
        if uniform_density:
            self.xyz_density = torch.full((self.xyz.size(0),), 1.0e6, device=self.device)
        else:
            self.xyz_density = self._density(density_depth)
        self.xyz_depth = self._branches[self.ENCODER].build_hierarchy_adaptive(
            self.xyz, self.xyz_density, log_base, min_density, limit_adaptive_depth)

    def split_data(self, xyz, branch: int, data_depth: int, data):
        return self._get_branch(branch).split_data(xyz, data_depth, data)

    def splat_data(self, xyz, branch: int, data_depth: int, data=None, check_corr: bool = True,
                   return_nf_mask: bool = False):
        return self._get_branch(branch).splat_data(xyz, data_depth, data, check_corr, return_nf_mask)
