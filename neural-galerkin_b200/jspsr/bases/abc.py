"""Basis interface of the Galerkin solver (reference: ``jspsr/bases/abc.py:6-88``)."""
from abc import ABC, abstractmethod

import torch


class BaseBasis(torch.nn.Module, ABC):
    """A per-voxel basis function family B_k(x), evaluated relative to the voxel centre in voxel units."""

    @classmethod
    def get_domain_range(cls) -> int:
        """Support of a basis function, in voxels (3 for the quadratic B-spline)."""
        return 3

    def get_feature_size(self) -> int:
        """Feature channels a voxel needs to describe its basis function (0: fixed basis)."""
        return 0

    @abstractmethod
    def initialize_feature_value(self, feat: torch.Tensor) -> None:
        """Initialise features (M, K) so that the basis starts as the B-spline."""

    @abstractmethod
    def evaluate(self, feat, xyz, feat_ids) -> torch.Tensor:
        """Values (N,) at local coordinates xyz (N, 3) of the voxels feat_ids (N,)."""

    @abstractmethod
    def evaluate_derivative(self, feat, xyz, feat_ids, stride: int) -> torch.Tensor:
        """Gradients (N, 3) per finest-voxel unit (local derivative / stride)."""

    @abstractmethod
    def integrate_deriv_deriv_product(self, source_feat, target_feat, rel_pos, source_stride: int,
                                      target_stride: int, source_ids, target_ids) -> torch.Tensor:
        """int grad B_source . grad B_target for each pair (N,) (the LHS stiffness)."""

    @abstractmethod
    def integrate_const_deriv_product(self, data, target_feat, rel_pos, data_stride: int, target_stride: int,
                                      target_ids) -> torch.Tensor:
        """int grad B_target . data over a constant data voxel, for each pair (N,) (the RHS)."""
