"""The learned-basis (Neural Galerkin) forward/backward on one shape.

The flow of the reference's training step (``models/full_net.py:118-133`` with the splatting of
``jspsr/__init__.py:36-47``): density-adaptive tree, normals splatted with 1/density weights,
``Reconstructor.solve_multigrid`` with an ``AdditiveHermite`` basis and per-voxel features, field
evaluated at query points, MSE loss against a target field, gradients w.r.t. the normals and the
per-voxel basis features.  Assembly and solve are one ``galerkin.GalerkinSolve`` with a hand-written
adjoint; ``LearnedBatch`` runs many shapes through one such function, so that every level's forward
and adjoint solves of all shapes go to the device as one batched persistent PCG launch.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Dict

import numpy as np
import torch

from ..bases.hermite_ns import AdditiveHermite
from ..bases.additive_components import SinPeaks
from . import galerkin as G
from ._hash_backend import compute_density
from .hashtree import HashTree
from .reconstructor import Reconstructor


def hermite_basis() -> AdditiveHermite:
    """AdditiveHermite(n_degrees=6, SinPeaks(1..3)) as configured in ``configs/shapenet/full_net_base.yaml:54-59``."""
    return AdditiveHermite(6, [SinPeaks(1), SinPeaks(2), SinPeaks(3)], [0.0, 0.0, 0.0])


@dataclass
class LearnedStep:
    xyz: torch.Tensor
    normal: torch.Tensor
    query: torch.Tensor
    target: torch.Tensor
    voxel_size: float = 1.0 / 128
    depth: int = 3
    min_density: float = 2.0
    screen_alpha: float = 4.0
    solver: str = "cholmod"
    basis: AdditiveHermite = field(default_factory=hermite_basis)
    tree: HashTree = None
    sample_weight: torch.Tensor = None

    def build(self):
        """Tree and splatting weights (depend on positions only).  ``min_density=None`` layers the
        points at the median of their density (so that no level is empty on any shape)."""
        self.basis = self.basis.to(self.xyz.device)
        self.tree = HashTree(self.xyz, voxel_size=self.voxel_size, depth=self.depth)
        if self.min_density is None:
            dens = compute_density(self.xyz, 4 * self.voxel_size) / 16
            self.min_density = float(torch.median(dens))
        self.tree.build_encoder_hierarchy_adaptive(min_density=self.min_density)
        self.tree.reflect_decoder_coords()
        self.sample_weight = 1.0 / self.tree.xyz_density
        return self

    def init_features(self, sigma: float = 0.1, seed: int = 0) -> Dict[int, torch.Tensor]:
        """Bezier-like initial features plus N(0, sigma) noise, per level."""
        rng = np.random.default_rng(seed)
        out = {}
        for d in range(self.depth):
            f = torch.zeros((self.tree.get_coords_size(HashTree.DECODER, d), self.basis.get_feature_size()))
            self.basis.initialize_feature_value(f)
            f = f + torch.from_numpy(rng.normal(0, sigma, f.shape).astype(np.float32))
            out[d] = f.to(self.xyz.device)
        return out

    def normal_data(self, normal: torch.Tensor) -> Dict[int, torch.Tensor]:
        t, sw = self.tree, self.sample_weight
        out = {}
        for d in range(t.depth):
            m = t.xyz_depth == d
            if not torch.any(m):
                continue
            nd = t.splat_data(self.xyz[m], t.DECODER, d, normal[m] * sw[m, None])
            out[d] = nd / (t.get_stride(t.DECODER, d) ** 3)
        return out

    def forward(self, normal: torch.Tensor, feats: Dict[int, torch.Tensor]):
        """(loss, chi at the queries, reconstructor); differentiable in ``normal`` and ``feats``."""
        rec = Reconstructor(self.tree, self.basis, feats)
        rec.sample_weight = self.sample_weight
        rec.solve_multigrid(self.depth - 1, 0, self.normal_data(normal), screen_alpha=self.screen_alpha,
                            screen_xyz=self.xyz, solver=self.solver, verbose=False)
        chi = rec.evaluate_chi(self.query)
        return torch.mean((chi - self.target) ** 2), chi, rec

    def loss_and_grad(self, normal: torch.Tensor, feats: Dict[int, torch.Tensor]):
        n = normal.detach().clone().requires_grad_(True)
        f = {d: v.detach().clone().requires_grad_(True) for d, v in feats.items()}
        loss, chi, rec = self.forward(n, f)
        loss.backward()
        return float(loss.detach()), n.grad, {d: v.grad for d, v in f.items()}, chi.detach(), rec


class LearnedBatch:
    """Many shapes of the learned form at once: one ``GalerkinSolve`` for all of them."""

    def __init__(self, steps):
        self.steps = [st if st.tree is not None else st.build() for st in steps]
        self.basis = self.steps[0].basis
        self.shapes = None

    def geometry(self):
        """Geometry of every shape (depends on the positions only; built once)."""
        if self.shapes is None:
            self.shapes = []
            for st in self.steps:
                data_levels = [d for d in range(st.depth) if bool(torch.any(st.tree.xyz_depth == d))]
                self.shapes.append(G.ShapeGeometry.build(st.tree, st.tree.DECODER, st.depth - 1, 0, data_levels,
                                                         st.xyz, st.screen_alpha, 0.1,
                                                         self.basis.get_domain_range()))
        return self.shapes

    def forward(self, normals, feats_list):
        """(summed loss, per-shape losses, per-shape chi at the queries); differentiable in every
        shape's normals and features."""
        shapes = self.geometry()
        nd_list = [st.normal_data(n) for st, n in zip(self.steps, normals)]
        sols = G.galerkin_solve(self.basis, shapes, feats_list, nd_list, self.steps[0].solver)
        losses, chis = [], []
        for st, f, x in zip(self.steps, feats_list, sols):
            chi_pts = sum(st.tree.evaluate_interpolated(st.xyz, self.basis, f[d], d, x[d]) for d in x)
            iso = (chi_pts * st.sample_weight).sum() / st.sample_weight.sum()
            chi = sum(st.tree.evaluate_interpolated(st.query, self.basis, f[d], d, x[d]) for d in x) - iso
            losses.append(torch.mean((chi - st.target) ** 2))
            chis.append(chi)
        return torch.stack(losses).sum(), losses, chis
