"""Hierarchy builders and queries of the reference's HashTree beside the density-adaptive one,
rebuilt on libngs, against the reference's own run (``tests/golden/structure.npz``): dense and
policy-subdivided hierarchies, voxel status, expanded / conforming coordinates, test grid and the
trilinear split of voxel data."""
import sys
from pathlib import Path

import numpy as np
import pytest
import torch

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT / "neural-galerkin_b200"))

pytestmark = pytest.mark.gpu

G = np.load(ROOT / "tests" / "golden" / "structure.npz")


def _count_policy(xyz, inds, min_count=6):
    counts = torch.bincount(inds)
    return counts[inds] >= min_count


@pytest.fixture(scope="module")
def dense():
    from jspsr.core.hashtree import HashTree
    t = HashTree(torch.from_numpy(G["xyz"]).cuda(), voxel_size=1.0 / 64, depth=3)
    t.build_encoder_hierarchy_dense(expand_range=3)
    t.reflect_decoder_coords()
    return t


def test_dense_hierarchy_bit_exact(dense):
    for d in range(3):
        assert np.array_equal(dense.get_coords(dense.ENCODER, d).cpu().numpy(), G[f"dense{d}"]), d
    dens = dense.xyz_density.cpu().numpy()
    assert np.abs(dens - G["dense_density"]).max() <= 2e-6 * np.abs(G["dense_density"]).max()


def test_voxel_status(dense):
    for d in range(3):
        probe = torch.from_numpy(G[f"probe{d}"]).cuda()
        st = dense.evaluate_voxel_status(dense.ENCODER, probe, d).cpu().numpy()
        assert np.array_equal(st, G[f"status{d}"]), d


def test_expanded_and_conforming_coords(dense):
    for d in range(3):
        assert np.array_equal(dense._get_branch(dense.ENCODER).get_coords(d, expand=3).cpu().numpy(), G[f"expand{d}"]), d
        assert np.array_equal(dense._get_branch(dense.ENCODER).get_coords(d, conforming=True).cpu().numpy(), G[f"conform{d}"]), d


def test_split_data_and_test_grid(dense):
    xyz = torch.from_numpy(G["xyz"]).cuda()
    for d in range(3):
        got = dense.split_data(xyz, dense.ENCODER, d, torch.from_numpy(G[f"data{d}"]).cuda()).cpu().numpy()
        assert np.abs(got - G[f"split{d}"]).max() <= 1e-5, d
    q, base = dense.get_test_grid(3, 1, expand=0, conforming=False)
    assert np.array_equal(base.cpu().numpy(), G["test_grid_base"])
    assert np.abs(q.cpu().numpy() - G["test_grid_pos"]).max() <= 1e-6


def test_subdivision_hierarchy_bit_exact():
    from jspsr.core.hashtree import HashTree
    t = HashTree(torch.from_numpy(G["xyz"]).cuda(), voxel_size=1.0 / 64, depth=3)
    t.build_hierarchy_subdivide(_count_policy, expand=True, min_count=6)
    assert np.array_equal(t.xyz_depth.cpu().numpy(), G["sub_depth"])
    for d in range(3):
        assert np.array_equal(t.get_coords(t.ENCODER, d).cpu().numpy(), G[f"sub{d}"]), d
