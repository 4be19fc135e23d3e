"""The reference's top-level flow (``jspsr/__init__.py:21-61``) written against this package's
mirror of its classes (HashTree, Reconstructor, BezierTensorBasis, solve_sparse) on libngs,
checked against the reference's own run (golden fixtures)."""
import sys
from pathlib import Path

import numpy as np
import pytest
import torch

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT / "neural-galerkin_b200"))

pytestmark = pytest.mark.gpu


def _reference_flow(xyz, nrm, vs, depth, md, alpha, solver):
    from jspsr.core.hashtree import HashTree
    from jspsr.core.reconstructor import Reconstructor
    from jspsr.bases.bezier_tensor import BezierTensorBasis
    ht = HashTree(xyz, voxel_size=vs, depth=depth)
    ht.build_encoder_hierarchy_adaptive(min_density=md)
    ht.reflect_decoder_coords()
    normal_data = {}
    sw = 1.0 / ht.xyz_density
    for d in range(ht.depth):
        m = ht.xyz_depth == d
        if not torch.any(m):
            continue
        nd = ht.splat_data(xyz[m], ht.DECODER, d, nrm[m] * sw[m, None])
        normal_data[d] = nd / (ht.get_stride(ht.DECODER, d) ** 3)
    rec = Reconstructor(ht, BezierTensorBasis())
    rec.sample_weight = sw
    rec.solve_multigrid(ht.depth - 1, 0, normal_data, screen_alpha=alpha, screen_xyz=xyz, solver=solver,
                        verbose=False)
    v, f = rec.extract_multiscale_mesh(n_upsample=2, build_o3d_mesh=False)
    return ht, rec, v, f


@pytest.mark.parametrize("case", ["torus_small", "sq_noisy"])
def test_reference_flow_matches_golden(case):
    g = np.load(ROOT / "tests" / "golden" / f"{case}.npz")
    vs, depth, md, alpha = float(g["params"][0]), int(g["params"][1]), float(g["params"][2]), float(g["params"][3])
    dev = torch.device("cuda:0")
    ht, rec, v, f = _reference_flow(torch.from_numpy(g["xyz"]).to(dev), torch.from_numpy(g["nrm"]).to(dev), vs,
                                    depth, md, alpha, "cholmod")
    assert np.array_equal(ht.xyz_depth.cpu().numpy(), g["levels"])
    for d in range(depth):
        assert np.array_equal(ht.get_coords(ht.DECODER, d).cpu().numpy(), g[f"coords{d}"]), d
        x = rec.solutions[d].detach().cpu().numpy().astype(np.float64)
        ref = g[f"x{d}"].astype(np.float64)
        assert np.linalg.norm(x - ref) <= 1e-5 * np.linalg.norm(ref), d
    vv, ff = v.cpu().numpy(), f.cpu().numpy()
    if ff.shape == g["faces"].shape and np.array_equal(ff, g["faces"]):
        assert np.abs(vv - g["vertices"]).max() < 1e-4
    else:
        # a dual-corner value within rounding of the iso level can flip one cube's sign pattern
        assert abs(ff.shape[0] - g["faces"].shape[0]) <= 0.002 * g["faces"].shape[0]


def test_reference_flow_pcg_solver_matches_pipeline():
    """The reference's default solver string ("pcg", rel-tol 1e-5) through solve_sparse, against the
    production pipeline's FP64-refined solve on the same cloud."""
    import jspsr
    from jspsr.synthetic import torus
    xyz, nrm = torus(n=10000, seed=0)
    dev = torch.device("cuda:0")
    ht, rec, v, f = _reference_flow(torch.from_numpy(xyz).to(dev), torch.from_numpy(nrm).to(dev), 1 / 128, 3, 1.5,
                                    4.0, "pcg")
    r = jspsr.reconstruct(torch.from_numpy(xyz).to(dev), torch.from_numpy(nrm).to(dev), 1 / 128, depth=3,
                          min_density=1.5, screen_alpha=4.0, return_reconstruction=True)
    recon = r[2]
    for d in range(3):
        assert torch.equal(ht.get_coords(ht.DECODER, d), recon.levels[d].coords.to(torch.int32)), d
        a = rec.solutions[d].detach().double()
        b = recon.levels[d].x64
        assert float(torch.linalg.norm(a - b) / torch.linalg.norm(b)) < 5e-4, d
