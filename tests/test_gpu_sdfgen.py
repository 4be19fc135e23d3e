"""Exact k nearest neighbours and the signed distance from oriented points (``jspsr.sdfgen``)
against the oracle (scipy's exact k-d tree and a numpy restatement of the reference's voting,
``ext/sdfgen/sdf_from_points.cu:31-68``), at the training loop's k = 8, stdv = 0.02."""
import numpy as np
import pytest
import torch

from oracle import ops as O

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda", 0)


def cloud(n_ref, n_query, seed):
    from jspsr import synthetic
    xyz, nrm, _ = synthetic.superquadrics(n_ref, k=2, seed=seed)
    rng = np.random.default_rng(seed)
    near = xyz[rng.integers(0, n_ref, n_query)] + rng.normal(0, 0.02, (n_query, 3))
    far = rng.uniform(-0.5, 1.5, (n_query // 10, 3))                 # also queries well off the surface
    return xyz, nrm, np.concatenate([near, far]).astype(np.float32)


@pytest.mark.parametrize("k", [1, 8, 16])
def test_knn_exact_sets(k):
    from jspsr import sdfgen
    xyz, nrm, q = cloud(50000, 20000, seed=k)
    idx, d2 = sdfgen.knn(torch.from_numpy(q).to(DEV), torch.from_numpy(xyz).to(DEV), k)
    idx, d2 = idx.cpu().numpy(), d2.cpu().numpy()
    ref_idx, ref_d2 = O.knn(q, xyz, k + 1)
    # FP32 distances against FP64 ones
    assert np.abs(d2 - ref_d2[:, :k]).max() <= 1e-5 * max(1.0, ref_d2.max())
    # the index sets wherever the k-th and (k+1)-th distances are not tied within FP32 rounding
    sep = ref_d2[:, k] - ref_d2[:, k - 1] > 1e-5 * ref_d2[:, k]
    assert sep.mean() > 0.99
    got = np.sort(idx[sep], 1)
    want = np.sort(ref_idx[sep, :k], 1)
    assert np.array_equal(got, want)


def test_sdf_from_points_matches_reference_rule():
    from jspsr import sdfgen
    xyz, nrm, q = cloud(60000, 30000, seed=7)
    sdf = sdfgen.sdf_from_points(torch.from_numpy(q).to(DEV), torch.from_numpy(xyz).to(DEV),
                                 torch.from_numpy(nrm).to(DEV), 8, 0.02).cpu().numpy()
    ref, idx = O.sdf_from_points(q, xyz, nrm, 8, 0.02)
    _, d2 = O.knn(q, xyz, 9)
    # decided cases: the 8-neighbour set is not tied, no vote within rounding of 0, the magnitude rule
    # not within rounding of stdv
    ray = q[:, None, :].astype(np.float64) - xyz[idx]
    dots = np.sum(nrm[idx].astype(np.float64) * ray, -1)
    clear = (d2[:, 8] - d2[:, 7] > 1e-5 * d2[:, 8]) & (np.abs(dots).min(1) > 1e-6) & \
        (np.abs(np.sqrt(d2[:, 0]) - 0.02) > 1e-6)
    assert clear.mean() > 0.99
    np.testing.assert_array_equal(np.sign(sdf[clear]), np.sign(ref[clear]))
    assert np.abs(sdf[clear] - ref[clear]).max() <= 1e-5
