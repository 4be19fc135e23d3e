"""Parity at the benchmark's own configurations, against the FP64 oracle on the same clouds.

The throughput numbers are measured on 300,000 points on 4 superquadrics (voxel 1/512, 4 levels,
min_density 2, screening 4, solver ``pcg-mixed@tol=1e-7``); this test runs exactly that
reconstruction and the C/OpenMP oracle (``oracle/fast.py``, FP64, every level solved to a relative
residual of 1e-12) on the same cloud and checks every stage:

* point levels, voxel coordinates of every level, and the CSR pattern of every level's matrix:
  equal (integer structure is bit-exact);
* matrix values and right-hand sides: relative L2 <= 1e-6 (FP32 screening inputs, FP64 assembly);
* solutions, the field at the mesh samples and the mesh vertices: relative L2 <= 1e-5;
* marching-cubes topology: the oracle's field, fed through the production dual-MC and vertex
  kernels, gives the oracle's faces exactly; with the GPU's own field, every sample whose sign
  differs from the oracle's is counted and reported (the field error near 1e-7 can flip a sample
  that lies within that distance of the level set).

A deep hierarchy (7 levels: level ratios up to 64, beyond the reference's tables, which stop at
16) is checked the same way, through both dual-centre routes (the rank bitmap and the sorted keys
that very deep scenes use).
"""
import numpy as np
import pytest
import torch

from oracle import fast as F

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda", 0)
TOL = 1e-5           # solution / field / vertex relative L2 against the FP64 oracle
TOL_SYSTEM = 1e-6    # matrix values and right-hand sides


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def run_both(xyz, nrm, vs, depth, md, alpha, solver, dual_grid_max_words=None):
    from jspsr.core.pipeline import Reconstruction
    ref = F.reconstruct(xyz, nrm, vs, depth, md, alpha, cg_tol=1e-12)
    rec = Reconstruction(torch.from_numpy(xyz).to(DEV), torch.from_numpy(nrm).to(DEV), vs, depth, md, alpha,
                         solver=solver)
    if dual_grid_max_words is not None:
        rec.dual_grid_max_words = dual_grid_max_words
    v, f = rec.run()
    return ref, rec, v.cpu().numpy(), f.cpu().numpy()


def check_parity(ref, rec, v, f, depth, report):
    np.testing.assert_array_equal(rec.point_level.cpu().numpy(), ref["levels"])
    for d in range(depth):
        lv = rec.levels[d]
        np.testing.assert_array_equal(lv.coords.cpu().numpy(), ref[f"coords{d}"], err_msg=f"level {d}")
        np.testing.assert_array_equal(lv.rowptr.cpu().numpy(), ref[f"rowptr{d}"], err_msg=f"level {d}")
        np.testing.assert_array_equal(lv.cols.cpu().numpy(), ref[f"cols{d}"], err_msg=f"level {d}")
        e_a = rel(lv.vals64.cpu().numpy(), ref[f"vals{d}"])
        e_b = rel(lv.rhs.cpu().numpy(), ref[f"rhs{d}"])
        e_x = rel(lv.x64.cpu().numpy(), ref[f"x{d}"])
        report[f"level{d}"] = dict(voxels=lv.n, nnz=lv.nnz, matrix=e_a, rhs=e_b, solution=e_x)
        assert e_a <= TOL_SYSTEM and e_b <= TOL_SYSTEM, (d, e_a, e_b)
        assert e_x <= TOL, (d, e_x)
    # field at the mesh samples
    vals = rec.mesh_info["values"].cpu().numpy()
    assert vals.shape == ref["dual_values"].shape
    e_f = rel(vals, ref["dual_values"])
    flips = int(np.count_nonzero((vals < 0) != (ref["dual_values"] < 0)))
    report["field"] = e_f
    report["sign_flips"] = flips
    report["samples"] = int(vals.size)
    assert e_f <= TOL, e_f
    own_vids = rec.mesh_vids.cpu().numpy().astype(np.int64)       # the GPU mesh's own vertex pairs
    # topology: the oracle's field through the production marching cubes
    cubes = rec.dual_cubes()[:, :, 0].cpu().numpy()
    np.testing.assert_array_equal(cubes, ref["cubes"])
    acc, cnt, pos = rec.mesh_info["acc_ids"], rec.mesh_info["cnt"], rec.mesh_info["positions"]
    v_o, f_o = rec.marching_cubes(acc, cnt, pos, torch.from_numpy(ref["dual_values"]).to(DEV).float())
    np.testing.assert_array_equal(f_o.cpu().numpy(), ref["faces"])
    report["faces_from_oracle_field_equal"] = True
    # vertices of the GPU's own mesh against the oracle's, matched by primal-sample pair
    vids = own_vids
    keys = np.empty(v.shape[0], np.int64)
    keys[f.reshape(-1)] = (vids[:, 0] << 32) | vids[:, 1]
    common, ia, ib = np.intersect1d(keys, ref["vertex_keys"], assume_unique=True, return_indices=True)
    e_v = rel(v[ia], ref["vertices"][ib])
    report["vertices"] = e_v
    report["vertices_compared"] = int(common.size)
    report["vertices_gpu_only"] = int(v.shape[0] - common.size)
    report["vertices_oracle_only"] = int(ref["vertices"].shape[0] - common.size)
    assert e_v <= TOL, e_v
    if flips == 0:
        np.testing.assert_array_equal(f, ref["faces"])
    # a sign flip changes the cubes around one sample: bounded by what one sample can touch
    assert report["vertices_gpu_only"] <= 12 * 8 * flips and report["vertices_oracle_only"] <= 12 * 8 * flips


def test_parity_superquadrics_300k_benchmark_config(record_property):
    from jspsr import synthetic
    xyz, nrm, _ = synthetic.superquadrics(300000, k=4, seed=0)
    ref, rec, v, f = run_both(xyz, nrm, 1.0 / 512, 4, 2.0, 4.0, "pcg-mixed@tol=1e-7")
    report = {}
    check_parity(ref, rec, v, f, 4, report)
    print("superquadrics-300k parity:", report)
    record_property("parity", report)


@pytest.mark.parametrize("route", ["bitmap", "sorted_keys"])
def test_parity_deep_hierarchy_7_levels(route, record_property):
    """A room scene at 2 cm with 7 levels: cross-level ratios up to 64 (tables extended beyond the
    reference's 16), coarse cells of 64 voxels in the dual grid."""
    from jspsr import synthetic
    xyz, nrm = synthetic.room(n=200_000, seed=0, n_objects=12)
    ref, rec, v, f = run_both(xyz, nrm, 0.02, 7, 2.0, 4.0, "pcg-mixed@tol=1e-7",
                              dual_grid_max_words=0 if route == "sorted_keys" else None)
    report = {}
    check_parity(ref, rec, v, f, 7, report)
    print(f"room-200k 7 levels ({route}) parity:", report)
    record_property("parity", report)
