"""The C / OpenMP restatement of the reconstruction (``oracle/spsr_omp.c``) against the golden
vectors of the reference's own Python run and against the numpy restatement.

This is the checker for the full-size parity tests and the timed CPU baseline, so it is pinned the
same way as ``oracle/spsr.py``: integer structure (point levels, voxel coordinates, matrix pattern,
dual cubes, faces) equal, FP quantities to the FP32 rounding of the reference's torch arithmetic.
"""
import numpy as np
import pytest

from oracle import fast as F
from oracle import spsr as S

CASES = ["torus_small", "torus_adaptive", "sq_noisy"]


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("name", CASES)
def test_fast_oracle_matches_reference_path(golden, name):
    g = golden(name)
    vs, depth, md, alpha = g["params"]
    depth = int(depth)
    r = F.reconstruct(g["xyz"], g["nrm"], vs, depth, md, alpha, cg_tol=1e-14, threads=4)
    assert rel(r["density"], g["density"]) < 2e-6
    np.testing.assert_array_equal(r["levels"], g["levels"])
    for d in range(depth):
        np.testing.assert_array_equal(r[f"coords{d}"], g[f"coords{d}"])
        assert r[f"cols{d}"].size == int(g[f"lhs{d}_nnz"])
        assert rel(r[f"rhs{d}"], g[f"lhs{d}_rhs"]) < 5e-6
        rp, cols, vals = r[f"rowptr{d}"], r[f"cols{d}"], r[f"vals{d}"]
        probe = g[f"lhs{d}_probe"].astype(np.float64)
        av = np.add.reduceat(vals * probe[cols], rp[:-1]) if vals.size else np.zeros(0)
        assert rel(av, g[f"lhs{d}_av"]) < 5e-6
        assert rel(r[f"x{d}"], g[f"x{d}"]) < 1e-5
    np.testing.assert_array_equal(r["faces"], g["faces"])
    assert np.abs(r["vertices"] - g["vertices"]).max() < 1e-5


def test_fast_oracle_matches_numpy_oracle():
    """Same algorithm, same structure decisions: identical integers, FP64 rounding-level differences."""
    from jspsr import synthetic
    xyz, nrm = synthetic.torus(n=3000, seed=0)
    vs, depth, md, alpha = 1 / 64, 3, 0.5, 4.0
    sol = S.solve_multigrid(xyz, nrm, vs, depth, md, alpha)
    mesh = S.extract_multiscale_mesh(sol, xyz)
    for threads in (1, 4):
        r = F.reconstruct(xyz, nrm, vs, depth, md, alpha, cg_tol=1e-14, threads=threads)
        np.testing.assert_array_equal(r["levels"], sol.levels)
        for d in range(depth):
            np.testing.assert_array_equal(r[f"coords{d}"], sol.grids[d].coords)
            assert rel(r[f"rhs{d}"], sol.rhs[d]) < 1e-12
            assert rel(r[f"x{d}"], sol.x[d]) < 1e-11
        np.testing.assert_array_equal(r["cubes"], mesh.acc[:, :, 0])
        assert np.abs(r["dual_values"] - mesh.dual_values).max() < 1e-12
        np.testing.assert_array_equal(r["faces"], mesh.faces)
        assert np.abs(r["vertices"] - mesh.vertices).max() < 1e-12


def test_fast_oracle_refuses_empty_level():
    from jspsr import synthetic
    xyz, nrm = synthetic.torus(n=2000, seed=0)
    with pytest.raises(ValueError):
        F.reconstruct(xyz, nrm, 1 / 64, 3, 1e9, 4.0)
