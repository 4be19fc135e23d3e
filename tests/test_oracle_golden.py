"""The FP64 oracle against golden vectors produced by the reference's own Python code.

``tests/golden/make_golden.py`` ran the reference's unmodified ``jspsr``
package on CPU (CUDA ops replaced by CPU restatements, linear solves exact) and
stored intermediates.  Integer structure must match exactly; FP quantities to
the FP32 rounding of the reference's torch arithmetic.
"""
import numpy as np
import pytest

from oracle import spsr as S
from oracle import tables as T
from oracle import mc_tables as MC
from oracle import ops as O

CASES = ["torus_small", "torus_adaptive", "sq_noisy"]


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("name", CASES)
def test_oracle_matches_reference_path(golden, name):
    g = golden(name)
    vs, depth, md, alpha = g["params"]
    depth = int(depth)
    sol = S.solve_multigrid(g["xyz"], g["nrm"], vs, depth, md, alpha, keep_lhs=True)
    assert rel(sol.density, g["density"]) < 2e-6
    np.testing.assert_array_equal(sol.levels, g["levels"])
    for d in range(depth):
        np.testing.assert_array_equal(sol.grids[d].coords, g[f"coords{d}"])
        assert sol.lhs[d].nnz == int(g[f"lhs{d}_nnz"])
        assert rel(sol.rhs[d], g[f"lhs{d}_rhs"]) < 5e-6
        assert rel(sol.lhs[d] @ g[f"lhs{d}_probe"].astype(np.float64), g[f"lhs{d}_av"]) < 5e-6
        assert rel(sol.x[d], g[f"x{d}"]) < 1e-5
    mesh = S.extract_multiscale_mesh(sol, g["xyz"])
    np.testing.assert_array_equal(mesh.faces, g["faces"])
    assert np.abs(mesh.vertices - g["vertices"]).max() < 1e-5


def test_bezier_tables_match_reference_definition(golden):
    g = golden("bezier_tables")
    t = T.bezier_tables(3)
    for m in range(3):
        M = 2 ** m
        np.testing.assert_allclose(t["SHIFTED_SELF_INTEGRAL"][m], g[f"ff{m}"], atol=1e-12)
        np.testing.assert_allclose(t["SHIFTED_DERIVATIVE_INTEGRAL"][m], M * g[f"dfdf{m}"], atol=1e-11)
        np.testing.assert_allclose(t["DERIVATIVE_PARTIAL_INTEGRAL"][m], g[f"f{m}"], atol=1e-12)
        np.testing.assert_allclose(t["PARTIAL_INTEGRAL"][m], M * g[f"df{m}"], atol=1e-11)
        if m:
            np.testing.assert_allclose(t["INV_DERIVATIVE_PARTIAL_INTEGRAL"][m - 1], g[f"finv{m}"], atol=1e-12)
            np.testing.assert_allclose(t["INV_PARTIAL_INTEGRAL"][m - 1], g[f"dfinv{m}"], atol=1e-12)


def test_bezier_known_answers():
    t = T.bezier_tables(2)
    assert abs(t["SHIFTED_SELF_INTEGRAL"][0][2] - 11 / 5) < 1e-14          # int B^2 = 4 * 11/20
    assert abs(t["SHIFTED_DERIVATIVE_INTEGRAL"][0][2] - 4.0) < 1e-14        # int B'^2
    assert abs(sum(t["DERIVATIVE_PARTIAL_INTEGRAL"][1]) - 4.0) < 1e-13      # int B(x/2) dx = 2 * 2


def test_mc_tables_match_reference(golden):
    g = golden("mc_tables")
    np.testing.assert_array_equal(MC.TRI_TABLE.reshape(-1), g["tri"])
    np.testing.assert_array_equal(MC.EDGE_TABLE, g["edge"])
    np.testing.assert_array_equal(MC.NUM_VERTS_TABLE, g["numverts"])


def test_fnv_known_answers(golden):
    g = golden("fnv_keys")
    np.testing.assert_array_equal(O.hash_cuda(g["coords"]), g["keys"])
    # hand-computed FNV-1a of (0,0,0): fold of the 64-bit hash
    h = 14695981039346656037
    for _ in range(3):
        h = ((h ^ 0) * 1099511628211) % (1 << 64)
    assert int(O.hash_cuda(np.zeros((1, 3), np.int32))[0]) == (h >> 60) ^ (h & 0x0FFFFFFFFFFFFFFF)


def test_range_kernel_prefix_property():
    k = S.range_kernel(7)
    assert tuple(k[0]) == (0, 0, 0)
    assert np.abs(k[:27]).max() == 1 and np.abs(k[:125]).max() == 2
    assert len({tuple(r) for r in k}) == 343
