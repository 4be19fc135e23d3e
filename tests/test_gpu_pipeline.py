"""Parity of the B200 reconstruction pipeline with the FP64 oracle and the golden vectors.

Integer structure (voxel coordinates, levels, neighbour structure, dual grid,
mesh topology for a given sign pattern) must be bit-exact.  Floating-point
results (density, assembled systems, per-level solutions, field, vertices) must
agree with the FP64 oracle within 1e-5 relative L2 (the tolerance the path is
specified to), written per assertion below.
"""
import numpy as np
import pytest
import torch

from oracle import spsr as S

pytestmark = pytest.mark.gpu
CASES = ["torus_small", "torus_adaptive", "sq_noisy"]
TOL = 1e-5


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(scope="module")
def cases(golden):
    out = {}
    for name in CASES:
        g = golden(name)
        vs, depth, md, alpha = g["params"]
        sol = S.solve_multigrid(g["xyz"], g["nrm"], vs, int(depth), md, alpha, keep_lhs=True)
        mesh = S.extract_multiscale_mesh(sol, g["xyz"])
        out[name] = (g, sol, mesh)
    return out


def pairs_of(rec, lv):
    """The level's point basis transposed per row, built through the C ABI."""
    from jspsr import _lib as L
    st = L.stream()
    counts = torch.zeros(lv.n, dtype=torch.int32, device=lv.rows.device)
    mx = torch.zeros(1, dtype=torch.int32, device=lv.rows.device)
    L.call("ngs_mf_count", L.ptr(lv.rows), rec.n, lv.n, L.ptr(counts), L.ptr(mx), st)
    t_ptr = torch.empty(lv.n + 1, dtype=torch.int64, device=lv.rows.device)
    L.scan(counts, out=t_ptr[:lv.n], total=t_ptr[lv.n:])
    E = int(t_ptr[lv.n])
    cursor = torch.zeros(lv.n, dtype=torch.int32, device=lv.rows.device)
    tmp = (torch.empty(E, dtype=torch.int32, device=lv.rows.device), torch.empty(E, device=lv.rows.device))
    t_point = torch.empty(E, dtype=torch.int32, device=lv.rows.device)
    t_phi = torch.empty(E, device=lv.rows.device)
    L.call("ngs_mf_fill", L.ptr(lv.rows), L.ptr(lv.phi), rec.n, L.ptr(t_ptr), lv.n, L.ptr(cursor), L.ptr(tmp[0]),
           L.ptr(tmp[1]), L.ptr(t_point), L.ptr(t_phi), st)
    return t_ptr, t_point, t_phi


def run_gpu(g, solver="pcg-mixed@tol=1e-9"):
    from jspsr.core.pipeline import Reconstruction
    vs, depth, md, alpha = g["params"]
    xyz = torch.from_numpy(g["xyz"]).cuda()
    nrm = torch.from_numpy(g["nrm"]).cuda()
    rec = Reconstruction(xyz, nrm, vs, int(depth), md, alpha, solver=solver)
    v, f = rec.run()
    rec.check_solves()
    return rec, v.cpu().numpy(), f.cpu().numpy()


@pytest.fixture(scope="module")
def gpu_runs(cases):
    return {name: run_gpu(g) for name, (g, _, _) in cases.items()}


@pytest.mark.parametrize("name", CASES)
def test_tree_bit_exact(cases, gpu_runs, name):
    g, sol, _ = cases[name]
    rec = gpu_runs[name][0]
    dens = rec.density.cpu().numpy()
    assert np.max(np.abs(dens - sol.density) / sol.density) < TOL          # FP32 KDE vs FP64
    np.testing.assert_array_equal(rec.point_level.cpu().numpy(), g["levels"])
    for d, lv in enumerate(rec.levels):
        np.testing.assert_array_equal(lv.coords.cpu().numpy(), g[f"coords{d}"])


@pytest.mark.parametrize("name", CASES)
def test_system_matches_oracle(cases, gpu_runs, name):
    import scipy.sparse as sp
    g, sol, _ = cases[name]
    rec = gpu_runs[name][0]
    for d, lv in enumerate(rec.levels):
        a = sp.csr_matrix((lv.vals64.cpu().numpy(), lv.cols.cpu().numpy(), lv.rowptr.cpu().numpy()),
                          shape=(lv.n, lv.n))
        ref = sol.lhs[d]
        assert a.nnz == ref.nnz == int(g[f"lhs{d}_nnz"])
        np.testing.assert_array_equal(a.indptr, ref.indptr)
        np.testing.assert_array_equal(a.indices, ref.indices)
        assert rel(a.data, ref.data) < 1e-6                                 # FP32 basis values, FP64 sums
        assert rel(lv.rhs.cpu().numpy(), sol.rhs[d]) < TOL


@pytest.mark.parametrize("name", CASES)
def test_solution_matches_oracle(cases, gpu_runs, name):
    _, sol, _ = cases[name]
    rec = gpu_runs[name][0]
    for d, lv in enumerate(rec.levels):
        assert rel(lv.x64.cpu().numpy(), sol.x[d]) < TOL, (d, rec.solve_stats[d])


@pytest.mark.parametrize("name", CASES)
def test_field_matches_oracle(cases, gpu_runs, name):
    g, sol, _ = cases[name]
    rec = gpu_runs[name][0]
    rng = np.random.default_rng(0)
    q = (g["xyz"] + rng.normal(0, 0.01, g["xyz"].shape)).astype(np.float32)
    ours = rec.chi_raw(torch.from_numpy(q).cuda()).cpu().numpy()
    assert rel(ours, S.evaluate_chi_raw(sol, q)) < TOL
    grad = rec.chi_raw(torch.from_numpy(q).cuda(), grad=True).cpu().numpy()
    assert rel(grad, S.evaluate_chi_raw(sol, q, grad=True)) < TOL


@pytest.mark.parametrize("name", CASES)
def test_dual_grid_bit_exact(cases, gpu_runs, name):
    _, _, mesh = cases[name]
    rec = gpu_runs[name][0]
    assert rec.mesh_info["counts"] == [mesh.n_primal[d] for d in sorted(mesh.n_primal)]
    np.testing.assert_array_equal(rec.dual_cubes().cpu().numpy(), mesh.acc)
    assert rel(rec.mesh_info["values"].cpu().numpy(), mesh.dual_values) < TOL


@pytest.mark.parametrize("name", CASES)
def test_cell_field_matches_point_field(gpu_runs, name):
    """The per-cell evaluation of the mesh samples (one neighbourhood read per cell and level,
    contracted axis by axis) sums the same terms as the per-sample evaluation: equal up to FP32
    rounding of the different summation order."""
    rec = gpu_runs[name][0]
    info = rec.mesh_info
    cells = rec.chi_cells(info["positions"]).cpu().numpy()
    points = rec.chi_raw(info["positions"]).cpu().numpy()
    assert np.abs(cells - points).max() <= 1e-6 * max(np.abs(points).max(), 1e-30)


@pytest.mark.parametrize("name", CASES)
def test_grouped_screening_terms(gpu_runs, name):
    """Cell keys from the kernel equal the torch formula; the screening RHS summed per run of a cell's
    points (segmented warp scans) equals the per-point atomics up to FP64 summation order."""
    from jspsr import _lib as L
    rec = gpu_runs[name][0]
    assert rec.alpha > 0
    for lv in rec.levels:
        present = lv.rows >= 0
        first = present.to(torch.int8).argmax(1)
        ref = lv.rows.gather(1, first[:, None]).squeeze(1).long() * 27 + first
        ref = torch.where(present.any(1), ref, torch.full_like(ref, -1))
        keys = torch.empty_like(ref)
        L.call("ngs_point_cell_keys", L.ptr(lv.rows), rec.n, L.ptr(keys), L.stream())
        assert torch.equal(keys, ref)
        skeys, order = torch.sort(keys)
        field = torch.rand(rec.n, device=lv.rows.device)
        for f in (None, field):
            a = torch.zeros(lv.n, dtype=torch.float64, device=lv.rows.device)
            b = torch.zeros_like(a)
            if f is None:
                L.call("ngs_screen_rhs", L.ptr(lv.rows), L.ptr(lv.phi), rec.n, None, 0.75, L.ptr(a), L.stream())
            else:
                L.call("ngs_correction_screen", L.ptr(lv.rows), L.ptr(lv.phi), rec.n, None, L.ptr(f), 0.75, L.ptr(a),
                       L.stream())
            L.call("ngs_screen_rhs_grouped", L.ptr(lv.rows), L.ptr(lv.phi), rec.n, None,
                   L.ptr(f) if f is not None else None, L.ptr(order), L.ptr(skeys), 0.75 if f is None else -0.75,
                   L.ptr(b), L.stream())
            assert rel(b.cpu().numpy(), a.cpu().numpy()) < 1e-12
            t_ptr, t_point, t_phi = pairs_of(rec, lv)   # the pair form: gathered per row
            c = torch.zeros_like(a)
            L.call("ngs_mf_screen_rhs", L.ptr(t_ptr), L.ptr(t_point), L.ptr(t_phi), lv.n,
                   L.ptr(f) if f is not None else None, 0.75 if f is None else -0.75, L.ptr(c), L.stream())
            assert rel(c.cpu().numpy(), a.cpu().numpy()) < 1e-12


@pytest.mark.parametrize("name", CASES)
def test_gram_from_pairs_equals_cell_grouped_atomics(gpu_runs, name):
    """The production screening Gram (per row from the transposed pairs, no atomics) equals the
    cell-grouped Gram with FP64 atomics up to FP64 summation order, on the assembled pattern."""
    from jspsr import _lib as L
    rec = gpu_runs[name][0]
    for d, lv in enumerate(rec.levels):
        st = L.stream()
        t_ptr, t_point, t_phi = pairs_of(rec, lv)
        a = torch.zeros(lv.nnz, dtype=torch.float64, device=lv.rows.device)
        b = torch.zeros_like(a)
        L.call("ngs_mf_gram", L.ptr(t_ptr), L.ptr(t_point), L.ptr(t_phi), lv.n, L.ptr(lv.rows),
               L.ptr(lv.phi), L.ptr(lv.masks), L.ptr(lv.rowptr), 1.5, L.ptr(a), st)
        keys = torch.empty(rec.n, dtype=torch.int64, device=lv.rows.device)
        L.call("ngs_point_cell_keys", L.ptr(lv.rows), rec.n, L.ptr(keys), st)
        skeys, order = torch.sort(keys)
        L.call("ngs_screen_gram_grouped", L.ptr(lv.rows), L.ptr(lv.phi), rec.n, None, L.ptr(order), L.ptr(skeys),
               L.ptr(lv.masks), L.ptr(lv.rowptr), 1.5, L.ptr(b), st)
        assert float(torch.linalg.norm(a - b) / torch.linalg.norm(b)) < 1e-13, d


@pytest.mark.parametrize("name", CASES)
def test_pair_form_reconstruction_equals_cell_grouping(cases, gpu_runs, name):
    """The whole reconstruction with every level's screening terms in pair form (the Gram per row
    from the transposed pairs, no atomics, no sort) solves the same systems."""
    from jspsr.core.pipeline import Reconstruction
    g, _, _ = cases[name]
    vs, depth, md, alpha = g["params"]
    rec = Reconstruction(torch.from_numpy(g["xyz"]).cuda(), torch.from_numpy(g["nrm"]).cuda(), vs, int(depth), md,
                         alpha, solver="pcg-mixed@tol=1e-9")
    rec.pair_row_limit = 1 << 30
    rec.run()
    rec.check_solves()
    assert all(lv.pair_form for lv in rec.levels)
    for lv, ref in zip(rec.levels, gpu_runs[name][0].levels):
        assert rel(lv.vals64.cpu().numpy(), ref.vals64.cpu().numpy()) < 1e-13
        assert rel(lv.rhs.cpu().numpy(), ref.rhs.cpu().numpy()) < 1e-6      # coarse solutions enter at tol
        assert rel(lv.x64.cpu().numpy(), ref.x64.cpu().numpy()) < TOL


@pytest.mark.parametrize("name", CASES)
def test_mesh_matches_oracle(cases, gpu_runs, name, record_property):
    """Topology is bit-exact for a given sign pattern: the oracle's field, fed through the production
    dual marching cubes and vertex de-duplication, gives the oracle's faces exactly.  The GPU's own
    field (solved to 1e-9) must then have the oracle's sign at every sample of these golden cases, so
    that its own mesh equals the oracle's too; the number of sign differences is recorded."""
    g, _, mesh = cases[name]
    rec, v, f = gpu_runs[name]
    acc, cnt, pos = rec.mesh_info["acc_ids"], rec.mesh_info["cnt"], rec.mesh_info["positions"]
    v_o, f_o = rec.marching_cubes(acc, cnt, pos, torch.from_numpy(mesh.dual_values).cuda().float())
    np.testing.assert_array_equal(f_o.cpu().numpy(), mesh.faces)
    assert rel(v_o.cpu().numpy(), mesh.vertices) < TOL
    ours = rec.mesh_info["values"].cpu().numpy()
    flips = int(np.count_nonzero((ours < 0) != (mesh.dual_values < 0)))
    record_property("sign_flips", flips)
    assert flips == 0, f"{flips} samples with the other sign than the oracle's"
    np.testing.assert_array_equal(f, mesh.faces)
    assert rel(v, mesh.vertices) < TOL


def test_reference_solver_semantics(cases):
    """solver="pcg" reproduces the reference's FP32 PCG (tol 1e-5 on the recursive residual)."""
    g, sol, _ = cases["torus_small"]
    rec, _, _ = run_gpu(g, solver="pcg")
    for d, lv in enumerate(rec.levels):
        st = rec.solve_stats[d]
        assert st["status"] == 0 and st["resid"] <= 1e-5 * st["bnorm"] * 1.0001
        assert rel(lv.x64.cpu().numpy(), sol.x[d]) < 1e-3


def test_plain_fp64_comparator(cases):
    g, sol, _ = cases["torus_small"]
    rec, _, _ = run_gpu(g, solver="plain-fp64@tol=1e-10")
    for d, lv in enumerate(rec.levels):
        assert rel(lv.x64.cpu().numpy(), sol.x[d]) < 1e-6                  # system assembled from FP32 basis values


def test_public_reconstruct_roundtrip(cases):
    import jspsr
    g, _, mesh = cases["torus_small"]
    vs, depth, md, alpha = g["params"]
    v, f = jspsr.reconstruct(g["xyz"], g["nrm"], vs, int(depth), md, alpha, solver="pcg-mixed@tol=1e-9")
    assert isinstance(v, np.ndarray) and v.dtype == np.float32 and f.dtype == np.int64
    np.testing.assert_array_equal(f, mesh.faces)
    assert rel(v, mesh.vertices) < TOL


def test_empty_level_raises():
    import jspsr
    from jspsr import synthetic
    xyz, nrm = synthetic.torus(n=2000)
    with pytest.raises(ValueError, match="empty"):
        jspsr.reconstruct(xyz, nrm, 1.0 / 128, depth=3, min_density=32.0)


@pytest.mark.parametrize("name", ["torus_adaptive", "sq_noisy"])
def test_sorted_key_dual_centres_match_bitmap(cases, name):
    """Deep hierarchies de-duplicate dual centres by sorting packed corner keys instead of a rank
    bitmap over the box; forcing that route gives the same dual grid and mesh."""
    from jspsr.core.pipeline import Reconstruction
    g, _, _ = cases[name]
    vs, depth, md, alpha = g["params"]
    xyz = torch.from_numpy(g["xyz"]).cuda()
    nrm = torch.from_numpy(g["nrm"]).cuda()
    out = []
    rec = Reconstruction(xyz, nrm, vs, int(depth), md, alpha, solver="pcg-mixed@tol=1e-9")
    rec.build_tree().assemble().solve()
    for max_words in (1 << 27, 0):
        rec.dual_grid_max_words = max_words
        v, f = rec.extract_mesh()
        out.append((rec.dual_cubes().cpu().numpy(), v.cpu().numpy(), f.cpu().numpy()))
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][2], out[1][2])
    assert np.abs(out[0][1] - out[1][1]).max() <= 1e-5
