"""The matrix-free level operator against the assembled CSR of the same level.

A = K (*) v + alpha * Phi^T (Phi v) applied without a matrix (the 5x5x5 stencil over the level's rank
bitmap, the screening through the point basis and its per-row transpose) must equal the assembled
CSR product of the same level in FP64 up to summation order (relative 1e-13); its Jacobi diagonal
and its screening right-hand side must equal the CSR path's; and a level solved through the operator
must agree with the same level solved through the CSR, in the mixed and in the FP64 mode, on the
cooperative grid and on a thread-block cluster.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda", 0)
CASES = ["torus_small", "torus_adaptive", "sq_noisy"]


def rel(a, b):
    a = a.double()
    b = b.double()
    return float(torch.linalg.norm(a - b) / max(float(torch.linalg.norm(b)), 1e-300))


@pytest.fixture(scope="module")
def recs(golden):
    from jspsr.core.pipeline import Reconstruction
    out = {}
    for name in CASES:
        g = golden(name)
        vs, depth, md, alpha = g["params"]
        rec = Reconstruction(torch.from_numpy(g["xyz"]).to(DEV), torch.from_numpy(g["nrm"]).to(DEV), vs, int(depth),
                             md, alpha, solver="pcg-mixed@tol=1e-9")
        rec.keep_csr = True
        rec.run()
        rec.check_solves()
        out[name] = rec
    return out


def pairs_of(rec, lv):
    """The transposed point basis of any level through the C ABI (whatever operator the level uses)."""
    from jspsr import _lib as L
    st = L.stream()
    counts = torch.zeros(lv.n, dtype=torch.int32, device=DEV)
    mx = torch.zeros(1, dtype=torch.int32, device=DEV)
    L.call("ngs_mf_count", L.ptr(lv.rows), rec.n, lv.n, L.ptr(counts), L.ptr(mx), st)
    t_ptr = torch.empty(lv.n + 1, dtype=torch.int64, device=DEV)
    L.scan(counts, out=t_ptr[:lv.n], total=t_ptr[lv.n:])
    E = int(t_ptr[lv.n])
    cursor = torch.zeros(lv.n, dtype=torch.int32, device=DEV)
    tmp_p = torch.empty(E, dtype=torch.int32, device=DEV)
    tmp_f = torch.empty(E, dtype=torch.float32, device=DEV)
    t_point = torch.empty(E, dtype=torch.int32, device=DEV)
    t_phi = torch.empty(E, dtype=torch.float32, device=DEV)
    L.call("ngs_mf_fill", L.ptr(lv.rows), L.ptr(lv.phi), rec.n, L.ptr(t_ptr), lv.n, L.ptr(cursor), L.ptr(tmp_p),
           L.ptr(tmp_f), L.ptr(t_point), L.ptr(t_phi), st)
    assert int(mx) == int(counts.max())
    return t_ptr, t_point, t_phi


def operator_of(rec, lv, d, pairs):
    from jspsr import _lib as L
    t_ptr, t_point, t_phi = pairs
    op = L.PcgOperator()
    op.grid = lv.grid
    op.coords, op.stencil, op.alpha, op.n_points = lv.coords.data_ptr(), lv.stencil.data_ptr(), \
        rec._screen_scale(d), rec.n
    op.point_rows, op.point_phi = lv.rows.data_ptr(), lv.phi.data_ptr()
    op.t_ptr, op.t_point, op.t_phi = t_ptr.data_ptr(), t_point.data_ptr(), t_phi.data_ptr()
    s32 = torch.empty(rec.n, dtype=torch.float32, device=DEV)
    s64 = torch.empty(rec.n, dtype=torch.float64, device=DEV)
    op.scratch32, op.scratch64 = s32.data_ptr(), s64.data_ptr()
    return op, (pairs, s32, s64)


@pytest.mark.parametrize("name", CASES)
def test_pairs_are_the_point_basis_transposed(recs, name):
    rec = recs[name]
    for lv in rec.levels:
        t_ptr, t_point, t_phi = pairs_of(rec, lv)
        rows = lv.rows.reshape(-1)
        keep = rows >= 0
        pts = torch.arange(rec.n, device=DEV).repeat_interleave(27)[keep]
        order = torch.argsort(rows[keep].long() * rec.n + pts)        # by row, then point
        exp_point = pts[order].int()
        exp_phi = lv.phi.reshape(-1)[keep][order]
        assert torch.equal(t_point, exp_point) and torch.equal(t_phi, exp_phi)
        assert torch.equal(t_ptr[1:] - t_ptr[:-1], torch.bincount(rows[keep].long(), minlength=lv.n))


@pytest.mark.parametrize("name", CASES)
def test_operator_equals_assembled_matrix(recs, name):
    from jspsr import _lib as L
    rec = recs[name]
    gen = torch.Generator(device="cpu").manual_seed(7)
    for d, lv in enumerate(rec.levels):
        op, keep = operator_of(rec, lv, d, pairs_of(rec, lv))
        x = torch.randn(lv.n, generator=gen, dtype=torch.float64).to(DEV)
        y_mf = torch.empty_like(x)
        y_csr = torch.empty_like(x)
        L.call("ngs_mf_apply64", L.C.byref(op), lv.n, L.ptr(x), L.ptr(y_mf), L.stream())
        L.call("ngs_spmv64", lv.n, L.ptr(lv.rowptr), L.ptr(lv.cols), L.ptr(lv.vals64), L.ptr(x), L.ptr(y_csr),
               L.stream())
        assert rel(y_mf, y_csr) <= 1e-13, (name, d)


@pytest.mark.parametrize("name", CASES)
def test_diagonal_and_screening_rhs_equal_csr_path(recs, name):
    from jspsr import _lib as L
    rec = recs[name]
    st = L.stream()
    for d, lv in enumerate(rec.levels):
        t_ptr, t_point, t_phi = pairs_of(rec, lv)
        inv = torch.empty(lv.n, dtype=torch.float32, device=DEV)
        L.call("ngs_mf_diag", L.ptr(t_ptr), L.ptr(t_phi), lv.n, float(lv.stencil[62]), rec._screen_scale(d),
               L.ptr(inv), st)
        inv_csr = (1.0 / lv.vals64[lv.diag_slot]).float()
        assert rel(inv, inv_csr) <= 1e-7, (name, d)
        cell = torch.empty(rec.n, dtype=torch.int64, device=DEV)
        L.call("ngs_point_cell_keys", L.ptr(lv.rows), rec.n, L.ptr(cell), st)
        keys, order = torch.sort(cell)
        field = torch.rand(rec.n, device=DEV)
        for f in (None, field):
            a = torch.zeros(lv.n, dtype=torch.float64, device=DEV)
            b = torch.zeros_like(a)
            L.call("ngs_mf_screen_rhs", L.ptr(t_ptr), L.ptr(t_point), L.ptr(t_phi), lv.n,
                   L.ptr(f) if f is not None else None, 0.75, L.ptr(a), st)
            L.call("ngs_screen_rhs_grouped", L.ptr(lv.rows), L.ptr(lv.phi), rec.n, None,
                   L.ptr(f) if f is not None else None, L.ptr(order), L.ptr(keys), 0.75, L.ptr(b), st)
            assert rel(a, b) <= 1e-12, (name, d)


def solve_level(rec, lv, d, mode, use_op, blocks=0, tol=1e-12):
    from jspsr import _lib as L
    lib = L.load()
    x32 = torch.empty(lv.n, dtype=torch.float32, device=DEV)
    x64 = torch.empty(lv.n, dtype=torch.float64, device=DEV)
    info = torch.zeros(4, dtype=torch.int64, device=DEV)
    resid = torch.zeros(2, dtype=torch.float64, device=DEV)
    sysd = L.PcgSystem()
    sysd.n = lv.n
    keep = []
    if use_op:
        pairs = pairs_of(rec, lv)
        op, k = operator_of(rec, lv, d, pairs)
        keep += [op, k]
        inv = torch.empty(lv.n, dtype=torch.float32, device=DEV)
        L.call("ngs_mf_diag", L.ptr(pairs[0]), L.ptr(pairs[2]), lv.n, float(lv.stencil[62]), rec._screen_scale(d),
               L.ptr(inv), L.stream())
        keep.append(inv)
        sysd.op = L.C.pointer(op)
        sysd.nnz = 60 * lv.n + 2 * int(pairs[0][lv.n])
        sysd.inv_diag = inv.data_ptr()
    else:
        inv = (1.0 / lv.vals64[lv.diag_slot]).float()
        keep.append(inv)
        sysd.nnz = lv.nnz
        sysd.rowptr, sysd.cols, sysd.inv_diag = lv.rowptr.data_ptr(), lv.cols.data_ptr(), inv.data_ptr()
        sysd.vals32, sysd.vals64 = lv.vals32.data_ptr(), lv.vals64.data_ptr()
    sysd.b64 = lv.rhs.data_ptr()
    sysd.x32, sysd.x64 = x32.data_ptr(), x64.data_ptr()
    cfg = L.PcgConfig()
    cfg.mode, cfg.max_iter, cfg.tol, cfg.res_fix = mode, 5000, tol, 0
    cfg.replace_every, cfg.blocks, cfg.timeout_s = 50, blocks, 10.0
    ws_bytes = lib.ngs_pcg_workspace_bytes(lv.n, mode)
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device=DEV)
    rc = lib.ngs_pcg_solve(L.C.byref(sysd), L.C.byref(cfg), L.ptr(ws), ws_bytes, L.ptr(info), L.ptr(resid),
                           L.stream())
    assert rc == 0, lib.ngs_status_string(rc)
    torch.cuda.synchronize()
    assert int(info[1]) == 0, (int(info[1]), int(info[0]))
    assert float(resid[0]) <= tol * float(resid[1]) * 1.0001
    cluster = lib.ngs_pcg_cluster_size(lv.n, sysd.nnz, mode) if blocks == 0 else 0
    return x64, cluster


@pytest.mark.parametrize("name", CASES)
def test_operator_solves_equal_csr_solves(recs, name):
    """Mixed and FP64 modes; every level once on its default path (a cluster for the small ones),
    once forced onto the cooperative grid (blocks = 2)."""
    from jspsr import _lib as L
    rec = recs[name]
    clusters = 0
    for d, lv in enumerate(rec.levels):
        for mode in (L.PCG_MIXED, L.PCG_FP64):
            x_csr, _ = solve_level(rec, lv, d, mode, use_op=False)
            x_mf, cl = solve_level(rec, lv, d, mode, use_op=True)
            x_grid, _ = solve_level(rec, lv, d, mode, use_op=True, blocks=2)
            clusters += cl > 0
            assert rel(x_mf, x_csr) <= 1e-8, (name, d, mode)
            assert rel(x_grid, x_csr) <= 1e-8, (name, d, mode)
    assert clusters > 0


def test_benchmark_cloud_levels_take_the_operator_where_it_pays():
    """300,000 points on 4 superquadrics at 1/512 (the benchmark cloud) with operator="matrix-free":
    the finest levels' point pairs are far fewer than their stiffness non-zeros, so they are solved
    matrix-free; the coarse ones, where many points share a cell, keep the assembled Gram.  The
    solutions equal the all-CSR reconstruction's."""
    from jspsr import synthetic
    from jspsr.core.pipeline import Reconstruction
    xyz, nrm, _ = synthetic.superquadrics(300000, k=4, seed=0)
    rec = Reconstruction(torch.from_numpy(xyz).to(DEV), torch.from_numpy(nrm).to(DEV), 1.0 / 512, 4, 2.0, 4.0,
                         solver="pcg-mixed@tol=1e-7", operator="matrix-free")
    rec.build_tree().assemble()
    assert rec.levels[0].mf
    for lv in rec.levels:
        assert lv.mf == (2 * lv.n_pairs <= lv.nnz and lv.max_pairs <= 4096)
    csr = Reconstruction(torch.from_numpy(xyz).to(DEV), torch.from_numpy(nrm).to(DEV), 1.0 / 512, 4, 2.0, 4.0,
                         solver="pcg-mixed@tol=1e-7", operator="csr")
    csr.build_tree().assemble()
    assert not any(lv.mf for lv in csr.levels)
    rec.solve()
    csr.solve()
    rec.check_solves()
    csr.check_solves()
    for a, b in zip(rec.levels, csr.levels):
        assert rel(a.x64, b.x64) <= 1e-6
