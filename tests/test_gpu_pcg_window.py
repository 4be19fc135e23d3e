"""The PCG's shared-memory vector window and its two SpMV forms, through the C ABI.

A system whose ``band`` (bound on |column - row|) lets every block's column range fit stages the
search vector in shared memory; with ``band = 0`` the launch reserves none and the gathers read
global memory.  The window changes only where the same values are read, so the two solutions are
bit-identical.  With the window the solver reads the 2-byte column deltas, if given, in the
software-pipelined SpMV (four entries per round); without it, the 4-byte columns in the
row-at-a-time one (eight per round) -- given deltas are then ignored, which this also checks bit for
bit.  The two forms' products round differently, and both converge to the same solution within the
solve tolerance.  Systems: 7-point Laplacians plus a shift (sorted columns within every row), one
solved by a thread-block cluster and one by a cooperative grid.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from test_zz_no_alloc import laplacian_system

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda", 0)
SOLVE_TOL = 1e-10       # relative residual every solve reaches


def solve(m, b64, band, deltas):
    from jspsr import _lib as L
    lib = L.load()
    x32 = torch.empty(m["n"], dtype=torch.float32, device=DEV)
    x64 = torch.empty(m["n"], dtype=torch.float64, device=DEV)
    info = torch.zeros(4, dtype=torch.int64, device=DEV)
    resid = torch.zeros(2, dtype=torch.float64, device=DEV)
    sysd = L.PcgSystem()
    sysd.n, sysd.nnz = m["n"], m["nnz"]
    sysd.rowptr, sysd.cols, sysd.inv_diag = m["rowptr"].data_ptr(), m["cols"].data_ptr(), m["inv_diag"].data_ptr()
    sysd.vals32, sysd.vals64 = m["vals32"].data_ptr(), m["vals64"].data_ptr()
    sysd.b32, sysd.b64 = None, b64.data_ptr()
    sysd.x32, sysd.x64 = x32.data_ptr(), x64.data_ptr()
    sysd.band = band
    delta = None
    if deltas:
        delta = torch.empty(m["nnz"], dtype=torch.int16, device=DEV)
        assert lib.ngs_csr_col_delta(L.ptr(m["rowptr"]), L.ptr(m["cols"]), m["n"], L.ptr(delta), L.stream()) == 0
        sysd.col_delta = delta.data_ptr()
    cfg = L.PcgConfig()
    cfg.mode, cfg.max_iter, cfg.tol, cfg.res_fix = L.PCG_MIXED, 2000, SOLVE_TOL, 0
    cfg.replace_every, cfg.blocks, cfg.timeout_s = 50, 0, 10.0
    ws_bytes = lib.ngs_pcg_workspace_bytes(m["n"], L.PCG_MIXED)
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device=DEV)
    rc = lib.ngs_pcg_solve(C.byref(sysd), C.byref(cfg), L.ptr(ws), ws_bytes, L.ptr(info), L.ptr(resid), L.stream())
    assert rc == 0, lib.ngs_status_string(rc)
    torch.cuda.synchronize()
    assert int(info[1]) == 0, f"solve status {int(info[1])}"
    return x64.clone(), int(info[0])


@pytest.mark.parametrize("side", [40, 60])
def test_window_changes_no_bit_and_both_spmv_forms_converge(side):
    from jspsr import _lib as L
    lib = L.load()
    m = laplacian_system(side, 0.05, DEV)
    # side 40: one cluster; side 60 (216,000 rows): a cooperative grid
    assert (lib.ngs_pcg_cluster_size(m["n"], m["nnz"], L.PCG_MIXED) > 0) == (side == 40)
    gen = torch.Generator(device="cpu").manual_seed(side)
    b = torch.randn(m["n"], generator=gen, dtype=torch.float64).to(DEV)
    band = side * side                      # the +-x neighbours are the farthest columns
    assert lib.ngs_pcg_window(m["n"], m["nnz"], band, L.PCG_MIXED) == 1
    assert lib.ngs_pcg_window(m["n"], m["nnz"], 0, L.PCG_MIXED) == 0
    x_glob, it_glob = solve(m, b, 0, False)
    x_win, it_win = solve(m, b, band, False)
    assert it_glob == it_win
    assert torch.equal(x_glob, x_win), "the window must not change a bit"
    x_glob_d, _ = solve(m, b, 0, True)      # no window: the deltas are not read
    assert torch.equal(x_glob, x_glob_d)
    x_win_d, _ = solve(m, b, band, True)    # window: the deltas, the pipelined form
    rel = float(torch.linalg.norm(x_win - x_win_d) / torch.linalg.norm(x_win))
    # both solutions are within the solve tolerance of the exact one; the Laplacian's condition
    # number at these sizes (< 1e3 with the shift) bounds their distance well below 1e-6
    assert rel < 1e-6, rel
