"""The allocation-free solve entry point against the regular one.

``ngs_pcg_solve_noalloc`` serves callers that cannot allocate device memory when they
solve (host callbacks, contexts where cudaMalloc is not allowed, embedders that only
hand over their own buffers): its scratch is a static device array inside the library.
This file runs last (it is named so that pytest collects it after every other test
file) and checks, through the C ABI, that two calls in a row give the same solution as
``ngs_pcg_solve`` with a caller-provided workspace, and that oversized systems are
refused before any launch.
"""
import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
TOL = 1e-12      # both paths run the same deterministic kernel: equal up to rounding-free identity


def laplacian_system(side, shift, dev):
    """7-point Laplacian plus a positive shift on a side^3 lattice: an SPD CSR system."""
    n = side ** 3
    idx = np.arange(n).reshape(side, side, side)
    rows, cols, vals = [idx.ravel()], [idx.ravel()], [np.full(n, 6.0 + shift)]
    for ax in range(3):
        for d in (-1, 1):
            src = np.take(idx, range(max(0, -d), side - max(0, d)), axis=ax)
            dst = np.take(idx, range(max(0, d), side - max(0, -d)), axis=ax)
            rows.append(src.ravel())
            cols.append(dst.ravel())
            vals.append(np.full(src.size, -1.0))
    r, c, v = np.concatenate(rows), np.concatenate(cols), np.concatenate(vals)
    order = np.lexsort((c, r))
    r, c, v = r[order], c[order], v[order]
    rowptr = np.zeros(n + 1, np.int64)
    np.add.at(rowptr, r + 1, 1)
    rowptr = np.cumsum(rowptr)
    diag = np.full(n, 6.0 + shift)
    return dict(n=n, nnz=len(v), rowptr=torch.from_numpy(rowptr).to(dev),
                cols=torch.from_numpy(c.astype(np.int32)).to(dev),
                vals64=torch.from_numpy(v).to(dev), vals32=torch.from_numpy(v.astype(np.float32)).to(dev),
                inv_diag=torch.from_numpy((1.0 / diag).astype(np.float32)).to(dev))


def solve(lib, L, m, b64, noalloc):
    dev = b64.device
    x32 = torch.empty(m["n"], dtype=torch.float32, device=dev)
    x64 = torch.empty(m["n"], dtype=torch.float64, device=dev)
    info = torch.zeros(4, dtype=torch.int64, device=dev)
    resid = torch.zeros(2, dtype=torch.float64, device=dev)
    sysd = L.PcgSystem()
    sysd.n, sysd.nnz = m["n"], m["nnz"]
    sysd.rowptr, sysd.cols, sysd.inv_diag = m["rowptr"].data_ptr(), m["cols"].data_ptr(), m["inv_diag"].data_ptr()
    sysd.vals32, sysd.vals64 = m["vals32"].data_ptr(), m["vals64"].data_ptr()
    sysd.b32, sysd.b64 = None, b64.data_ptr()
    sysd.x32, sysd.x64 = x32.data_ptr(), x64.data_ptr()
    cfg = L.PcgConfig()
    cfg.mode, cfg.max_iter, cfg.tol, cfg.res_fix = L.PCG_MIXED, 2000, 1e-10, 0
    cfg.replace_every, cfg.blocks, cfg.timeout_s = 50, 0, 10.0
    stream = L.stream()
    if noalloc:
        rc = lib.ngs_pcg_solve_noalloc(C.byref(sysd), C.byref(cfg), L.ptr(info), L.ptr(resid), stream)
        keep = None
    else:
        ws_bytes = lib.ngs_pcg_workspace_bytes(m["n"], L.PCG_MIXED)
        keep = torch.empty(ws_bytes, dtype=torch.uint8, device=dev)
        rc = lib.ngs_pcg_solve(C.byref(sysd), C.byref(cfg), L.ptr(keep), ws_bytes, L.ptr(info), L.ptr(resid),
                               stream)
    assert rc == 0, lib.ngs_status_string(rc)
    torch.cuda.synchronize()
    assert int(info[1]) == 0, f"solve status {int(info[1])}"
    return x64.cpu().numpy(), int(info[0])


@pytest.mark.parametrize("side", [40, 50])
def test_noalloc_matches_workspace_solve_twice(side):
    """side 40 (64,000 rows) is solved by one thread-block cluster, whose reductions live in
    distributed shared memory; side 50 (125,000 rows) needs more blocks than a cluster holds and takes
    the cooperative grid path, whose per-block partials, arrival counter, error word and deadline
    live in the shared static scratch -- the second call runs on what the first one left there."""
    from jspsr import _lib as L
    lib = L.load()
    dev = torch.device("cuda", 0)
    m = laplacian_system(side, 0.3, dev)
    assert m["n"] <= lib.ngs_pcg_noalloc_max_rows()
    cluster = lib.ngs_pcg_cluster_size(m["n"], m["nnz"], L.PCG_MIXED)
    assert (cluster > 0) == (side == 40), cluster
    gen = torch.Generator(device="cpu").manual_seed(side)
    for call in range(2):                                  # the second call runs on the first one's leftovers
        b = torch.randn(m["n"], generator=gen, dtype=torch.float64).to(dev)
        x_ref, it_ref = solve(lib, L, m, b, noalloc=False)
        x_new, it_new = solve(lib, L, m, b, noalloc=True)
        assert it_new == it_ref
        assert np.linalg.norm(x_new - x_ref) <= TOL * np.linalg.norm(x_ref), call


def test_noalloc_rejects_oversized_system():
    from jspsr import _lib as L
    lib = L.load()
    sysd = L.PcgSystem()
    sysd.n = lib.ngs_pcg_noalloc_max_rows() + 1
    cfg = L.PcgConfig()
    cfg.mode = L.PCG_MIXED
    rc = lib.ngs_pcg_solve_noalloc(C.byref(sysd), C.byref(cfg), None, None, L.stream())
    assert rc == 2                                         # NGS_ERR_OOM: larger than the built-in scratch
    sysd.n = -1
    rc = lib.ngs_pcg_solve_noalloc(C.byref(sysd), C.byref(cfg), None, None, L.stream())
    assert rc == 1                                         # NGS_ERR_INVALID_ARG, as ngs_pcg_solve
