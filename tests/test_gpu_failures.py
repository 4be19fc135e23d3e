"""Failure paths of the device code, exercised without faulting or hanging the GPU.

Every device-side wait of the persistent PCG is bounded by a time limit, after which the kernel
records NGS_ERR_TIMEOUT and returns; every solve is bounded by an iteration cap.  These tests make
those limits run out on purpose (a 1 microsecond limit, max_iter = 1), check that the status reaches
the caller -- through the C ABI and through ``jspsr.reconstruct`` -- and that the CUDA context is
still usable afterwards.  Host-side failures (a hash table too small for its keys) are injected
through the C ABI's own argument checks.  The reference ignores such failures
(``csrc/common/hashmap_cuda.cu:369``, ``csrc/sparse_solve/solve_pcg.cu:80-128`` has no cap on time).
"""
import ctypes as C
import warnings

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda", 0)


def laplacian(side, shift=0.3):
    """7-point Laplacian plus a positive shift on a side^3 lattice, CSR on the device."""
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
    rowptr = np.concatenate([[0], np.cumsum(np.bincount(r, minlength=n))]).astype(np.int64)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(DEV)   # noqa: E731
    return dict(n=n, nnz=len(v), rowptr=T(rowptr), cols=T(c.astype(np.int32)), vals64=T(v),
                vals32=T(v.astype(np.float32)), inv_diag=T(np.full(n, 1.0 / (6.0 + shift), np.float32)))


def pcg(m, max_iter=2000, timeout_s=10.0, tol=1e-10):
    from jspsr import _lib as L
    lib = L.load()
    b = torch.ones(m["n"], dtype=torch.float64, device=DEV)
    x32 = torch.empty(m["n"], dtype=torch.float32, device=DEV)
    x64 = torch.empty(m["n"], dtype=torch.float64, device=DEV)
    info = torch.full((4,), -1, dtype=torch.int64, device=DEV)
    resid = torch.zeros(2, dtype=torch.float64, device=DEV)
    sysd = L.PcgSystem()
    sysd.n, sysd.nnz = m["n"], m["nnz"]
    sysd.rowptr, sysd.cols, sysd.inv_diag = m["rowptr"].data_ptr(), m["cols"].data_ptr(), m["inv_diag"].data_ptr()
    sysd.vals32, sysd.vals64 = m["vals32"].data_ptr(), m["vals64"].data_ptr()
    sysd.b32, sysd.b64 = None, b.data_ptr()
    sysd.x32, sysd.x64 = x32.data_ptr(), x64.data_ptr()
    cfg = L.PcgConfig()
    cfg.mode, cfg.max_iter, cfg.tol, cfg.res_fix = L.PCG_MIXED, max_iter, tol, 0
    cfg.replace_every, cfg.blocks, cfg.timeout_s = 50, 0, timeout_s
    ws_bytes = lib.ngs_pcg_workspace_bytes(m["n"], L.PCG_MIXED)
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device=DEV)
    rc = lib.ngs_pcg_solve(C.byref(sysd), C.byref(cfg), L.ptr(ws), ws_bytes, L.ptr(info), L.ptr(resid), L.stream())
    assert rc == 0, lib.ngs_status_string(rc)
    torch.cuda.synchronize()
    return int(info[0]), int(info[1])


@pytest.mark.parametrize("side", [40, 50])      # one thread-block cluster / cooperative grid
def test_pcg_timeout_is_reported_and_context_survives(side):
    from jspsr import _lib as L
    m = laplacian(side)
    assert (L.load().ngs_pcg_cluster_size(m["n"], m["nnz"], L.PCG_MIXED) > 0) == (side == 40)
    _, status = pcg(m, timeout_s=1e-6)           # every bounded wait and the solve deadline: 1 us
    assert status == L.NGS_ERR_TIMEOUT
    it, status = pcg(m)                          # the same system again, normal limits
    assert status == L.NGS_OK and it > 0


@pytest.mark.parametrize("side", [40, 50])
def test_pcg_iteration_cap_is_reported(side):
    from jspsr import _lib as L
    it, status = pcg(laplacian(side), max_iter=1)
    assert (it, status) == (1, L.NGS_ERR_NOT_CONVERGED)


def _torus():
    from jspsr import synthetic
    xyz, nrm = synthetic.torus(n=3000, seed=0)
    return torch.from_numpy(xyz).to(DEV), torch.from_numpy(nrm).to(DEV)


def test_reconstruct_raises_on_solver_timeout():
    import jspsr
    from jspsr import _lib as L
    x, n = _torus()
    with pytest.raises(L.NgsError, match="timed out"):
        jspsr.reconstruct(x, n, 1.0 / 64, 3, 0.5, 4.0, solver="pcg-mixed@tol=1e-7@timeout=1e-6")
    v, f = jspsr.reconstruct(x, n, 1.0 / 64, 3, 0.5, 4.0)         # the context is still usable
    assert f.shape[0] > 0


def test_reconstruct_warns_at_requested_maxiter():
    import jspsr
    x, n = _torus()
    with warnings.catch_warnings(record=True) as w:
        warnings.simplefilter("always")
        v, f = jspsr.reconstruct(x, n, 1.0 / 64, 3, 0.5, 4.0, solver="pcg-mixed@tol=1e-7@maxiter=1")
    assert any("stopped at maxiter=1" in str(x.message) for x in w)


def test_hash_table_too_small_is_refused():
    from jspsr import _lib as L
    lib = L.load()
    keys = torch.arange(100, dtype=torch.int64, device=DEV)
    slots = torch.empty(16, dtype=torch.int64, device=DEV)             # 8 slots of 16 bytes
    status = torch.zeros(1, dtype=torch.int32, device=DEV)
    t = L.HashTable()
    t.slots, t.nslots = slots.data_ptr(), 8
    rc = lib.ngs_hash_table_build(C.byref(t), L.ptr(keys), None, 100, L.ptr(status), L.stream())
    assert rc == L.NGS_ERR_OOM
    assert int(status.item()) == 0                                     # nothing was launched
