"""Serving path on the GPU: the batched PCG launch against solo solves (bit for bit), and each
request's result alone against the same request in a concurrent mix."""
import sys
from pathlib import Path

import numpy as np
import pytest
import torch

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT / "neural-galerkin_b200"))

pytestmark = pytest.mark.gpu


def _requests(k, seed=0, n_range=(2000, 60000)):
    from jspsr import synthetic
    from jspsr.serving import Request
    rng = np.random.default_rng(seed)
    out = []
    for i in range(k):
        req = dict(n=int(np.exp(rng.uniform(np.log(n_range[0]), np.log(n_range[1])))), seed=1000 + i)
        x, n = synthetic.serving_request_device(req, "cuda")
        vs = 2.0 ** -int(rng.integers(6, 9))
        out.append(Request(x.cpu().pin_memory(), n.cpu().pin_memory(), vs, depth=4, rid=i))
    return out


def test_batched_pcg_is_bit_identical_to_solo_solves():
    from jspsr import _lib as L
    from jspsr.core.pipeline import Reconstruction
    lib = L.load()
    recs, items, solo = [], [], []
    for req in _requests(6, seed=1, n_range=(1500, 20000)):
        rec = Reconstruction(req.xyz.cuda(), req.normal.cuda(), req.voxel_size, 4, None, 4.0)
        rec.build_tree().assemble()
        d = rec.depth - 1
        lv = rec.levels[d]
        rec._rhs(d)
        item = rec.pcg_item(lv)
        L.call("ngs_pcg_solve", L.C.byref(item.sys), L.C.byref(item.cfg), item.ws, item.ws_bytes, item.info_dev,
               item.resid_dev, L.stream())
        solo.append((lv.x64.clone(), lv.info.clone()))
        lv.x64.zero_()
        lv.info.zero_()
        recs.append(rec)
        items.append(item)
    cap = lib.ngs_pcg_block_capacity(items[0].cfg.mode)
    # the largest prefix-greedy subset whose blocks fit one cooperative launch
    keep, used = [], 0
    for k, it in enumerate(items):
        b = lib.ngs_pcg_blocks(it.sys.n, it.sys.nnz, it.cfg.mode)
        if used + b <= cap:
            keep.append(k)
            used += b
    assert len(keep) >= 2, "need at least two systems in the batch"
    recs = [recs[k] for k in keep]
    solo = [solo[k] for k in keep]
    items = [items[k] for k in keep]
    arr = (L.PcgBatchItem * len(items))(*items)
    assert lib.ngs_pcg_solve_batch(arr, len(items), L.stream()) == 0
    torch.cuda.synchronize()
    for rec, (x, info) in zip(recs, solo):
        lv = rec.levels[rec.depth - 1]
        assert int(info[1]) == 0 and int(lv.info[1]) == 0
        assert torch.equal(lv.info[:3], info[:3])
        assert torch.equal(lv.x64, x)


def test_batched_pcg_rejects_oversubscription():
    """A batch whose blocks exceed one cooperative launch is refused before anything runs."""
    from jspsr import _lib as L
    from jspsr.core.pipeline import Reconstruction
    lib = L.load()
    cap = lib.ngs_pcg_block_capacity(L.PCG_MIXED)
    assert cap >= 148
    req = _requests(1, seed=3, n_range=(60000, 60001))[0]
    rec = Reconstruction(req.xyz.cuda(), req.normal.cuda(), 1 / 512, 4, None, 4.0)
    rec.build_tree().assemble()
    for d in range(rec.depth - 1, 0, -1):
        rec._rhs(d)
        rec._solve_level(rec.levels[d], d)
    rec._rhs(0)
    item = rec.pcg_item(rec.levels[0])
    b = lib.ngs_pcg_blocks(item.sys.n, item.sys.nnz, item.cfg.mode)
    if b == 0:
        pytest.skip("system solved by a thread-block cluster, outside the cooperative launch")
    copies = cap // b + 1
    if copies > L.PCG_BATCH_MAX:
        pytest.skip("system too small to oversubscribe within the batch limit")
    arr = (L.PcgBatchItem * copies)(*([item] * copies))
    info0 = rec.levels[0].info.clone()
    assert lib.ngs_pcg_solve_batch(arr, copies, L.stream()) == L.NGS_ERR_INVALID_ARG
    torch.cuda.synchronize()
    assert torch.equal(rec.levels[0].info, info0)          # nothing was launched or cleared


def test_serving_results_equal_alone_and_mixed():
    from jspsr.serving import ReconServer, run_sequential
    reqs = _requests(8, seed=2)
    alone = run_sequential(reqs, keep_solutions=True)
    srv = ReconServer(slots=4, keep_solutions=True)
    try:
        mixed = srv.run(reqs, realtime=False)
        launches, systems = srv.batcher.launches, srv.batcher.batched_systems
        direct_solves = srv.batcher.direct_solves
    finally:
        srv.close()
    assert all(r.error is None for r in mixed), [r.error for r in mixed]
    assert systems + direct_solves == 8 * 4 and launches <= max(systems, 1)
    for a, m in zip(alone, mixed):
        for xa, xm in zip(a.solutions, m.solutions):
            assert float(torch.linalg.norm(xa - xm) / torch.linalg.norm(xa)) <= 1e-6
        fa, fm = a.faces.numpy(), m.faces.numpy()
        if fa.shape == fm.shape and np.array_equal(fa, fm):
            assert np.abs(a.vertices.numpy() - m.vertices.numpy()).max() <= 1e-5
        else:
            assert abs(fa.shape[0] - fm.shape[0]) <= max(2, 0.001 * fa.shape[0])


def test_cluster_and_cooperative_solves_agree():
    """A small system solved by one thread-block cluster (the default at its size) and by the
    cooperative grid kernel (forced with a block count) reach the same solution."""
    from jspsr import _lib as L
    from jspsr.core.pipeline import Reconstruction
    lib = L.load()
    req = _requests(1, seed=4, n_range=(8000, 8001))[0]
    rec = Reconstruction(req.xyz.cuda(), req.normal.cuda(), 1 / 128, 4, None, 4.0)
    rec.build_tree().assemble()
    d = rec.depth - 1
    rec._rhs(d)
    lv = rec.levels[d]
    item = rec.pcg_item(lv)
    assert lib.ngs_pcg_cluster_size(item.sys.n, item.sys.nnz, item.cfg.mode) > 0
    item.cfg.tol = 1e-12
    out = []
    for blocks in (0, 24):
        item.cfg.blocks = blocks
        L.call("ngs_pcg_solve", L.C.byref(item.sys), L.C.byref(item.cfg), item.ws, item.ws_bytes, item.info_dev,
               item.resid_dev, L.stream())
        torch.cuda.synchronize()
        assert int(lv.info[1]) == 0, lv.info
        out.append(lv.x64.clone())
    assert float(torch.linalg.norm(out[0] - out[1]) / torch.linalg.norm(out[1])) < 1e-9
