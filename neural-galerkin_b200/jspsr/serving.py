"""Continuous-batching reconstruction server on one GPU.

Requests (oriented point clouds in host memory, each with its own voxel size) arrive over time.
The server admits a request when a slot is free and its estimated HBM footprint fits the budget,
and runs it on its own CUDA stream through the device-resident pipeline (tree, assembly, solve,
dual marching cubes, mesh copied back to pinned host memory).  Requests in flight overlap on the
device.  Their per-level PCG solves do not run as separate launches: a batcher collects the solves
that are ready, from every stream, and issues them as one cooperative launch
(``ngs_pcg_solve_batch``), each system keeping the block count of its solo solve, so that its
result is bit-identical to solving it alone.  Systems small enough for one thread-block cluster
skip the batcher: their cluster solve runs on the worker's own stream, concurrently with the rest.

Nothing here changes what a reconstruction computes: a request's mesh is the one
``jspsr.reconstruct`` returns for the same input, up to the order of floating-point atomics in
the assembly.
"""
from __future__ import annotations

import math
import queue
import threading
import time
from dataclasses import dataclass, field
from typing import Callable, List, Optional

import numpy as np

from . import _lib as L


@dataclass
class Request:
    xyz: "torch.Tensor"            # (N, 3) float32, host (pinned for asynchronous upload)
    normal: "torch.Tensor"
    voxel_size: float
    depth: int = 4
    min_density: Optional[float] = None     # None: the median point density of the request
    screen_alpha: float = 4.0
    arrival: float = 0.0           # seconds after the start of the stream
    rid: int = 0


@dataclass
class Result:
    rid: int
    vertices: Optional["torch.Tensor"] = None     # host
    faces: Optional["torch.Tensor"] = None
    arrival: float = 0.0
    admitted: float = 0.0
    done: float = 0.0
    error: Optional[str] = None
    solutions: Optional[list] = None              # per-level FP64 solutions (kept on request)
    n_vertices: int = 0
    n_faces: int = 0

    @property
    def latency(self) -> float:
        return self.done - self.arrival


def footprint_bytes(n_points: int, voxel_size: float, depth: int = 4) -> int:
    """Estimated peak device memory of one reconstruction.

    Per point: inputs, density / level / weight and the 27-entry basis rows of every level
    (about 0.25 KB per level).  Per voxel: the CSR row of up to 125 entries in FP64 + FP32 + int32
    (2 KB), solve vectors and mesh buffers.  The voxel count of a level is bounded by the points'
    trilinear corners (8 per point) and by the surface the cloud can span at that voxel size.
    """
    per_point = 96 + 256 * depth
    surf = 6.0 / (voxel_size * voxel_size)          # cells of a unit-cube-sized surface at the finest level
    voxels = min(6.0 * n_points, 3.0 * surf) * 1.4  # coarser levels add well under half of the finest
    return int(64 << 20) + int(per_point * n_points + 2000 * voxels)


class PinnedStage:
    """A worker's reusable pinned download buffers (grown by powers of two): allocating page-locked
    memory per mesh would cost more than the copy itself."""

    def __init__(self):
        self.bufs = {}

    def get(self, key, nbytes):
        import torch
        b = self.bufs.get(key)
        if b is None or b.numel() < nbytes:
            b = torch.empty(1 << max(20, (int(nbytes) - 1).bit_length()), dtype=torch.uint8, pin_memory=True)
            self.bufs[key] = b
        return b

    def download(self, v, f, keep: bool):
        """Enqueue the mesh's device-to-host copy on the current stream; returns host views (valid
        until the next download) or, with ``keep``, owned copies made after the caller's sync."""
        vb = self.get("v", v.numel() * v.element_size())[:v.numel() * v.element_size()].view(v.dtype).view(v.shape)
        fb = self.get("f", f.numel() * f.element_size())[:f.numel() * f.element_size()].view(f.dtype).view(f.shape)
        vb.copy_(v, non_blocking=True)
        fb.copy_(f, non_blocking=True)
        return vb, fb


class Admission:
    """Slots and an HBM budget shared by the requests in flight (first come, first admitted)."""

    def __init__(self, slots: int, budget_bytes: int):
        self.slots = slots
        self.budget = int(budget_bytes)
        self.busy = 0
        self.in_use = 0
        self.peak_in_use = 0
        self.waits = 0
        self.cv = threading.Condition()

    def acquire(self, need: int, timeout: float = None) -> int:
        """Block until a slot is free and ``need`` bytes fit; returns the bytes charged (a request
        larger than the whole budget is charged the budget and so runs alone)."""
        need = min(int(need), self.budget)
        t_end = None if timeout is None else time.perf_counter() + timeout
        with self.cv:
            waited = False
            while self.busy >= self.slots or self.in_use + need > self.budget:
                waited = True
                if t_end is not None and time.perf_counter() >= t_end:
                    raise TimeoutError("admission")
                self.cv.wait(0.01)
            self.waits += int(waited)
            self.busy += 1
            self.in_use += need
            self.peak_in_use = max(self.peak_in_use, self.in_use)
        return need

    def release(self, charged: int) -> None:
        with self.cv:
            self.busy -= 1
            self.in_use -= charged
            self.cv.notify_all()


class SolveBatcher:
    """Collects PCG solves from the worker streams and launches them together."""

    def __init__(self, device, window_s: float = 0.0015, busy: Callable[[], int] = None):
        import torch
        self.dev = device
        # highest priority: the blocks of a cooperative launch are scheduled ahead of the workers' kernels
        lo, hi = torch.cuda.Stream.priority_range()
        self.stream = torch.cuda.Stream(device, priority=min(lo, hi))
        self.window_s = window_s
        self.busy = busy or (lambda: 1)
        self.cv = threading.Condition()
        self.pending: list = []
        self.stop = False
        self.launches = 0
        self.batched_systems = 0
        self.direct_solves = 0
        self.inflight = None
        self.lib = L.load()
        self.thread = threading.Thread(target=self._loop, name="ngs-solve-batcher", daemon=True)
        self.thread.start()

    # called from a worker thread, on the worker's current stream
    def submit(self, rec, lv, d, item):
        import torch
        if self.lib.ngs_pcg_cluster_size(item.sys.n, item.sys.nnz, item.cfg.mode) > 0:
            # small system: one thread-block cluster solves it on the worker's own stream, next to
            # everything else in flight -- nothing to batch, nothing to wait for
            L.call("ngs_pcg_solve", L.C.byref(item.sys), L.C.byref(item.cfg), item.ws, item.ws_bytes, item.info_dev,
                   item.resid_dev, L.stream())
            self.direct_solves += 1
            return
        ready = torch.cuda.Event()
        ready.record()
        t = dict(item=item, ready=ready, done=None, rc=None, ev=threading.Event(),
                 blocks=self.lib.ngs_pcg_blocks(item.sys.n, item.sys.nnz, item.cfg.mode), mode=item.cfg.mode,
                 t=time.perf_counter())
        with self.cv:
            self.pending.append(t)
            self.cv.notify_all()
        if not t["ev"].wait(timeout=120.0):
            raise RuntimeError("solve batcher did not take the solve within 120 s")
        if t["rc"] != L.NGS_OK:
            raise L.NgsError(t["rc"], f"batched PCG, level {d}")
        torch.cuda.current_stream().wait_event(t["done"])

    def close(self):
        with self.cv:
            self.stop = True
            self.cv.notify_all()
        self.thread.join(timeout=30)

    def _take(self):
        """Continuous batching of solves: while a batched launch is on the GPU, the solves that
        become ready wait for it; when it finishes (or none is in flight), everything pending that
        fits one cooperative launch goes together.  No fixed window: a lone solve on an idle GPU
        launches at once."""
        with self.cv:
            while not self.pending and not self.stop:
                self.cv.wait(0.05)
            if self.stop and not self.pending:
                return None
        if self.inflight is not None:
            self.inflight.synchronize()          # the previous batch: let solves gather meanwhile
            self.inflight = None
        with self.cv:
            cap = self.lib.ngs_pcg_block_capacity(self.pending[0]["mode"])
            batch, used, rest = [], 0, []
            for t in self.pending:
                if t["mode"] == self.pending[0]["mode"] and len(batch) < L.PCG_BATCH_MAX and used + t["blocks"] <= cap:
                    batch.append(t)
                    used += t["blocks"]
                else:
                    rest.append(t)
            if not batch:                      # a single system larger than the capacity: alone
                batch, rest = [self.pending[0]], self.pending[1:]
            self.pending = rest
            return batch

    def _loop(self):
        import torch
        torch.cuda.set_device(self.dev)
        with torch.cuda.stream(self.stream):
            while True:
                batch = self._take()
                if batch is None:
                    return
                for t in batch:
                    self.stream.wait_event(t["ready"])
                arr = (L.PcgBatchItem * len(batch))(*[t["item"] for t in batch])
                rc = self.lib.ngs_pcg_solve_batch(arr, len(batch), L.stream())
                done = torch.cuda.Event()
                done.record(self.stream)
                self.inflight = done
                self.launches += 1
                self.batched_systems += len(batch)
                for t in batch:
                    t["rc"], t["done"] = rc, done
                    t["ev"].set()


class ReconServer:
    """Admission + worker slots + batched solves.  ``run`` replays a stream of requests."""

    def __init__(self, slots: int = 8, hbm_budget_bytes: Optional[int] = None, solver: str = "pcg-mixed@tol=1e-7",
                 window_s: float = 0.0015, device: int = 0, keep_solutions: bool = False, keep_meshes: bool = True,
                 footprint: Callable[[Request], int] = None):
        import sys
        import torch
        # the workers hand the interpreter to one another between their (GIL-free) launches and
        # waits; a short switch interval keeps a thread that has work from waiting 5 ms for its turn
        sys.setswitchinterval(min(sys.getswitchinterval(), 2e-4))
        self.slots = slots
        self.solver = solver
        self.dev = torch.device("cuda", device)
        if hbm_budget_bytes is None:
            free, _ = torch.cuda.mem_get_info(self.dev)
            hbm_budget_bytes = int(0.6 * free)
        self.budget = int(hbm_budget_bytes)
        self.keep_solutions = keep_solutions
        self.keep_meshes = keep_meshes
        self.footprint = footprint or (lambda r: footprint_bytes(r.xyz.shape[0], r.voxel_size, r.depth))
        self.adm = Admission(slots, self.budget)
        self.cv = threading.Condition()
        self.batcher = SolveBatcher(self.dev, window_s=window_s, busy=lambda: self.adm.busy)
        self.work: "queue.Queue" = queue.Queue()
        self.results: dict = {}
        self.workers = [threading.Thread(target=self._worker, args=(i,), name=f"ngs-worker-{i}", daemon=True)
                        for i in range(slots)]
        for w in self.workers:
            w.start()

    # ------------------------------------------------------------------ admission
    def admit(self, req: Request, t0: float, arrival: float) -> None:
        """Block until a slot is free and the request's footprint fits, then hand it to a worker."""
        need = self.adm.acquire(self.footprint(req))
        self.work.put((req, need, t0, arrival, time.perf_counter() - t0))

    # ------------------------------------------------------------------ worker
    def _worker(self, i):
        import torch
        from .core.pipeline import Reconstruction
        torch.cuda.set_device(self.dev)
        stream = torch.cuda.Stream(self.dev)
        stage = PinnedStage()
        with torch.cuda.stream(stream):
            while True:
                job = self.work.get()
                if job is None:
                    return
                req, need, t0, arrival, t_adm = job
                res = Result(rid=req.rid, arrival=arrival, admitted=t_adm)
                try:
                    x = req.xyz.to(self.dev, non_blocking=True)
                    n = req.normal.to(self.dev, non_blocking=True)
                    rec = Reconstruction(x, n, req.voxel_size, req.depth, req.min_density, req.screen_alpha,
                                         solver=self.solver)
                    rec.solve_hook = self.batcher.submit
                    v, f = rec.run()
                    vh, fh = stage.download(v, f, self.keep_meshes)
                    if self.keep_solutions:
                        res.solutions = [lv.x64.clone() for lv in rec.levels]
                    stream.synchronize()
                    res.n_vertices, res.n_faces = int(v.shape[0]), int(f.shape[0])
                    if self.keep_meshes:
                        res.vertices, res.faces = vh.clone(), fh.clone()
                    del rec, v, f, x, n
                except Exception as e:       # reported per request; the server keeps running
                    res.error = f"{type(e).__name__}: {e}"
                    stream.synchronize()
                res.done = time.perf_counter() - t0
                with self.cv:
                    self.results[req.rid] = res
                    self.cv.notify_all()
                self.adm.release(need)

    # ------------------------------------------------------------------ streams
    def run(self, requests: List[Request], realtime: bool = True) -> List[Result]:
        """Replay the requests at their arrival times (``realtime``) or all at once; returns results
        in request order once every request is done."""
        self.results = {}
        t0 = time.perf_counter()
        for req in sorted(requests, key=lambda r: r.arrival):
            if realtime:
                wait = req.arrival - (time.perf_counter() - t0)
                if wait > 0:
                    time.sleep(wait)
            self.admit(req, t0, req.arrival if realtime else 0.0)
        with self.cv:
            while len(self.results) < len(requests):
                self.cv.wait(0.05)
        return [self.results[r.rid] for r in requests]

    def close(self):
        for _ in self.workers:
            self.work.put(None)
        for w in self.workers:
            w.join(timeout=60)
        self.batcher.close()


def latency_stats(results: List[Result]) -> dict:
    lat = np.array([r.latency for r in results if r.error is None]) * 1e3
    if lat.size == 0:
        return {"p50_ms": math.nan, "p99_ms": math.nan, "mean_ms": math.nan}
    return {"p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "mean_ms": float(lat.mean()), "max_ms": float(lat.max())}


def run_sequential(requests: List[Request], solver: str = "pcg-mixed@tol=1e-7", keep_solutions: bool = False,
                   keep_meshes: bool = True, device: int = 0) -> List[Result]:
    """One request at a time through the plain path (``Reconstruction`` on the current stream, its own
    PCG launches), with the same upload and pinned download as the server; ``latency`` is the
    request's service time."""
    import torch
    from .core.pipeline import Reconstruction
    dev = torch.device("cuda", device)
    out = []
    stage = PinnedStage()
    t0 = time.perf_counter()
    for req in requests:
        torch.cuda.current_stream().synchronize()
        t_start = time.perf_counter() - t0
        res = Result(rid=req.rid, arrival=t_start, admitted=t_start)
        x = req.xyz.to(dev, non_blocking=True)
        n = req.normal.to(dev, non_blocking=True)
        rec = Reconstruction(x, n, req.voxel_size, req.depth, req.min_density, req.screen_alpha, solver=solver)
        v, f = rec.run()
        vh, fh = stage.download(v, f, keep_meshes)
        if keep_solutions:
            res.solutions = [lv.x64.clone() for lv in rec.levels]
        torch.cuda.current_stream().synchronize()
        res.n_vertices, res.n_faces = int(v.shape[0]), int(f.shape[0])
        if keep_meshes:
            res.vertices, res.faces = vh.clone(), fh.clone()
        res.done = time.perf_counter() - t0
        out.append(res)
    return out
