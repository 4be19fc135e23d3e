#!/usr/bin/env python
"""Reconstructions per second of the B200 screened-Poisson path.

Workload (one step = one full reconstruction, tree -> splat -> Galerkin solve ->
dual marching cubes): 300,000 points on a union of 4 random superquadrics in the
unit cube (exponents U[0.3,2], scales U[0.1,0.3], random rotations), normals
perturbed by N(0,0.02), positions by N(0,0.002); finest voxel 1/512, 4 levels,
min_density 2.0 (the reference default of 32 leaves the fine levels empty on
this cloud), screening weight 4.0; per-level FP32 PCG with FP64 dots and FP64
refinement to 1e-7 relative true residual.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun (N > 1) every rank runs independent replicas of the workload (the
path does not shard; there is no collective on the data path) and the job value
is the sum over ranks of reconstructions divided by the slowest rank's time.
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import os
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "neural-galerkin_b200"))

WORKLOADS = {
    # the headline workload (one step = one reconstruction)
    "superquadrics-300k": dict(workload="superquadrics-300k", n_points=300000, n_shapes=4, seed=0,
                               voxel_size=1.0 / 512, depth=4, min_density=2.0, screen_alpha=4.0,
                               solver="pcg-mixed@tol=1e-7"),
    # the same kind of cloud at a third of the size (profiling captures)
    "superquadrics-100k": dict(workload="superquadrics-100k", n_points=100000, n_shapes=4, seed=0,
                               voxel_size=1.0 / 512, depth=4, min_density=0.7, screen_alpha=4.0,
                               solver="pcg-mixed@tol=1e-7"),
    # 10k points on a torus, 3 levels at 1/128
    "torus-10k": dict(workload="torus-10k", n_points=10000, n_shapes=0, seed=0, voxel_size=1.0 / 128, depth=3,
                      min_density=1.5, screen_alpha=4.0, solver="pcg-mixed@tol=1e-7"),
    # 5M points in an 8 x 8 x 3 m room, 1 cm voxels, 11 levels
    "room-5m": dict(workload="room-5m", n_points=5_000_000, n_shapes=40, seed=0, voxel_size=0.01, depth=11,
                    min_density=2.0, screen_alpha=4.0, solver="pcg-mixed@tol=1e-7"),
}
WORKLOAD = dict(WORKLOADS["superquadrics-300k"])
PLAIN_SOLVER = "plain-fp64@tol=1e-7"
FP64_SOLVER = "pcg-fp64@tol=1e-7"          # the FP64 persistent kernel at the same tolerance (like for like)
EXACT_SOLVER = "pcg-fp64@tol=1e-12"        # the error reference: every level solved to 1e-12 in FP64



def workload_points():
    from jspsr import synthetic
    W = WORKLOAD
    if W["workload"].startswith("torus"):
        return synthetic.torus(n=W["n_points"], seed=W["seed"])
    if W["workload"].startswith("room"):
        return synthetic.room(n=W["n_points"], seed=W["seed"], n_objects=W["n_shapes"])
    xyz, nrm, _ = synthetic.superquadrics(W["n_points"], k=W["n_shapes"], seed=W["seed"])
    return xyz, nrm


def crop(xyz, nrm, n_keep, seed=1):
    """A bounded sample of the same cloud: the n_keep points nearest (L-inf) to a surface point."""
    c = xyz[np.random.default_rng(seed).integers(len(xyz))]
    d = np.abs(xyz - c).max(1)
    idx = np.argsort(d)[:n_keep]
    return xyz[idx], nrm[idx]


def cpu_reconstruct(xyz, nrm, threads=None):
    """The reference's path on the host's cores: the C/OpenMP FP64 oracle (structure decisions in
    FP32 as the reference's torch code, FP64 numerics, Jacobi CG to the same 1e-7 relative residual
    as the GPU solve), one full reconstruction including the mesh."""
    sys.path.insert(0, str(ROOT))
    from oracle import fast
    return fast.reconstruct(xyz, nrm, WORKLOAD["voxel_size"], WORKLOAD["depth"], WORKLOAD["min_density"],
                            WORKLOAD["screen_alpha"], cg_tol=1e-7, levels=False, threads=threads)


def cpu_cores():
    return len(os.sched_getaffinity(0))


def cpu_sample_text(threads):
    return (f"the full {WORKLOAD['workload']} workload per step (same cloud and parameters as the GPU arm), "
            f"C/OpenMP FP64 restatement of the reference path on {threads} host threads; every stage "
            f"multi-threaded (scatter sums by atomics, CG by parallel SpMV and reductions)")


# ----------------------------------------------------------------------------- replicas
def slowest_rank_ms(ms: float, world: int, device: str) -> float:
    """The timed region's duration on the slowest rank (every rank calls this, in the same order)."""
    if world <= 1:
        return ms
    import torch
    import torch.distributed as dist
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(ms: float, world: int, steps: int) -> float:
    """Reconstructions per second of the whole job: every rank ran ``steps`` independent replicas."""
    return world * steps / (ms / 1e3)


# ----------------------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None

    def __enter__(self):
        self.tmp = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.tmp,
                                         stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            self.proc.wait(timeout=10)

    def summary(self):
        if self.proc is None:
            return None
        rows = [r.split(",") for r in Path(self.tmp.name).read_text().strip().splitlines() if r.count(",") >= 8]
        os.unlink(self.tmp.name)
        if not rows:
            return None
        sm = np.array([float(r[1]) for r in rows])
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.strip() == "Active"})
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(rows[0][2]), "reasons": reasons,
                "samples": len(rows)}


# ----------------------------------------------------------------------------- reference arm
def run_reference(args, rank):
    """The reference's CPU path on the GPU box's host cores, on this arm's config and metric: one
    step = one full reconstruction of the same cloud.  Warm-up steps reconstruct a 30,000-point crop
    of the cloud (a CPU path has no device state to warm; this only faults in the code and the
    allocator), so that the timed steps dominate the run."""
    if rank != 0:
        return
    xyz, nrm = workload_points()
    threads = cpu_cores()
    wx, wn = crop(xyz, nrm, min(30000, len(xyz)))
    for _ in range(args.warmup):
        cpu_reconstruct(wx, wn, threads)
    stages = np.zeros(7)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        r = cpu_reconstruct(xyz, nrm, threads)
        stages += r["seconds"]
    dt = time.perf_counter() - t0
    value = args.steps / dt
    sample = cpu_sample_text(threads)
    line = {"impl": "reference", "metric": "recon/s", "value": value, "unit": "recon/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(WORKLOAD, warmup_sample="30,000-point L-inf crop of the same cloud"),
            "same_config": True,
            "cpu_baseline": {"value": value, "unit": "recon/s", "cores": threads, "kind": "port", "sample": sample},
            "stage_s_per_step": dict(zip(["tree", "assembly_solve", "mesh", "mesh_dual_centres", "mesh_dual_cubes",
                                          "mesh_field", "mesh_mc"], (stages / args.steps).round(4).tolist())),
            "e2e": {"value": value, "unit": "recon/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------- learned-basis leg
def learned_leg(n_shapes=32):
    """Neural Galerkin forward + adjoint on a batch of ``n_shapes`` random superquadrics (3,000
    points, voxel 1/128, 3 levels, AdditiveHermite basis with 18 features per voxel ~ init + N(0,
    0.1), loss = MSE of chi at 20,000 queries against the analytic target): the whole batch goes
    through one Galerkin solve function (every level's solves of all shapes in one batched launch,
    forward and adjoint); device time of the batch, median of three passes."""
    import torch
    from jspsr import synthetic
    from jspsr.core.learned import LearnedBatch, LearnedStep

    def make(seeds):
        steps = []
        for seed in seeds:
            xyz, nrm, q, tgt = synthetic.learned_problem(seed=seed)
            T = lambda a: torch.from_numpy(a).cuda()     # noqa: E731
            steps.append(LearnedStep(T(xyz), T(nrm), T(q), T(tgt), min_density=None).build())
        return LearnedBatch(steps)

    def run(batch):
        feats = [st.init_features(0.1, seed=k) for k, st in enumerate(batch.steps)]
        normals = [st.normal.clone().requires_grad_(True) for st in batch.steps]
        fl = [{d: v.clone().requires_grad_(True) for d, v in f.items()} for f in feats]
        torch.cuda.synchronize()
        e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        e[0].record()
        total, losses, _ = batch.forward(normals, fl)
        e[1].record()
        total.backward()
        e[2].record()
        torch.cuda.synchronize()
        return e[0].elapsed_time(e[1]), e[1].elapsed_time(e[2]), [float(x) for x in losses]

    warm = make(range(1000, 1002))
    run(warm)                                    # table uploads, allocator, kernels
    batch = make(range(n_shapes))
    batch.geometry()                             # positions only: built once per shape set
    # three passes over the batch, the median reported: the forward is host-bound Python and its
    # first pass over a new batch also grows the allocator's pools
    runs = [run(batch) for _ in range(3)]
    fw = float(np.median([r[0] for r in runs]))
    bw = float(np.median([r[1] for r in runs]))
    losses = runs[-1][2]
    voxels = [sum(st.tree.get_coords_size(st.tree.DECODER, d) for d in range(st.depth)) for st in batch.steps]
    return {"shapes": n_shapes, "batch_forward_ms": fw, "batch_adjoint_ms": bw,
            "batch_ms_passes": [[r[0], r[1]] for r in runs],
            "forward_ms_per_shape": fw / n_shapes, "adjoint_ms_per_shape": bw / n_shapes,
            "shapes_per_s": 1e3 * n_shapes / (fw + bw), "mean_voxels": float(np.mean(voxels)),
            "mean_loss": float(np.mean(losses)),
            "config": "3,000 points + N(0,0.005) on a random superquadric, voxel 1/128, 3 levels, "
                      "AdditiveHermite(6, SinPeaks(1..3)) 18 features/voxel, 20,000 queries, FP64 PCG to 1e-12 "
                      "forward and adjoint (cholmod-equivalent); gradients w.r.t. normals and features; "
                      "32 shapes in one batched Galerkin solve"}


# ----------------------------------------------------------------------------- sparse convolution leg
def conv_leg(cin=64, cout=64, reps=10):
    """One 3^3 sparse convolution layer (the Neural Galerkin U-Net's building block) on the finest voxel
    level of the benchmark cloud: forward, input gradient and weight gradient in bf16 with FP32
    accumulation on the tensor cores, device time per pass (mean of ``reps`` after warm-up), against
    the reference's algorithm in torch (per offset: gather, GEMM, scatter-add) on the same data."""
    import torch
    from jspsr import ext
    from jspsr.core._hash_backend import VoxelLevel
    from jspsr.core.pipeline import Reconstruction
    xyz, nrm = workload_points()
    W = WORKLOAD
    rec = Reconstruction(torch.from_numpy(xyz).cuda(), torch.from_numpy(nrm).cuda(), W["voxel_size"], W["depth"],
                         W["min_density"], W["screen_alpha"], solver=W["solver"])
    rec.build_tree()
    coords = rec.levels[0].coords
    lv = VoxelLevel(coords, 1)
    ax = torch.arange(-1, 2)
    offs = torch.cartesian_prod(ax, ax, ax).to(torch.int32).cuda()
    src, tgt, kidx, counts = lv.neighbours(coords, 1, offs, True, False)
    nbmaps = torch.stack([tgt, src], 1).int().contiguous()     # (input row, output row) per offset
    nbsizes = counts.int().cpu()
    n = coords.shape[0]
    pairs = int(nbsizes.sum())
    gen = torch.Generator(device="cpu").manual_seed(0)
    x = torch.randn(n, cin, generator=gen).cuda().bfloat16()
    w = (torch.randn(27, cin, cout, generator=gen) / cin ** 0.5).cuda().bfloat16()
    gy = torch.randn(n, cout, generator=gen).cuda().bfloat16()
    out = torch.zeros(n, cout, dtype=torch.bfloat16, device="cuda")
    gx = torch.zeros_like(x)
    gw = torch.zeros_like(w)

    def timed(fn):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        e = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        e[0].record()
        for _ in range(reps):
            fn()
        e[1].record()
        torch.cuda.synchronize()
        return e[0].elapsed_time(e[1]) / reps

    fwd = timed(lambda: ext.sparse_op.convolution_forward_cuda(x, out, w, nbmaps, nbsizes, False, False))
    bwd = timed(lambda: ext.sparse_op.convolution_backward_cuda(x, gx, gy, w, gw, nbmaps, nbsizes, False))
    # the input-gradient kernel alone (the rest of the backward pass is the weight gradient)
    starts_dev, _ = ext._offset_starts(nbsizes, 27, x.device)
    table_in = ext._conv_table(nbmaps, starts_dev, 27, 0, n, -1)
    dgrad = timed(lambda: ext._gather_gemm(gy, table_in, w, cin, gx))
    starts = np.concatenate([[0], np.cumsum(nbsizes.numpy())])

    def reference_forward():
        res = x[:, :0].new_zeros(n, cout)
        for k in range(27):
            a, b = int(starts[k]), int(starts[k + 1])
            res.index_add_(0, nbmaps[a:b, 1].long(), torch.mm(x[nbmaps[a:b, 0].long()], w[k]))
        return res
    ref_fwd = timed(reference_forward)
    flops = 2.0 * pairs * cin * cout
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    peak = peaks.get("bf16_tflops", 1590.0)
    return {"voxels": n, "pairs": pairs, "cin": cin, "cout": cout, "dtype": "bf16 in, fp32 accumulate",
            "forward_ms": fwd, "backward_ms": bwd, "input_grad_kernel_ms": dgrad,
            "weight_grad_ms": bwd - dgrad, "forward_tflops": flops / fwd / 1e9,
            "backward_tflops": 2 * flops / bwd / 1e9, "peak_bf16_tflops": peak,
            "forward_frac_of_peak": flops / fwd / 1e9 / peak,
            "reference_algorithm_torch_forward_ms": ref_fwd, "forward_speedup_vs_reference_algorithm": ref_fwd / fwd,
            "config": "3^3 kernel over the finest voxel level of the benchmark cloud, the U-Net's 64 -> 64 layer"}


# ----------------------------------------------------------------------------- serving leg
def serving_leg(n_requests=1024, slots=8, plain_every=8):
    """1,024 requests (points log-uniform in [1e3, 5e5], superquadric/torus unions, N(0,0.003) noise,
    finest voxel 2^-U{6..9}, 4 levels), Poisson arrivals at 200/s; host payloads in pinned memory,
    meshes back to pinned memory.  Compares the continuous-batching server against one request at
    a time (latency = service time alone)."""
    import torch
    from jspsr import synthetic
    from jspsr.serving import Request, ReconServer, run_sequential, latency_stats
    descs = synthetic.serving_stream(n_requests=n_requests)
    reqs = []
    for i, dsc in enumerate(descs):
        x, n = synthetic.serving_request_device(dsc, "cuda")
        reqs.append(Request(x.cpu().pin_memory(), n.cpu().pin_memory(), 2.0 ** -dsc["finest_depth"], depth=4,
                            arrival=dsc["arrival"], rid=i))
    torch.cuda.synchronize()
    run_sequential(reqs[:8], keep_meshes=False)                 # warm-up
    seq = run_sequential(reqs, keep_meshes=False)
    seq_s = seq[-1].done - seq[0].arrival
    sub = reqs[::plain_every]
    seq_plain = run_sequential(sub, solver="plain-fp64@tol=1e-7", keep_meshes=False)
    t_plain = sum(r.latency for r in seq_plain)
    t_mixed_sub = sum(seq[i].latency for i in range(0, n_requests, plain_every))
    plain_rps = n_requests / (seq_s * t_plain / t_mixed_sub)
    srv = ReconServer(slots=slots, keep_meshes=False)
    try:
        srv.run(reqs[:32], realtime=False)                      # warm-up (streams, allocator pools)
        l0, s0 = srv.batcher.launches, srv.batcher.batched_systems
        rt = srv.run(reqs, realtime=True)
        rt_s = max(r.done for r in rt) - min(r.arrival for r in rt)
        l1, s1 = srv.batcher.launches, srv.batcher.batched_systems
        sat = srv.run(reqs, realtime=False)
        sat_s = max(r.done for r in sat)
        # the same stream at a sustainable rate: arrivals slowed to half the saturated throughput
        half = 0.5 * (n_requests / sat_s)
        slow = [dataclasses.replace(r, arrival=r.arrival * 200.0 / half) for r in reqs[:max(64, n_requests // 4)]]
        low = srv.run(slow, realtime=True)
        waits, peak = srv.adm.waits, srv.adm.peak_in_use
        direct = srv.batcher.direct_solves
    finally:
        srv.close()
    errors = sum(r.error is not None for r in rt + sat + low)
    low_stats = latency_stats(low)
    seq_rps = n_requests / seq_s
    rt_stats, alone = latency_stats(rt), latency_stats(seq)
    return {"requests": n_requests, "slots": slots, "errors": errors,
            "offered_rate_rps": 200.0,
            "served_recon_per_s_at_offered_rate": n_requests / rt_s,
            "p50_ms": rt_stats["p50_ms"], "p99_ms": rt_stats["p99_ms"],
            "saturated_recon_per_s": n_requests / sat_s,
            "saturated": latency_stats(sat),
            "sequential_recon_per_s": seq_rps, "sequential_alone_latency": alone,
            "sequential_plain_fp64_recon_per_s": plain_rps,
            "plain_fp64_sample": f"every {plain_every}th request ({len(sub)}), scaled by the mixed-solver time of the same requests",
            "speedup_vs_sequential": (n_requests / sat_s) / seq_rps,
            "speedup_vs_sequential_plain_fp64": (n_requests / sat_s) / plain_rps,
            "p99_over_alone_p99": rt_stats["p99_ms"] / alone["p99_ms"],
            "at_half_saturated_rate": {"offered_rate_rps": half, "requests": len(low), **low_stats,
                                       "p99_over_alone_p99": low_stats["p99_ms"] / alone["p99_ms"]},
            "cluster_solves_on_worker_streams": direct,
            "pcg_launches_per_system": (l1 - l0) / max(1, s1 - s0),
            "admission_waits": waits, "peak_admitted_bytes": int(peak),
            "total_points": int(sum(r.xyz.shape[0] for r in reqs))}


# ----------------------------------------------------------------------------- our arm
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-comparators", action="store_true")
    ap.add_argument("--workload", default="superquadrics-300k", choices=sorted(WORKLOADS))
    ap.add_argument("--mode", default="all", choices=["all", "recon", "learned", "serving", "conv", "profile"],
                    help="all: reconstruction line with the learned-basis and serving legs attached; profile: "
                         "warm-up reconstructions, then one between cudaProfilerStart/Stop (for ncu "
                         "--profile-from-start off)")
    ap.add_argument("--serving-requests", type=int, default=1024)
    ap.add_argument("--learned-shapes", type=int, default=32)
    ap.add_argument("--serving-slots", type=int, default=8)
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    WORKLOAD.clear()
    WORKLOAD.update(WORKLOADS[args.workload])

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank)

    import torch
    import torch.distributed as dist
    from datetime import timedelta
    import jspsr
    from jspsr import _lib as L
    from jspsr.core.pipeline import Reconstruction

    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    lib = L.load()
    if args.mode in ("learned", "serving", "conv"):
        leg = learned_leg(args.learned_shapes) if args.mode == "learned" else \
            conv_leg() if args.mode == "conv" else serving_leg(args.serving_requests, slots=args.serving_slots)
        if rank == 0:
            print(json.dumps({"mode": args.mode, **leg}), flush=True)
        if world > 1:
            dist.destroy_process_group()
        return
    xyz, nrm = workload_points()
    X = torch.from_numpy(xyz).cuda()
    N = torch.from_numpy(nrm).cuda()
    W = WORKLOAD

    def step(solver=W["solver"], profile=False, operator="csr"):
        rec = Reconstruction(X, N, W["voxel_size"], W["depth"], W["min_density"], W["screen_alpha"], solver=solver,
                             operator=operator)
        rec.profile_pcg = profile
        v, f = rec.run()
        return rec, v, f

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if args.mode == "profile":
        torch.cuda.profiler.start()
        step()
        torch.cuda.synchronize()
        torch.cuda.profiler.stop()
        if rank == 0:
            print(json.dumps({"mode": "profile", "workload": W["workload"], "profiled_steps": 1}), flush=True)
        if world > 1:
            dist.destroy_process_group()
        return

    def barrier():
        if world > 1:
            dist.barrier()

    # ---------------------------------------------------------------- device-resident throughput
    with ClockSampler(local) as clocks:
        barrier()
        torch.cuda.synchronize()
        l0 = lib.ngs_launch_count()
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record()
        for _ in range(args.steps):
            step()
        t1.record()
        torch.cuda.synchronize()
        barrier()
    launches = lib.ngs_launch_count() - l0
    ms = slowest_rank_ms(t0.elapsed_time(t1), world, "cuda")
    value = job_throughput(ms, world, args.steps)

    # ---------------------------------------------------------------- end to end through the public API
    xyz_h = torch.from_numpy(xyz).pin_memory()
    nrm_h = torch.from_numpy(nrm).pin_memory()
    for _ in range(2):        # warm-up: the pinned host buffers of the mesh come from torch's host cache
        v, f = jspsr.reconstruct(xyz_h, nrm_h, W["voxel_size"], W["depth"], W["min_density"], W["screen_alpha"],
                                 solver=W["solver"])
        v = f = None
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    d2h = 0
    e0.record()
    for _ in range(args.steps):
        v, f = jspsr.reconstruct(xyz_h, nrm_h, W["voxel_size"], W["depth"], W["min_density"], W["screen_alpha"],
                                 solver=W["solver"])
        d2h = v.numel() * 4 + f.numel() * 8
        v = f = None          # the caller has consumed the mesh (host buffers go back to the cache)
    e1.record()
    torch.cuda.synchronize()
    barrier()
    e2e_ms = slowest_rank_ms(e0.elapsed_time(e1), world, "cuda")
    e2e = {"value": job_throughput(e2e_ms, world, args.steps), "unit": "recon/s",
           "h2d_bytes_per_step": int(xyz.nbytes + nrm.nbytes), "d2h_bytes_per_step": int(d2h)}

    # ---------------------------------------------------------------- roofline of the dominant kernel (level-0 PCG)
    rec, v, f = step(profile=True)
    stats = rec.check_solves()
    lv0 = rec.levels[0]
    pcg_ms = {d: rec.pcg_ms[d] for d in rec.pcg_ms}
    iters0 = stats[0]["iters"]
    # algorithmic bytes per PCG iteration: 8 B per non-zero (FP32 value + int32 column) + 48 B per row
    alg_bytes = iters0 * (8 * lv0.nnz + 48 * lv0.n)
    achieved = alg_bytes / (pcg_ms[0] / 1e3) / 1e9
    peaks = {}
    pk = ROOT / "MEASURED_PEAKS.json"
    if pk.exists():
        peaks = json.loads(pk.read_text())
    peak = peaks.get("hbm_gbs", 6650.0)
    traffic = None
    tf = ROOT / "profiles" / "pcg_mixed_superquadrics300k_traffic.txt"
    if tf.exists() and W["workload"] == "superquadrics-300k":    # the capture is of this workload
        for line in tf.read_text().splitlines():
            if line.startswith("dram_bytes_per_iteration_level0:"):
                traffic = float(line.split(":")[1]) * iters0
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "kernel": "pcg_form_kernel<MIXED> (level 0)",
                "peak_source": "measured" if pk.exists() else "fallback",
                "bytes_per_launch": alg_bytes, "launch_ms": pcg_ms[0], "iterations": iters0}

    # ---------------------------------------------------------------- comparators: plain FP64 GPU and FP64 field error
    extra = {}
    if not args.no_comparators:
        step(solver=PLAIN_SOLVER)        # warm-up: the comparator's kernels load on first use
        torch.cuda.synchronize()
        plain_steps = []
        for _ in range(5):               # host-driven: its time also depends on the host's speed, so
            c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            c0.record()                  # each step is timed alone and the median is reported
            step(solver=PLAIN_SOLVER)
            c1.record()
            torch.cuda.synchronize()
            plain_steps.append(c0.elapsed_time(c1))
        plain_ms = float(np.median(plain_steps))
        plain_rec, _, _ = step(solver=PLAIN_SOLVER, profile=True)
        plain_solve = plain_rec.pcg_ms
        plain_iters = {d: int(lv.info[0]) for d, lv in enumerate(plain_rec.levels)}
        plain_rec = None                 # each comparator's hierarchy is released once read (large scenes)
        step(solver=FP64_SOLVER)         # warm-up of the FP64 kernel, as above
        fp64_rec, _, _ = step(solver=FP64_SOLVER, profile=True)
        fp64_solve = fp64_rec.pcg_ms
        fp64_iters = {d: int(lv.info[0]) for d, lv in enumerate(fp64_rec.levels)}
        fp64_rec = None
        torch.cuda.empty_cache()
        # the matrix-free operator (stencil over the bitmap + point form of the screening) on the
        # levels where it applies, same solver
        step(operator="matrix-free")
        mf_rec, _, _ = step(profile=True, operator="matrix-free")
        mf_solve = mf_rec.pcg_ms
        mf_levels = [d for d, lv in enumerate(mf_rec.levels) if lv.mf]
        mf_rec = None
        torch.cuda.empty_cache()
        # errors against every level solved to 1e-12 in FP64 on the GPU: field at the input points,
        # solutions, and mesh vertices matched by their primal-sample pair
        ref64, v64, f64 = step(solver=EXACT_SOLVER)
        chi = rec.chi_raw(X) - rec.mean_chi()
        chi64 = ref64.chi_raw(X) - ref64.mean_chi()
        err = float(torch.linalg.norm(chi.double() - chi64.double()) / torch.linalg.norm(chi64.double()))
        xerr = max(float(torch.linalg.norm(a.x64 - b.x64) / torch.linalg.norm(b.x64))
                   for a, b in zip(rec.levels, ref64.levels))

        def keyed(r, vv, ff):
            k = torch.empty(vv.shape[0], dtype=torch.int64, device=vv.device)
            vids = r.mesh_vids.long()
            k[ff.reshape(-1)] = (vids[:, 0] << 32) | vids[:, 1]
            return k.cpu().numpy(), vv.cpu().numpy().astype(np.float64)
        ka, va = keyed(rec, v, f)
        kb, vb = keyed(ref64, v64, f64)
        common, ia, ib = np.intersect1d(ka, kb, assume_unique=True, return_indices=True)
        verr = float(np.linalg.norm(va[ia] - vb[ib]) / np.linalg.norm(vb[ib]))
        flips = int(torch.count_nonzero((rec.mesh_info["values"] < 0) != (ref64.mesh_info["values"] < 0)))
        mixed_solve = sum(pcg_ms.values())
        extra = {"plain_fp64_ms_per_step": plain_ms, "plain_fp64_ms_steps": plain_steps,
                 "speedup_vs_plain_fp64": plain_ms / (ms / args.steps),
                 "solve_ms": {"mixed": mixed_solve, "plain_fp64_host_driven": sum(plain_solve.values()),
                              "fp64_persistent_same_tol": sum(fp64_solve.values()),
                              "mixed_matrix_free_operator": sum(mf_solve.values())},
                 "matrix_free_levels": mf_levels,
                 "matrix_free_pcg_ms_per_level": mf_solve,
                 "solve_speedup_vs_plain_fp64": sum(plain_solve.values()) / mixed_solve,
                 "solve_speedup_vs_fp64_persistent": sum(fp64_solve.values()) / mixed_solve,
                 "error_vs_fp64_exact": {"reference": EXACT_SOLVER, "field": err, "solution": xerr, "vertices": verr,
                                         "vertices_compared": int(common.size),
                                         "vertices_unmatched": int(va.shape[0] + vb.shape[0] - 2 * common.size),
                                         "sample_sign_flips": flips},
                 "pcg_ms_per_level": pcg_ms, "pcg_iters_per_level": {d: s["iters"] for d, s in stats.items()},
                 "plain_fp64_iters_per_level": plain_iters,
                 "fp64_same_tol_iters_per_level": fp64_iters,
                 "mesh": {"vertices": int(v.shape[0]), "faces": int(f.shape[0])}}

    # ---------------------------------------------------------------- learned-basis and serving legs
    if args.mode == "all" and rank == 0 and world == 1:
        extra["learned"] = learned_leg(args.learned_shapes)
        extra["sparse_conv"] = conv_leg()
        extra["serving"] = serving_leg(args.serving_requests, slots=args.serving_slots)

    # ---------------------------------------------------------------- CPU baseline (the reference path on the host)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = cpu_cores()
        tc = time.perf_counter()
        cpu_reconstruct(xyz, nrm, threads)
        dt = time.perf_counter() - tc
        cpu = {"value": 1.0 / dt, "unit": "recon/s", "cores": threads, "kind": "port",
               "sample": cpu_sample_text(threads) + f"; one reconstruction, {dt:.2f} s"}

    mat_bytes = 8 * lv0.nnz + 8 * (lv0.n + 1)
    l2_note = (f"inputs larger than L2 (level-0 matrix {mat_bytes / 1e9:.2f} GB, L2 126 MB)" if mat_bytes > 126e6 else
               f"level-0 matrix {mat_bytes / 1e6:.0f} MB fits L2; steps run back to back without a flush")
    if rank == 0:
        line = {"metric": "recon/s", "value": value, "unit": "recon/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": dict(W, parallelism=f"replicas x{world}", precision="FP32 SpMV/vectors, FP64 dots + FP64 "
                               "refinement", l2=l2_note),
                "e2e": e2e, "gpu_launches": int(launches), "roofline": roofline, "cpu_baseline": cpu,
                "clocks": clocks.summary(), **extra}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
