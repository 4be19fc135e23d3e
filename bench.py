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

WORKLOAD = dict(workload="superquadrics-300k", n_points=300000, n_shapes=4, seed=0, voxel_size=1.0 / 512,
                depth=4, min_density=2.0, screen_alpha=4.0, solver="pcg-mixed@tol=1e-7")
PLAIN_SOLVER = "plain-fp64@tol=1e-7"
FP64_SOLVER = "pcg-fp64@tol=1e-12"


def workload_points():
    from jspsr import synthetic
    xyz, nrm, _ = synthetic.superquadrics(WORKLOAD["n_points"], k=WORKLOAD["n_shapes"], seed=WORKLOAD["seed"])
    return xyz, nrm


def crop(xyz, nrm, n_keep, seed=1):
    """A bounded sample of the same cloud: the n_keep points nearest (L-inf) to a surface point."""
    c = xyz[np.random.default_rng(seed).integers(len(xyz))]
    d = np.abs(xyz - c).max(1)
    idx = np.argsort(d)[:n_keep]
    return xyz[idx], nrm[idx]


def cpu_reconstruct(xyz, nrm):
    sys.path.insert(0, str(ROOT))
    from oracle import spsr
    return spsr.reconstruct(xyz, nrm, WORKLOAD["voxel_size"], WORKLOAD["depth"], WORKLOAD["min_density"],
                            WORKLOAD["screen_alpha"], cg_tol=1e-7)


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
    if rank != 0:
        return
    xyz, nrm = workload_points()
    n_sample = 4000
    sx, sn = crop(xyz, nrm, n_sample)
    for _ in range(args.warmup):
        cpu_reconstruct(sx, sn)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        cpu_reconstruct(sx, sn)
    dt = time.perf_counter() - t0
    value = (n_sample / WORKLOAD["n_points"]) * args.steps / dt
    sample = (f"{n_sample}-point L-inf crop of the {WORKLOAD['workload']} cloud per step, scaled by "
              f"{n_sample}/{WORKLOAD['n_points']}; FP64 numpy/scipy oracle, Jacobi CG to 1e-7")
    line = {"impl": "reference", "metric": "recon/s", "value": value, "unit": "recon/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(WORKLOAD, sample=sample),
            "cpu_baseline": {"value": value, "unit": "recon/s", "cores": 1, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": "recon/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------- our arm
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-comparators", action="store_true")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

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
    xyz, nrm = workload_points()
    X = torch.from_numpy(xyz).cuda()
    N = torch.from_numpy(nrm).cuda()
    W = WORKLOAD

    def step(solver=W["solver"], profile=False):
        rec = Reconstruction(X, N, W["voxel_size"], W["depth"], W["min_density"], W["screen_alpha"], solver=solver)
        rec.profile_pcg = profile
        v, f = rec.run()
        return rec, v, f

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()

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
    ms = t0.elapsed_time(t1)
    if world > 1:
        tt = torch.tensor([ms], device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms = float(tt.item())
    value = world * args.steps / (ms / 1e3)

    # ---------------------------------------------------------------- end to end through the public API
    xyz_h = torch.from_numpy(xyz).pin_memory()
    nrm_h = torch.from_numpy(nrm).pin_memory()
    jspsr.reconstruct(xyz_h, nrm_h, W["voxel_size"], W["depth"], W["min_density"], W["screen_alpha"], solver=W["solver"])
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    d2h = 0
    e0.record()
    for _ in range(args.steps):
        v, f = jspsr.reconstruct(xyz_h, nrm_h, W["voxel_size"], W["depth"], W["min_density"], W["screen_alpha"],
                                 solver=W["solver"])
        d2h = v.numel() * 4 + f.numel() * 8
    e1.record()
    torch.cuda.synchronize()
    barrier()
    e2e_ms = e0.elapsed_time(e1)
    if world > 1:
        tt = torch.tensor([e2e_ms], device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e_ms = float(tt.item())
    e2e = {"value": world * args.steps / (e2e_ms / 1e3), "unit": "recon/s",
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
    if tf.exists():
        for line in tf.read_text().splitlines():
            if line.startswith("dram_bytes_per_iteration_level0:"):
                traffic = float(line.split(":")[1]) * iters0
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "kernel": "pcg_kernel<MIXED> (level 0)",
                "peak_source": "measured" if pk.exists() else "fallback",
                "bytes_per_launch": alg_bytes, "launch_ms": pcg_ms[0], "iterations": iters0}

    # ---------------------------------------------------------------- comparators: plain FP64 GPU and FP64 field error
    extra = {}
    if not args.no_comparators:
        torch.cuda.synchronize()
        c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        c0.record()
        for _ in range(2):
            step(solver=PLAIN_SOLVER)
        c1.record()
        torch.cuda.synchronize()
        plain_ms = c0.elapsed_time(c1) / 2
        ref64, _, _ = step(solver=FP64_SOLVER)
        chi = rec.chi_raw(X) - rec.mean_chi()
        chi64 = ref64.chi_raw(X) - ref64.mean_chi()
        err = float(torch.linalg.norm(chi.double() - chi64.double()) / torch.linalg.norm(chi64.double()))
        extra = {"plain_fp64_ms_per_step": plain_ms, "speedup_vs_plain_fp64": plain_ms / (ms / args.steps),
                 "field_rel_err_vs_fp64_solve": err,
                 "pcg_ms_per_level": pcg_ms, "pcg_iters_per_level": {d: s["iters"] for d, s in stats.items()},
                 "mesh": {"vertices": int(v.shape[0]), "faces": int(f.shape[0])}}

    # ---------------------------------------------------------------- CPU baseline (oracle on a bounded sample)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        n_sample = 4000
        sx, sn = crop(xyz, nrm, n_sample)
        tc = time.perf_counter()
        cpu_reconstruct(sx, sn)
        dt = time.perf_counter() - tc
        cpu = {"value": (n_sample / W["n_points"]) / dt, "unit": "recon/s", "cores": 1, "kind": "port",
               "sample": f"{n_sample}-point L-inf crop of the same cloud, one reconstruction in {dt:.1f} s, "
                         f"scaled by {n_sample}/{W['n_points']}; FP64 numpy/scipy oracle, Jacobi CG to 1e-7"}

    if rank == 0:
        line = {"metric": "recon/s", "value": value, "unit": "recon/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": dict(W, parallelism=f"replicas x{world}", precision="FP32 SpMV/vectors, FP64 dots + FP64 "
                               "refinement", l2="inputs larger than L2 (level-0 matrix 0.6 GB)"),
                "e2e": e2e, "gpu_launches": int(launches), "roofline": roofline, "cpu_baseline": cpu,
                "clocks": clocks.summary(), **extra}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
