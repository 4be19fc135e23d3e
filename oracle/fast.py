"""Python wrapper of the C / OpenMP restatement of the reconstruction path (``oracle/spsr_omp.c``).

TEST INFRASTRUCTURE ONLY.  Only ``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` /
``--impl reference`` legs of ``bench.py`` may use it, as the checker or as the timed CPU baseline;
the product (``neural-galerkin_b200/jspsr``) never imports it.

``oracle/spsr.py`` is the readable numpy restatement, pinned by the reference's own golden runs;
this is the same algorithm stage for stage on all of the host's cores, so that full-size clouds
finish in seconds (``tests/test_oracle_fast.py`` checks the two against each other).  The 1-D
integral tables come from ``oracle/tables.py`` and the triangle table from ``oracle/mc_tables.py``.

    python oracle/fast.py          # build oracle/_build/libspsr_omp.so
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
SRC = HERE / "spsr_omp.c"
LIB = HERE / "_build" / "libspsr_omp.so"
KINDS = ("SHIFTED_SELF_INTEGRAL", "SHIFTED_DERIVATIVE_INTEGRAL", "DERIVATIVE_PARTIAL_INTEGRAL", "PARTIAL_INTEGRAL",
         "INV_DERIVATIVE_PARTIAL_INTEGRAL", "INV_PARTIAL_INTEGRAL")


def build(force: bool = False) -> Path:
    """Compile the restatement with gcc (-O3, OpenMP, IEEE arithmetic: no fast-math, no FMA contraction)."""
    if not force and LIB.exists() and LIB.stat().st_mtime >= SRC.stat().st_mtime:
        return LIB
    LIB.parent.mkdir(exist_ok=True)
    tmp = LIB.with_suffix(".so.tmp")
    cmd = ["gcc", "-O3", "-fopenmp", "-fPIC", "-shared", "-ffp-contract=off", "-std=gnu11", str(SRC), "-o", str(tmp),
           "-lm"]
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


_lib = None


def load():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        lib = C.CDLL(str(LIB))
        vp, i64, f64 = C.c_void_p, C.c_int64, C.c_double
        lib.spsr_reconstruct.argtypes = [vp, vp, i64, f64, C.c_int, f64, f64, f64, f64, C.c_int, C.c_int, vp, vp,
                                         C.c_int, vp, C.c_int, C.c_int]
        lib.spsr_reconstruct.restype = vp
        lib.spsr_free.argtypes = [vp]
        lib.spsr_sizes.argtypes = [vp, vp]
        lib.spsr_points.argtypes = [vp, vp, vp]
        lib.spsr_level.argtypes = [vp, C.c_int, vp, vp, vp, vp, vp, vp, vp]
        lib.spsr_mesh.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, vp]
        _lib = lib
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def default_threads() -> int:
    return len(os.sched_getaffinity(0))


def reconstruct(xyz, normal, voxel_size, depth=4, min_density=32.0, screen_alpha=4.0, screen_delta=0.1,
                cg_tol=1e-12, cg_maxiter=100000, n_upsample=2, mesh=True, threads=None, levels=True):
    """Full reconstruction on the host's cores; returns a dict of numpy arrays.

    Keys: ``density``, ``levels`` (per point); per level d: ``coords{d}``, ``rhs{d}``, ``x{d}``,
    ``rowptr{d}``, ``cols{d}``, ``vals{d}``, ``iters{d}``, ``normals{d}`` (when ``levels``); mesh:
    ``vertices``, ``faces``, ``dual_values`` (field minus mean chi at the primal samples),
    ``dual_pos``, ``cubes`` (complete dual cubes), ``vertex_keys`` (larger << 32 | smaller primal-sample
    id of each vertex's edge), ``mean_chi``; ``seconds`` (tree, solve, mesh; mesh parts: dual centres,
    dual-cube accumulation, field, marching cubes).
    """
    from . import tables as T
    from .mc_tables import TRI_TABLE
    lib = load()
    xyz = np.ascontiguousarray(xyz, dtype=np.float32)
    nrm = np.ascontiguousarray(normal, dtype=np.float32)
    tabs = T.bezier_tables(max(depth, 1))
    flat, lens = [], []
    for k in KINDS:
        for m in range(depth):
            arrs = tabs[k]
            a = np.asarray(arrs[m] if m < len(arrs) else np.zeros(1), dtype=np.float64)
            flat.append(a)
            lens.append(a.size)
    flat = np.ascontiguousarray(np.concatenate(flat))
    lens = np.asarray(lens, dtype=np.int64)
    tri = np.ascontiguousarray(np.asarray(TRI_TABLE, dtype=np.int32).reshape(256, 16))
    nthr = threads or default_threads()
    t0 = time.perf_counter()
    ctx = lib.spsr_reconstruct(_p(xyz), _p(nrm), xyz.shape[0], float(voxel_size), int(depth), float(min_density),
                               float(screen_alpha), float(screen_delta), float(cg_tol), int(cg_maxiter),
                               int(n_upsample), _p(flat), _p(lens), int(depth), _p(tri), int(nthr), int(mesh))
    wall = time.perf_counter() - t0
    if not ctx:
        raise ValueError("empty hierarchy level (lower min_density) or invalid arguments")
    try:
        sizes = np.zeros(8 + 4 * depth, dtype=np.int64)
        lib.spsr_sizes(ctx, _p(sizes))
        out = {"wall_s": wall, "threads": nthr}
        n = xyz.shape[0]
        out["density"] = np.empty(n, np.float64)
        out["levels"] = np.empty(n, np.int32)
        lib.spsr_points(ctx, _p(out["density"]), _p(out["levels"]))
        for d in range(depth):
            V, nnz, it, has_n = (int(v) for v in sizes[8 + 4 * d:12 + 4 * d])
            out[f"iters{d}"] = it
            out[f"coords{d}"] = np.empty((V, 3), np.int32)
            out[f"x{d}"] = np.empty(V, np.float64)
            if levels:
                out[f"rhs{d}"] = np.empty(V, np.float64)
                out[f"rowptr{d}"] = np.empty(V + 1, np.int64)
                out[f"cols{d}"] = np.empty(nnz, np.int64)
                out[f"vals{d}"] = np.empty(nnz, np.float64)
                if has_n:
                    out[f"normals{d}"] = np.empty((V, 3), np.float64)
            g = lambda k: _p(out[k]) if k in out else None          # noqa: E731
            lib.spsr_level(ctx, d, g(f"coords{d}"), g(f"rhs{d}"), g(f"x{d}"), g(f"rowptr{d}"), g(f"cols{d}"),
                           g(f"vals{d}"), g(f"normals{d}"))
        secs = np.zeros(7, np.float64)
        mc = np.zeros(1, np.float64)
        if mesh:
            n_primal, n_dual, n_cubes, nv, nf = (int(v) for v in sizes[:5])
            out["vertices"] = np.empty((nv, 3), np.float64)
            out["faces"] = np.empty((nf, 3), np.int64)
            out["dual_values"] = np.empty(n_primal, np.float64)
            out["dual_pos"] = np.empty((n_primal, 3), np.float64)
            out["cubes"] = np.empty((n_cubes, 8), np.int32)
            out["vertex_keys"] = np.empty(nv, np.int64)
            out["n_dual"] = n_dual
            lib.spsr_mesh(ctx, _p(out["vertices"]), _p(out["faces"]), _p(out["dual_values"]), _p(out["dual_pos"]),
                          _p(out["cubes"]), _p(mc), _p(secs), _p(out["vertex_keys"]))
        else:
            lib.spsr_mesh(ctx, None, None, None, None, None, _p(mc), _p(secs), None)
        out["mean_chi"] = float(mc[0])
        out["seconds"] = secs
        return out
    finally:
        lib.spsr_free(ctx)


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
