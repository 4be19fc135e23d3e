"""Build libngs.so (sm_100a) in-tree: nvcc compiles csrc/*.cu, links one shared library.

    python neural-galerkin_b200/build.py [--force]

The library lands in ``neural-galerkin_b200/jspsr/libngs.so`` so that it travels
with the source tree; object files go to ``neural-galerkin_b200/_build/``.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
INCLUDE = HERE.parent / "include"
BUILD = HERE / "_build"
LIB = HERE / "jspsr" / "libngs.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
              "-Xptxas", "-warn-spills", f"-I{INCLUDE}", f"-I{CSRC}"]
# Per-file flags.  pcg.cu: no multiply-add contraction, so that the single-system and the batched
# kernel (the same solver body inlined into two kernels) round every operation identically and a
# batched solve is bit-identical to the solo one; the SpMV is bound by memory, not by the extra adds.
FILE_FLAGS = {"pcg.cu": ["-fmad=false"]}


def nvcc() -> str:
    cand = [os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"]
    for c in cand:
        if c and Path(c).exists():
            return c
    raise RuntimeError("nvcc not found")


def _newest_dep() -> float:
    deps = list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.inc")) + list(INCLUDE.glob("*.h"))
    return max(p.stat().st_mtime for p in deps)


def compile_one(src: Path, force: bool, verbose_ptxas: bool) -> Path:
    obj = BUILD / (src.stem + ".o")
    if not force and obj.exists() and obj.stat().st_mtime >= max(src.stat().st_mtime, _newest_dep()):
        return obj
    cmd = [nvcc(), *ARCH, *NVCC_FLAGS, *FILE_FLAGS.get(src.name, []), "-c", str(src), "-o", str(obj)]
    if verbose_ptxas:
        cmd[1:1] = ["-Xptxas", "-v"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{res.stderr}")
    if verbose_ptxas:
        (BUILD / (src.stem + ".ptxas.txt")).write_text(res.stderr)
    return obj


def build(force: bool = False, verbose_ptxas: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    srcs = sorted(CSRC.glob("*.cu"))
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(lambda s: compile_one(s, force, verbose_ptxas), srcs))
    if force or not LIB.exists() or LIB.stat().st_mtime < max(o.stat().st_mtime for o in objs):
        tmp = LIB.with_suffix(".so.tmp")
        cmd = [nvcc(), *ARCH, "-shared", "-cudart", "static", "-o", str(tmp), *map(str, objs)]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stderr}")
        os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--ptxas", action="store_true", help="keep -Xptxas -v reports in _build/")
    a = ap.parse_args()
    print(build(a.force, a.ptxas))
    sys.exit(0)
