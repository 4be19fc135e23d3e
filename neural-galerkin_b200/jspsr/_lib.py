"""ctypes binding of libngs.so (the C ABI declared in include/ngs.h).

The library is built in-tree by ``neural-galerkin_b200/build.py``.  There is no
CPU fallback: every op raises if the library is missing or if a CUDA call
fails, with the library's status message.
"""
from __future__ import annotations

import ctypes as C
import math
import threading
from pathlib import Path

import numpy as np
import torch

LIB_PATH = Path(__file__).resolve().parent / "libngs.so"

STATUS = {0: "ok", 1: "invalid argument", 2: "buffer or workspace too small", 3: "hash insert failed",
          4: "not converged", 5: "topology error", 6: "CUDA error", 7: "device-side wait timed out"}
NGS_OK, NGS_ERR_INVALID_ARG, NGS_ERR_OOM, NGS_ERR_HASH_INSERT, NGS_ERR_NOT_CONVERGED = 0, 1, 2, 3, 4
NGS_ERR_TOPOLOGY, NGS_ERR_CUDA, NGS_ERR_TIMEOUT = 5, 6, 7
PCG_REFERENCE, PCG_MIXED, PCG_FP64 = 0, 1, 2
NGS_F16, NGS_BF16, NGS_F32 = 0, 1, 2
MAX_FIELD_LEVELS = 16

vp, i32, i64, f32, f64, sz = C.c_void_p, C.c_int32, C.c_int64, C.c_float, C.c_double, C.c_size_t


class Grid(C.Structure):
    _fields_ = [("origin", C.c_int32 * 3), ("dims", C.c_int32 * 3), ("stride", C.c_int32),
                ("log2_stride", C.c_int32), ("zwords", C.c_int32), ("pad_", C.c_int32),
                ("nwords", C.c_int64), ("words", C.c_void_p)]


class HashTable(C.Structure):
    _fields_ = [("slots", C.c_void_p), ("nslots", C.c_int64), ("inserted", C.c_int64)]


class PcgOperator(C.Structure):
    """ngs_pcg_operator: the matrix-free level operator (stencil over the bitmap + point screening)."""
    _fields_ = [("grid", Grid), ("coords", vp), ("stencil", vp), ("alpha", C.c_double), ("n_points", C.c_int64),
                ("point_rows", vp), ("point_phi", vp), ("t_ptr", vp), ("t_point", vp), ("t_phi", vp),
                ("scratch32", vp), ("scratch64", vp)]


class PcgSystem(C.Structure):
    _fields_ = [("n", C.c_int64), ("nnz", C.c_int64), ("rowptr", vp), ("cols", vp), ("vals32", vp),
                ("vals64", vp), ("b32", vp), ("b64", vp), ("inv_diag", vp), ("x32", vp), ("x64", vp),
                ("col_delta", vp), ("op", C.POINTER(PcgOperator)), ("band", C.c_int64)]


class PcgConfig(C.Structure):
    _fields_ = [("mode", C.c_int), ("max_iter", C.c_int), ("tol", C.c_double), ("res_fix", C.c_int),
                ("replace_every", C.c_int), ("blocks", C.c_int), ("timeout_s", C.c_double)]


G, H = Grid, C.POINTER(HashTable)
PCG_BATCH_MAX = 64


class PcgBatchItem(C.Structure):
    _fields_ = [("sys", PcgSystem), ("cfg", PcgConfig), ("ws", vp), ("ws_bytes", sz), ("info_dev", vp),
                ("resid_dev", vp)]


_SIGS = {
    "ngs_status_string": ([C.c_int], C.c_char_p),
    "ngs_last_cuda_error": ([], C.c_char_p),
    "ngs_version": ([], C.c_int),
    "ngs_launch_count": ([], i64),
    "ngs_reset_launch_count": ([], None),
    "ngs_hash_coords": ([vp, C.c_int, i64, C.c_int, vp, vp], C.c_int),
    "ngs_kernel_hash": ([vp, C.c_int, i64, C.c_int, vp, i64, vp, vp], C.c_int),
    "ngs_hash_table_slots": ([i64, C.c_int], i64),
    "ngs_hash_table_build": ([H, vp, vp, i64, vp, vp], C.c_int),
    "ngs_hash_table_query": ([H, vp, i64, vp, vp], C.c_int),
    "ngs_hash_table_query_coords": ([H, vp, i64, vp, vp], C.c_int),
    "ngs_scan_workspace_bytes": ([i64], sz),
    "ngs_exclusive_scan_i64": ([vp, i64, vp, vp, vp, sz, vp], C.c_int),
    "ngs_exclusive_scan_i32": ([vp, i64, vp, vp, vp, sz, vp], C.c_int),
    "ngs_points_bbox": ([vp, i64, vp, vp], C.c_int),
    "ngs_grid_mark_points": ([G, vp, i64, f32, vp, C.c_int, vp], C.c_int),
    "ngs_grid_mark_coords": ([G, vp, i64, vp, C.c_int, C.c_int, vp], C.c_int),
    "ngs_grid_workspace_bytes": ([C.POINTER(Grid)], sz),
    "ngs_grid_finalize": ([G, vp, sz, vp, vp], C.c_int),
    "ngs_grid_emit_coords": ([G, vp, vp], C.c_int),
    "ngs_grid_band_bound": ([G, i64, vp, vp], C.c_int),
    "ngs_grid_lookup": ([G, vp, i64, vp, vp], C.c_int),
    "ngs_grid_neighbours_tiles": ([i64], i64),
    "ngs_grid_neighbours_count": ([G, vp, vp, C.c_int, i64, C.c_int, C.c_int, vp, C.c_int, C.c_int, vp, vp, vp,
                                   vp, vp], C.c_int),
    "ngs_grid_neighbours_fill": ([G, vp, vp, C.c_int, i64, C.c_int, C.c_int, vp, C.c_int, C.c_int, vp, vp, vp, vp,
                                  vp, vp], C.c_int),
    "ngs_knn_mark_cells": ([G, vp, i64, f32, vp], C.c_int),
    "ngs_knn_bucket": ([G, vp, i64, f32, vp, vp, vp], C.c_int),
    "ngs_knn_scatter": ([vp, i64, vp, vp, vp, vp], C.c_int),
    "ngs_knn_sdf": ([G, vp, vp, vp, vp, vp, i64, f32, f32, C.c_int, f32, vp, vp, vp, vp], C.c_int),
    "ngs_splat_weights": ([G, vp, i64, f32, f64, vp, vp], C.c_int),
    "ngs_density_eval": ([G, vp, i64, f32, f64, vp, f32, C.c_int, vp, vp, vp, vp], C.c_int),
    "ngs_splat_data": ([G, vp, i64, f32, f64, vp, C.c_int, vp, vp, C.c_int, f32, vp, vp], C.c_int),
    "ngs_point_basis": ([G, vp, i64, f32, f64, vp, vp, vp], C.c_int),
    "ngs_point_field": ([vp, vp, i64, vp, vp, C.c_int, vp], C.c_int),
    "ngs_eval_field": ([G, vp, i64, f32, f64, vp, C.c_int, vp, vp], C.c_int),
    "ngs_eval_field_cells": ([C.POINTER(Grid), C.POINTER(vp), C.c_int, i64, vp, f32, f64, vp, vp], C.c_int),
    "ngs_eval_field_levels": ([C.POINTER(Grid), C.POINTER(vp), C.c_int, vp, i64, f32, f64, C.c_int, vp, vp], C.c_int),
    "ngs_weighted_sum": ([vp, vp, i64, vp, vp], C.c_int),
    "ngs_stencil_count": ([G, vp, i64, vp, vp, vp], C.c_int),
    "ngs_stencil_fill": ([G, vp, i64, vp, vp, vp, vp, vp, vp, vp], C.c_int),
    "ngs_screen_gram": ([vp, vp, i64, vp, vp, vp, f64, vp, vp], C.c_int),
    "ngs_point_cell_keys": ([vp, i64, vp, vp], C.c_int),
    "ngs_screen_gram_grouped": ([vp, vp, i64, vp, vp, vp, vp, vp, f64, vp, vp], C.c_int),
    "ngs_screen_rhs": ([vp, vp, i64, vp, f64, vp, vp], C.c_int),
    "ngs_screen_rhs_grouped": ([vp, vp, i64, vp, vp, vp, vp, f64, vp, vp], C.c_int),
    "ngs_rhs_normals": ([G, vp, i64, vp, G, vp, i64, vp, vp, C.c_int, vp, vp], C.c_int),
    "ngs_correction_stiffness": ([vp, i64, C.c_int, G, vp, vp, vp, C.c_int, vp, vp], C.c_int),
    "ngs_correction_screen": ([vp, vp, i64, vp, vp, f64, vp, vp], C.c_int),
    "ngs_finish_system": ([vp, i64, vp, i64, vp, vp, vp], C.c_int),
    "ngs_csr_col_delta": ([vp, vp, i64, vp, vp], C.c_int),
    "ngs_mf_count": ([vp, i64, i64, vp, vp, vp], C.c_int),
    "ngs_mf_fill": ([vp, vp, i64, vp, i64, vp, vp, vp, vp, vp, vp], C.c_int),
    "ngs_mf_diag": ([vp, vp, i64, f64, f64, vp, vp], C.c_int),
    "ngs_mf_screen_rhs": ([vp, vp, vp, i64, vp, f64, vp, vp], C.c_int),
    "ngs_mf_apply64": ([C.POINTER(PcgOperator), i64, vp, vp, vp], C.c_int),
    "ngs_mf_gram": ([vp, vp, vp, i64, vp, vp, vp, vp, f64, vp, vp], C.c_int),
    "ngs_conv_table": ([vp, vp, C.c_int, C.c_int, i64, C.c_int, vp, vp], C.c_int),
    "ngs_conv_transpose_weight": ([vp, C.c_int, C.c_int, C.c_int, C.c_int, vp, vp], C.c_int),
    "ngs_conv_tensor_core_ok": ([C.c_int, C.c_int, C.c_int], C.c_int),
    "ngs_conv_gather_gemm": ([vp, i64, C.c_int, vp, i64, C.c_int, vp, C.c_int, C.c_int, vp, C.c_int, vp, vp],
                             C.c_int),
    "ngs_conv_weight_grad_ws_bytes": ([C.c_int, C.c_int, C.c_int, i64], sz),
    "ngs_conv_weight_grad": ([vp, i64, C.c_int, vp, i64, C.c_int, vp, vp, C.c_int, i64, C.c_int, C.c_int, vp,
                              C.c_int, vp, sz, vp, vp], C.c_int),
    "ngs_pcg_workspace_bytes": ([i64, C.c_int], sz),
    "ngs_pcg_solve": ([C.POINTER(PcgSystem), C.POINTER(PcgConfig), vp, sz, vp, vp, vp], C.c_int),
    "ngs_pcg_block_capacity": ([C.c_int], C.c_int),
    "ngs_pcg_blocks": ([i64, i64, C.c_int], C.c_int),
    "ngs_pcg_window": ([i64, i64, i64, C.c_int], C.c_int),
    "ngs_pcg_cluster_size": ([i64, i64, C.c_int], C.c_int),
    "ngs_pcg_solve_batch": ([C.POINTER(PcgBatchItem), C.c_int, vp], C.c_int),
    "ngs_pcg_noalloc_max_rows": ([], i64),
    "ngs_pcg_solve_noalloc": ([C.POINTER(PcgSystem), C.POINTER(PcgConfig), vp, vp, vp], C.c_int),
    "ngs_spmv64": ([i64, vp, vp, vp, vp, vp, vp], C.c_int),
    "ngs_dot64": ([vp, vp, i64, vp, vp], C.c_int),
    "ngs_axpby64": ([i64, f64, vp, f64, vp, vp], C.c_int),
    "ngs_mul64": ([i64, vp, vp, vp, vp], C.c_int),
    "ngs_sparse_meshgrid": ([vp, vp, vp, vp, vp, i64, vp, vp, vp], C.c_int),
    "ngs_screened_multiplication": ([H, vp, vp, C.c_int, vp, vp, vp, vp, vp, vp, vp, i64, vp, vp], C.c_int),
    "ngs_screened_multiplication_backward": ([H, vp, vp, C.c_int, vp, vp, vp, vp, vp, vp, vp, i64, vp, vp, vp,
                                              vp, vp], C.c_int),
    "ngs_ddi_forward": ([vp, vp, vp, vp, vp, i64, C.c_int, C.c_int, vp, vp, vp], C.c_int),
    "ngs_ddi_backward": ([vp, vp, vp, vp, vp, vp, vp, i64, C.c_int, C.c_int, vp, vp, vp], C.c_int),
    "ngs_primal_mc_count": ([vp, i64, C.c_int, vp, vp], C.c_int),
    "ngs_primal_mc_emit": ([vp, vp, i64, C.c_int, vp, vp, vp, vp, vp, vp], C.c_int),
    "ngs_dual_mc_indices_cells": ([G, vp, i64, C.c_int, i64, vp, C.c_int, vp, vp], C.c_int),
    "ngs_grid_mark_cell_corners": ([G, vp, i64, C.c_int, vp], C.c_int),
    "ngs_dual_mc_indices_grid": ([G, vp, i64, C.c_int, C.c_int, i64, vp, C.c_int, vp, vp], C.c_int),
    "ngs_dual_mc_indices_hash": ([H, vp, i64, C.c_int, C.c_int, i64, vp, C.c_int, vp, vp], C.c_int),
    "ngs_dual_mc_select": ([vp, i64, vp, vp], C.c_int),
    "ngs_dual_mc_compact": ([vp, C.c_int, vp, vp, i64, vp, vp], C.c_int),
    "ngs_dual_mc_count": ([vp, C.c_int, vp, i64, vp, vp, vp], C.c_int),
    "ngs_dual_mc_emit": ([vp, C.c_int, vp, i64, vp, vp, vp, vp, vp, vp], C.c_int),
    "ngs_vdedup_count": ([vp, i64, vp, vp], C.c_int),
    "ngs_vdedup_sort": ([vp, i64, vp, i64, vp, vp, vp, vp], C.c_int),
    "ngs_vdedup_emit": ([vp, vp, i64, vp, vp, vp, vp, vp, vp, vp], C.c_int),
    "ngs_conformal_children": ([vp, i64, C.c_int, vp, vp], C.c_int),
    "ngs_leaf_flags": ([vp, i64, G, vp, vp], C.c_int),
    "ngs_compact_coords": ([vp, vp, vp, i64, vp, vp], C.c_int),
    "ngs_expand_cells": ([vp, i64, C.c_int, C.c_int, f32, vp, vp, vp], C.c_int),
}

_lib = None


def load():
    """Load libngs.so and attach prototypes (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"libngs.so not found at {LIB_PATH}; build it with neural-galerkin_b200/build.py")
        # PyDLL: the interpreter lock is kept across calls.  Every entry point only enqueues work on
        # a stream and returns in microseconds; releasing and re-acquiring the lock around each of
        # the few hundred calls of a reconstruction makes concurrent host threads (the serving
        # workers) queue for the lock at every call.
        lib = C.PyDLL(str(LIB_PATH))
        for name, (args, ret) in _SIGS.items():
            fn = getattr(lib, name)
            fn.argtypes, fn.restype = args, ret
        _lib = lib
    return _lib


def exported_symbols():
    return list(_SIGS)


class NgsError(RuntimeError):
    def __init__(self, status, where):
        lib = load()
        msg = lib.ngs_status_string(status).decode()
        if status == 6:
            msg += ": " + lib.ngs_last_cuda_error().decode()
        super().__init__(f"{where}: {msg}")
        self.status = status


def call(name, *args):
    """Call a libngs entry point; raise NgsError on a non-OK status."""
    rc = getattr(load(), name)(*args)
    if rc != NGS_OK:
        raise NgsError(rc, name)
    return rc


def require_cuda(t: torch.Tensor, name="tensor"):
    if not t.is_cuda:
        raise RuntimeError(f"{name} must be a CUDA tensor (libngs has no CPU path)")


def ptr(t):
    return None if t is None else C.c_void_p(t.data_ptr())


_raw_stream = getattr(torch._C, "_cuda_getCurrentRawStream", None)
_cur_device = getattr(torch._C, "_cuda_getDevice", None)


def stream():
    """The calling thread's current CUDA stream (torch's), as a handle for the C-ABI."""
    if _raw_stream is not None and _cur_device is not None:
        return C.c_void_p(_raw_stream(_cur_device()))
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


_dev_tables: dict = {}
_dev_tables_lock = threading.Lock()


def device_table(key, make, device) -> torch.Tensor:
    """A constant table uploaded once per device: ``make()`` -> numpy / torch host array.  The
    upload of a pageable host array waits for the stream, so per-call uploads would serialise the
    host with the GPU."""
    dev = torch.device(device)
    k = (key, dev.index)
    t = _dev_tables.get(k)
    if t is None:
        with _dev_tables_lock:
            t = _dev_tables.get(k)
            if t is None:
                a = make()
                t = (torch.from_numpy(a) if not isinstance(a, torch.Tensor) else a).to(dev)
                torch.cuda.synchronize(dev)
                _dev_tables[k] = t
    return t


# ----------------------------------------------------------------------------- helpers
def scan(values: torch.Tensor, out: torch.Tensor = None, total: torch.Tensor = None):
    """Exclusive prefix sum (int32 or int64 values) -> int64; returns (out, total_dev)."""
    n = values.numel()
    out = torch.empty(n, dtype=torch.int64, device=values.device) if out is None else out
    total = torch.empty(1, dtype=torch.int64, device=values.device) if total is None else total
    ws_bytes = load().ngs_scan_workspace_bytes(n)
    ws = torch.empty(max(ws_bytes, 8), dtype=torch.uint8, device=values.device)
    fn = "ngs_exclusive_scan_i64" if values.dtype == torch.int64 else "ngs_exclusive_scan_i32"
    call(fn, ptr(values), n, ptr(out), ptr(total), ptr(ws), ws_bytes, stream())
    return out, total


def make_grid(origin, dims, stride, device) -> tuple[Grid, torch.Tensor]:
    """A zeroed rank-bitmap over the box origin + [0, dims) * stride."""
    stride = int(stride)
    assert stride > 0 and stride & (stride - 1) == 0
    dims = [max(int(d), 1) for d in dims]
    zwords = (dims[2] + 63) // 64
    nwords = dims[0] * dims[1] * zwords
    if nwords > (1 << 33):
        raise RuntimeError(f"voxel index box too large ({dims} cells at stride {stride})")
    words = torch.zeros(nwords * 2, dtype=torch.int64, device=device)
    g = Grid()
    for a in range(3):
        g.origin[a] = int(origin[a])
        g.dims[a] = dims[a]
    g.stride, g.log2_stride, g.zwords, g.nwords = stride, int(math.log2(stride)), zwords, nwords
    g.words = words.data_ptr()
    return g, words


def grid_finalize(g: Grid, words: torch.Tensor, count: torch.Tensor):
    ws_bytes = load().ngs_grid_workspace_bytes(C.byref(g))
    ws = torch.empty(max(ws_bytes, 8), dtype=torch.uint8, device=words.device)
    call("ngs_grid_finalize", g, ptr(ws), ws_bytes, ptr(count), stream())
    return ws


def null_grid() -> Grid:
    g = Grid()
    g.stride, g.log2_stride, g.zwords, g.nwords, g.words = 1, 0, 1, 0, None
    return g


def f32_inv(vs: float) -> float:
    """fp32(1 / fp32(vs)): the reciprocal torch multiplies by when dividing by a Python float on CUDA."""
    return float(np.float32(1.0) / np.float32(vs))
