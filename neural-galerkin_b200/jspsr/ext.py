"""The reference's op modules, on libngs.

Drop-in for ``jspsr/ext.py`` of the reference, which re-exports five pybind11
CUDA modules (``jspsr._common``, ``_sparse_op``, ``_integration``,
``_sparse_solve``, ``_marching_cubes``; ``setup.py:17-48``) and defines
``CuckooHashTable`` (``ext.py:14-84``).  Same names, argument meaning, tensor
dtypes and return conventions; every op runs libngs kernels on torch's current
stream and raises ``RuntimeError`` on failure.
"""
from __future__ import annotations

import ctypes as C
from types import SimpleNamespace

import numpy as np
import torch

from . import _lib as L


def _check_cuda(*ts):
    for t in ts:
        if isinstance(t, torch.Tensor):
            L.require_cuda(t)


class HashLookupData:
    """Device key -> value table (the reference's ``HashLookupData``, ``hashmap_cuda.cuh:64-87``)."""

    def __init__(self, keys: torch.Tensor, vals: torch.Tensor | None, enlarge: bool):
        _check_cuda(keys)
        n = keys.numel()
        lib = L.load()
        nslots = lib.ngs_hash_table_slots(n, int(enlarge))
        self.slots = torch.empty(nslots * 2, dtype=torch.int64, device=keys.device)
        self.table = L.HashTable()
        self.table.slots, self.table.nslots = self.slots.data_ptr(), nslots
        status = torch.zeros(1, dtype=torch.int32, device=keys.device)
        use_vals = vals is not None and vals.numel() > 0
        L.call("ngs_hash_table_build", C.byref(self.table), L.ptr(keys.contiguous().long()),
               L.ptr(vals.contiguous().long()) if use_vals else None, n, L.ptr(status), L.stream())
        self.inserted_size = n
        # the reference synchronises after its insert and ignores a failed one
        # (hashmap_cuda.cu:152,187,369); here the insert status is read at that sync and raised
        rc = int(status.item())
        if rc != L.NGS_OK:
            raise L.NgsError(rc, "build_hash_table")

    def device(self):
        return self.slots.device


def hash_cuda(idx: torch.Tensor) -> torch.Tensor:
    """FNV-1a-60 key of each row of int32/int64 [N, D], D in {2,3,4} (``hashmap_cuda.cu:269``)."""
    _check_cuda(idx)
    idx = idx.contiguous()
    out = torch.empty(idx.shape[0], dtype=torch.int64, device=idx.device)
    L.call("ngs_hash_coords", L.ptr(idx), int(idx.dtype == torch.int64), idx.shape[0], idx.shape[1], L.ptr(out),
           L.stream())
    return out


def kernel_hash_cuda(idx: torch.Tensor, kernel_offset: torch.Tensor) -> torch.Tensor:
    """Keys of coord + offset for every (offset k, coord i): int64 [K, N] (``hashmap_cuda.cu:307``)."""
    _check_cuda(idx, kernel_offset)
    idx = idx.contiguous()
    off = kernel_offset.contiguous().int()
    out = torch.empty((off.shape[0], idx.shape[0]), dtype=torch.int64, device=idx.device)
    L.call("ngs_kernel_hash", L.ptr(idx), int(idx.dtype == torch.int64), idx.shape[0], idx.shape[1], L.ptr(off),
           off.shape[0], L.ptr(out), L.stream())
    return out


def build_hash_table(hash_target: torch.Tensor, idx_target: torch.Tensor, enlarge: bool) -> HashLookupData:
    """Table of keys -> idx_target (or row index when idx_target is empty) (``hashmap_cuda.cu:341``)."""
    return HashLookupData(hash_target, idx_target, enlarge)


def hash_table_query(hash_data: HashLookupData, hash_query: torch.Tensor) -> torch.Tensor:
    """value + 1 for present keys, 0 for absent ones (``hashmap_cuda.cu:381``)."""
    _check_cuda(hash_query)
    q = hash_query.contiguous().long()
    out = torch.empty(q.numel(), dtype=torch.int64, device=q.device)
    L.call("ngs_hash_table_query", C.byref(hash_data.table), L.ptr(q), q.numel(), L.ptr(out), L.stream())
    return out


# ----------------------------------------------------------------------------- sparse ops
def _starts(lengths: torch.Tensor):
    lengths = lengths.contiguous().long()
    start, total = L.scan(lengths)
    return lengths, start, total


def sparse_meshgrid(a_lengths: torch.Tensor, b_lengths: torch.Tensor):
    """Per-point meshgrid of index ranges (``sparse_product.cu:52-82``)."""
    _check_cuda(a_lengths, b_lengths)
    al, a0, _ = _starts(a_lengths)
    bl, b0, _ = _starts(b_lengths)
    ab0, ab_total = L.scan(al * bl)
    n = int(ab_total.item())
    ai = torch.empty(n, dtype=torch.int64, device=al.device)
    bi = torch.empty(n, dtype=torch.int64, device=al.device)
    L.call("ngs_sparse_meshgrid", L.ptr(a0), L.ptr(al), L.ptr(b0), L.ptr(bl), L.ptr(ab0), al.numel(), L.ptr(ai),
           L.ptr(bi), L.stream())
    return ai, bi


def screened_multiplication(hash_data, a_val, b_val, a_inds, b_inds, a_lengths, b_lengths, weight):
    """res[pair(a_inds[a], b_inds[b])] += a_val[a] . b_val[b] * weight[p] (``sparse_product.cu:202-258``)."""
    _check_cuda(a_val, b_val, a_inds, b_inds, a_lengths, b_lengths, weight)
    al, a0, _ = _starts(a_lengths)
    bl, b0, _ = _starts(b_lengths)
    dim = 1 if a_val.dim() == 1 else 3
    res = torch.zeros(hash_data.inserted_size, dtype=torch.float32, device=a_val.device)
    L.call("ngs_screened_multiplication", C.byref(hash_data.table), L.ptr(a_val.contiguous().float()),
           L.ptr(b_val.contiguous().float()), dim, L.ptr(a_inds.contiguous().long()), L.ptr(b_inds.contiguous().long()),
           L.ptr(a0), L.ptr(al), L.ptr(b0), L.ptr(bl), L.ptr(weight.contiguous().float()), al.numel(), L.ptr(res),
           L.stream())
    return res


def screened_multiplication_backward(hash_data, a_val, b_val, a_inds, b_inds, a_lengths, b_lengths, weight,
                                     grad_res):
    """Gradients of ``screened_multiplication`` w.r.t. a_val, b_val, weight (``sparse_product.cu:260-322``)."""
    _check_cuda(a_val, b_val, grad_res)
    al, a0, _ = _starts(a_lengths)
    bl, b0, _ = _starts(b_lengths)
    dim = 1 if a_val.dim() == 1 else 3
    ga = torch.zeros_like(a_val, dtype=torch.float32)
    gb = torch.zeros_like(b_val, dtype=torch.float32)
    gw = torch.zeros(weight.shape[0], dtype=torch.float32, device=a_val.device)
    L.call("ngs_screened_multiplication_backward", C.byref(hash_data.table), L.ptr(a_val.contiguous().float()),
           L.ptr(b_val.contiguous().float()), dim, L.ptr(a_inds.contiguous().long()), L.ptr(b_inds.contiguous().long()),
           L.ptr(a0), L.ptr(al), L.ptr(b0), L.ptr(bl), L.ptr(weight.contiguous().float()), al.numel(),
           L.ptr(grad_res.contiguous().float()), L.ptr(ga), L.ptr(gb), L.ptr(gw), L.stream())
    return [ga, gb, gw]


# ----------------------------------------------------------------------------- learned-basis integrals
def ddi_forward(source_expanded, target_expanded, rel_pos, f_f_i, df_df_i):
    """Per pair and axis bilinear forms of the learned basis (``ddi.cu:51-76``)."""
    _check_cuda(source_expanded, target_expanded, rel_pos, f_f_i, df_df_i)
    P = source_expanded.shape[0]
    C_, R = f_f_i.shape[0], f_f_i.shape[2]
    p = torch.empty((P, 3), dtype=torch.float32, device=source_expanded.device)
    q = torch.empty_like(p)
    L.call("ngs_ddi_forward", L.ptr(source_expanded.contiguous().float()), L.ptr(target_expanded.contiguous().float()),
           L.ptr(rel_pos.contiguous().long()), L.ptr(f_f_i.contiguous().float()), L.ptr(df_df_i.contiguous().float()),
           P, C_, R, L.ptr(p), L.ptr(q), L.stream())
    return p, q


def ddi_backward(source_expanded, target_expanded, rel_pos, f_f_i, df_df_i, grad_p, grad_q):
    """Gradients of ``ddi_forward`` (``ddi.cu:113-141``)."""
    _check_cuda(source_expanded, target_expanded, grad_p, grad_q)
    P = source_expanded.shape[0]
    C_, R = f_f_i.shape[0], f_f_i.shape[2]
    gs = torch.empty((P, 3 * C_), dtype=torch.float32, device=source_expanded.device)
    gt = torch.empty_like(gs)
    L.call("ngs_ddi_backward", L.ptr(source_expanded.contiguous().float()), L.ptr(target_expanded.contiguous().float()),
           L.ptr(rel_pos.contiguous().long()), L.ptr(f_f_i.contiguous().float()), L.ptr(df_df_i.contiguous().float()),
           L.ptr(grad_p.contiguous().float()), L.ptr(grad_q.contiguous().float()), P, C_, R, L.ptr(gs), L.ptr(gt),
           L.stream())
    return gs, gt


# ----------------------------------------------------------------------------- solvers
def _pcg(ap, aj, ax, b, inv_diag, tol, max_iter, res_fix, mode, b64=None, ax64=None):
    n = b.shape[0]
    dev = b.device
    rowptr = ap.contiguous().long()
    cols = aj.contiguous().int()
    x32 = torch.empty(n, dtype=torch.float32, device=dev)
    x64 = torch.empty(n, dtype=torch.float64, device=dev)
    info = torch.zeros(4, dtype=torch.int64, device=dev)
    resid = torch.zeros(2, dtype=torch.float64, device=dev)
    s = L.PcgSystem()
    s.n, s.nnz = n, cols.numel()
    s.rowptr, s.cols, s.inv_diag = rowptr.data_ptr(), cols.data_ptr(), inv_diag.contiguous().float().data_ptr()
    ax32 = ax.contiguous().float()
    s.vals32 = ax32.data_ptr()
    s.vals64 = ax64.data_ptr() if ax64 is not None else None
    b32 = b.contiguous().float()
    s.b32 = b32.data_ptr()
    s.b64 = b64.data_ptr() if b64 is not None else None
    s.x32, s.x64 = x32.data_ptr(), x64.data_ptr()
    cfg = L.PcgConfig()
    cfg.mode, cfg.max_iter, cfg.tol, cfg.res_fix, cfg.replace_every, cfg.blocks, cfg.timeout_s = \
        mode, int(max_iter), float(tol), int(bool(res_fix)), 50, 0, 30.0
    ws_bytes = L.load().ngs_pcg_workspace_bytes(n, mode)
    ws = torch.empty(max(ws_bytes, 8), dtype=torch.uint8, device=dev)
    keep = (rowptr, cols, ax32, b32, ws)
    L.call("ngs_pcg_solve", C.byref(s), C.byref(cfg), L.ptr(ws), ws_bytes, L.ptr(info), L.ptr(resid), L.stream())
    st = info.cpu().numpy()
    del keep
    if st[1] not in (L.NGS_OK, L.NGS_ERR_NOT_CONVERGED):
        raise L.NgsError(int(st[1]), "pcg")
    return (x32 if mode == L.PCG_REFERENCE else x64.float()), int(st[0])


def solve_pcg_diag(Ap, Aj, Ax, b, inv_diag_A, tol: float, max_iter: int, res_fix: bool):
    """Jacobi-PCG on CSR with the reference's stopping rule (``solve_pcg.cu:15-136``) -> (x, iterations)."""
    _check_cuda(Ap, Aj, Ax, b, inv_diag_A)
    return _pcg(Ap, Aj, Ax, b, inv_diag_A, tol, max_iter, res_fix, L.PCG_REFERENCE)


def solve_cusparse(Ap, Aj, Ax, b, tol: float):
    """Direct-solve replacement (``solve_cusparse.cu:15-42``): FP64 PCG to 1e-12 relative residual."""
    _check_cuda(Ap, Aj, Ax, b)
    n = b.shape[0]
    rowptr = Ap.long()
    rows = torch.repeat_interleave(torch.arange(n, device=b.device), rowptr[1:] - rowptr[:-1])
    ax64 = Ax.double()
    diag = torch.zeros(n, dtype=torch.float64, device=b.device).index_add_(0, rows[Aj.long() == rows],
                                                                            ax64[Aj.long() == rows])
    x, _ = _pcg(Ap, Aj, Ax, b, (1.0 / diag).float(), 1e-12, -1, False, L.PCG_FP64, b64=b.double(), ax64=ax64)
    return x


def init_cusolver():
    """No-op: there is no cuSOLVER handle to create (``solve_cusparse.cu:10``)."""


# ----------------------------------------------------------------------------- marching cubes
def marching_cubes_sparse(cube_base: torch.Tensor, cube_sdf: torch.Tensor):
    """Primal sparse MC on r^3 sub-cells (``primal_mc.cu:170-235``)."""
    _check_cuda(cube_base, cube_sdf)
    base = cube_base.contiguous().float()
    sdf = cube_sdf.contiguous().float()
    M, r = base.shape[0], sdf.shape[1] - 1
    dev = base.device
    vc = torch.empty(M * r * r * r, dtype=torch.int32, device=dev)
    L.call("ngs_primal_mc_count", L.ptr(sdf), M, r, L.ptr(vc), L.stream())
    off, tot = L.scan(vc)
    nv = int(tot.item())
    T = nv // 3
    tris = torch.empty((T, 3, 3), dtype=torch.float32, device=dev)
    vids = torch.empty((T, 3, 4), dtype=torch.int32, device=dev)
    sids = torch.empty((T, 3, 2), dtype=torch.int32, device=dev)
    sw = torch.empty((T, 3, 1), dtype=torch.float32, device=dev)
    L.call("ngs_primal_mc_emit", L.ptr(base), L.ptr(sdf), M, r, L.ptr(off), L.ptr(tris), L.ptr(vids), L.ptr(sids),
           L.ptr(sw), L.stream())
    return [tris, vids, sids, sw]


def dual_marching_cubes_sparse(cube_corner_inds: torch.Tensor, corner_pos: torch.Tensor, corner_value: torch.Tensor):
    """Dual MC over cubes whose corners index arbitrary points (``dual_mc.cu:135-189``)."""
    _check_cuda(cube_corner_inds, corner_pos, corner_value)
    acc = cube_corner_inds.contiguous().int()
    pos = corner_pos[:, :3].contiguous().float()
    val = corner_value.contiguous().float()
    M = acc.shape[0]
    dev = acc.device
    vc = torch.empty(M, dtype=torch.int32, device=dev)
    L.call("ngs_dual_mc_count", L.ptr(acc), 2, None, M, L.ptr(val), L.ptr(vc), L.stream())
    off, tot = L.scan(vc)
    nv = int(tot.item())
    tris = torch.empty((nv // 3, 3, 3), dtype=torch.float32, device=dev)
    vids = torch.empty((nv // 3, 3, 2), dtype=torch.int32, device=dev)
    L.call("ngs_dual_mc_emit", L.ptr(acc), 2, None, M, L.ptr(pos), L.ptr(val), L.ptr(off), L.ptr(tris), L.ptr(vids), L.stream())
    return [tris, vids]


def dual_marching_cubes_indices(dual_centers_hash_data: HashLookupData, expand_primal_base: dict,
                                primal_strides: dict, primal_inds_base: dict):
    """Dual-cube corner accumulation through the dual-centre key table (``dual_mc_inds.cu:143-182``)."""
    n = dual_centers_hash_data.inserted_size
    dev = dual_centers_hash_data.device()
    acc = torch.zeros((n, 8, 2), dtype=torch.int32, device=dev)
    cnt = torch.zeros(n, dtype=torch.int32, device=dev)
    for d, stride in primal_strides.items():
        base = expand_primal_base[d].contiguous().int()
        L.call("ngs_dual_mc_indices_hash", C.byref(dual_centers_hash_data.table), L.ptr(base), base.shape[0],
               int(stride), int(d), int(primal_inds_base[d]), L.ptr(acc), 2, L.ptr(cnt), L.stream())
    return [acc, cnt]


# ----------------------------------------------------------------------------- sparse convolution
_CONV_DTYPES = {torch.float16: L.NGS_F16, torch.bfloat16: L.NGS_BF16, torch.float32: L.NGS_F32}


def _conv_dtype(t: torch.Tensor) -> int:
    if t.dtype not in _CONV_DTYPES:
        raise TypeError(f"sparse convolution takes float16, bfloat16 or float32 features, not {t.dtype}")
    return _CONV_DTYPES[t.dtype]


def _offset_starts(neighbor_offset, K: int, device):
    """int64 [K+1] exclusive prefix of the per-offset pair counts, on the device, and the largest count."""
    sizes = torch.as_tensor(neighbor_offset).reshape(-1).to(device="cpu", dtype=torch.int64)
    if sizes.numel() != K:
        raise ValueError(f"neighbor_offset has {sizes.numel()} entries for a kernel of {K} offsets")
    starts = torch.zeros(K + 1, dtype=torch.int64)
    starts[1:] = torch.cumsum(sizes, 0)
    return starts.to(device), int(sizes.max()) if K else 0


def _conv_table(neighbor_map, starts, K, key_col, n_rows, mid):
    table = torch.empty((n_rows, K), dtype=torch.int32, device=neighbor_map.device)
    L.call("ngs_conv_table", L.ptr(neighbor_map), L.ptr(starts), K, key_col, n_rows, mid, L.ptr(table), L.stream())
    return table


def _gather_gemm(x, table, bt, ncols, out):
    err = torch.zeros(1, dtype=torch.int32, device=x.device)
    dt = _conv_dtype(x)
    out_f32 = int(out.dtype == torch.float32)
    L.call("ngs_conv_gather_gemm", L.ptr(x), x.shape[0], x.shape[1], L.ptr(table), table.shape[0], table.shape[1],
           L.ptr(bt), ncols, dt, L.ptr(out), out_f32, L.ptr(err), L.stream())
    return err


def _raise_device_error(err):
    code = int(err.item())
    if code:
        raise L.NgsError(code, "sparse convolution")


def convolution_forward_cuda(in_feat, out_feat, kernel, neighbor_map, neighbor_offset, transpose: bool,
                             no_acc: bool):
    """``sparse_op.convolution_forward_cuda`` (convolution_cuda.cu:52-174): out_feat [M, Cout] receives
    sum over offsets k and pairs (i, o) of offset k of in_feat[i] @ kernel[k] (pairs (map[:,0], map[:,1]),
    read the other way round when ``transpose``).  As in the reference, when the kernel volume is odd,
    the input and output counts agree and ``no_acc`` is false, the centre offset is the identity over
    all rows and out_feat is overwritten; otherwise the sum is added to out_feat.  One fused gather-GEMM
    kernel on the tensor cores (16-bit features, FP32 accumulation)."""
    _check_cuda(in_feat, out_feat, kernel, neighbor_map)
    if in_feat.shape[1] != kernel.shape[1]:
        raise ValueError("Input feature size and kernel size mismatch")
    K, cin, cout = kernel.shape
    x = in_feat.contiguous()
    w = kernel.contiguous().to(x.dtype)
    nbmap = neighbor_map.int().contiguous()
    starts, _ = _offset_starts(neighbor_offset, K, x.device)
    n_out = out_feat.shape[0]
    precompute_mid = K % 2 == 1 and x.shape[0] == n_out and not no_acc
    key_col = 0 if transpose else 1
    table = _conv_table(nbmap, starts, K, key_col, n_out, K // 2 if precompute_mid else -1)
    wt = torch.empty((K, cout, cin), dtype=w.dtype, device=w.device)
    L.call("ngs_conv_transpose_weight", L.ptr(w), K, cin, cout, _conv_dtype(w), L.ptr(wt), L.stream())
    if precompute_mid and out_feat.is_contiguous() and out_feat.dtype == x.dtype:
        err = _gather_gemm(x, table, wt, cout, out_feat)
    else:
        res = torch.empty((n_out, cout), dtype=out_feat.dtype, device=x.device)
        err = _gather_gemm(x, table, wt, cout, res)
        if precompute_mid:
            out_feat.copy_(res)
        else:
            out_feat.add_(res)
    _raise_device_error(err)


def convolution_backward_cuda(in_feat, grad_in_feat, grad_out_feat, kernel, grad_kernel, neighbor_map,
                              neighbor_offset, transpose: bool):
    """``sparse_op.convolution_backward_cuda`` (convolution_cuda.cu:176-282): grad_in_feat = sum over pairs
    (i, o) of offset k of grad_out[o] @ kernel[k]^T (gathered per input row, no scatter) and
    grad_kernel[k] = sum over the pairs of in_feat[i]^T grad_out[o] (a GEMM over the pairs, split over
    CTAs and reduced in a fixed order); both are overwritten, as the reference zeroes them."""
    _check_cuda(in_feat, grad_in_feat, grad_out_feat, kernel, grad_kernel, neighbor_map)
    K, cin, cout = kernel.shape
    x = in_feat.contiguous()
    gy = grad_out_feat.contiguous().to(x.dtype)
    w = kernel.contiguous().to(x.dtype)
    nbmap = neighbor_map.int().contiguous()
    starts, max_pairs = _offset_starts(neighbor_offset, K, x.device)
    in_col = 1 if transpose else 0
    table = _conv_table(nbmap, starts, K, in_col, x.shape[0], -1)
    grad_in_feat.resize_(x.shape)
    grad_kernel.resize_(kernel.shape)
    gi = grad_in_feat if (grad_in_feat.is_contiguous() and grad_in_feat.dtype == x.dtype) else \
        torch.empty(x.shape, dtype=x.dtype, device=x.device)
    err = _gather_gemm(gy, table, w, cin, gi)
    if gi is not grad_in_feat:
        grad_in_feat.copy_(gi)
    dt = _conv_dtype(x)
    gk = grad_kernel if (grad_kernel.is_contiguous() and grad_kernel.dtype == x.dtype) else \
        torch.empty(kernel.shape, dtype=x.dtype, device=x.device)
    ws_bytes = L.load().ngs_conv_weight_grad_ws_bytes(K, cin, cout, max_pairs)
    ws = torch.empty(max(ws_bytes, 16), dtype=torch.uint8, device=x.device)
    L.call("ngs_conv_weight_grad", L.ptr(x), x.shape[0], cin, L.ptr(gy), gy.shape[0], cout, L.ptr(nbmap), L.ptr(starts),
           K, max_pairs, in_col, dt, L.ptr(gk), int(gk.dtype == torch.float32), L.ptr(ws), ws.numel(), L.ptr(err),
           L.stream())
    if gk is not grad_kernel:
        grad_kernel.copy_(gk)
    _raise_device_error(err)


# ----------------------------------------------------------------------------- module namespaces
common = _common = SimpleNamespace(hash_cuda=hash_cuda, kernel_hash_cuda=kernel_hash_cuda,
                                   build_hash_table=build_hash_table, hash_table_query=hash_table_query,
                                   HashLookupData=HashLookupData)
sparse_op = _sparse_op = SimpleNamespace(sparse_meshgrid=sparse_meshgrid, screened_multiplication=screened_multiplication,
                                         screened_multiplication_backward=screened_multiplication_backward,
                                         convolution_forward_cuda=convolution_forward_cuda,
                                         convolution_backward_cuda=convolution_backward_cuda)
integration = _integration = SimpleNamespace(ddi_forward=ddi_forward, ddi_backward=ddi_backward)
sparse_solve = _sparse_solve = SimpleNamespace(solve_pcg_diag=solve_pcg_diag, solve_cusparse=solve_cusparse,
                                               init_cusolver=init_cusolver)
marching_cubes = _marching_cubes = SimpleNamespace(marching_cubes_sparse=marching_cubes_sparse,
                                                   dual_marching_cubes_sparse=dual_marching_cubes_sparse,
                                                   dual_marching_cubes_indices=dual_marching_cubes_indices)


class CuckooHashTable:
    """Key table for positional queries (``ext.py:14-84``): same constructor and query API.

    The device table is open addressing rather than cuckoo hashing; query results are the same.
    """

    def __init__(self, data: torch.Tensor = None, hashed_data: torch.Tensor = None, enlarged: bool = False):
        if data is not None:
            self.dim = data.size(1)
            assert data.size(0) > 0
            source_hash = hash_cuda(data.contiguous())
        else:
            self.dim = -1
            source_hash = hashed_data
        self.object = build_hash_table(source_hash, torch.tensor([], device=source_hash.device), enlarged)

    @classmethod
    def _sphash(cls, coords: torch.Tensor, offsets=None) -> torch.Tensor:
        assert coords.dtype in [torch.int, torch.long], coords.dtype
        coords = coords.contiguous()
        if offsets is None:
            assert coords.ndim == 2 and coords.shape[1] in [2, 3, 4], coords.shape
            if coords.size(0) == 0:
                return torch.empty((0,), dtype=torch.int64, device=coords.device)
            return hash_cuda(coords)
        assert offsets.dtype == torch.int, offsets.dtype
        assert offsets.ndim == 2 and offsets.shape[1] == 3, offsets.shape
        assert coords.ndim == 2 and coords.shape[1] in [3, 4], coords.shape
        if coords.size(0) == 0 or offsets.size(0) == 0:
            return torch.empty((offsets.size(0), coords.size(0)), dtype=torch.int64, device=coords.device)
        return kernel_hash_cuda(coords, offsets.contiguous())

    def query(self, coords, offsets=None):
        assert coords.size(1) == self.dim
        return self.query_hashed(self._sphash(coords, offsets))

    def query_hashed(self, hashed_query: torch.Tensor):
        sizes = hashed_query.size()
        hashed_query = hashed_query.view(-1)
        if hashed_query.size(0) == 0:
            return torch.zeros(sizes, dtype=torch.int64, device=hashed_query.device) - 1
        output = hash_table_query(self.object, hashed_query.contiguous())
        return (output - 1).view(*sizes)
