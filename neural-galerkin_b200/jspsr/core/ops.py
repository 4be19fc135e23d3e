"""Differentiable wrappers and helpers (reference: ``jspsr/core/ops.py:9-145``)."""
from __future__ import annotations

import numpy as np
import torch

from .. import _lib as L
from .. import ext


def _scatter_sum(src, index, n):
    return torch.zeros((n,) + src.shape[1:], dtype=src.dtype, device=src.device).index_add_(0, index.long(), src)


def torch_unique(input: torch.Tensor, sorted: bool = False, return_inverse: bool = False,
                 return_counts: bool = False, dim: int = None):
    """Row-unique with the reference's empty-input fix (``ops.py:103-127``).

    int32 [N, 3] coordinates on the GPU (voxel sets, the case on the reconstruction path) go
    through the rank bitmap of libngs: sorted lexicographic rows and inverse indices without a
    sort.  Everything else falls back to ``torch.unique``.
    """
    if (dim == 0 and input.is_cuda and input.dtype == torch.int32 and input.dim() == 2 and input.size(1) == 3
            and input.size(0) > 0 and not return_counts):
        return _unique_coords(input, return_inverse)
    res = torch.unique(input, sorted, return_inverse, return_counts, dim)
    if dim is not None and input.size(dim) == 0:
        shape = list(input.size())
        shape[dim] = 0
        if isinstance(res, torch.Tensor):
            res = res.reshape(shape)
        else:
            res = list(res)
            res[0] = res[0].reshape(shape)
    return res


def _unique_coords(c: torch.Tensor, return_inverse: bool):
    c = c.contiguous()
    lo = c.min(0).values.cpu().numpy().astype(np.int64)
    hi = c.max(0).values.cpu().numpy().astype(np.int64)
    g, words = L.make_grid(lo, hi - lo + 1, 1, c.device)
    st = L.stream()
    L.call("ngs_grid_mark_coords", g, L.ptr(c), c.shape[0], None, 1, 0, st)
    cnt = torch.empty(1, dtype=torch.int64, device=c.device)
    ws = L.grid_finalize(g, words, cnt)
    n = int(cnt.item())
    out = torch.empty((n, 3), dtype=torch.int32, device=c.device)
    L.call("ngs_grid_emit_coords", g, L.ptr(out), st)
    if not return_inverse:
        return out
    inv = torch.empty(c.shape[0], dtype=torch.int64, device=c.device)
    L.call("ngs_grid_lookup", g, L.ptr(c), c.shape[0], L.ptr(inv), st)
    del ws
    return out, inv


class MarchingCubes(torch.autograd.Function):
    """Primal sparse MC with the MeshSDF-style backward to the grid values (``ops.py:9-61``)."""

    @staticmethod
    def forward(ctx, base_coords, sdf_val, bandwidth=1.0):
        tris, vert_ids, src_ids, src_w = ext.marching_cubes_sparse(base_coords, sdf_val)
        unq, tri_idx = torch.unique(vert_ids.view(-1, 4), dim=0, return_inverse=True)
        # each vertex takes the edge data of its first occurrence, whole: the occurrences of an edge
        # may list its two grid samples in either order (with w and 1 - w), so mixing columns of
        # different occurrences would pair a sample with the other one's weight
        n_occ = tri_idx.numel()
        first = torch.full((unq.size(0),), n_occ, dtype=torch.int64, device=vert_ids.device)
        first.scatter_reduce_(0, tri_idx, torch.arange(n_occ, device=vert_ids.device), reduce="amin")
        vertices = tris.view(-1, 3)[first].float()
        vsrc = src_ids.view(-1, 2)[first]
        vw = src_w.view(-1, 1)[first]
        triangles = tri_idx.view(-1, 3)
        normals = compute_normal(vertices, triangles)
        ctx.save_for_backward(normals, vsrc.long(), vw)
        ctx.bandwidth, ctx.res = bandwidth, sdf_val.size()
        return vertices, triangles, normals, unq

    @staticmethod
    def backward(ctx, grad_vert, grad_face, grad_normal, grad_unq):
        normals, vsrc, vw = ctx.saved_tensors
        g = ctx.bandwidth * (grad_vert * normals).sum(-1)
        w = vw[:, 0]
        grid = torch.zeros(ctx.res, device=grad_vert.device).view(-1)
        grid.index_add_(0, vsrc[:, 0], w * g)
        grid.index_add_(0, vsrc[:, 1], (1 - w) * g)
        return None, grid.view(ctx.res), None


marching_cubes_op = MarchingCubes.apply


class ScreenedMultiplication(torch.autograd.Function):
    """Screening products into matrix entries located by a pair-key table (``ops.py:64-82``)."""

    @staticmethod
    def forward(ctx, domain_hash_data, a_val, b_val, a_inds, b_inds, a_lengths, b_lengths, pt_w):
        res = ext.screened_multiplication(domain_hash_data, a_val, b_val, a_inds, b_inds, a_lengths, b_lengths, pt_w)
        ctx.save_for_backward(a_val, b_val, a_inds, b_inds, a_lengths, b_lengths, pt_w)
        ctx.hash_data = domain_hash_data
        return res

    @staticmethod
    def backward(ctx, grad_res):
        a_val, b_val, a_inds, b_inds, a_lengths, b_lengths, pt_w = ctx.saved_tensors
        ga, gb, gw = ext.screened_multiplication_backward(ctx.hash_data, a_val, b_val, a_inds, b_inds, a_lengths,
                                                          b_lengths, pt_w, grad_res.contiguous())
        return None, ga, gb, None, None, None, None, gw


screened_multiplication = ScreenedMultiplication.apply


def compute_normal(vertices: torch.Tensor, triangles: torch.Tensor):
    """Area-weighted vertex normals (``ops.py:85-100``)."""
    e1 = vertices[triangles[:, 1]] - vertices[triangles[:, 0]]
    e2 = vertices[triangles[:, 2]] - vertices[triangles[:, 0]]
    fn = torch.linalg.cross(e1, e2)
    vn = _scatter_sum(fn.repeat_interleave(3, dim=0), triangles.reshape(-1), vertices.size(0))
    return vn / (torch.linalg.norm(vn, dim=-1, keepdim=True) + 1e-6)
