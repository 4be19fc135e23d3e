"""Galerkin assembly and solve of the multi-level screened-Poisson system for any basis, with its
adjoint, over a batch of shapes (reference: ``jspsr/core/reconstructor.py:79-195`` for the system,
``jspsr/core/solver.py:76-98`` for the adjoint rule).

The system of level d (coarse to fine, every coarser solution known):

    A_d x_d = b_d,   A_d = K_d + G_dd,
    K_d[i, j]   = int grad B_i . grad B_j                        (stiffness, 5^3 stencil)
    G_de[i, j]  = sf_d sum_p a_p B_i(p) B_j(p)                   (screening Gram, sf_d = 4^-d)
    b_d[i]      = sum_data -int grad B_i . n  +  sf_d sum_p (a delta)_p B_i(p)
                  - sum_{e coarser} (K_de + G_de) x_e            (cross-level correction)

Storage is libngs': the stencil CSR of each level comes from the level's rank bitmap
(``ngs_stencil_count / _fill``); the basis integrals of every CSR slot are evaluated for the slot's
(row, column) pair and written straight into the CSR values; the Gram is added in place from the
points grouped by cell (``ngs_screen_gram_grouped``); each level is solved by the persistent PCG,
the levels of all shapes of a batch in one launch (``ngs_pcg_solve_batch``).

``GalerkinSolve`` is one autograd function over all of it.  Its backward is the adjoint of the
whole coarse-to-fine chain, written out:

    for d from the finest level to the coarsest:
        lambda_d = A_d^-1 gx_d                                    (PCG on the same CSR, batched)
        gx_e    -= (K_de + G_de)^T lambda_d   for every coarser e (the correction's transpose)
    dL/dA_d[i, j] = -lambda_d[i] x_d[j],  dL/db_d = lambda_d

and then, term by term, the local derivatives of the assembly: the stiffness and cross-level
integrals of every pair (the basis' own pair kernels, DDI for the learned bases), the point values
B_i(p) through dL/dB_i(p) = -sf_d a_p (lambda_i chi_x(p) + x_i chi_lambda(p)) + ... (closed forms
below), and the normal data through the divergence integrals.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from types import SimpleNamespace
from typing import Dict, List, Optional

import numpy as np
import torch

from .. import _lib as L
from ..bases import tables as TB
from ._hash_backend import VoxelLevel
from .pipeline import Reconstruction, parse_solver


# ----------------------------------------------------------------------------- geometry of one level
@dataclass
class LevelGeometry:
    """Everything of one level that depends on positions only."""
    depth: int
    stride: int
    level: VoxelLevel
    n: int
    masks: torch.Tensor = None        # int32 [n, 4]: which of the 125 stencil offsets exist
    rowptr: torch.Tensor = None       # int64 [n + 1]
    cols: torch.Tensor = None         # int32 [nnz]
    diag_slot: torch.Tensor = None    # int64 [n]
    slot_row: torch.Tensor = None     # int64 [nnz]: row of every CSR slot
    slot_rel: torch.Tensor = None     # float [nnz, 3]: column centre - row centre, in voxels
    nnz: int = 0
    band: int = 0                     # bound on |column - row| (the solver's shared-memory window)
    pt_rows: torch.Tensor = None      # int32 [N, 27]: the basis functions touching each screening point
    pt_local: torch.Tensor = None     # float [N, 27, 3]: the point relative to each of their centres, voxels
    group: tuple = None               # (cell keys sorted, point order): the Gram's point grouping
    cross: Dict[int, tuple] = field(default_factory=dict)   # coarser e -> (i, j, rel) pairs
    data: Dict[int, tuple] = field(default_factory=dict)    # data level -> (data ids, target ids, rel)


def _stencil(geo: LevelGeometry):
    st, dev = L.stream(), geo.level.device
    n = geo.n
    geo.masks = torch.empty((n, 4), dtype=torch.int32, device=dev)
    counts = torch.empty(n, dtype=torch.int64, device=dev)
    L.call("ngs_stencil_count", geo.level.grid, L.ptr(geo.level.coords), n, L.ptr(geo.masks), L.ptr(counts), st)
    geo.rowptr = torch.empty(n + 1, dtype=torch.int64, device=dev)
    L.scan(counts, out=geo.rowptr[:n], total=geo.rowptr[n:])
    # the non-zero count and a bound on |column - row| from the rank bitmap: one synchronisation
    if n > 0:
        lvb = SimpleNamespace(grid=geo.level.grid, words=geo.level.words, n=n)
        host = torch.stack([geo.rowptr[n], Reconstruction._row_span_bound(lvb)]).cpu()
        geo.nnz, geo.band = int(host[0]), int(host[1])
    else:
        geo.nnz, geo.band = 0, 0
    geo.cols = torch.empty(geo.nnz, dtype=torch.int32, device=dev)
    scratch = torch.empty(geo.nnz, dtype=torch.float64, device=dev)
    geo.diag_slot = torch.empty(n, dtype=torch.int64, device=dev)
    st125 = L.device_table(("stencil125", geo.stride), lambda s=geo.stride: TB.stencil125(s), dev)
    L.call("ngs_stencil_fill", geo.level.grid, L.ptr(geo.level.coords), n, L.ptr(geo.masks), L.ptr(geo.rowptr),
           L.ptr(st125), L.ptr(geo.cols), L.ptr(scratch), L.ptr(geo.diag_slot), st)
    geo.slot_row = torch.repeat_interleave(torch.arange(n, device=dev), counts)
    c = geo.level.coords
    geo.slot_rel = ((c[geo.cols.long()] - c[geo.slot_row]) // geo.stride).float()


def _point_basis(geo: LevelGeometry, xyz: torch.Tensor, voxel_size: float):
    """The 27 basis functions around every screening point (``ngs_point_basis`` rows, lexicographic
    offsets) and the point's position relative to each of their centres in voxel units."""
    st, dev, n = L.stream(), xyz.device, xyz.shape[0]
    inv = L.f32_inv(voxel_size)
    geo.pt_rows = torch.empty((n, 27), dtype=torch.int32, device=dev)
    phi = torch.empty((n, 27), dtype=torch.float32, device=dev)
    L.call("ngs_point_basis", geo.level.grid, L.ptr(xyz), n, np.float32(inv), float(voxel_size), L.ptr(geo.pt_rows),
           L.ptr(phi), st)
    s = geo.stride
    pos = xyz.double() / voxel_size - 0.5
    snap = torch.floor((xyz * np.float32(inv) - 0.5 + 0.5) / s) * s                 # the fp32 lattice snap
    k = torch.arange(-1, 2, device=dev, dtype=torch.float64)
    off = torch.cartesian_prod(k, k, k)                                              # [27, 3] lexicographic
    geo.pt_local = ((pos[:, None, :] - snap.double()[:, None, :] - off[None] * s - 0.5 * (s - 1)) / s).float()
    keys = torch.empty(n, dtype=torch.int64, device=dev)
    L.call("ngs_point_cell_keys", L.ptr(geo.pt_rows), n, L.ptr(keys), st)
    skeys, order = torch.sort(keys)
    geo.group = (skeys, order)


@dataclass
class ShapeGeometry:
    """One shape: per-level geometry plus the screening points and their weights."""
    levels: Dict[int, LevelGeometry]
    order: List[int]                       # solve order: coarsest first
    xyz: Optional[torch.Tensor]            # screening points (or None: no screening)
    alpha: Optional[torch.Tensor]          # per-point screening weight a_p
    alpha_delta: Optional[torch.Tensor]    # per-point (a delta)_p
    data_levels: List[int]                 # levels carrying normal data
    voxel_size: float
    stats: Dict[int, dict] = field(default_factory=dict)   # last forward solve of every level

    @staticmethod
    def build(tree, branch, start_depth: int, end_depth: int, data_levels, screen_xyz, screen_alpha, screen_delta,
              basis_range: int):
        order = list(range(start_depth, end_depth - 1, -1))
        screen = screen_xyz is not None and (isinstance(screen_alpha, torch.Tensor) or screen_alpha > 0)
        n = screen_xyz.shape[0] if screen else 0
        dev = tree.device
        xyz = screen_xyz.detach().float().contiguous() if screen else None
        alpha = alpha_delta = None
        if screen:
            a = screen_alpha if isinstance(screen_alpha, torch.Tensor) else torch.full((n,), float(screen_alpha), device=dev)
            dl = screen_delta if isinstance(screen_delta, torch.Tensor) else torch.full((n,), float(screen_delta), device=dev)
            alpha = a.detach().float().contiguous()
            alpha_delta = (a * dl).detach().float().contiguous()
        hier = tree._get_branch(branch)
        levels = {}
        for d in order:
            lv = hier.level(d)
            geo = LevelGeometry(depth=d, stride=hier.get_stride(d), level=lv, n=len(lv))
            _stencil(geo)
            if screen:
                _point_basis(geo, xyz, tree.voxel_size)
            for e in order:
                if e > d:
                    i, j, rel, _ = tree.get_neighbours(d, e, target_range=2 * basis_range - 1, branch=branch)
                    geo.cross[e] = (i, j, rel)
            for dd in data_levels:
                v, t, rel, _ = tree.get_neighbours(dd, d, basis_range, branch)
                geo.data[dd] = (v, t, rel)
            levels[d] = geo
        return ShapeGeometry(levels, order, xyz, alpha, alpha_delta, list(data_levels), tree.voxel_size)


# ----------------------------------------------------------------------------- basis terms (torch)
def _phi(basis, feat, geo: LevelGeometry):
    """B_i(p) for the 27 slots of every point ([N, 27], 0 where the slot has no voxel)."""
    rows = geo.pt_rows.long()
    valid = rows >= 0
    ids = rows.clamp(min=0).reshape(-1)
    val = basis.evaluate(feat=feat, xyz=geo.pt_local.reshape(-1, 3), feat_ids=ids).reshape(rows.shape)
    return torch.where(valid, val, torch.zeros((), device=val.device, dtype=val.dtype))


def _slot_stiffness(basis, feat, geo: LevelGeometry):
    return basis.integrate_deriv_deriv_product(source_feat=feat, target_feat=feat, rel_pos=geo.slot_rel,
                                               source_stride=geo.stride, target_stride=geo.stride,
                                               source_ids=geo.slot_row, target_ids=geo.cols.long())


def _cross_stiffness(basis, feat_d, feat_e, geo_d: LevelGeometry, geo_e: LevelGeometry):
    i, j, rel = geo_d.cross[geo_e.depth]
    return basis.integrate_deriv_deriv_product(source_feat=feat_d, target_feat=feat_e, rel_pos=rel,
                                               source_stride=geo_d.stride, target_stride=geo_e.stride,
                                               source_ids=i, target_ids=j)


def _divergence(basis, nd, feat, geo_d: LevelGeometry, data_stride: int, dd: int):
    """-int grad B_t . n_v of every (data voxel v, target t) pair."""
    v, t, rel = geo_d.data[dd]
    return basis.integrate_const_deriv_product(data=-nd[v], target_feat=feat, rel_pos=rel, data_stride=data_stride,
                                               target_stride=geo_d.stride, target_ids=t)


def _point_field(phi, rows, x):
    """chi(p) = sum over the 27 slots of x[row] B_row(p)."""
    r = rows.long()
    return (phi * torch.where(r >= 0, x[r.clamp(min=0)], torch.zeros((), device=x.device, dtype=x.dtype))).sum(1)


def _scatter_points(weights, rows, n):
    """sum over points and slots of weights[p, k] into row rows[p, k]."""
    r = rows.long().reshape(-1)
    ok = r >= 0
    return torch.zeros(n, dtype=weights.dtype, device=weights.device).index_add_(0, r[ok], weights.reshape(-1)[ok])


# ----------------------------------------------------------------------------- systems and solves
@dataclass
class LevelSystem:
    vals64: torch.Tensor
    vals32: torch.Tensor
    inv_diag: torch.Tensor
    phi: Optional[torch.Tensor]


def _finish(geo: LevelGeometry, vals64: torch.Tensor) -> LevelSystem:
    vals32 = torch.empty(geo.nnz, dtype=torch.float32, device=vals64.device)
    inv_diag = torch.empty(geo.n, dtype=torch.float32, device=vals64.device)
    L.call("ngs_finish_system", L.ptr(vals64), geo.nnz, L.ptr(geo.diag_slot), geo.n, L.ptr(vals32), L.ptr(inv_diag),
           L.stream())
    return LevelSystem(vals64, vals32, inv_diag, None)


def solve_levels(jobs, spec):
    """Solve independent systems ``jobs = [(geo, system, b64)]`` with the persistent PCG of the
    solver spec; systems go to the device in batches that fit one cooperative launch."""
    dev = jobs[0][2].device
    lib = L.load()
    mode = spec.mode if spec.mode is not None else L.PCG_FP64
    outs, items, keep = [], [], []
    for geo, sysm, b in jobs:
        x64 = torch.empty(geo.n, dtype=torch.float64, device=dev)
        x32 = torch.empty(geo.n, dtype=torch.float32, device=dev)
        info = torch.zeros(4, dtype=torch.int64, device=dev)
        resid = torch.zeros(2, dtype=torch.float64, device=dev)
        b = b.contiguous()
        b32 = b.float()
        it = L.PcgBatchItem()
        s = it.sys
        s.n, s.nnz = geo.n, geo.nnz
        s.rowptr, s.cols, s.inv_diag = geo.rowptr.data_ptr(), geo.cols.data_ptr(), sysm.inv_diag.data_ptr()
        s.vals32, s.vals64 = sysm.vals32.data_ptr(), sysm.vals64.data_ptr()
        s.b32, s.b64, s.x32, s.x64 = b32.data_ptr(), b.data_ptr(), x32.data_ptr(), x64.data_ptr()
        s.band = geo.band
        c = it.cfg
        c.mode, c.max_iter, c.tol, c.res_fix = mode, spec.maxiter, spec.tol, int(spec.res_fix)
        c.replace_every, c.blocks, c.timeout_s = spec.replace, 0, spec.timeout
        ws_bytes = lib.ngs_pcg_workspace_bytes(geo.n, mode)
        ws = torch.empty(max(ws_bytes, 8), dtype=torch.uint8, device=dev)
        it.ws, it.ws_bytes = ws.data_ptr(), ws_bytes
        it.info_dev, it.resid_dev = info.data_ptr(), resid.data_ptr()
        items.append(it)
        keep.append((b, b32, ws))
        outs.append((x64, x32, info, resid))
    cap = lib.ngs_pcg_block_capacity(mode)
    st = L.stream()
    group, used = [], 0
    for it in items:
        need = lib.ngs_pcg_blocks(it.sys.n, it.sys.nnz, mode)
        if group and (used + need > cap or len(group) == L.PCG_BATCH_MAX):
            arr = (L.PcgBatchItem * len(group))(*group)
            L.call("ngs_pcg_solve_batch", arr, len(group), st)
            group, used = [], 0
        group.append(it)
        used += need
    if group:
        arr = (L.PcgBatchItem * len(group))(*group)
        L.call("ngs_pcg_solve_batch", arr, len(group), st)
    status = torch.cat([torch.stack([o[2].double() for o in outs]), torch.stack([o[3] for o in outs])], 1).cpu().numpy()
    for k, row in enumerate(status):
        if row[1] not in (L.NGS_OK, L.NGS_ERR_NOT_CONVERGED) or (row[1] == L.NGS_ERR_NOT_CONVERGED and spec.maxiter < 0):
            raise L.NgsError(int(row[1]), f"Galerkin level solve {k}")
    del keep
    # the reference mode solves in FP32 throughout and writes only the FP32 solution
    sols = [o[1].double() if mode == L.PCG_REFERENCE else o[0] for o in outs]
    return sols, status


# ----------------------------------------------------------------------------- forward of one shape, one level
def _assemble_level(basis, shape: ShapeGeometry, d: int, feats, normal_data, x_coarse):
    """System and right-hand side of level d given the coarser solutions (no autograd)."""
    geo = shape.levels[d]
    sf = 0.25 ** d
    dev = geo.level.device
    feat_d = feats.get(d)
    K = _slot_stiffness(basis, feat_d, geo)
    vals64 = K.double().contiguous()
    b = torch.zeros(geo.n, dtype=torch.float64, device=dev)
    for dd in shape.data_levels:
        part = _divergence(basis, normal_data[dd], feat_d, geo, shape_stride(shape, dd), dd)
        b.index_add_(0, geo.data[dd][1], part.double())
    phi = None
    if shape.xyz is not None:
        phi = _phi(basis, feat_d, geo).float().contiguous()
        keys, order = geo.group
        L.call("ngs_screen_gram_grouped", L.ptr(geo.pt_rows), L.ptr(phi), shape.xyz.shape[0], L.ptr(shape.alpha),
               L.ptr(order), L.ptr(keys), L.ptr(geo.masks), L.ptr(geo.rowptr), sf, L.ptr(vals64), L.stream())
        b += sf * _scatter_points(phi.double() * shape.alpha_delta.double()[:, None], geo.pt_rows, geo.n)
    for e, (xe, phi_e) in x_coarse.items():
        geo_e = shape.levels[e]
        a = _cross_stiffness(basis, feat_d, feats.get(e), geo, geo_e)
        i, j, _ = geo.cross[e]
        b.index_add_(0, i, -(a.double() * xe[j]))
        if phi is not None:
            chi_e = _point_field(phi_e.double(), geo_e.pt_rows, xe)
            b -= sf * _scatter_points(phi.double() * (shape.alpha.double() * chi_e)[:, None], geo.pt_rows, geo.n)
    sysm = _finish(geo, vals64)
    sysm.phi = phi
    return sysm, b


def shape_stride(shape: ShapeGeometry, d: int) -> int:
    return 1 << d


# ----------------------------------------------------------------------------- the autograd function
class GalerkinSolve(torch.autograd.Function):
    """Solutions of every level of every shape; inputs per shape: basis features per level and
    normal data per data level (``None`` where absent).  ``spec`` is the parsed solver string."""

    @staticmethod
    def forward(ctx, basis, shapes, spec, layout, *tensors):
        feats, normals = _unflatten(layout, tensors)
        S = len(shapes)
        systems = [dict() for _ in range(S)]
        xs = [dict() for _ in range(S)]
        with torch.no_grad():
            depths = shapes[0].order
            for d in depths:
                jobs = []
                for s in range(S):
                    coarse = {e: (xs[s][e], systems[s][e].phi) for e in xs[s]}
                    sysm, b = _assemble_level(basis, shapes[s], d, feats[s], normals[s], coarse)
                    systems[s][d] = sysm
                    jobs.append((shapes[s].levels[d], sysm, b))
                sol, status = solve_levels(jobs, spec)
                for s in range(S):
                    xs[s][d] = sol[s]
                    shapes[s].stats[d] = dict(iters=int(status[s][0]), status=int(status[s][1]), resid=float(status[s][4]),
                                              bnorm=float(status[s][5]))
        ctx.basis, ctx.shapes, ctx.spec, ctx.layout = basis, shapes, spec, layout
        ctx.systems, ctx.xs = systems, xs
        ctx.save_for_backward(*[t for t in tensors if t is not None])
        ctx.has = [t is not None for t in tensors]
        out = []
        for s in range(S):
            for d in shapes[s].order:
                out.append(xs[s][d].float())
        return tuple(out)

    @staticmethod
    def backward(ctx, *grads):
        basis, shapes, spec, layout = ctx.basis, ctx.shapes, ctx.spec, ctx.layout
        saved = iter(ctx.saved_tensors)
        tensors = [next(saved) if h else None for h in ctx.has]
        feats, normals = _unflatten(layout, tensors)
        S = len(shapes)
        gi = iter(grads)
        gx = [dict() for _ in range(S)]
        for s in range(S):
            for d in shapes[s].order:
                g = next(gi)
                gx[s][d] = (g.double() if g is not None else
                            torch.zeros(shapes[s].levels[d].n, dtype=torch.float64, device=shapes[s].levels[d].level.device))
        lam = [dict() for _ in range(S)]
        # adjoint solves, finest level first; each pushes its correction's transpose to the coarser levels
        with torch.no_grad():
            for d in reversed(shapes[0].order):
                jobs = [(shapes[s].levels[d], ctx.systems[s][d], gx[s][d]) for s in range(S)]
                sol, _ = solve_levels(jobs, spec)
                for s in range(S):
                    lam[s][d] = sol[s]
                    shape, geo = shapes[s], shapes[s].levels[d]
                    sf = 0.25 ** d
                    phi_d = ctx.systems[s][d].phi
                    for e in geo.cross:
                        a = _cross_stiffness(basis, feats[s].get(d), feats[s].get(e), geo, shape.levels[e])
                        i, j, _ = geo.cross[e]
                        gx[s][e].index_add_(0, j, -(a.double() * lam[s][d][i]))
                        if phi_d is not None:
                            geo_e = shape.levels[e]
                            chi_l = _point_field(phi_d.double(), geo.pt_rows, lam[s][d])
                            gx[s][e] -= sf * _scatter_points(ctx.systems[s][e].phi.double() *
                                                             (shape.alpha.double() * chi_l)[:, None],
                                                             geo_e.pt_rows, geo_e.n)
        # local derivatives of the assembly, term by term
        grad_tensors = [None] * len(tensors)
        need = [t is not None and ctx.needs_input_grad[4 + k] for k, t in enumerate(tensors)]
        if not any(need):
            return (None, None, None, None) + tuple(grad_tensors)
        with torch.enable_grad():
            for s in range(S):
                _shape_vjp(basis, shapes[s], layout, s, feats[s], normals[s], ctx.xs[s], lam[s], ctx.systems[s],
                           need, grad_tensors)
        return (None, None, None, None) + tuple(grad_tensors)


def _shape_vjp(basis, shape: ShapeGeometry, layout, s, feats, normals, xs, lam, systems, need, grad_tensors):
    """dL/d(features) and dL/d(normal data) of one shape from its solutions and adjoints."""
    fidx, nidx = layout[s]
    f_in = {d: (feats[d].detach().requires_grad_(True) if need[fidx[d]] else feats[d].detach())
            for d in feats if feats[d] is not None}
    n_in = {d: (normals[d].detach().requires_grad_(True) if need[nidx[d]] else normals[d].detach())
            for d in normals if normals[d] is not None}
    outs, gouts = [], []
    for d in shape.order:
        geo = shape.levels[d]
        sf = 0.25 ** d
        x, l = xs[d], lam[d]
        fd = f_in.get(d)
        learned = fd is not None and fd.requires_grad
        # stiffness of every slot (i, j): dL/dK = -lambda_i x_j
        if learned:
            outs.append(_slot_stiffness(basis, fd, geo))
            gouts.append((-(l[geo.slot_row] * x[geo.cols.long()])).float())
        # divergence terms: dL/db_t = lambda_t
        for dd in shape.data_levels:
            nd = n_in[dd]
            if not (learned or nd.requires_grad):
                continue
            outs.append(_divergence(basis, nd, fd, geo, shape_stride(shape, dd), dd))
            gouts.append(l[geo.data[dd][1]].float())
        # cross-level stiffness of every pair: dL/dK_de = -lambda_d[i] x_e[j]
        for e in geo.cross:
            fe = f_in.get(e)
            if not (learned or (fe is not None and fe.requires_grad)):
                continue
            i, j, _ = geo.cross[e]
            outs.append(_cross_stiffness(basis, fd, fe, geo, shape.levels[e]))
            gouts.append((-(l[i] * xs[e][j])).float())
        # point values B_i(p) of this level: screening Gram (same level and towards every coarser
        # level), screening target, and the finer levels' Gram towards this one
        if shape.xyz is not None and learned:
            a = shape.alpha.double()
            phi_d = systems[d].phi.double()
            chi_x = _point_field(phi_d, geo.pt_rows, x)
            chi_l = _point_field(phi_d, geo.pt_rows, l)
            rows = geo.pt_rows.long().clamp(min=0)
            lr, xr = l[rows], x[rows]
            # same level: -sf a_p (lambda_i chi_x(p) + x_i chi_lambda(p)); target: sf (a delta)_p lambda_i
            gphi = -sf * a[:, None] * (lr * chi_x[:, None] + xr * chi_l[:, None]) + \
                sf * shape.alpha_delta.double()[:, None] * lr
            # rows of level d against coarser e: -sf a_p lambda_i chi_{x_e}(p)
            for e in geo.cross:
                chi_xe = _point_field(systems[e].phi.double(), shape.levels[e].pt_rows, xs[e])
                gphi = gphi - sf * a[:, None] * lr * chi_xe[:, None]
            # columns of level d from every finer f: -sf_f a_p x_j chi_{lambda_f}(p)
            for f in shape.order:
                if f < d:
                    geo_f = shape.levels[f]
                    chi_lf = _point_field(systems[f].phi.double(), geo_f.pt_rows, lam[f])
                    gphi = gphi - (0.25 ** f) * a[:, None] * xr * chi_lf[:, None]
            gphi = torch.where(geo.pt_rows >= 0, gphi, torch.zeros((), dtype=gphi.dtype, device=gphi.device))
            outs.append(_phi(basis, fd, geo))
            gouts.append(gphi.float())
    inputs = [t for t in list(f_in.values()) + list(n_in.values()) if t.requires_grad]
    if not inputs or not outs:
        return
    grads = torch.autograd.grad(outs, inputs, grad_outputs=gouts, allow_unused=True)
    gmap = dict(zip([id(t) for t in inputs], grads))
    for d, t in f_in.items():
        if t.requires_grad and gmap.get(id(t)) is not None:
            grad_tensors[fidx[d]] = gmap[id(t)]
    for d, t in n_in.items():
        if t.requires_grad and gmap.get(id(t)) is not None:
            grad_tensors[nidx[d]] = gmap[id(t)]


def _flatten(feats_list, normals_list, depths):
    """Flat tensor list (features per level, then normal data per level, per shape) and its layout."""
    tensors, layout = [], []
    for feats, normals in zip(feats_list, normals_list):
        fidx, nidx = {}, {}
        for d in depths:
            fidx[d] = len(tensors)
            tensors.append(feats.get(d) if feats is not None else None)
        for d in depths:
            nidx[d] = len(tensors)
            tensors.append(normals.get(d))
        layout.append((fidx, nidx))
    return tensors, layout


def _unflatten(layout, tensors):
    feats, normals = [], []
    for fidx, nidx in layout:
        feats.append({d: tensors[k] for d, k in fidx.items()})
        normals.append({d: tensors[k] for d, k in nidx.items() if tensors[k] is not None})
    return feats, normals


def galerkin_solve(basis, shapes: List[ShapeGeometry], feats_list, normals_list, solver: str = "cholmod"):
    """Solve every level of every shape; returns per shape a dict level -> solution (float32),
    differentiable w.r.t. the features and the normal data."""
    spec = parse_solver(solver)
    depths = shapes[0].order
    for sh in shapes:
        assert sh.order == depths, "every shape of a batch needs the same levels"
    tensors, layout = _flatten(feats_list, normals_list, depths)
    outs = GalerkinSolve.apply(basis, shapes, spec, layout, *tensors)
    res, k = [], 0
    for sh in shapes:
        res.append({d: outs[k + i] for i, d in enumerate(sh.order)})
        k += len(sh.order)
    return res
