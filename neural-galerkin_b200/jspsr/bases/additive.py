"""Learned (additive) basis: per axis B(x) = sum_u m_u q_u(x) with per-voxel coefficients m
(reference: ``jspsr/bases/additive.py:55-414``).

Galerkin integrals of two such functions are bilinear in their coefficients; the per-pair
forms run in the DDI kernels (``ngs_ddi_forward / _backward``) behind ``DDIFunc``.
"""
from __future__ import annotations

from functools import lru_cache
from typing import List, Union

import numpy as np
import torch

from .abc import BaseBasis
from .additive_components import *          # noqa: F401,F403  (component names usable in basis specs)
from .additive_components import AdditiveComponent, Bezier, Power, Sinusoid, SinPeaks, Product
from . import tables as T
from .. import ext


def _scatter_sum(src, index, n):
    return torch.zeros((n,) + src.shape[1:], dtype=src.dtype, device=src.device).index_add_(0, index, src)


class DDIFunc(torch.autograd.Function):
    """(p, q) = per-pair integrals of basis and basis-gradient products; hand-written adjoint."""

    @staticmethod
    def forward(ctx, source_expanded, target_expanded, rel_pos, f_f_i, df_df_i):
        p, q = ext.ddi_forward(source_expanded, target_expanded, rel_pos, f_f_i, df_df_i)
        ctx.save_for_backward(rel_pos, source_expanded, target_expanded, f_f_i, df_df_i)
        return p, q

    @staticmethod
    def backward(ctx, grad_p, grad_q):
        rel_pos, s, t, ff, dd = ctx.saved_tensors
        gs, gt = ext.ddi_backward(s, t, rel_pos, ff, dd, grad_p.contiguous(), grad_q.contiguous())
        return gs, gt, None, None, None


class EvalFunc(torch.autograd.Function):
    """Per-axis basis values (N, 3) = sum_u q_u(x) m_u; gradient to the coefficients only."""

    @staticmethod
    def forward(ctx, xyz, coeffs, feat_ids, components):
        with torch.no_grad():
            out = 0
            for ci, comp in enumerate(components):
                out = out + comp.evaluate(xyz) * coeffs[feat_ids, 3 * ci:3 * ci + 3]
        ctx.save_for_backward(xyz, feat_ids)
        ctx.components, ctx.n = components, coeffs.size(0)
        return out

    @staticmethod
    def backward(ctx, grad):
        xyz, ids = ctx.saved_tensors
        with torch.no_grad():
            g = [_scatter_sum(grad * comp.evaluate(xyz), ids, ctx.n) for comp in ctx.components]
        return None, torch.cat(g, dim=1), None, None


class EvalDerivFunc(torch.autograd.Function):
    """Per-axis values and derivatives (each (N, 3)); gradient to the coefficients only."""

    @staticmethod
    def forward(ctx, xyz, coeffs, feat_ids, components, stride):
        with torch.no_grad():
            f, d = 0, 0
            for ci, comp in enumerate(components):
                c = coeffs[feat_ids, 3 * ci:3 * ci + 3]
                f = f + comp.evaluate(xyz) * c
                d = d + comp.evaluate_derivative(xyz) * c / stride
        ctx.save_for_backward(xyz, feat_ids)
        ctx.components, ctx.n, ctx.stride = components, coeffs.size(0), stride
        return f, d

    @staticmethod
    def backward(ctx, grad_f, grad_d):
        xyz, ids = ctx.saved_tensors
        with torch.no_grad():
            g = [_scatter_sum(grad_f * comp.evaluate(xyz) + grad_d * comp.evaluate_derivative(xyz) / ctx.stride,
                              ids, ctx.n) for comp in ctx.components]
        return None, torch.cat(g, dim=1), None, None, None


@lru_cache(maxsize=None)
def _pair_tables(ci: str, cj: str, n_mult: int, comps: tuple):
    a, b = comps[0], comps[1]
    return T.component_pair_tables(a, b, n_mult)


class AdditiveBasis(BaseBasis):
    """B(x) = sum_u m_u q_u(x) per axis, m from per-voxel features."""

    def __init__(self, components: List[Union[str, AdditiveComponent]], init_vals: List[float], n_multiples: int = 5):
        super().__init__()
        assert len(components) == len(init_vals)
        self.components = [eval(c, {k: v for k, v in globals().items() if k[0].isupper()}) if isinstance(c, str)
                           else c for c in components]
        self.init_vals = list(init_vals)
        self.n_multiples = n_multiples
        C = len(self.components)
        ff = [[None] * C for _ in range(C)]
        for s, cs in enumerate(self.components):
            for t, ct in enumerate(self.components):
                ff[s][t] = _pair_tables(repr(cs), repr(ct), n_multiples, (cs, ct))
        for m in range(n_multiples):
            self.register_buffer(f"ff_{m}", torch.tensor(np.stack([[ff[s][t][0][m] for t in range(C)]
                                                                   for s in range(C)]), dtype=torch.float32))
            self.register_buffer(f"dfdf_{m}", torch.tensor(np.stack([[ff[s][t][1][m] for t in range(C)]
                                                                     for s in range(C)]), dtype=torch.float32))
        for ci, c in enumerate(self.components):
            f, df, fi, dfi = T.component_tables(c, n_multiples)
            for m in range(n_multiples):
                self.register_buffer(f"f_{ci}_{m}", torch.tensor(f[m], dtype=torch.float32))
                self.register_buffer(f"df_{ci}_{m}", torch.tensor(df[m], dtype=torch.float32))
            for m in range(1, n_multiples):
                self.register_buffer(f"finv_{ci}_{m}", torch.tensor(fi[m - 1], dtype=torch.float32))
                self.register_buffer(f"dfinv_{ci}_{m}", torch.tensor(dfi[m - 1], dtype=torch.float32))

    def _buf(self, name, device):
        b = getattr(self, name)
        return b if b.device == device else b.to(device)

    def feature_to_coefficient(self, feat: torch.Tensor) -> torch.Tensor:
        return feat

    def initialize_feature_value(self, feat: torch.Tensor) -> None:
        assert feat.size(1) == self.get_feature_size()
        for ci, v in enumerate(self.init_vals):
            feat[:, 3 * ci:3 * ci + 3] = v

    def get_feature_size(self) -> int:
        return 3 * len(self.components)

    def evaluate(self, feat, xyz, feat_ids):
        assert feat_ids.size(0) == xyz.size(0), "Input sizes not equal!"
        f = EvalFunc.apply(xyz, self.feature_to_coefficient(feat), feat_ids, self.components)
        return f[:, 0] * f[:, 1] * f[:, 2]

    def evaluate_derivative(self, feat, xyz, feat_ids, stride: int):
        f, d = EvalDerivFunc.apply(xyz, self.feature_to_coefficient(feat), feat_ids, self.components, stride)
        return torch.stack([d[:, 0] * f[:, 1] * f[:, 2], f[:, 0] * d[:, 1] * f[:, 2], f[:, 0] * f[:, 1] * d[:, 2]], 1)

    def integrate_deriv_deriv_product(self, source_feat, target_feat, rel_pos, source_stride: int,
                                      target_stride: int, source_ids, target_ids):
        assert source_stride <= target_stride, "Query must be smaller than reference."
        assert source_ids.size(0) == target_ids.size(0) == rel_pos.size(0), "Input sizes not equal!"
        M = target_stride // source_stride
        m = T.ratio_log2(M)
        assert m < self.n_multiples, f"level ratio {M} beyond the basis tables"
        idx = (rel_pos + 1.5 * M + 0.5).round().long()
        ff = self._buf(f"ff_{m}", rel_pos.device)
        dd = self._buf(f"dfdf_{m}", rel_pos.device)
        R = ff.shape[-1]
        ok = (idx >= 0) & (idx < R)
        idx = idx.clamp(0, R - 1)
        src = self.feature_to_coefficient(source_feat)[source_ids]
        tgt = self.feature_to_coefficient(target_feat)[target_ids]
        p, q = DDIFunc.apply(src, tgt, idx, ff * source_stride, dd / source_stride)
        z = torch.zeros((), device=p.device)
        p, q = torch.where(ok, p, z), torch.where(ok, q, z)
        return q[:, 0] * p[:, 1] * p[:, 2] + p[:, 0] * q[:, 1] * p[:, 2] + p[:, 0] * p[:, 1] * q[:, 2]

    def integrate_const_deriv_product(self, data, target_feat, rel_pos, data_stride: int, target_stride: int,
                                      target_ids):
        assert data.size(0) == target_ids.size(0) == rel_pos.size(0), "Input sizes not equal!"
        dev = rel_pos.device
        if target_stride >= data_stride:
            M = target_stride // data_stride
            idx = (rel_pos + (3 * M - 1) / 2.0).round().long()
            m, fk, dk, scale = T.ratio_log2(M), "f", "df", data_stride
        else:
            M = data_stride // target_stride
            idx = (rel_pos * M + M / 2 + 0.5).round().long()
            m, fk, dk, scale = T.ratio_log2(M), "finv", "dfinv", target_stride
        tgt = self.feature_to_coefficient(target_feat)[target_ids]
        p, q = 0, 0
        for si in range(len(self.components)):
            c = tgt[:, 3 * si:3 * si + 3]
            p = p + c * (self._buf(f"{fk}_{si}_{m}", dev)[idx] * scale)
            q = q + c * self._buf(f"{dk}_{si}_{m}", dev)[idx]
        return data[:, 0] * q[:, 0] * p[:, 1] * p[:, 2] + data[:, 1] * p[:, 0] * q[:, 1] * p[:, 2] + \
            data[:, 2] * p[:, 0] * p[:, 1] * q[:, 2]

    @staticmethod
    def get_bezier():
        return AdditiveBasis([Bezier()], [1.0])

    @staticmethod
    def get_poly_6():
        return AdditiveBasis([Power(p) for p in range(7)], [0.7394, 0.0, -0.6572, 0.0, 0.1461, 0.0, 0.0])
