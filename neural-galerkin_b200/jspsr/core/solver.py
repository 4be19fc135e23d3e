"""Sparse systems and the differentiable solve (reference: ``jspsr/core/solver.py:11-202``)."""
from __future__ import annotations

import time
from functools import cached_property

import torch

from .. import ext
from .pipeline import parse_solver


def _scatter_sum(src, index, n):
    return torch.zeros((n,) + src.shape[1:], dtype=src.dtype, device=src.device).index_add_(0, index.long(), src)


class SparseMatrixStorage:
    """COO matrix with cached CSR / CSC / diagonal views."""

    def __init__(self, a_i, a_j, a_x, dim: int, dim_j: int = None):
        self.a_i, self.a_j, self.a_x = a_i.detach(), a_j.detach(), a_x.detach()
        self.dim_i = dim
        self.dim_j = dim_j or dim
        self.device = self.a_i.device

    def __matmul__(self, v):
        return _scatter_sum(v[self.a_j] * self.a_x, self.a_i, self.dim_i)

    @property
    def shape(self):
        return self.dim_i, self.dim_j

    @classmethod
    def from_dict(cls, data: dict, dim: int, dim_j: int = None):
        return SparseMatrixStorage(data["i"], data["j"], data["x"], dim, dim_j)

    @cached_property
    def _csr(self):
        order = torch.argsort(self.a_i * self.dim_j + self.a_j)
        counts = torch.bincount(self.a_i, minlength=self.dim_i)
        ptr = torch.zeros(self.dim_i + 1, dtype=torch.long, device=self.device)
        ptr[1:] = torch.cumsum(counts, 0)
        return ptr, self.a_j[order], self.a_x[order]

    def csr(self):
        return self._csr

    def csc(self):
        order = torch.argsort(self.a_j * self.dim_i + self.a_i)
        counts = torch.bincount(self.a_j, minlength=self.dim_j)
        ptr = torch.zeros(self.dim_j + 1, dtype=torch.long, device=self.device)
        ptr[1:] = torch.cumsum(counts, 0)
        return ptr, self.a_i[order], self.a_x[order]

    @cached_property
    def _diag(self):
        m = self.a_i == self.a_j
        d = torch.zeros(self.dim_i, device=self.device, dtype=self.a_x.dtype)
        d[self.a_i[m]] = self.a_x[m]
        return d

    def diagonal(self):
        return self._diag

    def dense(self):
        return torch.sparse_coo_tensor(torch.stack([self.a_i, self.a_j]), self.a_x, (self.dim_i, self.dim_j)).to_dense()


class Solver(torch.autograd.Function):
    """x = A^-1 b with the adjoint: grad_b = A^-T grad_x (a second solve with the same SPD A),
    grad_A[i, j] = -grad_b[i] x[j] on A's pattern (``solver.py:76-98``)."""

    @staticmethod
    def forward(ctx, a: SparseMatrixStorage, a_x, b, forward_solver, backward_solver):
        with torch.no_grad():
            x = forward_solver(a=a, b=b.detach())
        ctx.save_for_backward(x, b)
        ctx.a, ctx.backward_solver = a, backward_solver
        return x

    @staticmethod
    def backward(ctx, grad_x):
        x, b = ctx.saved_tensors
        with torch.no_grad():
            grad_b = ctx.backward_solver(ctx.a, grad_x.contiguous())
            grad_a_x = -grad_b[ctx.a.a_i] * x[ctx.a.a_j]
        return None, grad_a_x, grad_b, None, None


def _pcg_solver(spec):
    def run(a: SparseMatrixStorage, b: torch.Tensor):
        if b.size(0) == 0:
            return torch.zeros_like(b)
        ptr, cols, vals = a.csr()
        dinv = (1.0 / a.diagonal()).float()
        mode = spec.mode
        if spec.name == "pcg":
            x, _ = ext.solve_pcg_diag(ptr, cols.int(), vals.float(), b.float(), dinv, spec.tol, spec.maxiter,
                                      spec.res_fix)
            return x
        if spec.name == "plain-fp64":
            mode = 2
        x, _ = ext._pcg(ptr, cols.int(), vals.float(), b.float(), dinv, spec.tol, spec.maxiter, False, mode,
                        b64=b.double().contiguous(), ax64=vals.double().contiguous())
        return x
    return run


def solve_cholmod(a: SparseMatrixStorage, b: torch.Tensor):
    """The reference's direct solve (cuSOLVER Cholesky, ``solver.py:148-164``): here an FP64 PCG to 1e-12."""
    if b.size(0) == 0:
        return torch.zeros_like(b)
    return _pcg_solver(parse_solver("pcg-fp64@tol=1e-12"))(a, b)


def solve_mixed(a, b, fast_solver, fallback_solver, tol: float = 0.01, name: str = None):
    """Fast solve, re-solved with the fallback when the residual is above tol (``solver.py:167-177``)."""
    if b.size(0) == 0:
        return torch.zeros_like(b)
    x = fast_solver(a, b)
    if float(torch.linalg.norm(a @ x - b)) > tol:
        x = fallback_solver(a, b)
    return x


def _parse_solver_type(solver_type: str):
    """``name@key=value@...`` -> (name, config); values are parsed, never ``eval``-ed."""
    spec = parse_solver(solver_type)
    return spec.name, spec


def solve_pcg(a: SparseMatrixStorage, b: torch.Tensor, pcg_conf):
    return _pcg_solver(pcg_conf)(a, b)


def solve_sparse(a_i, a_j, a_x, b, solver_type: str, verbose_str: str = None):
    """Differentiable solve of A x = b for COO A (``solver.py:101-145``)."""
    if verbose_str is not None:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
    a = SparseMatrixStorage(a_i, a_j, a_x, dim=b.size(0))
    name = solver_type.split("@")[0]
    if name == "mixed":
        fast = _pcg_solver(parse_solver("pcg@tol=1e-4@maxiter=1000"))
        fwd = lambda a, b: solve_mixed(a, b, fast, solve_cholmod, tol=1e-2)     # noqa: E731
        x = Solver.apply(a, a_x, b, fwd, solve_cholmod)
    elif name == "cholmod":
        x = Solver.apply(a, a_x, b, solve_cholmod, solve_cholmod)
    else:
        fn = _pcg_solver(parse_solver(solver_type))
        x = Solver.apply(a, a_x, b, fn, fn)
    if verbose_str is not None:
        torch.cuda.synchronize()
        with torch.no_grad():
            resid = float(torch.linalg.norm(a @ x - b))
        print(verbose_str.format(time=time.perf_counter() - t0, residual=resid))
    return x
