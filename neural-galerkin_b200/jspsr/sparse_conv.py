"""Sparse convolution as an autograd function, on the tensor-core gather-GEMM of libngs.

Mirrors ``ConvolutionFunction`` of the reference (``models/ascn/utils.py:108-190``): the same
``apply(input, weight, nbmaps, nbsizes, sizes, transposed=False, no_acc=False)`` signature, the
output of ``sizes[1]`` rows (``sizes[0]`` when transposed) and the gradients w.r.t. the input
features and the weights.  Under autocast the reference casts its inputs to float16
(``custom_fwd(cast_inputs=torch.half)``); this function does the same, and also takes bfloat16
and float32 features as given.
"""
from __future__ import annotations

from typing import Tuple

import torch
from torch.amp import custom_bwd, custom_fwd

from . import ext


class ConvolutionFunction(torch.autograd.Function):

    @staticmethod
    @custom_fwd(device_type="cuda", cast_inputs=torch.half)
    def forward(ctx, input: torch.Tensor, weight: torch.Tensor, nbmaps: torch.Tensor, nbsizes: torch.Tensor,
                sizes: Tuple[int, int], transposed: bool = False, no_acc: bool = False) -> torch.Tensor:
        input = input.contiguous()
        weight = weight.contiguous().to(input.dtype)
        nbmaps = nbmaps.int().contiguous()
        nbsizes = nbsizes.int().contiguous()
        rows = sizes[0] if transposed else sizes[1]
        output = torch.zeros(rows, weight.size(-1), dtype=input.dtype, device=input.device)
        ext.sparse_op.convolution_forward_cuda(input, output, weight, nbmaps, nbsizes.cpu(), transposed, no_acc)
        ctx.for_backwards = (input, weight, nbmaps, nbsizes, transposed)
        return output

    @staticmethod
    @custom_bwd(device_type="cuda")
    def backward(ctx, grad_output: torch.Tensor):
        input, weight, nbmaps, nbsizes, transposed = ctx.for_backwards
        grad_input = torch.zeros_like(input)
        grad_weight = torch.zeros_like(weight)
        ext.sparse_op.convolution_backward_cuda(input, grad_input, grad_output.contiguous(), weight, grad_weight,
                                                nbmaps, nbsizes.cpu(), transposed)
        return grad_input, grad_weight, None, None, None, None, None


def sparse_conv(input, weight, nbmaps, nbsizes, sizes, transposed=False, no_acc=False):
    """Functional form of :class:`ConvolutionFunction`."""
    return ConvolutionFunction.apply(input, weight, nbmaps, nbsizes, sizes, transposed, no_acc)
