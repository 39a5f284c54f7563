"""Reverse-mode AD through the device einsum: the counterpart of the
reference's ChainRules rule for ``einsum`` (src/autodiff.jl:35-44), so that
code differentiated with ``torch.autograd`` runs both passes on this
library's kernels.

The pullback of y = einsum(ixs -> iy)(xs...) for input i is ``einsum_grad``
(src/autodiff.jl:24-30): contract conj(dy) in place of input i into ixs[i]
and conjugate; a real input of a complex contraction takes the real part.
torch's complex-gradient convention (dL/dRe + i dL/dIm) is the one this rule
assumes.  A NestedEinsum is differentiated node by node (every node is one
differentiable einsum), as the reference's AD does through the tree;
``cost_and_gradient`` remains the specialised tree pullback for a scalar
output.
"""
from __future__ import annotations

from typing import Any, Dict, Sequence

import torch

from ._lib import ArgumentError
from .core import EinCode, NestedEinsum, SlicedEinsum, get_size_dict
from .engine import einsum, einsum_grad


class _EinsumFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, code: EinCode, size_dict: Dict[Any, int], *xs):
        ctx.code = code
        ctx.size_dict = size_dict
        ctx.save_for_backward(*xs)
        with torch.no_grad():
            return einsum(code, [x.detach() for x in xs], size_dict)

    @staticmethod
    def backward(ctx, dy):
        xs = [x.detach() for x in ctx.saved_tensors]
        code = ctx.code
        grads = []
        for i in range(len(xs)):
            if ctx.needs_input_grad[2 + i]:
                grads.append(einsum_grad(code.ixs, xs, code.iy, ctx.size_dict, dy, i))
            else:
                grads.append(None)
        return (None, None, *grads)


def ad_einsum(code, xs: Sequence[torch.Tensor], size_dict: Dict[Any, int] | None = None) -> torch.Tensor:
    """``einsum(code, xs)`` recorded for ``torch.autograd``: flat codes are one
    differentiable contraction, NestedEinsum trees one per node.  Inputs are
    CUDA tensors (real or complex); gradients flow to those with
    ``requires_grad``."""
    if isinstance(code, SlicedEinsum):
        code = code.eins   # gradients run unsliced, as in the reference (src/bp.jl:26-28)
    if size_dict is None:
        size_dict = get_size_dict(code.getixsv() if isinstance(code, NestedEinsum) else code.getixs(), xs)
    if isinstance(code, NestedEinsum):
        if code.isleaf:
            raise ArgumentError("a bare leaf is not a contraction")

        def rec(n: NestedEinsum):
            args = [xs[a.tensorindex] if a.isleaf else rec(a) for a in n.args]
            return _EinsumFunction.apply(n.eins, size_dict, *args)

        return rec(code)
    return _EinsumFunction.apply(code, size_dict, *xs)
