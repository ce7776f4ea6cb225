"""torch.autograd.Function over the batched engine.

forward: params -> <O_{c,o}> for every circuit c and observable o (one
persistent launch).  backward: the adjoint vector-Jacobian product with a
single bra sum_o dy_o O_o psi per circuit (the Hamiltonian trick the reference
uses for its vjp, pennylane_lightning/lightning_qubit/lightning_qubit.py:747-772),
one more persistent launch.  Both run on torch's current stream.
"""
from __future__ import annotations

import torch

from .batch import BatchedCircuits


class BatchedExpval(torch.autograd.Function):
    @staticmethod
    def forward(ctx, params: torch.Tensor, engine: BatchedCircuits):
        p = params.detach().to(torch.float64).contiguous()
        out = engine.forward(p)
        ctx.engine = engine
        ctx.save_for_backward(p)
        ctx.in_dtype = params.dtype
        return out.to(params.dtype)

    @staticmethod
    def backward(ctx, dy: torch.Tensor):
        (p,) = ctx.saved_tensors
        grad = ctx.engine.vjp(p, dy.detach().to(torch.float64).contiguous())
        return grad.to(ctx.in_dtype), None


def batched_expval(params: torch.Tensor, engine: BatchedCircuits) -> torch.Tensor:
    """Differentiable expectation values of every circuit of `engine` at `params`."""
    return BatchedExpval.apply(params, engine)
