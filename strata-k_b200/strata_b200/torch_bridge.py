"""torch.autograd bridge for provenance circuits.

`ProvProbability.apply(p, circuits)` returns the weighted model count of
every compiled query for the FP32 leaf probabilities `p` (a CUDA tensor with
requires_grad), and its backward is the circuits' adjoint kernel: for an
upstream gradient dL/dP it returns dL/dp = Σ_q dL/dP_q · ∂P_q/∂p — the role
`wmc_grad` plays inside a user's autograd Function in the reference's Python
bridge (strata-py/src/lib.rs:436-441, examples/python/train_gnn.py:49-60).
"""
from __future__ import annotations

import torch


class ProvProbability(torch.autograd.Function):
    @staticmethod
    def forward(ctx, p: torch.Tensor, circuits) -> torch.Tensor:
        if p.dtype != torch.float32 or not p.is_cuda:
            raise TypeError("leaf probabilities must be a float32 CUDA tensor")
        p = p.contiguous()
        ctx.circuits = circuits
        ctx.save_for_backward(p)
        return circuits.forward(p)

    @staticmethod
    def backward(ctx, grad_out: torch.Tensor):
        (p,) = ctx.saved_tensors
        seed = grad_out.contiguous().to(torch.float32)
        g32, _ = ctx.circuits.vjp(p, seed)
        return g32.clone(), None


def prov_probability(p: torch.Tensor, circuits) -> torch.Tensor:
    """P(query) for every query of `circuits`, differentiable in `p`."""
    return ProvProbability.apply(p, circuits)
