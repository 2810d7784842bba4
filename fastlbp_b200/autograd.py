"""torch.autograd bridge for gradients through unrolled synchronous sweeps.

`unrolled_beliefs(p, engine, q, sweeps, every)` returns the beliefs after
`sweeps` sweeps from init() as a differentiable function of every factor's
firing probability p (reference factor order; singleton factors' p is the
input prior). The forward pass runs the CUDA engine with checkpoints every
`every` sweeps; the backward pass runs its hand-written adjoint kernels
(flbp_adjoint_backward) backwards through the sweeps, recomputing each
segment from its checkpoint. The engine keeps the state of its last forward
call, so each forward must be followed by its backward before the next
forward on the same engine.
"""

from __future__ import annotations

import numpy as np
import torch

from .api import Engine


class UnrolledBeliefs(torch.autograd.Function):
    @staticmethod
    def forward(ctx, p: torch.Tensor, engine: Engine, q: np.ndarray, sweeps: int, every: int):
        engine.set_factor_probs(p.detach().to("cpu", torch.float64).numpy(), q)
        b = engine.adjoint_forward(int(sweeps), int(every))
        ctx.engine = engine
        return torch.from_numpy(b).to(p.device)

    @staticmethod
    def backward(ctx, grad_b: torch.Tensor):
        gp, _ = ctx.engine.adjoint_backward(grad_b.detach().to("cpu", torch.float64).numpy())
        return torch.from_numpy(gp).to(grad_b.device), None, None, None, None


def unrolled_beliefs(p: torch.Tensor, engine: Engine, q, sweeps: int, every: int) -> torch.Tensor:
    return UnrolledBeliefs.apply(p, engine, np.ascontiguousarray(q, np.float64), sweeps, every)
