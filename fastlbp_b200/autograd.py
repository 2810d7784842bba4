"""torch.autograd bridge for gradients through unrolled synchronous sweeps.

`unrolled_beliefs(p, engine, q, sweeps, every)` returns the beliefs after
`sweeps` sweeps from init() as a differentiable function of every factor's
firing probability p (reference factor order; singleton factors' p is the
input prior). The forward pass runs the CUDA engine with checkpoints every
`every` sweeps; the backward pass runs its hand-written adjoint kernels
(flbp_adjoint_backward) backwards through the sweeps, recomputing each
segment from its checkpoint. The engine keeps the state of its last forward
call, so each forward must be followed by its backward before the next
forward on the same engine. With p on the engine's CUDA device, beliefs and
gradients stay on the device (flbp_get_beliefs_device,
flbp_adjoint_backward_device), and so does p: flbp_set_factor_probs_device
takes it from device memory (q too, when given as a CUDA tensor; a host q
is copied to the device once per call).
"""

from __future__ import annotations

import numpy as np
import torch

from .api import Engine


class UnrolledBeliefs(torch.autograd.Function):
    @staticmethod
    def forward(ctx, p: torch.Tensor, engine: Engine, q, sweeps: int, every: int):
        ctx.engine = engine
        ctx.on_device = p.is_cuda
        if p.is_cuda:
            pd = p.detach().to(torch.float64).contiguous()
            qd = torch.as_tensor(q, dtype=torch.float64, device=p.device).contiguous()
            torch.cuda.current_stream(p.device).synchronize()  # the engine's stream does not wait for torch's
            engine.set_factor_probs_device(pd, qd)
            engine.adjoint_forward(int(sweeps), int(every), fetch=False)
            b = torch.empty(engine.n_vars, dtype=torch.float64, device=p.device)
            engine.beliefs_device(b)
            return b
        qh = q.detach().to("cpu", torch.float64).numpy() if isinstance(q, torch.Tensor) else q
        engine.set_factor_probs(p.detach().to("cpu", torch.float64).numpy(), qh)
        return torch.from_numpy(engine.adjoint_forward(int(sweeps), int(every)))

    @staticmethod
    def backward(ctx, grad_b: torch.Tensor):
        if ctx.on_device:
            g = grad_b.detach().to(torch.float64).contiguous()
            gp = torch.empty(ctx.engine.n_factors, dtype=torch.float64, device=g.device)
            ctx.engine.adjoint_backward_device(g, gp)
            return gp, None, None, None, None
        gp, _ = ctx.engine.adjoint_backward(grad_b.detach().to("cpu", torch.float64).numpy(), want_q=False)
        return torch.from_numpy(gp), None, None, None, None


def unrolled_beliefs(p: torch.Tensor, engine: Engine, q, sweeps: int, every: int) -> torch.Tensor:
    if not isinstance(q, torch.Tensor):
        q = np.ascontiguousarray(q, np.float64)
    return UnrolledBeliefs.apply(p, engine, q, sweeps, every)
