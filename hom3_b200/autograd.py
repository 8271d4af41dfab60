"""torch.autograd binding of the discrete adjoint (h3c_adjoint).

`solve(q0, solver, nsteps)` returns the state after `nsteps` steps of
`solver` started from `q0` at time 0; its backward pass is the library's
discrete adjoint with the forward time steps frozen (the CFL step size is
treated as a constant, as the adjoint does).  Tensors are float64 of shape
[nv][n_cells] in the caller's cell numbering; ghost entries of the gradient
are zero.  The forward pass runs on the GPU through the solver, the backward
pass re-runs the forward with checkpoints and then the adjoint sweep.  CUDA
tensors stay on the device (state, output, cotangent and gradient are copied
device to device); CPU tensors go through host memory.
"""
from __future__ import annotations

import numpy as np
import torch

from .solver import Solver


class _Solve(torch.autograd.Function):
    @staticmethod
    def forward(ctx, q0: torch.Tensor, solver: Solver, nsteps: int, every):
        solver.set_state(_arg(q0), 0)
        solver.reset_time()
        solver.solve(nsteps)
        if q0.is_cuda:
            out = torch.empty(q0.shape, dtype=torch.float64, device=q0.device)
            solver.state(0, out=out)
        else:
            out = torch.from_numpy(solver.state(0))
        ctx.solver, ctx.nsteps, ctx.every = solver, nsteps, every
        ctx.save_for_backward(q0.detach())
        return out

    @staticmethod
    def backward(ctx, grad_out: torch.Tensor):
        (q0,) = ctx.saved_tensors
        s = ctx.solver
        s.set_state(_arg(q0), 0)
        s.reset_time()
        grad, _ = s.adjoint(ctx.nsteps, _arg(grad_out), every=ctx.every)
        if not torch.is_tensor(grad):
            grad = torch.from_numpy(np.ascontiguousarray(grad))
        return grad.to(grad_out.device), None, None, None


def _arg(t: torch.Tensor):
    """A float64 CUDA tensor as it is, anything else as a host numpy array."""
    t = t.detach()
    if t.is_cuda:
        return t.to(torch.float64).contiguous()
    return t.to(torch.float64).contiguous().numpy()


def solve(q0: torch.Tensor, solver: Solver, nsteps: int, every: int = 0) -> torch.Tensor:
    """q_N = solve(q0): nsteps steps of `solver` from q0 at time 0, differentiable in q0."""
    return _Solve.apply(q0, solver, nsteps, every)
