"""torch.autograd binding of the discrete adjoint (h3c_adjoint).

`solve(q0, solver, nsteps)` returns the state after `nsteps` steps of
`solver` started from `q0` at time 0; its backward pass is the library's
discrete adjoint with the forward time steps frozen (the CFL step size is
treated as a constant, as the adjoint does).  Tensors are float64 of shape
[nv][n_cells] in the caller's cell numbering; ghost entries of the gradient
are zero.  The forward pass runs on the GPU through the solver, the backward
pass re-runs the forward with checkpoints and then the adjoint sweep.
"""
from __future__ import annotations

import numpy as np
import torch

from .solver import Solver


class _Solve(torch.autograd.Function):
    @staticmethod
    def forward(ctx, q0: torch.Tensor, solver: Solver, nsteps: int, every):
        q = q0.detach().to("cpu", torch.float64).contiguous().numpy()
        solver.set_state(q, 0)
        solver.reset_time()
        solver.solve(nsteps)
        out = torch.from_numpy(solver.state(0).copy()).to(q0.device)
        ctx.solver, ctx.nsteps, ctx.every = solver, nsteps, every
        ctx.save_for_backward(q0.detach())
        return out

    @staticmethod
    def backward(ctx, grad_out: torch.Tensor):
        (q0,) = ctx.saved_tensors
        s = ctx.solver
        s.set_state(q0.to("cpu", torch.float64).contiguous().numpy(), 0)
        s.reset_time()
        lam = grad_out.detach().to("cpu", torch.float64).contiguous().numpy()
        grad, _ = s.adjoint(ctx.nsteps, lam, every=ctx.every)
        return torch.from_numpy(np.ascontiguousarray(grad)).to(grad_out.device), None, None, None


def solve(q0: torch.Tensor, solver: Solver, nsteps: int, every: int = 0) -> torch.Tensor:
    """q_N = solve(q0): nsteps steps of `solver` from q0 at time 0, differentiable in q0."""
    return _Solve.apply(q0, solver, nsteps, every)
