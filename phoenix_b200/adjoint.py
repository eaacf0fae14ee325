"""Gradients of an RK4 trajectory through torch.autograd.

`evolve(solver, pump, psi0, n0, iterations, potential=V)` runs `iterations`
RK4 iterations of the GP equation with reservoir in phoenix_b200's kernels
and returns the final (psi, n) as torch tensors that carry a backward: the
library's adjoint (phx_adjoint_forward / phx_adjoint_backward) recomputes
the trajectory from checkpoints kept every ceil(sqrt(iterations))
iterations and applies hand-written vector-Jacobian products of the RK4
stages, giving dL/dP (pump), dL/dV (potential), dL/dpsi_0 and dL/dn_0.  The
reference has no adjoint; the forward map is its RK4 (runge_kutta.cu:74-94)
bit for bit, with the pump and the potential entering as in gp_scalar
(include/kernel/kernel_gp_compute.cuh:86-98).

The solver is configured by its SystemParameters (scalar, RK4, periodic on
both axes, one pump group, at most one potential group, constant envelopes,
no filter, no noise).  A solver serves one forward/backward pair at a time.
"""
from __future__ import annotations

import torch

from .solver import Solver


class _Trajectory(torch.autograd.Function):
    @staticmethod
    def forward(ctx, pump, psi0, n0, potential, solver: Solver, iterations: int, checkpoint_every: int):
        solver.set_field_tensor("pump_plus", pump.detach().contiguous(), 0)
        if potential is not None:
            solver.set_field_tensor("potential_plus", potential.detach().contiguous(), 0)
        solver.set_field_tensor("psi_plus", psi0.detach().contiguous())
        solver.set_field_tensor("n_plus", n0.detach().contiguous())
        solver.adjoint_forward(iterations, checkpoint_every)
        psi_T = solver.get_field_tensor("psi_plus")
        n_T = solver.get_field_tensor("n_plus")
        ctx.solver = solver
        return psi_T, n_T

    @staticmethod
    def backward(ctx, g_psi, g_n):
        solver = ctx.solver
        if g_psi is None:
            g_psi = torch.zeros_like(solver.get_field_tensor("psi_plus"))
        g_psi0, g_n0, g_p, g_v = solver.adjoint_backward(
            g_psi.contiguous(), None if g_n is None else g_n.contiguous(), want_psi0=ctx.needs_input_grad[1],
            want_n0=ctx.needs_input_grad[2], want_pump=ctx.needs_input_grad[0],
            want_potential=ctx.needs_input_grad[3])
        return g_p, g_psi0, g_n0, g_v, None, None, None


def evolve(solver: Solver, pump, psi0, n0, iterations: int, checkpoint_every: int = 0, potential=None):
    """Final (psi, n) after `iterations` RK4 iterations, differentiable in pump,
    psi0, n0 and, when given, the potential (the solver needs a potential group
    for it; without it the solver's own potential, if any, is used as is)."""
    return _Trajectory.apply(pump, psi0, n0, potential, solver, int(iterations), int(checkpoint_every))
