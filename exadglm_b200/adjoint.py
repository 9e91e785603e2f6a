"""Gradients of final-time objectives through the DGLM time integration.

``evolve(u0, solver, nsteps)`` (the autograd Function ``DGLMStep``) advances
the state ``u0`` (a CUDA float64 tensor of shape (nvar, K*Np), the
reference's nodal layout) by ``nsteps`` LSERK steps on ``solver`` and returns
u(T) as a differentiable tensor.  The backward pass is the library's discrete adjoint (``dglm_adjoint_backward``):
the exact transpose of the FP64 step with dt and the face penalty tau held at
the values of the forward run.  Those two are maxima over the state (a global
CFL max and per-face wave speeds), so they are frozen rather than
differentiated; finite-difference checks must replay them
(``Solver.adjoint_replay``).

Memory: the forward run keeps a checkpoint every ``checkpoint_every`` steps;
the backward pass recomputes each segment once from its checkpoint, keeping
its 5 stage inputs per step, and sweeps it in reverse.  With ``max_bytes``
the tape instead stays under that many bytes of device memory by binomial
checkpointing (revolve): fewer checkpoints, more forward steps recomputed,
the same gradient.

The reference has no adjoint; this module has no counterpart there.
"""
from __future__ import annotations

import torch

from .capi import Solver


class DGLMStep(torch.autograd.Function):
    """``DGLMStep.apply(u0, solver, nsteps, checkpoint_every, max_bytes)``:
    u(T) after ``nsteps`` CFL steps from u0; its backward is the discrete
    adjoint (max_bytes: None, or a cap on the tape's device memory)."""

    @staticmethod
    def forward(ctx, u0, solver, nsteps, checkpoint_every, max_bytes=None):
        nv = solver.p.nvar
        if u0.dtype != torch.float64 or not u0.is_cuda or tuple(u0.shape) != (
                nv, solver.p.K * solver.p.Np):
            raise ValueError("evolve: u0 must be a CUDA float64 tensor of shape (nvar, K*Np)")
        u0c = u0.detach().contiguous()
        torch.cuda.current_stream(u0c.device).synchronize()
        solver.set_state_device([u0c[v].data_ptr() for v in range(nv)])
        if max_bytes is None:
            solver.adjoint_record(int(nsteps), int(checkpoint_every))
        else:
            solver.adjoint_record_capped(int(nsteps), int(max_bytes))
        uT = torch.empty_like(u0c)
        solver.get_state_device([uT[v].data_ptr() for v in range(nv)])
        solver._tape_id = getattr(solver, "_tape_id", 0) + 1
        ctx.solver, ctx.tape_id = solver, solver._tape_id
        return uT

    @staticmethod
    def backward(ctx, g):
        s = ctx.solver
        if getattr(s, "_tape_id", None) != ctx.tape_id:
            raise RuntimeError("evolve: the solver recorded another run since this forward; "
                               "call backward before the next evolve on the same solver")
        nv = s.p.nvar
        g = g.contiguous()
        torch.cuda.current_stream(g.device).synchronize()
        lam0 = torch.empty_like(g)
        s.adjoint_backward_device([g[v].data_ptr() for v in range(nv)],
                                  [lam0[v].data_ptr() for v in range(nv)])
        return lam0, None, None, None, None


def evolve(u0: torch.Tensor, solver: Solver, nsteps: int, checkpoint_every: int = 50,
           max_bytes: int | None = None):
    """u(T) after nsteps CFL steps from u0, differentiable with respect to u0;
    max_bytes caps the tape's device memory (binomial checkpointing)."""
    return DGLMStep.apply(u0, solver, nsteps, checkpoint_every, max_bytes)


def density_misfit(uT: torch.Tensor, rho_target: torch.Tensor) -> torch.Tensor:
    """J = 1/2 ||rho(T) - rho_target||^2 (the objective of the gradient check)."""
    d = uT[0] - rho_target
    return 0.5 * torch.dot(d, d)
