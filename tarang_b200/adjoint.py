"""Gradients through the IF-RK4 time stepper: a torch.autograd.Function over the
CUDA library's discrete adjoint (FFF basis, rotational form, unforced).

``rk4_evolve(u0, plan, nsteps, window)`` returns u(nsteps) and, under autograd,
back-propagates with checkpointed recomputation: the forward pass keeps the
state only every ``window`` steps; the backward pass re-runs each window from
its checkpoint (keeping that window's states and stage fields in one work
buffer) and runs the window's adjoint steps last step first
(``ts_adjoint_window``).  Memory: nsteps/window checkpoints of 3 components plus
one work buffer of 12 * window components.

The gradient convention is torch's for a real loss of a complex tensor: the
cotangent G of a field A satisfies dJ = Re sum G conj(dA) over the stored
half-spectrum entries.  The reference has no adjoint (its solvers only step
forward); this module has no counterpart there.
"""
from __future__ import annotations

import torch

from .solver import Plan


class RK4Evolve(torch.autograd.Function):
    @staticmethod
    def forward(ctx, u0: torch.Tensor, plan: Plan, nsteps: int, window: int):
        if nsteps < 1 or window < 1:
            raise ValueError("nsteps and window must be >= 1")
        u = u0.detach().contiguous().clone()
        ckpts = []
        for s in range(0, nsteps, window):
            ckpts.append(u.clone())
            plan.rk4_step(u, min(window, nsteps - s))
        ctx.plan, ctx.nsteps, ctx.window = plan, nsteps, window
        ctx.ckpts = ckpts
        return u

    @staticmethod
    def backward(ctx, grad):
        plan, nsteps, window = ctx.plan, ctx.nsteps, ctx.window
        lam = grad.detach().contiguous().clone()
        nb = plan.adjoint_work_bytes(min(window, nsteps))
        work = torch.empty(nb, dtype=torch.uint8, device=lam.device)
        for w in reversed(range(len(ctx.ckpts))):
            n = min(window, nsteps - w * window)
            plan.adjoint_window(ctx.ckpts[w], n, lam, work)
        ctx.ckpts = None
        return lam, None, None, None


def rk4_evolve(u0: torch.Tensor, plan: Plan, nsteps: int, window: int = 20) -> torch.Tensor:
    """u(nsteps) from u0 by `plan`'s IF-RK4 step, differentiable with respect to u0."""
    return RK4Evolve.apply(u0, plan, nsteps, window)


def energy_norm_loss(u: torch.Tensor, target: torch.Tensor) -> torch.Tensor:
    """J = 1/2 ||u - target||^2 with the Tarang energy weights (1, and 1/2 on the kz = 0 plane),
    i.e. the total energy of the difference field."""
    d = u - target
    w = torch.ones(d.shape[-1], dtype=torch.float64, device=d.device)
    w[0] = 0.5
    return ((d.real.double() ** 2 + d.imag.double() ** 2) * w).sum()
