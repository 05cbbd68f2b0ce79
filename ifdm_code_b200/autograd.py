"""torch.autograd binding of the adjoint split step.

``evolve(psi0, sim, a0, nsteps, dt_scale, checkpoint_every)`` runs ``nsteps``
fixed-mode leap-frog steps of ``sim`` (a :class:`Simulation`) from the complex128
CUDA tensor ``psi0`` at scale factor ``a0`` and returns psi after the last
step.  Its backward pass is the hand-written adjoint behind the C ABI
(``ifdm_record_steps`` / ``ifdm_adjoint``): checkpoints every
``checkpoint_every`` steps, segments replayed forward, then swept backwards.
Gradients follow torch's convention for real losses of complex tensors,
dL/dRe + i dL/dIm, which is what the adjoint computes.  The step schedule is
the recorded one (it depends on max reductions, which are not
differentiated).
"""

from __future__ import annotations

import torch

from .simulation import Simulation


class _Evolve(torch.autograd.Function):
    @staticmethod
    def forward(ctx, psi0, sim: Simulation, a0: float, nsteps: int, dt_scale: float, checkpoint_every: int):
        if psi0.dtype != torch.complex128 or not psi0.is_cuda:
            raise TypeError("psi0 must be a complex128 CUDA tensor")
        x = psi0.detach().contiguous()
        torch.cuda.current_stream().synchronize()  # x is read on the library's own stream
        sim.set_psi(x, a0)
        sim.record_steps(nsteps, dt_scale, checkpoint_every)
        out = torch.empty_like(x)
        sim.get_psi_into(out)
        ctx.sim = sim
        return out

    @staticmethod
    def backward(ctx, g):
        g = g.detach().to(torch.complex128).contiguous()
        g0 = torch.empty_like(g)
        torch.cuda.current_stream().synchronize()
        ctx.sim.adjoint(g, g0)
        return g0, None, None, None, None, None


def evolve(psi0: torch.Tensor, sim: Simulation, a0: float, nsteps: int, dt_scale: float = 1.0,
           checkpoint_every: int = 20) -> torch.Tensor:
    """psi after ``nsteps`` steps from ``psi0``; differentiable through the adjoint."""
    return _Evolve.apply(psi0, sim, a0, nsteps, dt_scale, checkpoint_every)
