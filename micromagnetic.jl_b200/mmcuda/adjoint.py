"""Reverse-mode gradients through fixed-step RK4 on the device
(mm_adjoint_record / mm_adjoint_backward).

The reference has no differentiation of this path; this is the Python
counterpart of the ChainRulesCore.rrule that julia/MMCuda.jl defines:
`rk4_grad` for a host loss, and `RK4Function`, a torch.autograd.Function
whose input is m0 and whose output is m after nsteps RK4 steps.
"""
from __future__ import annotations

import numpy as np

from . import _lib


def record(sim, nsteps: int, dt: float | None = None, ckpt_every: int = 100) -> np.ndarray:
    """Run nsteps RK4 steps from the Sim's m, keeping checkpoints every
    ckpt_every steps; returns m_T (AoS, 3N)."""
    h = float(sim.driver.integrator._step if dt is None else dt)
    sim._h.call("mm_adjoint_record", h, int(nsteps), int(ckpt_every))
    return sim.spin


def backward(sim, dL_dmT) -> dict:
    """Gradients of L for dL/dm_T: dict with m0 (3N), Ms (N, per A/m),
    Ku (N) and D (N, interfacial DMI per cell)."""
    n = sim.n_total
    out = {"m0": np.zeros(3 * n), "Ms": np.zeros(n), "Ku": np.zeros(n), "D": np.zeros(n)}
    g = np.ascontiguousarray(np.asarray(dL_dmT, dtype=np.float64).reshape(-1))
    if g.size != 3 * n:
        raise ValueError("dL/dm_T must have 3N entries")
    d = _lib.dptr
    sim._h.call("mm_adjoint_backward", d(g), d(out["m0"]), d(out["Ms"]), d(out["Ku"]), d(out["D"]))
    return out


def rk4_grad(sim, loss_and_grad, nsteps: int, dt: float | None = None, ckpt_every: int = 100):
    """L and its gradients for a loss of the final state:
    loss_and_grad(m_T) -> (L, dL/dm_T).  Returns (L, grads) with grads as in
    `backward`; the Sim is left at m_T."""
    mT = record(sim, nsteps, dt, ckpt_every)
    L, g = loss_and_grad(mT)
    return L, backward(sim, g)


def _torch_function():
    import torch

    class RK4Function(torch.autograd.Function):
        """m_T = RK4^nsteps(m0) for a Sim; backward returns dL/dm0 and stores
        the parameter gradients in sim.adjoint_grads (Ms, Ku, D)."""

        @staticmethod
        def forward(ctx, m0, sim, nsteps, dt, ckpt_every):
            sim.spin = m0.detach().double().cpu().numpy()
            mT = record(sim, nsteps, dt, ckpt_every)
            ctx.sim = sim
            return torch.from_numpy(mT).to(m0.device, m0.dtype)

        @staticmethod
        def backward(ctx, grad_mT):
            grads = backward(ctx.sim, grad_mT.detach().double().cpu().numpy())
            ctx.sim.adjoint_grads = grads
            return torch.from_numpy(grads["m0"]).to(grad_mT.device, grad_mT.dtype), None, None, None, None

    return RK4Function


def __getattr__(name):
    if name == "RK4Function":
        return _torch_function()
    raise AttributeError(name)

