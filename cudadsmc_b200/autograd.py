"""torch.autograd wrapper of the engine's pathwise adjoint (dsmc_adjoint_run).

    theta = torch.tensor([B', B0, eta_0, ..., eta_8], dtype=torch.float64, requires_grad=True)
    loss = smoothed_knife_loss(theta, run, cloud, steps=2000)
    loss.backward()          # theta.grad = d loss / d theta, by the hand-written adjoint

Each forward call runs one physical simulation at theta (the cloud is initialised with the given
seed), records its collisions and evaluates the smoothed-knife loss: the final mean energy per
retained atom in units of kB T0 plus the retained fraction, with each atom's survival weight the
product over steps of sigmoid((cut - E) / (width kB T0)).  The gradient holds every random choice
of the run fixed, and the initial cloud too (it is an input of the run, not differentiated).
"""
from __future__ import annotations

import torch

from . import _abi
from .engine import Simulation


def _cloud_at(cloud: _abi.CloudParams, theta) -> _abi.CloudParams:
    c = cloud.copy()
    c.dBdz = float(theta[0])
    c.B0 = float(theta[1])
    for k in range(9):
        c.knife_eta[k] = float(theta[2 + k])
    return c


class SmoothedKnifeLoss(torch.autograd.Function):
    @staticmethod
    def forward(ctx, theta, run, cloud, steps, checkpoint_every, precision, width_kT, seed):
        th = theta.detach().to("cpu", torch.float64)
        sim = Simulation(run, _cloud_at(cloud, th))
        try:
            sim.init_cloud(seed)
            g = sim.adjoint_run(steps, checkpoint_every, precision, width_kT)
        finally:
            sim.close()
        grad = torch.tensor([g["dL_dBp"], g["dL_dB0"]] + list(g["dL_deta"]), dtype=torch.float64)
        ctx.save_for_backward(grad.to(theta.device, theta.dtype))
        return torch.tensor(g["loss"], dtype=theta.dtype, device=theta.device)

    @staticmethod
    def backward(ctx, grad_out):
        (grad,) = ctx.saved_tensors
        return grad_out * grad, None, None, None, None, None, None, None


def smoothed_knife_loss(theta: torch.Tensor, run: _abi.RunParams, cloud: _abi.CloudParams, steps: int,
                        checkpoint_every: int = 100, precision: int = _abi.FP64, width_kT: float = 0.2,
                        seed: int = 1234) -> torch.Tensor:
    """Differentiable smoothed-knife loss of a DSMC run at theta = (B', B0, eta_0..eta_8)."""
    return SmoothedKnifeLoss.apply(theta, run, cloud, steps, checkpoint_every, precision, width_kT, seed)
