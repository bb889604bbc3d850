"""torch.autograd wrapper of the engine's pathwise adjoint (dsmc_adjoint_run).

    theta = torch.tensor([B', B0, eta_0, ..., eta_8], dtype=torch.float64, requires_grad=True)
    energy, retained = smoothed_loss_terms(theta, run, cloud, steps=2000)
    (energy + retained).backward()   # theta.grad by the hand-written adjoint

Each forward call runs one physical simulation at theta (the cloud is initialised with the given
seed), records its collisions and evaluates the smoothed model: every atom kept with a survival
weight, the product over steps of the knife's sigmoid((cut - E) / (width kB T0)) and, when the
cloud has Majorana loss, of sigmoid(<s.B^> / majorana_width), the spinors precessing about the
local field as in the run.  Its two terms are the final mean energy per retained atom in units of
kB T0 and the retained fraction; the adjoint gives the gradient of each, so any weighting of the
two differentiates exactly.  The gradient holds every random choice of the run fixed, and the
initial cloud too (it is an input of the run, not differentiated).
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


class SmoothedLossTerms(torch.autograd.Function):
    @staticmethod
    def forward(ctx, theta, run, cloud, steps, checkpoint_every, precision, width_kT, majorana_width, seed):
        th = theta.detach().to("cpu", torch.float64)
        sim = Simulation(run, _cloud_at(cloud, th))
        try:
            sim.init_cloud(seed)
            g = sim.adjoint_run(steps, checkpoint_every, precision, width_kT, majorana_width)
        finally:
            sim.close()
        jac = torch.tensor([g["dE_dtheta"], g["dN_dtheta"]], dtype=torch.float64)
        ctx.save_for_backward(jac.to(theta.device, theta.dtype))
        return torch.tensor([g["mean_energy_kT"], g["retained_fraction"]], dtype=theta.dtype, device=theta.device)

    @staticmethod
    def backward(ctx, grad_out):
        (jac,) = ctx.saved_tensors
        return grad_out @ jac, None, None, None, None, None, None, None, None


def smoothed_loss_terms(theta: torch.Tensor, run: _abi.RunParams, cloud: _abi.CloudParams, steps: int,
                        checkpoint_every: int = 100, precision: int = _abi.FP64, width_kT: float = 0.2,
                        majorana_width: float = 0.05, seed: int = 1234) -> torch.Tensor:
    """(final mean energy per retained atom / kB T0, retained fraction) of a DSMC run at
    theta = (B', B0, eta_0..eta_8), differentiable by the pathwise adjoint."""
    return SmoothedLossTerms.apply(theta, run, cloud, steps, checkpoint_every, precision, width_kT, majorana_width,
                                   seed)


def smoothed_knife_loss(theta: torch.Tensor, run: _abi.RunParams, cloud: _abi.CloudParams, steps: int,
                        checkpoint_every: int = 100, precision: int = _abi.FP64, width_kT: float = 0.2,
                        seed: int = 1234, majorana_width: float = 0.05) -> torch.Tensor:
    """The sum of the two terms: the loss dsmc_adjoint_run reports."""
    return smoothed_loss_terms(theta, run, cloud, steps, checkpoint_every, precision, width_kT, majorana_width,
                               seed).sum()
