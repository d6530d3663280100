"""torch.autograd bridge to the discrete adjoint (bfx_adjoint).

    theta = torch.tensor([stroke, pitch, phase, deviation], dtype=torch.float64, requires_grad=True)
    J = kinematic_objective(theta, build, steps=2000, force_weight=(0, 0, 1))
    J.backward()            # theta.grad = dJ/dtheta from one forward + adjoint run

``build(theta)`` returns a fresh :class:`bfx.simulation.Lattice` whose wing
kinematics are ``theta`` (for example ``cases.with_kinematic_parameters``).
The forward call runs the simulation and its adjoint once and keeps the
gradient; backward scales it by the incoming gradient.  The reference's Python
tooling (``Reference/*.py``) can call this like any other torch function.
"""
from __future__ import annotations

from typing import Callable, Optional, Sequence

import torch


class KinematicObjective(torch.autograd.Function):
    @staticmethod
    def forward(ctx, theta: torch.Tensor, build: Callable, steps: int, force_weight: Sequence[float],
                power_weight: float, window: Optional[Sequence[int]], checkpoint_interval: int):
        params = tuple(float(v) for v in theta.detach().cpu().reshape(-1).tolist())
        if len(params) != 4:
            raise ValueError("theta holds the four kinematic parameters")
        lattice = build(params)
        try:
            res = lattice.adjoint(steps, force_weight, power_weight, window, checkpoint_interval)
        finally:
            lattice.close()
        ctx.save_for_backward(torch.tensor(list(res.gradient), dtype=theta.dtype, device=theta.device))
        ctx.result = res
        return torch.tensor(res.objective, dtype=theta.dtype, device=theta.device)

    @staticmethod
    def backward(ctx, grad_output: torch.Tensor):
        (gradient,) = ctx.saved_tensors
        return grad_output * gradient, None, None, None, None, None, None


def kinematic_objective(theta: torch.Tensor, build: Callable, steps: int, force_weight=(0.0, 0.0, 1.0),
                        power_weight: float = 0.0, window=None, checkpoint_interval: int = 0) -> torch.Tensor:
    """J(theta) as a differentiable torch scalar (see the module docstring)."""
    return KinematicObjective.apply(theta, build, int(steps), tuple(float(w) for w in force_weight),
                                    float(power_weight), None if window is None else tuple(window),
                                    int(checkpoint_interval))
