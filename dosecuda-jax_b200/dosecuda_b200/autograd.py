"""torch.autograd wrappers: dose as a differentiable function of spot weights.

``dose(mu, plan)`` runs the forward pencil-beam kernel; its backward runs the
hand-written adjoint kernel (matrix-free: spot footprints are recomputed,
the spot-voxel influence matrix is never stored).  ``quadratic_objective``
reduces sum_v w_v (D_v - P_v)^2 in FP64 on the device; its backward is
2 w (D - P).

The reference has no gradient path; the closest is the JAX restatement's
claim of differentiability (DoseCUDA/Jax/impt_jax.py, never differentiated
in the reference).  The forward it differentiates is
DoseCUDA/dose_kernels/IMPTClasses.cu:204-271.
"""
from __future__ import annotations

import numpy as np
import torch

from . import engine


class PencilBeamDose(torch.autograd.Function):
    """mu (plan row order) -> dose (V, float32)."""

    @staticmethod
    def forward(ctx, mu_plan: torch.Tensor, dp: "engine.DevicePlan", scale: float):
        mu_sorted = dp.to_sorted(mu_plan.detach().to(torch.float32).contiguous())
        dose = dp.forward(mu_sorted, scale=scale)
        ctx.dp = dp
        ctx.scale = scale
        return dose

    @staticmethod
    def backward(ctx, grad_dose: torch.Tensor):
        g = ctx.dp.adjoint(grad_dose.to(torch.float32).contiguous(), scale=ctx.scale)
        return ctx.dp.to_plan(g), None, None


class QuadraticObjective(torch.autograd.Function):
    """(dose, prescription, weights) -> sum w (D - P)^2 as a float64 scalar."""

    @staticmethod
    def forward(ctx, dose: torch.Tensor, presc: torch.Tensor, weight: torch.Tensor):
        resid = torch.empty_like(dose)
        obj = engine.objective(dose.detach(), presc, weight, resid)
        ctx.save_for_backward(resid)
        return obj.reshape(())

    @staticmethod
    def backward(ctx, g: torch.Tensor):
        (resid,) = ctx.saved_tensors
        return resid * g.to(torch.float32), None, None


def dose(mu: torch.Tensor, dp: "engine.DevicePlan", scale: float = 1.0) -> torch.Tensor:
    return PencilBeamDose.apply(mu, dp, float(scale))


def quadratic_objective(d: torch.Tensor, presc: torch.Tensor, weight: torch.Tensor):
    return QuadraticObjective.apply(d, presc, weight)


def _as_device(x, n, device):
    t = torch.as_tensor(np.asarray(x, dtype=np.float32).reshape(-1) if not torch.is_tensor(x)
                        else x.reshape(-1).to(torch.float32))
    if t.numel() != n:
        raise ValueError(f"expected {n} voxel values, got {t.numel()}")
    return t.to(device).contiguous()


def plan_objective_and_grad(dp: "engine.DevicePlan", target_dose, voxel_weights,
                            scale: float = 1.0, mu_plan=None):
    """Objective (float) and d objective / d mu (float32 ndarray, plan order)."""
    presc = _as_device(target_dose, dp.n_vox, dp.device)
    w = _as_device(voxel_weights, dp.n_vox, dp.device)
    mu_sorted = dp.mu_sorted if mu_plan is None else dp.to_sorted(
        torch.as_tensor(mu_plan, dtype=torch.float32, device=dp.device))
    d = dp.forward(mu_sorted, scale=scale)
    resid = torch.empty_like(d)
    obj = engine.objective(d, presc, w, resid)
    g = dp.adjoint(resid, scale=scale)
    return float(obj.item()), dp.to_plan(g).cpu().numpy()
