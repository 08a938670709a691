"""Projected gradient descent on spot weights, all state on the device.

    mu <- max(0, mu - eta * d/dmu sum_v w_v (D_v(mu) - P_v)^2)

with D = scale * K mu the pencil-beam dose (forward kernel), the gradient
from the adjoint kernel and the objective reduced in FP64 on the device.
The step eta = 1 / L uses L, an upper estimate of the largest eigenvalue of
the objective's Hessian 2 scale^2 K^T W K, from power iteration (each
iteration is one forward and one adjoint), so every step decreases the
objective.  One iteration is captured once as a CUDA graph and replayed;
the objective of every iteration is kept in a device buffer.

The reference has no optimiser; its dose is the forward of
DoseCUDA/dose_kernels/IMPTClasses.cu:204-271.
"""
from __future__ import annotations

from typing import Optional

import torch

from . import engine


class ProjectedGradient:

    def __init__(self, dp: "engine.DevicePlan", presc: torch.Tensor, weight: torch.Tensor,
                 scale: float = 1.0, mu_plan: Optional[torch.Tensor] = None):
        self.dp = dp
        dev = dp.device
        self.presc = presc.to(dev, torch.float32).reshape(-1).contiguous()
        self.weight = weight.to(dev, torch.float32).reshape(-1).contiguous()
        if self.presc.numel() != dp.n_vox or self.weight.numel() != dp.n_vox:
            raise ValueError("prescription and weights need one value per voxel")
        self.scale = float(scale)
        self.mu = (dp.mu_sorted if mu_plan is None else dp.to_sorted(
            mu_plan.to(dev, torch.float32))).clone()
        self.dose = torch.empty(dp.n_vox, dtype=torch.float32, device=dev)
        self.resid = torch.empty_like(self.dose)
        self.grad = torch.empty(max(dp.n_spots, 1), dtype=torch.float32, device=dev)
        self.obj = torch.zeros(1, dtype=torch.float64, device=dev)
        self.eta = None
        self.graph = None

    def lipschitz(self, iters: int = 10) -> float:
        """Power-iteration estimate of the Hessian's largest eigenvalue."""
        v = self.mu.clone()
        v /= torch.linalg.vector_norm(v)
        lam = 0.0
        for _ in range(iters):
            self.dp.forward(v, scale=self.scale, out=self.dose)
            torch.mul(self.dose, self.weight, out=self.resid)
            self.resid.mul_(2.0)
            self.dp.adjoint(self.resid, scale=self.scale, out=self.grad)
            hv = self.grad[: self.dp.n_spots]
            lam = float(torch.dot(v.double(), hv.double()))
            v = hv / torch.linalg.vector_norm(hv)
        return lam

    def step(self) -> None:
        """One iteration, stream-ordered (capturable)."""
        self.dp.forward(self.mu, scale=self.scale, out=self.dose)
        engine.objective(self.dose, self.presc, self.weight, self.resid, out=self.obj)
        self.dp.adjoint(self.resid, scale=self.scale, out=self.grad)
        self.mu.sub_(self.grad[: self.dp.n_spots], alpha=self.eta).clamp_(min=0.0)

    def prepare(self, capture: bool = True, safety: float = 1.05) -> None:
        if self.eta is None:
            self.eta = 1.0 / (safety * self.lipschitz())
        if capture:
            self.step()                       # warm-up outside the capture
            torch.cuda.synchronize(self.dp.device)
            self.graph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(self.graph):
                self.step()

    def run(self, iters: int) -> torch.Tensor:
        """Run `iters` iterations; returns the FP64 objective before each
        step (device tensor)."""
        if self.eta is None:
            self.prepare()
        hist = torch.empty(iters, dtype=torch.float64, device=self.dp.device)
        for i in range(iters):
            if self.graph is not None:
                self.graph.replay()
            else:
                self.step()
            hist[i : i + 1].copy_(self.obj)
        return hist

    def final_dose(self) -> torch.Tensor:
        self.dp.forward(self.mu, scale=self.scale, out=self.dose)
        return self.dose

    def mu_plan(self) -> torch.Tensor:
        return self.dp.to_plan(self.mu)
