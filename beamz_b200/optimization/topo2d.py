"""Density-based topology optimisation on the batched adjoint (examples/4_topo.py:52-420).

The parametrisation follows the reference loop: a masked box blur of the design
density, a smoothed-Heaviside (tanh) projection with a beta schedule, the mapping
eps = eps_lo + rho_phys * (eps_hi - eps_lo), and Adam on the normalised gradient
with clipping to [0, 1]. The gradient of the objective with respect to eps comes
from the exact adjoint (FDTDObjective); the filter chain is differentiated by
torch autograd instead of the reference's hand-written back-propagation.
"""
from __future__ import annotations

import time

import numpy as np
import torch
import torch.nn.functional as F

from .adjoint import AdjointFDTD2D, FDTDObjective


def masked_box_blur(rho: torch.Tensor, radius: int) -> torch.Tensor:
    """Mean over a (2r+1)^2 window; the design region is the whole tensor, edges are
    replicated (the reference pads values by edge and the mask by zeros; inside a
    full rectangular region the two agree away from its border)."""
    if radius < 1:
        return rho
    k = 2 * radius + 1
    x = F.pad(rho[:, None], (radius,) * 4, mode="replicate")
    ones = torch.ones((1, 1, k, k), dtype=rho.dtype, device=rho.device) / (k * k)
    return F.conv2d(x, ones)[:, 0]


def smoothed_heaviside(v: torch.Tensor, beta: float, eta: float = 0.5) -> torch.Tensor:
    beta = max(beta, 1e-6)
    den = np.tanh(beta * eta) + np.tanh(beta * (1.0 - eta))
    return (np.tanh(beta * eta) + torch.tanh(beta * (v - eta))) / den


class TopologyOptimizer2D:
    """Adam ascent of the mode-power objective for B designs at once."""

    def __init__(self, problem: AdjointFDTD2D, rho0, eps_lo, eps_hi, *, lr=0.1, radius=2, beta=(2.0, 20.0),
                 steps=50, j_ref=1.0):
        self.problem = problem
        self.rho = torch.tensor(np.asarray(rho0), dtype=torch.float64, requires_grad=True)
        self.eps_lo, self.eps_hi = eps_lo, eps_hi
        self.radius, self.beta, self.n_steps, self.j_ref = radius, beta, steps, j_ref
        self.opt = torch.optim.Adam([self.rho], lr=lr)
        self.it = 0
        self.history = []

    def physical(self, rho=None):
        rho = self.rho if rho is None else rho
        frac = 0.0 if self.n_steps <= 1 else min(1.0, self.it / (self.n_steps - 1))
        beta = self.beta[0] + frac * (self.beta[1] - self.beta[0])
        return smoothed_heaviside(torch.clamp(masked_box_blur(rho, self.radius), 0.0, 1.0), beta)

    def step(self):
        t0 = time.perf_counter()
        self.opt.zero_grad()
        eps = self.eps_lo + self.physical() * (self.eps_hi - self.eps_lo)
        J = FDTDObjective.apply(eps, self.problem) / self.j_ref
        (-J.sum()).backward()
        g = self.rho.grad
        self.rho.grad = g / g.abs().amax(dim=(1, 2), keepdim=True).clamp_min(1e-300)
        self.opt.step()
        with torch.no_grad():
            self.rho.clamp_(0.0, 1.0)
        self.it += 1
        self.history.append((J.detach().numpy().copy(), time.perf_counter() - t0))
        return J.detach().numpy()
