"""Density filters and the masked density update of a topology loop, on torch tensors
batched over designs (the operations of beamz/optimization/topology.py:31-178).

Every function takes densities shaped ``(..., H, W)`` -- one design or a batch of
designs sharing leading dimensions -- as NumPy arrays or torch tensors. The arithmetic
runs in float64 on the tensor's device (a CUDA batch stays on the GPU), and the result
comes back as the kind of array that was passed in.

* ``masked_box_blur``: normalised box average over a (2r+1)^2 window counting only
  cells inside the mask; values are continued past the border by their edge value,
  the mask by zeros; a window holding no mask cell divides by one.
* ``apply_density_update``: ``clip(rho + lr * g_s, 0, 1)`` inside the mask, where
  ``g_s`` is the gradient restricted to the mask and optionally smoothed; returns the
  new density, ``g_s``, the change, and the L2 norm and largest magnitude of the
  change inside the mask (floats for one design, one value per design for a batch).
* ``blur_density``: separable box filter with zero padding ('same' size).
* ``project_density``: logistic projection ``1 / (1 + exp(-beta (rho - eta)))``.
* ``compute_overlap_gradient``: ``Re(conj(E_adj) E_fwd)`` over the common extent.

The exact discrete adjoint gradient of a monitor objective is
``beamz_b200.optimization.adjoint``; the tanh-projected filter chain of the topology
loop is ``beamz_b200.optimization.topo2d``.
"""
from __future__ import annotations

from typing import Callable, Optional

import numpy as np
import torch
import torch.nn.functional as F


def _tensor(x, device=None) -> torch.Tensor:
    if isinstance(x, torch.Tensor):
        return x.to(dtype=torch.float64, device=device if device is not None else x.device)
    return torch.as_tensor(np.asarray(x, dtype=np.float64), device=device)


def _like(t: torch.Tensor, template):
    return t if isinstance(template, torch.Tensor) else t.cpu().numpy()


def _planes(t: torch.Tensor) -> tuple[torch.Tensor, tuple]:
    """(N, 1, H, W) view of a (..., H, W) tensor, and the leading shape."""
    lead = tuple(t.shape[:-2])
    return t.reshape((-1, 1) + tuple(t.shape[-2:])), lead


def _box_sum(x: torch.Tensor, r: int) -> torch.Tensor:
    """Sum over the (2r+1)^2 window of an already padded (N, 1, H+2r, W+2r) tensor."""
    k = torch.ones((1, 1, 2 * r + 1, 2 * r + 1), dtype=x.dtype, device=x.device)
    return F.conv2d(x, k)


def masked_box_blur(values, mask, radius):
    """Normalised box average of ``values`` over the cells of ``mask`` (see module)."""
    r = int(max(0, round(radius)))
    if r < 1:
        return values
    v = _tensor(values)
    m = _tensor(mask, device=v.device).expand_as(v)
    vp, lead = _planes(v)
    mp, _ = _planes(m)
    num = _box_sum(F.pad(vp, (r, r, r, r), mode="replicate") * F.pad(mp, (r, r, r, r)), r)
    den = _box_sum(F.pad(mp, (r, r, r, r)), r)
    out = (num / torch.where(den == 0, torch.ones_like(den), den)).reshape(v.shape)
    return _like(out, values)


def apply_density_update(density, gradient, mask, *, learning_rate: float, blur_radius: int = 0,
                         blur_fn: Optional[Callable] = None):
    """Masked, clipped density step (see module). Returns
    ``(new_density, applied_gradient, delta, change_norm, max_update)``."""
    rho = _tensor(density)
    g = _tensor(gradient, device=rho.device)
    if g.shape != rho.shape:
        raise ValueError(f"gradient shape {tuple(g.shape)} differs from density shape {tuple(rho.shape)}")
    m = torch.as_tensor(np.asarray(mask) if not isinstance(mask, torch.Tensor) else mask, device=rho.device)
    if m.shape != rho.shape[-m.dim():] or m.dim() < 2:
        raise ValueError(f"mask shape {tuple(m.shape)} does not match density shape {tuple(rho.shape)}")
    m = m.to(torch.bool).expand_as(rho)
    zero = torch.zeros((), dtype=rho.dtype, device=rho.device)
    gs = torch.where(m, g, zero)
    if blur_fn is not None:
        gs = _tensor(blur_fn(_like(gs, density), _like(m, density)), device=rho.device)
    elif blur_radius > 0:
        gs = _tensor(masked_box_blur(gs, m.to(rho.dtype), blur_radius))
    gs = torch.where(m, gs, zero)
    new = torch.where(m, torch.clamp(rho + learning_rate * gs, 0.0, 1.0), rho)
    delta = torch.where(m, new - rho, zero)
    flat = delta.reshape(delta.shape[:-2] + (-1,))
    norm = torch.linalg.vector_norm(flat, dim=-1)
    peak = flat.abs().amax(dim=-1) if flat.shape[-1] else torch.zeros(flat.shape[:-1], dtype=rho.dtype)
    if rho.dim() == 2:
        norm, peak = float(norm), float(peak)
    else:
        norm, peak = _like(norm, density), _like(peak, density)
    return _like(new, density), _like(gs, density), _like(delta, density), norm, peak


def blur_density(density, radius: float, *, backend: str = "torch"):
    """Separable (2r+1)-point box filter along x then y, zero padded, same size."""
    r = max(0, int(round(radius)))
    if r <= 0:
        return density
    t = _tensor(density)
    p, _ = _planes(t)
    k = torch.full((1, 1, 1, 2 * r + 1), 1.0 / (2 * r + 1), dtype=t.dtype, device=t.device)
    p = F.conv2d(F.pad(p, (r, r, 0, 0)), k)
    p = F.conv2d(F.pad(p, (0, 0, r, r)), k.transpose(-1, -2))
    return _like(p.reshape(t.shape), density)


def project_density(density, beta: float, eta: float):
    """Logistic projection towards 0/1 around eta; beta <= 0 leaves the density as is."""
    if beta <= 0:
        return density
    t = _tensor(density)
    return _like(torch.sigmoid(beta * (t - eta)), density)


def _ez(container):
    if container is None:
        return None
    v = container.get("Ez") if isinstance(container, dict) else getattr(container, "Ez", None)
    if isinstance(v, (list, tuple)):
        v = v[-1] if v else None
    return v


def compute_overlap_gradient(forward_fields, adjoint_fields, *, monitor=None):
    """Re(conj(E_adj) * E_fwd) of the two runs' Ez (a dict or object with ``Ez``; a list
    holds snapshots, the last is used), over the extent common to both."""
    fwd, adj = _ez(forward_fields), _ez(adjoint_fields)
    if fwd is None or adj is None:
        raise ValueError("forward and adjoint results both need an 'Ez' field")
    ft = torch.as_tensor(fwd) if isinstance(fwd, torch.Tensor) else torch.as_tensor(np.asarray(fwd))
    at = torch.as_tensor(adj, device=ft.device) if isinstance(adj, torch.Tensor) else \
        torch.as_tensor(np.asarray(adj), device=ft.device)
    common = tuple(slice(0, min(a, b)) for a, b in zip(ft.shape, at.shape))
    ft, at = ft[common], at[common]
    g = (at.conj() * ft).real if (ft.is_complex() or at.is_complex()) else at * ft
    return _like(g.to(torch.float64), fwd)


__all__ = ["masked_box_blur", "apply_density_update", "blur_density", "project_density",
           "compute_overlap_gradient"]
