"""Topology-optimisation building blocks (beamz/optimization/topology.py:22-306).

Density arrays live on the host as NumPy float64 (they are small: one value per
design-region cell). The masked box blur, sigmoid projection, masked update with
clipping, Adam step and overlap gradient follow the reference's definitions.
"""
from __future__ import annotations

from typing import Callable, Optional, Tuple

import numpy as np
from numpy.lib.stride_tricks import sliding_window_view

from .optimizers import Optimizer

DensityArray = np.ndarray
MaskArray = np.ndarray


def _validate_shapes(density, gradient, mask) -> None:
    if density.shape != gradient.shape:
        raise ValueError("Gradient and density must share shape.")
    if mask.shape != density.shape:
        raise ValueError("Mask must share the same shape as density.")


def _masked_box_blur(values, mask, radius):
    """Mean over the (2r+1)^2 window of the cells inside ``mask`` (edge-padded values,
    zero-padded mask); windows with no mask cell return the weighted sum over 1."""
    radius = int(max(0, round(radius)))
    if radius < 1:
        return values
    pv = np.pad(values, radius, mode="edge")
    pm = np.pad(mask.astype(float), radius, mode="constant", constant_values=0.0)
    win = (2 * radius + 1, 2 * radius + 1)
    vv, mv = sliding_window_view(pv, win), sliding_window_view(pm, win)
    num = (vv * mv).sum(axis=(-2, -1))
    den = mv.sum(axis=(-2, -1))
    return num / np.where(den == 0.0, 1.0, den)


def apply_density_update(density, gradient, mask, *, learning_rate: float, blur_radius: int = 0,
                         blur_fn: Optional[Callable] = None) -> Tuple[np.ndarray, np.ndarray, np.ndarray, float, float]:
    """``clip(density + lr * smooth(gradient inside mask), 0, 1)`` inside ``mask``.

    Returns (new_density, applied_gradient, density_delta, change_norm, max_update).
    """
    _validate_shapes(density, gradient, mask)
    g = np.where(mask, gradient, 0.0).astype(float, copy=False)
    if blur_fn is not None:
        sm = blur_fn(g, mask)
    elif blur_radius > 0:
        sm = _masked_box_blur(g, mask, blur_radius)
    else:
        sm = g
    sm = np.where(mask, sm, 0.0)
    new = np.where(mask, np.clip(density + learning_rate * sm, 0.0, 1.0), density)
    delta = np.where(mask, new - density, 0.0)
    if np.any(mask):
        change_norm = float(np.linalg.norm(delta[mask]))
        max_update = float(np.max(np.abs(delta[mask])))
    else:
        change_norm = max_update = 0.0
    return new, sm, delta, change_norm, max_update


def initialize_density_from_region(design_region, resolution: float) -> DensityArray:
    width = getattr(design_region, "width", None)
    height = getattr(design_region, "height", None)
    if width is None or height is None:
        raise ValueError("Design region must expose width and height attributes.")
    nx = max(1, int(round(width / resolution)))
    ny = max(1, int(round(height / resolution)))
    density = np.full((ny, nx), 0.5, dtype=float)
    grid = getattr(getattr(design_region, "material", None), "permittivity_grid", None)
    if grid is not None:
        density = _resample_to_shape(grid, (ny, nx))
    return density


def blur_density(density, radius: float, *, backend: str = "numpy") -> DensityArray:
    """Separable box blur (``np.convolve`` 'same' along rows then columns)."""
    r = max(0, int(round(radius)))
    if r <= 0:
        return density
    k = np.ones((2 * r + 1,), dtype=float)
    k /= k.size
    out = np.apply_along_axis(lambda row: np.convolve(row, k, mode="same"), axis=1, arr=density)
    return np.apply_along_axis(lambda col: np.convolve(col, k, mode="same"), axis=0, arr=out)


def project_density(density, beta: float, eta: float) -> DensityArray:
    if beta <= 0:
        return density
    return 1.0 / (1.0 + np.exp(-beta * (density - eta)))


def compute_overlap_gradient(forward_fields, adjoint_fields, *, monitor=None) -> DensityArray:
    """Re(conj(adjoint Ez) * forward Ez) over the common extent of the two fields."""
    fwd = _extract_field(forward_fields, "Ez")
    adj = _extract_field(adjoint_fields, "Ez")
    if fwd is None or adj is None:
        raise ValueError("Forward/adjoint data must contain an 'Ez' entry.")
    fwd, adj = np.asarray(fwd), np.asarray(adj)
    g = np.real(np.conj(adj) * fwd)
    return g[tuple(slice(0, min(a, b)) for a, b in zip(fwd.shape, adj.shape))]


def run_forward(sim, source, monitor, *, live: bool = False):
    sim.sources = [source]
    sim.initialize_simulation(save=True, live=live)
    while sim.step():
        pass
    return sim.finalize_simulation()


def run_adjoint(density, sim, source, forward_results, monitor=None, *, live: bool = False) -> DensityArray:
    """Runs the adjoint simulation and returns a zero gradient, as the reference's
    placeholder does (topology.py:191-207). The exact discrete adjoint of this
    package is ``beamz_b200.optimization.adjoint``."""
    sim.sources = [source]
    sim.initialize_simulation(save=True, live=live)
    while sim.step():
        pass
    sim.finalize_simulation()
    return np.zeros_like(density, dtype=float)


def compute_objective(results, monitor=None) -> float:
    ez = _extract_field(results, "Ez")
    return 0.0 if ez is None else float(np.sum(np.abs(ez) ** 2))


def apply_optimizer_step(density, gradient, optimizer_state, *, method="adam", learning_rate=1e-2, **kwargs):
    if gradient.shape != density.shape:
        raise ValueError("Gradient and density must share shape.")
    opt = Optimizer(method=method, learning_rate=learning_rate, options=kwargs) if optimizer_state is None \
        else optimizer_state["optimizer"]
    return np.clip(density + opt.step(gradient), 0.0, 1.0), {"optimizer": opt}


def update_design_region_material(design_region, density) -> None:
    material = getattr(design_region, "material", None)
    if material is None or not hasattr(material, "update_grid"):
        return
    material.update_grid("permittivity", np.interp(density, [0.0, 1.0], [_background_eps(), _target_eps()]))


def _normalize_to_unit_interval(values):
    lo, hi = values.min(), values.max()
    return np.zeros_like(values) if np.isclose(lo, hi) else (values - lo) / (hi - lo)


def _resample_to_shape(grid, shape):
    ny, nx = shape
    ys, yd = np.linspace(0.0, 1.0, grid.shape[0]), np.linspace(0.0, 1.0, ny)
    xs, xd = np.linspace(0.0, 1.0, grid.shape[1]), np.linspace(0.0, 1.0, nx)
    tmp = np.stack([np.interp(yd, ys, grid[:, c]) for c in range(grid.shape[1])], axis=1)
    out = np.stack([np.interp(xd, xs, tmp[r, :]) for r in range(ny)], axis=0)
    return _normalize_to_unit_interval(out)


def _background_eps() -> float:
    return 1.444 ** 2


def _target_eps() -> float:
    return 2.25 ** 2


def _extract_field(container, key):
    if container is None:
        return None
    if isinstance(container, dict):
        v = container.get(key)
        return v[-1] if isinstance(v, list) and v else v
    return getattr(container, key, None)
