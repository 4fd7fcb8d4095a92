"""Design builders shared by the golden-fixture generator and the tests.

Each builder takes a module namespace ``bz`` that provides the beamz API (the
reference package when fixtures are generated, ``beamz_b200`` in the tests) and
builds the same design with the same calls, so both sides rasterise and step
identical inputs.
"""
from __future__ import annotations

import numpy as np

from pathlib import Path

HERE = Path(__file__).resolve().parent
UM = 1e-6
RES = 0.05 * UM  # 50 nm cells keep the fixtures small


def raster_shapes(bz):
    """Every rasteriser path: rectangle fast path (with partial cells), circle,
    ring, circular bend (ring path), taper and negative-height rectangle (polygon
    path), polygon with a hole, order-3 PML with a sigma factor."""
    d = bz.Design(width=3.02 * UM, height=2.51 * UM, material=bz.Material(2.085), pml_size=0.4 * UM)
    d += bz.Rectangle(position=(0.0, 1.13 * UM), width=1.6 * UM, height=0.27 * UM, material=bz.Material(12.25))
    d += bz.Circle(position=(2.1 * UM, 0.9 * UM), radius=0.33 * UM, material=bz.Material(6.0))
    d += bz.Ring(position=(1.2 * UM, 0.75 * UM), inner_radius=0.21 * UM, outer_radius=0.42 * UM,
                 material=bz.Material(9.0, 1.0, 0.0))
    d += bz.CircularBend(position=(2.4 * UM, 2.0 * UM), inner_radius=0.2 * UM, outer_radius=0.35 * UM, angle=120,
                         rotation=30, material=bz.Material(4.0))
    d += bz.Taper(position=(0.55 * UM, 1.95 * UM), input_width=0.5 * UM, output_width=0.12 * UM,
                  length=0.9 * UM, material=bz.Material(7.5))
    d += bz.Rectangle(position=(1.9 * UM, 2.4 * UM), width=0.3 * UM, height=-0.6 * UM, material=bz.Material(3.3))
    d += bz.Polygon(vertices=[(0.3 * UM, 0.3 * UM), (1.0 * UM, 0.45 * UM), (0.85 * UM, 0.95 * UM),
                              (0.35 * UM, 0.8 * UM)],
                    interiors=[[(0.5 * UM, 0.5 * UM), (0.7 * UM, 0.55 * UM), (0.6 * UM, 0.7 * UM)]],
                    material=bz.Material(5.0, 1.0, 0.0))
    d += bz.Rectangle(position=(1.45 * UM, 0.12 * UM), width=0.37 * UM, height=0.33 * UM,
                      material=bz.Material(2.5, 1.0, 1e3))
    for b in d.boundaries:
        b.polynomial_order = 3
        b.sigma_factor = 1.151
    return d


def raster_custom(bz):
    """CustomMaterial on the rectangle path: a function-defined permittivity and
    conductivity, and a grid-defined permittivity interpolated over its bounds, next to a
    plain rectangle; default automatic PML."""
    d = bz.Design(width=2.51 * UM, height=2.02 * UM, material=bz.Material(2.085), pml_size=0.3 * UM)
    f = bz.CustomMaterial(permittivity_func=lambda x, y, z=0: 2.0 + 1.5 * np.sin(x / (0.31 * UM)) ** 2
                          + 0.7 * np.cos(y / (0.17 * UM)),
                          conductivity_func=lambda x, y, z=0: 50.0 * (x / UM) * (y / UM))
    d += bz.Rectangle(position=(0.42 * UM, 0.37 * UM), width=0.93 * UM, height=0.61 * UM, material=f)
    grid = 3.0 + np.add.outer(np.linspace(0.0, 2.0, 7), np.linspace(0.0, 5.0, 9))
    g = bz.CustomMaterial(permittivity_grid=grid, bounds=((1.2 * UM, 2.1 * UM), (1.0 * UM, 1.7 * UM)))
    d += bz.Rectangle(position=(1.18 * UM, 0.97 * UM), width=0.96 * UM, height=0.77 * UM, material=g)
    d += bz.Rectangle(position=(0.2 * UM, 1.5 * UM), width=0.7 * UM, height=0.21 * UM, material=bz.Material(9.0))
    return d


def raster_pml_only(bz):
    """Vacuum box with the default (order-2) automatic PML."""
    return bz.Design(width=2.0 * UM, height=1.5 * UM, pml_size=0.35 * UM)


def wg_design(bz):
    """Straight Si waveguide in SiO2 for the stepping fixtures."""
    d = bz.Design(width=2.4 * UM, height=2.0 * UM, material=bz.Material(2.085), pml_size=0.4 * UM)
    d += bz.Rectangle(position=(0.0, 0.8 * UM), width=2.4 * UM, height=0.4 * UM, material=bz.Material(12.25))
    return d


def time_axis(bz, n_steps, res=RES):
    dt = 0.99 * res / (bz.LIGHT_SPEED * np.sqrt(2))
    return np.arange(n_steps) * dt


def gauss_signal(bz, t):
    return bz.gaussian_pulse(t, 1.0, 6e-15, 2e-15, bz.LIGHT_SPEED / (1.55 * UM), 0.0) \
        if hasattr(bz, "gaussian_pulse") else None


def cw_signal(bz, t):
    return bz.ramped_cosine(t, amplitude=1.0, frequency=bz.LIGHT_SPEED / (1.55 * UM), phase=0,
                            ramp_duration=5e-15, t_max=t[-1])


def design_3d(bz):
    """Small 3D stack: substrate slab, strip waveguide, a disc (3D rasteriser paths)."""
    d = bz.Design(width=1.5 * UM, height=1.2 * UM, depth=0.8 * UM, material=bz.Material(1.0), pml_size=0.2 * UM)
    d += bz.Rectangle(position=(0, 0, 0), width=1.5 * UM, height=1.2 * UM, depth=0.4 * UM, material=bz.Material(2.085))
    d += bz.Rectangle(position=(0, 0.45 * UM, 0.4 * UM), width=1.5 * UM, height=0.3 * UM, depth=0.22 * UM,
                      material=bz.Material(12.25))
    d += bz.Circle(position=(1.0 * UM, 0.6 * UM, 0.4 * UM), radius=0.2 * UM, material=bz.Material(6.0))
    return d


def step3d_design(bz):
    return bz.Design(width=0.85 * UM, height=0.75 * UM, depth=0.65 * UM, material=bz.Material(1.0), pml_size=0.1 * UM)


def step3d_arrays(shape, seed=5):
    rng = np.random.default_rng(seed)
    nz, ny, nx = shape
    zz, yy, xx = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    eps = 1.0 + 5.0 * (1 + np.sin(0.7 * xx + 0.3 * yy) * np.cos(0.5 * zz)) + rng.random(shape)
    sig = np.zeros(shape)
    for a, n in ((xx, nx), (yy, ny), (zz, nz)):
        d = np.maximum(0, np.maximum(3 - a, a - (n - 4))) / 3.0
        sig += 4e4 * d ** 3
    return eps, sig
