"""Synthetic benchmark workloads: the design, time axis, sources and monitors of
the standard configurations, built through the public API.

* ``dipole_2d``  400x400 cells at 20 nm, vacuum, 20-cell order-3 PML, point-like
  Gaussian source with a Gaussian-pulsed carrier at 1.55 um, 2000 steps, four edge
  line monitors.
* ``mmi_2d``     2000x1000 cells at 20 nm, SiO2 cladding (eps 2.085) with a Si
  (eps 12.25) 1x2 MMI: 500 nm input/output guides, 6 x 3 um body, outputs at
  +-0.75 um; 30-cell PML; CW (ramped cosine) fundamental-mode source at 1.55 um;
  20000 steps; DFT flux monitors at 1.50..1.60 um on the input and both ports.
* ``soi_mmi_3d`` 600x300x150 cells at 20 nm, the SOI strip + MMI stack (see the
  function), 16-cell PML on all faces, 8000 steps.

PML grading: order 3 with sigma_max set for a normal-incidence reflection R = 1e-6,
sigma_max = (m+1) ln(1/R) / (2 eta0 d), d = thickness; expressed through the
PML's ``sigma_factor`` relative to its default 1.2/(eta0 dx).

The 2D/3D builders take ``api``: the namespace whose classes build the design
(default: this package). The same geometry can so be built with the reference
package's own Design/Rectangle/ModeSource/Monitor classes, which have the same
constructors; its Monitor has no DFT, so ``wavelengths`` is passed only to a
Monitor that accepts it. This module imports nothing from the package at module
level, so it can be loaded by path without loading the native library.
"""
from __future__ import annotations

import inspect

import numpy as np

UM = 1e-6


def _api(api):
    if api is None:
        import beamz_b200 as api
    return api


def _signal(api, name):
    fn = getattr(api, name, None)
    if fn is None:  # the reference exports gaussian_pulse from its signals module only
        import importlib

        fn = getattr(importlib.import_module(api.__name__ + ".devices.signals"), name)
    return fn


def _monitor(api, wavelengths=None, **kw):
    if wavelengths is not None and "wavelengths" in inspect.signature(api.Monitor.__init__).parameters:
        kw["wavelengths"] = wavelengths
    elif "record_fields" in kw and wavelengths is not None:
        kw["record_fields"] = True  # no DFT: the time series carries the same information
    return api.Monitor(**kw)


def pml_sigma_factor(n_cells: int, order: int = 3, reflection: float = 1e-6) -> float:
    """sigma_factor giving sigma_max = (m+1) ln(1/R) / (2 eta0 n dx) (eta0 cancels)."""
    return (order + 1) * np.log(1.0 / reflection) / (2.0 * n_cells) / 1.2


def _grade(design, n_cells):
    for b in design.boundaries:
        b.polynomial_order = 3
        b.sigma_factor = pml_sigma_factor(n_cells)
    return design


def courant_dt(dx, dims=2):
    return 0.99 * dx / (299792458.0 * np.sqrt(dims))


def dipole_2d(n=400, dx=0.02 * UM, n_steps=2000, pml=20, api=None, monitors=True):
    bz = _api(api)
    W = (n + 0.5) * dx
    d = _grade(bz.Design(width=W, height=W, material=bz.Material(1.0), pml_size=pml * dx), pml)
    t = np.arange(n_steps) * courant_dt(dx)
    sig = _signal(bz, "gaussian_pulse")(t, 1.0, 3 * 10e-15, 10e-15, bz.LIGHT_SPEED / (1.55 * UM), 0.0)
    d += bz.GaussianSource(position=(n // 2 * dx, n // 2 * dx), width=dx / 10, signal=sig)
    if monitors:
        k = (pml + 10) * dx
        lo, hi = k, (n - pml - 10) * dx
        mons = [bz.Monitor(design=d, start=(lo, lo), end=(lo, hi), name="left"),
                bz.Monitor(design=d, start=(hi, lo), end=(hi, hi), name="right"),
                bz.Monitor(design=d, start=(lo, lo), end=(hi, lo), name="bottom"),
                bz.Monitor(design=d, start=(lo, hi), end=(hi, hi), name="top")]
        for m in mons:
            d += m
    return d, t, dx


MMI_WAVELENGTHS = np.array([1.50, 1.525, 1.55, 1.575, 1.60]) * UM


def mmi_2d(nx=2000, ny=1000, dx=0.02 * UM, n_steps=20000, pml=30, mode_solver="num_eigen", api=None, monitors=True):
    bz = _api(api)
    µm = UM
    W, H = (nx + 0.5) * dx, (ny + 0.5) * dx
    d = _grade(bz.Design(width=W, height=H, material=bz.Material(2.085), pml_size=pml * dx), pml)
    yc, xc = H / 2, W / 2
    si = bz.Material(12.25)
    wg, L, B, off = 0.5 * µm, 6.0 * µm, 3.0 * µm, 0.75 * µm
    d += bz.Rectangle(position=(0, yc - wg / 2), width=xc - L / 2, height=wg, material=si)
    d += bz.Rectangle(position=(xc - L / 2, yc - B / 2), width=L, height=B, material=si)
    for s in (+1, -1):
        d += bz.Rectangle(position=(xc + L / 2, yc + s * off - wg / 2), width=W - (xc + L / 2), height=wg, material=si)
    t = np.arange(n_steps) * courant_dt(dx)
    sig = bz.ramped_cosine(t, amplitude=1.0, frequency=bz.LIGHT_SPEED / (1.55 * µm), phase=0,
                           ramp_duration=20 * 1.55 * µm / bz.LIGHT_SPEED, t_max=t[-1] * 2)
    x_src = pml * dx + 1.0 * µm
    d += bz.ModeSource(design=d, position=(x_src, yc), width=2.0 * µm, wavelength=1.55 * µm, signal=sig,
                       direction="+x", num_modes=1, mode_solver=mode_solver)
    if monitors:
        x_in, x_out = x_src + 1.0 * µm, W - pml * dx - 1.0 * µm
        mons = [_monitor(bz, design=d, start=(x_in, yc - 1.0 * µm), end=(x_in, yc + 1.0 * µm), name="in",
                         wavelengths=MMI_WAVELENGTHS, record_fields=False, accumulate_power=False)]
        for s, name in ((+1, "port_top"), (-1, "port_bottom")):
            y0 = yc + s * off
            mons.append(_monitor(bz, design=d, start=(x_out, y0 - 0.6 * µm), end=(x_out, y0 + 0.6 * µm), name=name,
                                 wavelengths=MMI_WAVELENGTHS, record_fields=False, accumulate_power=False))
        for m in mons:
            d += m
    return d, t, dx


def soi_mmi_3d(nx=600, ny=300, nz=150, dx=0.02 * UM, n_steps=8000, pml=16, grid_resolution=500,
               mode_solver="num_eigen", api=None, monitors=True):
    """600x300x150 cells at 20 nm: SiO2 box (eps 2.085) / 220 nm Si (eps 12.25) / air,
    500 nm strip into a 6 x 3 um MMI with outputs at +-0.75 um, 16-cell PML on all faces
    (the grid is built with RegularGrid3D(extrude=True)), Gaussian-pulse mode source at
    1.55 um, DFT flux planes at 5 wavelengths on both outputs, 8000 steps.
    ``mode_solver="cross_section"`` takes the source profile from the 2D cross-section
    eigenproblem instead of the reference's separable slab approximation."""
    bz = _api(api)
    µm = UM
    W, H, Dz = (nx + 0.5) * dx, (ny + 0.5) * dx, (nz + 0.5) * dx
    d = _grade(bz.Design(width=W, height=H, depth=Dz, material=bz.Material(1.0), pml_size=pml * dx), pml)
    yc = H / 2
    z_box, t_si = 1.4 * µm, 0.22 * µm
    si, sio2 = bz.Material(12.25), bz.Material(2.085)
    d += bz.Rectangle(position=(0, 0, 0), width=W, height=H, depth=z_box, material=sio2)
    x0, L, B, wg, off = 3.0 * µm, 6.0 * µm, 3.0 * µm, 0.5 * µm, 0.75 * µm
    d += bz.Rectangle(position=(0, yc - wg / 2, z_box), width=x0, height=wg, depth=t_si, material=si)
    d += bz.Rectangle(position=(x0, yc - B / 2, z_box), width=L, height=B, depth=t_si, material=si)
    for s in (+1, -1):
        d += bz.Rectangle(position=(x0 + L, yc + s * off - wg / 2, z_box), width=W - x0 - L, height=wg, depth=t_si,
                          material=si)
    t = np.arange(n_steps) * courant_dt(dx, dims=3)
    sig = _signal(bz, "gaussian_pulse")(t, 1.0, 30e-15, 10e-15, bz.LIGHT_SPEED / (1.55 * µm), 0.0)
    d += bz.ModeSource(design=d, position=(pml * dx + 0.7 * µm, yc, z_box + t_si / 2), width=1.5 * µm,
                       height=1.0 * µm, wavelength=1.55 * µm, signal=sig, direction="+x", num_modes=1,
                       grid_resolution=grid_resolution, mode_solver=mode_solver)
    if monitors:
        x_out = W - pml * dx - 0.8 * µm
        for s, name in ((+1, "port_top"), (-1, "port_bottom")):
            d += _monitor(bz, design=d, start=(0.0, yc + s * off - 0.6 * µm, z_box - 0.4 * µm), plane_normal="x",
                          plane_position=x_out, size=(1.2 * µm, 1.0 * µm), name=name, wavelengths=MMI_WAVELENGTHS,
                          record_fields=False, accumulate_power=False)
    return d, t, dx


def topo_2d(n_designs=64, nx=600, ny=400, dx=0.02 * UM, n_steps=8000, pml=20, region_cells=120, seed=1234,
            mode_points=None, wavelengths=None):
    """Batched topology-optimisation problem: B densities (120x120 cells, uniform in
    [0, 1] then Gaussian-smoothed with sigma = 3 cells, seeds seed+b) mapped to
    eps = 2.085 + rho * (12.25 - 2.085), centred in a 600x400 grid between 500 nm input
    and output Si waveguides in SiO2; CW mode source at 1.55 um; the objective is the
    power in the output guide's fundamental slab mode at 1.55 um (monitor line 1 um
    before the right PML). Returns a dict of AdjointFDTD2D arguments plus rho0 and the
    material mapping.

    With ``wavelengths`` (a list), the source is a Gaussian-pulsed carrier at 1.55 um
    (10 fs width, the signal of the dipole workload) and the objective has one term
    per wavelength, each with the slab mode of that wavelength; ``rho_straight`` is
    then the density of an uninterrupted guide (the transmission reference)."""
    from scipy.ndimage import gaussian_filter

    bz = _api(None)
    from .devices.mode import slab_mode_source
    from .simulation.meshing import RegularGrid

    µm = UM

    W, H = (nx + 0.5) * dx, (ny + 0.5) * dx
    d = _grade(bz.Design(width=W, height=H, material=bz.Material(2.085), pml_size=pml * dx), pml)
    yc = H / 2
    wg = 0.5 * µm
    r = region_cells
    y0, x0 = ny // 2 - r // 2, nx // 2 - r // 2
    d += bz.Rectangle(position=(0, yc - wg / 2), width=x0 * dx, height=wg, material=bz.Material(12.25))
    d += bz.Rectangle(position=((x0 + r) * dx, yc - wg / 2), width=W - (x0 + r) * dx, height=wg,
                   material=bz.Material(12.25))
    t = np.arange(n_steps) * courant_dt(dx)
    f0 = bz.LIGHT_SPEED / (1.55 * µm)
    if wavelengths is None:
        sig = bz.ramped_cosine(t, amplitude=1.0, frequency=f0, phase=0, ramp_duration=20 / f0, t_max=t[-1] * 2)
    else:
        sig = bz.gaussian_pulse(t, 1.0, 3 * 10e-15, 10e-15, f0, 0.0)
    src = bz.ModeSource(design=d, position=(pml * dx + 0.6 * µm, yc), width=2.0 * µm, wavelength=1.55 * µm, signal=sig,
                        direction="+x", num_modes=1)
    # a transparent (soft) line source, as the reference's topology example sets it
    # (examples/4_topo.py:246): with the zeroed cell behind each point the source line
    # reflects returning light, and a design could then pump the mode beyond the straight
    # guide's power
    src.enforce_direction = False
    grid = RegularGrid(d, dx)
    x_mon = (nx - pml - 50) * dx
    mon = bz.Monitor(start=(x_mon, yc - 1.0 * µm), end=(x_mon, yc + 1.0 * µm))
    pts = mon.get_grid_points_2d(dx, dx)
    ys = np.array([p[1] * dx for p in pts]) + 0.5 * dx - yc
    if wavelengths is None:
        mode, _ = slab_mode_source(x=ys, w=wg, n_WG=np.sqrt(12.25), n0=np.sqrt(2.085), wavelength=1.55 * µm,
                                   ind_m=0)
        freq = f0
    else:
        mode = np.stack([slab_mode_source(x=ys, w=wg, n_WG=np.sqrt(12.25), n0=np.sqrt(2.085), wavelength=lam,
                                          ind_m=0)[0] for lam in wavelengths])
        freq = [bz.LIGHT_SPEED / lam for lam in wavelengths]
    import torch

    rho = np.stack([gaussian_filter(torch.rand((r, r), generator=torch.Generator().manual_seed(seed + b),
                                               dtype=torch.float64).numpy(), sigma=3) for b in range(n_designs)])
    straight = np.zeros((r, r))
    rows = (np.arange(r) + y0 + 0.5) * dx
    straight[(rows >= yc - wg / 2) & (rows <= yc + wg / 2), :] = 1.0
    return dict(eps_base=grid.permittivity, sigma=grid.conductivity, dx=dx, dt=t[1] - t[0], n_steps=n_steps,
                sources=[src], monitor=mon, mode_profile=mode, frequency=freq, region=(y0, x0, r, r), rho0=rho,
                eps_lo=2.085, eps_hi=12.25, design=d, rho_straight=straight)


SURROGATE_WAVELENGTHS = [1.50 * UM, 1.525 * UM, 1.55 * UM, 1.575 * UM, 1.60 * UM]


def surrogate_2d(n_designs=64, seed=10000, n_steps=8000, **kw):
    """The topology problem with a pulsed source and the transmission objective at
    1.50, 1.525, 1.55, 1.575 and 1.60 um (the surrogate's outputs); densities from
    seeds seed+b as in topo_2d."""
    return topo_2d(n_designs=n_designs, seed=seed, n_steps=n_steps, wavelengths=SURROGATE_WAVELENGTHS, **kw)
