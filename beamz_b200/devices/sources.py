"""Sources (beamz/devices/sources.py:7-376).

Sources are set up on the host exactly as in the reference. During stepping
they are not applied point by point: the simulation compiles all sources into
a list of per-cell operations (``compile_injection``), executed on the GPU inside
the step kernel after the E update.
"""
from __future__ import annotations

import numpy as np

from ..const import LIGHT_SPEED, µm
from .mode import slab_mode_source, solve_modes, solve_modes_2d


def _xyz(position):
    if position is None:
        return None
    if len(position) == 2:
        return (position[0], position[1], 0)
    if len(position) == 3:
        return tuple(position)
    raise ValueError(f"Position must be 2D (x,y) or 3D (x,y,z), got {len(position)} dimensions")


class GaussianSource:
    """Soft source: a Gaussian patch (std ``width``) times ``signal[step]`` added to Ez.

    In 2D the patch amplitude is divided by 4 (helper.py:116); in 3D it is not."""

    def __init__(self, position=(0, 0), width=1.0 * µm, signal=0):
        self.position = _xyz(position)
        self.width = width
        self.signal = signal

    @property
    def position_2d(self):
        return (self.position[0], self.position[1])

    def copy(self):
        return GaussianSource(position=self.position, width=self.width, signal=self.signal)

    def add_to_plot(self, *args, **kwargs):
        raise NotImplementedError("plotting is not part of beamz_b200")


_ORIENTATION = {"+x": "yz", "-x": "yz", "+y": "xz", "-y": "xz", "+z": "xy", "-z": "xy"}


class ModeSource:
    """Eigenmode line (2D) or plane (3D) source.

    ``mode_profiles[m]`` is a list of ``[amplitude, x, y, z]`` points; only
    ``mode_profiles[0]`` is injected (helper.py:9). With ``enforce_direction``
    (default True) each injection also zeroes Ez one cell behind the line.
    """

    def __init__(self, design, position=None, width=None, height=None, wavelength=1.55 * µm, signal=0,
                 direction="+x", orientation=None, npml=20, num_modes=2, grid_resolution=2000,
                 mode_solver="num_eigen", start=None, end=None):
        if start is not None and end is not None:
            self.start, self.end = _xyz(start), _xyz(end)
            self._position = tuple((self.start[i] + self.end[i]) / 2 for i in range(3))
            self.width = np.linalg.norm(np.array([self.end[i] - self.start[i] for i in range(3)]))
            self.height = 0
        else:
            if position is None:
                raise ValueError("Either (start, end) or position must be specified")
            self._position = _xyz(position)
            self.width = width if width is not None else wavelength
            self.height = height if height is not None else 0
            self.orientation = orientation if orientation is not None else _ORIENTATION.get(direction, "yz")
            self.start, self.end = self._line_from_position()
        self.wavelength = wavelength
        self.design = design
        self.signal = signal
        self.direction = direction
        self.npml = npml
        self.num_modes = num_modes
        self.grid_resolution = grid_resolution
        self.mode_solver = mode_solver
        self.dL = self.wavelength / grid_resolution
        eps_1d = self.get_eps_1d()
        self.omega = 2 * np.pi * LIGHT_SPEED / self.wavelength
        if mode_solver == "analytical":
            self._analytic_modes(eps_1d)
        else:
            self.effective_indices, self.mode_vectors = solve_modes(eps_1d, self.omega, self.dL, npml=self.npml,
                                                                    m=self.num_modes)
        self.mode_profiles = []
        if self.height and self.height > 0 and mode_solver == "cross_section":
            self.mode_profiles = self._build_3d_cross_section_profiles()
        elif self.height and self.height > 0:
            try:
                self.mode_profiles = self._build_3d_rect_mode_profiles() or []
            except Exception:  # noqa: BLE001 - same fallback as the reference
                self.mode_profiles = []
        if not self.mode_profiles:
            self.mode_profiles = [self.get_xy_mode_line(self.mode_vectors, m)
                                  for m in range(self.mode_vectors.shape[1])]

    def _analytic_modes(self, eps_1d):
        try:
            n = eps_1d.size
            x = np.linspace(0, np.hypot(self.end[0] - self.start[0], self.end[1] - self.start[1]), n)
            n_core, n_clad = np.sqrt(np.max(eps_1d)), np.sqrt(np.min(eps_1d))
            core = np.where(eps_1d > (np.max(eps_1d) * 0.9))[0]
            core_w = (core[-1] - core[0]) * self.dL if len(core) > 0 else 1.0 * self.wavelength
            self.mode_vectors = np.zeros((n, self.num_modes), dtype=complex)
            neff = []
            for m in range(self.num_modes):
                try:
                    E, ne = slab_mode_source(x=x, w=core_w, n_WG=n_core, n0=n_clad, wavelength=self.wavelength,
                                             ind_m=m)
                    self.mode_vectors[:, m] = E
                    neff.append(ne)
                except Exception:  # noqa: BLE001
                    self.mode_vectors[:, m] = 0
                    neff.append(0)
            self.effective_indices = np.array(neff)
        except Exception:  # noqa: BLE001 - reference falls back to the numerical solver
            self.effective_indices, self.mode_vectors = solve_modes(eps_1d, self.omega, self.dL, npml=self.npml,
                                                                    m=self.num_modes)

    def _line_from_position(self):
        x, y, z = self._position
        if self.orientation == "yz":
            return (x, y - self.width / 2, z), (x, y + self.width / 2, z)
        if self.orientation in ("xz", "xy"):
            return (x - self.width / 2, y, z), (x + self.width / 2, y, z)
        raise ValueError(f"Invalid orientation: {self.orientation}. Must be 'xy', 'xz', or 'yz'")

    @property
    def position(self):
        return self._position

    @property
    def position_2d(self):
        return ((self.start[0] + self.end[0]) / 2, (self.start[1] + self.end[1]) / 2)

    def _line(self, n):
        return tuple(np.linspace(self.start[i], self.end[i], n) for i in range(3))

    def get_eps_1d(self):
        n = int(np.hypot(self.end[0] - self.start[0], self.end[1] - self.start[1]) / self.dL)
        xs, ys, zs = self._line(n)
        eps = np.zeros(n)
        for i in range(n):
            eps[i] = self.design.get_material_value(xs[i], ys[i], zs[i])[0]
        return eps

    def get_xy_mode_line(self, vecs, mode_number):
        xs, ys, zs = self._line(vecs.shape[0])
        return [[vecs[j, mode_number], xs[j], ys[j], zs[j]] for j in range(vecs.shape[0])]

    def _build_3d_rect_mode_profiles(self):
        """Separable cross-section profile for 3D plane injection (sources.py:323-376)."""
        x0, y0, z0 = self.position
        dL = self.dL
        ny = max(8, int(round(self.width / dL)))
        nz = max(8, int(round(self.height / dL)))
        ys = np.linspace(y0 - self.width / 2, y0 + self.width / 2, ny)
        zs = np.linspace(z0 - self.height / 2, z0 + self.height / 2, nz)
        eps_y = np.array([self.design.get_material_value(x0, y, z0)[0] for y in ys])
        eps_z = np.array([self.design.get_material_value(x0, y0, z)[0] for z in zs])

        def core_width(coords, eps_line):
            idx = np.where(eps_line >= 0.9 * np.max(eps_line))[0]
            return coords[idx[-1]] - coords[idx[0]] if idx.size > 0 else max(coords[-1] - coords[0], dL)

        try:
            fy, _ = slab_mode_source(x=ys, w=core_width(ys, eps_y), n_WG=np.sqrt(np.max(eps_y)),
                                     n0=np.sqrt(np.min(eps_y)), wavelength=self.wavelength, ind_m=0, x0=y0)
        except Exception:  # noqa: BLE001
            fy = np.ones_like(ys)
        try:
            fz, _ = slab_mode_source(x=zs, w=core_width(zs, eps_z), n_WG=np.sqrt(np.max(eps_z)),
                                     n0=np.sqrt(np.min(eps_z)), wavelength=self.wavelength, ind_m=0, x0=z0)
        except Exception:  # noqa: BLE001
            fz = np.ones_like(zs)
        fy = fy / np.max(np.abs(fy) + 1e-12)
        fz = fz / np.max(np.abs(fz) + 1e-12)
        plane = np.outer(np.abs(fy), np.abs(fz))
        plane /= np.max(plane) + 1e-12
        return [[[plane[iy, iz], x0, y, z] for iy, y in enumerate(ys) for iz, z in enumerate(zs)]]

    def _build_3d_cross_section_profiles(self, max_points=200):
        """Modes of the source plane's own 2D cross-section (``mode_solver="cross_section"``).

        The plane (width x height, orientation yz / xz / xy) is sampled on at most
        ``max_points`` nodes per side; ``solve_modes_2d`` finds ``num_modes`` modes, with
        the semi-vectorial operator for a field along the height axis (z, the injected
        Ez) for x- and y-normal planes and the scalar one for z-normal planes. Each
        profile is scaled to peak 1 and then by (node area / dL^2), so that every grid
        cell receives the same summed amplitude as from the reference's profiles, whose
        points are dL apart. Sets ``effective_indices_2d``."""
        x0, y0, z0 = self.position
        nu = int(min(max_points, max(16, round(self.width / self.dL))))
        nv = int(min(max_points, max(16, round(self.height / self.dL))))
        us = np.linspace(-self.width / 2, self.width / 2, nu)
        vs = np.linspace(-self.height / 2, self.height / 2, nv)
        du, dv = us[1] - us[0], vs[1] - vs[0]
        U, V = np.meshgrid(us, vs, indexing="ij")
        orient = getattr(self, "orientation", "yz")
        if orient == "yz":
            X, Y, Z = np.full_like(U, x0), y0 + U, z0 + V
        elif orient == "xz":
            X, Y, Z = x0 + U, np.full_like(U, y0), z0 + V
        else:
            X, Y, Z = x0 + U, y0 + V, np.full_like(U, z0)
        eps = np.array([[self.design.get_material_value(X[i, j], Y[i, j], Z[i, j])[0] for j in range(nv)]
                        for i in range(nu)], dtype=float)
        neff, modes = solve_modes_2d(eps, self.omega, du, dv, m=max(1, self.num_modes),
                                     polarization="scalar" if orient == "xy" else "v")
        self.effective_indices_2d = neff
        scale = du * dv / self.dL ** 2
        profiles = []
        for mode in modes:
            a = np.real(mode)
            a = a / np.max(np.abs(a)) * scale
            profiles.append(np.stack([a.ravel(), X.ravel(), Y.ravel(), Z.ravel()], axis=1).tolist())
        return profiles

    def copy(self):
        return ModeSource(design=self.design, start=self.start, end=self.end, wavelength=self.wavelength,
                          signal=self.signal, direction=self.direction, npml=self.npml, num_modes=self.num_modes,
                          grid_resolution=self.grid_resolution, mode_solver=self.mode_solver)

    def show(self):
        raise NotImplementedError("plotting is not part of beamz_b200")

    def add_to_plot(self, *args, **kwargs):
        raise NotImplementedError("plotting is not part of beamz_b200")
