"""Graded-conductivity absorbing boundary regions (beamz/design/pml.py:5-74).

A boundary is a rectangle strip ("left", "right", "top", "bottom") or a quarter
disc at a domain corner. Its conductivity at a point is
``sigma_max * profile(d) / (1 + alpha_max * d**2)`` with
``sigma_max = sigma_factor * 1.2 / (eta * dx)``, ``eta = sqrt(mu0 / (eps0 * eps))`` and
``d`` the normalised depth into the layer. The profile is quadratic up to d = 0.05
(reaching 0.01) and ``((d - 0.05) / 0.95) ** polynomial_order`` beyond.
"""
from __future__ import annotations

import numpy as np

from ..const import EPS_0, MU_0


class PML:
    def __init__(self, region_type, position, size, orientation, polynomial_order=2.0, sigma_factor=1.0,
                 alpha_max=0.1):
        self.region_type = region_type
        self.position = position
        self.orientation = orientation
        self.polynomial_order = polynomial_order
        self.sigma_factor = sigma_factor
        self.alpha_max = alpha_max
        if region_type == "rect":
            self.width, self.height = size
        else:
            self.radius = size

    def get_profile(self, normalized_distance):
        d = min(max(normalized_distance, 0.0), 1.0)
        if d < 0.05:
            sigma = 0.01 * (d / 0.05) ** 2
        else:
            sigma = ((d - 0.05) / 0.95) ** self.polynomial_order
        return sigma, self.alpha_max * d ** 2

    def depth_at(self, x, y):
        """Normalised depth d of (x, y) into the layer, or None outside it."""
        if self.region_type == "rect":
            px, py = self.position[0], self.position[1]
            if not (px <= x <= px + self.width and py <= y <= py + self.height):
                return None
            o = self.orientation
            if o == "left":
                return 1.0 - (x - px) / self.width
            if o == "right":
                return (x - px) / self.width
            if o == "top":
                return (y - py) / self.height
            if o == "bottom":
                return 1.0 - (y - py) / self.height
            return None
        r = np.hypot(x - self.position[0], y - self.position[1])
        if r > self.radius:
            return None
        dx, dy = x - self.position[0], y - self.position[1]
        o = self.orientation
        if (o == "top-left" and (dx > 0 or dy < 0)) or (o == "top-right" and (dx < 0 or dy < 0)) or \
                (o == "bottom-left" and (dx > 0 or dy > 0)) or (o == "bottom-right" and (dx < 0 or dy > 0)):
            return None
        return r / self.radius

    def profile_factors(self, x, y, with_dt=True):
        """(profile, frequency_factor) at a point, or None where the layer adds nothing.

        This is the position-only part of :meth:`get_conductivity`; the GPU
        rasteriser multiplies it by the eps-dependent sigma_max per cell.
        """
        d = self.depth_at(x, y)
        if d is None:
            return None
        s, a = self.get_profile(d)
        return s, (1.0 / (1.0 + a) if with_dt else 1.0)

    def get_conductivity(self, x, y, dx=None, dt=None, eps_avg=None):
        if dx is not None and eps_avg is not None:
            eta = np.sqrt(MU_0 / (EPS_0 * eps_avg))
            sigma_max = 1.2 / (eta * dx)
            sigma_max *= self.sigma_factor
        else:
            sigma_max = 1.0
        pf = self.profile_factors(x, y, with_dt=dt is not None)
        if pf is None:
            return 0.0
        conductivity = sigma_max * pf[0]
        if dt is not None:
            conductivity *= pf[1]
        return conductivity

    def copy(self):
        size = (self.width, self.height) if self.region_type == "rect" else self.radius
        return PML(self.region_type, self.position, size, self.orientation, self.polynomial_order, self.sigma_factor,
                   self.alpha_max)

    def add_to_plot(self, *args, **kwargs):
        raise NotImplementedError("plotting is not part of beamz_b200")
