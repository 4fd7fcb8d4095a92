"""Stability and parameter helpers (beamz/helpers.py:21-87) plus a quiet status log.

The reference prints rich-formatted panels; this package logs through the
standard ``logging`` module instead (logger ``beamz_b200``) so the stepping loop
stays silent unless the caller enables it.
"""
from __future__ import annotations

import datetime
import logging

import numpy as np

from .const import LIGHT_SPEED

log = logging.getLogger("beamz_b200")


def display_status(message: str, status: str = "info") -> None:
    level = {"error": logging.ERROR, "warning": logging.WARNING}.get(status, logging.INFO)
    log.log(level, message)


def display_parameters(params: dict, title: str = "Parameters") -> None:
    log.info("%s: %s", title, ", ".join(f"{k}={v}" for k, v in params.items()))


def display_time_elapsed(start_time) -> None:
    if start_time is not None:
        log.info("elapsed %s", datetime.datetime.now() - start_time)


def get_si_scale_and_label(value):
    if value >= 1e-3:
        return 1e3, "mm"
    if value >= 1e-6:
        return 1e6, "µm"
    if value >= 1e-9:
        return 1e9, "nm"
    return 1e12, "pm"


def check_fdtd_stability(dt, dx, dy=None, dz=None, n_max=1.0, safety_factor=1.0):
    """CFL check with the vacuum speed of light (helpers.py:21-53).

    Returns ``(is_stable, courant_number, limit)`` where the limit is
    ``safety_factor / sqrt(dims)`` and dims counts the spacings given.
    """
    spacings = [s for s in (dx, dy, dz) if s is not None]
    if dz is not None and dy is None:
        spacings = [dx, dz]
    dims = len(spacings)
    courant = LIGHT_SPEED * dt / min(spacings)
    limit = safety_factor * (1.0 / np.sqrt(dims))
    return courant <= limit, courant, limit


def calc_optimal_fdtd_params(wavelength, n_max, dims=2, safety_factor=0.999, points_per_wavelength=10):
    """Grid spacing and time step for a wavelength and peak index (helpers.py:55-87).

    resolution = (wavelength / n_max) / points_per_wavelength and
    dt = safety_factor * resolution / (c * sqrt(dims)).
    """
    resolution = (wavelength / n_max) / points_per_wavelength
    dt = safety_factor * (resolution / (LIGHT_SPEED * np.sqrt(dims)))
    _, courant, limit = check_fdtd_stability(
        dt, resolution, dy=resolution if dims >= 2 else None, dz=resolution if dims >= 3 else None, n_max=n_max
    )
    if courant > limit + 1e-15:
        raise AssertionError("time step exceeds the stability limit")
    return resolution, dt
