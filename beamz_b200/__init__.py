"""beamz_b200 — B200-native FDTD stepping with the beamz design/simulation API.

``from beamz_b200 import *`` exports the same names as ``from beamz import *`` for
the simulation path (constants, materials, structures, sources, monitors,
signals, mode solvers, RegularGrid, FDTD, get_backend, Optimizer,
compute_overlap_gradient, calc_optimal_fdtd_params). Plotting and rich-console
helpers of the reference are not part of this package.
"""
from .const import EPS_0, LIGHT_SPEED, MU_0, VAC_PERMEABILITY, VAC_PERMITTIVITY, nm, um, µm, μm
from .design import CustomMaterial, Design, Material, Circle, CircularBend, Polygon, Rectangle, Ring, Taper
from .devices import GaussianSource, ModeSource, Monitor, gaussian_pulse, ramped_cosine, slab_mode_source, solve_modes
from .devices.signals import plot_signal
from .helpers import calc_optimal_fdtd_params, check_fdtd_stability, display_status, get_si_scale_and_label
from .optimization.optimizers import Optimizer
from .optimization.topology import compute_overlap_gradient
from .simulation import FDTD, RegularGrid, RegularGrid3D, get_backend

__version__ = "0.1.0"

__all__ = ["LIGHT_SPEED", "VAC_PERMITTIVITY", "VAC_PERMEABILITY", "EPS_0", "MU_0", "um", "nm", "µm", "μm",
           "Material", "CustomMaterial", "Design", "Rectangle", "Circle", "Ring", "CircularBend", "Polygon",
           "Taper", "ModeSource", "GaussianSource", "Monitor", "ramped_cosine", "gaussian_pulse", "plot_signal",
           "solve_modes", "slab_mode_source", "RegularGrid", "RegularGrid3D", "FDTD", "get_backend", "Optimizer",
           "compute_overlap_gradient", "display_status", "get_si_scale_and_label", "calc_optimal_fdtd_params",
           "check_fdtd_stability"]
