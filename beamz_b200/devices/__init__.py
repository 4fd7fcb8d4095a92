"""Sources, monitors, mode solvers and time signals."""
from .mode import compute_derivative_matrices, slab_mode_source, solve_modes
from .monitors import Monitor
from .signals import cosine, gaussian, gaussian_pulse, plot_signal, ramped_cosine, sigmoid
from .sources import GaussianSource, ModeSource

__all__ = ["GaussianSource", "ModeSource", "Monitor", "solve_modes", "slab_mode_source",
           "compute_derivative_matrices", "ramped_cosine", "gaussian_pulse", "gaussian", "cosine", "sigmoid",
           "plot_signal"]
