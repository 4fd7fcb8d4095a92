"""Learned surrogate of the topology objective: a Fourier neural operator on the
library's bf16 kernels, its FDTD-generated training data, and the
surrogate-proposal / FDTD-verification optimisation loop."""
from .fno import FNO2d, spectral_bases

__all__ = ["FNO2d", "spectral_bases"]
