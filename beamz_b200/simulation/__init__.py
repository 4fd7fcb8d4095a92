"""Meshing, the FDTD simulation object and the backend registry."""
from .backends import get_backend
from .fdtd import FDTD
from .meshing import RegularGrid, RegularGrid3D

__all__ = ["RegularGrid", "RegularGrid3D", "FDTD", "get_backend"]
