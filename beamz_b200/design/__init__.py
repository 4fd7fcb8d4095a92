"""Design-side API: materials, structures, PML regions and the Design container."""
from .core import Design
from .materials import CustomMaterial, Material
from .pml import PML
from .structures import Circle, CircularBend, Polygon, Rectangle, Ring, Taper

__all__ = ["Material", "CustomMaterial", "Design", "Rectangle", "Circle", "Ring", "CircularBend", "Polygon",
           "Taper", "PML"]
