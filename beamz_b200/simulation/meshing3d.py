"""3D rasterisation (beamz/simulation/meshing.py:569-893)."""
from __future__ import annotations


def init_regular_grid_3d(grid, design, resolution_xy=None, resolution_z=None, **kwargs):
    raise NotImplementedError("3D meshing is provided by a later module of beamz_b200")
