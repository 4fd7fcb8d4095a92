"""The design container (beamz/design/core.py:15-607).

A Design holds, in painter's order, a background rectangle followed by the
structures, sources and monitors added to it, plus the absorbing boundaries.
With ``auto_pml`` it adds four edge strips and four corner regions of
thickness ``pml_size`` and four display-only rectangles flagged ``is_pml``.
GDS import/export (core.py:445-553) reads and writes the GDSII stream itself
(``design/gds.py``); polygon union (core.py:159-440) needs shapely and is not provided.
"""
from __future__ import annotations

import random

import numpy as np

from ..const import µm
from ..helpers import display_status
from .materials import Material
from .pml import PML
from .structures import Circle, CircularBend, Polygon, Rectangle, Ring


class Design:
    def __init__(self, width=5 * µm, height=5 * µm, depth=0, material=None, color=None, border_color="black",
                 auto_pml=True, pml_size=None):
        if material is None:
            material = Material(permittivity=1.0, permeability=1.0, conductivity=0.0)
        self.structures = [Rectangle(position=(0, 0, 0), width=width, height=height, depth=depth, material=material,
                                     color=color)]
        self.sources = []
        self.monitors = []
        self.boundaries = []
        self.width = width
        self.height = height
        self.depth = depth
        self.border_color = border_color
        self.time = 0
        self.layers: dict = {}
        self.is_3d = not (depth is None or depth == 0)
        if auto_pml:
            self._init_boundaries(pml_size)
        display_status(f"Created design with size: {self.width:.2e} x {self.height:.2e} m")

    def __str__(self):
        return f"Design with {len(self.structures)} structures ({'3D' if self.is_3d else '2D'})"

    def __iadd__(self, structure):
        self.add(structure)
        return self

    def _init_boundaries(self, pml_size=None):
        if pml_size is None:
            eps_max = 1.0
            for s in self.structures:
                if hasattr(s, "material") and hasattr(s.material, "permittivity"):
                    eps_max = max(eps_max, s.material.permittivity)
            lam = 1.55e-6 / np.sqrt(eps_max)
            pml_size = max(1.5 * lam, min(min(self.width, self.height) * 0.3, min(self.width, self.height) / 3))
        W, H = self.width, self.height
        self.boundaries += [
            PML("rect", (0, 0), (pml_size, H), "left"),
            PML("rect", (W - pml_size, 0), (pml_size, H), "right"),
            PML("rect", (0, H - pml_size), (W, pml_size), "top"),
            PML("rect", (0, 0), (W, pml_size), "bottom"),
            PML("corner", (0, 0), pml_size, "bottom-left"),
            PML("corner", (W, 0), pml_size, "bottom-right"),
            PML("corner", (0, H), pml_size, "top-left"),
            PML("corner", (W, H), pml_size, "top-right"),
        ]
        vac = Material(permittivity=1.0, permeability=1.0, conductivity=0.0)
        for pos, w, h in [((0, 0), pml_size, H), ((W - pml_size, 0), pml_size, H), ((0, 0), W, pml_size),
                          ((0, H - pml_size), W, pml_size)]:
            self.structures.append(Rectangle(position=pos, width=w, height=h, material=vac, color="none",
                                             is_pml=True))

    def add(self, structure):
        from ..devices.monitors import Monitor
        from ..devices.sources import GaussianSource, ModeSource

        if isinstance(structure, (ModeSource, GaussianSource)):
            self.sources.append(structure)
        elif isinstance(structure, Monitor):
            self.monitors.append(structure)
        self.structures.append(structure)
        if hasattr(structure, "depth") and structure.depth != 0:
            self.is_3d = True
        elif hasattr(structure, "position") and len(structure.position) > 2 and structure.position[2] != 0:
            self.is_3d = True
        elif getattr(structure, "vertices", None):
            if any(len(v) > 2 and v[2] != 0 for v in structure.vertices):
                self.is_3d = True

    def scatter(self, structure, n=1000, xyrange=(-5 * µm, 5 * µm), scale_range=(0.05, 1)):
        for _ in range(n):
            s = structure.copy()
            s.shift(random.uniform(*xyrange), random.uniform(*xyrange))
            s.rotate(random.uniform(0, 360))
            s.scale(random.uniform(*scale_range))
            self.add(s)

    def get_material_value(self, x, y, z=0, dx=None, dt=None):
        """Material of the topmost structure containing (x, y), plus PML conductivity
        when ``dx`` is given (core.py:399-443).

        As in the reference every Polygon subclass (rectangles, circles, rings,
        bends, and the vacuum display rectangles of the PML strips) is tested
        with its vertex polygon, and a material is sampled without coordinates.
        """
        eps, mu, sig = 1.0, 1.0, 0.0
        for s in reversed(self.structures):
            if isinstance(s, Polygon) and s.point_in_polygon(x, y, z):
                eps, mu, sig = s.material.get_sample()
                break
        pml = 0.0
        if dx is not None:
            for b in self.boundaries:
                pml += b.get_conductivity(x, y, dx=dx, dt=dt, eps_avg=eps)
        return [eps, mu, sig + pml]

    def copy(self):
        bg = self.structures[0].material if self.structures and hasattr(self.structures[0], "material") else None
        new = Design(width=self.width, height=self.height, material=bg, auto_pml=False)
        new.structures, new.sources, new.monitors, new.boundaries = [], [], [], []
        from ..devices.monitors import Monitor
        from ..devices.sources import GaussianSource, ModeSource

        for s in self.structures:
            if hasattr(s, "copy"):
                c = s.copy()
                if getattr(c, "material", None) is not None and hasattr(c.material, "copy"):
                    c.material = c.material.copy()
                if hasattr(c, "design"):
                    c.design = new
                new.structures.append(c)
                if isinstance(c, (ModeSource, GaussianSource)):
                    new.sources.append(c)
                elif isinstance(s, Monitor):
                    new.monitors.append(c)
            else:
                new.structures.append(s)
        new.boundaries = [b.copy() if hasattr(b, "copy") else b for b in self.boundaries]
        new.is_3d, new.depth, new.border_color, new.time = self.is_3d, self.depth, self.border_color, self.time
        new.layers = dict(self.layers)
        return new

    def show(self, *args, **kwargs):
        raise NotImplementedError("plotting is not part of beamz_b200")

    def unify_polygons(self):
        raise NotImplementedError("polygon union needs shapely, which beamz_b200 does not use")

    @staticmethod
    def import_gds(gds_file: str, default_depth=1e-6):
        """New Design holding every polygon of the file's flattened top cells
        (core.py:445-478): ``layers[layer]`` lists the polygons of each GDS layer, all
        with ``default_depth`` (a positive depth makes the design 3D). The polygons carry
        no material, as in the reference. Read by ``design/gds.py``."""
        from .gds import read_gds

        design = Design()
        n = 0
        for (layer, _datatype), polys in read_gds(gds_file).items():
            design.layers.setdefault(layer, [])
            for pts in polys:
                poly = Polygon(vertices=[(float(x), float(y)) for x, y in pts], depth=default_depth)
                design.layers[layer].append(poly)
                design.structures.append(poly)
                n += 1
        if default_depth > 0:
            design.is_3d = True
            design.depth = default_depth
        display_status(f"Imported {n} polygons from '{gds_file}' into Design object.")
        return design

    def export_gds(self, output_file):
        """Writes the structures (not sources, monitors or PML strips) as GDS polygons,
        one layer per distinct (permittivity, permeability, conductivity) in order of
        first appearance, as core.py:480-553 does; user unit 1 um, database unit 1 nm,
        cell "main". Unlike the reference, touching polygons of one material are not
        merged first (that union needs shapely); each structure is its own boundary,
        holes written as keyholes."""
        from .gds import write_gds

        groups: dict = {}
        for st in self.structures:
            if getattr(st, "is_pml", False) or not isinstance(st, Polygon):
                continue
            mat = getattr(st, "material", None)
            if mat is None or not st.vertices:
                continue
            key = (getattr(mat, "permittivity", 1.0), getattr(mat, "permeability", 1.0),
                   getattr(mat, "conductivity", 0.0))
            outline = np.asarray([(v[0], v[1]) for v in st.vertices], dtype=float)
            holes = [np.asarray([(v[0], v[1]) for v in h], dtype=float) for h in getattr(st, "interiors", []) if h]
            groups.setdefault(key, []).append((outline, holes))
        write_gds(output_file, {layer: polys for layer, polys in enumerate(groups.values())})
        display_status(f"GDS file saved as '{output_file}' with {len(groups)} material-based layers")
        for layer, key in enumerate(groups):
            display_status(f"Layer {layer}: eps_r={key[0]:.1f}, mu_r={key[1]:.1f}, sigma={key[2]:.2e} S/m")


# Circle, Ring and CircularBend are Polygon subclasses, so get_material_value's
# point_in_polygon test covers them; the names are imported for re-export.
__all__ = ["Design", "Circle", "Ring", "CircularBend"]
