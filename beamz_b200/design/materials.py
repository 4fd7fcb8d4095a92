"""Materials (beamz/design/materials.py:1-217).

``Material`` is a constant (eps_r, mu_r, sigma) triple. ``CustomMaterial`` gives
spatially varying values from callables or from grids interpolated with
``scipy.interpolate.RegularGridInterpolator`` over ``bounds``; the rasteriser
evaluates it at cell centres on the host and hands the table to the GPU.
"""
from __future__ import annotations

import numpy as np


class Material:
    def __init__(self, permittivity=1.0, permeability=1.0, conductivity=0.0):
        self.permittivity = permittivity
        self.permeability = permeability
        self.conductivity = conductivity

    def get_sample(self):
        return self.permittivity, self.permeability, self.conductivity

    def __repr__(self):
        return f"Material(eps={self.permittivity}, mu={self.permeability}, sigma={self.conductivity})"


_PROPS = ("permittivity", "permeability", "conductivity")


class CustomMaterial:
    """Function- or grid-defined material for inverse design.

    Each property is taken, in order of precedence, from ``<prop>_func(x, y[, z])``,
    from the interpolated ``<prop>_grid`` (rows = y, columns = x, spanning
    ``bounds = ((x_min, x_max), (y_min, y_max))``), or from the default
    (1, 1, 0). Out-of-bounds grid lookups return the default.
    """

    def __init__(self, permittivity_func=None, permeability_func=None, conductivity_func=None,
                 permittivity_grid=None, permeability_grid=None, conductivity_grid=None,
                 bounds=None, interpolation="linear"):
        self.permittivity_func = permittivity_func
        self.permeability_func = permeability_func
        self.conductivity_func = conductivity_func
        self.permittivity_grid = permittivity_grid
        self.permeability_grid = permeability_grid
        self.conductivity_grid = conductivity_grid
        self.bounds = bounds
        self.interpolation = interpolation
        self.default_permittivity = 1.0
        self.default_permeability = 1.0
        self.default_conductivity = 0.0
        for prop in _PROPS:
            if getattr(self, f"{prop}_grid") is not None and bounds is not None:
                self._create_grid_interpolator(prop)

    def _summary(self, prop):
        grid = getattr(self, f"{prop}_grid")
        if grid is not None:
            return f"grid({np.min(grid):.3f}-{np.max(grid):.3f})"
        if getattr(self, f"{prop}_func") is not None:
            return "function"
        return getattr(self, f"default_{prop}")

    permittivity = property(lambda self: self._summary("permittivity"))
    permeability = property(lambda self: self._summary("permeability"))
    conductivity = property(lambda self: self._summary("conductivity"))

    def _create_grid_interpolator(self, prop):
        from scipy.interpolate import RegularGridInterpolator

        grid = getattr(self, f"{prop}_grid")
        if grid is None:
            return
        xs = np.linspace(self.bounds[0][0], self.bounds[0][1], grid.shape[1])
        ys = np.linspace(self.bounds[1][0], self.bounds[1][1], grid.shape[0])
        interp = RegularGridInterpolator((ys, xs), grid, method=self.interpolation, bounds_error=False,
                                         fill_value=getattr(self, f"default_{prop}"))
        setattr(self, f"_{prop}_interpolator", interp)

    def _get(self, prop, x, y, z=None):
        fn = getattr(self, f"{prop}_func")
        if fn is not None:
            return fn(x, y, z) if z is not None else fn(x, y)
        interp = getattr(self, f"_{prop}_interpolator", None)
        if interp is not None:
            return interp(np.column_stack([np.atleast_1d(y), np.atleast_1d(x)]))
        return getattr(self, f"default_{prop}")

    def get_permittivity(self, x, y, z=None):
        return self._get("permittivity", x, y, z)

    def get_permeability(self, x, y, z=None):
        return self._get("permeability", x, y, z)

    def get_conductivity(self, x, y, z=None):
        return self._get("conductivity", x, y, z)

    def get_sample(self, x=0, y=0, z=None):
        return self.get_permittivity(x, y, z), self.get_permeability(x, y, z), self.get_conductivity(x, y, z)

    def update_grid(self, property_name, new_grid):
        if property_name not in _PROPS:
            raise ValueError(f"Unknown property: {property_name}")
        setattr(self, f"{property_name}_grid", new_grid)
        self._create_grid_interpolator(property_name)

    def copy(self):
        grids = {f"{p}_grid": (None if getattr(self, f"{p}_grid") is None else getattr(self, f"{p}_grid").copy())
                 for p in _PROPS}
        return CustomMaterial(permittivity_func=self.permittivity_func, permeability_func=self.permeability_func,
                              conductivity_func=self.conductivity_func, bounds=self.bounds,
                              interpolation=self.interpolation, **grids)


def material_triple(material, x=0.0, y=0.0, z=0.0):
    """(eps, mu, sigma) of a material at a point, as meshing.py:21-56 resolves it.

    A CustomMaterial whose evaluation raises falls back to its defaults, like the
    reference; an object with neither getters nor attributes is vacuum.
    """
    if material is None:
        return 1.0, 1.0, 0.0
    if hasattr(material, "get_permittivity"):
        try:
            vals = [material.get_permittivity(x, y, z), material.get_permeability(x, y, z),
                    material.get_conductivity(x, y, z)]
            return tuple(v.item() if hasattr(v, "item") else v for v in vals)
        except Exception:  # noqa: BLE001 - same fallback as the reference
            return (getattr(material, "default_permittivity", 1.0), getattr(material, "default_permeability", 1.0),
                    getattr(material, "default_conductivity", 0.0))
    if hasattr(material, "permittivity"):
        return (getattr(material, "permittivity", 1.0), getattr(material, "permeability", 1.0),
                getattr(material, "conductivity", 0.0))
    return 1.0, 1.0, 0.0
