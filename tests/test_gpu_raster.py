"""GPU rasteriser against the reference's RegularGrid output (golden fixtures).

eps and mu are compared bit for bit (the kernel reproduces every sample test
and blend with identically rounded float64 operations); sigma includes the PML
pass, whose eps-dependent factor is also bit-reproducible, so it is compared
bit for bit too."""
import numpy as np
import pytest

import designs as D

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,builder", [("shapes", D.raster_shapes), ("pml_only", D.raster_pml_only)])
def test_rasterizer_bit_exact(bz, golden, name, builder):
    g = golden(f"raster_{name}")
    grid = bz.RegularGrid(builder(bz), D.RES)
    assert grid.permittivity.shape == g["eps"].shape
    np.testing.assert_array_equal(grid.permittivity, g["eps"])
    np.testing.assert_array_equal(grid.permeability, g["mu"])
    np.testing.assert_array_equal(grid.conductivity, g["sigma"])


def test_rasterizer_shapes_nontrivial(bz):
    grid = bz.RegularGrid(D.raster_shapes(bz), D.RES)
    assert len(np.unique(grid.permittivity)) > 30
    assert (grid.conductivity > 0).sum() > 500


def test_custom_material_raster_bit_exact(bz, golden):
    """CustomMaterial rectangles (function- and grid-defined properties) against the
    reference's RegularGrid output."""
    import designs as D

    g = golden("raster_custom")
    grid = bz.RegularGrid(D.raster_custom(bz), D.RES)
    np.testing.assert_array_equal(grid.permittivity, g["eps"])
    np.testing.assert_array_equal(grid.permeability, g["mu"])
    np.testing.assert_array_equal(grid.conductivity, g["sigma"])
