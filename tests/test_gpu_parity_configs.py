"""The benchmark configurations against the CPU oracle (the reference's float64 NumPy
loop restated in oracle/): GPU fields after N steps, relative L2 over all field
components, at the tolerances the design states for each precision:
float64 <= 1e-11, float32 <= 1e-5.

* 2D dipole (400 x 400, 20-cell PML, Gaussian-pulsed point source): the full grid and
  the full 2000 steps.
* 2D MMI (2000 x 1000, 30-cell PML, CW mode source): the full grid for 200 steps.
* 3D SOI MMI stack, reduced (120 x 64 x 40 cells: SiO2 box, 220 nm Si strip into an
  MMI, air; 8-cell PML on all faces; Gaussian-pulse mode source), extruded grid,
  250 steps.

The measured errors are printed (``pytest -s``) and carried in the assertion messages.
"""
import numpy as np
import pytest

from oracle import fdtd2d, fdtd3d, raster2d, raster3d

pytestmark = pytest.mark.gpu


def _rel(pairs):
    num = sum(float(np.linalg.norm(np.asarray(a, dtype=np.float64) - np.real(b))) ** 2 for a, b in pairs)
    den = sum(float(np.linalg.norm(np.real(b))) ** 2 for a, b in pairs)
    return (num / den) ** 0.5


def _gpu_run(bz, grid, t, precision, n):
    sim = bz.FDTD(design=grid, time=t, backend_options={"precision": precision, "n_comp": 1})
    sim.initialize_simulation(save=False, live=False, save_memory_mode=True)
    sim.engine.run_steps(n)
    return sim


def _fields(sim, keys):
    return {k: sim.engine.field(k).cpu().numpy() for k in keys}


@pytest.fixture(scope="module")
def dipole_case(bz):
    from beamz_b200 import workloads as W

    d, t, dx = W.dipole_2d()
    grid = bz.RegularGrid(d, dx)
    eps, sig = raster2d.rasterize(d, dx)
    np.testing.assert_array_equal(grid.permittivity, eps)
    np.testing.assert_array_equal(grid.conductivity, sig)
    ref = fdtd2d.run(eps, sig, dx, dx, t[1] - t[0], len(t), d.sources, d.monitors, record=True,
                     complex_fields=False)
    return d, t, dx, grid, ref


def test_dipole_full_run_fp64_vs_oracle(bz, dipole_case):
    d, t, dx, grid, ref = dipole_case
    sim = _gpu_run(bz, grid, t, "fp64", len(t))
    got = _fields(sim, ("Ez", "Hx", "Hy"))
    err = _rel([(got[k], ref[k]) for k in ("Ez", "Hx", "Hy")])
    print(f"dipole 400x400, {len(t)} steps, fp64: relative L2 {err:.2e}")
    assert err <= 1e-11, f"dipole fp64: relative L2 {err:.3e}"


def test_dipole_full_run_fp32_monitors_vs_oracle(bz, dipole_case):
    """The 4-edge monitors of the float32 run against the oracle's: every sample within
    1e-5 of the series' peak, the summed |S| power within 1e-4."""
    d, t, dx, grid, ref = dipole_case
    sim = bz.FDTD(design=grid, time=t, backend_options={"precision": "fp32", "n_comp": 1})
    sim.run(live=False, save=False, save_memory_mode=True)
    worst = {}
    for i, name in enumerate(("left", "right", "bottom", "top")):
        m = next(mm for mm in sim.monitors if mm.name == name)
        rec = ref["records"][i]
        for k in ("Ez", "Hx", "Hy"):
            got = np.array([np.asarray(v) for v in m.fields[k]], dtype=np.float64)
            exp = np.real(rec[k])
            assert got.shape == exp.shape and got.shape[0] == len(t)
            worst[(name, k)] = np.abs(got - exp).max() / np.abs(exp).max()
        p_got, p_exp = float(np.sum(m.power_history)), float(np.sum(np.real(rec["power"])))
        worst[(name, "power")] = abs(p_got - p_exp) / abs(p_exp)
    series = max(v for (n, k), v in worst.items() if k != "power")
    power = max(v for (n, k), v in worst.items() if k == "power")
    print(f"dipole fp32 monitors: worst sample error / peak {series:.2e}, summed power {power:.2e}")
    assert series <= 1e-5, f"monitor series {series:.3e}"
    assert power <= 1e-4, f"summed power {power:.3e}"


@pytest.mark.parametrize("precision,tol", [("fp32", 1e-5), ("fp64", 1e-11)])
def test_mmi_full_grid_vs_oracle(bz, precision, tol):
    from beamz_b200 import workloads as W

    n = 200
    d, t, dx = W.mmi_2d(n_steps=n)
    grid = bz.RegularGrid(d, dx)
    eps, sig = raster2d.rasterize(d, dx)
    np.testing.assert_array_equal(grid.permittivity, eps)
    ref = fdtd2d.run(eps, sig, dx, dx, t[1] - t[0], n, d.sources, [], record=False)
    sim = _gpu_run(bz, grid, t, precision, n)
    got = _fields(sim, ("Ez", "Hx", "Hy"))
    err = _rel([(got[k], ref[k]) for k in ("Ez", "Hx", "Hy")])
    print(f"MMI 2000x1000, {n} steps, {precision}: relative L2 {err:.2e}")
    assert err <= tol, f"MMI {precision}: relative L2 {err:.3e} > {tol:g}"


def soi_stack_small(bz, n_steps=250):
    """The 3D SOI MMI stack shrunk to 120 x 64 x 40 cells at 20 nm."""
    dx = 20e-9
    nx, ny, nz, pml = 120, 64, 40, 8
    W, H, D = (nx + 0.5) * dx, (ny + 0.5) * dx, (nz + 0.5) * dx
    d = bz.Design(width=W, height=H, depth=D, material=bz.Material(1.0), pml_size=pml * dx)
    from beamz_b200.workloads import pml_sigma_factor

    for b in d.boundaries:
        b.polynomial_order = 3
        b.sigma_factor = pml_sigma_factor(pml)
    yc, z_box, t_si = H / 2, 0.3e-6, 0.22e-6
    si, sio2 = bz.Material(12.25), bz.Material(2.085)
    d += bz.Rectangle(position=(0, 0, 0), width=W, height=H, depth=z_box, material=sio2)
    d += bz.Rectangle(position=(0, yc - 0.2e-6, z_box), width=0.8e-6, height=0.4e-6, depth=t_si, material=si)
    d += bz.Rectangle(position=(0.8e-6, yc - 0.45e-6, z_box), width=1.0e-6, height=0.9e-6, depth=t_si, material=si)
    d += bz.Rectangle(position=(1.8e-6, yc - 0.2e-6, z_box), width=W - 1.8e-6, height=0.4e-6, depth=t_si,
                      material=si)
    dt = 0.99 * dx / (bz.LIGHT_SPEED * np.sqrt(3))
    t = np.arange(n_steps) * dt
    sig = bz.gaussian_pulse(t, 1.0, 60 * dt, 20 * dt, bz.LIGHT_SPEED / 1.55e-6, 0.0)
    d += bz.ModeSource(design=d, position=(0.35e-6, yc, z_box + t_si / 2), width=0.8e-6, height=0.6e-6,
                       wavelength=1.55e-6, signal=sig, direction="+x", num_modes=1, grid_resolution=300)
    return d, t, dx


@pytest.mark.parametrize("precision,tol", [("fp32", 1e-5), ("fp64", 1e-11)])
def test_soi_stack_reduced_vs_oracle(bz, precision, tol):
    d, t, dx = soi_stack_small(bz)
    grid = bz.RegularGrid3D(d, dx, extrude=True)
    eps, _, sig = raster3d.rasterize3d(d, dx, extrude=True)
    np.testing.assert_array_equal(grid.permittivity, eps)
    np.testing.assert_array_equal(grid.conductivity, sig)
    n = len(t)
    ref = fdtd3d.run(eps, sig, dx, dx, dx, t[1] - t[0], n, d.sources, [])
    keys = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")
    sim = _gpu_run(bz, grid, t, precision, n)
    got = _fields(sim, keys)
    err = _rel([(got[k], ref["fields"][k]) for k in keys])
    print(f"SOI stack 120x64x40, {n} steps, {precision}: relative L2 {err:.2e}")
    assert np.linalg.norm(np.real(ref["fields"]["Ez"])) > 0
    assert err <= tol, f"SOI stack {precision}: relative L2 {err:.3e} > {tol:g}"
