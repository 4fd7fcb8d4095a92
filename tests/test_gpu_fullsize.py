"""The benchmark configurations at their full sizes: float32 against a float64 run of
the same workload on the GPU (the float64 path matches the reference's own runs to
1e-11 on the golden fixtures), through the quantities each configuration reports.

* 2D dipole, 400 x 400, 2000 steps: monitor time series within 1e-5 of their peak;
  integrated edge power within 1e-4.
* 2D MMI, 2000 x 1000, 20000 steps (CW): per-port, per-wavelength transmission
  |dT| <= 1e-4; final field relative L2 <= 1e-4.
* 3D SOI MMI, 600 x 300 x 150, 8000 steps: port flux at every wavelength within 1e-4
  of the largest port flux.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _run(bz, name, precision):
    from beamz_b200 import workloads as W

    d, t, dx = getattr(W, name)()
    grid = bz.RegularGrid3D(d, dx, extrude=True) if d.is_3d and d.depth else bz.RegularGrid(d, dx)
    sim = bz.FDTD(design=grid, time=t, backend_options={"precision": precision, "n_comp": 1})
    sim.run(live=False, save=False, save_memory_mode=True)
    return sim


def _mon(sim, name):
    return next(m for m in sim.monitors if m.name == name)


def test_dipole_full_size_fp32_matches_fp64(bz):
    s32, s64 = _run(bz, "dipole_2d", "fp32"), _run(bz, "dipole_2d", "fp64")
    for name in ("left", "right", "bottom", "top"):
        a, b = _mon(s32, name), _mon(s64, name)
        ez32, ez64 = np.array(a.fields["Ez"]), np.array(b.fields["Ez"])
        assert ez32.shape == ez64.shape and ez32.shape[0] == 2000
        assert np.abs(ez32 - ez64).max() <= 1e-5 * np.abs(ez64).max(), name
        p32, p64 = np.sum(a.power_history), np.sum(b.power_history)
        assert abs(p32 - p64) <= 1e-4 * abs(p64), name


def test_mmi_full_size_fp32_transmission_matches_fp64(bz):
    s32, s64 = _run(bz, "mmi_2d", "fp32"), _run(bz, "mmi_2d", "fp64")
    T = {}
    for prec, sim in (("fp32", s32), ("fp64", s64)):
        fin = _mon(sim, "in").flux()
        T[prec] = np.array([_mon(sim, p).flux() / fin for p in ("port_top", "port_bottom")])
    dT = np.abs(T["fp32"] - T["fp64"]).max()
    print(f"MMI max |dT| fp32 vs fp64 = {dT:.2e}; T = {np.round(T['fp64'], 4)}")
    assert dT <= 1e-4
    e32 = s32.engine.field("Ez").cpu().numpy().astype(np.float64)
    e64 = s64.engine.field("Ez").cpu().numpy()
    assert np.linalg.norm(e32 - e64) <= 1e-4 * np.linalg.norm(e64)


def test_soi_3d_full_size_fp32_flux_matches_fp64(bz):
    s32, s64 = _run(bz, "soi_mmi_3d", "fp32"), _run(bz, "soi_mmi_3d", "fp64")
    f32 = np.array([_mon(s32, p).flux() for p in ("port_top", "port_bottom")])
    f64 = np.array([_mon(s64, p).flux() for p in ("port_top", "port_bottom")])
    err = np.abs(f32 - f64).max() / np.abs(f64).max()
    print(f"3D port flux max relative difference fp32 vs fp64 = {err:.2e}")
    assert np.abs(f64).max() > 0 and err <= 1e-4
