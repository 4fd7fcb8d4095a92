"""The benchmark configurations at their full sizes and lengths: float32 against a float64
run of the same workload on the GPU (the float64 path matches the CPU oracle to 1e-11 on
these grids, tests/test_gpu_parity_configs.py), through the fields after the last step
and the quantities each configuration reports.

* 2D MMI, 2000 x 1000, 20000 steps (CW): relative L2 of (Ez, Hx, Hy) <= 1e-5;
  per-port, per-wavelength transmission |dT| <= 1e-4.
* 3D SOI MMI, 600 x 300 x 150, 8000 steps: relative L2 of the six components <= 1e-5;
  port flux at every wavelength within 1e-4 of the largest port flux.

The measured errors are printed (``pytest -s``) and carried in the assertion messages.
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


def _rel(s32, s64, keys):
    num = den = 0.0
    for k in keys:
        a = s32.engine.field(k).double()
        b = s64.engine.field(k)
        num += float((a - b).square().sum())
        den += float(b.square().sum())
    return (num / den) ** 0.5


def test_mmi_full_size_fp32_matches_fp64(bz):
    s32, s64 = _run(bz, "mmi_2d", "fp32"), _run(bz, "mmi_2d", "fp64")
    T = {}
    for prec, sim in (("fp32", s32), ("fp64", s64)):
        fin = _mon(sim, "in").flux()
        T[prec] = np.array([_mon(sim, p).flux() / fin for p in ("port_top", "port_bottom")])
    dT = np.abs(T["fp32"] - T["fp64"]).max()
    err = _rel(s32, s64, ("Ez", "Hx", "Hy"))
    print(f"MMI 20000 steps: fields relative L2 fp32 vs fp64 {err:.2e}; max |dT| {dT:.2e}; "
          f"T = {np.round(T['fp64'], 4)}")
    assert dT <= 1e-4, f"MMI max |dT| {dT:.3e}"
    assert err <= 1e-5, f"MMI fields relative L2 {err:.3e}"


def test_soi_3d_full_size_fp32_matches_fp64(bz):
    s32, s64 = _run(bz, "soi_mmi_3d", "fp32"), _run(bz, "soi_mmi_3d", "fp64")
    f32 = np.array([_mon(s32, p).flux() for p in ("port_top", "port_bottom")])
    f64 = np.array([_mon(s64, p).flux() for p in ("port_top", "port_bottom")])
    ferr = np.abs(f32 - f64).max() / np.abs(f64).max()
    err = _rel(s32, s64, ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz"))
    print(f"3D SOI MMI 8000 steps: fields relative L2 fp32 vs fp64 {err:.2e}; port flux {ferr:.2e}")
    assert np.abs(f64).max() > 0 and ferr <= 1e-4, f"3D port flux relative difference {ferr:.3e}"
    assert err <= 1e-5, f"3D fields relative L2 {err:.3e}"
