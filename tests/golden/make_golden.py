"""Generate the golden fixtures in this directory by running the reference beamz.

Run in a container where the reference source tree is available:

    python tests/golden/make_golden.py /path/to/beamz-reference

The reference is imported from that path with stand-ins for its plotting/GDS
imports (matplotlib, mpl_toolkits, gdspy are not installed and are not on the
simulation path), and its own NumPy backend (float64 / complex128) produces:

* raster_*.npz   RegularGrid permittivity / permeability / conductivity
* step_*.npz     final Ez/Hx/Hy, monitor samples, power history and accumulated
                 power of short 2D runs (Gaussian source; mode sources with the
                 injected profile exported, since ARPACK's phase is arbitrary)
* modes.npz      slab_mode_source profiles and solve_modes effective indices
* signals.npz    ramped_cosine / gaussian_pulse samples
* raster3d.npz   RegularGrid3D output (the reference's own 3D rasteriser)
* step3d.npz     final six field components, z-normal plane monitor records and
                 accumulated power of a short 3D run on prescribed eps/sigma
* raster_custom.npz  RegularGrid output for CustomMaterial rectangles (function- and
                 grid-defined properties)
* monitor_saved.npz  a line monitor's recorded fields and power written by the
                 reference's own Monitor.save_data after a short 2D run

``--only name1,name2`` regenerates just those fixtures (the mode-source runs depend on
ARPACK's random start vector, so a full regeneration changes their files).

The tests rebuild the same designs through beamz_b200 (``designs.py``) and compare.
"""
from __future__ import annotations

import sys
import types
from pathlib import Path
from unittest.mock import MagicMock

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
import designs as D  # noqa: E402


def import_reference(path: str):
    for m in ["matplotlib", "matplotlib.pyplot", "matplotlib.patches", "matplotlib.path", "matplotlib.animation",
              "mpl_toolkits", "mpl_toolkits.mplot3d", "gdspy"]:
        sys.modules.setdefault(m, MagicMock())
    sys.path.insert(0, path)
    import beamz
    from beamz.devices import signals
    from beamz.devices.mode import slab_mode_source, solve_modes
    from beamz.simulation.meshing import RegularGrid, RegularGrid3D

    ns = {k: getattr(beamz, k) for k in dir(beamz) if not k.startswith("_")}
    ns.update(gaussian_pulse=signals.gaussian_pulse, ramped_cosine=signals.ramped_cosine, RegularGrid=RegularGrid,
              RegularGrid3D=RegularGrid3D,
              slab_mode_source=slab_mode_source, solve_modes=solve_modes)
    return types.SimpleNamespace(**ns)


def gauss_run(bz, n_steps=160):
    d = D.wg_design(bz)
    t = D.time_axis(bz, n_steps)
    sig = D.gauss_signal(bz, t)
    d += bz.GaussianSource(position=(1.2 * D.UM, 1.0 * D.UM), width=0.1 * D.UM, signal=sig)
    mons = [bz.Monitor(design=d, start=(1.8 * D.UM, 0.5 * D.UM), end=(1.8 * D.UM, 1.5 * D.UM), name="v"),
            bz.Monitor(design=d, start=(0.4 * D.UM, 1.6 * D.UM), end=(2.0 * D.UM, 1.6 * D.UM), name="h",
                       record_interval=3),
            bz.Monitor(design=d, start=(2.3 * D.UM, 0.1 * D.UM), end=(2.45 * D.UM, 1.9 * D.UM), name="edge")]
    for m in mons:
        d += m
    return d, t, mons


def mode_run(bz, n_steps=200, direction="+x", enforce=True):
    d = D.wg_design(bz)
    t = D.time_axis(bz, n_steps)
    sig = D.cw_signal(bz, t)
    if direction == "+x":
        src = bz.ModeSource(design=d, start=(0.6 * D.UM, 0.45 * D.UM), end=(0.6 * D.UM, 1.55 * D.UM),
                            wavelength=1.55 * D.UM, signal=sig, direction="+x", num_modes=1)
        mon = bz.Monitor(design=d, start=(1.9 * D.UM, 0.5 * D.UM), end=(1.9 * D.UM, 1.5 * D.UM), name="out")
    else:
        src = bz.ModeSource(design=d, position=(1.2 * D.UM, 1.5 * D.UM), width=1.0 * D.UM,
                            wavelength=1.55 * D.UM, signal=sig, direction="-y", num_modes=1)
        mon = bz.Monitor(design=d, start=(0.7 * D.UM, 0.6 * D.UM), end=(1.7 * D.UM, 0.6 * D.UM), name="out")
    if not enforce:
        src.enforce_direction = False
    d += src
    d += mon
    return d, t, src, [mon]


def _pack_monitor(prefix, m, out):
    for k in ("Ez", "Hx", "Hy"):
        out[f"{prefix}_{k}"] = np.array([np.asarray(v, dtype=complex) for v in m.fields[k]])
    out[f"{prefix}_t"] = np.asarray(m.fields["t"], dtype=float)
    out[f"{prefix}_power"] = np.asarray(m.power_history)


def run_and_pack(bz, d, t, mons, extra=None):
    sim = bz.FDTD(design=d, time=t, mesh="regular", resolution=D.RES, backend="numpy")
    sim.run(live=False, save=False, save_memory_mode=True, accumulate_power=True)
    out = dict(Ez=np.asarray(sim.Ez), Hx=np.asarray(sim.Hx), Hy=np.asarray(sim.Hy),
               power=np.asarray(sim.power_accumulated), eps=sim.mesh.permittivity, sigma=sim.mesh.conductivity)
    for i, m in enumerate(mons):
        _pack_monitor(f"m{i}", m, out)
    if extra:
        out.update(extra)
    return out


def step3d_run(bz, n_steps=60):
    """Small 3D run on prescribed eps/sigma (copied into the mesh, as examples/4_topo.py
    does in 2D): Gaussian source, 3D mode source plane, two plane monitors."""
    d = D.step3d_design(bz)
    res = D.RES
    grid = bz.RegularGrid3D(d, res)
    eps, sig = D.step3d_arrays(grid.permittivity.shape)
    np.copyto(grid.permittivity, eps)
    np.copyto(grid.conductivity, sig)
    dt = 0.99 * res / (bz.LIGHT_SPEED * np.sqrt(3))
    t = np.arange(n_steps) * dt
    sg = bz.gaussian_pulse(t, 1.0, 10 * dt, 4 * dt, bz.LIGHT_SPEED / (1.55 * D.UM), 0.0)
    cw = bz.ramped_cosine(t, amplitude=1.0, frequency=bz.LIGHT_SPEED / (1.55 * D.UM), phase=0,
                          ramp_duration=8 * dt, t_max=t[-1])
    g = bz.GaussianSource(position=(0.4 * D.UM, 0.35 * D.UM, 0.3 * D.UM), width=0.06 * D.UM, signal=sg)
    m = bz.ModeSource(design=d, position=(0.25 * D.UM, 0.38 * D.UM, 0.33 * D.UM), width=0.3 * D.UM,
                      height=0.25 * D.UM, wavelength=1.55 * D.UM, signal=cw, direction="+x", num_modes=1)
    mz = bz.Monitor(design=d, start=(0.1 * D.UM, 0.1 * D.UM, 0.32 * D.UM), end=(0.7 * D.UM, 0.6 * D.UM, 0.32 * D.UM))
    # only z-normal planes: the reference's x/y-normal plane slicing falls back to whole arrays and fails
    mx = bz.Monitor(design=d, start=(0.2 * D.UM, 0.05 * D.UM, 0.45 * D.UM), end=(0.8 * D.UM, 0.7 * D.UM, 0.45 * D.UM),
                    record_interval=2)
    for dev in (g, m, mz, mx):  # through the design: the reference's devices= path fails for GaussianSource
        d += dev
    return d, grid, t, [g, m], [mz, mx]


def custom_fixture(bz):
    g = bz.RegularGrid(D.raster_custom(bz), D.RES)
    np.savez_compressed(HERE / "raster_custom.npz", eps=g.permittivity, mu=g.permeability, sigma=g.conductivity)


def monitor_saved_fixture(bz):
    """A short Gaussian-source run with one recording line monitor (power on), saved by
    the reference's Monitor.save_data."""
    d = D.wg_design(bz)
    t = D.time_axis(bz, 40)
    d += bz.GaussianSource(position=(1.0 * D.UM, 1.0 * D.UM), width=0.1 * D.UM, signal=D.gauss_signal(bz, t))
    mon = bz.Monitor(design=d, start=(1.6 * D.UM, 0.6 * D.UM), end=(1.6 * D.UM, 1.4 * D.UM), name="m",
                     record_interval=2)
    d += mon
    sim = bz.FDTD(design=bz.RegularGrid(d, D.RES), time=t)
    sim.run(live=False, save=False, save_memory_mode=True)
    mon.save_data(str(HERE / "monitor_saved.npz"))


def main(ref_path: str, only=None):
    bz = import_reference(ref_path)
    if only:
        for name in only:
            {"raster_custom": custom_fixture, "monitor_saved": monitor_saved_fixture}[name](bz)
        print("fixtures written to", HERE)
        return
    custom_fixture(bz)
    monitor_saved_fixture(bz)
    for name, builder in (("shapes", D.raster_shapes), ("pml_only", D.raster_pml_only)):
        g = bz.RegularGrid(builder(bz), D.RES)
        np.savez_compressed(HERE / f"raster_{name}.npz", eps=g.permittivity, mu=g.permeability, sigma=g.conductivity)

    d, t, mons = gauss_run(bz)
    np.savez_compressed(HERE / "step_gauss.npz", **run_and_pack(bz, d, t, mons))
    for tag, direction, enforce in (("mode_x", "+x", True), ("mode_y", "-y", False)):
        d, t, src, mons = mode_run(bz, direction=direction, enforce=enforce)
        prof = src.mode_profiles[0]
        extra = dict(prof_amp=np.array([p[0] for p in prof], dtype=complex),
                     prof_x=np.array([p[1] for p in prof]), prof_y=np.array([p[2] for p in prof]))
        np.savez_compressed(HERE / f"step_{tag}.npz", **run_and_pack(bz, d, t, mons, extra))

    g3 = bz.RegularGrid3D(D.design_3d(bz), D.RES)
    np.savez_compressed(HERE / "raster3d.npz", eps=g3.permittivity, mu=g3.permeability, sigma=g3.conductivity)
    d, grid, t, srcs, mons = step3d_run(bz)
    sim = bz.FDTD(design=grid, time=t, backend="numpy")
    sim.run(live=False, save=False, save_memory_mode=True, accumulate_power=True)
    out = {k: np.asarray(getattr(sim, k)) for k in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")}
    out["power"] = np.asarray(sim.power_accumulated)
    prof = srcs[1].mode_profiles[0]
    amps = np.array([p[0] for p in prof], dtype=complex)  # deterministic (analytic slab modes): summarised only
    out.update(prof_n=len(prof), prof_sum=amps.sum(), prof_xyz_sum=np.array([p[1:4] for p in prof]).sum(axis=0))
    for i, m in enumerate(mons):
        for k in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz"):
            out[f"m{i}_{k}"] = np.array(m.fields[k])
        out[f"m{i}_t"] = np.asarray(m.fields["t"], dtype=float)
        out[f"m{i}_power"] = np.asarray(m.power_history)
    np.savez_compressed(HERE / "step3d.npz", **out)

    x = np.linspace(-1.5e-6, 1.5e-6, 301)
    modes = {}
    for k, (w, n1, n0, m) in enumerate([(0.5e-6, 3.5, 1.444, 0), (0.5e-6, 2.25, 1.444, 0), (2.0e-6, 3.5, 1.444, 1),
                                        (2.0e-6, 3.5, 1.444, 2)]):
        E, ne = bz.slab_mode_source(x=x, w=w, n_WG=n1, n0=n0, wavelength=1.55e-6, ind_m=m)
        modes[f"slab{k}_E"] = E
        modes[f"slab{k}_neff"] = ne
    eps1d = np.where(np.abs(np.linspace(-1e-6, 1e-6, 400)) < 0.25e-6, 12.25, 2.085)
    neff, vecs = bz.solve_modes(eps1d, 2 * np.pi * bz.LIGHT_SPEED / 1.55e-6, 2e-6 / 400, npml=20, m=2)
    modes.update(solve_neff=neff, solve_abs=np.abs(vecs), solve_eps=eps1d)
    np.savez_compressed(HERE / "modes.npz", x=x, **modes)

    tt = np.linspace(0, 60e-15, 500)
    np.savez_compressed(HERE / "signals.npz", t=tt,
                        ramped=bz.ramped_cosine(tt, 1.0, 1.9e14, phase=0.3, ramp_duration=8e-15, t_max=60e-15),
                        pulse=bz.gaussian_pulse(tt, 1.3, 20e-15, 5e-15, 1.9e14, 0.1))
    print("fixtures written to", HERE)


if __name__ == "__main__":
    import argparse

    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("reference", help="path of the reference beamz source tree")
    ap.add_argument("--only", default="", help="comma-separated fixture names (raster_custom, monitor_saved)")
    a = ap.parse_args()
    main(a.reference, [n for n in a.only.split(",") if n])
