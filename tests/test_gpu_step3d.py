"""3D stepping, sources, plane monitors, power and the 3D rasteriser on the GPU,
against the reference's runs (golden fixtures) and the oracle.
Tolerances: fp64 relative L2 <= 1e-11; fp32 relative L2 <= 1e-5 (short runs, live
fields); rasteriser output bit-exact."""
import numpy as np
import pytest

import designs as D
from oracle import fdtd3d

pytestmark = pytest.mark.gpu
KEYS = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")


def rel_l2(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(np.asarray(b)), 1e-300)


def test_rasterizer3d_reference_mode_bit_exact(bz, golden):
    g = golden("raster3d")
    grid = bz.RegularGrid3D(D.design_3d(bz), D.RES)
    np.testing.assert_array_equal(grid.permittivity, g["eps"])
    np.testing.assert_array_equal(grid.permeability, g["mu"])
    np.testing.assert_array_equal(grid.conductivity, g["sigma"])


def test_rasterizer3d_extrude_mode_fills_thickness(bz):
    d = D.design_3d(bz)
    grid = bz.RegularGrid3D(d, D.RES, extrude=True)
    eps = grid.permittivity
    # substrate 0..0.4 um fills layers 0..7 at the centre column; Si strip 0.4..0.62 um above it
    i, j = int(0.6e-6 / D.RES), int(0.3e-6 / D.RES)
    assert np.all(eps[:8, i, j] == 2.085)
    assert np.all(eps[8:12, i, j] == 12.25)
    assert np.all(eps[13:, i, j] == 1.0)
    assert grid.conductivity[0].max() > 0 and grid.conductivity[-1].max() > 0  # z-face PML


@pytest.mark.parametrize("which", ["stack", "soi_mmi_3d"])
def test_rasterizer3d_extrude_mode_bit_exact_vs_oracle(bz, which):
    """extrude=True against the oracle's restatement (the reference's 27-sample rule
    with the structure's z range tested, plus z-face PML), bit for bit: the small
    stack of the fixtures and the full 600 x 300 x 150 SOI MMI grid of the 3D
    workload."""
    from oracle import raster3d
    from beamz_b200 import workloads as W

    if which == "stack":
        d, res = D.design_3d(bz), D.RES
    else:
        d, _, res = W.soi_mmi_3d()
    grid = bz.RegularGrid3D(d, res, extrude=True)
    eps, mu, sig = raster3d.rasterize3d(d, res, extrude=True)
    assert grid.permittivity.shape == eps.shape
    np.testing.assert_array_equal(grid.permittivity, eps)
    np.testing.assert_array_equal(grid.permeability, mu)
    np.testing.assert_array_equal(grid.conductivity, sig)
    assert sig[0].max() > 0 and sig[-1].max() > 0


def _golden_3d(bz, golden, precision):
    g = golden("step3d")
    d = D.step3d_design(bz)
    grid = bz.RegularGrid3D(d, D.RES)
    eps, sig = D.step3d_arrays(grid.permittivity.shape)
    np.copyto(grid.permittivity, eps)
    np.copyto(grid.conductivity, sig)
    res = D.RES
    dt = 0.99 * res / (bz.LIGHT_SPEED * np.sqrt(3))
    t = np.arange(60) * dt
    sg = bz.gaussian_pulse(t, 1.0, 10 * dt, 4 * dt, bz.LIGHT_SPEED / 1.55e-6, 0.0)
    cw = bz.ramped_cosine(t, amplitude=1.0, frequency=bz.LIGHT_SPEED / 1.55e-6, phase=0, ramp_duration=8 * dt,
                          t_max=t[-1])
    srcs = [bz.GaussianSource(position=(0.4e-6, 0.35e-6, 0.3e-6), width=0.06e-6, signal=sg),
            bz.ModeSource(design=d, position=(0.25e-6, 0.38e-6, 0.33e-6), width=0.3e-6, height=0.25e-6,
                          wavelength=1.55e-6, signal=cw, direction="+x", num_modes=1)]
    mons = [bz.Monitor(design=d, start=(0.1e-6, 0.1e-6, 0.32e-6), end=(0.7e-6, 0.6e-6, 0.32e-6)),
            bz.Monitor(design=d, start=(0.2e-6, 0.05e-6, 0.45e-6), end=(0.8e-6, 0.7e-6, 0.45e-6), record_interval=2)]
    sim = bz.FDTD(design=grid, time=t, devices=srcs + mons, backend_options={"precision": precision})
    sim.run(live=False, save=False, save_memory_mode=True, accumulate_power=True)
    return g, sim, mons


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-11), ("fp32", 1e-5)])
def test_step3d_matches_reference_run(bz, golden, precision, tol):
    g, sim, mons = _golden_3d(bz, golden, precision)
    for k in KEYS:
        got = sim.engine.field(k).cpu().numpy()
        assert got.shape == g[k].shape
        assert rel_l2(got, np.real(g[k])) <= tol, (k, rel_l2(got, np.real(g[k])))
    assert rel_l2(sim.power_accumulated, g["power"]) <= 10 * tol
    for i, m in enumerate(mons):
        assert len(m.fields["Ez"]) == len(g[f"m{i}_t"])
        for k in KEYS:
            got = np.array(m.fields[k])
            want = np.real(g[f"m{i}_{k}"])
            assert got.shape == want.shape
            assert np.abs(got - want).max() <= tol * max(np.abs(want).max(), 1e-300), (i, k)
        np.testing.assert_array_equal(m.fields["t"], g[f"m{i}_t"])
        want_p = np.real(g[f"m{i}_power"])
        assert np.abs(np.real(np.asarray(m.power_history)) - want_p).max() <= 10 * tol * np.abs(want_p).max()


def _odd_problem(bz, n_steps=50, seed=4, shape=(9, 11, 13)):
    rng = np.random.default_rng(seed)
    nz, ny, nx = shape
    dx = 30e-9
    eps = 1.0 + 9.0 * rng.random((nz, ny, nx))
    sig = np.zeros((nz, ny, nx))
    sig[:, :, :3] = 1e5 * rng.random((nz, ny, 3))
    sig[-2:] += 5e4 * rng.random((2, ny, nx))
    dt = 0.99 * dx / (bz.LIGHT_SPEED * np.sqrt(3))
    t = np.arange(n_steps) * dt
    sgn = np.sin(2 * np.pi * 1.9e14 * t) * np.exp(-((t - 12 * dt) / (5 * dt)) ** 2)
    d = bz.Design(width=(nx + 0.5) * dx, height=(ny + 0.5) * dx, depth=(nz + 0.5) * dx, auto_pml=False)
    grid = bz.RegularGrid3D(d, dx)
    np.copyto(grid.permittivity, eps)
    np.copyto(grid.conductivity, sig)
    from beamz_b200.devices.sources import ModeSource

    src = ModeSource.__new__(ModeSource)
    src.__dict__.update(direction="+x", enforce_direction=True, signal=sgn,
                        mode_profiles=[[[complex(rng.standard_normal(), rng.standard_normal()), 5 * dx, (2 + k) * dx,
                                         (2 + k % 5) * dx] for k in range(7)]])
    return d, grid, eps, sig, dx, dt, t, src, sgn


@pytest.mark.parametrize("precision,tol,tile_y", [("fp64", 1e-11, 8), ("fp32", 2e-5, 8), ("fp64", 1e-11, 16),
                                                   ("fp32", 2e-5, 16)])
def test_step3d_odd_grid_complex_vs_oracle(bz, precision, tol, tile_y):
    """Two-component (complex) fields; fp64 with 16-row tiles needs 64 KB of shared memory."""
    d, grid, eps, sig, dx, dt, t, src, _ = _odd_problem(bz)
    mon = bz.Monitor(design=d, start=(1 * dx, 1 * dx, 4 * dx), end=(11 * dx, 9 * dx, 4 * dx))
    sim = bz.FDTD(design=grid, time=t, devices=[mon], backend_options={"precision": precision, "tile_y": tile_y})
    sim.sources = [src]
    sim.run(live=False, save=False, save_memory_mode=True, accumulate_power=True)
    ref = fdtd3d.run(eps, sig, dx, dx, dx, dt, len(t), [src], [mon], accumulate_power=True)
    for k in KEYS:
        got = sim.engine.field(k).cpu().numpy()
        assert np.iscomplexobj(got)
        assert rel_l2(got, ref["fields"][k]) <= tol, k
    assert rel_l2(sim.power_accumulated * len(t), ref["power"]) <= 10 * tol
    got = np.array(mon.fields["Ez"])
    want = ref["records"][0]["fields"]["Ez"]
    assert np.abs(got - want).max() <= tol * np.abs(want).max()


@pytest.mark.parametrize("x_cells", [4, 2, 1])
@pytest.mark.parametrize("shape", [(9, 11, 13), (12, 17, 131), (10, 9, 128), (7, 10, 250), (37, 23, 70)])
@pytest.mark.parametrize("tile_z,tile_y", [(0, 8), (16, 8), (8, 8), (0, 16), (16, 16), (8, 16)])
def test_step3d_real_fp32_vs_oracle(bz, shape, tile_z, tile_y, x_cells):
    """Real float32 fields stepped four, two or one x cells per thread: nx not a multiple
    of the cells per thread (the last group ends in row padding), several x tiles (124 or
    62 owned columns each), several z blocks (tile_z 0 is the default, 16)."""
    if x_cells == 1 and (tile_z, tile_y) != (16, 8):
        pytest.skip("one layout is enough for the scalar kernel")
    if x_cells == 2 and tile_z == 0:
        pytest.skip("the same layout as tile_z 16")
    d, grid, eps, sig, dx, dt, t, _, sgn = _odd_problem(bz, shape=shape)
    nz, ny, nx = shape
    g = bz.GaussianSource(position=((nx - 3) * dx, 5 * dx, 4 * dx), width=dx / 10, signal=sgn)
    g2 = bz.GaussianSource(position=(2 * dx, (ny - 3) * dx, (nz - 4) * dx), width=dx / 10, signal=sgn)
    sim = bz.FDTD(design=grid, time=t, backend_options={"precision": "fp32", "tile_z": tile_z, "tile_y": tile_y,
                                                        "x_cells": x_cells})
    sim.sources = [g, g2]
    sim.run(live=False, save=False, save_memory_mode=True)
    assert sim.engine.n_comp == 1
    ref = fdtd3d.run(eps, sig, dx, dx, dx, dt, len(t), [g, g2], [])
    for k in KEYS:
        got = sim.engine.field(k).cpu().numpy()
        assert rel_l2(got, ref["fields"][k]) <= 2e-5, (k, rel_l2(got, ref["fields"][k]))


def test_step3d_graph_equals_direct(bz):
    d, grid, eps, sig, dx, dt, t, src, sgn = _odd_problem(bz, n_steps=100)
    g = bz.GaussianSource(position=(6 * dx, 5 * dx, 4 * dx), width=dx / 10, signal=sgn)
    outs = []
    for graph in (True, False):
        sim = bz.FDTD(design=grid, time=t, backend_options={"graph": graph})
        sim.sources = [g]
        sim.run(live=False, save=False, save_memory_mode=True)
        outs.append(sim.engine.field("Ez").cpu().numpy())
    np.testing.assert_array_equal(outs[0], outs[1])


def test_dft3d_with_runs_split_off_graph_chunks(bz):
    """Plane-monitor DFT sums with run_steps counts off the graph chunk equal the ones
    of direct launches (single-step samples are folded before a chunk reuses the ring)."""
    from beamz_b200.simulation.engine3d import Engine3D

    d, grid, eps, sig, dx, dt, t, src, sgn = _odd_problem(bz, n_steps=120)
    g = bz.GaussianSource(position=(6 * dx, 5 * dx, 3 * dx), width=dx / 10, signal=sgn)
    mon = bz.Monitor(design=d, start=(1 * dx, 1 * dx, 6 * dx), end=(11 * dx, 9 * dx, 6 * dx), frequencies=[1.9e14],
                     record_fields=False, accumulate_power=False)
    outs = []
    for graphs, parts in ((False, [120]), (True, [20, 40, 5, 32, 23])):
        eng = Engine3D(eps, sig, dx, dx, dx, dt, len(t), [g], [mon], precision="fp64", record=False,
                       use_graphs=graphs)
        for p in parts:
            eng.run_steps(p)
        eng._fold()
        outs.append(eng.dft.cpu().numpy())
    assert rel_l2(outs[1], outs[0]) <= 1e-12


def test_step3d_tile_heights_agree(bz):
    d, grid, eps, sig, dx, dt, t, src, sgn = _odd_problem(bz, n_steps=60)
    g = bz.GaussianSource(position=(6 * dx, 5 * dx, 4 * dx), width=dx / 10, signal=sgn)
    outs = []
    for tz, ty in ((16, 8), (8, 8), (16, 16), (8, 16)):
        sim = bz.FDTD(design=grid, time=t, backend_options={"tile_z": tz, "tile_y": ty})
        sim.sources = [g]
        sim.run(live=False, save=False, save_memory_mode=True)
        outs.append(sim.engine.field("Ey").cpu().numpy())
    for o in outs[1:]:
        assert rel_l2(o, outs[0]) <= 1e-6


def test_dft3d_flux_vs_oracle(bz):
    d, grid, eps, sig, dx, dt, t, src, sgn = _odd_problem(bz, n_steps=120)
    g = bz.GaussianSource(position=(6 * dx, 5 * dx, 3 * dx), width=dx / 10, signal=sgn)
    freqs = np.array([1.8e14, 2.0e14])
    mon = bz.Monitor(design=d, start=(1 * dx, 1 * dx, 6 * dx), end=(11 * dx, 9 * dx, 6 * dx), frequencies=freqs,
                     record_fields=False, accumulate_power=False)
    sim = bz.FDTD(design=grid, time=t, devices=[mon], backend_options={"precision": "fp64"})
    sim.sources = [g]
    sim.run(live=False, save=False, save_memory_mode=True)
    ref = fdtd3d.run(eps, sig, dx, dx, dx, dt, len(t), [g], [mon], dft_freqs=freqs)
    want = ref["dft"][0]  # (nf, n0, n1, 6)
    for i, k in enumerate(KEYS):
        assert rel_l2(mon.dft[k], want[..., i]) <= 1e-10, k
    s = want[..., 0] * np.conj(want[..., 4]) - want[..., 1] * np.conj(want[..., 3])
    flux = 0.5 * np.real(s.reshape(len(freqs), -1).sum(axis=1)) * dx * dx
    np.testing.assert_allclose(mon.flux(), flux, rtol=1e-9)


def test_cross_section_mode_source_run_vs_oracle(bz):
    """A 3D run driven by a ModeSource with mode_solver="cross_section" (its profile from
    the 2D cross-section eigenproblem) against the oracle's run of the same source."""
    d = bz.Design(width=3e-6, height=2e-6, depth=1.2e-6, material=bz.Material(permittivity=2.085), auto_pml=False)
    d.add(bz.Rectangle(position=(0, 0.75e-6, 0.5e-6), width=3e-6, height=0.5e-6, depth=0.22e-6,
                       material=bz.Material(permittivity=12.25)))
    dx = 50e-9
    dt = 0.99 * dx / (bz.LIGHT_SPEED * np.sqrt(3))
    t = np.arange(60) * dt
    sig = bz.ramped_cosine(t, amplitude=1.0, frequency=bz.LIGHT_SPEED / 1.55e-6, phase=0, ramp_duration=10 * dt,
                           t_max=t[-1])
    src = bz.ModeSource(design=d, position=(0.6e-6, 1.0e-6, 0.61e-6), width=1.2e-6, height=0.8e-6,
                        wavelength=1.55e-6, signal=sig, direction="+x", num_modes=1, mode_solver="cross_section")
    grid = bz.RegularGrid3D(d, dx, extrude=True)
    eps, sig_grid = grid.permittivity.copy(), grid.conductivity.copy()
    sim = bz.FDTD(design=grid, time=t, backend_options={"precision": "fp64", "n_comp": 1})
    sim.sources = [src]
    sim.run(live=False, save=False, save_memory_mode=True)
    ref = fdtd3d.run(eps, sig_grid, dx, dx, dx, dt, len(t), [src], [])
    for k in KEYS:
        got = sim.engine.field(k).cpu().numpy()
        assert np.abs(got).max() > 0, k
        assert rel_l2(got, np.real(ref["fields"][k])) <= 1e-11, k
