"""2D stepping on the GPU against the reference's runs (golden fixtures) and the
oracle. Tolerances:
  * precision="fp64": relative L2 error <= 1e-11 (same arithmetic up to
    reassociation of the coefficient products);
  * precision="fp32": relative L2 error <= 1e-5 of the field norm while the
    field is live (these runs end before the pulse is absorbed); monitor samples
    within 1e-5 of their peak magnitude.
"""
import numpy as np
import pytest

import make_golden as MG
from designs import RES
from oracle import fdtd2d

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(np.asarray(b)), 1e-300)


def _golden_sim(bz, golden, name, precision):
    g = golden(f"step_{name}")
    if name == "gauss":
        d, t, mons = MG.gauss_run(bz)
    else:
        direction, enforce = {"mode_x": ("+x", True), "mode_y": ("-y", False)}[name]
        d, t, src, mons = MG.mode_run(bz, direction=direction, enforce=enforce)
        src.mode_profiles[0] = [[a, x, y, 0.0] for a, x, y in zip(g["prof_amp"], g["prof_x"], g["prof_y"])]
    grid = bz.RegularGrid(d, RES)
    np.copyto(grid.permittivity, g["eps"])
    np.copyto(grid.conductivity, g["sigma"])
    sim = bz.FDTD(design=grid, time=t, backend_options={"precision": precision})
    sim.run(live=False, save=False, save_memory_mode=True, accumulate_power=True)
    return g, sim, mons


@pytest.mark.parametrize("name", ["gauss", "mode_x", "mode_y"])
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-11), ("fp32", 1e-5)])
def test_step2d_matches_reference_run(bz, golden, name, precision, tol):
    g, sim, mons = _golden_sim(bz, golden, name, precision)
    for k in ("Ez", "Hx", "Hy"):
        got = sim.engine.field(k).cpu().numpy()
        want = g[k] if name != "gauss" else np.real(g[k])
        if name == "gauss":
            assert np.abs(np.imag(g[k])).max() == 0
        assert rel_l2(got, want) <= tol, (k, rel_l2(got, want))
    pw = sim.power_accumulated
    assert rel_l2(pw, g["power"]) <= 10 * tol
    for i, m in enumerate(mons):
        for k in ("Ez", "Hx", "Hy"):
            got = np.array([np.asarray(v) for v in m.fields[k]])
            want = g[f"m{i}_{k}"]
            if name == "gauss":
                want = np.real(want)
            assert got.shape == want.shape
            scale = max(np.abs(want).max(), 1e-300)
            assert np.abs(got - want).max() <= tol * scale, (i, k)
        np.testing.assert_allclose(m.fields["t"], g[f"m{i}_t"], rtol=0, atol=0)
        want_p = g[f"m{i}_power"]
        assert np.abs(np.asarray(m.power_history) - want_p).max() <= 10 * tol * max(np.abs(want_p).max(), 1e-300)


def _random_problem(seed, ny=29, nx=37, n_steps=120):
    rng = np.random.default_rng(seed)
    eps = 1.0 + 11.0 * rng.random((ny, nx))
    sigma = np.zeros((ny, nx))
    sigma[:, :5] = 2e5 * rng.random((ny, 5))
    sigma[-4:, :] = 1e5 * rng.random((4, nx))
    dx = 20e-9
    dt = 0.99 * dx / (299792458.0 * np.sqrt(2))
    t = np.arange(n_steps) * dt
    sig = np.sin(2 * np.pi * 1.9e14 * t) * np.exp(-((t - 20 * dt) / (10 * dt)) ** 2)

    class Pt:  # minimal ModeSource-like point list with complex amplitudes
        direction = "+x"
        enforce_direction = True
        signal = sig
        mode_profiles = [[[complex(rng.standard_normal(), rng.standard_normal()), 11 * dx, (3 + k) * dx, 0.0]
                          for k in range(20)]]

    return eps, sigma, dx, dt, t, sig, Pt


def _sim_from_arrays(bz, eps, sigma, dx, t, sources, monitors, precision, **kw):
    ny, nx = eps.shape
    d = bz.Design(width=(nx + 0.5) * dx, height=(ny + 0.5) * dx, auto_pml=False)
    grid = bz.RegularGrid(d, dx)
    np.copyto(grid.permittivity, eps)
    np.copyto(grid.conductivity, sigma)
    sim = bz.FDTD(design=grid, time=t, devices=list(monitors), backend_options={"precision": precision, **kw})
    sim.sources = list(sources)
    return sim


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-11), ("fp32", 2e-5)])
def test_step2d_odd_grid_complex_vs_oracle(bz, precision, tol):
    from beamz_b200.devices.sources import ModeSource

    eps, sigma, dx, dt, t, sig, Pt = _random_problem(3)
    src = ModeSource.__new__(ModeSource)
    src.__dict__.update(direction="+x", enforce_direction=True, signal=sig, mode_profiles=Pt.mode_profiles)
    mon = bz.Monitor(start=(30 * dx, 2 * dx), end=(30 * dx, 26 * dx))
    sim = _sim_from_arrays(bz, eps, sigma, dx, t, [src], [mon], precision)
    sim.run(live=False, save=False, save_memory_mode=True, accumulate_power=True)
    ref = fdtd2d.run(eps, sigma, dx, dx, dt, len(t), [src], [mon], accumulate_power=True)
    got = sim.engine.field("Ez").cpu().numpy()
    assert np.iscomplexobj(got)
    assert rel_l2(got, ref["Ez"]) <= tol
    assert rel_l2(sim.engine.field("Hx").cpu().numpy(), ref["Hx"]) <= tol
    assert rel_l2(sim.power_accumulated * len(t), ref["power"]) <= 10 * tol
    rec = ref["records"][0]
    got_ez = np.array([np.asarray(v) for v in mon.fields["Ez"]])
    assert np.abs(got_ez - rec["Ez"]).max() <= tol * np.abs(rec["Ez"]).max()


def _tiled_problem(bz, seed=21, n_steps=160):
    """83x141 grid (several temporal tiles each way) with a complex line source, a
    Gaussian source straddling tile edges, and two monitors on tile edges."""
    from beamz_b200.devices.sources import ModeSource

    eps, sigma, dx, dt, t, sig, Pt = _random_problem(seed, ny=83, nx=141, n_steps=n_steps)
    src = ModeSource.__new__(ModeSource)
    src.__dict__.update(direction="+x", enforce_direction=True, signal=sig, mode_profiles=Pt.mode_profiles)
    g = bz.GaussianSource(position=(54 * dx, 54 * dx), width=dx / 10, signal=sig)
    freqs = np.array([1.8e14, 2.0e14])
    mv = bz.Monitor(start=(54 * dx, 2 * dx), end=(54 * dx, 80 * dx), frequencies=freqs)
    mh = bz.Monitor(start=(3 * dx, 50 * dx), end=(137 * dx, 50 * dx), frequencies=freqs)
    return eps, sigma, dx, dt, t, [src, g], [mv, mh], freqs


@pytest.mark.parametrize("tb,tile", [(1, 0), (3, 1), (5, 2), (5, 3), (7, 0), (9, 0), (9, 5)])
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-11), ("fp32", 2e-5)])
def test_time_blocked_run_vs_oracle(bz, tb, tile, precision, tol):
    eps, sigma, dx, dt, t, srcs, mons, freqs = _tiled_problem(bz)
    sim = _sim_from_arrays(bz, eps, sigma, dx, t, srcs, mons, precision, time_block=tb, tb_tile=tile)
    sim.run(live=False, save=False, save_memory_mode=True)
    assert sim.engine.time_block == tb
    ref = fdtd2d.run(eps, sigma, dx, dx, dt, len(t), srcs, mons, dft_freqs=freqs)
    assert rel_l2(sim.engine.field("Ez").cpu().numpy(), ref["Ez"]) <= tol
    assert rel_l2(sim.engine.field("Hx").cpu().numpy(), ref["Hx"]) <= tol
    assert rel_l2(sim.engine.field("Hy").cpu().numpy(), ref["Hy"]) <= tol
    for m, rec in zip(mons, ref["records"]):
        for k in ("Ez", "Hx", "Hy"):
            got = np.array([np.asarray(v) for v in m.fields[k]])
            assert np.abs(got - rec[k]).max() <= tol * np.abs(rec[k]).max(), k
    # DFT sums of the real field (component 0): [points][freq][5] per monitor block
    d = sim.engine.dft_fields()[0, 0]
    for i, (sl, dft) in enumerate(zip(sim.engine.mp.slices, ref["dft"])):
        got = d[sl, i * len(freqs):(i + 1) * len(freqs)].transpose(1, 0, 2)
        errs = [rel_l2(got[..., q], dft[..., q]) for q in range(5)]
        assert max(errs) <= 10 * tol, (i, errs)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_time_blocked_batch_matches_single_steps(bz, precision):
    """Batched designs with their own materials: time-blocked launches (graphs and
    direct, split runs) give the same bits as single-step launches for fields and
    records (both kernels round every operation explicitly); DFT sums differ only by
    the grouping of the float64 fold."""
    from beamz_b200.simulation.engine2d import Engine2D

    eps, sigma, dx, dt, t, srcs, mons, freqs = _tiled_problem(bz, seed=23, n_steps=150)
    rng = np.random.default_rng(5)
    eps_b = np.stack([eps, eps[::-1, :], 1.0 + 11.0 * rng.random(eps.shape)])
    outs = []
    for tb, graphs, parts in ((1, False, [150]), (5, True, [71, 64, 15]), (7, False, [150]), (3, True, [150]),
                              (9, True, [55, 80, 15])):
        eng = Engine2D(eps_b, sigma, dx, dx, dt, len(t), srcs, mons, precision=precision, n_comp=2, n_designs=3,
                       record=True, use_graphs=graphs, time_block=tb)
        for p in parts:
            eng.run_steps(p)
        outs.append(([eng.field(k, d).cpu().numpy() for k in ("Ez", "Hx", "Hy") for d in range(3)]
                     + [eng.take_records()], eng.dft_fields()))
    for exact, dft in outs[1:]:
        for a, b in zip(exact, outs[0][0]):
            np.testing.assert_array_equal(a, b)
        assert rel_l2(dft, outs[0][1]) <= 1e-12


def test_graph_replay_equals_direct_launches(bz):
    eps, sigma, dx, dt, t, sig, _ = _random_problem(5, n_steps=300)
    src = bz.GaussianSource(position=(18 * dx, 14 * dx), width=dx / 10, signal=sig)
    outs = []
    for graph in (True, False):
        sim = _sim_from_arrays(bz, eps, sigma, dx, t, [src], [], "fp32", graph=graph)
        sim.run(live=False, save=False, save_memory_mode=True)
        outs.append(sim.engine.field("Ez").cpu().numpy())
    np.testing.assert_array_equal(outs[0], outs[1])


def test_step_api_and_snapshots(bz):
    eps, sigma, dx, dt, t, sig, _ = _random_problem(7, n_steps=40)
    src = bz.GaussianSource(position=(18 * dx, 14 * dx), width=dx / 10, signal=sig)
    sim = _sim_from_arrays(bz, eps, sigma, dx, t, [src], [], "fp64")
    sim.initialize_simulation(save=True, live=False, fields_to_cache=["Ez"])
    n = 0
    while sim.step():
        n += 1
    res = sim.finalize_simulation()
    assert n == 40 and len(res["Ez"]) == 40 and np.iscomplexobj(res["Ez"][0])
    ref = fdtd2d.run(eps, sigma, dx, dx, dt, len(t), [src], [], snapshot_steps=(0, 17, 39))
    for k in (0, 17, 39):
        assert rel_l2(res["Ez"][k], ref["snapshots"][k][0]) <= 1e-11


def test_dft_flux_vs_oracle(bz):
    eps, sigma, dx, dt, t, sig, _ = _random_problem(11, n_steps=400)
    src = bz.GaussianSource(position=(10 * dx, 14 * dx), width=dx / 10, signal=sig)
    freqs = np.array([1.7e14, 1.9e14, 2.1e14])
    mv = bz.Monitor(start=(25 * dx, 3 * dx), end=(25 * dx, 25 * dx), frequencies=freqs, record_fields=False,
                    accumulate_power=False)
    mh = bz.Monitor(start=(4 * dx, 20 * dx), end=(32 * dx, 20 * dx), frequencies=freqs, record_fields=False,
                    accumulate_power=False)
    sim = _sim_from_arrays(bz, eps, sigma, dx, t, [src], [mv, mh], "fp64")
    sim.run(live=False, save=False, save_memory_mode=True)
    ref = fdtd2d.run(eps, sigma, dx, dx, dt, len(t), [src], [mv, mh], dft_freqs=freqs, record=False)
    for m, d, vert in ((mv, ref["dft"][0], True), (mh, ref["dft"][1], False)):
        assert rel_l2(m.dft["Ez"], d[:, :, 0]) <= 1e-10
        want = fdtd2d.flux_from_dft(d, vert, dx, dx)
        np.testing.assert_allclose(m.flux(), want, rtol=1e-9, atol=1e-12 * np.abs(want).max())


def test_dft_with_runs_split_off_graph_chunks(bz):
    """run_steps counts that are not multiples of the graph chunk leave single-step
    samples in the monitor ring; the DFT must equal the one of direct launches."""
    from beamz_b200.simulation.engine2d import Engine2D

    eps, sigma, dx, dt, t, sig, _ = _random_problem(11, n_steps=400)
    src = bz.GaussianSource(position=(10 * dx, 14 * dx), width=dx / 10, signal=sig)
    mv = bz.Monitor(start=(25 * dx, 3 * dx), end=(25 * dx, 25 * dx), frequencies=[1.7e14, 2.1e14],
                    record_fields=False, accumulate_power=False)
    outs = []
    for graphs, parts in ((False, [400]), (True, [52, 128, 7, 64, 149])):
        eng = Engine2D(eps, sigma, dx, dx, dt, len(t), [src], [mv], precision="fp64", record=False,
                       use_graphs=graphs)
        for p in parts:
            eng.run_steps(p)
        outs.append(eng.dft_fields())
    assert rel_l2(outs[1], outs[0]) <= 1e-12


def test_tiny_grid_rejected(bz):
    d = bz.Design(width=1.5e-8, height=1e-6, auto_pml=False)
    with pytest.raises(ValueError):
        sim = bz.FDTD(design=d, time=np.arange(4) * 1e-17, resolution=1e-8)
        sim.run(live=False)


@pytest.mark.parametrize("rows", [4, 8, 32])
def test_tile_heights_agree(bz, rows):
    eps, sigma, dx, dt, t, sig, _ = _random_problem(13, ny=45, nx=70, n_steps=150)
    src = bz.GaussianSource(position=(30 * dx, 20 * dx), width=dx / 10, signal=sig)
    outs = []
    for tr in (16, rows):
        sim = _sim_from_arrays(bz, eps, sigma, dx, t, [src], [], "fp32", tile_rows=tr)
        sim.run(live=False, save=False, save_memory_mode=True)
        outs.append(sim.engine.field("Ez").cpu().numpy())
    assert rel_l2(outs[1], outs[0]) <= 1e-6


def test_autotune_picks_a_candidate_and_keeps_results(bz):
    from beamz_b200.simulation import engine2d as E

    eps, sigma, dx, dt, t, srcs, mons, freqs = _tiled_problem(bz, seed=29, n_steps=140)
    outs = []
    for tb in ("auto", 1):
        eng = E.Engine2D(eps, sigma, dx, dx, dt, len(t), srcs, mons, precision="fp32", record=True, time_block=tb)
        eng.run_steps(140)
        outs.append((eng.field("Ez").cpu().numpy(), eng.take_records(), eng))
    chosen = (outs[0][2].time_block, outs[0][2].tb_tile)
    assert chosen in E.TUNE_CANDIDATES
    np.testing.assert_array_equal(outs[0][0], outs[1][0])
    np.testing.assert_array_equal(outs[0][1], outs[1][1])
