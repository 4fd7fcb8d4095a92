"""The oracle reproduces the reference's own outputs (golden fixtures from
tests/golden/make_golden.py) — this pins the oracle before the GPU path is compared with it."""
import numpy as np
import pytest

import make_golden as MG
from designs import RES
from oracle import fdtd2d


def _patch_profile(src, g):
    src.mode_profiles[0] = [[a, x, y, 0.0] for a, x, y in zip(g["prof_amp"], g["prof_x"], g["prof_y"])]


def _run_case(bz, name, golden):
    g = golden(f"step_{name}")
    if name == "gauss":
        d, t, mons = MG.gauss_run(bz)
    else:
        direction, enforce = {"mode_x": ("+x", True), "mode_y": ("-y", False)}[name]
        d, t, src, mons = MG.mode_run(bz, direction=direction, enforce=enforce)
        _patch_profile(src, g)
    res = fdtd2d.run(g["eps"], g["sigma"], RES, RES, t[1] - t[0], len(t), d.sources, mons, accumulate_power=True)
    return g, res


@pytest.mark.parametrize("name", ["gauss", "mode_x", "mode_y"])
def test_oracle_matches_reference_run(bz, golden, name):
    g, res = _run_case(bz, name, golden)
    for k in ("Ez", "Hx", "Hy"):
        np.testing.assert_array_equal(res[k], g[k])
    np.testing.assert_allclose(res["power"], g["power"] * res["count"], rtol=1e-12, atol=0)
    for i, rec in enumerate(res["records"]):
        for k in ("Ez", "Hx", "Hy"):
            np.testing.assert_array_equal(rec[k], g[f"m{i}_{k}"])
        np.testing.assert_array_equal(rec["t"], g[f"m{i}_t"])
        np.testing.assert_array_equal(rec["power"], g[f"m{i}_power"])


def test_oracle_is_not_trivial(bz, golden):
    g, res = _run_case(bz, "gauss", golden)
    assert np.abs(res["Ez"]).max() > 1e-3
    assert all(len(r["Ez"]) > 10 for r in res["records"])


@pytest.mark.parametrize("name", ["shapes", "pml_only"])
def test_oracle_rasteriser_matches_reference(bz, golden, name):
    import designs as D
    from oracle import raster2d

    g = golden(f"raster_{name}")
    builder = {"shapes": D.raster_shapes, "pml_only": D.raster_pml_only}[name]
    eps, mu, sig = raster2d.rasterize_all(builder(bz), D.RES)
    np.testing.assert_array_equal(eps, g["eps"])
    np.testing.assert_array_equal(mu, g["mu"])
    np.testing.assert_array_equal(sig, g["sigma"])


def test_oracle_rasteriser3d_matches_reference(bz, golden):
    """The 3D restatement in its reference mode reproduces RegularGrid3D's grids
    (z-collapsed bounding boxes, 2D PML over every layer) bit for bit."""
    import designs as D
    from oracle import raster3d

    g = golden("raster3d")
    eps, mu, sig = raster3d.rasterize3d(D.design_3d(bz), D.RES)
    np.testing.assert_array_equal(eps, g["eps"])
    np.testing.assert_array_equal(mu, g["mu"])
    np.testing.assert_array_equal(sig, g["sigma"])


def test_oracle_rasteriser3d_extrude_fills_layers(bz):
    """extrude=True fills each structure's [z, z + depth) and grades the z faces."""
    import designs as D
    from oracle import raster3d

    eps, mu, sig = raster3d.rasterize3d(D.design_3d(bz), D.RES, extrude=True)
    i, j = int(0.6e-6 / D.RES), int(0.3e-6 / D.RES)
    assert np.all(eps[:8, i, j] == 2.085) and np.all(eps[8:12, i, j] == 12.25) and np.all(eps[13:, i, j] == 1.0)
    ref_eps, _, ref_sig = raster3d.rasterize3d(D.design_3d(bz), D.RES)
    assert not np.array_equal(eps, ref_eps)
    assert sig[0].max() > 0 and sig[-1].max() > 0 and sig[len(sig) // 2].max() <= ref_sig.max() + 1e-9


def _step3d_setup(bz, golden):
    import designs as D

    g = golden("step3d")
    d = D.step3d_design(bz)
    nz, ny, nx = int(0.65e-6 / D.RES), int(0.75e-6 / D.RES), int(0.85e-6 / D.RES)
    eps, sig = D.step3d_arrays((nz, ny, nx))
    res = D.RES
    dt = 0.99 * res / (bz.LIGHT_SPEED * np.sqrt(3))
    t = np.arange(60) * dt
    sg = bz.gaussian_pulse(t, 1.0, 10 * dt, 4 * dt, bz.LIGHT_SPEED / (1.55e-6), 0.0)
    cw = bz.ramped_cosine(t, amplitude=1.0, frequency=bz.LIGHT_SPEED / 1.55e-6, phase=0, ramp_duration=8 * dt,
                          t_max=t[-1])
    src_g = bz.GaussianSource(position=(0.4e-6, 0.35e-6, 0.3e-6), width=0.06e-6, signal=sg)
    src_m = bz.ModeSource(design=d, position=(0.25e-6, 0.38e-6, 0.33e-6), width=0.3e-6, height=0.25e-6,
                          wavelength=1.55e-6, signal=cw, direction="+x", num_modes=1)
    mz = bz.Monitor(design=d, start=(0.1e-6, 0.1e-6, 0.32e-6), end=(0.7e-6, 0.6e-6, 0.32e-6))
    mx = bz.Monitor(design=d, start=(0.2e-6, 0.05e-6, 0.45e-6), end=(0.8e-6, 0.7e-6, 0.45e-6), record_interval=2)
    for dev in (src_g, src_m, mz, mx):
        d += dev
    return g, d, eps, sig, res, dt, t, [src_g, src_m], [mz, mx]


def test_mode_source_3d_profile_matches_reference(bz, golden):
    g, d, eps, sig, res, dt, t, srcs, mons = _step3d_setup(bz, golden)
    prof = srcs[1].mode_profiles[0]
    assert len(prof) == int(g["prof_n"])
    assert np.sum(np.array([p[0] for p in prof], dtype=complex)) == g["prof_sum"]
    np.testing.assert_array_equal(np.array([p[1:4] for p in prof]).sum(axis=0), g["prof_xyz_sum"])


def test_oracle_3d_matches_reference_run(bz, golden):
    from oracle import fdtd3d

    g, d, eps, sig, res, dt, t, srcs, mons = _step3d_setup(bz, golden)
    out = fdtd3d.run(eps, sig, res, res, res, dt, len(t), srcs, mons, accumulate_power=True)
    for k in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz"):
        np.testing.assert_array_equal(out["fields"][k], g[k])
    np.testing.assert_allclose(out["power"], g["power"] * len(t), rtol=1e-12)
    for i, rec in enumerate(out["records"]):
        for k in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz"):
            np.testing.assert_array_equal(rec["fields"][k], g[f"m{i}_{k}"])
        np.testing.assert_array_equal(rec["t"], g[f"m{i}_t"])
        np.testing.assert_array_equal(rec["power"], g[f"m{i}_power"])


def test_fno_oracle_spectral_round_trip():
    """The oracle's truncated DFT followed by its inverse reproduces a field made of
    the kept modes (pins the basis, the Hermitian weights and the 1/P scale)."""
    import torch

    from oracle import fno_ref

    n, m = 16, 4
    cos, sin, w = fno_ref.bases(n, m)
    rng = np.random.default_rng(0)
    a = rng.standard_normal(cos.shape[1])
    b = rng.standard_normal(cos.shape[1])
    KX = np.tile(np.arange(m), 2 * m)
    KY = np.repeat(np.concatenate([np.arange(m), np.arange(n - m, n)]), m)
    # kx = 0 modes come in +ky/-ky pairs (each carries half), except ky = 0 (alone) and
    # ky = -m, whose partner +m is not kept: leave that one out of the test field
    amp = np.where(KX == 0, np.where(KY == 0, 1.0, 0.5), 1.0)
    amp[(KX == 0) & (KY == n - m)] = 0.0
    v = (cos.numpy() @ (a * amp)) - (sin.numpy() @ (b * amp))
    V = torch.as_tensor(v)
    ur, ui = V @ cos, -(V @ sin)
    back = (ur * w) @ cos.T - (ui * w) @ sin.T
    np.testing.assert_allclose(back.numpy(), v, rtol=1e-9, atol=1e-9 * np.abs(v).max())
