"""Host-side parts of the API against the reference (no GPU): mode solvers,
signals, PML profile, source compilation, topology helpers and Adam."""
import numpy as np
import pytest

import make_golden as MG
from designs import RES
from oracle import fdtd2d


def test_slab_mode_source_bit_exact(bz, golden):
    g = golden("modes")
    for k, (w, n1, n0, m) in enumerate([(0.5e-6, 3.5, 1.444, 0), (0.5e-6, 2.25, 1.444, 0), (2.0e-6, 3.5, 1.444, 1),
                                        (2.0e-6, 3.5, 1.444, 2)]):
        E, ne = bz.slab_mode_source(x=g["x"], w=w, n_WG=n1, n0=n0, wavelength=1.55e-6, ind_m=m)
        np.testing.assert_array_equal(E, g[f"slab{k}_E"])
        assert ne == g[f"slab{k}_neff"]


def test_solve_modes_matches_up_to_phase(bz, golden):
    g = golden("modes")
    neff, vecs = bz.solve_modes(g["solve_eps"], 2 * np.pi * bz.LIGHT_SPEED / 1.55e-6, 2e-6 / 400, npml=20, m=2)
    order = np.argsort(-np.real(neff))
    gorder = np.argsort(-np.real(g["solve_neff"]))
    np.testing.assert_allclose(neff[order], g["solve_neff"][gorder], rtol=1e-10)
    np.testing.assert_allclose(np.abs(vecs[:, order]), g["solve_abs"][:, gorder], rtol=1e-6, atol=1e-9)
    # the phase convention: repeatable, largest entry real and positive
    _, again = bz.solve_modes(g["solve_eps"], 2 * np.pi * bz.LIGHT_SPEED / 1.55e-6, 2e-6 / 400, npml=20, m=2)
    np.testing.assert_array_equal(again, vecs)
    peak = vecs[np.argmax(np.abs(vecs), axis=0), [0, 1]]
    assert np.all(peak.real > 0) and np.all(np.abs(peak.imag) <= 1e-15 * np.abs(peak))


def test_signals_bit_exact(bz, golden):
    from beamz_b200.devices.signals import gaussian_pulse, ramped_cosine

    g = golden("signals")
    t = g["t"]
    np.testing.assert_array_equal(ramped_cosine(t, 1.0, 1.9e14, phase=0.3, ramp_duration=8e-15, t_max=60e-15),
                                  g["ramped"])
    np.testing.assert_array_equal(gaussian_pulse(t, 1.3, 20e-15, 5e-15, 1.9e14, 0.1), g["pulse"])


def test_stability_and_params(bz):
    res, dt = bz.calc_optimal_fdtd_params(1.55e-6, 2.25, dims=2, safety_factor=0.99, points_per_wavelength=9)
    ok, c, lim = bz.check_fdtd_stability(dt, res, dy=res)
    assert ok and c == pytest.approx(0.99 / np.sqrt(2))


def _apply_ops(ops, ez, step, n_comp):
    """Apply compiled source ops to a flat field copy (the kernel's post phase)."""
    out = ez.copy()
    for c, m, w, s in zip(ops.cell, ops.mul, ops.weight, ops.sig):
        val = ops.signals[s, step]
        out[c] = m * out[c] + (w[0] + 1j * w[1]) * val
    return out


@pytest.mark.parametrize("case", ["gauss", "mode_x", "mode_y"])
def test_compiled_source_ops_equal_sequential_injection(bz, golden, case):
    """The merged per-cell operations give the reference's point-by-point result."""
    from beamz_b200.simulation.compile_ops import compile_sources

    if case == "gauss":
        d, t, _ = MG.gauss_run(bz)
    else:
        d, t, src, _ = MG.mode_run(bz, direction="+x" if case == "mode_x" else "-y", enforce=case == "mode_x")
        g = golden(f"step_{case}")
        src.mode_profiles[0] = [[a, x, y, 0.0] for a, x, y in zip(g["prof_amp"], g["prof_x"], g["prof_y"])]
    ny, nx = 40, 48
    ops = compile_sources(d.sources, (ny, nx), (RES, RES), len(t))
    rng = np.random.default_rng(0)
    for step in (3, 77):
        ez = rng.standard_normal((ny, nx)) + 1j * rng.standard_normal((ny, nx))
        want = ez.copy()
        for s in d.sources:
            inj = fdtd2d._ModeInjector(s, RES, RES, nx, ny) if hasattr(s, "mode_profiles") else \
                fdtd2d._GaussInjector(s, RES, RES, nx, ny)
            inj.apply(want, step)
        got = _apply_ops(ops, ez.ravel(), step, 2).reshape(ny, nx)
        np.testing.assert_allclose(got, want, rtol=1e-13, atol=1e-13 * np.abs(want).max())


def test_compiled_ops_enforce_zero_then_add_order(bz):
    """A zeroed cell that is injected later keeps only the later injections."""
    from beamz_b200.simulation.compile_ops import compile_sources

    class Src:
        direction = "+x"
        enforce_direction = True
        signal = np.ones(4)
        mode_profiles = [[[1.0, 2 * RES, 1 * RES, 0], [2.0, 3 * RES, 1 * RES, 0], [5.0, 2 * RES, 1 * RES, 0]]]

    from beamz_b200.devices.sources import ModeSource

    s = ModeSource.__new__(ModeSource)
    s.__dict__.update({k: getattr(Src, k) for k in ("direction", "enforce_direction", "signal", "mode_profiles")})
    ops = compile_sources([s], (4, 6), (RES, RES), 4)
    ez = np.arange(24, dtype=complex) + 10
    got = _apply_ops(ops, ez, 1, 1).reshape(4, 6)
    want = ez.reshape(4, 6).copy()
    want[1, 2] += 1.0; want[1, 1] = 0  # noqa: E702
    want[1, 3] += 2.0; want[1, 2] = 0  # noqa: E702
    want[1, 2] += 5.0; want[1, 1] = 0  # noqa: E702
    np.testing.assert_allclose(got, want)


# ---- topology helpers: the reference's own tests (tests/test_topology_updates.py) ----

def test_apply_density_update_changes_masked_region():
    from beamz_b200.optimization.topology import apply_density_update

    density = np.zeros((3, 3))
    mask = np.zeros_like(density, dtype=bool)
    mask[1, 1] = True
    new, applied, delta, norm, mx = apply_density_update(density, np.ones_like(density), mask, learning_rate=0.2)
    assert pytest.approx(new[1, 1]) == 0.2
    assert norm > 0.0 and pytest.approx(mx) == norm
    assert np.all(new[~mask] == 0.0) and np.all(delta[~mask] == 0.0)
    assert applied[1, 1] == pytest.approx(1.0)


def test_apply_density_update_obeys_clip_and_mask():
    from beamz_b200.optimization.topology import apply_density_update

    density = np.full((3, 3), 0.95)
    mask = np.zeros_like(density, dtype=bool)
    mask[1, 1] = True
    new, _, delta, norm, mx = apply_density_update(density, np.ones_like(density), mask, learning_rate=0.5)
    assert pytest.approx(new[1, 1]) == 1.0
    assert np.all(new[~mask] == density[~mask]) and np.all(delta[~mask] == 0.0)
    assert norm == pytest.approx(mx)


def test_apply_density_update_zero_gradient_returns_no_change():
    from beamz_b200.optimization.topology import apply_density_update

    density = np.random.default_rng(1).random((4, 4))
    mask = np.ones_like(density, dtype=bool)
    new, applied, delta, norm, mx = apply_density_update(density, np.zeros_like(density), mask, learning_rate=0.3)
    assert np.allclose(new, density) and np.allclose(applied, 0.0) and np.allclose(delta, 0.0)
    assert norm == 0.0 and mx == 0.0


def test_masked_blur_matches_window_loop():
    """masked_box_blur against an explicit window loop (edge-continued values, zero
    mask outside, empty windows divided by one), on a ragged mask."""
    from beamz_b200.optimization.topology import masked_box_blur

    rng = np.random.default_rng(3)
    v = rng.random((6, 7))
    m = rng.random((6, 7)) > 0.4
    m[0, :] = False
    r = 1
    vp = np.pad(v, r, mode="edge")
    mp = np.pad(m.astype(float), r)
    want = np.zeros_like(v)
    for i in range(6):
        for j in range(7):
            w = mp[i:i + 3, j:j + 3]
            den = w.sum()
            want[i, j] = (vp[i:i + 3, j:j + 3] * w).sum() / (den if den else 1.0)
    np.testing.assert_allclose(masked_box_blur(v, m, r), want, rtol=1e-14)
    assert masked_box_blur(np.arange(25.0).reshape(5, 5), np.ones((5, 5), bool), 1)[2, 2] == pytest.approx(12.0)


def test_density_update_batched_equals_per_design():
    """A batch of designs (leading dimension) gives each design's own update."""
    import torch

    from beamz_b200.optimization.topology import apply_density_update

    rng = np.random.default_rng(5)
    rho, g = rng.random((4, 9, 8)), rng.standard_normal((4, 9, 8))
    mask = rng.random((9, 8)) > 0.3
    new_b, app_b, d_b, n_b, mx_b = apply_density_update(torch.as_tensor(rho), torch.as_tensor(g), mask,
                                                        learning_rate=0.3, blur_radius=1)
    assert isinstance(new_b, torch.Tensor) and n_b.shape == (4,)
    for b in range(4):
        new, app, dl, n, mx = apply_density_update(rho[b], g[b], mask, learning_rate=0.3, blur_radius=1)
        np.testing.assert_allclose(new_b[b].numpy(), new, rtol=1e-14)
        np.testing.assert_allclose(app_b[b].numpy(), app, rtol=1e-14)
        assert float(n_b[b]) == pytest.approx(n) and float(mx_b[b]) == pytest.approx(mx)
        assert np.all(new[~mask] == rho[b][~mask]) and np.all((new >= 0) & (new <= 1))


def test_adam_steps_follow_the_published_rule():
    """Three Adam steps against the bias-corrected moment formulas written out here."""
    import torch

    from beamz_b200.optimization.optimizers import Optimizer

    rng = np.random.default_rng(7)
    grads = [rng.standard_normal((2, 3)) for _ in range(3)]
    opt = Optimizer(learning_rate=0.05, options={"beta1": 0.8, "beta2": 0.99})
    m = v = np.zeros((2, 3))
    for t, g in enumerate(grads, start=1):
        m = 0.8 * m + 0.2 * g
        v = 0.99 * v + 0.01 * g * g
        want = -0.05 * (m / (1 - 0.8 ** t)) / (np.sqrt(v / (1 - 0.99 ** t)) + 1e-8)
        np.testing.assert_allclose(opt.step(g), want, rtol=1e-12)
    np.testing.assert_allclose(Optimizer(learning_rate=0.1).step(np.array([1.0, -2.0])), [-0.1, 0.1], rtol=1e-6)
    out = Optimizer().step(torch.ones(3))
    assert isinstance(out, torch.Tensor)
    assert Optimizer().step(np.zeros(0)).shape == (0,)
    with pytest.raises(ValueError):
        Optimizer(method="lbfgs")
    with pytest.raises(TypeError):
        Optimizer().step([1.0, 2.0])


def test_filters_and_overlap_gradient():
    from beamz_b200.optimization.topology import blur_density, compute_overlap_gradient, project_density

    rho = np.zeros((5, 5))
    rho[2, 2] = 9.0
    b = blur_density(rho, 1)
    np.testing.assert_allclose(b[1:4, 1:4], np.ones((3, 3)))
    assert b.sum() == pytest.approx(9.0)
    p = project_density(np.array([0.5, 1.0]), 10.0, 0.5)
    assert p[0] == pytest.approx(0.5) and p[1] == pytest.approx(1 / (1 + np.exp(-5.0)))
    fwd = {"Ez": [np.ones((3, 4)) * (1 + 1j)]}
    adj = {"Ez": np.full((2, 5), 2.0 + 0j)}
    g = compute_overlap_gradient(fwd, adj)
    assert g.shape == (2, 4) and np.allclose(g, 2.0)
    with pytest.raises(ValueError):
        compute_overlap_gradient({}, adj)


@pytest.mark.parametrize("save,memory,cache,decimate,n", [(False, True, [], 1, 20000), (True, False, [], 1, 20000),
                                                          (True, True, ["Ez"], 1, 5000), (True, False, [], 3, 997),
                                                          (True, False, ["Hx"], 2, 123), (True, True, [], 1, 50)])
def test_next_save_step_matches_per_step_scan(bz, save, memory, cache, decimate, n):
    """FDTD._next_save gives the step a scan with _save_due stops at, from every start."""
    sim = bz.FDTD.__new__(bz.FDTD)
    freq = (max(10, n // 100) if save else 1) * decimate
    sim.__dict__.update(num_steps=n, _save_results=save, save_memory_mode=memory, _cache_fields=list(cache),
                        _effective_save_freq=freq, _cache_frequency=1 if cache else freq)
    starts = range(n + 1) if n <= 1000 else list(range(0, 400)) + list(range(n - 400, n + 1))
    for s in starts:
        want = s
        while want < n and not sim._save_due(want):
            want += 1
        assert sim._next_save(s) == want, s


def test_time_accumulation_matches_repeated_addition():
    dt = 2.3456789e-17
    t_loop = 1.0e-15
    for _ in range(20000):
        t_loop += dt
    t_acc = float(np.add.accumulate(np.r_[1.0e-15, np.full(20000, dt)])[-1])
    assert t_acc == t_loop


def test_adjoint_history_auto_takes_at_most_half_the_free_memory(monkeypatch):
    """store_history="auto" keeps the forward region history when (n_steps + 1) x designs x
    region cells fit in half the free device memory (a faked memory query; no GPU)."""
    import types

    import torch

    from beamz_b200.optimization.adjoint import AdjointFDTD2D

    p = AdjointFDTD2D.__new__(AdjointFDTD2D)
    p.store_history, p._hist, p.region, p.n_steps, p.B = "auto", None, (0, 0, 120, 120), 8000, 64
    p.engine = types.SimpleNamespace(dtype=torch.float32, dev=None)
    need = 8001 * 64 * 120 * 120 * 4  # 29.5 GB
    monkeypatch.setattr(torch.cuda, "mem_get_info", lambda dev=None: (2 * need, 4 * need))
    assert p._use_history()
    monkeypatch.setattr(torch.cuda, "mem_get_info", lambda dev=None: (2 * need - 2, 4 * need))
    assert not p._use_history()
    p._hist = object()  # once allocated, it is kept
    assert p._use_history()
    p._hist = None
    p.store_history = False
    assert not p._use_history()
    p.store_history = True
    assert p._use_history()
