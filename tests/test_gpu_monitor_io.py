"""Monitor output of GPU runs in the reference's formats: a line monitor's samples saved
with Monitor.save_data against the file the reference's own Monitor.save_data wrote for
the same run (float64 path, 1e-11 of each series' peak), and the DFT mode overlap
against the oracle's DFT of the same run."""
import numpy as np
import pytest

import designs as D
from oracle import fdtd2d

pytestmark = pytest.mark.gpu


def test_saved_monitor_matches_reference_file(bz, tmp_path):
    d = D.wg_design(bz)
    t = D.time_axis(bz, 40)
    d += bz.GaussianSource(position=(1.0 * D.UM, 1.0 * D.UM), width=0.1 * D.UM, signal=D.gauss_signal(bz, t))
    mon = bz.Monitor(design=d, start=(1.6 * D.UM, 0.6 * D.UM), end=(1.6 * D.UM, 1.4 * D.UM), name="m",
                     record_interval=2)
    d += mon
    sim = bz.FDTD(design=bz.RegularGrid(d, D.RES), time=t, backend_options={"precision": "fp64"})
    sim.run(live=False, save=False, save_memory_mode=True)
    out = tmp_path / "gpu.npz"
    mon.save_data(str(out))
    got = np.load(out, allow_pickle=True)
    ref = np.load(D.HERE / "monitor_saved.npz", allow_pickle=True)
    assert sorted(got.files) == sorted(ref.files)
    assert got["monitor_info"].item() == ref["monitor_info"].item()
    gf, rf = got["fields"].item(), ref["fields"].item()
    np.testing.assert_array_equal(np.array(gf["t"]), np.array(rf["t"]))
    for k in ("Ez", "Hx", "Hy"):
        a, b = np.real(np.array(gf[k])), np.real(np.array(rf[k]))
        assert a.shape == b.shape
        assert np.abs(a - b).max() <= 1e-11 * np.abs(b).max(), k
    pa, pb = np.real(got["power_history"]), np.real(ref["power_history"])
    assert np.abs(pa - pb).max() <= 1e-11 * np.abs(pb).max()
    np.testing.assert_array_equal(got["power_timestamps"], ref["power_timestamps"])


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("fp32", 1e-5)])
def test_mode_overlap_matches_oracle(bz, precision, tol):
    """Monitor.mode_overlap of the DFT line (per frequency) against the same normalised
    overlap of the oracle's DFT, for a slab-mode profile on the monitor's points."""
    d = D.wg_design(bz)
    t = D.time_axis(bz, 400)
    sig = bz.ramped_cosine(t, amplitude=1.0, frequency=bz.LIGHT_SPEED / 1.55e-6, phase=0, ramp_duration=8e-15,
                           t_max=t[-1] * 2)
    d += bz.GaussianSource(position=(0.8 * D.UM, 1.0 * D.UM), width=0.1 * D.UM, signal=sig)
    freqs = [bz.LIGHT_SPEED / lam for lam in (1.5e-6, 1.55e-6, 1.6e-6)]
    mon = bz.Monitor(design=d, start=(1.8 * D.UM, 0.5 * D.UM), end=(1.8 * D.UM, 1.5 * D.UM), name="out",
                     wavelengths=[bz.LIGHT_SPEED / f for f in freqs], record_fields=False, accumulate_power=False)
    d += mon
    grid = bz.RegularGrid(d, D.RES)
    sim = bz.FDTD(design=grid, time=t, backend_options={"precision": precision})
    sim.run(live=False, save=False, save_memory_mode=True)
    pts = mon.get_grid_points_2d(D.RES, D.RES)
    ys = np.array([p[1] * D.RES for p in pts]) + 0.5 * D.RES - 1.0 * D.UM
    profile, _ = bz.slab_mode_source(x=ys, w=0.4 * D.UM, n_WG=3.5, n0=np.sqrt(2.085), wavelength=1.55e-6, ind_m=0)
    got = mon.mode_overlap(profile)
    ref = fdtd2d.run(grid.permittivity, grid.conductivity, D.RES, D.RES, t[1] - t[0], len(t), d.sources, [mon],
                     record=False, dft_freqs=np.asarray(mon.frequencies), complex_fields=False)
    ez = ref["dft"][0][:, :, 0]  # [freq][point]
    m = np.asarray(profile, dtype=complex)
    want = np.abs(ez @ np.conj(m)) / (np.linalg.norm(m) * np.linalg.norm(ez, axis=1))
    assert got.shape == want.shape == (3,)
    assert np.all(want > 0.05)
    np.testing.assert_allclose(got, want, rtol=tol)
