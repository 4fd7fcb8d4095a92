"""Monitor npz I/O in the reference's format (beamz/devices/monitors.py:569-589: keys
fields, power_history, power_timestamps, monitor_info) and CustomMaterial rasterisation
on the host restatement, against files the reference itself wrote (tests/golden/)."""
import numpy as np
import pytest

import designs as D
from oracle import fdtd2d, raster2d


def _monitor_case(bz):
    d = D.wg_design(bz)
    t = D.time_axis(bz, 40)
    d += bz.GaussianSource(position=(1.0 * D.UM, 1.0 * D.UM), width=0.1 * D.UM, signal=D.gauss_signal(bz, t))
    mon = bz.Monitor(design=d, start=(1.6 * D.UM, 0.6 * D.UM), end=(1.6 * D.UM, 1.4 * D.UM), name="m",
                     record_interval=2)
    d += mon
    return d, t, mon


def test_load_reference_saved_monitor(bz, tmp_path):
    """A file written by the reference's Monitor.save_data loads into this Monitor, holds
    the oracle's records of the same run, and survives a save/load round trip with the
    same keys."""
    d, t, mon = _monitor_case(bz)
    mon.load_data(str(D.HERE / "monitor_saved.npz"))
    assert set(mon.fields) == {"Ez", "Hx", "Hy", "t"} and len(mon.fields["Ez"]) == 20
    eps, sig = raster2d.rasterize(d, D.RES)
    ref = fdtd2d.run(eps, sig, D.RES, D.RES, t[1] - t[0], len(t), d.sources, [mon], record=True)
    rec = ref["records"][0]
    for k in ("Ez", "Hx", "Hy"):
        np.testing.assert_array_equal(np.array(mon.fields[k]), rec[k])
    np.testing.assert_array_equal(np.array(mon.fields["t"]), rec["t"])
    np.testing.assert_array_equal(np.array(mon.power_history), rec["power"])
    out = tmp_path / "again.npz"
    mon.save_data(str(out))
    a = np.load(out, allow_pickle=True)
    assert sorted(a.files) == ["fields", "monitor_info", "power_history", "power_timestamps"]
    assert a["monitor_info"].item() == {"type": "line", "is_3d": False}
    for k in ("Ez", "Hx", "Hy", "t"):
        np.testing.assert_array_equal(np.array(a["fields"].item()[k]), np.array(mon.fields[k]))
    np.testing.assert_array_equal(a["power_history"], np.array(mon.power_history))
    with pytest.raises(ValueError):
        mon.save_data(str(tmp_path / "x.h5"), format="hdf5")


def test_custom_material_raster_oracle_matches_reference(bz, golden):
    g = golden("raster_custom")
    eps, mu, sig = raster2d.rasterize_all(D.raster_custom(bz), D.RES)
    np.testing.assert_array_equal(eps, g["eps"])
    np.testing.assert_array_equal(mu, g["mu"])
    np.testing.assert_array_equal(sig, g["sigma"])
    assert len(np.unique(g["eps"])) > 50  # the functions and the grid really vary
