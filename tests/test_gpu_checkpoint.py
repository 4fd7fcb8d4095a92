"""Step-state checkpoint and resume (FDTD.save_checkpoint / FDTD.resume): a run stopped
after a whole number of graph chunks, saved, and continued by a new simulation object
from the file ends with the same bits as the uninterrupted run -- fields, monitor
records and the float64 DFT sums -- in 2D and 3D; a checkpoint of another problem is
refused."""
import numpy as np
import pytest

import designs as D

pytestmark = pytest.mark.gpu


def _case2d(bz, n_steps=560):
    d = D.wg_design(bz)
    t = D.time_axis(bz, n_steps)
    sig = bz.ramped_cosine(t, amplitude=1.0, frequency=bz.LIGHT_SPEED / 1.55e-6, phase=0, ramp_duration=8e-15,
                           t_max=t[-1] * 2)
    d += bz.GaussianSource(position=(0.8 * D.UM, 1.0 * D.UM), width=0.1 * D.UM, signal=sig)
    d += bz.Monitor(design=d, start=(1.8 * D.UM, 0.5 * D.UM), end=(1.8 * D.UM, 1.5 * D.UM), name="dft",
                    wavelengths=[1.5e-6, 1.55e-6], record_fields=False, accumulate_power=False)
    d += bz.Monitor(design=d, start=(1.2 * D.UM, 0.4 * D.UM), end=(1.2 * D.UM, 1.6 * D.UM), name="rec")
    return bz.RegularGrid(d, D.RES), t


def _case3d(bz, n_steps=256):
    dx = 30e-9
    d = bz.Design(width=(40 + 0.5) * dx, height=(30 + 0.5) * dx, depth=(24 + 0.5) * dx, material=bz.Material(2.0),
                  pml_size=5 * dx)
    t = np.arange(n_steps) * 0.99 * dx / (bz.LIGHT_SPEED * np.sqrt(3))
    sig = np.sin(2 * np.pi * 1.9e14 * t) * np.exp(-((t - 40 * t[1]) / (15 * t[1])) ** 2)
    d += bz.GaussianSource(position=(12 * dx, 15 * dx, 12 * dx), width=dx / 10, signal=sig)
    d += bz.Monitor(design=d, start=(0.0, 5 * dx, 5 * dx), plane_normal="x", plane_position=28 * dx,
                    size=(20 * dx, 14 * dx), name="plane", wavelengths=[1.5e-6, 1.6e-6], record_fields=False,
                    accumulate_power=False)
    return bz.RegularGrid3D(d, dx, extrude=True), t


@pytest.mark.parametrize("dims", [2, 3])
def test_resume_matches_uninterrupted_run(bz, dims, tmp_path):
    grid, t = _case2d(bz) if dims == 2 else _case3d(bz)
    opts = {"precision": "fp32", "time_block": 7} if dims == 2 else {"precision": "fp32"}
    kw = dict(live=False, save=False, save_memory_mode=True)
    full = bz.FDTD(design=grid, time=t, backend_options=opts)
    full.run(**kw)
    # the monitors belong to the design, which every run below shares: keep this run's data
    want_flux = {m.name: np.array(m.flux()) for m in full.monitors if m.frequencies is not None}
    want_rec = {m.name: np.array(m.fields["Ez"]) for m in full.monitors if m.frequencies is None}
    keys = ("Ez", "Hx", "Hy") if dims == 2 else ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")
    want_fields = {k: full.engine.field(k).cpu().numpy().copy() for k in keys}
    for m in full.monitors:  # start the next runs from empty monitors
        for v in m.fields.values():
            v.clear()
    first = bz.FDTD(design=grid, time=t, backend_options=opts)
    first.initialize_simulation(**kw)
    chunk = first.engine.chunk if dims == 2 else 32
    first_chunk = (len(t) // 2) // chunk * chunk
    first.run_for(first_chunk)
    assert first.current_step == first_chunk
    path = tmp_path / "state.pt"
    first.save_checkpoint(path)
    second = bz.FDTD(design=grid, time=t, backend_options=opts)
    second.resume(path, **kw)
    assert second.current_step == len(t)
    for k in keys:
        np.testing.assert_array_equal(second.engine.field(k).cpu().numpy(), want_fields[k])
    for m in second.monitors:
        if m.frequencies is not None:
            np.testing.assert_array_equal(np.array(m.flux()), want_flux[m.name])
            assert np.abs(want_flux[m.name]).max() > 0
        elif dims == 2:
            np.testing.assert_array_equal(np.array(m.fields["Ez"]), want_rec[m.name])
            assert len(m.fields["Ez"]) == len(t)


def test_checkpoint_of_another_problem_is_refused(bz, tmp_path):
    grid, t = _case2d(bz, n_steps=112)
    a = bz.FDTD(design=grid, time=t, backend_options={"time_block": 7})
    a.run_for(56, live=False, save=False, save_memory_mode=True)
    path = tmp_path / "state.pt"
    a.save_checkpoint(path)
    other = bz.FDTD(design=grid, time=t, backend_options={"time_block": 7, "precision": "fp64"})
    with pytest.raises(ValueError):
        other.resume(path, live=False, save=False, save_memory_mode=True)
