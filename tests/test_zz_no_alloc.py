"""The allocation-free entry point against the regular path.

Some callers cannot call cudaMalloc, for example a binding whose runtime owns all
device memory through its own pool, or a host with a fixed device-memory budget.
For them ``bz_step2d_dft_static`` keeps the monitor-sample ring, which the regular
path (``bz_step2d`` + ``bz_dft_fold``) takes from the caller, in a fixed array
inside the library. This test calls it through the C ABI twice in a row and checks
that the fields and the float64 DFT sums match the regular path after each call.

This file is named so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N = 150  # steps per call; not a multiple of the 64-step ring, so the tail fold runs too


def _engine(bz):
    rng = np.random.default_rng(21)
    ny, nx = 41, 53
    dx = 20e-9
    eps = 1.0 + 11.0 * rng.random((ny, nx))
    sigma = np.zeros((ny, nx))
    sigma[:, :6] = 2e5 * rng.random((ny, 6))
    dt = 0.99 * dx / (bz.LIGHT_SPEED * np.sqrt(2))
    t = np.arange(2 * N) * dt
    sig = np.sin(2 * np.pi * 1.9e14 * t) * np.exp(-((t - 30 * dt) / (12 * dt)) ** 2)
    d = bz.Design(width=(nx + 0.5) * dx, height=(ny + 0.5) * dx, auto_pml=False)
    grid = bz.RegularGrid(d, dx)
    np.copyto(grid.permittivity, eps)
    np.copyto(grid.conductivity, sigma)
    freqs = np.array([1.8e14, 1.9e14, 2.0e14])
    mons = [bz.Monitor(start=(40 * dx, 3 * dx), end=(40 * dx, 37 * dx), frequencies=freqs, record_fields=False,
                       accumulate_power=False),
            bz.Monitor(start=(5 * dx, 30 * dx), end=(45 * dx, 30 * dx), frequencies=freqs, record_fields=False,
                       accumulate_power=False)]
    sim = bz.FDTD(design=grid, time=t, devices=mons, backend_options={"graph": False, "time_block": 1})
    sim.sources = [bz.GaussianSource(position=(15 * dx, 20 * dx), width=dx / 10, signal=sig)]
    sim.initialize_simulation(save=False, live=False, save_memory_mode=True)
    return sim.engine


def test_static_ring_entry_matches_caller_ring_path(bz):
    import torch

    from beamz_b200 import _native as nat

    eng = _engine(bz)
    # regular path: bz_step2d with the engine's own ring, folded by bz_dft_fold
    want = []
    for _ in range(2):
        eng.run_steps(N)
        eng._fold()
        torch.cuda.synchronize()
        want.append((eng.field("Ez").cpu().numpy().copy(), eng.dft.cpu().numpy().copy()))

    # allocation-free path from the same initial state
    eng.reset()
    dft = torch.zeros_like(eng.dft)
    mon = nat.MonitorOps.from_buffer_copy(eng.mops)
    mon.ring, mon.ring_len = None, 0
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        st = nat._step2d_dft_static(C.byref(eng.grid), C.byref(eng._fields()), C.byref(eng.sops), C.byref(mon),
                                    call * N, N, len(eng.freqs), eng.phasor.data_ptr(), eng.n_steps,
                                    dft.data_ptr(), stream)
        assert st == nat.BZ_OK, nat.last_error()
        torch.cuda.synchronize()
        eng.step_index = (call + 1) * N
        ez = eng.field("Ez").cpu().numpy()
        got = dft.cpu().numpy()
        np.testing.assert_array_equal(ez, want[call][0])
        np.testing.assert_allclose(got, want[call][1], rtol=1e-12, atol=1e-12 * np.abs(want[call][1]).max())
        assert np.abs(got).max() > 0


def test_static_ring_shorter_than_64_steps(bz):
    """float64 samples of 50 designs x 76 points take 152 KB a step, so the 8 MiB array
    holds 55 steps: the folds fall every 55 steps instead of 64. Same check as above."""
    import torch

    from beamz_b200 import _native as nat
    from beamz_b200.simulation.engine2d import Engine2D

    rng = np.random.default_rng(8)
    ny, nx, dx = 41, 53, 20e-9
    eps = 1.0 + 11.0 * rng.random((ny, nx))
    sigma = np.zeros((ny, nx))
    dt = 0.99 * dx / (bz.LIGHT_SPEED * np.sqrt(2))
    t = np.arange(2 * N) * dt
    sig = np.sin(2 * np.pi * 1.9e14 * t) * np.exp(-((t - 30 * dt) / (12 * dt)) ** 2)
    freqs = np.array([1.8e14, 2.0e14])
    mons = [bz.Monitor(start=(40 * dx, 3 * dx), end=(40 * dx, 37 * dx), frequencies=freqs, record_fields=False,
                       accumulate_power=False),
            bz.Monitor(start=(5 * dx, 30 * dx), end=(45 * dx, 30 * dx), frequencies=freqs, record_fields=False,
                       accumulate_power=False)]
    src = [bz.GaussianSource(position=(15 * dx, 20 * dx), width=dx / 10, signal=sig)]
    eng = Engine2D(eps, sigma, dx, dx, dt, len(t), src, mons, precision="fp64", n_designs=50, record=False,
                   use_graphs=False, time_block=1)
    items = eng.n_designs * eng.n_comp * eng.mp.n_points
    assert items * 5 * 8 > (8 << 20) // 64  # the ring is shorter than 64 steps
    eng.run_steps(N)
    eng._fold()
    torch.cuda.synchronize()
    want_ez, want_dft = eng.field("Ez", design=49).cpu().numpy().copy(), eng.dft.cpu().numpy().copy()
    eng.reset()
    dft = torch.zeros_like(eng.dft)
    mon = nat.MonitorOps.from_buffer_copy(eng.mops)
    mon.ring, mon.ring_len = None, 0
    st = nat._step2d_dft_static(C.byref(eng.grid), C.byref(eng._fields()), C.byref(eng.sops), C.byref(mon), 0, N,
                                len(eng.freqs), eng.phasor.data_ptr(), eng.n_steps, dft.data_ptr(),
                                torch.cuda.current_stream().cuda_stream)
    assert st == nat.BZ_OK, nat.last_error()
    torch.cuda.synchronize()
    eng.step_index = N
    np.testing.assert_array_equal(eng.field("Ez", design=49).cpu().numpy(), want_ez)
    got = dft.cpu().numpy()
    np.testing.assert_allclose(got, want_dft, rtol=1e-12, atol=1e-12 * np.abs(want_dft).max())


def test_static_ring_rejects_a_step_above_8_mib(bz):
    """A step whose samples exceed the array is refused with BZ_ERR_INVALID before any
    launch: the fields are left as they were."""
    import torch

    from beamz_b200 import _native as nat

    eng = _engine(bz)
    eng.run_steps(10)
    torch.cuda.synchronize()
    before = eng.field("Ez").cpu().numpy().copy()
    mon = nat.MonitorOps.from_buffer_copy(eng.mops)
    mon.ring, mon.ring_len = None, 0
    mon.n_points = 300000
    grid = nat.Grid2D.from_buffer_copy(eng.grid)
    grid.dtype = nat.BZ_F64  # 300000 x 5 x 8 bytes = 12 MB > 8 MiB
    dft = torch.zeros_like(eng.dft)
    st = nat._step2d_dft_static(C.byref(grid), C.byref(eng._fields()), C.byref(eng.sops), C.byref(mon), 10, 5,
                                len(eng.freqs), eng.phasor.data_ptr(), eng.n_steps, dft.data_ptr(),
                                torch.cuda.current_stream().cuda_stream)
    assert st == nat.BZ_ERR_INVALID
    assert "static ring" in nat.last_error()[1]
    torch.cuda.synchronize()
    np.testing.assert_array_equal(eng.field("Ez").cpu().numpy(), before)
    assert float(dft.abs().max()) == 0.0
