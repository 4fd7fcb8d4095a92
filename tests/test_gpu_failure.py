"""Failure paths on the GPU, made to happen without faulting anything:

* divergence: a run whose time step breaks the Courant limit grows without bound
  (float overflow to inf is an ordinary value); the engines' periodic field check
  records it on the device and FDTD.run() raises NativeError(BZ_ERR_DIVERGED) with the
  step, while the same run at a stable time step finishes;
* a bounded device wait: the tcgen05 GEMM's wait for an MMA commit that never comes
  runs out after a given number of polls; the kernel frees its tensor memory and
  returns, the call reports BZ_ERR_TIMEOUT, and the next GEMM on the same context is
  correct.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _run(bz, courant, n_steps, is3d=False, precision="fp32"):
    dx = 20e-9
    n = 24
    dims = 3 if is3d else 2
    kw = dict(width=(n + 0.5) * dx, height=(n + 0.5) * dx, material=bz.Material(2.0), pml_size=4 * dx)
    if is3d:
        kw["depth"] = (16 + 0.5) * dx
    d = bz.Design(**kw)
    dt = courant * dx / (bz.LIGHT_SPEED * np.sqrt(dims))
    t = np.arange(n_steps) * dt
    sig = np.sin(2 * np.pi * bz.LIGHT_SPEED / 1.55e-6 * t) * np.exp(-((t - 20 * dt) / (8 * dt)) ** 2)
    pos = (12 * dx, 12 * dx, 8 * dx) if is3d else (12 * dx, 12 * dx)
    d += bz.GaussianSource(position=pos, width=dx / 10, signal=sig)
    grid = bz.RegularGrid3D(d, dx, extrude=True) if is3d else bz.RegularGrid(d, dx)
    sim = bz.FDTD(design=grid, time=t, backend_options={"precision": precision})
    return sim


@pytest.mark.parametrize("is3d", [False, True])
def test_unstable_time_step_raises_diverged(bz, is3d):
    from beamz_b200 import _native as nat

    sim = _run(bz, 2.5, 1500, is3d)
    with pytest.raises(nat.NativeError) as err:
        sim.run(live=False, save=False, save_memory_mode=True)
    assert err.value.code == nat.BZ_ERR_DIVERGED
    assert "diverged by step" in str(err.value)
    step = int(str(err.value).split("step ")[1].split(":")[0])
    assert 0 < step <= 1500
    # the context is still usable: a stable run on the same grid finishes
    ok = _run(bz, 0.99, 300, is3d)
    ok.run(live=False, save=False, save_memory_mode=True)
    assert torch.isfinite(ok.engine.field("Ez")).all()


def test_gemm_bounded_wait_runs_out_and_context_survives(bz):
    from beamz_b200 import _native as nat

    dev = "cuda"
    A = torch.randn(128, 64, device=dev).to(torch.bfloat16)
    B = torch.randn(256, 64, device=dev).to(torch.bfloat16)
    C = torch.full((128, 256), 7.0, device=dev)
    rc = nat.gemm_wait_selftest(A.data_ptr(), B.data_ptr(), C.data_ptr(), 2000,
                                torch.cuda.current_stream().cuda_stream)
    assert rc == nat.BZ_ERR_TIMEOUT, rc
    assert "ran out" in nat.last_error()[1]
    assert torch.all(C == 7.0)  # the epilogue was skipped
    assert nat.gemm_error(reset=True) == 0  # the self-test cleared the word
    # an ordinary tcgen05 GEMM on the same context
    p = nat.Gemm()
    out = torch.empty(128, 256, device=dev)
    p.M, p.N, p.K, p.batch, p.act, p.ta, p.tb, p.engine = 128, 256, 64, 1, 0, 0, 1, 2
    p.A, p.lda, p.sa = A.data_ptr(), 64, 128 * 64
    p.B, p.ldb, p.sb = B.data_ptr(), 64, 256 * 64
    p.alpha, p.splitk, p.atomic = 1.0, 1, 0
    p.outf, p.ldc, p.sc = out.data_ptr(), 256, 128 * 256
    nat.gemm(p, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    want = A.float() @ B.float().T
    assert float((out - want).norm() / want.norm()) <= 1e-5
    assert nat.gemm_error(reset=True) == 0
