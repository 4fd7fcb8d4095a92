"""The Backend interface's update_h_fields / update_e_field on the GPU against
the oracle's restatement of the NumPy backend."""
import numpy as np
import pytest

from oracle import fdtd2d

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("cplx", [False, True])
def test_backend_updates_match_numpy_backend(bz, cplx):
    rng = np.random.default_rng(2)
    ny, nx = 23, 31
    ez = rng.standard_normal((ny, nx)) + (1j * rng.standard_normal((ny, nx)) if cplx else 0)
    hx = rng.standard_normal((ny, nx - 1)) * 1e-3
    hy = rng.standard_normal((ny - 1, nx)) * 1e-3
    sigma = np.abs(rng.standard_normal((ny, nx))) * 1e4
    eps = 1 + 5 * rng.random((ny, nx))
    dx = dy = 20e-9
    dt = 0.99 * dx / (299792458.0 * np.sqrt(2))
    be = bz.get_backend("b200")
    hx_w, hy_w = fdtd2d.update_h(hx, hy, ez, sigma, dx, dy, dt)
    ez_w = fdtd2d.update_e(ez.copy(), hx_w, hy_w, sigma, eps, dx, dy, dt)
    Hx, Hy = be.update_h_fields(be.from_numpy(hx.astype(ez.dtype)), be.from_numpy(hy.astype(ez.dtype)),
                                be.from_numpy(ez), sigma, dx, dy, dt, bz.MU_0, bz.EPS_0)
    np.testing.assert_allclose(be.to_numpy(Hx), hx_w, rtol=1e-12, atol=1e-18)
    np.testing.assert_allclose(be.to_numpy(Hy), hy_w, rtol=1e-12, atol=1e-18)
    Ez = be.update_e_field(be.from_numpy(ez.copy()), Hx, Hy, sigma, eps, dx, dy, dt, bz.EPS_0)
    np.testing.assert_allclose(be.to_numpy(Ez), ez_w, rtol=1e-11, atol=1e-14)


def test_backend_registry(bz):
    assert type(bz.get_backend("numpy")).__name__ == "B200Backend"
    with pytest.raises(ValueError):
        bz.get_backend("tpu")
