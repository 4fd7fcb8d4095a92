"""Cross-section mode solver of 3D plane sources (``mode_solver="cross_section"``),
checked on the CPU against exact discrete eigenvalues and an independent 1D assembly."""
import numpy as np
import pytest

from beamz_b200.const import LIGHT_SPEED
from beamz_b200.devices.mode import solve_modes_2d

WL = 1.55e-6
OMEGA = 2 * np.pi * LIGHT_SPEED / WL
K0 = OMEGA / LIGHT_SPEED


def _lap_eig(n, h, k=1):
    """k-th eigenvalue of the Dirichlet second difference on n nodes."""
    return -4.0 / h ** 2 * np.sin(k * np.pi / (2 * (n + 1))) ** 2


@pytest.mark.parametrize("pol", ["scalar", "v"])
def test_uniform_box_matches_discrete_eigenvalue(pol):
    nu, nv, du, dv, e = 31, 23, 20e-9, 25e-9, 4.0
    neff, modes = solve_modes_2d(np.full((nu, nv), e), OMEGA, du, dv, m=2, polarization=pol)
    beta2 = K0 ** 2 * e + _lap_eig(nu, du) + _lap_eig(nv, dv)
    assert abs(neff[0] ** 2 * K0 ** 2 - beta2) <= 1e-9 * beta2
    m0 = modes[0]
    assert np.all(m0.real > 0) and abs(np.linalg.norm(m0) - 1) < 1e-12
    want = np.outer(np.sin(np.pi * np.arange(1, nu + 1) / (nu + 1)), np.sin(np.pi * np.arange(1, nv + 1) / (nv + 1)))
    assert np.abs(m0.real - want / np.linalg.norm(want)).max() < 1e-8


def test_slab_separates_into_1d_operator_plus_u_mode():
    """eps(u, v) = f(v): beta^2 = (largest eigenvalue of the 1D v-operator) + first
    u-eigenvalue; the 1D semi-vectorial operator is assembled here independently."""
    nu, nv, du, dv = 25, 60, 30e-9, 15e-9
    v = (np.arange(nv) - nv / 2) * dv
    f = np.where(np.abs(v) < 110e-9, 12.25, 2.085)
    neff, _ = solve_modes_2d(np.tile(f, (nu, 1)), OMEGA, du, dv, m=1, polarization="v")
    A = np.zeros((nv, nv))
    for j in range(nv):
        up = (f[j] + f[j + 1]) / 2 if j + 1 < nv else f[j]
        dn = (f[j] + f[j - 1]) / 2 if j > 0 else f[j]
        A[j, j] = -(f[j] / up + f[j] / dn) / dv ** 2 + K0 ** 2 * f[j]
        if j + 1 < nv:
            A[j, j + 1] = f[j + 1] / up / dv ** 2
        if j > 0:
            A[j, j - 1] = f[j - 1] / dn / dv ** 2
    beta2 = np.max(np.linalg.eigvals(A).real) + _lap_eig(nu, du)
    assert abs(neff[0] ** 2 * K0 ** 2 - beta2) <= 1e-9 * beta2


def test_soi_strip_cross_section():
    """500 x 220 nm Si strip in SiO2: a guided mode between the indices; the field along
    the 220 nm direction jumps by the permittivity ratio at the Si faces (eps E is
    continuous), so eps E peaks in the core and E just outside it, and its index is
    below the scalar one."""
    nu, nv, h = 80, 60, 20e-9
    u = (np.arange(nu) - (nu - 1) / 2) * h
    v = (np.arange(nv) - (nv - 1) / 2) * h
    core = (np.abs(u)[:, None] <= 250e-9) & (np.abs(v)[None, :] <= 110e-9)
    eps = np.where(core, 12.25, 2.085)
    n_v, m_v = solve_modes_2d(eps, OMEGA, h, h, m=1, polarization="v")
    n_s, _ = solve_modes_2d(eps, OMEGA, h, h, m=1, polarization="scalar")
    assert np.sqrt(2.085) < n_v[0] < n_s[0] < 3.5
    i, j = np.unravel_index(np.argmax(np.abs(eps * m_v[0])), m_v[0].shape)
    assert core[i, j]
    a = np.abs(m_v[0])
    ie, je = np.unravel_index(np.argmax(a), a.shape)
    assert not core[ie, je] and (core[ie, je - 1] or core[ie, min(je + 1, nv - 1)])  # next to a Si face
    assert a[0, 0] < 1e-3 * a.max()


def test_mode_source_cross_section_option(bz):
    d = bz.Design(width=3e-6, height=2e-6, depth=1.2e-6, material=bz.Material(permittivity=2.085), auto_pml=False)
    d.add(bz.Rectangle(position=(0, 0.75e-6, 0.5e-6), width=3e-6, height=0.5e-6, depth=0.22e-6,
                       material=bz.Material(permittivity=12.25)))
    t = np.arange(10) * 1e-17
    src = bz.ModeSource(design=d, position=(0.5e-6, 1.0e-6, 0.61e-6), width=1.2e-6, height=0.8e-6, wavelength=WL,
                        signal=np.ones(10), direction="+x", num_modes=1, mode_solver="cross_section")
    prof = np.asarray(src.mode_profiles[0], dtype=float)
    assert prof.shape[1] == 4 and len(prof) == len(np.unique(prof[:, 1:], axis=0))
    assert np.all(prof[:, 1] == 0.5e-6)  # x-normal plane at the source position
    assert np.all(prof[:, 0] > -1e-12 * prof[:, 0].max())  # fundamental: one sign
    top = prof[np.argmax(prof[:, 0])]
    # the strip spans y 0.75-1.25 um, z 0.50-0.72 um; Ez peaks on a Si face
    assert abs(top[2] - 1.0e-6) < 0.1e-6 and 0.47e-6 < top[3] < 0.75e-6
    assert np.sqrt(2.085) < src.effective_indices_2d[0] < 3.5
    assert t.size == 10
