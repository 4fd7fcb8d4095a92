"""1D waveguide mode solvers used to build mode sources (beamz/devices/mode.py:9-227).

Both run once on the host when a source is created:

* ``solve_modes``: finite-difference eigenproblem eps + (DfDb + DbDf)/(2 k0^2) on a
  line, with a complex coordinate-stretching absorber of ``npml`` points per
  side, solved with ARPACK shift-invert around n_max^2 (scipy ``eigs``). The
  reference lets ARPACK start from a random vector, so the overall phase of each
  mode (and with it the real part a real-field run injects) changes from run to
  run. Here the start vector is a fixed pseudo-random one and each mode is
  rotated so that its largest-magnitude entry is real and positive: the same
  modes up to a phase, reproducible across runs.
* ``solve_modes_2d``: modes of a 2D cross-section (the optional ``cross_section``
  solver of 3D plane sources), semi-vectorial or scalar, sparse shift-invert.
* ``slab_mode_source``: analytic TE mode of a symmetric slab; the propagation
  constant is bracketed by a 2000-point scan of the even/odd dispersion relations
  and refined by 50 bisection steps, then the profile is normalised to unit
  trapezoidal power. The same scan and bisection are used so results agree
  with the reference to the last bit.
"""
from __future__ import annotations

import warnings

import numpy as np
import scipy.sparse as sps
import scipy.sparse.linalg as spl

from ..const import LIGHT_SPEED


def compute_derivative_matrices(N, dL, npml=0):
    fwd = sps.diags([-1.0, 1.0], [0, 1], shape=(N, N), format="csr", dtype=float) / dL
    bwd = sps.diags([-1.0, 1.0], [-1, 0], shape=(N, N), format="csr", dtype=float) / dL
    if npml > 1:
        stretch = np.ones(N, dtype=complex)
        strength, power = 3.0, 3
        for i in range(npml):  # left layer: depth 1 at index 0, 0 at npml-1
            stretch[i] = 1.0 / (1.0 + 1j * strength * (((npml - 1) - i) / (npml - 1)) ** power)
        for k in range(npml):  # right layer: depth 0 at N-npml, 1 at N-1
            stretch[N - npml + k] = 1.0 / (1.0 + 1j * strength * (k / (npml - 1)) ** power)
        s = sps.diags(stretch, 0)
        s_inv = sps.diags(1 / stretch, 0)
        fwd = s_inv @ fwd @ s
        bwd = s_inv @ bwd @ s
    return fwd, bwd


def solve_modes(eps, omega, dL, npml=0, m=2):
    """Effective indices and unit-norm profiles of the m modes nearest n_max."""
    k0 = omega / LIGHT_SPEED
    N = eps.size
    fwd, bwd = compute_derivative_matrices(N, dL, npml)
    A = sps.diags(eps.flatten(), 0) + 0.5 * (fwd @ bwd + bwd @ fwd) * (1 / k0) ** 2
    n_max = np.sqrt(np.max(eps))
    v0 = np.random.default_rng(0).standard_normal(N)
    vals, vecs = spl.eigs(A, k=m, sigma=n_max ** 2, which="LM", v0=v0)
    vecs = vecs / np.sqrt(np.sum(np.square(np.abs(vecs)), axis=0))
    peak = vecs[np.argmax(np.abs(vecs), axis=0), np.arange(vecs.shape[1])]
    vecs = vecs * (np.abs(peak) / np.where(peak == 0, 1.0, peak))[None, :]
    return np.sqrt(vals), vecs


def solve_modes_2d(eps, omega, du, dv, m=1, polarization="v"):
    """Guided modes of a 2D cross-section ``eps[nu][nv]`` (uniform steps du, dv; the
    field is zero outside the window).

    ``polarization="v"``: semi-vectorial operator for a field along v,
    d2E/du2 + d/dv[(1/eps) d(eps E)/dv] + k0^2 eps E = beta^2 E (the eps jumps across
    v-interfaces enter through eps at the half points, their mean); ``"scalar"``:
    d2E/du2 + d2E/dv2 + k0^2 eps E = beta^2 E. Second-order central differences on the
    nodes, ARPACK shift-invert around k0^2 n_max^2 with a fixed start vector. Returns
    (neff[m], modes[m][nu][nv]) by decreasing neff, each mode of unit norm with its
    largest entry real and positive. No counterpart in the reference, whose 3D mode
    source multiplies two 1D slab profiles (sources.py:323-376)."""
    eps = np.asarray(eps, dtype=float)
    nu, nv = eps.shape
    k0 = omega / LIGHT_SPEED
    lap_u = sps.diags([1.0, -2.0, 1.0], [-1, 0, 1], shape=(nu, nu), format="csr", dtype=float) / du ** 2
    A = sps.kron(lap_u, sps.identity(nv, format="csr"), format="csr")
    if polarization == "scalar":
        lap_v = sps.diags([1.0, -2.0, 1.0], [-1, 0, 1], shape=(nv, nv), format="csr", dtype=float) / dv ** 2
        A = A + sps.kron(sps.identity(nu, format="csr"), lap_v, format="csr")
    elif polarization == "v":
        e = eps
        e_up = np.concatenate([(e[:, 1:] + e[:, :-1]) / 2, e[:, -1:]], axis=1)  # eps at j + 1/2
        e_dn = np.concatenate([e[:, :1], (e[:, 1:] + e[:, :-1]) / 2], axis=1)   # eps at j - 1/2
        diag = -(e / e_up + e / e_dn) / dv ** 2
        upper = np.zeros_like(e)
        upper[:, :-1] = e[:, 1:] / e_up[:, :-1] / dv ** 2      # coefficient of E[j+1] in row j
        lower = np.zeros_like(e)
        lower[:, 1:] = e[:, :-1] / e_dn[:, 1:] / dv ** 2       # coefficient of E[j-1] in row j
        n = nu * nv
        A = A + sps.diags([lower.ravel()[1:], diag.ravel(), upper.ravel()[:-1]], [-1, 0, 1], shape=(n, n),
                          format="csr")
    else:
        raise ValueError(f"polarization must be 'v' or 'scalar', got {polarization!r}")
    A = A + sps.diags(k0 ** 2 * eps.ravel(), 0, format="csr")
    v0 = np.random.default_rng(0).standard_normal(nu * nv)
    vals, vecs = spl.eigs(A, k=m, sigma=k0 ** 2 * np.max(eps), which="LM", v0=v0)
    order = np.argsort(-vals.real)
    vals, vecs = vals[order], vecs[:, order]
    vecs = vecs / np.linalg.norm(vecs, axis=0)
    peak = vecs[np.argmax(np.abs(vecs), axis=0), np.arange(vecs.shape[1])]
    vecs = vecs * (np.abs(peak) / np.where(peak == 0, 1.0, peak))[None, :]
    neff = np.sqrt(np.maximum(vals.real, 0.0)) / k0  # 0 for a mode below cutoff
    return neff, [vecs[:, i].reshape(nu, nv) for i in range(vecs.shape[1])]


def _slab_branches(w, n_wg, n0, k0):
    def common(beta):
        if beta < n0 * k0 or beta > n_wg * k0:
            return None
        inside = n_wg ** 2 * k0 ** 2 - beta ** 2
        outside = beta ** 2 - n0 ** 2 * k0 ** 2
        if inside <= 0 or outside <= 0:
            return None
        return np.sqrt(inside), np.sqrt(outside)

    def even(beta):
        kk = common(beta)
        if kk is None:
            return None
        kx, kappa = kk
        return kx * np.tan(kx * w / 2) - kappa

    def odd(beta):
        kk = common(beta)
        if kk is None:
            return None
        kx, kappa = kk
        s = np.sin(kx * w / 2)
        if abs(s) < 1e-12:
            return None
        return -kx * (np.cos(kx * w / 2) / s) - kappa

    return even, odd


def _branch_index(beta, w, n_wg, k0):
    inside = n_wg ** 2 * k0 ** 2 - beta ** 2
    if inside <= 0:
        return None, None
    theta = np.sqrt(inside) * w / 2
    return int(np.floor(2 * theta / np.pi)), theta


def _bisect(f, lo, hi):
    mid = lo
    for _ in range(50):
        mid = 0.5 * (lo + hi)
        fm = f(mid)
        if fm is None:
            hi = mid
            continue
        if abs(fm) < 1e-9:
            return mid
        fl = f(lo)
        if fl is None or fl * fm > 0:
            lo = mid
        else:
            hi = mid
    return mid


def slab_mode_source(x, w, n_WG, n0, wavelength, ind_m=0, x0=0):
    """Normalised TE profile and effective index of slab mode ``ind_m``."""
    k0 = 2 * np.pi / wavelength
    even, odd = _slab_branches(w, n_WG, n0, k0)
    scan = np.linspace(n0 * k0, n_WG * k0, 2000)
    fe = [even(b) for b in scan]
    fo = [odd(b) for b in scan]
    brackets = {"even": [], "odd": []}
    for i in range(len(scan) - 1):
        for name, vals in (("even", fe), ("odd", fo)):
            if vals[i] is not None and vals[i + 1] is not None and vals[i] * vals[i + 1] < 0:
                brackets[name].append((scan[i], scan[i + 1]))
    roots = []
    for lo, hi in brackets["even"]:
        b = _bisect(even, lo, hi)
        m, theta = _branch_index(b, w, n_WG, k0)
        if m is not None and m % 2 == 0 and not (m == 0 and theta > (np.pi / 2 - 0.1)):
            roots.append(("even", b))
    for lo, hi in brackets["odd"]:
        b = _bisect(odd, lo, hi)
        m, _ = _branch_index(b, w, n_WG, k0)
        if m is not None and m % 2 == 1:
            roots.append(("odd", b))
    roots.sort(key=lambda t: t[1], reverse=True)
    if not roots:
        raise ValueError("No guided slab modes found in [n0*k0, n_WG*k0].")
    if ind_m >= len(roots):
        warnings.warn(f"Requested mode index {ind_m} >= found modes ({len(roots)}). "
                      f"Using highest mode index {len(roots) - 1}.", UserWarning)
        ind_m = len(roots) - 1
    parity, beta = roots[ind_m]
    kx = np.sqrt(n_WG ** 2 * k0 ** 2 - beta ** 2)
    kappa = np.sqrt(beta ** 2 - n0 ** 2 * k0 ** 2)
    E = np.zeros_like(x, dtype=np.complex128)
    for i, xi in enumerate(x):
        xp = xi - x0
        if abs(xp) <= w / 2:
            E[i] = np.cos(kx * xp) if parity == "even" else np.sin(kx * xp)
        elif parity == "even":
            E[i] = np.cos(kx * (w / 2)) * np.exp(-kappa * (abs(xp) - w / 2))
        else:
            E[i] = np.sign(xp) * np.sin(kx * (w / 2)) * np.exp(-kappa * (abs(xp) - w / 2))
    E /= np.sqrt(np.trapezoid(np.abs(E) ** 2, x))
    return E, beta / k0
