"""3D Yee FDTD loop in float64 / complex128 NumPy (test oracle, see oracle/__init__.py).

One step, in the reference's order (beamz/simulation/fdtd.py:411-429):
  1. H then E update   fdtd.py:200-310 (E on interior slices only)
  2. sources           helper.py:8-47 (ModeSource into Ez at z_target),
                       helper.py:62-95 (GaussianSource 3D patch, no 1/4 factor)
  3. plane monitors    helper.py:235-244 -> monitors.py:317-396, 426-439
  4. power             helper.py:124-151 (|Re(E x H*)| over the common region)
Arrays are [z, y, x]: Ex (nz, ny, nx-1), Ey (nz, ny-1, nx), Ez (nz-1, ny, nx),
Hx (nz-1, ny-1, nx), Hy (nz-1, ny, nx-1), Hz (nz, ny-1, nx-1).
"""
from __future__ import annotations

import numpy as np

EPS_0 = 8.85e-12
MU_0 = 1.256e-6


def zeros_fields(nz, ny, nx, dtype=np.complex128):
    return dict(Ex=np.zeros((nz, ny, nx - 1), dtype), Ey=np.zeros((nz, ny - 1, nx), dtype),
                Ez=np.zeros((nz - 1, ny, nx), dtype), Hx=np.zeros((nz - 1, ny - 1, nx), dtype),
                Hy=np.zeros((nz - 1, ny, nx - 1), dtype), Hz=np.zeros((nz, ny - 1, nx - 1), dtype))


def update(F, eps_r, sigma, dx, dy, dz, dt, mu0=MU_0, eps0=EPS_0):
    """fdtd.py:200-310 with the same expressions, in place on the dict F."""
    Ex, Ey, Ez, Hx, Hy, Hz = (F[k] for k in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz"))
    smx = sigma[:-1, :-1, :] * mu0 / eps0
    smy = sigma[:-1, :, :-1] * mu0 / eps0
    smz = sigma[:, :-1, :-1] * mu0 / eps0
    cx = (Ez[:, 1:, :] - Ez[:, :-1, :]) / dy - (Ey[1:, :, :] - Ey[:-1, :, :]) / dz
    cy = (Ex[1:, :, :] - Ex[:-1, :, :]) / dz - (Ez[:, :, 1:] - Ez[:, :, :-1]) / dx
    cz = (Ey[:, :, 1:] - Ey[:, :, :-1]) / dx - (Ex[:, 1:, :] - Ex[:, :-1, :]) / dy
    for H, sm, c in ((Hx, smx, cx), (Hy, smy, cy), (Hz, smz, cz)):
        den = 1.0 + sm * dt / (2.0 * mu0)
        H[:] = ((1.0 - sm * dt / (2.0 * mu0)) / den) * H - ((dt / mu0) / den) * c
    e_x, s_x = eps_r[1:-1, 1:-1, :-1], sigma[1:-1, 1:-1, :-1]
    e_y, s_y = eps_r[1:-1, :-1, 1:-1], sigma[1:-1, :-1, 1:-1]
    e_z, s_z = eps_r[:-1, 1:-1, 1:-1], sigma[:-1, 1:-1, 1:-1]
    chx = ((Hz[:, 1:, :] - Hz[:, :-1, :]) / dy)[1:-1, :, :] - ((Hy[1:, :, :] - Hy[:-1, :, :]) / dz)[:, 1:-1, :]
    chy = ((Hx[1:, :, :] - Hx[:-1, :, :]) / dz)[:, :, 1:-1] - ((Hz[:, :, 1:] - Hz[:, :, :-1]) / dx)[1:-1, :, :]
    chz = ((Hy[:, :, 1:] - Hy[:, :, :-1]) / dx)[:, 1:-1, :] - ((Hx[:, 1:, :] - Hx[:, :-1, :]) / dy)[:, :, 1:-1]
    for E, sl, e, s, c in ((Ex, np.s_[1:-1, 1:-1, :], e_x, s_x, chx), (Ey, np.s_[1:-1, :, 1:-1], e_y, s_y, chy),
                           (Ez, np.s_[:, 1:-1, 1:-1], e_z, s_z, chz)):
        den = 1.0 + s * dt / (2.0 * eps0 * e)
        f1 = (1.0 - s * dt / (2.0 * eps0 * e)) / den
        f2 = (dt / (eps0 * e)) / den
        E[sl] = f1 * E[sl] + f2 * c


_BEHIND = {"+x": (0, 0, -1), "-x": (0, 0, 1), "+y": (0, -1, 0), "-y": (0, 1, 0), "+z": (-1, 0, 0), "-z": (1, 0, 0)}


class _ModeInjector3D:
    """helper.py:8-47 for one 3D ModeSource: each point adds amplitude*signal[n] to
    Ez[z_target, y, x] and, with enforce_direction, zeroes the cell behind it. When no
    zeroed cell is also injected the point sequence equals "add all, then zero all"
    and is applied vectorised; otherwise points are replayed one by one."""

    def __init__(self, src, dx, dy, dz, shape, nez):
        nz, ny, nx = shape
        self.signal = np.asarray(src.signal)
        enforce = getattr(src, "enforce_direction", True)
        amp, iz, iy, ix, zz_, zy_, zx_, seq = [], [], [], [], [], [], [], []
        for p in src.mode_profiles[0]:
            a, xr, yr, zr = (p[0], p[1], p[2], p[3]) if len(p) == 4 else (p[0], p[1], p[2], 0)
            x, y, z = int(round(xr / dx)), int(round(yr / dy)), int(round(zr / dz))
            if x < 0 or x >= nx or y < 0 or y >= ny or z < 0 or z >= nz:
                continue
            zt = min(z, nez - 1) if z < nez else nez // 2
            amp.append(a); iz.append(zt); iy.append(y); ix.append(x)  # noqa: E702
            zc = None
            if enforce and src.direction in _BEHIND:
                bz_, by, bx = _BEHIND[src.direction]
                ok = {"+x": x > 0, "-x": x < nx - 1, "+y": y > 0, "-y": y < ny - 1, "+z": zt > 0,
                      "-z": zt < nez - 1}[src.direction]
                if ok:
                    zc = (zt + bz_, y + by, x + bx)
                    zz_.append(zc[0]); zy_.append(zc[1]); zx_.append(zc[2])  # noqa: E702
            seq.append((a, zt, y, x, zc))
        self.amp = np.asarray(amp, dtype=complex)
        self.idx = tuple(np.asarray(v, dtype=int) for v in (iz, iy, ix))
        self.zidx = tuple(np.asarray(v, dtype=int) for v in (zz_, zy_, zx_))
        self.seq = seq
        inj = set(zip(iz, iy, ix))
        self.vectorised = not any(c in inj for c in zip(zz_, zy_, zx_))

    def apply(self, Ez, n):
        mod = self.signal[n]
        if self.vectorised:
            np.add.at(Ez, self.idx, self.amp * mod)
            if len(self.zidx[0]):
                Ez[self.zidx] = 0
            return
        for a, zt, y, x, zc in self.seq:
            Ez[zt, y, x] += a * mod
            if zc is not None:
                Ez[zc] = 0


class _GaussInjector3D:
    """helper.py:62-95: 3D Gaussian patch (no 1/4 factor) times signal[n]."""

    def __init__(self, src, dx, dy, dz, shape, nez):
        nz, ny, nx = shape
        self.signal = np.asarray(src.signal)
        cx, cy, cz = src.position[0] / dx, src.position[1] / dy, src.position[2] / dz
        wx, wy, wz = src.width / dx, src.width / dy, src.width / dz
        hx, hy, hz = (max(1, int(round(3 * w))) for w in (wx, wy, wz))
        ix, iy, iz = int(round(cx)), int(round(cy)), int(round(cz))
        self.x0, self.x1 = max(0, ix - hx), min(nx, ix + hx + 1)
        self.y0, self.y1 = max(0, iy - hy), min(ny, iy + hy + 1)
        self.z0, z1 = max(0, iz - hz), min(nz, iz + hz + 1)
        self.z1 = min(z1, nez)
        zg, yg, xg = np.meshgrid(np.arange(self.z0, self.z1), np.arange(self.y0, self.y1),
                                 np.arange(self.x0, self.x1), indexing="ij")
        e = 1e-9
        self.amp = np.exp(-((xg - cx) ** 2 / (2 * (wx ** 2 + e)) + (yg - cy) ** 2 / (2 * (wy ** 2 + e))
                            + (zg - cz) ** 2 / (2 * (wz ** 2 + e))))
        self.ze = max(0, min(nez - 1, self.z0))

    def apply(self, Ez, n):
        k = self.z1 - self.z0
        Ez[self.ze:self.ze + k, self.y0:self.y1, self.x0:self.x1] += self.amp[:k, :, :] * self.signal[n]


def make_injectors(sources, dx, dy, dz, shape):
    nez = shape[0] - 1
    return [(_ModeInjector3D if hasattr(s, "mode_profiles") else _GaussInjector3D)(s, dx, dy, dz, shape, nez)
            for s in sources]


def plane_slices(mon, dx, dy, dz, F):
    """Per-component index tuples of a plane monitor (monitors.py:317-371)."""
    return mon.plane_slices_3d(dx, dy, dz, {k: F[k].shape for k in F})


def run(eps_r, sigma, dx, dy, dz, dt, n_steps, sources=(), monitors=(), accumulate_power=False, fields=None,
        dft_freqs=None):
    """Run n_steps; ``dft_freqs`` additionally accumulates, per monitor, the DFT of the
    real part of the six plane samples (E at (n+1)dt, H at (n+1/2)dt), times dt."""
    nz, ny, nx = eps_r.shape
    F = zeros_fields(nz, ny, nx) if fields is None else {k: np.array(v) for k, v in fields.items()}
    keys = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")
    mons = [dict(m=m, last=-1, k=getattr(m, "record_interval", 1), rec={c: [] for c in keys}, power=[], t=[])
            for m in monitors]
    power = None
    inj = make_injectors(sources, dx, dy, dz, (nz, ny, nx))
    freqs = None if dft_freqs is None else np.asarray(dft_freqs, dtype=float)
    dft = [None] * len(mons)
    t = 0
    for n in range(n_steps):
        update(F, eps_r, sigma, dx, dy, dz, dt)
        for j in inj:
            j.apply(F["Ez"], n)
        for md in mons:
            if (n - md["last"]) >= md["k"]:
                sl = plane_slices(md["m"], dx, dy, dz, F)
                parts = [F[c][s].copy() for c, s in zip(keys, sl)]
                for c, p in zip(keys, parts):
                    md["rec"][c].append(p)
                ex, ey, ez, hx, hy, hz = parts
                sx, sy, sz = ey * hz - ez * hy, ez * hx - ex * hz, ex * hy - ey * hx
                md["power"].append(np.sum(np.sqrt(sx ** 2 + sy ** 2 + sz ** 2)))
                md["t"].append(t)
                md["last"] = n
        if freqs is not None:
            w = 2 * np.pi * freqs
            pe, ph = np.exp(-1j * w * ((n + 1.0) * dt)), np.exp(-1j * w * ((n + 0.5) * dt))
            for i, md in enumerate(mons):
                sl = plane_slices(md["m"], dx, dy, dz, F)
                parts = np.stack([np.real(F[c][s]) for c, s in zip(keys, sl)], axis=-1)  # (n0, n1, 6)
                phase = np.stack([pe] * 3 + [ph] * 3, axis=-1)  # (nf, 6)
                term = parts[None] * phase[:, None, None, :]
                dft[i] = term if dft[i] is None else dft[i] + term
        if accumulate_power:
            mz = min(F[c].shape[0] for c in keys)
            my = min(F[c].shape[1] for c in keys)
            mx = min(F[c].shape[2] for c in keys)
            Ex, Ey, Ez, Hx, Hy, Hz = (F[c][:mz, :my, :mx] for c in keys)
            sx = np.real(Ey * np.conj(Hz) - Ez * np.conj(Hy))
            sy = np.real(Ez * np.conj(Hx) - Ex * np.conj(Hz))
            sz = np.real(Ex * np.conj(Hy) - Ey * np.conj(Hx))
            pm = np.sqrt(sx ** 2 + sy ** 2 + sz ** 2)
            power = pm.copy() if power is None else power + pm
        t += dt
    recs = [dict(fields={c: np.array(md["rec"][c]) for c in keys}, power=np.asarray(md["power"]),
                 t=np.asarray(md["t"], dtype=float)) for md in mons]
    if freqs is not None:
        dft = [None if d is None else d * dt for d in dft]
    return dict(fields=F, power=power, records=recs, dft=dft)
