"""2D Ez-mode FDTD loop in float64 / complex128 NumPy (test oracle, see oracle/__init__.py).

One step, in the reference's order (beamz/simulation/fdtd.py:411-429):
  1. H update     numpy_backend.py:34-61  (Hx, Hy promoted to complex128 with Ez)
  2. E update     numpy_backend.py:63-88  (interior; the outer ring is left as is)
  3. sources      helper.py:5-118         (ModeSource points, GaussianSource patch)
  4. monitors     helper.py:245-256 -> monitors.py:279-315 / 407-424
  5. power        helper.py:152-187       (only when accumulate_power)
and, as additions checked against the GPU path (the reference has no DFT): the
DFT of Ez and of the H samples centred on the monitor cells, with E stamped at
(n+1)dt and H at (n+1/2)dt.

Arrays follow the reference: Ez (ny, nx) complex128, Hx (ny, nx-1), Hy (ny-1, nx).
"""
from __future__ import annotations

import numpy as np

EPS_0 = 8.85e-12  # beamz/const.py
MU_0 = 1.256e-6


def update_h(Hx, Hy, Ez, sigma, dx, dy, dt, mu_0=MU_0, eps_0=EPS_0):
    """numpy_backend.py:34-61, same expressions and order."""
    if np.iscomplexobj(Ez):
        if not np.iscomplexobj(Hx):
            Hx = Hx.astype(np.complex128)
        if not np.iscomplexobj(Hy):
            Hy = Hy.astype(np.complex128)
    smx = sigma[:, :-1] * mu_0 / eps_0
    smy = sigma[:-1, :] * mu_0 / eps_0
    cex = (Ez[:, 1:] - Ez[:, :-1]) / dy
    cey = (Ez[1:, :] - Ez[:-1, :]) / dx
    dnx = 1.0 + smx * dt / (2.0 * mu_0)
    Hx = ((1.0 - smx * dt / (2.0 * mu_0)) / dnx) * Hx - ((dt / mu_0) / dnx) * cex
    dny = 1.0 + smy * dt / (2.0 * mu_0)
    Hy = ((1.0 - smy * dt / (2.0 * mu_0)) / dny) * Hy + ((dt / mu_0) / dny) * cey
    return Hx, Hy


def update_e(Ez, Hx, Hy, sigma, eps_r, dx, dy, dt, eps_0=EPS_0):
    """numpy_backend.py:63-88 (in place on Ez's interior)."""
    cplx = np.iscomplexobj(Ez) or np.iscomplexobj(Hx) or np.iscomplexobj(Hy)
    chx = np.zeros_like(Ez, dtype=np.complex128) if cplx else np.zeros_like(Ez)
    chy = np.zeros_like(Ez, dtype=np.complex128) if cplx else np.zeros_like(Ez)
    chx[1:-1, 1:-1] = (Hx[1:-1, 1:] - Hx[1:-1, :-1]) / dy
    chy[1:-1, 1:-1] = (Hy[1:, 1:-1] - Hy[:-1, 1:-1]) / dx
    s = sigma[1:-1, 1:-1]
    e = eps_r[1:-1, 1:-1]
    den = 1.0 + s * dt / (2.0 * eps_0 * e)
    f1 = (1.0 - s * dt / (2.0 * eps_0 * e)) / den
    f2 = (dt / (eps_0 * e)) / den
    Ez[1:-1, 1:-1] = f1 * Ez[1:-1, 1:-1] + f2 * (-chx[1:-1, 1:-1] + chy[1:-1, 1:-1])
    return Ez


_BEHIND_2D = {"+x": (0, -1), "-x": (0, 1), "+y": (-1, 0), "-y": (1, 0)}


class _ModeInjector:
    """helper.py:8-54 for one ModeSource. Points are added in order and, with
    enforce_direction, each addition zeroes the cell behind it. When no zeroed
    cell is also an injected cell (true for axis-aligned lines) the per-point
    sequence equals "add all, then zero all", which is applied vectorised;
    otherwise the points are replayed one by one."""

    def __init__(self, src, dx, dy, nx, ny):
        self.signal = np.asarray(src.signal)
        pts = src.mode_profiles[0]
        self.amp, self.ix, self.iy, self.zx, self.zy = [], [], [], [], []
        self.seq = []
        enforce = getattr(src, "enforce_direction", True)
        beh = _BEHIND_2D.get(src.direction)
        for p in pts:
            amp, xr, yr = p[0], p[1], p[2]
            x, y = int(round(xr / dx)), int(round(yr / dy))
            if x < 0 or x >= nx or y < 0 or y >= ny:
                continue
            self.amp.append(amp)
            self.ix.append(x)
            self.iy.append(y)
            z = None
            if enforce and beh is not None:
                by, bx = beh
                yy, xx = y + by, x + bx
                ok = {"+x": x > 0, "-x": x < nx - 1, "+y": y > 0, "-y": y < ny - 1}[src.direction]
                if ok:
                    z = (yy, xx)
                    self.zy.append(yy)
                    self.zx.append(xx)
            self.seq.append((amp, y, x, z))
        self.amp = np.asarray(self.amp, dtype=complex)
        inj = set(zip(self.iy, self.ix))
        self.vectorised = not any((zy, zx) in inj for zy, zx in zip(self.zy, self.zx))

    def apply(self, Ez, n):
        mod = self.signal[n]
        if self.vectorised:
            np.add.at(Ez, (np.asarray(self.iy, dtype=int), np.asarray(self.ix, dtype=int)), self.amp * mod)
            if self.zx:
                Ez[np.asarray(self.zy, dtype=int), np.asarray(self.zx, dtype=int)] = 0
            return
        for amp, y, x, z in self.seq:
            Ez[y, x] += amp * mod
            if z is not None:
                Ez[z] = 0


class _GaussInjector:
    """helper.py:96-118 (2D): patch exp(-r^2/2w^2)/4 times signal[step]."""

    def __init__(self, src, dx, dy, nx, ny):
        self.signal = np.asarray(src.signal)
        cx, cy = src.position[0] / dx, src.position[1] / dy
        wx, wy = src.width / dx, src.width / dy
        hx, hy = max(1, int(round(3 * wx))), max(1, int(round(3 * wy)))
        ix, iy = int(round(cx)), int(round(cy))
        self.x0, self.x1 = max(0, ix - hx), min(nx, ix + hx + 1)
        self.y0, self.y1 = max(0, iy - hy), min(ny, iy + hy + 1)
        yg, xg = np.meshgrid(np.arange(self.y0, self.y1), np.arange(self.x0, self.x1), indexing="ij")
        eps = 1e-9
        ex = -((xg - cx) ** 2 / (2 * (wx ** 2 + eps)) + (yg - cy) ** 2 / (2 * (wy ** 2 + eps)))
        self.amp = np.exp(ex) / 4

    def apply(self, Ez, n):
        Ez[self.y0:self.y1, self.x0:self.x1] += self.amp * self.signal[n]


def monitor_points(mon, dx, dy):
    """monitors.py:204-220."""
    sx, sy = int(round(mon.start[0] / dx)), int(round(mon.start[1] / dy))
    ex, ey = int(round(mon.end[0] / dx)), int(round(mon.end[1] / dy))
    n = max(abs(ex - sx), abs(ey - sy)) + 1
    return np.linspace(sx, ex, n, dtype=int), np.linspace(sy, ey, n, dtype=int)


def _sample(arr, ys, xs):
    ok = (ys >= 0) & (ys < arr.shape[0]) & (xs >= 0) & (xs < arr.shape[1])
    out = np.zeros(len(xs), dtype=arr.dtype)
    out[ok] = arr[ys[ok], xs[ok]]
    return out


def run(eps_r, sigma, dx, dy, dt, n_steps, sources=(), monitors=(), accumulate_power=False, complex_fields=True,
        dft_freqs=None, record=True, snapshot_steps=(), fields=None):
    """Run n_steps of the reference loop. ``sources`` are ModeSource / GaussianSource
    like objects (duck-typed: mode_profiles/signal/direction/enforce_direction or
    position/width/signal). ``monitors`` are objects with start/end/record_interval.

    Returns dict(Ez, Hx, Hy, power (summed, not averaged), count, records: list per
    monitor of dict(Ez, Hx, Hy, t, power), dft: per monitor [freq][point][5],
    snapshots: {step: (Ez, Hx, Hy)})."""
    ny, nx = eps_r.shape
    if fields is None:
        Ez = np.zeros((ny, nx), dtype=np.complex128 if complex_fields else np.float64)
        Hx = np.zeros((ny, nx - 1))
        Hy = np.zeros((ny - 1, nx))
    else:
        Ez, Hx, Hy = (np.array(f) for f in fields)
    inj = []
    for s in sources:
        if hasattr(s, "mode_profiles"):
            inj.append(_ModeInjector(s, dx, dy, nx, ny))
        else:
            inj.append(_GaussInjector(s, dx, dy, nx, ny))
    mons = []
    for m in monitors:
        xs, ys = monitor_points(m, dx, dy)
        mons.append(dict(xs=xs, ys=ys, k=getattr(m, "record_interval", 1), last=-1, Ez=[], Hx=[], Hy=[], t=[],
                         power=[]))
    freqs = None if dft_freqs is None else np.asarray(dft_freqs, dtype=float)
    dft = [np.zeros((len(freqs), len(m["xs"]), 5), dtype=complex) for m in mons] if freqs is not None else None
    power = np.zeros((ny, nx)) if accumulate_power else None
    snaps = {}
    t = 0
    for n in range(n_steps):
        Hx, Hy = update_h(Hx, Hy, Ez, sigma, dx, dy, dt)
        Ez = update_e(Ez, Hx, Hy, sigma, eps_r, dx, dy, dt)
        for j in inj:
            j.apply(Ez, n)
        for i, m in enumerate(mons):
            if record and (n - m["last"]) >= m["k"]:
                ez, hx, hy = _sample(Ez, m["ys"], m["xs"]), _sample(Hx, m["ys"], m["xs"]), _sample(Hy, m["ys"], m["xs"])
                m["Ez"].append(ez)
                m["Hx"].append(hx)
                m["Hy"].append(hy)
                m["t"].append(t)
                sx, sy = -ez * hy, ez * hx
                m["power"].append(np.sum(np.sqrt(sx ** 2 + sy ** 2)))
                m["last"] = n
            if dft is not None:
                xs, ys = m["xs"], m["ys"]
                q = np.stack([_sample(Ez, ys, xs), _sample(Hx, ys, xs), _sample(Hx, ys, xs - 1),
                              _sample(Hy, ys, xs), _sample(Hy, ys - 1, xs)], axis=-1)
                q = np.real(q)
                w = 2 * np.pi * freqs
                pe = np.exp(-1j * w * ((n + 1.0) * dt))
                ph = np.exp(-1j * w * ((n + 0.5) * dt))
                dft[i][:, :, 0] += pe[:, None] * q[None, :, 0]
                dft[i][:, :, 1:] += ph[:, None, None] * q[None, :, 1:]
        if accumulate_power:
            Hxf = np.zeros_like(Ez, dtype=np.complex128)
            Hyf = np.zeros_like(Ez, dtype=np.complex128)
            Hxf[:, :-1] = Hx
            Hyf[:-1, :] = Hy
            er, ei = np.real(Ez), np.imag(Ez)
            sx = -er * np.real(Hyf) - ei * np.imag(Hyf)
            sy = er * np.real(Hxf) + ei * np.imag(Hxf)
            power += sx ** 2 + sy ** 2
        if n in snapshot_steps:
            snaps[n] = (Ez.copy(), Hx.copy(), Hy.copy())
        t += dt
    recs = [{k: (np.array(m[k]) if k != "t" else np.asarray(m[k], dtype=float)) for k in ("Ez", "Hx", "Hy", "t", "power")}
            for m in mons]
    if dft is not None:
        dft = [d * dt for d in dft]
    return dict(Ez=Ez, Hx=Hx, Hy=Hy, power=power, count=n_steps, records=recs, dft=dft, snapshots=snaps)


def flux_from_dft(d, vertical, dx, dy):
    """Flux per frequency of a monitor's DFT [freq][point][5] (see beamz_b200 Monitor.flux)."""
    ez = d[:, :, 0]
    if vertical:
        hc = 0.5 * (d[:, :, 1] + d[:, :, 2])
        return 0.5 * np.real(np.sum(ez * np.conj(hc), axis=1)) * dy
    hc = 0.5 * (d[:, :, 3] + d[:, :, 4])
    return -0.5 * np.real(np.sum(ez * np.conj(hc), axis=1)) * dx
