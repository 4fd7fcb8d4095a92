"""Host-side compilation of sources and monitors into device cell operations.

Sources (beamz/simulation/helper.py:5-118) become a list of per-cell events in
application order — "add amplitude * signal[step]" for every ModeSource profile
point and GaussianSource patch cell, and "set to 0" for the cell behind a
ModeSource point when ``enforce_direction`` holds. Events on the same cell are
merged into ``v = mul * v + sum_s W_s * signal_s[step]`` (exact composition of the
sequence), which the step kernel applies after the E update.

Monitors become the list of cells they sample (monitors.py:204-220).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from ..devices.monitors import Monitor
from ..devices.sources import GaussianSource, ModeSource

_BEHIND = {"+x": (0, 0, -1), "-x": (0, 0, 1), "+y": (0, -1, 0), "-y": (0, 1, 0), "+z": (-1, 0, 0), "-z": (1, 0, 0)}


@dataclass
class SourceOps:
    cell: np.ndarray          # int32 [n_ops], sorted (stable) by linear cell index
    mul: np.ndarray           # float64 [n_ops]
    weight: np.ndarray        # float64 [n_ops, 2]: (Re, Im) of the per-op weight
    sig: np.ndarray           # int32 [n_ops]: signal row
    signals: np.ndarray       # float64 [n_signals, n_steps]
    complex_weights: bool     # any weight has a non-zero imaginary part
    rows: int = 0             # number of grid rows (for the CSR row pointer)
    row_ptr: np.ndarray = field(default=None)  # int32 [rows + 1]


class _Signals:
    def __init__(self, n_steps: int):
        self.rows: list[np.ndarray] = []
        self.n_steps = n_steps

    def add(self, sig) -> tuple[int, int | None]:
        """Register a signal; returns (real row, imag row or None)."""
        a = np.asarray(sig)
        if a.ndim == 0:
            raise TypeError("source signal must be an array indexed by time step, got a scalar")
        row = np.zeros(self.n_steps)
        im = None
        n = min(len(a), self.n_steps)
        row[:n] = np.real(a[:n])
        self.rows.append(row)
        r = len(self.rows) - 1
        if np.iscomplexobj(a) and np.any(np.imag(a[:n]) != 0):
            irow = np.zeros(self.n_steps)
            irow[:n] = np.imag(a[:n])
            self.rows.append(irow)
            im = len(self.rows) - 1
        return r, im


def _gaussian_patch(src, grid_shape, spacing, is_3d):
    """Cells and weights of a GaussianSource patch (helper.py:56-118)."""
    if is_3d:
        nz, ny, nx = grid_shape
        dx, dy, dz = spacing
        cx, cy, cz = src.position[0] / dx, src.position[1] / dy, src.position[2] / dz
        w = [src.width / dx, src.width / dy, src.width / dz]
        half = [max(1, int(round(3 * v))) for v in w]
        ci = [int(round(cx)), int(round(cy)), int(round(cz))]
        xs0, xs1 = max(0, ci[0] - half[0]), min(nx, ci[0] + half[0] + 1)
        ys0, ys1 = max(0, ci[1] - half[1]), min(ny, ci[1] + half[1] + 1)
        zs0, zs1 = max(0, ci[2] - half[2]), min(nz, ci[2] + half[2] + 1)
        zs1 = min(zs1, nz - 1)  # Ez has nz-1 layers
        zg, yg, xg = np.meshgrid(np.arange(zs0, zs1), np.arange(ys0, ys1), np.arange(xs0, xs1), indexing="ij")
        eps = 1e-9
        expo = -((xg - cx) ** 2 / (2 * (w[0] ** 2 + eps)) + (yg - cy) ** 2 / (2 * (w[1] ** 2 + eps))
                 + (zg - cz) ** 2 / (2 * (w[2] ** 2 + eps)))
        amp = np.exp(expo)
        z_ez = max(0, min(nz - 2, zs0))
        zz = zg - zs0 + z_ez
        keep = zz < nz - 1
        return (zz[keep], yg[keep], xg[keep]), amp[keep]
    ny, nx = grid_shape
    dx, dy = spacing
    cx, cy = src.position[0] / dx, src.position[1] / dy
    wx, wy = src.width / dx, src.width / dy
    hx, hy = max(1, int(round(3 * wx))), max(1, int(round(3 * wy)))
    ix, iy = int(round(cx)), int(round(cy))
    x0, x1 = max(0, ix - hx), min(nx, ix + hx + 1)
    y0, y1 = max(0, iy - hy), min(ny, iy + hy + 1)
    yg, xg = np.meshgrid(np.arange(y0, y1), np.arange(x0, x1), indexing="ij")
    eps = 1e-9
    expo = -((xg - cx) ** 2 / (2 * (wx ** 2 + eps)) + (yg - cy) ** 2 / (2 * (wy ** 2 + eps)))
    return (yg.ravel(), xg.ravel()), (np.exp(expo) / 4).ravel()


def compile_sources(sources, grid_shape, spacing, n_steps, is_3d=False) -> SourceOps:
    """Merge every source's injection into per-cell operations.

    grid_shape is (ny, nx) or (nz, ny, nx) of the material grid; spacing is
    (dx, dy) or (dx, dy, dz). In 3D the operations act on Ez (nz-1 layers)."""
    sigs = _Signals(n_steps)
    ev_cell, ev_mul, ev_w, ev_sig = [], [], [], []

    def lin(*idx):
        if is_3d:
            z, y, x = idx
            return (z * grid_shape[1] + y) * grid_shape[2] + x
        y, x = idx
        return y * grid_shape[1] + x

    def add(cell, w, row_re, row_im):
        ev_cell.append(cell); ev_mul.append(1.0); ev_w.append(complex(w)); ev_sig.append(row_re)  # noqa: E702
        if row_im is not None:  # w * (s_re + i s_im): the i*w part rides on the imaginary row
            ev_cell.append(cell); ev_mul.append(1.0); ev_w.append(1j * complex(w)); ev_sig.append(row_im)  # noqa: E702

    def zero(cell):
        ev_cell.append(cell); ev_mul.append(0.0); ev_w.append(0j); ev_sig.append(0)  # noqa: E702

    for src in sources:
        if isinstance(src, ModeSource):
            rr, ri = sigs.add(src.signal)
            enforce = getattr(src, "enforce_direction", True)
            behind = _BEHIND.get(src.direction)
            if is_3d:
                nz, ny, nx = grid_shape
                dx, dy, dz = spacing
                n_ez = nz - 1
            else:
                ny, nx = grid_shape
                dx, dy = spacing
            for pt in src.mode_profiles[0]:
                if len(pt) == 4:
                    amp, xr, yr, zr = pt
                else:
                    amp, xr, yr = pt
                    zr = 0
                x, y = int(round(xr / dx)), int(round(yr / dy))
                if is_3d:
                    z = int(round(zr / dz))
                    if x < 0 or x >= nx or y < 0 or y >= ny or z < 0 or z >= nz:
                        continue
                    zt = min(z, n_ez - 1) if z < n_ez else n_ez // 2
                    add(lin(zt, y, x), amp, rr, ri)
                    if enforce and behind is not None:
                        bz_, by, bx = behind
                        zz, yy, xx = zt + bz_, y + by, x + bx
                        if 0 <= xx < nx and 0 <= yy < ny and 0 <= zz < n_ez:
                            zero(lin(zz, yy, xx))
                else:
                    if x < 0 or x >= nx or y < 0 or y >= ny:
                        continue
                    add(lin(y, x), amp, rr, ri)
                    if enforce and behind is not None and behind[0] == 0:
                        yy, xx = y + behind[1], x + behind[2]
                        if 0 <= xx < nx and 0 <= yy < ny:
                            zero(lin(yy, xx))
        elif isinstance(src, GaussianSource):
            rr, ri = sigs.add(src.signal)
            idx, amp = _gaussian_patch(src, grid_shape, spacing, is_3d)
            cells = lin(*idx)
            for c, a in zip(np.ravel(cells), np.ravel(amp)):
                add(int(c), a, rr, ri)
        else:
            raise TypeError(f"Unsupported source type: {type(src)}")

    rows = grid_shape[0] * grid_shape[1] if is_3d else grid_shape[0]
    row_len = grid_shape[2] if is_3d else grid_shape[1]
    if not ev_cell:
        empty = np.zeros(0)
        return SourceOps(np.zeros(0, np.int32), empty, np.zeros((0, 2)), np.zeros(0, np.int32),
                         np.zeros((max(1, len(sigs.rows)), n_steps)), False, rows, np.zeros(rows + 1, np.int32))
    cell = np.asarray(ev_cell, dtype=np.int64)
    order = np.argsort(cell, kind="stable")
    o_cell, o_mul, o_w, o_sig = [], [], [], []
    k = 0
    n = len(order)
    while k < n:
        c = cell[order[k]]
        m = 1.0
        weights: dict[int, complex] = {}
        while k < n and cell[order[k]] == c:
            e = order[k]
            if ev_mul[e] == 0.0:
                m = 0.0
                weights = {s: 0j for s in weights}
            else:
                weights[ev_sig[e]] = weights.get(ev_sig[e], 0j) + ev_w[e]
            k += 1
        items = [(s, w) for s, w in weights.items() if w != 0] or [(0, 0j)]
        for q, (s, w) in enumerate(items):
            o_cell.append(c)
            o_mul.append(m if q == 0 else 1.0)
            o_w.append((w.real, w.imag))
            o_sig.append(s)
    ops_cell = np.asarray(o_cell, dtype=np.int64)
    row_ptr = np.searchsorted(ops_cell // row_len, np.arange(rows + 1), side="left").astype(np.int32)
    w = np.asarray(o_w, dtype=np.float64).reshape(-1, 2)
    signals = np.stack(sigs.rows) if sigs.rows else np.zeros((1, n_steps))
    return SourceOps(ops_cell.astype(np.int32), np.asarray(o_mul), w, np.asarray(o_sig, dtype=np.int32), signals,
                     bool(np.any(w[:, 1] != 0)), rows, row_ptr)


@dataclass
class MonitorPoints:
    monitors: list              # monitors sampled on the device
    slices: list                # per monitor: slice of the global point index range
    valid: list                 # per monitor: boolean mask of in-grid points
    cell: np.ndarray            # int32 [n_ops] sorted cells
    point: np.ndarray           # int32 [n_ops] global point slot of each op
    n_points: int
    row_ptr: np.ndarray


def compile_monitors_2d(monitors, nx, ny, dx, dy) -> MonitorPoints:
    mons, slices, valid = [], [], []
    cells, slots = [], []
    base = 0
    for m in monitors:
        if not isinstance(m, Monitor) or getattr(m, "is_3d", False):
            continue
        pts = m.get_grid_points_2d(dx, dy)
        ok = np.array([0 <= x < nx and 0 <= y < ny for x, y in pts], dtype=bool)
        for k, (x, y) in enumerate(pts):
            if ok[k]:
                cells.append(int(y) * nx + int(x))
                slots.append(base + k)
        mons.append(m)
        slices.append(slice(base, base + len(pts)))
        valid.append(ok)
        base += len(pts)
    cell = np.asarray(cells, dtype=np.int64)
    order = np.argsort(cell, kind="stable")
    cell = cell[order]
    slot = np.asarray(slots, dtype=np.int64)[order]
    row_ptr = np.searchsorted(cell // nx, np.arange(ny + 1), side="left").astype(np.int32)
    return MonitorPoints(mons, slices, valid, cell.astype(np.int32), slot.astype(np.int32), base, row_ptr)
