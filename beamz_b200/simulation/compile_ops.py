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
    # events in application order, as arrays per source: cell, mul, complex weight, signal row
    ev_cell, ev_mul, ev_w, ev_sig = [], [], [], []

    def lin(*idx):
        if is_3d:
            z, y, x = idx
            return (z * grid_shape[1] + y) * grid_shape[2] + x
        y, x = idx
        return y * grid_shape[1] + x

    def emit(cells, amps, zero_cells, zero_ok, row_re, row_im):
        """Per point i, in this order: add amps[i] on row_re at cells[i], the i*amps[i]
        part on row_im (complex signals), then zero zero_cells[i] where zero_ok[i]."""
        n = len(cells)
        amps = np.asarray(amps, dtype=np.complex128)
        parts = [(np.asarray(cells, np.int64), np.ones(n), amps, np.full(n, row_re), np.ones(n, bool))]
        if row_im is not None:  # w * (s_re + i s_im): the i*w part rides on the imaginary row
            parts.append((np.asarray(cells, np.int64), np.ones(n), 1j * amps, np.full(n, row_im), np.ones(n, bool)))
        if zero_cells is not None:
            parts.append((np.asarray(zero_cells, np.int64), np.zeros(n), np.zeros(n, np.complex128), np.zeros(n, int),
                          np.asarray(zero_ok, bool)))
        k = len(parts)
        cell = np.stack([q[0] for q in parts], axis=1).reshape(-1)  # point-major interleave
        keep = np.stack([q[4] for q in parts], axis=1).reshape(-1)
        ev_cell.append(cell[keep])
        ev_mul.append(np.stack([q[1] for q in parts], axis=1).reshape(-1)[keep])
        ev_w.append(np.stack([q[2] for q in parts], axis=1).reshape(-1)[keep])
        ev_sig.append(np.stack([q[3] for q in parts], axis=1).reshape(-1)[keep].astype(np.int64))
        del k

    for src in sources:
        if isinstance(src, ModeSource):
            rr, ri = sigs.add(src.signal)
            enforce = getattr(src, "enforce_direction", True)
            behind = _BEHIND.get(src.direction)
            pts = src.mode_profiles[0]
            if len(pts) == 0:
                continue
            tab = np.asarray(pts, dtype=np.complex128)  # rows (amp, x, y[, z])
            amp, xr, yr = tab[:, 0], tab[:, 1].real, tab[:, 2].real
            zr = tab[:, 3].real if tab.shape[1] == 4 else np.zeros(len(tab))
            if is_3d:
                nz, ny, nx = grid_shape
                dx, dy, dz = spacing
                n_ez = nz - 1
                x, y, z = np.round(xr / dx).astype(np.int64), np.round(yr / dy).astype(np.int64), \
                    np.round(zr / dz).astype(np.int64)
                ok = (x >= 0) & (x < nx) & (y >= 0) & (y < ny) & (z >= 0) & (z < nz)
                x, y, z, amp = x[ok], y[ok], z[ok], amp[ok]
                zt = np.where(z < n_ez, np.minimum(z, n_ez - 1), n_ez // 2)
                zc = zok = None
                if enforce and behind is not None:
                    zz, yy, xx = zt + behind[0], y + behind[1], x + behind[2]
                    zok = (xx >= 0) & (xx < nx) & (yy >= 0) & (yy < ny) & (zz >= 0) & (zz < n_ez)
                    zc = lin(zz, yy, xx)
                emit(lin(zt, y, x), amp, zc, zok, rr, ri)
            else:
                ny, nx = grid_shape
                dx, dy = spacing
                x, y = np.round(xr / dx).astype(np.int64), np.round(yr / dy).astype(np.int64)
                ok = (x >= 0) & (x < nx) & (y >= 0) & (y < ny)
                x, y, amp = x[ok], y[ok], amp[ok]
                zc = zok = None
                if enforce and behind is not None and behind[0] == 0:
                    yy, xx = y + behind[1], x + behind[2]
                    zok = (xx >= 0) & (xx < nx) & (yy >= 0) & (yy < ny)
                    zc = lin(yy, xx)
                emit(lin(y, x), amp, zc, zok, rr, ri)
        elif isinstance(src, GaussianSource):
            rr, ri = sigs.add(src.signal)
            idx, amp = _gaussian_patch(src, grid_shape, spacing, is_3d)
            emit(np.ravel(lin(*idx)), np.ravel(amp), None, None, rr, ri)
        else:
            raise TypeError(f"Unsupported source type: {type(src)}")

    rows = grid_shape[0] * grid_shape[1] if is_3d else grid_shape[0]
    row_len = grid_shape[2] if is_3d else grid_shape[1]
    cell = np.concatenate(ev_cell) if ev_cell else np.zeros(0, np.int64)
    if len(cell) == 0:
        empty = np.zeros(0)
        return SourceOps(np.zeros(0, np.int32), empty, np.zeros((0, 2)), np.zeros(0, np.int32),
                         np.zeros((max(1, len(sigs.rows)), n_steps)), False, rows, np.zeros(rows + 1, np.int32))
    mul, wts, sgs = np.concatenate(ev_mul), np.concatenate(ev_w), np.concatenate(ev_sig)
    # Merge each cell's events in application order (stable sort by cell): a zeroing
    # event sets the cell's factor to 0 and drops the weights added before it, so
    # the merged weight of a signal is the sum of its adds after the cell's last
    # zeroing; signals keep the order in which they first appear on the cell, zero
    # weights are dropped, and a cell left with none gets one (0, 0) operation.
    order = np.argsort(cell, kind="stable")
    sc, sm, sw, ss = cell[order], mul[order], wts[order], sgs[order]
    n = len(sc)
    start = np.r_[True, sc[1:] != sc[:-1]]
    grp = np.cumsum(start) - 1
    n_grp = int(grp[-1]) + 1
    pos = np.arange(n)
    zero = sm == 0.0
    last_zero = np.full(n_grp, -1, dtype=np.int64)
    np.maximum.at(last_zero, grp[zero], pos[zero])
    has_zero = last_zero >= 0
    adds = ~zero
    key = grp * (int(ss.max()) + 1 if n else 1) + ss
    ukey, first, inv = np.unique(np.where(adds, key, -1), return_index=True, return_inverse=True)
    live = adds & (pos > last_zero[grp])
    wsum = np.zeros(len(ukey), dtype=np.complex128)
    np.add.at(wsum, inv[live], sw[live])
    pair = ukey >= 0
    p_grp, p_sig, p_first, p_w = grp[first[pair]], ss[first[pair]], first[pair], wsum[pair]
    keep = p_w != 0
    p_grp, p_sig, p_first, p_w = p_grp[keep], p_sig[keep], p_first[keep], p_w[keep]
    empty_grp = np.setdiff1d(np.arange(n_grp), p_grp)
    g_all = np.concatenate([p_grp, empty_grp])
    f_all = np.concatenate([p_first, np.full(len(empty_grp), -1)])
    srt = np.lexsort((f_all, g_all))
    g_all = g_all[srt]
    o_sig = np.concatenate([p_sig, np.zeros(len(empty_grp), dtype=np.int64)])[srt]
    o_wc = np.concatenate([p_w, np.zeros(len(empty_grp), dtype=np.complex128)])[srt]
    lead = np.r_[True, g_all[1:] != g_all[:-1]]
    o_mul = np.where(lead & has_zero[g_all], 0.0, 1.0)
    o_cell = sc[start][g_all]
    o_w = np.stack([o_wc.real, o_wc.imag], axis=1)
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
