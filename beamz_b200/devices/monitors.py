"""Field monitors (beamz/devices/monitors.py:7-589).

A 2D monitor is a line sampled at grid cells; a 3D monitor is a plane slice.
The reference copies every field to the host every step and samples it in
Python; here the step kernel samples the monitor cells on the GPU into a device
record buffer (and, when frequencies are requested, into float64 DFT
accumulators) and the simulation fills ``fields``, ``power_history`` and
``power_timestamps`` from that buffer when the run ends, with the same layout and
values as the reference (``fields['Ez']`` is one sample vector per recorded step).

Additions over the reference (it has no frequency-domain monitors):
``frequencies`` / ``wavelengths`` enable on-the-fly DFT of Ez and of H centred on
the E nodes; ``flux(i)`` and ``mode_overlap(profile, i)`` read them out.
"""
from __future__ import annotations

from typing import Callable, Optional

import numpy as np

from ..const import LIGHT_SPEED


class Monitor:
    def __init__(self, design=None, start=(0, 0), end=None, plane_normal=None, plane_position=0, size=None,
                 record_fields=True, accumulate_power=True, live_update=False, record_interval=1,
                 max_history_steps=None, objective_function: Optional[Callable[["Monitor"], float]] = None,
                 name: Optional[str] = None, frequencies=None, wavelengths=None):
        self.design = design
        self.should_record_fields = record_fields
        self.accumulate_power = accumulate_power
        self.live_update = live_update
        self.record_interval = record_interval
        self.max_history_steps = max_history_steps
        self.objective_function = objective_function
        self.objective_value: Optional[float] = None
        self.name = name
        self.is_3d = self._determine_3d_mode(start, end, design)
        keys = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz") if self.is_3d else ("Ez", "Hx", "Hy")
        self.fields = {k: [] for k in keys}
        self.fields["t"] = []
        self.power_accumulated = None
        self.energy_history = []
        self.power_history = []
        self.power_timestamps = []
        self.power_accumulation_count = 0
        self.step_count = 0
        self.last_record_step = -1
        if frequencies is None and wavelengths is not None:
            frequencies = LIGHT_SPEED / np.asarray(wavelengths, dtype=float)
        self.frequencies = None if frequencies is None else np.atleast_1d(np.asarray(frequencies, dtype=float))
        self.dft = None  # filled after a run: dict of complex arrays
        if self.is_3d:
            self._init_3d_monitor(start, end, plane_normal, plane_position, size)
        else:
            self._init_2d_monitor(start, end)

    # ---- geometry ----------------------------------------------------------
    def _determine_3d_mode(self, start, end, design):
        if end is not None and len(end) == 3:
            return True
        if len(start) == 3:
            return True
        if end is not None and len(start) == 2 and len(end) == 2:
            return False
        return bool(design is not None and getattr(design, "is_3d", False))

    def _init_2d_monitor(self, start, end):
        if end is None:
            end = start
        self.start, self.end = start, end
        self.position = ((start[0] + end[0]) / 2, (start[1] + end[1]) / 2)
        self.monitor_type = "line"

    def _init_3d_monitor(self, start, end, plane_normal, plane_position, size):
        if len(start) == 2:
            start = (start[0], start[1], 0.0)
        self.start = start
        if end is not None:
            if len(end) == 2:
                end = (end[0], end[1], start[2])
            self.end = end
            self.size = (abs(end[0] - start[0]), abs(end[1] - start[1]))
            self.plane_position = start[2]
            self.plane_normal = "z"
            self.start = (min(start[0], end[0]), min(start[1], end[1]), start[2])
        else:
            self.end = None
            self.plane_normal = plane_normal or "z"
            self.plane_position = plane_position
            if size is None:
                if self.design:
                    d = self.design
                    size = {"z": (d.width, d.height), "y": (d.width, d.depth or d.width)}.get(
                        self.plane_normal, (d.height, d.depth or d.height))
                else:
                    size = (1e-6, 1e-6)
            self.size = size
        self.monitor_type = "plane"
        self.position = self._get_plane_center()
        self.vertices = self._generate_plane_vertices()

    def _xy_plane(self):
        return self.plane_normal == "z" or getattr(self, "end", None) is not None

    def _generate_plane_vertices(self):
        s0, s1 = self.size
        if self._xy_plane():
            x, y, z = self.start[0], self.start[1], self.plane_position
            return [(x, y, z), (x + s0, y, z), (x + s0, y + s1, z), (x, y + s1, z)]
        if self.plane_normal == "y":
            x, z, y = self.start[0], self.start[2], self.plane_position
            return [(x, y, z), (x + s0, y, z), (x + s0, y, z + s1), (x, y, z + s1)]
        y, z, x = self.start[1], self.start[2], self.plane_position
        return [(x, y, z), (x, y + s0, z), (x, y + s0, z + s1), (x, y, z + s1)]

    def _get_plane_center(self):
        s0, s1 = self.size
        if self._xy_plane():
            return (self.start[0] + s0 / 2, self.start[1] + s1 / 2, self.plane_position)
        if self.plane_normal == "y":
            return (self.start[0] + s0 / 2, self.plane_position, self.start[2] + s1 / 2)
        return (self.plane_position, self.start[1] + s0 / 2, self.start[2] + s1 / 2)

    def get_grid_points_2d(self, dx, dy):
        """Cells sampled by a line monitor (monitors.py:204-220): the endpoints are
        rounded to cells and joined by np.linspace with integer truncation."""
        sx, sy = int(round(self.start[0] / dx)), int(round(self.start[1] / dy))
        ex, ey = int(round(self.end[0] / dx)), int(round(self.end[1] / dy))
        n = max(abs(ex - sx), abs(ey - sy)) + 1
        xs = np.linspace(sx, ex, n, dtype=int)
        ys = np.linspace(sy, ey, n, dtype=int)
        return list(zip(xs, ys))

    def get_grid_slice_3d(self, dx, dy, dz, field_shape=None):
        """Plane slice indices (monitors.py:222-273): (y, x, z_index) for z-normal
        planes, (y_index, x, z) for y-normal, (y, x_index, z) for x-normal."""
        bnx = max(1, int(round(getattr(self.design, "width", 0.0) / dx)))
        bny = max(1, int(round(getattr(self.design, "height", 0.0) / dy)))
        bnz = max(1, int(round((getattr(self.design, "depth", 0.0) or 0.0) / dz)))
        clamp = lambda v, hi: max(0, min(v, hi))  # noqa: E731
        s0, s1 = self.size
        if self.plane_normal == "z":
            zi = clamp(int(round(self.plane_position / dz)), bnz - 1)
            xs, xe = int(round(self.start[0] / dx)), int(round((self.start[0] + s0) / dx))
            ys, ye = int(round(self.start[1] / dy)), int(round((self.start[1] + s1) / dy))
            return slice(clamp(ys, bny - 1), clamp(ye, bny)), slice(clamp(xs, bnx - 1), clamp(xe, bnx)), zi
        if self.plane_normal == "y":
            yi = clamp(int(round(self.plane_position / dy)), bny - 1)
            xs, xe = int(round(self.start[0] / dx)), int(round((self.start[0] + s0) / dx))
            zs, ze = int(round(self.start[2] / dz)), int(round((self.start[2] + s1) / dz))
            return yi, slice(clamp(xs, bnx - 1), clamp(xe, bnx)), slice(clamp(zs, bnz - 1), clamp(ze, bnz))
        xi = clamp(int(round(self.plane_position / dx)), bnx - 1)
        ys, ye = int(round(self.start[1] / dy)), int(round((self.start[1] + s0) / dy))
        zs, ze = int(round(self.start[2] / dz)), int(round((self.start[2] + s1) / dz))
        return slice(clamp(ys, bny - 1), clamp(ye, bny)), xi, slice(clamp(zs, bnz - 1), clamp(ze, bnz))

    # ---- host-side recording (API compatibility; the GPU path records on device)
    def should_record(self, step):
        return (step - self.last_record_step) >= self.record_interval

    def record_fields(self, *args, **kwargs):
        if self.is_3d and len(args) >= 6:
            return self.record_fields_3d(*args, **kwargs)
        return self.record_fields_2d(*args, **kwargs)

    def record_fields_2d(self, Ez, Hx, Hy, t, dx, dy, step=0):
        if not self.should_record(step):
            return
        vals = {k: [] for k in ("Ez", "Hx", "Hy")}
        for xi, yi in self.get_grid_points_2d(dx, dy):
            for k, arr in (("Ez", Ez), ("Hx", Hx), ("Hy", Hy)):
                if 0 <= yi < arr.shape[0] and 0 <= xi < arr.shape[1]:
                    v = arr[yi, xi]
                    vals[k].append(complex(v) if np.iscomplexobj(v) else float(v))
                else:
                    vals[k].append(0.0)
        self._append_2d(vals["Ez"], vals["Hx"], vals["Hy"], t)
        self.last_record_step = step
        self._manage_memory()

    def _append_2d(self, ez, hx, hy, t):
        if self.should_record_fields:
            self.fields["Ez"].append(ez)
            self.fields["Hx"].append(hx)
            self.fields["Hy"].append(hy)
            self.fields["t"].append(t)
        if self.accumulate_power:
            self._calculate_power_2d(ez, hx, hy, t)

    def record_fields_3d(self, Ex, Ey, Ez, Hx, Hy, Hz, t, dx, dy, dz, step=0):
        if not self.should_record(step):
            return
        sl = self.plane_slices_3d(dx, dy, dz, {k: a.shape for k, a in
                                               zip(("Ex", "Ey", "Ez", "Hx", "Hy", "Hz"), (Ex, Ey, Ez, Hx, Hy, Hz))})
        parts = [a[s].copy() for a, s in zip((Ex, Ey, Ez, Hx, Hy, Hz), sl)]
        self._append_3d(parts, t)
        self.last_record_step = step
        self._manage_memory()

    def plane_slices_3d(self, dx, dy, dz, shapes):
        """Per-component index tuples of the recorded plane (monitors.py:317-371):
        the plane slice clamped to each staggered array, then cropped to the common
        overlap of all six components. z-normal planes follow the reference exactly;
        for x- and y-normal planes the reference's slicing falls back to whole arrays
        and fails, so here they are sliced the same way along their own axes."""
        si = self.get_grid_slice_3d(dx, dy, dz)
        out = []
        for k in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz"):
            a0, a1, a2 = shapes[k]
            if isinstance(si[2], int):
                zi = min(max(0, si[2]), a0 - 1)
                ys = max(0, min(si[0].start or 0, a1 - 1))
                ye = max(ys, min(si[0].stop or a1, a1))
                xs = max(0, min(si[1].start or 0, a2 - 1))
                xe = max(xs, min(si[1].stop or a2, a2))
                out.append([zi, ys, ye, xs, xe, "z"])
            elif self.plane_normal == "y":
                fixed, s1, s0 = si  # (y index, x slice, z slice)
                fe = max(0, min(fixed, a1 - 1))
                xs = max(0, min(s1.start or 0, a2 - 1))
                xe = max(xs, min(s1.stop or a2, a2))
                zs = max(0, min(s0.start or 0, a0 - 1))
                ze = max(zs, min(s0.stop or a0, a0))
                out.append([fe, zs, ze, xs, xe, "y"])
            else:
                s0, fixed, s1 = si  # (y slice, x index, z slice)
                fe = max(0, min(fixed, a2 - 1))
                ys = max(0, min(s0.start or 0, a1 - 1))
                ye = max(ys, min(s0.stop or a1, a1))
                zs = max(0, min(s1.start or 0, a0 - 1))
                ze = max(zs, min(s1.stop or a0, a0))
                out.append([fe, zs, ze, ys, ye, "x"])
        n0 = min(o[2] - o[1] for o in out)
        n1 = min(o[4] - o[3] for o in out)
        res = []
        for fixed, a, _, b, _, kind in out:
            if kind == "z":
                res.append((fixed, slice(a, a + n0), slice(b, b + n1)))
            elif kind == "y":
                res.append((slice(a, a + n0), fixed, slice(b, b + n1)))
            else:
                res.append((slice(a, a + n0), slice(b, b + n1), fixed))
        return res

    def _append_3d(self, parts, t):
        if self.should_record_fields:
            for k, p in zip(("Ex", "Ey", "Ez", "Hx", "Hy", "Hz"), parts):
                self.fields[k].append(p)
            self.fields["t"].append(t)
        if self.accumulate_power:
            self._calculate_power_3d(*parts, t)

    def _calculate_power_2d(self, Ez_values, Hx_values, Hy_values, t):
        ez, hx, hy = np.array(Ez_values), np.array(Hx_values), np.array(Hy_values)
        sx = -ez * hy
        sy = ez * hx
        mag = np.sqrt(sx ** 2 + sy ** 2)
        if self.power_accumulated is None:
            self.power_accumulated = mag
        else:
            self.power_accumulated += mag
        self.power_history.append(np.sum(mag))
        self.power_timestamps.append(float(t))
        self.power_accumulation_count += 1

    def _calculate_power_3d(self, Ex, Ey, Ez, Hx, Hy, Hz, t):
        sx = Ey * Hz - Ez * Hy
        sy = Ez * Hx - Ex * Hz
        sz = Ex * Hy - Ey * Hx
        mag = np.sqrt(sx ** 2 + sy ** 2 + sz ** 2)
        if self.power_accumulated is None:
            self.power_accumulated = mag.copy()
        else:
            self.power_accumulated += mag
        self.power_history.append(np.sum(mag))
        self.power_timestamps.append(float(t))
        self.power_accumulation_count += 1

    def _manage_memory(self):
        n = self.max_history_steps
        if n is None:
            return
        for k in self.fields:
            if len(self.fields[k]) > n:
                self.fields[k] = self.fields[k][len(self.fields[k]) - n:]
        if len(self.power_history) > n:
            self.power_history = self.power_history[-n:]
            self.power_timestamps = self.power_timestamps[-n:]

    # ---- batch fill from the device record ----------------------------------
    def load_record_2d(self, ez, hx, hy, times):
        """Fill fields/power from device samples [n_rec][n_points] (complex or real),
        in one vectorised pass with the reference's per-step semantics."""
        if self.should_record_fields:
            self.fields["Ez"].extend(list(ez))
            self.fields["Hx"].extend(list(hx))
            self.fields["Hy"].extend(list(hy))
            self.fields["t"].extend(float(t) for t in times)
        if self.accumulate_power and len(times):
            sx = -ez * hy
            sy = ez * hx
            mag = np.sqrt(sx ** 2 + sy ** 2)
            acc = mag.sum(axis=0) if self.power_accumulated is None else self.power_accumulated + mag.sum(axis=0)
            self.power_accumulated = acc
            self.power_history.extend(list(mag.sum(axis=1)))
            self.power_timestamps.extend(float(t) for t in times)
            self.power_accumulation_count += len(times)
        self._manage_memory()

    # ---- objectives and I/O ---------------------------------------------------
    def evaluate_objective(self) -> Optional[float]:
        if self.objective_function is None:
            return None
        try:
            value = self.objective_function(self)
        except Exception as exc:  # noqa: BLE001 - reference swallows objective errors
            print(f"Warning: monitor objective evaluation failed: {exc}")
            return None
        if value is None:
            return None
        try:
            self.objective_value = float(value)
        except (TypeError, ValueError):
            return None
        return self.objective_value

    def get_field_statistics(self):
        if not self.fields["t"]:
            return {}
        t = self.fields["t"]
        stats = {"total_records": len(t), "time_span": t[-1] - t[0] if len(t) > 1 else 0,
                 "avg_power": np.mean(self.power_history) if self.power_history else 0,
                 "max_power": np.max(self.power_history) if self.power_history else 0,
                 "monitor_type": self.monitor_type, "is_3d": self.is_3d}
        if self.is_3d:
            stats.update(plane_normal=self.plane_normal, plane_position=self.plane_position, plane_size=self.size)
        else:
            stats.update(line_start=self.start, line_end=self.end)
        return stats

    def save_data(self, filename, format="npz"):  # noqa: A002
        if format != "npz":
            raise ValueError(f"Unsupported format: {format}")
        np.savez(filename, fields=self.fields, power_history=self.power_history,
                 power_timestamps=self.power_timestamps,
                 monitor_info={"type": self.monitor_type, "is_3d": self.is_3d})

    def load_data(self, filename):
        data = np.load(filename, allow_pickle=True)
        self.fields = data["fields"].item()
        self.power_history = list(data["power_history"])
        self.power_timestamps = list(data["power_timestamps"]) if "power_timestamps" in data else \
            list(range(len(self.power_history)))

    # ---- frequency-domain readout (DFT monitors) -------------------------------
    def flux(self, freq_index=None):
        """Time-averaged Poynting flux through the line at each DFT frequency.

        Uses Ez and H centred on the E node (mean of the two staggered samples):
        a line at constant x gives +x flux 0.5*Re(sum Ez conj(Hx_c))*dy, a line at
        constant y gives +y flux -0.5*Re(sum Ez conj(Hy_c))*dx; Hx and Hy are the
        reference's staggered components (Hx_ref = -Hy, Hy_ref = -Hx of a
        right-handed TMz field). Component 0 (the real field) is used."""
        if self.dft is None:
            raise RuntimeError("monitor has no DFT data; pass frequencies= and run a simulation")
        d = self.dft
        out = d["flux"]
        return out if freq_index is None else out[freq_index]

    def mode_overlap(self, profile, freq_index=None):
        """Normalised overlap |<m, E>| / (|m| |E|) of the DFT Ez line with a mode profile."""
        if self.dft is None:
            raise RuntimeError("monitor has no DFT data")
        ez = self.dft["Ez"]  # [n_freq][n_points]
        m = np.asarray(profile, dtype=complex)
        num = np.abs(ez @ np.conj(m))
        den = np.linalg.norm(m) * np.linalg.norm(ez, axis=1)
        ov = np.where(den > 0, num / np.where(den > 0, den, 1), 0.0)
        return ov if freq_index is None else ov[freq_index]

    def add_to_plot(self, *args, **kwargs):
        raise NotImplementedError("plotting is not part of beamz_b200")

    def start_live_visualization(self, *args, **kwargs):
        pass  # live plotting is not part of beamz_b200
