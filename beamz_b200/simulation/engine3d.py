"""Device state and time loop of the 3D Yee solver.

Six components, each two ping-pong copies of [design][component][nz][ny][pitch]
(x contiguous, pitch a multiple of 32); positions outside a component's
reference shape stay zero. Per time step: ``bz_step3d`` (H then E), the compiled
source operations on Ez (``bz_cell_ops``), the plane-monitor gather
(``bz_gather``: record rows and the DFT ring) and, when requested, the |S|
accumulation (``bz_power3d``); replayed in CUDA-graph chunks.
"""
from __future__ import annotations

import numpy as np
import torch

from .. import _native as nat
from ..const import EPS_0, MU_0
from ..devices.monitors import Monitor
from .compile_ops import compile_sources
from .graphs import capture, dft_phasors
from .guard import DivergenceGuard

GRAPH_CHUNK = 32
RING_LEN = GRAPH_CHUNK
COMPONENTS = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")


def _round_up(n, m):
    return (n + m - 1) // m * m


class Engine3D:
    def __init__(self, eps_r, sigma, dx, dy, dz, dt, n_steps, sources, monitors, *, precision="fp32", n_comp=None,
                 power=False, n_designs=1, record=True, use_graphs=True, tile_z=0, tile_y=8, x_cells=0, device=None):
        if not torch.cuda.is_available():
            raise RuntimeError("beamz_b200 needs a CUDA GPU (sm_100a); none is visible")
        self.dev = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
        eps_r = np.asarray(eps_r, dtype=np.float64)
        sigma = np.asarray(sigma, dtype=np.float64)
        if eps_r.ndim == 3:
            eps_r, sigma = eps_r[None], sigma[None]
        self.n_mat, self.nz, self.ny, self.nx = eps_r.shape
        if min(self.nx, self.ny, self.nz) < 2:
            raise ValueError("3D grid must be at least 2 x 2 x 2 cells")
        self.n_designs = n_designs
        self.dx, self.dy, self.dz, self.dt = float(dx), float(dy), float(dz), float(dt)
        self.n_steps = int(n_steps)
        self.h2d_bytes = 0
        self.d2h_bytes = 0
        self.dtype = {"fp32": torch.float32, "fp64": torch.float64}[precision]
        self.bz_dtype = nat.BZ_F32 if precision == "fp32" else nat.BZ_F64
        self.src = compile_sources(sources, (self.nz, self.ny, self.nx), (self.dx, self.dy, self.dz), self.n_steps,
                                   is_3d=True)
        self.n_comp = n_comp if n_comp is not None else (2 if self.src.complex_weights else 1)
        self.pitch = _round_up(self.nx, 32)
        self.vol = self.nz * self.ny * self.pitch
        shape = (n_designs, self.n_comp, self.nz, self.ny, self.pitch)
        self.f = {c: [torch.zeros(shape, dtype=self.dtype, device=self.dev) for _ in range(2)] for c in COMPONENTS}
        self.ce = torch.empty((self.n_mat, self.nz, self.ny, self.pitch), dtype=self.dtype, device=self.dev)
        self.loss = torch.empty_like(self.ce)
        self._keep = []
        te = torch.as_tensor(np.ascontiguousarray(eps_r)).to(self.dev)
        ts = torch.as_tensor(np.ascontiguousarray(sigma)).to(self.dev)
        self.h2d_bytes += eps_r.nbytes + sigma.nbytes
        nat.prepare_coeffs(te.data_ptr(), ts.data_ptr(), self.n_mat * self.nz * self.ny, self.nx, self.pitch,
                           self.bz_dtype, self.dt, EPS_0, self.dy, self.ce.data_ptr(), self.loss.data_ptr(),
                           self._stream())
        self.power = torch.zeros((n_designs, self.nz - 1, self.ny - 1, self.nx - 1), dtype=torch.float64,
                                 device=self.dev) if power else None
        g = nat.Grid3D()
        g.nx, g.ny, g.nz, g.pitch = self.nx, self.ny, self.nz, self.pitch
        g.n_designs, g.n_comp, g.n_mat, g.dtype, g.tile_z = n_designs, self.n_comp, self.n_mat, self.bz_dtype, tile_z
        g.tile_y = int(tile_y)
        g.x_cells = int(x_cells)
        g.chx, g.chy, g.chz = self.dt / (MU_0 * self.dx), self.dt / (MU_0 * self.dy), self.dt / (MU_0 * self.dz)
        g.qx, g.qz = self.dy / self.dx, self.dy / self.dz
        g.inv_kd2 = 2.0 * EPS_0 * self.dy / self.dt
        self.grid = g
        self.step_index = 0
        self._folded = 0
        self._setup_sources()
        self._setup_monitors(monitors, record)
        self.d_step = torch.zeros(1, dtype=torch.int64, device=self.dev)
        self.use_graphs = use_graphs
        self._graphs = {}
        self.kernel_timer = None  # graphs.KernelTimer around the step launches (direct launches only)
        self.guard = DivergenceGuard(self.dev)
        # kernels per step: the step itself, source operations, monitor gather, power
        self.kernels_per_step = 1 + (self.sops.n_ops > 0) + (self.gops is not None) + (self.power is not None)
        self.n_step_launches = 0  # bz_step3d launches (one per step, graph nodes included)
        self.n_kernel_launches = 0  # every launch of this library, folds included
        self.n_fold_launches = 0
        torch.cuda.current_stream().synchronize()

    @staticmethod
    def _stream():
        return torch.cuda.current_stream().cuda_stream

    def _kept(self, t):
        self._keep.append(t)
        self.h2d_bytes += t.numel() * t.element_size()
        return t

    def _setup_sources(self):
        s = self.src
        self.sops = nat.SourceOps()
        self.sops.n_ops = 0
        if len(s.cell) == 0:
            return
        t = lambda a, dt: self._kept(torch.as_tensor(np.ascontiguousarray(a)).to(self.dev, dt))  # noqa: E731
        self._src_t = dict(row=t(s.row_ptr, torch.int32), cell=t(s.cell, torch.int32), mul=t(s.mul, self.dtype),
                           w=t(s.weight[:, :self.n_comp], self.dtype), sig=t(s.sig, torch.int32),
                           signals=t(s.signals, self.dtype))
        so = self.sops
        so.n_ops, so.n_steps = len(s.cell), s.signals.shape[1]
        so.row_ptr, so.cell = self._src_t["row"].data_ptr(), self._src_t["cell"].data_ptr()
        so.mul, so.weight = self._src_t["mul"].data_ptr(), self._src_t["w"].data_ptr()
        so.sig, so.signals = self._src_t["sig"].data_ptr(), self._src_t["signals"].data_ptr()

    def _setup_monitors(self, monitors, record):
        shapes = {"Ex": (self.nz, self.ny, self.nx - 1), "Ey": (self.nz, self.ny - 1, self.nx),
                  "Ez": (self.nz - 1, self.ny, self.nx), "Hx": (self.nz - 1, self.ny - 1, self.nx),
                  "Hy": (self.nz - 1, self.ny, self.nx - 1), "Hz": (self.nz, self.ny - 1, self.nx - 1)}
        self.mons, self.mon_slices, self.mon_shape = [], [], []
        offs = []
        base = 0
        for m in monitors:
            if not isinstance(m, Monitor) or not m.is_3d:
                continue
            sl = m.plane_slices_3d(self.dx, self.dy, self.dz, shapes)
            per_c = []
            for idx in sl:
                zz, yy, xx = (np.arange(a.start, a.stop) if isinstance(a, slice) else np.array([a]) for a in idx)
                g = np.meshgrid(zz, yy, xx, indexing="ij")
                lin = ((g[0] * self.ny + g[1]) * self.pitch + g[2]).reshape(-1)
                per_c.append(lin)
            n_pts = len(per_c[0])
            two_d = tuple(a.stop - a.start for a in sl[0] if isinstance(a, slice))
            offs.append(np.stack(per_c, axis=1))
            self.mons.append(m)
            self.mon_slices.append(slice(base, base + n_pts))
            self.mon_shape.append(two_d)
            base += n_pts
        self.n_points = base
        self.gops = None
        self.record = None
        self.ring = None
        self.dft = None
        self.freqs = np.zeros(0)
        if base == 0:
            return
        self._offsets = self._kept(torch.as_tensor(np.concatenate(offs).astype(np.int64)).to(self.dev))
        go = nat.GatherOps()
        go.n_points, go.n_q, go.offset = base, 6, self._offsets.data_ptr()
        if record and any(m.should_record_fields or m.accumulate_power for m in self.mons):
            row = self.n_designs * self.n_comp * base * 6 * torch.finfo(self.dtype).bits // 8
            self.rec_rows = max(1, min(self.n_steps, (512 << 20) // max(1, row)))
            self.record = torch.zeros((self.rec_rows, self.n_designs, self.n_comp, base, 6), dtype=self.dtype,
                                      device=self.dev)
            go.record, go.n_rec, go.rec_step0 = self.record.data_ptr(), self.rec_rows, 0
        freqs = [np.asarray(m.frequencies, dtype=float) for m in self.mons if m.frequencies is not None]
        if freqs:
            self.freqs = np.concatenate(freqs)
            self.phasor = dft_phasors(self.freqs, self.n_steps, self.dt, self.dev)
            self.h2d_bytes += self.freqs.nbytes
            self.ring = torch.zeros((RING_LEN, self.n_designs, self.n_comp, base, 6), dtype=self.dtype, device=self.dev)
            self.dft = torch.zeros((self.n_designs, self.n_comp, base, len(self.freqs), 6, 2), dtype=torch.float64,
                                   device=self.dev)
            go.ring, go.ring_len = self.ring.data_ptr(), RING_LEN
        self.gops = go
        self._rec_host = []

    # ---- stepping ---------------------------------------------------------------
    def _fields(self):
        f = nat.Fields3D()
        for cp in range(2):
            for i, c in enumerate(("Ex", "Ey", "Ez")):
                f.e[cp][i] = self.f[c][cp].data_ptr()
            for i, c in enumerate(("Hx", "Hy", "Hz")):
                f.h[cp][i] = self.f[c][cp].data_ptr()
        f.ce, f.loss = self.ce.data_ptr(), self.loss.data_ptr()
        return f

    def _launch(self, step_arg, d_step_ptr):
        st = self._stream()
        fields = self._fields()
        timer = self.kernel_timer
        if timer is not None:
            timer.before()
        nat.step3d(self.grid, fields, step_arg, st)
        if timer is not None:
            timer.after()
        dst = (step_arg & 1) ^ 1
        if self.sops.n_ops:
            nat.cell_ops(self.f["Ez"][dst].data_ptr(), self.bz_dtype, self.n_designs, self.n_comp, self.vol, self.nx,
                         self.pitch, self.sops, step_arg, d_step_ptr, st)
        if self.gops is not None and (self.record is not None or self.ring is not None):
            for i, c in enumerate(COMPONENTS):
                self.gops.src[i] = self.f[c][dst].data_ptr()
            nat.gather(self.gops, self.bz_dtype, self.n_designs, self.n_comp, self.vol, step_arg, d_step_ptr, st)
        if self.power is not None:
            nat.power3d(self.grid, fields, dst, self.power.data_ptr(), st)

    def step_once(self):
        self._maybe_drain()
        self._launch(self.step_index, None)
        self.n_step_launches += 1
        self.n_kernel_launches += self.kernels_per_step
        self.step_index += 1
        if self.dft is not None and self.step_index - self._folded >= RING_LEN:
            self._fold()

    def _graph_for(self, phase):
        g = self._graphs.get(phase)
        if g is None:
            def launches():
                for k in range(GRAPH_CHUNK):
                    self._launch(phase + k, self.d_step.data_ptr())

            g = capture(launches)
            self._graphs[phase] = g
        return g

    def run_steps(self, n):
        """Advance n steps (see _run_steps); the E field is scanned for divergence every
        guard.every steps."""
        while n > 0:
            k = min(n, max(1, self.guard.next - self.step_index))
            self._run_steps(k)
            n -= k
            self.guard.maybe_check(self.f["Ez"][self.cur], self.bz_dtype, self.step_index)

    def check_divergence(self):
        """Scan the current E field and raise NativeError(BZ_ERR_DIVERGED) if this run
        diverged at any check so far (synchronizes)."""
        self.guard.check(self.f["Ez"][self.cur], self.bz_dtype, self.step_index)
        self.guard.raise_if_diverged()

    def _run_steps(self, n):
        while n > 0:
            self._maybe_drain()
            room = n
            if self.record is not None:
                room = min(room, self.gops.rec_step0 + self.rec_rows - self.step_index)
            if self.use_graphs and self.kernel_timer is None and room >= GRAPH_CHUNK:
                # fold samples left by single steps before the chunk overwrites their slots
                if self.step_index - self._folded > RING_LEN - GRAPH_CHUNK:
                    self._fold()
                phase = self.step_index & 1
                g = self._graph_for(phase)
                self.d_step.fill_(self.step_index - phase)
                g.replay()
                self.n_step_launches += GRAPH_CHUNK
                self.n_kernel_launches += GRAPH_CHUNK * self.kernels_per_step
                self.step_index += GRAPH_CHUNK
                n -= GRAPH_CHUNK
                self._fold()
                continue
            self.step_once()
            n -= 1

    def _fold(self):
        while self.dft is not None and self._folded < self.step_index:
            cnt = min(RING_LEN, self.step_index - self._folded)
            nat.dft_fold_q(self.ring.data_ptr(), self.bz_dtype, RING_LEN, self.n_designs * self.n_comp * self.n_points,
                           6, 3, len(self.freqs), self.phasor.data_ptr(), self.n_steps, self._folded, cnt,
                           self.dft.data_ptr(), self._stream())
            self.n_fold_launches += 1
            self.n_kernel_launches += 1
            self._folded += cnt

    def reset(self):
        for c in COMPONENTS:
            for b in self.f[c]:
                b.zero_()
        for t in (self.dft, self.power, self.ring):
            if t is not None:
                t.zero_()
        self.step_index = 0
        self._folded = 0
        self.guard.reset()
        if self.record is not None:
            self._rec_host = []
            self.gops.rec_step0 = 0
            self._graphs.clear()

    def _maybe_drain(self, force=False):
        if self.record is None:
            return
        used = self.step_index - self.gops.rec_step0
        if used >= self.rec_rows or (force and used > 0):
            self._rec_host.append(self.record[:used].cpu().numpy())
            self.d2h_bytes += self._rec_host[-1].nbytes
            self.gops.rec_step0 = self.step_index
            self._graphs.clear()

    def take_records(self):
        if self.record is None:
            return None
        self._maybe_drain(force=True)
        if not self._rec_host:
            return np.zeros((0, self.n_designs, self.n_comp, self.n_points, 6))
        out = np.concatenate(self._rec_host).astype(np.float64)
        self._rec_host = []
        return out

    # ---- results ----------------------------------------------------------------
    @property
    def cur(self):
        return self.step_index & 1

    def field(self, name, design=0):
        nz, ny, nx = self.nz, self.ny, self.nx
        shp = {"Ex": (nz, ny, nx - 1), "Ey": (nz, ny - 1, nx), "Ez": (nz - 1, ny, nx), "Hx": (nz - 1, ny - 1, nx),
               "Hy": (nz - 1, ny, nx - 1), "Hz": (nz, ny - 1, nx - 1)}[name]
        buf = self.f[name][self.cur][design][:, :shp[0], :shp[1], :shp[2]]
        if self.n_comp == 2:
            return torch.complex(buf[0].double(), buf[1].double())
        return buf[0]

    def power_map(self, design=0):
        if self.power is None:
            return None
        out = self.power[design].cpu().numpy()
        self.d2h_bytes += out.nbytes
        return out

    def collect_monitors(self, recs, times):
        """Fill plane monitors from the device records (monitors.py:317-396, 426-439)."""
        if recs is not None:
            for m, sl, shp in zip(self.mons, self.mon_slices, self.mon_shape):
                part = recs[:, 0, :, sl, :]  # [steps][comp][points][6]
                vals = part[:, 0] + 1j * part[:, 1] if self.n_comp == 2 else part[:, 0]
                k = m.record_interval
                sel = np.arange(k - 1, len(times), k) if k > 1 else np.arange(len(times))
                for n in sel:
                    comps = [vals[n, :, q].reshape(shp) for q in range(6)]
                    if self.n_comp == 2:
                        comps = [c.astype(np.complex128) for c in comps]
                    m._append_3d(comps, times[n])
                    m.last_record_step = int(n)
                m._manage_memory()
        if self.dft is not None:
            self._fold()
            a = self.dft.cpu().numpy()
            self.d2h_bytes += a.nbytes
            d = (a[..., 0] + 1j * a[..., 1]) * self.dt  # [designs][comp][points][freq][6]
            f0 = 0
            for m, sl, shp in zip(self.mons, self.mon_slices, self.mon_shape):
                if m.frequencies is None:
                    continue
                nf = len(m.frequencies)
                q = d[0, 0, sl, f0:f0 + nf, :]  # [points][freq][6]
                f0 += nf
                comps = {c: q[..., i].T.reshape((nf,) + shp) for i, c in enumerate(COMPONENTS)}
                area = {"z": self.dx * self.dy, "y": self.dx * self.dz, "x": self.dy * self.dz}[m.plane_normal]
                ex, ey, ez, hx, hy, hz = (comps[c] for c in COMPONENTS)
                if m.plane_normal == "z":
                    s = ex * np.conj(hy) - ey * np.conj(hx)
                elif m.plane_normal == "y":
                    s = ez * np.conj(hx) - ex * np.conj(hz)
                else:
                    s = ey * np.conj(hz) - ez * np.conj(hy)
                flux = 0.5 * np.real(s.reshape(nf, -1).sum(axis=1)) * area
                m.dft = dict(frequencies=np.asarray(m.frequencies), flux=flux, **comps)
