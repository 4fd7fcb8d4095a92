"""Device state and time loop of the 2D Ez-mode solver.

Holds the ping-pong field buffers ([design][component][ny][pitch], x contiguous,
pitch a multiple of 32 elements), the update coefficients, the compiled source
and monitor operations, and drives the step kernels: ``bz_step2d_multi`` advances
``time_block`` steps per launch (temporal blocking), ``bz_step2d`` one step (single
steps, power accumulation, region capture); launches are replayed in CUDA-graph
chunks when no host work is due between steps.
"""
from __future__ import annotations

import warnings

import numpy as np
import torch

from .. import _native as nat
from ..const import EPS_0, MU_0
from .compile_ops import SourceOps, compile_monitors_2d, compile_sources
from .graphs import capture, dft_phasors
from .guard import DivergenceGuard

GRAPH_CHUNK = 64  # at most this many steps per captured graph
RING_LEN = GRAPH_CHUNK  # monitor samples kept between DFT folds
# (steps per launch, register-tile shape) tried by the autotuner
TUNE_CANDIDATES = ((9, 0), (9, 5), (7, 0), (7, 4), (7, 5), (7, 1), (7, 3), (5, 0), (5, 4), (5, 1), (3, 1))
_TUNED: dict = {}  # (device name, nx, ny, designs, components, dtype) -> (time_block, tb_tile)


def _round_up(n: int, m: int) -> int:
    return (n + m - 1) // m * m


class Engine2D:
    def __init__(self, eps_r, sigma, dx, dy, dt, n_steps, sources, monitors, *, precision="fp32", n_comp=None,
                 power=False, n_designs=1, record=True, use_graphs=True, device=None, tile_rows=16, time_block=7,
                 tb_tile=0):
        if not torch.cuda.is_available():
            raise RuntimeError("beamz_b200 needs a CUDA GPU (sm_100a); none is visible")
        self.dev = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
        eps_r = np.asarray(eps_r, dtype=np.float64)
        sigma = np.asarray(sigma, dtype=np.float64)
        if eps_r.ndim == 2:
            eps_r = eps_r[None]
        self.n_mat, self.ny, self.nx = eps_r.shape
        if self.nx < 2 or self.ny < 2:
            raise ValueError("2D grid must be at least 2 x 2 cells")
        self.n_designs = n_designs
        if self.n_mat not in (1, n_designs):
            raise ValueError("material batch must be 1 or n_designs")
        self.dx, self.dy, self.dt = float(dx), float(dy), float(dt)
        self.n_steps = int(n_steps)
        self.h2d_bytes = 0  # host->device traffic of set-up (material, op tables, phasors)
        self.d2h_bytes = 0  # device->host traffic of results (records, DFT, power, snapshots)
        self.dtype = {"fp32": torch.float32, "fp64": torch.float64}[precision]
        self.bz_dtype = nat.BZ_F32 if precision == "fp32" else nat.BZ_F64
        self.src = compile_sources(sources, (self.ny, self.nx), (self.dx, self.dy), self.n_steps)
        if n_comp is None:
            n_comp = 2 if self.src.complex_weights else 1
        self.n_comp = n_comp
        self.pitch = _round_up(self.nx, 32)
        shape = (n_designs, n_comp, self.ny, self.pitch)
        z = lambda: torch.zeros(shape, dtype=self.dtype, device=self.dev)  # noqa: E731
        self.ez, self.hx, self.hy = [z(), z()], [z(), z()], [z(), z()]
        self.ce = torch.empty((self.n_mat, self.ny, self.pitch), dtype=self.dtype, device=self.dev)
        self.loss = torch.empty_like(self.ce)
        self.set_material(eps_r, sigma)
        self.power = torch.zeros((n_designs, self.ny, self.pitch), dtype=torch.float64, device=self.dev) \
            if power else None
        self.step_index = 0
        self._setup_sources()
        self._setup_monitors(monitors, record)
        self.d_step = torch.zeros(1, dtype=torch.int64, device=self.dev)
        self.use_graphs = use_graphs
        self._graphs: dict[int, torch.cuda.CUDAGraph] = {}
        self.kernel_timer = None  # graphs.KernelTimer around the step launches (direct launches only)
        self._autotune = time_block == "auto"
        if self._autotune:
            time_block = 7
        if int(time_block) not in (1, 3, 5, 7, 9):
            raise ValueError(f"time_block must be 1, 3, 5, 7, 9 or 'auto' (got {time_block})")
        # power accumulation runs on the single-step kernel
        self.time_block = 1 if power else int(time_block)
        self._autotune = self._autotune and not power
        self.tb_tile = int(tb_tile)
        # steps per graph: an even number of steps keeps the copy parity, so one
        # graph serves every chunk of a run
        self.chunk = GRAPH_CHUNK // (2 * self.time_block) * (2 * self.time_block)
        self.guard = DivergenceGuard(self.dev, every=8 * self.chunk)  # checks fall on chunk boundaries
        self.n_step_launches = 0  # step-kernel launches issued (graph nodes included)
        self.n_fold_launches = 0
        g = nat.Grid2D()
        g.nx, g.ny, g.pitch = self.nx, self.ny, self.pitch
        g.n_designs, g.n_comp, g.n_mat, g.dtype = n_designs, n_comp, self.n_mat, self.bz_dtype
        g.tile_rows = int(tile_rows)
        # x-differences use dy and y-differences dx, as the reference pairs them
        g.chx = self.dt / (MU_0 * self.dy)
        g.chy = self.dt / (MU_0 * self.dx)
        g.qy = self.dy / self.dx
        g.inv_kd2 = 2.0 * EPS_0 * self.dy / self.dt
        self.grid = g

    # ---- set-up ---------------------------------------------------------------
    def set_material(self, eps_r, sigma):
        """Uploads new material ([n_mat][ny][nx] or (ny, nx), sigma may be shared) and
        recomputes the update coefficients."""
        shape = (self.n_mat, self.ny, self.nx)
        eps_r = np.ascontiguousarray(np.broadcast_to(np.asarray(eps_r, dtype=np.float64), shape))
        sigma = np.ascontiguousarray(np.broadcast_to(np.asarray(sigma, dtype=np.float64), shape))
        self.h2d_bytes += eps_r.nbytes + sigma.nbytes
        with warnings.catch_warnings():  # a read-only broadcast view is only read by the copy
            warnings.filterwarnings("ignore", message="The given NumPy array is not writable")
            te, ts = torch.as_tensor(eps_r).to(self.dev), torch.as_tensor(sigma).to(self.dev)
        self.set_material_tensors(te, ts)

    def set_material_tensors(self, eps_r: torch.Tensor, sigma: torch.Tensor):
        """As set_material, from float64 device tensors of shape [n_mat][ny][nx]."""
        shape = (self.n_mat, self.ny, self.nx)
        if tuple(eps_r.shape) != shape or tuple(sigma.shape) != shape:
            raise ValueError(f"material tensors must have shape {shape}")
        te = eps_r.to(self.dev, torch.float64).contiguous()
        ts = sigma.to(self.dev, torch.float64).contiguous()
        nat.prepare_coeffs(te.data_ptr(), ts.data_ptr(), self.n_mat * self.ny, self.nx, self.pitch, self.bz_dtype,
                           self.dt, EPS_0, self.dy, self.ce.data_ptr(), self.loss.data_ptr(), self._stream())
        torch.cuda.current_stream().synchronize()

    def _setup_sources(self):
        s: SourceOps = self.src
        self.sops = nat.SourceOps()
        self._keep = []
        if len(s.cell) == 0:
            self.sops.n_ops = 0
            return
        # n_comp = 1 with complex amplitudes carries Re(field), the physical field:
        # the update is real-linear, so the real part evolves on its own.
        t = lambda a, dt: self._kept(torch.as_tensor(np.ascontiguousarray(a)).to(self.dev, dt))  # noqa: E731
        self._src_t = dict(row=t(s.row_ptr, torch.int32), cell=t(s.cell, torch.int32),
                           mul=t(s.mul, self.dtype), w=t(s.weight[:, :self.n_comp], self.dtype),
                           sig=t(s.sig, torch.int32), signals=t(s.signals, self.dtype))
        so = self.sops
        so.n_ops, so.n_steps = len(s.cell), s.signals.shape[1]
        so.row_ptr, so.cell = self._src_t["row"].data_ptr(), self._src_t["cell"].data_ptr()
        so.mul, so.weight = self._src_t["mul"].data_ptr(), self._src_t["w"].data_ptr()
        so.sig, so.signals = self._src_t["sig"].data_ptr(), self._src_t["signals"].data_ptr()

    def _kept(self, t):
        self._keep.append(t)
        self.h2d_bytes += t.numel() * t.element_size()
        return t

    def _setup_monitors(self, monitors, record):
        self.mp = compile_monitors_2d(monitors, self.nx, self.ny, self.dx, self.dy)
        self.mops = nat.MonitorOps()
        self.mops.n_points = 0
        self.freqs = np.zeros(0)
        self.record = None
        self.dft = None
        self.ring = None
        self._folded = 0
        if self.mp.n_points == 0 or len(self.mp.cell) == 0:
            return
        mp = self.mp
        self._mon_t = dict(row=self._kept(torch.as_tensor(mp.row_ptr).to(self.dev)),
                           cell=self._kept(torch.as_tensor(mp.cell).to(self.dev)),
                           point=self._kept(torch.as_tensor(mp.point).to(self.dev)))
        mo = self.mops
        mo.n_points = mp.n_points
        mo.row_ptr, mo.cell, mo.point = (self._mon_t[k].data_ptr() for k in ("row", "cell", "point"))
        want_rec = record and any(m.should_record_fields or m.accumulate_power for m in mp.monitors)
        if want_rec:
            row_bytes = self.n_designs * self.n_comp * mp.n_points * 3 * torch.finfo(self.dtype).bits // 8
            self.rec_rows = max(1, min(self.n_steps, (256 << 20) // max(1, row_bytes)))
            self.record = torch.zeros((self.rec_rows, self.n_designs, self.n_comp, mp.n_points, 3), dtype=self.dtype,
                                      device=self.dev)
            mo.record, mo.n_rec = self.record.data_ptr(), self.rec_rows
            mo.rec_step0 = 0
        freqs = [np.asarray(m.frequencies, dtype=float) for m in mp.monitors if m.frequencies is not None]
        if freqs:
            self.freqs = np.concatenate(freqs)
            nf = len(self.freqs)
            self.phasor = dft_phasors(self.freqs, self.n_steps, self.dt, self.dev)
            self.h2d_bytes += self.freqs.nbytes
            self.ring = torch.zeros((RING_LEN, self.n_designs, self.n_comp, mp.n_points, 5), dtype=self.dtype,
                                    device=self.dev)
            self.dft = torch.zeros((self.n_designs, self.n_comp, mp.n_points, nf, 5, 2), dtype=torch.float64,
                                   device=self.dev)
            mo.ring, mo.ring_len = self.ring.data_ptr(), RING_LEN
        self._rec_host: list[np.ndarray] = []
        self._rec_first = 0

    # ---- stepping -------------------------------------------------------------
    @staticmethod
    def _stream() -> int:
        return torch.cuda.current_stream().cuda_stream

    def _fields(self) -> nat.Fields2D:
        # The copy holding the current fields is always (step_index & 1): every
        # step flips it, and a launch with host step argument n reads copy n & 1.
        f = nat.Fields2D()
        f.ez[0], f.ez[1] = self.ez[0].data_ptr(), self.ez[1].data_ptr()
        f.hx[0], f.hx[1] = self.hx[0].data_ptr(), self.hx[1].data_ptr()
        f.hy[0], f.hy[1] = self.hy[0].data_ptr(), self.hy[1].data_ptr()
        f.ce, f.loss = self.ce.data_ptr(), self.loss.data_ptr()
        f.power = self.power.data_ptr() if self.power is not None else None
        return f

    @property
    def cur(self) -> int:
        return self.step_index & 1

    def _launch(self, step_arg: int, d_step_ptr):
        timer = self.kernel_timer
        if timer is not None:
            timer.before()
        nat.step2d(self.grid, self._fields(), self.sops if self.sops.n_ops else None,
                   self.mops if self.mops.n_points else None, step_arg, d_step_ptr, self._stream())
        if timer is not None:
            timer.after()

    def _launch_tb(self, step_arg: int, d_step_ptr):
        timer = self.kernel_timer
        if timer is not None:
            timer.before(self.time_block)
        nat.step2d_multi(self.grid, self._fields(), self.sops if self.sops.n_ops else None,
                         self.mops if self.mops.n_points else None, step_arg, self.time_block, self.tb_tile,
                         d_step_ptr, self._stream())
        if timer is not None:
            timer.after()

    def _block(self) -> int:
        """Steps per launch available now."""
        return self.time_block

    def advance_direct(self, n: int):
        """Advance n steps with direct launches (blocked where possible, no graphs): for
        runs whose launch parameters change between calls, such as the adjoint's
        segment recompute with region capture."""
        while n > 0:
            tb = self.time_block if n >= self.time_block else 1
            (self._launch_tb if tb > 1 else self._launch)(self.step_index, None)
            self.n_step_launches += 1
            self.step_index += tb
            n -= tb

    def step_once(self):
        """Advance one time step with a direct launch."""
        self._maybe_drain()
        self._launch(self.step_index, None)
        self.n_step_launches += 1
        self.step_index += 1
        if self.dft is not None and self.step_index - self._folded >= RING_LEN:
            self._fold()

    def _fold(self):
        """Fold the monitor samples of steps [folded, step_index) into the DFT sums."""
        while self.dft is not None and self._folded < self.step_index:
            cnt = min(RING_LEN, self.step_index - self._folded)
            nat.dft_fold(self.ring.data_ptr(), self.bz_dtype, RING_LEN, self.n_designs * self.n_comp * self.mp.n_points,
                         len(self.freqs), self.phasor.data_ptr(), self.n_steps, self._folded, cnt,
                         self.dft.data_ptr(), self._stream())
            self.n_fold_launches += 1
            self._folded += cnt

    def reset(self):
        """Zero the fields and accumulators and rewind to step 0 (material and
        compiled operations are kept)."""
        for bufs in (self.ez, self.hx, self.hy):
            for b in bufs:
                b.zero_()
        for t in (self.dft, self.power, self.ring):
            if t is not None:
                t.zero_()
        self.step_index = 0
        self._folded = 0
        self.guard.reset()
        if self.record is not None:
            self._rec_host = []
            self.mops.rec_step0 = 0
            self._graphs.clear()

    def _graph_for(self, phase: int) -> torch.cuda.CUDAGraph:
        """Graph of the launches of `chunk` steps starting at a step of parity `phase`;
        the time index comes from the device counter (d_step = first step - phase)."""
        g = self._graphs.get(phase)
        if g is None:
            tb = self.time_block

            def launches():
                for k in range(0, self.chunk, tb):
                    (self._launch_tb if tb > 1 else self._launch)(phase + k, self.d_step.data_ptr())

            g = capture(launches)
            self._graphs[phase] = g
        return g

    def autotune(self, candidates=TUNE_CANDIDATES, launches: int = 12, rounds: int = 2):
        """Pick (time_block, tb_tile) by timing blocked launches on this grid (CUDA events).

        Every candidate gives the same results (same arithmetic per cell), and a launch
        only writes the copy that the next step overwrites and ring/record slots of steps
        not yet taken, so timing from the current state changes nothing. Each candidate
        is launched once to warm up, then timed over ``launches`` launches in ``rounds``
        interleaved rounds (best time kept). The choice is cached per (device, grid,
        designs, components, dtype) for the process."""
        key = (torch.cuda.get_device_name(self.dev), self.nx, self.ny, self.n_designs, self.n_comp, self.bz_dtype)
        if key not in _TUNED:
            times = {c: float("inf") for c in candidates}
            for tb, tile in candidates:
                self.time_block, self.tb_tile = tb, tile
                self._launch_tb(self.step_index, None)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            for _ in range(rounds):
                for tb, tile in candidates:
                    self.time_block, self.tb_tile = tb, tile
                    a.record()
                    for _ in range(launches):
                        self._launch_tb(self.step_index, None)
                    b.record()
                    b.synchronize()
                    times[(tb, tile)] = min(times[(tb, tile)], a.elapsed_time(b) / (launches * tb))
            _TUNED[key] = min(times, key=times.get)
            self.tune_times = times
        self.time_block, self.tb_tile = _TUNED[key]
        self.chunk = GRAPH_CHUNK // (2 * self.time_block) * (2 * self.time_block)
        self.guard.every = 8 * self.chunk  # checks fall on chunk boundaries
        self.guard.next = (self.step_index // self.guard.every + 1) * self.guard.every
        self._graphs.clear()
        self._autotune = False
        return _TUNED[key]

    def run_steps(self, n: int):
        """Advance n steps (see _run_steps); the E field is scanned for divergence every
        guard.every steps."""
        while n > 0:
            k = min(n, max(1, self.guard.next - self.step_index))
            self._run_steps(k)
            n -= k
            self.guard.maybe_check(self.ez[self.cur], self.bz_dtype, self.step_index)

    def check_divergence(self):
        """Scan the current E field and raise NativeError(BZ_ERR_DIVERGED) if this run
        diverged at any check so far (synchronizes)."""
        self.guard.check(self.ez[self.cur], self.bz_dtype, self.step_index)
        self.guard.raise_if_diverged()

    def _run_steps(self, n: int):
        """Advance n steps, replaying graph chunks where the record buffer allows."""
        if self._autotune:
            self.autotune()
        while n > 0:
            self._maybe_drain()
            room = n
            if self.record is not None:
                room = min(room, self.mops.rec_step0 + self.rec_rows - self.step_index)
            tb = self._block()
            if self.use_graphs and self.kernel_timer is None and not self.mops.region and room >= self.chunk:
                # the chunk writes `chunk` ring slots: fold what earlier launches left
                # there first, or those samples are overwritten before they are read
                if self.step_index - self._folded > RING_LEN - self.chunk:
                    self._fold()
                phase = self.step_index & 1
                g = self._graph_for(phase)
                self.d_step.fill_(self.step_index - phase)
                g.replay()
                self.n_step_launches += self.chunk // self.time_block
                self.step_index += self.chunk
                n -= self.chunk
                self._fold()
                continue
            if tb > 1 and room >= tb:
                if self.step_index - self._folded > RING_LEN - tb:
                    self._fold()
                self._launch_tb(self.step_index, None)
                self.n_step_launches += 1
                self.step_index += tb
                n -= tb
                continue
            self.step_once()
            n -= 1

    # ---- records --------------------------------------------------------------
    def _maybe_drain(self, force=False):
        if self.record is None:
            return
        used = self.step_index - self.mops.rec_step0
        if used >= self.rec_rows or (force and used > 0):
            self._rec_host.append(self.record[:used].cpu().numpy())
            self.d2h_bytes += self._rec_host[-1].nbytes
            self.mops.rec_step0 = self.step_index
            self._graphs.clear()  # graphs bake rec_step0

    def take_records(self) -> np.ndarray | None:
        """All samples recorded so far: [steps][designs][comp][points][3] (float64)."""
        if self.record is None:
            return None
        self._maybe_drain(force=True)
        if not self._rec_host:
            return np.zeros((0, self.n_designs, self.n_comp, self.mp.n_points, 3))
        out = np.concatenate(self._rec_host).astype(np.float64)
        self._rec_host = []
        return out

    # ---- field access ---------------------------------------------------------
    def field(self, name: str, design: int = 0) -> torch.Tensor:
        """Current field with the reference's shape: Ez (ny, nx), Hx (ny, nx-1), Hy (ny-1, nx);
        complex when the run carries two components."""
        buf = {"Ez": self.ez, "Hx": self.hx, "Hy": self.hy}[name][self.cur][design]
        ny, nx = self.ny, self.nx
        sl = {"Ez": (slice(0, ny), slice(0, nx)), "Hx": (slice(0, ny), slice(0, nx - 1)),
              "Hy": (slice(0, ny - 1), slice(0, nx))}[name]
        if self.n_comp == 2:
            return torch.complex(buf[0][sl].double(), buf[1][sl].double())
        return buf[0][sl]

    def power_map(self, design: int = 0) -> np.ndarray | None:
        if self.power is None:
            return None
        out = self.power[design, :, :self.nx].cpu().numpy()
        self.d2h_bytes += out.nbytes
        return out

    def dft_fields(self) -> np.ndarray | None:
        """DFT sums times dt, complex [designs][comp][points][freq][5]."""
        if self.dft is None:
            return None
        self._fold()
        a = self.dft.cpu().numpy()
        self.d2h_bytes += a.nbytes
        return (a[..., 0] + 1j * a[..., 1]) * self.dt
