"""The FDTD simulation object (beamz/simulation/fdtd.py:16-549), stepping on the GPU.

Same constructor, ``initialize_simulation`` / ``step`` / ``finalize_simulation`` /
``run`` / ``simulate_step`` entries, ``results`` dict and monitor side effects as
the reference. What changes is where the loop runs: fields stay in HBM, one
fused kernel per time step does H + E + sources + monitors (+ power), and
``run`` replays CUDA-graph chunks of steps. Host copies happen only for the
snapshots the caller asked for (``save`` / ``fields_to_cache``) and once at the
end for monitor records, DFT sums and accumulated power.

Not provided: live plotting and animation (``live``/``save_animation`` are
accepted and ignored), ``plot_field``/``plot_power``.
"""
from __future__ import annotations

import datetime
from typing import Dict, Optional, Sequence

import numpy as np

from ..const import EPS_0, MU_0, µm
from ..devices.monitors import Monitor
from ..devices.sources import GaussianSource, ModeSource
from ..helpers import check_fdtd_stability, display_status
from .backends import get_backend
from .meshing import BaseMeshGrid, RegularGrid, RegularGrid3D

__all__ = ["FDTD"]


class FDTD:
    def __init__(self, design, time, mesh: str = "regular", resolution: float = 0.02 * µm, backend="b200",
                 backend_options=None, devices=None):
        provided = None
        if isinstance(design, BaseMeshGrid):
            provided = design
            if getattr(provided, "design", None) is None:
                raise ValueError("Provided mesh must expose its originating design via the `design` attribute.")
            design = provided.design
        self.design = design
        self.is_3d = bool(design.is_3d and design.depth and design.depth > 0)
        if provided is not None:
            mesh_obj = provided
        elif isinstance(mesh, BaseMeshGrid):
            mesh_obj = mesh
        elif mesh == "regular":
            mesh_obj = RegularGrid3D(design, resolution_xy=resolution) if self.is_3d else \
                RegularGrid(design, resolution)
        else:
            raise ValueError(f"Unsupported mesh specification: {mesh!r}")
        if getattr(mesh_obj, "design", None) is not None and mesh_obj.design is not self.design:
            raise ValueError("Provided mesh was generated from a different design instance.")
        if self.is_3d and not isinstance(mesh_obj, RegularGrid3D):
            raise ValueError("3D designs require a RegularGrid3D mesh.")
        if not self.is_3d and not isinstance(mesh_obj, RegularGrid):
            raise ValueError("2D designs require a RegularGrid mesh.")
        self.mesh = mesh_obj
        self.resolution = getattr(mesh_obj, "resolution", None) or getattr(mesh_obj, "resolution_xy", resolution)
        self.dx = mesh_obj.dx
        self.dy = mesh_obj.dy
        if self.is_3d:
            self.dz = mesh_obj.dz
            self.nz, self.ny, self.nx = mesh_obj.permittivity.shape
        else:
            self.ny, self.nx = mesh_obj.permittivity.shape
        self.backend_options = dict(backend_options or {})
        self.backend = get_backend(name=backend, **self.backend_options)
        # material arrays are read when the engine is built (initialize_simulation),
        # so edits to mesh.permittivity before then are honoured
        self.epsilon_r = mesh_obj.permittivity
        self.mu_r = mesh_obj.permeability
        self.sigma = mesh_obj.conductivity
        self.time = time
        self.dt = time[1] - time[0]
        self.num_steps = len(time)
        self.sources = list(design.sources)
        self.monitors = list(design.monitors)
        for dev in devices or []:
            if isinstance(dev, (ModeSource, GaussianSource)):
                if getattr(dev, "design", "n/a") is None:
                    dev.design = design
                self.sources.append(dev)
            elif isinstance(dev, Monitor):
                if dev.design is None:
                    dev.design = design
                self.monitors.append(dev)
            else:
                raise TypeError(f"Unsupported device type: {type(dev)}")
        keys = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz") if self.is_3d else ("Ez", "Hx", "Hy")
        self.results = {k: [] for k in keys}
        self.results["t"] = []
        self.monitor_data = {}
        self.power_accumulated = None
        self.power_accumulation_count = 0
        self.start_time = None
        self.engine = None
        self.t = 0
        self.current_step = 0
        self.fig = None
        self._live = False
        self.accumulate_power = False
        self.save_memory_mode = False

    # ---- engine ---------------------------------------------------------------
    def _build_engine(self, accumulate_power: bool):
        opts = self.backend_options
        precision = opts.get("precision", "fp32")
        n_comp = opts.get("n_comp")
        graphs = opts.get("graph", True)
        if self.is_3d:
            from .engine3d import Engine3D

            self.engine = Engine3D(self.mesh.permittivity, self.mesh.conductivity, self.dx, self.dy, self.dz,
                                   self.dt, self.num_steps, self.sources, self.monitors, precision=precision,
                                   n_comp=n_comp, power=accumulate_power, use_graphs=graphs,
                                   tile_z=opts.get("tile_z", 0), tile_y=opts.get("tile_y", 8),
                                   x_cells=opts.get("x_cells", 0))
        else:
            from .engine2d import Engine2D

            self.engine = Engine2D(self.mesh.permittivity, self.mesh.conductivity, self.dx, self.dy, self.dt,
                                   self.num_steps, self.sources, self.monitors, precision=precision, n_comp=n_comp,
                                   power=accumulate_power, use_graphs=graphs, tile_rows=opts.get("tile_rows", 16),
                                   time_block=opts.get("time_block", "auto"), tb_tile=opts.get("tb_tile", 0))

    def __getattr__(self, name):
        # field access with the reference's names and shapes (device tensors)
        if name in ("Ez", "Hx", "Hy", "Ex", "Ey", "Hz") and self.__dict__.get("engine") is not None:
            return self.__dict__["engine"].field(name)
        raise AttributeError(name)

    # ---- API ------------------------------------------------------------------
    def simulate_step(self):
        """Advance the fields by one step (H, E, sources and monitors run fused)."""
        if self.engine is None:
            self.initialize_simulation(save=False, live=False)
        self.engine.step_once()

    def initialize_simulation(self, save=True, live=True, axis_scale=(-1, 1), save_animation=False,
                              animation_filename="fdtd_animation.mp4", clean_visualization=True, save_fields=None,
                              decimate_save=1, accumulate_power=False, save_memory_mode=False,
                              fields_to_cache: Optional[Sequence[str]] = None):
        if save_fields is None:
            save_fields = ["Ex", "Ey", "Ez", "Hx", "Hy", "Hz"] if self.is_3d else ["Ez", "Hx", "Hy"]
        self._cache_fields = list(fields_to_cache) if fields_to_cache else []
        self._cache_frequency = 1 if self._cache_fields else None
        self.start_time = datetime.datetime.now()
        self.t = 0
        self.current_step = 0
        self._total_steps = self.num_steps
        self._save_results = save
        self._save_fields = save_fields
        self._decimate_save = decimate_save
        self._live = False
        self._axis_scale = axis_scale
        for k in list(self.results.keys()):
            self.results[k] = []
        self.save_memory_mode = save_memory_mode
        self.accumulate_power = accumulate_power
        n_max = np.sqrt(np.max(self.mesh.permittivity))
        ok, courant, limit = check_fdtd_stability(dt=self.dt, dx=self.dx, dy=self.dy, n_max=n_max, safety_factor=1.0)
        if not ok:
            display_status(f"Simulation may be unstable! Courant number = {courant:.3f} > {limit:.3f}", "warning")
        if accumulate_power:
            shape = (self.nz, self.ny, self.nx) if self.is_3d else (self.ny, self.nx)
            self.power_accumulated = np.zeros(shape)
            self.power_accumulation_count = 0
        # the reference's GPU-backend rule (fdtd.py:390-397): batch saves on device backends
        save_freq = max(10, self.num_steps // 100) if save else 1
        self._effective_save_freq = save_freq * decimate_save
        if self._cache_frequency is None:
            self._cache_frequency = self._effective_save_freq
        self._build_engine(accumulate_power)
        self._t_host = 0.0

    def _save_due(self, step: int) -> bool:
        last = step == self.num_steps - 1
        full = self._save_results and not self.save_memory_mode and \
            (step % self._effective_save_freq == 0 or last)
        cache = bool(self._save_results and self._cache_fields and (step % self._cache_frequency == 0 or last))
        return full or cache

    def _save_step_results(self):
        """helper.py:189-229 for the step just completed."""
        step = self.current_step
        last = step == self.num_steps - 1
        full = self._save_results and not self.save_memory_mode and \
            (step % self._effective_save_freq == 0 or last)
        cache = bool(self._save_results and self._cache_fields and (step % self._cache_frequency == 0 or last))
        if not (full or cache):
            return
        self.results.setdefault("t", []).append(self.t)
        names = list(self._save_fields) if full else []
        if cache:
            names += [f for f in self._cache_fields if f not in names]
        for name in names:
            arr = self.engine.field(name).cpu().numpy()
            if name in self._cache_fields:
                arr = arr.astype(np.complex128)
            else:
                arr = np.abs(arr)  # the reference's fields are complex; saved magnitudes
            self.results.setdefault(name, []).append(arr)

    def step(self) -> bool:
        if self.current_step >= self.num_steps:
            return False
        if self.engine is None:
            self.initialize_simulation(save=False, live=False)
        self.engine.step_once()
        self._save_step_results()
        self.t += self.dt
        self.current_step += 1
        return True

    def _next_save(self, step: int) -> int:
        """First step >= ``step`` for which _save_due holds (num_steps if none does)."""
        n = self.num_steps
        full = self._save_results and not self.save_memory_mode
        cache = bool(self._save_results and self._cache_fields)
        if step >= n or not (full or cache):
            return n
        nxt = n - 1  # the last step is always saved
        for on, f in ((full, self._effective_save_freq), (cache, self._cache_frequency)):
            if on:
                f = max(1, int(f))
                nxt = min(nxt, -(-step // f) * f)
        return nxt

    def _run_until_end(self):
        """Steps to the end, in graph chunks between the steps that need host copies."""
        self._run_until(self.num_steps)

    def _run_until(self, stop: int):
        stop = min(int(stop), self.num_steps)
        while self.current_step < stop:
            n_free = min(self._next_save(self.current_step), stop) - self.current_step
            if n_free > 0:
                self.engine.run_steps(n_free)
                # t advances by repeated addition, as one step at a time would
                # (accumulate adds in order, so the rounding is the same)
                self.t = float(np.add.accumulate(np.r_[self.t, np.full(n_free, self.dt)])[-1])
                self.current_step += n_free
            if self.current_step < stop:
                self.step()

    def _collect_monitors(self):
        eng = self.engine
        recs = eng.take_records() if hasattr(eng, "take_records") else None
        steps = np.arange(eng.step_index)
        times = np.zeros(len(steps))
        if len(steps) > 1:
            times[1:] = np.cumsum(np.full(len(steps) - 1, self.dt))
        if hasattr(eng, "collect_monitors"):
            eng.collect_monitors(recs, times)
            return
        if recs is not None:
            self._load_records(eng, recs, times, steps)
        self._collect_dft()

    def _load_records(self, eng, recs, times, steps):
        for mon, sl, ok in zip(eng.mp.monitors, eng.mp.slices, eng.mp.valid):
            part = recs[:, 0, :, sl, :]  # [steps][comp][points][3]
            vals = part[:, 0] + 1j * part[:, 1] if eng.n_comp == 2 else part[:, 0]
            k = mon.record_interval
            sel = np.arange(k - 1, len(steps), k) if k > 1 else np.arange(len(steps))
            sel = sel[sel >= 0]
            vals = vals[sel]
            ez, hx, hy = vals[..., 0], vals[..., 1], vals[..., 2]
            if eng.n_comp == 2:
                ez, hx, hy = ez.astype(np.complex128), hx.astype(np.complex128), hy.astype(np.complex128)
            mon.load_record_2d(ez, hx, hy, times[sel])
            mon.last_record_step = int(sel[-1]) if len(sel) else mon.last_record_step

    def _collect_dft(self):
        eng = self.engine
        d = eng.dft_fields()
        if d is None:
            return
        f0 = 0
        for mon, sl in zip(eng.mp.monitors, eng.mp.slices):
            if mon.frequencies is None:
                continue
            nf = len(mon.frequencies)
            q = d[0, 0, sl, f0:f0 + nf, :]  # [points][freq][5], component 0 = real field
            f0 += nf
            ez = q[..., 0].T
            hx_c = 0.5 * (q[..., 1] + q[..., 2]).T
            hy_c = 0.5 * (q[..., 3] + q[..., 4]).T
            vertical = abs(mon.end[0] - mon.start[0]) < abs(mon.end[1] - mon.start[1])
            if vertical:
                flux = 0.5 * np.real(np.sum(ez * np.conj(hx_c), axis=1)) * self.dy
            else:
                flux = -0.5 * np.real(np.sum(ez * np.conj(hy_c), axis=1)) * self.dx
            mon.dft = {"frequencies": np.asarray(mon.frequencies), "Ez": ez, "Hx": hx_c, "Hy": hy_c, "flux": flux}
            if eng.n_comp == 2:
                mon.dft["Ez_imag_part"] = d[0, 1, sl, f0 - nf:f0, 0].T

    def finalize_simulation(self):
        if self.engine is not None:
            # raises NativeError(BZ_ERR_DIVERGED) if the fields ran away (the reference
            # only warns about the Courant number before the run, fdtd.py:375-383)
            self.engine.check_divergence()
            self._collect_monitors()
            if self.accumulate_power:
                pm = self.engine.power_map()
                if pm is not None:
                    self.power_accumulated = pm
                    self.power_accumulation_count = self.engine.step_index
                if self.power_accumulation_count > 0:
                    self.power_accumulated = self.power_accumulated / self.power_accumulation_count
        objectives: Dict[str, float] = {}
        for idx, mon in enumerate(self.monitors):
            value = mon.evaluate_objective() if hasattr(mon, "evaluate_objective") else None
            if value is None:
                continue
            objectives[getattr(mon, "name", None) or f"monitor_{idx}"] = value
        if objectives:
            self.results["objectives"] = objectives
        else:
            self.results.pop("objectives", None)
        self.last_objectives = objectives
        return self.results

    def run(self, steps: Optional[int] = None, save=True, live=True, axis_scale=(-1, 1), save_animation=False,
            animation_filename="fdtd_animation.mp4", clean_visualization=True, save_fields=None, decimate_save=1,
            accumulate_power=False, save_memory_mode=False, fields_to_cache: Optional[Sequence[str]] = None) -> Dict:
        self.initialize_simulation(save=save, live=live, axis_scale=axis_scale, save_fields=save_fields,
                                   decimate_save=decimate_save, accumulate_power=accumulate_power,
                                   save_memory_mode=save_memory_mode, fields_to_cache=fields_to_cache)
        self._run_until_end()
        return self.finalize_simulation()

    # ---- partial runs and checkpoints (no counterpart in the reference) -------------
    def run_for(self, n_steps: int, **run_kwargs) -> None:
        """Advance n_steps (initialising first, with run()'s keyword arguments, if the
        simulation has not started); finalise with finalize_simulation() or continue."""
        if self.engine is None:
            self.initialize_simulation(**run_kwargs)
        self._run_until(self.current_step + int(n_steps))

    def save_checkpoint(self, path) -> None:
        """Write the run's state after the steps taken so far: fields (both copies),
        monitor DFT sums and records, accumulated power, step index, time and saved
        results (``simulation.checkpoint``). Resuming after a whole number of graph
        chunks continues with the bits of the uninterrupted run."""
        import torch

        from .checkpoint import engine_state

        if self.engine is None:
            raise RuntimeError("nothing to save: the simulation has not started")
        st = engine_state(self.engine)
        st["fdtd"] = {"current_step": self.current_step, "t": self.t, "t_host": getattr(self, "_t_host", 0.0),
                      "results": {k: list(v) for k, v in self.results.items()}}
        torch.save(st, path)

    def resume(self, path, **run_kwargs) -> Dict:
        """Continue a run from a save_checkpoint file: initialise with run()'s keyword
        arguments, restore the state, step to the end and finalise (returns results)."""
        import torch

        from .checkpoint import load_engine_state

        self.initialize_simulation(**run_kwargs)
        st = torch.load(path, weights_only=False)
        load_engine_state(self.engine, st)
        f = st["fdtd"]
        self.current_step, self.t = int(f["current_step"]), f["t"]
        self._t_host = f.get("t_host", 0.0)
        for k, v in f["results"].items():
            self.results[k] = list(v)
        self._run_until_end()
        return self.finalize_simulation()

    def estimate_memory_usage(self, time_steps=None, save_fields=None):
        time_steps = self.num_steps if time_steps is None else time_steps
        itemsize = 4 if self.backend_options.get("precision", "fp32") == "fp32" else 8
        n = self.nx * self.ny * (self.nz if self.is_3d else 1)
        comps = 6 if self.is_3d else 3
        total = n * comps * 2 * itemsize + n * 2 * itemsize
        return {"Full simulation": {"Total memory (MB)": total / 2 ** 20, "Time steps": time_steps}}

    def plot_field(self, *args, **kwargs):
        raise NotImplementedError("plotting is not part of beamz_b200")

    def plot_power(self, *args, **kwargs):
        raise NotImplementedError("plotting is not part of beamz_b200")

    def animate_live(self, *args, **kwargs):
        raise NotImplementedError("plotting is not part of beamz_b200")

    def save_animation(self, *args, **kwargs):
        raise NotImplementedError("plotting is not part of beamz_b200")
