"""Batched adjoint FDTD for 2D topology optimisation.

The reference's topology loop (examples/4_topo.py:310-420) estimates the gradient
by overlapping a forward field history with a separately driven adjoint run
(``grad += Re(Ez_adj * conj(Ez_fwd))``), and its library adjoint
(beamz/optimization/topology.py:191-207) returns zeros. Here the gradient is the
exact reverse-mode derivative of the discrete update (``bz_adjoint_step2d``), so it
agrees with finite differences of the same simulation.

Objective: the power in a target mode, measured on a line monitor at one or more
frequencies, ``J = sum_f c_f |a_f|^2`` with ``a_f = sum_p w_fp E_f(p)``,
``E_f(p) = sum_n E_{n+1}(p) exp(-i w_f (n+1) dt) dt`` (the DFT convention of the
frequency-domain monitors) and ``w_fp = conj(m_f(p)) ds`` for the mode profile m_f of
each frequency on the monitor cells (c_f = 1 by default).

Memory/compute trade: the backward pass needs the forward Ez of the design region at
every step. Where it fits (by default when it takes at most half the free device
memory), the forward run writes it to one device buffer ((n_steps + 1) x region cells
per design) and the backward pass runs only reverse steps. Otherwise the forward states
are checkpointed every K steps and each K-step segment is recomputed once during the
backward sweep with the region captured per step (K x region cells per design), so the
backward pass costs one extra forward pass.
"""
from __future__ import annotations

import math

import numpy as np
import torch

from .. import _native as nat
from ..devices.monitors import Monitor
from ..simulation.compile_ops import SourceOps, compile_sources
from ..simulation.engine2d import Engine2D


class AdjointFDTD2D:
    """B designs that differ only inside one rectangular design region.

    Parameters
    ----------
    eps_base, sigma : (ny, nx) float64 arrays; eps_base outside the design region is
        used for every design, sigma must be 0 inside the region.
    dx, dt, n_steps : grid spacing, time step and number of steps (dy = dx).
    sources : beamz_b200 sources (GaussianSource / ModeSource) driving the forward run.
    monitor : a 2D line Monitor; its cells carry the objective.
    mode_profile : complex values m_p on the monitor's cells (length = its point count),
        or one row per frequency.
    frequency : objective frequency in Hz, or a sequence of them.
    weights : optional c_f per frequency.
    region : (y0, x0, h, w) cell box of the design region.
    store_history : where the backward pass gets the forward Ez of the design region.
        True keeps it for every step on the device during the forward run ((n_steps + 1)
        x n_designs x h x w values, 29.5 GB for 64 designs of 120 x 120 over 8000 float32
        steps): the backward pass then runs no forward steps. False keeps the fields every
        ``checkpoint_every`` steps and recomputes each segment in the backward pass.
        "auto" keeps the history when it takes at most half the free device memory.
    """

    def __init__(self, eps_base, sigma, dx, dt, n_steps, sources, monitor, mode_profile, frequency, region, *,
                 n_designs=1, precision="fp32", checkpoint_every=500, weights=None, store_history="auto"):
        self.eps_base = np.asarray(eps_base, dtype=np.float64)
        self.sigma = np.asarray(sigma, dtype=np.float64)
        self.ny, self.nx = self.eps_base.shape
        self.dx, self.dt, self.n_steps = float(dx), float(dt), int(n_steps)
        self.sources = list(sources)
        self.region = tuple(int(v) for v in region)
        y0, x0, h, w = self.region
        if np.any(self.sigma[y0:y0 + h, x0:x0 + w] != 0):
            raise ValueError("the design region must be free of conductivity")
        self.B = int(n_designs)
        self.precision = precision
        self.K = int(checkpoint_every)
        self.freqs = np.atleast_1d(np.asarray(frequency, dtype=float))
        self.frequency = float(self.freqs[0])
        nf = len(self.freqs)
        self.c_f = np.ones(nf) if weights is None else np.asarray(weights, dtype=float).reshape(nf)
        mon = Monitor(start=monitor.start, end=monitor.end, frequencies=list(self.freqs), record_fields=False,
                      accumulate_power=False)
        self.monitor = mon
        mode = np.asarray(mode_profile, dtype=complex)
        self.mode = np.broadcast_to(mode if mode.ndim == 2 else mode[None], (nf, mode.shape[-1])).copy()
        pts = mon.get_grid_points_2d(dx, dx)
        if len(pts) != self.mode.shape[1]:
            raise ValueError(f"mode profile has {self.mode.shape[1]} values, the monitor {len(pts)} cells")
        self.ds = dx
        self.wp = np.conj(self.mode) * self.ds  # [F][P]
        self.mon_cells = [(int(y), int(x)) for x, y in pts]
        src_ops = compile_sources(self.sources, (self.ny, self.nx), (dx, dx), self.n_steps)
        for c in src_ops.cell:
            yy, xx = divmod(int(c), self.nx)
            if y0 <= yy < y0 + h and x0 <= xx < x0 + w:
                raise ValueError("sources may not act inside the design region")
        self._fwd_ops = src_ops
        self.engine = None
        self._adj_block = None  # reverse steps per launch, timed on the first backward
        if store_history not in (True, False, "auto"):
            raise ValueError(f"store_history must be True, False or 'auto' (got {store_history!r})")
        self.store_history = store_history
        self._hist = None  # [n_steps + 1][B][h][w] region Ez of the last forward run
        self._hist_ready = False

    # ---- helpers -------------------------------------------------------------
    def _eps_full(self, eps_region):
        eps_region = np.asarray(eps_region, dtype=np.float64).reshape(self.B, self.region[2], self.region[3])
        y0, x0, h, w = self.region
        full = np.repeat(self.eps_base[None], self.B, axis=0)
        full[:, y0:y0 + h, x0:x0 + w] = eps_region
        return full, eps_region

    def _build(self, eps_region):
        if self.engine is None:
            full, er = self._eps_full(eps_region)
            self.engine = Engine2D(full, self.sigma, self.dx, self.dx, self.dt, self.n_steps, self.sources,
                                   [self.monitor], precision=self.precision, n_comp=1, n_designs=self.B,
                                   record=False, use_graphs=True, time_block="auto")
            dev = self.engine.dev
            self._eps_t = torch.as_tensor(self.eps_base).to(dev)
            self._sigma_t = torch.as_tensor(self.sigma).to(dev).expand(self.B, self.ny, self.nx).contiguous()
        else:
            # only the design region crosses to the device
            er = np.asarray(eps_region, dtype=np.float64).reshape(self.B, self.region[2], self.region[3])
            y0, x0, h, w = self.region
            full_t = self._eps_t.expand(self.B, self.ny, self.nx).clone()
            full_t[:, y0:y0 + h, x0:x0 + w] = torch.as_tensor(er).to(full_t.device)
            self.engine.h2d_bytes += er.nbytes
            self.engine.set_material_tensors(full_t, self._sigma_t)
        self.eps_region = er

    # ---- forward ---------------------------------------------------------------
    def forward(self, eps_region, keep_checkpoints=True):
        """Runs the B forward simulations; returns J (B,) and keeps checkpoints."""
        self._build(eps_region)
        eng = self.engine
        eng.reset()
        self.ckpt = []
        self._hist_ready = False
        if keep_checkpoints and self._use_history():
            self._run_with_history()
        else:
            for s in range(math.ceil(self.n_steps / self.K)):
                if keep_checkpoints:
                    cur = eng.cur
                    self.ckpt.append(tuple(b[cur].clone() for b in (eng.ez, eng.hx, eng.hy)))
                eng.run_steps(min(self.K, self.n_steps - s * self.K))
        d = eng.dft_fields()  # [B][1][P][F][5]
        ew = d[:, 0, :, :, 0]  # E_f at the monitor cells, [B][P][F]
        self.a = np.einsum("bpf,fp->bf", ew, self.wp)
        self.power = np.abs(self.a) ** 2  # [B][F]
        return self.power @ self.c_f

    def _use_history(self) -> bool:
        if self.store_history != "auto":
            return bool(self.store_history)
        if self._hist is not None:
            return True
        _, _, h, w = self.region
        need = (self.n_steps + 1) * self.B * h * w * torch.empty((), dtype=self.engine.dtype).element_size()
        free, _ = torch.cuda.mem_get_info(self.engine.dev)
        return need <= free // 2

    def _run_with_history(self):
        """The forward run with the design region's Ez captured after every step
        (slot k = Ez at step k; slot 0 from the initial fields)."""
        eng = self.engine
        y0, x0, h, w = self.region
        if self._hist is None:
            self._hist = torch.empty((self.n_steps + 1, self.B, h, w), dtype=eng.dtype, device=eng.dev)
        self._hist[0].copy_(eng.ez[eng.cur][:, 0, y0:y0 + h, x0:x0 + w])
        mo = eng.mops
        saved = (mo.region, mo.rx0, mo.ry0, mo.rw, mo.rh, mo.reg_step0, mo.n_reg)
        mo.region, mo.rx0, mo.ry0, mo.rw, mo.rh = self._hist.data_ptr(), x0, y0, w, h
        mo.reg_step0, mo.n_reg = 0, self.n_steps + 1
        try:
            eng.run_steps(self.n_steps)  # direct launches while a region is set
        finally:
            mo.region, mo.rx0, mo.ry0, mo.rw, mo.rh, mo.reg_step0, mo.n_reg = saved
        self._hist_ready = True

    # ---- backward -----------------------------------------------------------------
    def _adjoint_ops(self):
        """Operations preparing dJ/dEt from dJ/dE: the forward sources' zeroing mask and
        the objective terms sum_f Re(alpha_fp phi_f(n)), phi_f(n) = exp(-i w_f (n+1) dt) dt."""
        fo = self._fwd_ops
        M = {}
        for c, m in zip(fo.cell, fo.mul):
            M[int(c)] = M.get(int(c), 1.0) * m  # composite multiplier of each cell
        nf = len(self.freqs)
        alpha = 2.0 * (self.c_f[None, :] * np.conj(self.a))[:, :, None] * self.wp[None]  # [B][F][P]
        per_cell = {}
        for p, (y, x) in enumerate(self.mon_cells):
            if 0 <= x < self.nx and 0 <= y < self.ny:
                c = y * self.nx + x
                per_cell[c] = per_cell.get(c, 0) + alpha[:, :, p]
        cells = sorted(set(per_cell) | {c for c, m in M.items() if m != 1.0})
        n = np.arange(self.n_steps, dtype=np.float64)
        phi = np.exp(-1j * 2 * np.pi * self.freqs[:, None] * (n[None, :] + 1.0) * self.dt) * self.dt  # [F][n]
        signals = np.stack([phi.real, phi.imag], axis=1).reshape(2 * nf, self.n_steps)
        op_cell, op_mul, op_sig, w_cols = [], [], [], []
        for c in cells:
            m = M.get(c, 1.0)
            a = per_cell.get(c, np.zeros((self.B, nf), dtype=complex))
            for f in range(nf):  # v <- m*v + m*Re(alpha_0 phi_0), then + m*Re(alpha_f phi_f)
                op_cell += [c, c]
                op_mul += [m if f == 0 else 1.0, 1.0]
                op_sig += [2 * f, 2 * f + 1]
                w_cols += [m * a[:, f].real, -m * a[:, f].imag]
        weight = np.stack(w_cols, axis=1) if w_cols else np.zeros((self.B, 0))  # [B][n_ops]
        # The seed is ~|a| dx dt (tiny in SI units); the adjoint is linear, so each
        # design's seed is scaled to O(1) (keeps float32 adjoint fields in range) and
        # its gradient is divided by the same factor.
        peak = np.abs(weight).max(axis=1) * np.abs(signals).max() if w_cols else np.ones(self.B)
        self._adj_scale = np.where(peak > 0, 1.0 / np.where(peak > 0, peak, 1.0), 1.0)
        weight = weight * self._adj_scale[:, None]
        cell = np.asarray(op_cell, dtype=np.int64)
        row_ptr = np.searchsorted(cell // self.nx, np.arange(self.ny + 1), side="left").astype(np.int32)
        return cell.astype(np.int32), np.asarray(op_mul), np.asarray(op_sig, dtype=np.int32), weight, signals, row_ptr

    def backward(self):
        """dJ/d eps_r inside the design region, (B, h, w) float64."""
        eng = self.engine
        dev, dt_ = eng.dev, eng.dtype
        y0, x0, h, w = self.region
        cell, mul, sig, weight, signals, row_ptr = self._adjoint_ops()
        keep = []

        def t(a, dtype):
            x = torch.as_tensor(np.ascontiguousarray(a)).to(dev, dtype)
            keep.append(x)
            return x

        ops = nat.SourceOps()
        ops.n_ops, ops.n_steps = len(cell), self.n_steps
        ops.row_ptr, ops.cell = t(row_ptr, torch.int32).data_ptr(), t(cell, torch.int32).data_ptr()
        ops.mul, ops.weight = t(mul, dt_).data_ptr(), t(weight, dt_).data_ptr()
        ops.sig, ops.signals = t(sig, torch.int32).data_ptr(), t(signals, dt_).data_ptr()
        ops.weight_stride = len(cell)
        shape = (self.B, self.ny, eng.pitch)
        st = torch.cuda.current_stream().cuda_stream
        E = [torch.zeros(shape, dtype=dt_, device=dev) for _ in range(2)]
        HX = [torch.zeros_like(E[0]) for _ in range(2)]
        HY = [torch.zeros_like(E[0]) for _ in range(2)]
        grad = torch.zeros((self.B, h, w), dtype=torch.float64, device=dev)
        eps_reg = t(self.eps_region, torch.float64)
        hist = self._hist_ready
        if not hist and not self.ckpt:
            raise RuntimeError("backward() needs a forward() run with keep_checkpoints=True")
        cap = None if hist else torch.zeros((self.K + 1, self.B, h, w), dtype=dt_, device=dev)
        # dJ/dE_N through the last step's sources
        nat.cell_ops(E[0].data_ptr(), eng.bz_dtype, self.B, 1, self.ny * eng.pitch, self.nx, eng.pitch, ops,
                     self.n_steps - 1, None, st)
        st_ = nat.Adjoint2D()
        st_.ce, st_.loss = eng.ce.data_ptr(), eng.loss.data_ptr()
        st_.grad, st_.eps_region = grad.data_ptr(), eps_reg.data_ptr()
        st_.fwd_region = (self._hist if hist else cap).data_ptr()
        st_.rx0, st_.ry0, st_.rw, st_.rh = x0, y0, w, h
        for i in range(2):
            st_.e[i], st_.hx[i], st_.hy[i] = E[i].data_ptr(), HX[i].data_ptr(), HY[i].data_ptr()
        phase = 0
        grid = eng.grid
        if self._adj_block is None:
            self._adj_block = self._time_adjoint(grid, st_, st)
        if hist:  # the whole forward history is on the device: reverse steps only
            st_.fwd_step0, st_.n_fwd = 0, self.n_steps + 1
            n, tb = self.n_steps - 1, self._adj_block
            while n >= 0:
                k = tb if n + 1 >= tb else 1
                nat.adjoint_step2d_multi(grid, st_, ops, n, k, phase, st)
                phase ^= 1
                n -= k
            torch.cuda.current_stream().synchronize()
            return grad.cpu().numpy() / self._adj_scale[:, None, None]
        mo = eng.mops
        saved = (mo.ring, mo.region, mo.n_reg)
        for s in range(len(self.ckpt) - 1, -1, -1):
            s0, s1 = s * self.K, min((s + 1) * self.K, self.n_steps)
            # restore the checkpoint and recompute the segment with the region captured
            eng.step_index = s0
            for buf, ck in zip((eng.ez, eng.hx, eng.hy), self.ckpt[s]):
                buf[s0 & 1].copy_(ck)
            cap[0].copy_(self.ckpt[s][0][:, 0, y0:y0 + h, x0:x0 + w])
            mo.ring, mo.region, mo.n_reg = None, cap.data_ptr(), s1 - s0 + 1
            mo.rx0, mo.ry0, mo.rw, mo.rh, mo.reg_step0 = x0, y0, w, h, s0
            eng.advance_direct(s1 - s0)
            st_.fwd_step0, st_.n_fwd = s0, s1 - s0 + 1
            n, tb = s1 - 1, self._adj_block
            while n >= s0:  # blocks of tb reverse steps, single steps for the rest
                k = tb if n - s0 + 1 >= tb else 1
                nat.adjoint_step2d_multi(grid, st_, ops, n, k, phase, st)
                phase ^= 1
                n -= k
        mo.ring, mo.region, mo.n_reg = saved
        eng._graphs.clear()
        torch.cuda.current_stream().synchronize()
        return grad.cpu().numpy() / self._adj_scale[:, None, None]

    def _time_adjoint(self, grid, state, stream, reps: int = 3) -> int:
        """Blocked or single reverse steps, whichever runs faster on this problem (a
        single design on a small grid leaves the blocked tiles too few to fill the GPU).
        Timed before the backward pass: no gradient, no operations, and every launch reads
        the still-zero current copy, so nothing changes."""
        tb = self.engine.time_block
        if tb <= 1:
            return 1
        grad = state.grad
        state.grad = None
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        best = {}
        for k in (tb, 1):
            nat.adjoint_step2d_multi(grid, state, None, tb - 1, k, 0, stream)  # warm-up
            t = float("inf")
            for _ in range(reps):
                a.record()
                for _ in range(tb // k):
                    nat.adjoint_step2d_multi(grid, state, None, tb - 1, k, 0, stream)
                b.record()
                b.synchronize()
                t = min(t, a.elapsed_time(b))
            best[k] = t
        state.grad = grad
        return min(best, key=best.get)

    def value_and_grad(self, eps_region):
        J = self.forward(eps_region)
        return J, self.backward()


class FDTDObjective(torch.autograd.Function):
    """J(eps_region) with the exact adjoint gradient; eps_region (B, h, w) float tensor."""

    @staticmethod
    def forward(ctx, eps_region, problem):
        J, g = problem.value_and_grad(eps_region.detach().cpu().numpy())
        ctx.save_for_backward(torch.as_tensor(g, dtype=eps_region.dtype, device=eps_region.device))
        return torch.as_tensor(J, dtype=eps_region.dtype, device=eps_region.device)

    @staticmethod
    def backward(ctx, gJ):
        (g,) = ctx.saved_tensors
        return gJ[:, None, None] * g, None
