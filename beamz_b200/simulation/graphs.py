"""CUDA-graph capture of an engine's launch sequence, and the DFT phasor table.

The engines capture a chunk of step launches once and replay it. Capture goes
through ``CUDAGraph.capture_begin``/``capture_end`` on a side stream rather than
the ``torch.cuda.graph`` context manager, which synchronizes the device and runs
the garbage collector on entry: a capture in the middle of a run would otherwise
stall the host until the GPU drains. The captured launches allocate nothing.
"""
from __future__ import annotations

import numpy as np
import torch


def capture(launches) -> torch.cuda.CUDAGraph:
    """Graph of the kernels that ``launches()`` issues on the current stream."""
    g = torch.cuda.CUDAGraph()
    cur = torch.cuda.current_stream()
    side = torch.cuda.Stream()
    side.wait_stream(cur)
    with torch.cuda.stream(side):
        g.capture_begin()
        try:
            launches()
        finally:
            g.capture_end()
    cur.wait_stream(side)
    return g


class KernelTimer:
    """CUDA-event timing of an engine's step-kernel launches, for direct (non-graph)
    launches: the engine calls ``before()``/``after()`` around each step-kernel launch
    on the launching stream; every ``every``-th launch is bracketed by an event pair.
    Events recorded during a graph capture cannot be timed, so engines run without
    graphs while a timer is attached."""

    def __init__(self, every: int = 1, capacity: int = 4096):
        self.every = max(1, int(every))
        self.pairs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                      for _ in range(capacity)]
        self.steps = []  # time steps advanced by each timed launch
        self.n_launch = 0
        self.used = 0
        self._open = False

    def before(self, steps: int = 1):
        self._open = self.n_launch % self.every == 0 and self.used < len(self.pairs)
        if self._open:
            self.pairs[self.used][0].record()
            self.steps.append(int(steps))

    def after(self):
        if self._open:
            self.pairs[self.used][1].record()
            self.used += 1
        self._open = False
        self.n_launch += 1

    def durations_ms(self):
        """Durations of the timed launches (synchronizes on the last one)."""
        if self.used == 0:
            return []
        self.pairs[self.used - 1][1].synchronize()
        return [a.elapsed_time(b) for a, b in self.pairs[:self.used]]


def dft_phasors(freqs, n_steps: int, dt: float, device) -> torch.Tensor:
    """[n_steps][n_freq][4] float64 table (cos wt_E, -sin wt_E, cos wt_H, -sin wt_H) with
    t_E = (n+1) dt and t_H = (n+1/2) dt, computed on the device (the angles are the
    same float64 products as a host computation; cos/sin agree to an ulp)."""
    n = torch.arange(n_steps, dtype=torch.float64, device=device)[:, None]
    w = torch.as_tensor(2 * np.pi * np.asarray(freqs, dtype=np.float64), device=device)[None, :]
    ae, ah = w * ((n + 1.0) * dt), w * ((n + 0.5) * dt)
    return torch.stack([torch.cos(ae), -torch.sin(ae), torch.cos(ah), -torch.sin(ah)], dim=-1).contiguous()
