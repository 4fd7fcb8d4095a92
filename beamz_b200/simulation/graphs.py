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


def dft_phasors(freqs, n_steps: int, dt: float, device) -> torch.Tensor:
    """[n_steps][n_freq][4] float64 table (cos wt_E, -sin wt_E, cos wt_H, -sin wt_H) with
    t_E = (n+1) dt and t_H = (n+1/2) dt, computed on the device (the angles are the
    same float64 products as a host computation; cos/sin agree to an ulp)."""
    n = torch.arange(n_steps, dtype=torch.float64, device=device)[:, None]
    w = torch.as_tensor(2 * np.pi * np.asarray(freqs, dtype=np.float64), device=device)[None, :]
    ae, ah = w * ((n + 1.0) * dt), w * ((n + 0.5) * dt)
    return torch.stack([torch.cos(ae), -torch.sin(ae), torch.cos(ah), -torch.sin(ah)], dim=-1).contiguous()
