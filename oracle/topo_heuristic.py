"""The reference's own topology gradient estimate (test oracle, see oracle/__init__.py).

Restates examples/4_topo.py:276-341: a forward run caches Ez every step; a second
run is driven at the output line with amplitudes 0.5 + 0.5 * target (the
transmission and mode weights of 4_topo.py:225-230, the target profile normalised
to unit norm) and the forward signal, no direction enforcement; the estimate is
grad = sum_n Re(Ez_adj[n] * conj(Ez_fwd[N-1-n])) (4_topo.py:338-340), i.e. the
cached forward fields are consumed from the last one backwards.
"""
from __future__ import annotations

import numpy as np

from . import fdtd2d


class _LineSource:
    def __init__(self, amps, xs, ys, signal, direction="-x"):
        self.mode_profiles = [[[a, x, y, 0.0] for a, x, y in zip(amps, xs, ys)]]
        self.signal = signal
        self.direction = direction
        self.enforce_direction = False


def heuristic_gradient(eps, sigma, dx, dt, n_steps, sources, monitor, mode, region):
    """Reference estimate of d(objective)/d(eps) over region (y0, x0, h, w)."""
    y0, x0, h, w = region
    steps = range(n_steps)
    fwd = fdtd2d.run(eps, sigma, dx, dx, dt, n_steps, sources, [], snapshot_steps=set(steps))
    xs, ys = fdtd2d.monitor_points(monitor, dx, dx)
    target = np.asarray(mode, dtype=complex)
    target = target / (np.linalg.norm(target) or 1.0)
    amps = 0.5 + 0.5 * target
    signal = np.asarray(sources[0].signal)
    adj_src = _LineSource(amps, xs * dx, ys * dx, signal)
    adj = fdtd2d.run(eps, sigma, dx, dx, dt, n_steps, [adj_src], [], snapshot_steps=set(steps))
    g = np.zeros((h, w))
    for n in steps:
        ea = adj["snapshots"][n][0][y0:y0 + h, x0:x0 + w]
        ef = fwd["snapshots"][n_steps - 1 - n][0][y0:y0 + h, x0:x0 + w]
        g += np.real(ea * np.conj(ef))
    return g
