"""Time signals (beamz/devices/signals.py:5-23), evaluated on the host in float64.

Sources index their signal by time-step number (helper.py:10,57), so a signal is
simply an array with one value per step of the simulation's time axis.
"""
from __future__ import annotations

import numpy as np


def cosine(t, amplitude, frequency, phase):
    return amplitude * np.cos(2 * np.pi * frequency * t + phase)


def sigmoid(t, duration=1, min=0, max=1, t0=0):  # noqa: A002 - reference keyword names
    return min + (max - min) * (1 / (1 + np.exp(-10 * (t - duration / 2 - t0) / duration)))


def ramped_cosine(t, amplitude, frequency, phase=None, ramp_duration=None, t_max=None):
    """Cosine with a sigmoid switch-on over ``ramp_duration`` and a switch-off
    ending at ``t_max`` (default ramp: t_max / 10)."""
    if phase is None:
        phase = 0
    if ramp_duration is None:
        ramp_duration = t_max / 10
    signal = sigmoid(t, min=0, max=1, duration=ramp_duration, t0=0)
    signal *= cosine(t, amplitude=amplitude, frequency=frequency, phase=phase)
    signal *= sigmoid(t, min=1, max=0, duration=ramp_duration, t0=t_max - ramp_duration)
    return signal


def gaussian(t, amplitude, center, width):
    return amplitude * np.exp(-(t - center) ** 2 / (2 * width ** 2))


def gaussian_pulse(t, amplitude, center, width, frequency, phase):
    """Gaussian envelope times cosine carrier; like the reference, the amplitude
    multiplies both factors (so the peak is amplitude**2)."""
    return gaussian(t, amplitude, center, width) * cosine(t, amplitude, frequency, phase)


def plot_signal(signals, t):
    raise NotImplementedError("plotting is not part of beamz_b200")
