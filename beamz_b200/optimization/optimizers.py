"""Optimizer wrapper for topology updates (beamz/optimization/optimizers.py:23-107).

Only Adam is registered, with the reference's defaults (beta1 0.9, beta2 0.999,
epsilon 1e-8, bias-corrected moments); ``step(gradient)`` returns the update to
add to the parameters.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Callable, Dict, Mapping, MutableMapping

import numpy as np

UpdateFn = Callable[[np.ndarray, float, MutableMapping[str, np.ndarray]], np.ndarray]


def _adam_update(grad, learning_rate, state, *, beta1=0.9, beta2=0.999, epsilon=1e-8):
    if "m" not in state:
        state["m"] = np.zeros_like(grad)
    if "v" not in state:
        state["v"] = np.zeros_like(grad)
    state["t"] = state.get("t", 0) + 1
    m, v, t = state["m"], state["v"], state["t"]
    m *= beta1
    m += (1.0 - beta1) * grad
    v *= beta2
    v += (1.0 - beta2) * (grad ** 2)
    m_hat = m / (1.0 - beta1 ** t)
    v_hat = v / (1.0 - beta2 ** t)
    return -learning_rate * m_hat / (np.sqrt(v_hat) + epsilon)


_OPTIMIZER_REGISTRY: Dict[str, UpdateFn] = {"adam": _adam_update}


@dataclass
class Optimizer:
    method: str = "adam"
    learning_rate: float = 1e-2
    options: Mapping[str, float] = field(default_factory=dict)
    _state: MutableMapping[str, np.ndarray] = field(default_factory=dict, init=False)

    def __post_init__(self) -> None:
        key = self.method.lower()
        if key not in _OPTIMIZER_REGISTRY:
            raise ValueError(f"Unknown optimizer method '{self.method}'. "
                             f"Available: {', '.join(sorted(_OPTIMIZER_REGISTRY))}.")
        self._update_fn = _OPTIMIZER_REGISTRY[key]

    def step(self, gradient: np.ndarray) -> np.ndarray:
        if not isinstance(gradient, np.ndarray):
            raise TypeError("Gradient must be a numpy.ndarray")
        if gradient.size == 0:
            return np.zeros_like(gradient)
        return self._update_fn(gradient, self.learning_rate, self._state, **self.options)

    def reset(self) -> None:
        self._state.clear()


__all__ = ["Optimizer"]
