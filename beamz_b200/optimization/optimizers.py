"""Gradient-step rules for density updates (the ``Optimizer`` of
beamz/optimization/optimizers.py:23-107), on torch tensors.

``Optimizer(method, learning_rate, options)`` keeps its moment estimates between calls;
``step(gradient)`` returns the update to add to the parameters (it does not change
them), as an array of the kind it was given, computed on the gradient's device in
float64. A batch of designs is one gradient array with leading batch dimensions, and
each element keeps its own moments.

Methods:
  "adam"  Kingma & Ba (2015): m = b1 m + (1-b1) g, v = b2 v + (1-b2) g^2 (both from
          zero), update = -lr (m / (1 - b1^t)) / (sqrt(v / (1 - b2^t)) + eps), with
          options beta1 (0.9), beta2 (0.999), epsilon (1e-8).
  "sgd"   update = -lr g.
"""
from __future__ import annotations

from typing import Mapping, Optional

import numpy as np
import torch


class _Adam:
    def __init__(self, beta1: float = 0.9, beta2: float = 0.999, epsilon: float = 1e-8):
        self.b1, self.b2, self.eps = float(beta1), float(beta2), float(epsilon)
        self.m = self.v = None
        self.t = 0

    def __call__(self, g: torch.Tensor, lr: float) -> torch.Tensor:
        if self.m is None or self.m.shape != g.shape or self.m.device != g.device:
            self.m, self.v, self.t = torch.zeros_like(g), torch.zeros_like(g), 0
        self.t += 1
        self.m.mul_(self.b1).add_(g, alpha=1.0 - self.b1)
        self.v.mul_(self.b2).addcmul_(g, g, value=1.0 - self.b2)
        m_hat = self.m / (1.0 - self.b1 ** self.t)
        v_hat = self.v / (1.0 - self.b2 ** self.t)
        return -lr * m_hat / (v_hat.sqrt() + self.eps)


class _Sgd:
    def __init__(self):
        pass

    def __call__(self, g: torch.Tensor, lr: float) -> torch.Tensor:
        return -lr * g


_RULES = {"adam": _Adam, "sgd": _Sgd}


class Optimizer:
    """Stateful update rule; see the module docstring."""

    def __init__(self, method: str = "adam", learning_rate: float = 1e-2, options: Optional[Mapping] = None):
        rule = _RULES.get(str(method).lower())
        if rule is None:
            raise ValueError(f"optimizer method {method!r} is not one of {sorted(_RULES)}")
        self.method = str(method).lower()
        self.learning_rate = float(learning_rate)
        self.options = dict(options or {})
        self._rule = rule(**self.options)

    def step(self, gradient):
        if not isinstance(gradient, (np.ndarray, torch.Tensor)):
            raise TypeError(f"gradient must be a NumPy array or a torch tensor, not {type(gradient).__name__}")
        g = gradient.to(torch.float64) if isinstance(gradient, torch.Tensor) else \
            torch.as_tensor(np.asarray(gradient, dtype=np.float64))
        if g.numel() == 0:
            out = torch.zeros_like(g)
        else:
            out = self._rule(g, self.learning_rate)
        return out if isinstance(gradient, torch.Tensor) else out.cpu().numpy()

    def reset(self) -> None:
        self._rule = _RULES[self.method](**self.options)


__all__ = ["Optimizer"]
