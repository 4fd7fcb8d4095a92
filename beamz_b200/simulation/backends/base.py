"""The compute-backend interface (beamz/simulation/backends/base.py:3-43)."""
from abc import ABC, abstractmethod


class Backend(ABC):
    """Array factory plus the two 2D Yee half-step updates."""

    @abstractmethod
    def zeros(self, shape):
        ...

    @abstractmethod
    def ones(self, shape):
        ...

    @abstractmethod
    def copy(self, array):
        ...

    @abstractmethod
    def to_numpy(self, array):
        ...

    @abstractmethod
    def from_numpy(self, array):
        ...

    @abstractmethod
    def roll(self, array, shift, axis=None):
        ...

    @abstractmethod
    def update_h_fields(self, Hx, Hy, Ez, sigma, dx, dy, dt, mu_0, eps_0):
        ...

    @abstractmethod
    def update_e_field(self, Ez, Hx, Hy, sigma, epsilon_r, dx, dy, dt, eps_0):
        ...
