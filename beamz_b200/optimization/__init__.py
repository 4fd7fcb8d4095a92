"""Topology-optimisation helpers."""
from . import topology
from .optimizers import Optimizer

__all__ = ["topology", "Optimizer"]
