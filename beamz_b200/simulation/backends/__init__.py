"""Backend registry (beamz/simulation/backends/__init__.py:8-36).

``get_backend(name, **options)`` returns the B200 backend for "b200" (aliases
"cuda", "gpu"). The reference's "numpy", "jax" and "torch" names are accepted as
requests for a stepping backend and are served by the same B200 backend, the
way the reference falls back when a requested backend is unavailable; any other
name raises ``ValueError``.
"""
import logging

from .base import Backend

logger = logging.getLogger("beamz_b200")

_ALIASES = {"b200": "b200", "cuda": "b200", "gpu": "b200", "numpy": "b200", "jax": "b200", "torch": "b200"}


def get_backend(name="b200", **kwargs):
    key = str(name).lower()
    if key not in _ALIASES:
        raise ValueError(f"Unknown backend: {name}")
    if key in ("numpy", "jax", "torch"):
        logger.info("backend %r is served by the B200 backend", name)
    from .b200 import B200Backend

    return B200Backend(**kwargs)


__all__ = ["get_backend", "Backend"]
