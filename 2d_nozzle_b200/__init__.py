"""B200-native nodal-DG backend for the 2D Euler nozzle solver.

The product is the CUDA library in ``csrc/`` (C ABI: ``include/nozzle_b200.h``)
and :class:`~.backend.B200Backend`, a drop-in implementation of the reference
solver's ``Backend`` interface that drives it.  The package directory name is
not a Python identifier, so import it with
``importlib.import_module("2d_nozzle_b200")``.
"""

from __future__ import annotations

from . import config, mesh, operators, refelem  # noqa: F401  (host-only, no torch)

__all__ = ["B200Backend", "get_backend", "config", "mesh", "operators", "refelem"]


def __getattr__(name):
    if name == "B200Backend":
        from .backend import B200Backend

        return B200Backend
    raise AttributeError(name)


def get_backend(name, ops, flow, opts):
    """The registry branch a host application adds: ``"b200"`` -> :class:`B200Backend`."""
    if name == "b200":
        from .backend import B200Backend

        return B200Backend(ops, flow, opts)
    raise ValueError(f"unknown backend {name!r}; this package provides 'b200'")
