"""openecloud_b200: the openECLOUD per-step particle-in-cell loop on B200.

Modules mirror the reference's module/class names (grid, particles,
particleBoundary, particleEmitter, particleManagement, poissonSolver, beam,
...).  Compute runs in liboec.so (hand-written sm_100a CUDA) through the C ABI
declared in include/oec.h.  The reference-API modules take device memory and
streams from torch; `session` drives a whole run through the library's own
context and run handles with numpy and scipy only.  Submodules load on first
use, so importing the package pulls in no GPU framework.
"""
import importlib

from . import _lib, constants  # noqa: F401

__all__ = ["constants", "grid", "particles", "particleBoundary", "particleEmitter", "poissonSolver", "grid_geom",
           "magneticField", "util", "beam", "buildup", "batch", "autotune", "checkpoint", "shard", "session",
           "lu_setup", "furman", "cnn", "particleManagement"]


def __getattr__(name):
    if name in __all__:
        return importlib.import_module(f".{name}", __name__)
    raise AttributeError(f"module {__name__!r} has no attribute {name!r}")
