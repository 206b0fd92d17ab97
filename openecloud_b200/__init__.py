"""openecloud_b200: the openECLOUD per-step particle-in-cell loop on B200.

Modules mirror the reference's module/class names (grid, particles,
particleBoundary, particleEmitter, particleManagement, poissonSolver, beam,
...).  Compute runs in liboec.so (hand-written sm_100a CUDA) through the C ABI
declared in include/oec.h; torch provides device memory and streams.
"""
from . import _lib, constants, grid_geom  # noqa: F401
from . import grid, particles, particleBoundary, particleEmitter, particleManagement, poissonSolver  # noqa: F401
from . import beam, buildup, cnn, magneticField, util, autotune, batch  # noqa: F401

__all__ = ["constants", "grid", "particles", "particleBoundary", "particleEmitter", "poissonSolver", "grid_geom",
           "magneticField", "util", "beam", "buildup", "batch", "autotune"]
