"""Diagnostics (util.pyx)."""
import ctypes

import torch

from . import _lib
from . import device as D
from .constants import elementary_charge

_lib.OTHER_DECLARED.update({"oec_average_energy_sums"})


def _declare():
    L = _lib.lib()
    if not getattr(L, "_util_declared", False):
        L.oec_average_energy_sums.restype = ctypes.c_int
        L.oec_average_energy_sums.argtypes = [ctypes.POINTER(_lib.Particles_t), ctypes.c_void_p, ctypes.c_void_p]
        L._util_declared = True
    return L


def averageEnergy(partObj):
    """util.pyx:8-20: weighted mean kinetic energy of the particles in eV
    (sums in f64 on the device; NaN for an empty store, where the reference
    divides by zero)."""
    sums = D.zeros(2, torch.float64)
    rc = _declare().oec_average_energy_sums(partObj.c_particles(), sums.data_ptr(), D.stream())
    if rc:
        raise _lib.OecError("oec_average_energy_sums", rc)
    e, w = D.to_numpy(sums)
    return float(e * partObj.getParticleMass() * 0.5 / elementary_charge / w) if w != 0 else float("nan")
