"""Magnetic field on the grid nodes (magneticField.pyx).

`multipoleExpansion` builds the multipole field of magneticField.pyx:23-59 on
the device: coefficients in T/m^n without a reference radius, the length of
`multipolesIn` setting the order, a shorter skew list padded with zeros.
The result feeds `Particles.bFieldToParticles` and the Boris push with
typeBField 2, or `Buildup(b_multipoles=...)`.
"""
import ctypes

import numpy as np
import torch

from . import _lib
from . import device as D

_lib.OTHER_DECLARED.update({"oec_multipole_field"})


def _declare():
    L = _lib.lib()
    if not getattr(L, "_field_declared", False):
        P = ctypes.c_void_p
        L.oec_multipole_field.restype = ctypes.c_int
        L.oec_multipole_field.argtypes = [ctypes.c_int32, ctypes.c_int32, P, P, P, ctypes.c_int32, P,
                                          ctypes.c_int32, P, P]
        L._field_declared = True
    return L


def multipoleExpansionDevice(gridObj, multipolesIn, skewMultipolesIn=()):
    """[Bx | By | Bz] f64 [3*npExt] on the device."""
    normal = np.ascontiguousarray(multipolesIn, dtype=np.float64).reshape(-1)
    skew = np.ascontiguousarray(skewMultipolesIn, dtype=np.float64).reshape(-1)
    nx, ny = gridObj.getNxExt(), gridObj.getNyExt()
    xm = D.to_device(np.asarray(gridObj.getXMesh(), np.float64), torch.float64)
    ym = D.to_device(np.asarray(gridObj.getYMesh(), np.float64), torch.float64)
    b = D.empty(3 * nx * ny, torch.float64)
    rc = _declare().oec_multipole_field(nx, ny, xm.data_ptr(), ym.data_ptr(),
                                        normal.ctypes.data_as(ctypes.c_void_p) if normal.size else None,
                                        normal.size, skew.ctypes.data_as(ctypes.c_void_p) if skew.size else None,
                                        skew.size, b.data_ptr(), D.stream())
    if rc:
        raise _lib.OecError("oec_multipole_field", rc)
    return b


def multipoleExpansion(gridObj, multipolesIn, skewMultipolesIn=()):
    """magneticField.pyx:23-59: [Bx | By | Bz] at the nodes (numpy copy)."""
    return D.to_numpy(multipoleExpansionDevice(gridObj, multipolesIn, skewMultipolesIn))
