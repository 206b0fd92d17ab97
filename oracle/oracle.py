"""Python access to the CPU oracle (``liboec_oracle.so``) -- TEST INFRASTRUCTURE.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg import this module, always as the checker.  The product package never
imports anything under ``oracle/``.

The shared object is built from ``oec_oracle.c`` (the FP64 restatement of the
reference routines, each citing its reference file:line) plus the
project-written GSL stand-in ``gsl_shim/oec_gsl_shim.c``.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboec_oracle.so")
SOURCES = [os.path.join(HERE, "oec_oracle.c"), os.path.join(HERE, "oec_oracle_emit.c"),
           os.path.join(HERE, "oec_oracle_manage.c"), os.path.join(HERE, "gsl_shim", "oec_gsl_shim.c")]

_lib = None


def build(force=False):
    """Compile liboec_oracle.so with gcc (no FMA contraction, like the reference build)."""
    srcs = [s for s in SOURCES if os.path.exists(s)]
    if not force and os.path.exists(LIB_PATH):
        t = os.path.getmtime(LIB_PATH)
        if all(os.path.getmtime(s) <= t for s in srcs):
            return LIB_PATH
    cmd = ["gcc", "-O2", "-fPIC", "-shared", "-ffp-contract=off", "-std=gnu11",
           "-I" + os.path.join(HERE, "gsl_shim"), "-o", LIB_PATH + ".tmp"] + srcs + ["-lm"]
    subprocess.run(cmd, check=True)
    os.replace(LIB_PATH + ".tmp", LIB_PATH)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = ctypes.CDLL(LIB_PATH)
        _declare(_lib)
    return _lib


_P = ctypes.c_void_p
_D = ctypes.c_double
_I64 = ctypes.c_int64
_U32 = ctypes.c_uint32
_I = ctypes.c_int


def _declare(L):
    def sig(name, res, args):
        if hasattr(L, name):
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
    sig("orc_seed", None, [ctypes.c_ulong])
    sig("orc_rand", _D, [])
    sig("orc_randn", _D, [])
    sig("orc_randi", ctypes.c_ulong, [ctypes.c_ulong])
    sig("orc_calc_grid_weights", None, [_P, _I64, _D, _D, _D, _D, _U32, _P, _P, _P, _P, _P])
    sig("orc_charge_to_grid", None, [_P, _I64, _P, _P, _P, _P, _P, _D, _U32, _U32, _P])
    sig("orc_field_to_particles", None, [_P, _I, _P, _P, _P, _P, _P, _U32, _U32, _I64, _P])
    sig("orc_boris_push", None, [_P, _I64, _P, _P, _P, _D, _D, _I])
    sig("orc_index_inside_rect", None, [_P, _I64, _D, _D, _P])
    sig("orc_index_inside_ellipse", None, [_P, _I64, _D, _D, _P])
    sig("orc_clip_to_grid", _I, [_P, _I64, _D, _D])
    sig("orc_index_inside_cutcell", None, [_P, _I64, _D, _D, _D, _D, _U32, _P, _P, _P, _P])
    sig("orc_save_absorbed", _I64, [_P, _I64, _P, _P])
    sig("orc_interaction_rect", None, [_P, _I64, _D, _D, _D, _D, _P])
    sig("orc_interaction_ellipse", None, [_P, _I64, _D, _D, _D, _D, _P])
    sig("orc_interaction_cutcell", _I64, [_P, _I64, _D, _D, _D, _D, _D, _U32, _P, _P, _P, _P, _P])


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _c(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


class GridGeom:
    """Scalar grid constants as the reference computes them (grid.pyx:57-68)."""

    def __init__(self, nx, ny, lx, ly):
        self.nx_in, self.ny_in = int(nx), int(ny)
        self.lx, self.ly = float(lx), float(ly)
        self.dx = self.lx / (self.nx_in - 1.)
        self.dy = self.ly / (self.ny_in - 1.)
        self.nx, self.ny = self.nx_in + 2, self.ny_in + 2
        self.np = self.nx * self.ny
        self.lxExt = self.lx + 2. * self.dx
        self.lyExt = self.ly + 2. * self.dy


def seed(s):
    lib().orc_seed(int(s))


def calc_grid_weights(pd, g):
    pd = _c(pd, np.float64)
    n = pd.shape[0]
    inc = np.empty(n, np.uint32)
    w = [np.empty(n, np.float64) for _ in range(4)]
    lib().orc_calc_grid_weights(_p(pd), n, 1. / g.dx, 1. / g.dy, g.lxExt * 0.5, g.lyExt * 0.5, g.nx,
                                _p(inc), *[_p(x) for x in w])
    return inc, w


def charge_to_grid(pd, g, charge):
    pd = _c(pd, np.float64)
    inc, w = calc_grid_weights(pd, g)
    q = np.empty(g.np, np.float64)
    lib().orc_charge_to_grid(_p(pd), pd.shape[0], _p(inc), *[_p(x) for x in w], float(charge), g.nx, g.np, _p(q))
    return q


def field_to_particles(pd, g, field, ncomp):
    pd = _c(pd, np.float64)
    field = _c(field, np.float64)
    inc, w = calc_grid_weights(pd, g)
    out = np.empty((pd.shape[0], ncomp), np.float64)
    lib().orc_field_to_particles(_p(field), ncomp, _p(inc), *[_p(x) for x in w], g.nx, g.np, pd.shape[0], _p(out))
    return out


def boris_push(pd, e_at, dt, qm, type_b, b_at=None, bconst=None):
    pd = np.array(pd, np.float64, copy=True, order="C")
    e_at = _c(e_at, np.float64)
    b_at = _c(b_at if b_at is not None else np.zeros((pd.shape[0], 3)), np.float64)
    bc = _c(bconst if bconst is not None else np.zeros(3), np.float64)
    lib().orc_boris_push(_p(pd), pd.shape[0], _p(e_at), _p(b_at), _p(bc), float(dt), float(qm), int(type_b))
    return pd


def index_inside(pd, g, kind, geom=None):
    """kind 0 rect, 1 ellipse, 2 cut-cell (geom: dict with faces, bpts, cpi). Returns (inside, pd')."""
    pd = np.array(pd, np.float64, copy=True, order="C")
    inside = np.empty(pd.shape[0], np.uint16)
    L = lib()
    if kind == 0:
        L.orc_index_inside_rect(_p(pd), pd.shape[0], g.lx, g.ly, _p(inside))
    elif kind == 1:
        L.orc_index_inside_ellipse(_p(pd), pd.shape[0], g.lx, g.ly, _p(inside))
    else:
        faces = _c(geom["insideFaces"], np.uint16)
        bpts = _c(geom["boundaryPoints"], np.float64)
        cpi = _c(geom["cutCellPointsInd"], np.int32)
        L.orc_index_inside_cutcell(_p(pd), pd.shape[0], g.lxExt * 0.5, g.lyExt * 0.5, g.dx, g.dy, g.nx,
                                   _p(faces), _p(bpts), _p(cpi), _p(inside))
    return inside, pd


def save_absorbed(pd, inside):
    pd = _c(pd, np.float64)
    inside = _c(inside, np.uint16)
    out = np.empty_like(pd)
    k = lib().orc_save_absorbed(_p(pd), pd.shape[0], _p(inside), _p(out))
    return out[:k].copy()


def interaction(ab, g, kind, dt=None, geom=None):
    """calculateInteractionPoint + calculateNormalVectors. Returns (ab', normals, n_missing)."""
    ab = np.array(ab, np.float64, copy=True, order="C")
    normals = np.empty((ab.shape[0], 2), np.float64)
    L = lib()
    missing = 0
    if kind == 0:
        L.orc_interaction_rect(_p(ab), ab.shape[0], g.lx, g.ly, g.dx, g.dy, _p(normals))
    elif kind == 1:
        L.orc_interaction_ellipse(_p(ab), ab.shape[0], g.lx, g.ly, g.dx, g.dy, _p(normals))
    else:
        faces = _c(geom["insideFaces"], np.uint16)
        bpts = _c(geom["boundaryPoints"], np.float64)
        cpi = _c(geom["cutCellPointsInd"], np.int32)
        cn = _c(geom["cutCellNormalVectors"], np.float64)
        missing = L.orc_interaction_cutcell(_p(ab), ab.shape[0], float(dt), g.lxExt * 0.5, g.lyExt * 0.5, g.dx,
                                            g.dy, g.nx, _p(faces), _p(bpts), _p(cpi), _p(cn), _p(normals))
    return ab, normals, int(missing)
