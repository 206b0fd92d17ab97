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


# ------------------------------------------------------------- emission
# Furman-Pivi tables as the reference sets them (particleEmitter.pyx:107-152).
FURMAN_TABLES = {
    "stainless": dict(p1EInf=0.07, p1Ehat=0.5, eEHat=0., w=100., p=0.9, e1=0.26, e2=2., q=0.4, sigmaE=1.9,
                      p1RInf=0.74, eR=40., r=1., r1=0.26, r2=2., deltaTSHat=1.22, s=1.813, eHat0=310., t3=0.7,
                      t4=1., t1=0.66, t2=0.8, epsN=[3.9, 6.2, 13., 8.8, 6.25, 2.25, 9.2, 5.3, 17.8, 10.],
                      pSmallN=[1.6, 2., 1.8, 4.7, 1.8, 2.4, 1.8, 1.8, 2.3, 1.8]),
    "copper": dict(p1EInf=0.02, p1Ehat=0.496, eEHat=0., w=60.86, p=1., e1=0.26, e2=2., sigmaE=2., p1RInf=0.2,
                   eR=0.041, r=0.104, q=0.5, r1=0.26, r2=2., deltaTSHat=1.8848, s=1.54, eHat0=276.8, t3=0.7,
                   t4=1., t1=0.66, t2=0.8, epsN=[2.5, 3.3, 2.5, 2.5, 2.8, 1.3, 1.5, 1.5, 1.5, 1.5],
                   pSmallN=[1.5, 1.75, 1., 3.75, 8.5, 11.5, 2.5, 3., 2.5, 3.]),
}


class OrcFurman(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in ("p1EInf", "p1Ehat", "eEHat", "w", "p", "e1", "e2", "p1RInf", "eR",
                                               "r", "r1", "r2", "q", "sigmaE", "deltaTSHat", "s", "eHat0", "t1",
                                               "t2", "t3", "t4", "theta0max", "deltaERmax")] + \
               [("epsN", ctypes.c_double * 10), ("pSmallN", ctypes.c_double * 10),
                ("particle_mass", ctypes.c_double), ("m", ctypes.c_int32), ("scaleSigmaE", ctypes.c_int32),
                ("compat_last", ctypes.c_int32), ("reserved", ctypes.c_int32)]


def furman(material="copper", seyMax=-1.0, eHat0=None, compat=True, scaleSigmaE=0):
    t = dict(FURMAN_TABLES[material])
    t["theta0max"] = 84. * 3.141592653589793 / 180
    t["deltaERmax"] = 0.99
    if seyMax >= 0.5:
        t["deltaTSHat"] = seyMax - t["p1RInf"] - t["p1EInf"]
    if eHat0 is not None:
        t["eHat0"] = eHat0
    f = OrcFurman()
    for k, v in t.items():
        if k in ("epsN", "pSmallN"):
            getattr(f, k)[:] = v
        else:
            setattr(f, k, v)
    f.particle_mass = 9.10938291e-31
    f.m = 10
    f.scaleSigmaE = scaleSigmaE
    f.compat_last = 1 if compat else 0
    return f


def furman_emit(params, rows, normals, mode=0, uniforms=None, seed=None):
    """generateSecondaries restated; mode 0: MT stream (seed first), mode 1: uniforms (n, 32)."""
    L = lib()
    if not getattr(L, "_emit_declared", False):
        L.orc_furman_emit.restype = _I64
        L.orc_furman_emit.argtypes = [ctypes.POINTER(OrcFurman), _P, _P, _I64, _I, _P, _P, _I64, _P]
        L.orc_betaincinv.restype = _D
        L.orc_betaincinv.argtypes = [_D, _D, _D]
        L.orc_gammaincinv.restype = _D
        L.orc_gammaincinv.argtypes = [_D, _D]
        L._emit_declared = True
    rows = _c(rows, np.float64)
    normals = _c(normals, np.float64)
    n = rows.shape[0]
    if seed is not None:
        L.orc_seed(int(seed))
    u = _c(uniforms if uniforms is not None else np.zeros((1, 32)), np.float64)
    cap = 10 * max(n, 1)
    out = np.empty((cap, 6), np.float64)
    warn = np.zeros(2, np.int32)
    k = L.orc_furman_emit(ctypes.byref(params), _p(rows), _p(normals), n, int(mode), _p(u), _p(out), cap, _p(warn))
    return out[:k].copy()


class OrcSecElec(ctypes.Structure):
    _fields_ = [("model", ctypes.c_int32), ("max_ts", ctypes.c_int32)] + \
        [(k, ctypes.c_double) for k in ("p1EInf", "p1Ehat", "eEHat", "w", "p", "e1", "e2", "p1RInf", "eR", "r", "r1",
                                        "r2", "deltaTSHat", "s", "eHat0", "t1", "t2", "t3", "t4", "sigmaETS",
                                        "muETS", "theta0max", "deltaERmax", "q", "particle_mass")]


# SecElecEmitter.stainlessMod (particleEmitter.pyx:331-352)
STAINLESS_SIMPLE = dict(p1EInf=0.07, p1Ehat=0.5, eEHat=0., w=100., p=0.9, e1=0.26, e2=2., q=0.4, p1RInf=0.74,
                        eR=40., r=1., r1=0.26, r2=2., deltaTSHat=1.22, s=1.813, eHat0=310., t3=0.7, t4=1., t1=0.66,
                        t2=0.8, sigmaETS=1.041, muETS=2.456)


def secelec(model=0, seyMax=-1.0, reflec=-1.0, max_ts=10):
    """Parameters of SecElecEmitter (model 0, stainlessMod with seyMax /
    reflec, particleEmitter.pyx:331-352) or SimpleSecEmitter (model 1)."""
    t = dict(STAINLESS_SIMPLE)
    t["theta0max"] = 84. * 3.141592653589793 / 180
    t["deltaERmax"] = 0.99
    if seyMax >= 0.5:
        t["deltaTSHat"] = seyMax - t["p1RInf"] - t["p1EInf"]
        if t["deltaTSHat"] < 0.:
            t["deltaTSHat"] = 1.e-6
    if reflec >= 0.:
        t["p1Ehat"] = reflec
    f = OrcSecElec()
    for k, v in t.items():
        setattr(f, k, v)
    f.model, f.max_ts = int(model), int(max_ts)
    f.particle_mass = 9.10938291e-31
    return f


def secelec_emit(params, rows, normals, mode=0, uniforms=None, seed=None):
    """SecElecEmitter / SimpleSecEmitter.generateSecondaries restated; mode 0:
    MT stream (seed first), mode 1: uniforms (n, 64)."""
    L = lib()
    if not getattr(L, "_secelec_declared", False):
        L.orc_secelec_emit.restype = _I64
        L.orc_secelec_emit.argtypes = [ctypes.POINTER(OrcSecElec), _P, _P, _I64, _I, _P, _P, _I64]
        L._secelec_declared = True
    rows = _c(rows, np.float64)
    normals = _c(normals, np.float64)
    n = rows.shape[0]
    if seed is not None:
        L.orc_seed(int(seed))
    u = _c(uniforms if uniforms is not None else np.zeros((1, 64)), np.float64)
    cap = (2 + params.max_ts) * max(n, 1)
    out = np.empty((cap, 6), np.float64)
    k = L.orc_secelec_emit(ctypes.byref(params), _p(rows), _p(normals), n, int(mode), _p(u), _p(out), cap)
    return out[:k].copy()


def betaincinv(a, b, p):
    furman_emit(furman(), np.zeros((0, 6)), np.zeros((0, 2)))  # declares signatures
    return lib().orc_betaincinv(float(a), float(b), float(p))


def gammaincinv(a, p):
    furman_emit(furman(), np.zeros((0, 6)), np.zeros((0, 2)))
    return lib().orc_gammaincinv(float(a), float(p))


# ------------------------------------------------------------ management
def _manage_declared():
    L = lib()
    if not getattr(L, "_manage_declared", False):
        L.orc_quicksort_by_column.restype = None
        L.orc_quicksort_by_column.argtypes = [_P, _I64, _I64, _I]
        L.orc_global_random.restype = _I64
        L.orc_global_random.argtypes = [_P, _I64, _I64, _P]
        L.orc_local_random_ellipse.restype = _I64
        L.orc_local_random_ellipse.argtypes = [_P, _I64, _I64, _I64, _D, _D, _D, _D, _I, _D, _D, _D, _I,
                                               ctypes.c_uint, _P]
        L.orc_add_and_remove.restype = _I64
        L.orc_add_and_remove.argtypes = [_P, _I64, _I64, _P, _I64, _P]
        L._manage_declared = True
    return L


def homo_loader(kind, lx, ly, n, w0, vsigma=10000. * 2.2250738585072014e-308, randomize=0, seed=None):
    """homoLoader (particleEmitter.pyx:41-72) with the MT stream: n rows
    uniform inside the rectangle (kind 0) or the ellipse (kind 1) of the
    particle boundary, Gaussian velocities of deviation vsigma (the
    reference's default: 1e4 times the smallest normal double), weight w0
    (or w0 (0.5 + U) with randomize)."""
    L = lib()
    if not getattr(L, "_homo_declared", False):
        L.orc_homo_loader.restype = None
        L.orc_homo_loader.argtypes = [_I, _D, _D, _I64, _D, _D, _I, _P]
        L._homo_declared = True
    if seed is not None:
        L.orc_seed(int(seed))
    pd = np.zeros((int(n), 6))
    L.orc_homo_loader(int(kind), float(lx), float(ly), int(n), float(w0), float(vsigma), int(randomize), _p(pd))
    return pd


def add_and_remove(pd, add, keep, array_len):
    """addAndRemoveParticles (particles.pyx:94-121, :201-269) on a particle
    array of `array_len` rows holding the rows of `pd`: returns the rows
    after the call and the array's row count (int(1.1 * count) when the
    call allocated a new array)."""
    L = _manage_declared()
    pd = np.asarray(pd, np.float64).reshape(-1, 6)
    add = np.ascontiguousarray(add, np.float64).reshape(-1, 6)
    keep = np.ascontiguousarray(keep, np.uint16)
    n, m = pd.shape[0], add.shape[0]
    a = np.zeros((max(n, int(keep[:n].sum()) + m, 1), 6))
    a[:n] = pd
    k = L.orc_add_and_remove(_p(a), int(array_len), n, _p(add) if m else None, m, _p(keep))
    if m and k > array_len:
        array_len = int(k * 1.1)
    return a[:k].copy(), int(array_len)


def sort_by_column(pd, col=5, seed=None):
    """sortByColumn (particles.pyx:49-50, :431-459) with the MT stream."""
    L = _manage_declared()
    if seed is not None:
        L.orc_seed(int(seed))
    a = np.array(pd, np.float64, copy=True, order="C")
    L.orc_quicksort_by_column(_p(a), 0, a.shape[0] - 1, int(col))
    return a


def global_random(pd, target, seed=None):
    """globalRandom (particleManagement.pyx:35-67) with the MT stream."""
    L = _manage_declared()
    if seed is not None:
        L.orc_seed(int(seed))
    n = pd.shape[0]
    a = np.zeros((max(n, target), 6))
    a[:n] = pd
    scratch = np.zeros((max(target - n, 1), 6))
    k = L.orc_global_random(_p(a), n, int(target), _p(scratch))
    return a[:k].copy()


def local_random(pd, target, g, kind=1, seed=None, threshold=2., lambda_factor=1., dis_limit=1., scheme=0,
                 leaf=10, array_len=None):
    """localRandom (particleManagement.pyx:74-238) with the MT stream.  The
    particle array holds n rows, as after setParticleData, or array_len rows
    when given; then the array's row count after the call is returned too
    (int(1.1 * count) when the refill needed a new array)."""
    L = _manage_declared()
    if seed is not None:
        L.orc_seed(int(seed))
    n = pd.shape[0]
    cap = n if array_len is None else int(array_len)
    room = 2 * n + 10
    a = np.zeros((room, 6))
    a[:n] = pd
    scratch = np.zeros((n + 10, 6))
    k = L.orc_local_random_ellipse(_p(a), cap, n, int(target), g.dx, g.dy, g.lx, g.ly, 1 if kind == 0 else 0,
                                   float(threshold), float(lambda_factor), float(dis_limit), int(scheme),
                                   int(leaf), _p(scratch))
    if array_len is None:
        return a[:k].copy()
    # more rows than the array holds can only come from added (split) rows
    return a[:k].copy(), (int(k * 1.1) if k > cap else cap)


# ------------------------------------------------- fixed-point deposit
def deposit_bits(total_capacity):
    """Fixed-point bits of a particle's charge: each particle's charge stays
    below 2^bits units, so capacity * 2^bits <= 2^63 keeps any node inside
    int64; at most 50."""
    lc = 0
    while (1 << lc) < total_capacity:
        lc += 1
    return min(50, 63 - lc)


def deposit_scale(w, total_capacity):
    """wscale = 2^(bits - ceil(log2 max|w|)) as the device computes it from
    the FP32 weights (the exponent e of frexp(max|w|))."""
    m = float(np.max(np.abs(np.asarray(w, np.float32)))) if len(w) else 0.0
    e = np.frexp(m)[1] if m > 0 and np.isfinite(m) else 0
    return float(np.ldexp(1.0, deposit_bits(total_capacity) - int(e)))


def fixed_point_deposit(cell, ox, oy, w, nx, n_nodes, wscale):
    """The order-independent int64 deposit of chargeToGrid
    (particles.pyx:336-351) in the units of wscale: per particle the charge
    qd = rint(w * wscale) is split into the CIC corner parts
    rint(qd * (1-fx)(1-fy)), rint(qd * fx(1-fy)), rint(qd * (1-fx)fy) and the
    remainder (so the four sum to qd exactly), all in round-to-nearest f64,
    added to nodes cell, cell+1, cell+nx, cell+nx+1.  Particles whose cell
    has a corner off the grid are skipped."""
    cell = np.asarray(cell, np.int64)
    gx = np.asarray(ox, np.float32).astype(np.float64)
    gy = np.asarray(oy, np.float32).astype(np.float64)
    qd = np.rint(np.asarray(w, np.float32).astype(np.float64) * wscale)
    ok = (cell >= 0) & (cell < n_nodes - nx - 1)
    cell, gx, gy, qd = cell[ok], gx[ok], gy[ok], qd[ok]
    hx, hy = 1.0 - gx, 1.0 - gy
    v0 = np.rint(qd * (hx * hy))
    v1 = np.rint(qd * (gx * hy))
    v2 = np.rint(qd * (hx * gy))
    v3 = qd - v0 - v1 - v2
    rho = np.zeros(n_nodes, np.int64)
    for off, v in ((0, v0), (1, v1), (nx, v2), (nx + 1, v3)):
        np.add.at(rho, cell + off, v.astype(np.int64))
    return rho
