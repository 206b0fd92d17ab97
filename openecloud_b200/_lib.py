"""ctypes binding of liboec.so (declared in include/oec.h).

The library is built in-tree by ``python -m openecloud_b200.build``.  There is
no fallback: if the shared object is missing the first call raises.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
# OEC_BOUNDS_CHECK=1 selects the bounds-checked build (liboec_checked.so:
# out-of-range indices are counted by oec_bound_violations and skipped)
LIB_PATH = os.path.join(_HERE, "liboec_checked.so" if os.environ.get("OEC_BOUNDS_CHECK") == "1" else "liboec.so")

OEC_OK = 0
ERRORS = {1: "invalid argument", 2: "CUDA runtime error", 3: "capacity exceeded",
          4: "iterative solve did not converge", 5: "fixed-point overflow", 6: "host failure"}

BOUNDARY_RECT, BOUNDARY_ELLIPSE, BOUNDARY_CUTCELL = 0, 1, 2


class OecError(RuntimeError):
    def __init__(self, name, code):
        super().__init__(f"{name} failed: {ERRORS.get(code, 'error')} (code {code})")
        self.code = code


class Particles_t(ctypes.Structure):
    _fields_ = [("cell", ctypes.c_void_p), ("ox", ctypes.c_void_p), ("oy", ctypes.c_void_p),
                ("vx", ctypes.c_void_p), ("vy", ctypes.c_void_p), ("vz", ctypes.c_void_p),
                ("w", ctypes.c_void_p), ("count", ctypes.c_void_p), ("capacity", ctypes.c_int64)]


class Grid_t(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("dx", ctypes.c_double),
                ("dy", ctypes.c_double), ("lx", ctypes.c_double), ("ly", ctypes.c_double)]


class Boundary_t(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("n_boundary_points", ctypes.c_int32),
                ("inside_faces_dev", ctypes.c_void_p), ("boundary_points_dev", ctypes.c_void_p),
                ("cut_cell_points_ind_dev", ctypes.c_void_p), ("cut_cell_normals_dev", ctypes.c_void_p)]


STATUS_FIELDS = ["n_absorbed", "n_secondaries", "n_nonfinite", "n_clipped", "n_not_found",
                 "n_capacity_drop", "deposit_overflow", "n_wait_timeout", "warn_derm", "warn_tsprime",
                 "n_out_of_grid", "n_rows_dropped", "n_emit_skipped"]
STATUS_WORDS = 16

_P = ctypes.c_void_p
_PP = ctypes.POINTER(Particles_t)
_PG = ctypes.POINTER(Grid_t)
_PB = ctypes.POINTER(Boundary_t)
_I32 = ctypes.c_int32
_I64 = ctypes.c_int64
_D = ctypes.c_double
_D3 = ctypes.c_double * 3

# name -> argtypes (all return int status)
SIGNATURES = {
    "oec_particles_from_aos": [_PG, _P, _I64, _PP, _P],
    "oec_particles_to_aos": [_PG, _PP, _P, _I64, _P],
    "oec_particles_upload_host": [_PG, _P, _I64, _PP, _P, _I64, _P],
    "oec_particles_download_host": [_PG, _PP, _P, _I64, _P, _I64, _P],
    "oec_calc_grid_weights": [_PG, _PP, _P, _P, _P, _P, _P, _P],
    "oec_field_prepare": [_PG, _P, _I32, _P, _P],
    "oec_gather": [_PG, _PP, _P, _I32, _P, _P],
    "oec_boris_push": [_PG, _PP, _P, _P, _P, _D, _D, _I32, _P],
    "oec_deposit_scale": [_PP, _P, _P],
    "oec_deposit_scale_capacity": [_PP, _I64, _P, _P],
    "oec_push_gather": [_PG, _PP, _P, _P, _P, _D, _D, _I32, _PB, _P, _P, _P, _P, _P],
    "oec_push_gather_host": [_PG, _PP, _P, _P, _I64, _P, _I64, _P, _P, _P, _D, _D, _I32, _PB, _P, _P, _P, _P,
                             _P],
    "oec_deposit": [_PG, _PP, _P, _P, _I32, _P, _P],
    "oec_deposit_finalize": [_PG, _P, _P, _D, _P, _P],
    "oec_deposit_charge_noalloc": [_PG, _PP, _D, _P, _P],
    "oec_index_inside": [_PG, _PP, _PB, _P, _P, _P],
    "oec_absorbed_index": [_PP, _P, _P, _I32, _P, _P, _P, _P],
    "oec_save_absorbed": [_PG, _PP, _P, _P, _I32, _P, _P],
    "oec_wall_interaction": [_PG, _PB, _D, _P, _P, _I32, _P, _P, _P],
    "oec_add_remove": [_PG, _PP, _PP, _P, _P, _P, _I32, _P, _P, _I32, _P, _P, _P, _P, _P],
    "oec_mask_from_keep": [_P, _I64, _P, _I64, _P],
    "oec_homo_load": [_PG, _PB, _PP, _I64, _D, _D, _I32, ctypes.c_uint64, _P, _P],
    "oec_sort_particles": [_PP, _PP, _I32, _P, _P],
    "oec_scale_weights": [_PP, _D, _P],
    "oec_roulette_select": [_I32, _I32, _P, _I64, ctypes.c_uint64, ctypes.c_uint32, _P, _P],
    "oec_clone_rows": [_PG, _PP, _I32, _I32, ctypes.c_uint64, ctypes.c_uint32, _P, _P],
    "oec_weight_stats": [_PP, _P, _P],
    "oec_weight_thresholds": [_PP, _D, _D, _P, _P],
    "oec_split_rows": [_PG, _PP, _I32, _I32, _P, _P],
    "oec_cell_merge": [_PG, _PP, _I32, _I32, _D, _D, _I32, ctypes.c_uint64, ctypes.c_uint32, _D, _P, _P, _P, _P],
    "oec_rhs_with_beam": [_PG, _P, _P, _D, _P, _P, _P, _I32, _P, _P],
    "oec_history": [_PP, _P, _I32, _P, _P, _P, _P],
    "oec_step_advance": [_P, _P],
    "oec_bound_violations": [_P, _I32],
}
_INT64_RETURNING = {"oec_sort_work_bytes": [_I64]}

_lib = None
# entry points whose ctypes signatures live next to their Python users
# (structure arguments defined there); registered at import of that module
OTHER_DECLARED = {"oec_sort_work_bytes"}


def lib():
    """Load liboec.so once; raise if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m openecloud_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        for name, args in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = ctypes.c_int
            f.argtypes = args
        for name, args in _INT64_RETURNING.items():
            f = getattr(L, name)
            f.restype = ctypes.c_int64
            f.argtypes = args
        _lib = L
    return _lib


def call(name, *args):
    rc = getattr(lib(), name)(*args)
    if rc != OEC_OK:
        raise OecError(name, rc)
    return rc


def d3(v):
    return _D3(*[float(x) for x in v])
