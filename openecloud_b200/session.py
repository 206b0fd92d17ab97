"""A buildup run driven through the library's own context and run handles.

This is the host side of a run for a program that brings no GPU framework:
numpy and scipy prepare what the reference prepares on the host -- the grid
geometry (Grid, host C++), the beam profile and its per-step factor
(beam.py), the Furman parameters (particleEmitter.pyx:107-152), the
assembled operator and its SuperLU factors (poissonSolver.pyx:33-67) -- and
the C ABI (include/oec.h: oec_ctx_*, oec_run_*) owns the device memory, the
stream and the step graph.  The loop itself is the reference's
(example01_basic.py:52-97) with the LU solve and globalRandom management.

    from openecloud_b200.session import Context, Run
    with Context(0) as ctx:
        run = Run(ctx, nx=128, ny=128, lx=0.04, ly=0.04, boundType=1, rows=rows)
        run.steps(2500)
        counts, weights = run.history()

Nothing here imports torch.
"""
import ctypes

import numpy as np

from . import _lib
from .beam import LHCBeam, LHCBeamEndless
from .constants import elementary_charge, m_e
from .furman import Furman_t, furman_params, furman_struct
from .grid import Grid
from .lu_setup import LU_t, factor, lu_host_arrays, lu_struct

_P = ctypes.c_void_p


class Status_t(ctypes.Structure):
    _fields_ = [(k, ctypes.c_int32) for k in _lib.STATUS_FIELDS] + \
               [("reserved", ctypes.c_int32 * (_lib.STATUS_WORDS - len(_lib.STATUS_FIELDS)))]


class RunDesc_t(ctypes.Structure):
    _fields_ = [("grid", _lib.Grid_t), ("boundary_kind", ctypes.c_int32), ("type_b", ctypes.c_int32),
                ("dt", ctypes.c_double), ("charge", ctypes.c_double), ("mass", ctypes.c_double),
                ("bconst", ctypes.c_double * 3), ("capacity", ctypes.c_int64), ("abs_cap", ctypes.c_int32),
                ("target", ctypes.c_int32), ("management_every", ctypes.c_int32), ("table_len", ctypes.c_int32),
                ("rows", _P), ("n_rows", ctypes.c_int64), ("furman", Furman_t), ("emit_seed", ctypes.c_uint64),
                ("manage_seed", ctypes.c_uint64), ("beam_profile", _P), ("beam_table", _P), ("lu", LU_t),
                ("e_ptr", _P), ("e_idx", _P), ("e_val", _P)]


_lib.OTHER_DECLARED.update({"oec_ctx_create", "oec_ctx_destroy", "oec_ctx_stream", "oec_ctx_synchronize",
                            "oec_ctx_alloc", "oec_status", "oec_run_create", "oec_run_steps", "oec_run_history",
                            "oec_run_get_rows", "oec_run_particles", "oec_run_destroy"})


def _declare():
    L = _lib.lib()
    if not getattr(L, "_session_declared", False):
        I32, I64 = ctypes.c_int32, ctypes.c_int64
        sig = {"oec_ctx_create": [I32, ctypes.POINTER(_P)], "oec_ctx_destroy": [_P],
               "oec_ctx_stream": [_P, ctypes.POINTER(_P)], "oec_ctx_synchronize": [_P],
               "oec_ctx_alloc": [_P, I64, ctypes.POINTER(_P)], "oec_status": [_P, ctypes.POINTER(Status_t)],
               "oec_run_create": [_P, ctypes.POINTER(RunDesc_t), ctypes.POINTER(_P)],
               "oec_run_steps": [_P, I32, I32], "oec_run_history": [_P, _P, _P, I32],
               "oec_run_get_rows": [_P, _P, I64, ctypes.POINTER(I64)],
               "oec_run_particles": [_P, ctypes.POINTER(_lib.Particles_t)], "oec_run_destroy": [_P]}
        for name, args in sig.items():
            f = getattr(L, name)
            f.restype = ctypes.c_int
            f.argtypes = args
        L._session_declared = True
    return L


def _call(name, *args):
    rc = getattr(_declare(), name)(*args)
    if rc != _lib.OEC_OK:
        raise _lib.OecError(name, rc)


def _ptr(a):
    return None if a is None else a.ctypes.data_as(_P).value


class Context:
    """oec_ctx_t: a device, its stream, its status block and its memory."""

    def __init__(self, device=0):
        h = _P()
        _call("oec_ctx_create", int(device), ctypes.byref(h))
        self.handle = h

    def status(self):
        st = Status_t()
        _call("oec_status", self.handle, ctypes.byref(st))
        return {k: int(getattr(st, k)) for k in _lib.STATUS_FIELDS}

    def synchronize(self):
        _call("oec_ctx_synchronize", self.handle)

    def close(self):
        if self.handle:
            _call("oec_ctx_destroy", self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class Run:
    """oec_run_t: one buildup run in `ctx`, set up on the host like
    Buildup (same parameters for the chamber, beam, emitter and management;
    LU solve, globalRandom) from the (N, 6) float64 initial rows."""

    def __init__(self, ctx, rows, nx=128, ny=128, lx=0.04, ly=0.04, boundType=1, dt=1e-11, beam="endless",
                 beam_particles=1.1e11, radius_sigma=0.002, bunch_length_sigma=0.25e-9 * 299792458.0,
                 material="copper", sey_max=1.6, e_hat0=300.0, type_b_field=0, b_const=(0., 0., 0.),
                 target=100000, management_every=50, capacity=None, abs_cap=None, seed=0, n_steps_table=2500,
                 tail=None):
        if boundType not in (0, 1):
            raise NotImplementedError("the run handle takes rectangular and elliptical chambers")
        self.ctx = ctx
        rows = np.ascontiguousarray(rows, np.float64).reshape(-1, 6)
        self.grid = g = Grid(nx, ny, lx, ly, boundType)
        cap = capacity or max(4 * int(target), 4 * rows.shape[0], 65536)
        beam_cls = LHCBeamEndless if beam == "endless" else LHCBeam
        bm = beam_cls(g, float(dt), nParticles=beam_particles, radiusSigma=radius_sigma,
                      bunchLengthSigma=bunch_length_sigma)
        self._keep = keep = {}
        keep["profile"] = np.ascontiguousarray(bm.getTransversalProfile(), np.float64)
        keep["table"] = np.ascontiguousarray(bm.scalarTable(int(n_steps_table)), np.float64)
        _, _, _, inside, lu, phi_to_e = factor(g)
        keep["lu"] = a = lu_host_arrays(lu, inside, g.getNpExt(), tail)
        E = phi_to_e.tocsr()
        E.sort_indices()
        keep["e_ptr"] = np.ascontiguousarray(E.indptr, np.int32)
        keep["e_idx"] = np.ascontiguousarray(E.indices, np.int32)
        keep["e_val"] = np.ascontiguousarray(E.data, np.float64)
        keep["rows"] = rows
        params = furman_params(material, sey_max)
        if e_hat0 is not None:
            params["eHat0"] = float(e_hat0)
        d = RunDesc_t()
        d.grid = g.c_grid()
        d.boundary_kind = boundType
        d.type_b = int(type_b_field)
        d.dt, d.charge, d.mass = float(dt), -elementary_charge, m_e
        d.bconst[:] = [float(b) for b in b_const]
        d.capacity = int(cap)
        d.abs_cap = int(abs_cap) if abs_cap is not None else max(4096, int(cap) // 8)
        d.target, d.management_every = int(target), int(management_every)
        d.table_len = int(n_steps_table)
        d.rows, d.n_rows = _ptr(rows), rows.shape[0]
        d.furman = furman_struct(params, m_e)
        d.emit_seed = int(seed) + 17      # the seed Buildup gives its FurmanEmitter
        d.manage_seed = int(seed)
        d.beam_profile, d.beam_table = _ptr(keep["profile"]), _ptr(keep["table"])
        d.lu = lu_struct(a, lambda name: _ptr(a.get(name)))
        d.e_ptr, d.e_idx, d.e_val = _ptr(keep["e_ptr"]), _ptr(keep["e_idx"]), _ptr(keep["e_val"])
        h = _P()
        _call("oec_run_create", ctx.handle, ctypes.byref(d), ctypes.byref(h))
        self.handle = h
        self.table_len = int(n_steps_table)
        self.steps_done = 0

    def steps(self, n, use_graph=True):
        _call("oec_run_steps", self.handle, int(n), 1 if use_graph else 0)
        self.steps_done += int(n)

    def history(self):
        """(macro count, sum of weights) at the start of every step so far."""
        n = self.steps_done + 1
        c = np.zeros(n, np.int32)
        w = np.zeros(n, np.float64)
        _call("oec_run_history", self.handle, _ptr(c), _ptr(w), n)
        return c, w

    def getParticleData(self):
        """(N, 6) float64 rows (particles.pyx:142)."""
        n = ctypes.c_int64(0)
        _call("oec_run_get_rows", self.handle, None, 0, ctypes.byref(n))
        out = np.zeros((max(n.value, 1), 6))
        _call("oec_run_get_rows", self.handle, _ptr(out), n.value, ctypes.byref(n))
        return out[:n.value]

    def close(self):
        if self.handle:
            _call("oec_run_destroy", self.handle)
            self.handle = None
