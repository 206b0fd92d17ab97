"""Secondary emission (Furman-Pivi) and the initial uniform loader.

Mirrors ``particleEmitter`` (particleEmitter.pyx): ``FurmanEmitter`` (:77-311)
with the reference's copper and stainless-steel parameter tables (:107-152)
and ``homoLoader`` (:41-72).  Emission runs on the GPU (``oec_furman_emit``):
each absorbed particle draws from its own Philox4x32-10 stream keyed by the
run seed, so a run is reproducible for a given seed.  The reference's single
secondary split reads the yields of the LAST absorbed particle of the first
pass (stale loop variables, :245-246); ``compat=True`` (default) reproduces
that, ``compat=False`` uses each particle's own yields.
"""
import ctypes

import numpy as np
import torch

from . import _lib
from . import device as D
from .constants import pi, doubleMinVal  # noqa: F401
from .furman import COPPER, STAINLESS, Furman_t, furman_params, furman_struct  # noqa: F401


_lib.OTHER_DECLARED.update({"oec_furman_emit", "oec_furman_work_bytes", "oec_secelec_emit", "oec_secelec_work_bytes"})


def _declare():
    L = _lib.lib()
    if not getattr(L, "_emit_declared", False):
        P = ctypes.c_void_p
        L.oec_furman_emit.restype = ctypes.c_int
        L.oec_furman_emit.argtypes = [ctypes.POINTER(Furman_t), P, P, P, ctypes.c_int32, P, ctypes.c_uint64,
                                      ctypes.c_uint32, P, P, P, P, ctypes.c_int32, P, P, P]
        L.oec_furman_work_bytes.restype = ctypes.c_int64
        L.oec_furman_work_bytes.argtypes = [ctypes.c_int32]
        L.oec_secelec_emit.restype = ctypes.c_int
        L.oec_secelec_emit.argtypes = [ctypes.POINTER(SecElec_t), P, P, P, ctypes.c_int32, P, ctypes.c_uint64,
                                       ctypes.c_uint32, P, P, P, P, ctypes.c_int32, P, P, P]
        L.oec_secelec_work_bytes.restype = ctypes.c_int64
        L.oec_secelec_work_bytes.argtypes = [ctypes.c_int32]
        L._emit_declared = True
    return L


class FurmanEmitter:
    """Reference: particleEmitter.pyx:77-311."""

    def __init__(self, particleBoundaryObj, particlesObj, material="copper", seyMax=-1., reflec=-1.,
                 scaleSigmaE=0, seed=0, compat=True):
        self.particlesObj = particlesObj
        self.particleBoundaryObj = particleBoundaryObj
        self.params = furman_params(material, seyMax, reflec)
        self.scaleSigmaE = int(scaleSigmaE)
        self.particleMass = particlesObj.getParticleMass()
        self.m = 10
        self.seed = int(seed)
        self.compat = bool(compat)
        self.step = 0
        self._work = None
        self._out = None
        self._n_out = None
        self.out_cap = None  # bound on the output rows (None: m per absorbed row)
        self.secondaryCount = 0

    def setEHat0(self, value):
        """E_max of the true-secondary yield (copperMod's eHat0)."""
        self.params["eHat0"] = float(value)

    def c_params(self):
        return furman_struct(self.params, self.particleMass, m=self.m, scaleSigmaE=self.scaleSigmaE,
                             compat=self.compat)

    def ensure_buffers(self, cap_abs):
        L = _declare()
        if self._work is None or self._cap_abs < cap_abs:
            self._cap_abs = int(cap_abs)
            self._work = D.empty(int(L.oec_furman_work_bytes(self._cap_abs)), torch.uint8)
            self._n_out = D.zeros(1, torch.int32)
        # output rows: m per absorbed row, or at most `out_cap` when the caller
        # fixes it (a buildup whose store cannot grow: secondaries beyond its
        # capacity could not be added, and the emission counts them dropped)
        out_rows = self.m * self._cap_abs
        if self.out_cap is not None:
            out_rows = min(out_rows, max(int(self.out_cap), 1))
        out_rows += 1
        if self._out is None or self._out.shape[0] < out_rows:
            self._out = D.zeros((out_rows, 6), torch.float64)

    def _launch(self, cap, step, step_dev, replay):
        """One emission over the boundary's first min(n_abs, cap) rows into
        this emitter's buffers (the step counter added to `step` when given
        on the device); no host synchronisation."""
        bd = self.particleBoundaryObj
        ids = bd._index.data_ptr() if bd._index is not None else None
        rc = _declare().oec_furman_emit(ctypes.byref(self.c_params()), bd._rows.data_ptr(), bd._normals.data_ptr(),
                                        bd._n_abs.data_ptr(), cap, ids, self.seed, step & 0xffffffff,
                                        step_dev.data_ptr() if step_dev is not None else None,
                                        replay.data_ptr() if replay is not None else None, self._work.data_ptr(),
                                        self._out.data_ptr(), self._out.shape[0], self._n_out.data_ptr(),
                                        self.particlesObj._status.data_ptr(), D.stream())
        if rc:
            raise _lib.OecError("oec_furman_emit", rc)

    def emitDevice(self, replay=None, step=None):
        """Launch the emission for the boundary's absorbed rows; returns the
        device rows buffer and the device count (no host synchronisation)."""
        bd = self.particleBoundaryObj
        bd._wall()
        cap = bd._rows.shape[0]
        self.ensure_buffers(cap)
        step = self.step if step is None else int(step)
        self._launch(cap, step, None, replay)
        self.step += 1
        return self._out, self._n_out

    def generateSecondaries(self, replay=None):
        """particleEmitter.pyx:154-308: the secondaries as a (n, 6) device tensor."""
        out, n = self.emitDevice(replay=replay)
        self.secondaryCount = int(n.item())
        return out[:self.secondaryCount]

    def getEmittedParticles(self):
        return D.to_numpy(self._out[:self.secondaryCount])


class SecElec_t(ctypes.Structure):
    _fields_ = [("model", ctypes.c_int32), ("max_ts", ctypes.c_int32)] + \
        [(k, ctypes.c_double) for k in ("p1EInf", "p1Ehat", "eEHat", "w", "p", "e1", "e2", "p1RInf", "eR", "r", "r1",
                                        "r2", "deltaTSHat", "s", "eHat0", "t1", "t2", "t3", "t4", "sigmaETS",
                                        "muETS", "theta0max", "deltaERmax", "q", "particle_mass")]


# SecElecEmitter.stainlessMod (particleEmitter.pyx:331-352)
STAINLESS_SECELEC = dict(p1EInf=0.07, p1Ehat=0.5, eEHat=0., w=100., p=0.9, e1=0.26, e2=2., q=0.4, p1RInf=0.74,
                         eR=40., r=1., r1=0.26, r2=2., deltaTSHat=1.22, s=1.813, eHat0=310., t3=0.7, t4=1., t1=0.66,
                         t2=0.8, sigmaETS=1.041, muETS=2.456)


class SecElecEmitter:
    """Reference: particleEmitter.pyx:316-484 -- a simplified Furman model
    for stainless steel: an elastic and a rediffused secondary with
    probabilities delta_E and delta_R and a Bernoulli-rounded number of true
    secondaries with lognormal energies, on the device (`oec_secelec_emit`).
    Draws come from per-row Philox streams keyed by `seed`, row and step;
    true secondaries of one absorbed particle are capped at `maxTrue` (the
    reference has no cap; capped rows count in the status block)."""

    MODEL = 0

    def __init__(self, particleBoundaryObj, particlesObj, seyMax=-1., reflec=-1., seed=0, maxTrue=10):
        self.particlesObj = particlesObj
        self.particleBoundaryObj = particleBoundaryObj
        self.particleMass = particlesObj.getParticleMass()
        self.seed = int(seed)
        self.max_ts = int(maxTrue)
        self.m = self.max_ts + 2  # rows per absorbed particle at most
        self.step = 0
        self._work = None
        self._out = None
        self._n_out = None
        self.out_cap = None  # bound on the output rows (None: m per absorbed row)
        self.secondaryCount = 0
        self.stainlessMod(seyMax, reflec)

    def stainlessMod(self, seyMax, reflec):
        """particleEmitter.pyx:331-352."""
        t = dict(STAINLESS_SECELEC, theta0max=84. * pi / 180., deltaERmax=0.99)
        if seyMax >= 0.5:
            t["deltaTSHat"] = seyMax - t["p1RInf"] - t["p1EInf"]
            if t["deltaTSHat"] < 0.:
                t["deltaTSHat"] = 1.e-6
                print("WARNING: Maximum SEY too small. Setting true SEY to zero.")
        if reflec >= 0.:
            t["p1Ehat"] = reflec
        self.params = t

    def c_params(self):
        f = SecElec_t()
        for k, v in self.params.items():
            setattr(f, k, float(v))
        f.model, f.max_ts = self.MODEL, self.max_ts
        f.particle_mass = self.particleMass
        return f

    def ensure_buffers(self, cap_abs):
        L = _declare()
        if self._work is None or self._cap_abs < cap_abs:
            self._cap_abs = int(cap_abs)
            self._work = D.empty(int(L.oec_secelec_work_bytes(self._cap_abs)), torch.uint8)
            self._n_out = D.zeros(1, torch.int32)
        # output rows: m per absorbed row, or at most `out_cap` when the caller
        # fixes it (a buildup whose store cannot grow: secondaries beyond its
        # capacity could not be added, and the emission counts them dropped)
        out_rows = self.m * self._cap_abs
        if self.out_cap is not None:
            out_rows = min(out_rows, max(int(self.out_cap), 1))
        out_rows += 1
        if self._out is None or self._out.shape[0] < out_rows:
            self._out = D.zeros((out_rows, 6), torch.float64)

    def _launch(self, cap, step, step_dev, replay):
        bd = self.particleBoundaryObj
        ids = bd._index.data_ptr() if bd._index is not None else None
        rc = _declare().oec_secelec_emit(ctypes.byref(self.c_params()), bd._rows.data_ptr(), bd._normals.data_ptr(),
                                         bd._n_abs.data_ptr(), cap, ids, self.seed, step & 0xffffffff,
                                         step_dev.data_ptr() if step_dev is not None else None,
                                         replay.data_ptr() if replay is not None else None, self._work.data_ptr(),
                                         self._out.data_ptr(), self._out.shape[0], self._n_out.data_ptr(),
                                         self.particlesObj._status.data_ptr(), D.stream())
        if rc:
            raise _lib.OecError("oec_secelec_emit", rc)

    emitDevice = FurmanEmitter.emitDevice

    def generateSecondaries(self, replay=None):
        """The secondaries as a (n, 6) device tensor (replay: injected
        uniforms, 64 per absorbed row)."""
        out, n = self.emitDevice(replay=replay)
        self.secondaryCount = int(n.item())
        return out[:self.secondaryCount]

    def getEmittedParticles(self):
        return D.to_numpy(self._out[:self.secondaryCount])


class SimpleSecEmitter(SecElecEmitter):
    """Reference: particleEmitter.pyx:489-597 ("currently only for
    testing"): fixed yields delta_E = 0.05, delta_R = 0.5 and a stainless-like
    true yield, secondaries along the reversed incident velocity (true ones
    with a uniform 0-5 eV energy); seyMax and reflec are ignored, as in the
    reference."""

    MODEL = 1


def homoLoader(gridObj, particlesObj, partBoundObj, macroParticleCount, weightInit, vsigma=10000. * doubleMinVal,
               randomizeWeight=0, seed=0):
    """particleEmitter.pyx:41-72 on the device: uniform rejection sampling
    inside the particle boundary, Gaussian velocities, weight w0 (or
    w0*(0.5+U))."""
    P = particlesObj
    P._bind(gridObj)
    n = int(macroParticleCount)
    P.ensure_capacity(n)
    failed = D.zeros(1, torch.int32)
    _lib.call("oec_homo_load", gridObj.c_grid(), partBoundObj.c_boundary(), P.c_particles(), n, float(weightInit),
              float(vsigma), int(randomizeWeight), int(seed) & 0xffffffffffffffff, failed.data_ptr(), D.stream())
    if int(failed.item()):
        raise RuntimeError("homoLoader: rejection sampling found no inside point for some particles")
    P._array_len.fill_(n)  # the reference stores the loaded rows with setParticleData
