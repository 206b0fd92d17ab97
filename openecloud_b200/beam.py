"""Rigid proton beam imprinted on the grid.

Mirrors ``beam.LHCBeam`` (beam.py:13-78) and ``beam.LHCBeamEndless``
(beam.py:81-136).  The transverse profile (integral of a round Gaussian over
each node's cell, cut at 5 sigma, normalised to one) is built once on the
host; the charge per node at time t is a scalar (the longitudinal Gaussian
integrated over one time step, times N_b e / (c dt)) times that profile.
The device path precomputes the scalars of a whole run (``scalarTable``) so
the per-step right-hand side is formed on the GPU in the same kernel that
converts the fixed-point electron deposit (``oec_rhs_with_beam``).

The radius and bunch-length sigmas are constructor arguments with the
reference's values as defaults (1 mm / 2 mm, 0.1 m).
"""
import numpy as np
import scipy.constants as spc
from scipy.special import ndtr

# beam.py takes e and c from scipy.constants (beam.py:9, :25-26), not from the
# reference's constants.pyx; the installed SciPy's values are used here too.
elementary_charge = spc.elementary_charge
c = spc.c


class _BeamBase:
    def __init__(self, gridObj, dt, nParticles, tBunchSpacing, radiusSigma, bunchLengthSigma):
        self.gridObj = gridObj
        self.nx = gridObj.getNxExt()
        self.ny = gridObj.getNyExt()
        self.np = gridObj.getNpExt()
        self.lx = gridObj.getLxExt()
        self.ly = gridObj.getLyExt()
        self.dx = gridObj.getDx()
        self.dy = gridObj.getDy()
        self.dt = dt
        self.nParticles = nParticles
        self.charge = elementary_charge
        self.beamVelocity = c
        self.circumference = 6900
        self.radiusSigma = radiusSigma
        self.radiusLimitSigma = 5
        self.xBeamCenter = 0.
        self.yBeamCenter = 0.
        self.tBunchSpacing = tBunchSpacing
        self.bunchLengthSigma = bunchLengthSigma
        self.tBunchLengthSigma = self.bunchLengthSigma / self.beamVelocity
        self.bunchLengthLimitSigma = 5
        self.qTransversalProfile = self._profile()

    def _profile(self):
        """beam.py:47-63: CDF differences over each node's cell."""
        xMesh = self.gridObj.getXMesh()
        yMesh = self.gridObj.getYMesh()
        x = np.tile(xMesh, self.ny)
        y = np.reshape(np.tile(yMesh, (self.nx, 1)).transpose(), self.np)
        s, lim = self.radiusSigma, self.radiusLimitSigma
        inside = ((lim * s + max([self.dx, self.dy])) ** 2 - x ** 2 - y ** 2) > 0
        prof = np.zeros(self.np)
        fx = (ndtr(np.clip((x - self.xBeamCenter + self.dx / 2.) / s, -lim, lim)) -
              ndtr(np.clip((x - self.xBeamCenter - self.dx / 2.) / s, -lim, lim)))
        fy = (ndtr(np.clip((y - self.yBeamCenter + self.dy / 2.) / s, -lim, lim)) -
              ndtr(np.clip((y - self.yBeamCenter - self.dy / 2.) / s, -lim, lim)))
        prof[inside] = (fx * fy)[inside]
        prof /= np.sum(prof)
        return prof

    def getTransversalProfile(self):
        return self.qTransversalProfile

    def _slice(self, tRed):
        lim, st = self.bunchLengthLimitSigma, self.tBunchLengthSigma
        return (ndtr(np.clip((tRed + self.dt / 2.) / st - lim, -lim, lim)) -
                ndtr(np.clip((tRed - self.dt / 2.) / st - lim, -lim, lim)))

    def chargeScalar(self, t):
        """Scalar s(t) with getCharge(t) = s(t) * profile."""
        raise NotImplementedError

    def getCharge(self, t):
        s = self.chargeScalar(t)
        return s * self.qTransversalProfile if s != 0 else 0

    def scalarTable(self, n_steps, t0=0.0):
        """s(t0 + i dt) for i < n_steps (float64 array)."""
        return np.array([self.chargeScalar(t0 + i * self.dt) for i in range(int(n_steps))], np.float64)


class LHCBeam(_BeamBase):
    """beam.py:13-78: 4 batches of 72 bunches, 8 empty slots between batches."""

    def __init__(self, gridObj, dt, nParticles=1.e11, tBunchSpacing=25.e-9, radiusSigma=0.001,
                 bunchLengthSigma=0.1):
        self.tRevolution = 6900 / c
        self.nBatches = 4
        self.nBunchesPerBatch = 72
        self.nEmptyBunches = 8
        super().__init__(gridObj, dt, nParticles, 25.e-9, radiusSigma, bunchLengthSigma)
        self.tBatchLength = self.nBunchesPerBatch * self.tBunchSpacing
        self.tBatchSpacing = self.nEmptyBunches * self.tBunchSpacing
        self.tTrainLength = (self.nBatches * self.nBunchesPerBatch + (self.nBatches - 1) * self.nEmptyBunches) * \
            self.tBunchSpacing
        del tBunchSpacing  # the reference fixes the spacing at 25 ns for the train (beam.py:36)

    def chargeScalar(self, t):
        """beam.py:68-78."""
        if (np.mod(t, self.tBunchSpacing) < 2 * self.bunchLengthLimitSigma * self.tBunchLengthSigma and
                np.mod(t, self.tBatchLength + self.tBatchSpacing) < self.tBatchLength and
                np.mod(t, self.tRevolution) < self.tTrainLength):
            tRed = np.mod(np.mod(t, self.tRevolution), self.tBunchSpacing)
            return float(self._slice(tRed) * self.nParticles / self.dt / self.beamVelocity * self.charge)
        return 0.0


class LHCBeamEndless(_BeamBase):
    """beam.py:81-136: an endless train of equal bunches."""

    def __init__(self, gridObj, dt, nParticles=1.e11, tBunchSpacing=25.e-9, radiusSigma=0.002,
                 bunchLengthSigma=0.1):
        super().__init__(gridObj, dt, nParticles, tBunchSpacing, radiusSigma, bunchLengthSigma)

    def chargeScalar(self, t):
        """beam.py:129-136."""
        if np.mod(t, self.tBunchSpacing) < 2 * self.bunchLengthLimitSigma * self.tBunchLengthSigma:
            tRed = np.mod(t, self.tBunchSpacing)
            return float(self._slice(tRed) * self.nParticles / self.dt / self.beamVelocity * self.charge)
        return 0.0
