"""Particle boundaries: absorption, wall intersection and wall normals.

Mirrors ``particleBoundary`` (particleBoundary.pyx): ``AbsorbRectangular``
(:77-221), ``AbsorbElliptical`` (:225-297) and ``AbsorbArbitraryCutCell``
(:302-481).  Everything runs on the GPU: the inside test
(``oec_index_inside``, or fused into ``oec_push_gather``) leaves one absorbed
bit per particle; ``saveAbsorbed`` turns the bits into the ascending list of
absorbed indices and their (n_abs, 6) float64 rows; the wall intersection
and the normals are one kernel (``oec_wall_interaction``).  ``isInside(x, y)``
is the scalar host predicate the reference exposes for loaders.
"""
import numpy as np
import torch

from . import _lib
from . import device as D


class ParticleBoundary:
    kind = None

    def __init__(self, gridObj, particlesObj):
        self.gridObj = gridObj
        self.particlesObj = particlesObj
        self.nx = gridObj.getNxExt()
        self.ny = gridObj.getNyExt()
        self.np = gridObj.getNpExt()
        self.lx = gridObj.getLx()
        self.ly = gridObj.getLy()
        self.dx = gridObj.getDx()
        self.dy = gridObj.getDy()
        self.absorbedMacroParticleCount = 0
        self._index = None         # device int32: ascending absorbed indices
        self._n_abs = None         # device int32 scalar
        self._scratch = None
        self._rows = None          # device (cap, 6) f64 absorbed rows
        self._normals = None       # device (cap, 2) f64 wall normals
        self._wall_done = False
        self._cb = None

    # ------------------------------------------------------------ plumbing
    def c_boundary(self):
        if self._cb is None:
            b = _lib.Boundary_t()
            b.kind = self.kind
            if self.kind == _lib.BOUNDARY_CUTCELL:
                g = self.gridObj
                b.n_boundary_points = int(g.getBoundaryPoints().shape[0])
                b.inside_faces_dev = g.device_array("insideFaces", torch.int16).data_ptr()
                b.boundary_points_dev = g.device_array("boundaryPoints", torch.float64).data_ptr()
                b.cut_cell_points_ind_dev = g.device_array("cutCellPointsInd", torch.int32).data_ptr()
                b.cut_cell_normals_dev = g.device_array("cutCellNormalVectors", torch.float64).data_ptr()
            self._cb = b
        return self._cb

    def ensure_buffers(self, rows):
        """Device buffers for the absorbed index list and `rows` absorbed rows."""
        P = self.particlesObj
        if self._index is None or self._index.shape[0] < P._cap:
            self._index = D.empty(max(P._cap, 1), torch.int32)
            self._n_abs = D.zeros(1, torch.int32)
            self._scratch = D.zeros(1024, torch.int32)
        if self._rows is None or self._rows.shape[0] < rows:
            cap = max(int(rows * 1.1) + 1, 1024)
            self._rows = D.zeros((cap, 6), torch.float64)
            self._normals = D.zeros((cap, 2), torch.float64)

    # ----------------------------------------------------------------- API
    def indexInside(self):
        """Absorbed bit per particle on the device (1 = outside)."""
        P = self.particlesObj
        P._bind(self.gridObj)
        _lib.call("oec_index_inside", self.gridObj.c_grid(), P.c_particles(), self.c_boundary(),
                  P._mask.data_ptr(), P._status.data_ptr(), D.stream())

    def absorbedIndex(self):
        """Device: ascending absorbed indices and their count (no host sync)."""
        P = self.particlesObj
        self.ensure_buffers(1)
        _lib.call("oec_absorbed_index", P.c_particles(), P._mask.data_ptr(), self._index.data_ptr(),
                  self._index.shape[0], self._n_abs.data_ptr(), self._scratch.data_ptr(), P._status.data_ptr(),
                  D.stream())
        return self._index, self._n_abs

    def saveAbsorbed(self):
        """particleBoundary.pyx:38-65: the absorbed rows, in index order."""
        P = self.particlesObj
        P._bind(self.gridObj)
        self.absorbedIndex()
        n = int(self._n_abs.item())
        self.ensure_buffers(n)
        _lib.call("oec_save_absorbed", self.gridObj.c_grid(), P.c_particles(), self._index.data_ptr(),
                  self._n_abs.data_ptr(), self._rows.shape[0], self._rows.data_ptr(), D.stream())
        self.absorbedMacroParticleCount = n
        self._wall_done = False

    def _wall(self):
        if self._wall_done:
            return
        P = self.particlesObj
        _lib.call("oec_wall_interaction", self.gridObj.c_grid(), self.c_boundary(), P.getDt(), self._rows.data_ptr(),
                  self._n_abs.data_ptr(), self._rows.shape[0], self._normals.data_ptr(), P._status.data_ptr(),
                  D.stream())
        self._wall_done = True

    def calculateInteractionPoint(self):
        """Move the absorbed rows back onto the wall (normals computed alongside)."""
        self._wall()

    def calculateNormalVectors(self):
        """Inward wall normals of the absorbed rows."""
        self._wall()

    def getAbsorbedParticles(self):
        return D.to_numpy(self._rows[:self.absorbedMacroParticleCount])

    def getNormalVectors(self):
        return D.to_numpy(self._normals[:self.absorbedMacroParticleCount])

    def getAbsorbedParticlesDevice(self):
        return self._rows[:self.absorbedMacroParticleCount]

    def getNormalVectorsDevice(self):
        return self._normals[:self.absorbedMacroParticleCount]

    def getAbsorbedMacroParticleCount(self):
        return self.absorbedMacroParticleCount


class AbsorbRectangular(ParticleBoundary):
    kind = _lib.BOUNDARY_RECT

    def isInside(self, x, y):
        """particleBoundary.pyx:99-105."""
        lxh, lyh = self.lx * 0.5, self.ly * 0.5
        return 0 if (x < -lxh or x > lxh or y < -lyh or y > lyh) else 1


class AbsorbElliptical(ParticleBoundary):
    kind = _lib.BOUNDARY_ELLIPSE

    def isInside(self, x, y):
        """particleBoundary.pyx:244-249."""
        a, b = 4. / self.lx ** 2, 4. / self.ly ** 2
        return 0 if (x ** 2 * a + y ** 2 * b) >= 1. else 1


class AbsorbArbitraryCutCell(ParticleBoundary):
    kind = _lib.BOUNDARY_CUTCELL

    def isInside(self, x, y):
        """particleBoundary.pyx:304-333."""
        g = self.gridObj
        faces = g.getInsideFaces()
        bp = g.getBoundaryPoints()
        cpi = g.getCutCellPointsInd()
        ix = int((x + 0.5 * g.getLxExt()) * (1. / g.getDx()))
        iy = int((y + 0.5 * g.getLyExt()) * (1. / g.getDy()))
        c = ix + iy * g.getNxExt()
        if faces[c] == 8:
            return 1
        if faces[c] == 0:
            return 0
        a, b = cpi[c, 0], cpi[c, 1]
        return 1 if (bp[a, 0] - x) * (bp[b, 1] - y) > (bp[b, 0] - x) * (bp[a, 1] - y) else 0
