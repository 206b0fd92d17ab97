"""Particle boundaries: absorption, wall intersection and wall normals.

Mirrors ``particleBoundary`` (particleBoundary.pyx): ``AbsorbRectangular``
(:77-221), ``AbsorbElliptical`` (:225-297) and ``AbsorbArbitraryCutCell``
(:302-481).  The inside test runs on the GPU (``oec_index_inside`` or fused in
``oec_push_gather``); the absorbed set, wall points, normals and the
secondary emission run on the GPU too (boundary.cu, emit.cu).
``isInside(x, y)`` is the scalar host predicate the reference exposes for
loaders.
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
        self._absorbed = None      # device (cap, 6) f64
        self._normals = None       # device (cap, 2) f64
        self._index = None         # device int32 indices of absorbed particles
        self._cb = None

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

    def indexInside(self):
        """Absorbed bit per particle on the device (1 = outside)."""
        P = self.particlesObj
        P._bind(self.gridObj)
        _lib.call("oec_index_inside", self.gridObj.c_grid(), P.c_particles(), self.c_boundary(),
                  P._mask.data_ptr(), P._status.data_ptr(), D.stream())

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
