"""Grid: extended equidistant grid with staircase or cut-cell boundary.

Mirrors ``grid.Grid`` of the reference (grid.pyx:34-105, getters :1338-1434).
The scalar constants are computed exactly as the reference computes them.
The geometry arrays (inside points/edges/faces, edge lengths, cut-cell
boundary points and normals, edge-to-node interpolation) are built by the
host C++ routine ``oec_grid_geometry`` in liboec.so (grid_geom.cpp) on first
use and are uploaded to the device when a kernel needs them.
"""
import numpy as np
import scipy.sparse as spsp

from . import _lib
from .constants import machineEpsilon  # noqa: F401  (re-exported like the reference)


def _boundFuncRectangular(x, y, lxHalf, lyHalf):
    """grid.pyx:1437-1441."""
    return 1 if (x < lxHalf and x > -lxHalf and y < lyHalf and y > -lyHalf) else 0


def _boundFuncElliptical(x, y, aSqInv, bSqInv):
    """grid.pyx:1443-1447."""
    return 1 if 1 > x ** 2 * aSqInv + y ** 2 * bSqInv else 0


class Grid:
    """Reference: grid.pyx:49-105 (constructor) and :1338-1434 (getters)."""

    def __init__(self, nx, ny, lx, ly, boundType, boundFunc=None, cutCellAcc=1e-12, scanAroundPoint=1.e-3):
        if boundType not in (0, 1, 2, 3, 4):
            raise NotImplementedError("Not yet implemented.")
        if int(nx) < 2 or int(ny) < 2:
            raise ValueError("nx and ny must be at least 2")
        self.nx = int(nx)
        self.ny = int(ny)
        self.np = self.nx * self.ny
        self.lx = float(lx)
        self.ly = float(ly)
        self.dx = self.lx / (self.nx - 1.)
        self.dy = self.ly / (self.ny - 1.)
        self.cutCellAcc = float(cutCellAcc)
        self.scanAroundPoint = float(scanAroundPoint)
        self.nxExt = self.nx + 2
        self.nyExt = self.ny + 2
        self.npExt = self.nxExt * self.nyExt
        self.lxExt = self.lx + 2. * self.dx
        self.lyExt = self.ly + 2. * self.dy
        self.xMesh = np.linspace(-self.lxExt / 2., self.lxExt / 2, self.nxExt)
        self.yMesh = np.linspace(-self.lyExt / 2., self.lyExt / 2, self.nyExt)
        self.boundType = int(boundType)
        self.boundFuncPoints = None
        if boundType == 0:
            lxh, lyh = self.lx * 0.5, self.ly * 0.5
            self.boundFunc = lambda x, y: _boundFuncRectangular(x, y, lxh, lyh)
        elif boundType == 1:
            a, b = 4. / self.lx ** 2, 4. / self.ly ** 2
            self.boundFunc = lambda x, y: _boundFuncElliptical(x, y, a, b)
        elif boundType in (2, 3):
            if boundFunc is None:
                raise ValueError("boundType 2/3 needs a boundFunc(x, y) -> 0/1")
            self.boundFunc = boundFunc
        else:
            self.boundFuncPoints = np.ascontiguousarray(boundFunc, dtype=np.float64)
            self.boundFunc = self.pointInPolygon
        self._geom = None
        self._dev = {}

    # ------------------------------------------------------------ geometry
    def _geometry(self):
        if self._geom is None:
            from . import grid_geom
            self._geom = grid_geom.compute(self)
        return self._geom

    def pointInPolygon(self, xx, yy):
        """grid.pyx:108-120: winding-number test of (|x|, |y|)."""
        from . import grid_geom
        return grid_geom.point_in_polygon(self, xx, yy)

    def c_grid(self):
        """The oec_grid_t descriptor of this grid."""
        return _lib.Grid_t(self.nxExt, self.nyExt, self.dx, self.dy, self.lx, self.ly)

    def device_array(self, name, dtype):
        """Geometry array uploaded once to the device (cached)."""
        import torch
        from . import device as D
        key = (name, dtype)
        if key not in self._dev:
            a = self._geometry()[name]
            self._dev[key] = D.to_device(np.ascontiguousarray(a), dtype=dtype)
        return self._dev[key]

    # ------------------------------------------------------------- getters
    def getXMesh(self): return self.xMesh
    def getYMesh(self): return self.yMesh
    def getLx(self): return self.lx
    def getLy(self): return self.ly
    def getLxExt(self): return self.lxExt
    def getLyExt(self): return self.lyExt
    def getDx(self): return self.dx
    def getDy(self): return self.dy
    def getNxExt(self): return self.nxExt
    def getNyExt(self): return self.nyExt
    def getNpExt(self): return self.npExt
    def getNx(self): return self.nx
    def getNy(self): return self.ny
    def getNp(self): return self.np
    def getBoundaryPoints(self): return self._geometry()["boundaryPoints"]
    def getBoundaryPointsInd(self): return self._geometry()["boundaryPointsInd"]
    def getCutCellPointsInd(self): return self._geometry()["cutCellPointsInd"]
    def getCutCellCenter(self): return self._geometry()["cutCellCenter"]
    def getCutCellNormalVectors(self): return self._geometry()["cutCellNormalVectors"]
    def getInsidePoints(self): return self._geometry()["insidePoints"]
    def getInsideEdges(self): return self._geometry()["insideEdges"]
    def getInsideFaces(self): return self._geometry()["insideFaces"]
    def getDs(self): return self._geometry()["ds"]
    def getDsi(self): return self._geometry()["dsi"]
    def getDa(self): return self._geometry()["da"]
    def getDai(self): return self._geometry()["dai"]
    def getDst(self): return self._geometry()["dst"]
    def getDat(self): return self._geometry()["dat"]
    def getDati(self): return self._geometry()["dati"]
    def getEdgeToNode(self): return self._geometry()["edgeToNode"]
    def getBoundFunc(self): return self.boundFunc
