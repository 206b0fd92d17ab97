"""Host glue for the grid geometry built by ``oec_grid_geometry`` (grid_geom.cpp).

Allocates the output arrays, picks the boundary function (built-in
rectangle / ellipse / polygon in C++, or a user ``boundFunc`` called back
from C++), and composes the three sparse interpolation stages into
``edgeToNode`` in the reference's order (grid.pyx:427, :456, :925, :1203,
:1330): ``stage3 @ (stage2 @ stage1)``.
"""
import ctypes

import numpy as np
import scipy.sparse as spsp

from . import _lib

BOUND_RECT, BOUND_ELLIPSE, BOUND_POLYGON, BOUND_CALLBACK = 0, 1, 2, 3
_CB = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_void_p)


class GeomIn(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("dx", ctypes.c_double), ("dy", ctypes.c_double),
                ("x_mesh", ctypes.c_void_p), ("y_mesh", ctypes.c_void_p), ("scan_around_point", ctypes.c_double),
                ("cut_cell_acc", ctypes.c_double), ("cut_cell", ctypes.c_int32), ("bound_kind", ctypes.c_int32),
                ("p0", ctypes.c_double), ("p1", ctypes.c_double), ("poly", ctypes.c_void_p),
                ("n_poly", ctypes.c_int32), ("fn", _CB), ("ctx", ctypes.c_void_p)]


class GeomOut(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in ("inside_points", "inside_edges", "inside_faces", "ds", "dsi", "da",
                                                 "dai", "dst", "dsti", "dat", "dati", "boundary_points",
                                                 "boundary_points_ind")] + \
               [("cap_boundary_points", ctypes.c_int32), ("n_boundary_points", ctypes.c_int32),
                ("cut_cell_points_ind", ctypes.c_void_p), ("cut_cell_center", ctypes.c_void_p),
                ("cut_cell_normals", ctypes.c_void_p), ("cap_coo", ctypes.c_int64),
                ("r1", ctypes.c_void_p), ("c1", ctypes.c_void_p), ("v1", ctypes.c_void_p), ("n1", ctypes.c_int64),
                ("r2", ctypes.c_void_p), ("c2", ctypes.c_void_p), ("v2", ctypes.c_void_p), ("n2", ctypes.c_int64),
                ("r3", ctypes.c_void_p), ("c3", ctypes.c_void_p), ("v3", ctypes.c_void_p), ("n3", ctypes.c_int64)]


_lib.OTHER_DECLARED.update({"oec_grid_geometry", "oec_point_in_polygon", "oec_polygon_prepare"})


def _declare():
    L = _lib.lib()
    if not getattr(L, "_geom_declared", False):
        L.oec_grid_geometry.restype = ctypes.c_int
        L.oec_grid_geometry.argtypes = [ctypes.POINTER(GeomIn), ctypes.POINTER(GeomOut)]
        L.oec_point_in_polygon.restype = ctypes.c_int
        L.oec_point_in_polygon.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_double, ctypes.c_double]
        L.oec_polygon_prepare.restype = ctypes.c_int
        L.oec_polygon_prepare.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p,
                                          ctypes.POINTER(ctypes.c_int32)]
        L._geom_declared = True
    return L


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def prepare_polygon(points):
    """grid.pyx:123-159 (drop collinear vertices)."""
    L = _declare()
    pts = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 2)
    out = np.empty_like(pts)
    m = ctypes.c_int32(0)
    rc = L.oec_polygon_prepare(_p(pts), pts.shape[0], _p(out), ctypes.byref(m))
    if rc:
        raise _lib.OecError("oec_polygon_prepare", rc)
    return out[:m.value].copy()


def point_in_polygon(grid, x, y):
    L = _declare()
    if getattr(grid, "_poly", None) is None:
        grid._poly = prepare_polygon(grid.boundFuncPoints)
    return int(L.oec_point_in_polygon(_p(grid._poly), grid._poly.shape[0], float(x), float(y)))


def compute(grid):
    """All geometry arrays of `grid` as a dict of numpy arrays (+ edgeToNode)."""
    L = _declare()
    nx, ny, G = grid.nxExt, grid.nyExt, grid.npExt
    gin = GeomIn()
    gin.nx, gin.ny, gin.dx, gin.dy = nx, ny, grid.dx, grid.dy
    xm = np.ascontiguousarray(grid.xMesh, np.float64)
    ym = np.ascontiguousarray(grid.yMesh, np.float64)
    gin.x_mesh, gin.y_mesh = _p(xm).value, _p(ym).value
    gin.scan_around_point = grid.scanAroundPoint
    gin.cut_cell_acc = grid.cutCellAcc
    bt = grid.boundType
    gin.cut_cell = 0 if bt in (0, 2) else 1
    keep = [xm, ym]
    cb = None
    if bt == 0:
        gin.bound_kind, gin.p0, gin.p1 = BOUND_RECT, grid.lx * 0.5, grid.ly * 0.5
    elif bt == 1:
        gin.bound_kind, gin.p0, gin.p1 = BOUND_ELLIPSE, 4. / grid.lx ** 2, 4. / grid.ly ** 2
    elif bt == 4:
        poly = prepare_polygon(grid.boundFuncPoints)
        grid._poly = poly
        keep.append(poly)
        gin.bound_kind, gin.poly, gin.n_poly = BOUND_POLYGON, _p(poly).value, poly.shape[0]
    else:
        f = grid.boundFunc

        def _call(x, y, ctx):
            return 1 if f(x, y) else 0
        cb = _CB(_call)
        gin.bound_kind, gin.fn = BOUND_CALLBACK, cb
    out = {
        "insidePoints": np.zeros(G, np.uint16), "insideEdges": np.zeros(2 * G, np.uint16),
        "insideFaces": np.zeros(G, np.uint16),
        "ds": np.zeros(2 * G), "dsi": np.zeros(2 * G), "da": np.zeros(G), "dai": np.zeros(G),
        "dst": np.zeros(2 * G), "dsti": np.zeros(2 * G), "dat": np.zeros(G), "dati": np.zeros(G),
        "boundaryPoints": np.zeros((2 * G, 2)), "boundaryPointsInd": np.zeros(2 * G, np.uint32),
        "cutCellPointsInd": np.zeros((G, 2), np.int32), "cutCellCenter": np.zeros((G, 2)),
        "cutCellNormalVectors": np.zeros((G, 2)),
    }
    cap = 8 * G
    coo = [(np.zeros(cap, np.int32), np.zeros(cap, np.int32), np.zeros(cap)) for _ in range(3)]
    go = GeomOut()
    for k, n in [("inside_points", "insidePoints"), ("inside_edges", "insideEdges"), ("inside_faces", "insideFaces"),
                 ("ds", "ds"), ("dsi", "dsi"), ("da", "da"), ("dai", "dai"), ("dst", "dst"), ("dsti", "dsti"),
                 ("dat", "dat"), ("dati", "dati"), ("boundary_points", "boundaryPoints"),
                 ("boundary_points_ind", "boundaryPointsInd"), ("cut_cell_points_ind", "cutCellPointsInd"),
                 ("cut_cell_center", "cutCellCenter"), ("cut_cell_normals", "cutCellNormalVectors")]:
        setattr(go, k, _p(out[n]).value)
    go.cap_boundary_points = 2 * G
    go.cap_coo = cap
    for s, (r, c, v) in zip("123", coo):
        setattr(go, "r" + s, _p(r).value)
        setattr(go, "c" + s, _p(c).value)
        setattr(go, "v" + s, _p(v).value)
    rc = L.oec_grid_geometry(ctypes.byref(gin), ctypes.byref(go))
    del keep, cb
    if rc:
        raise _lib.OecError("oec_grid_geometry", rc)
    nb = go.n_boundary_points
    out["boundaryPoints"] = out["boundaryPoints"][:nb].copy()
    out["boundaryPointsInd"] = out["boundaryPointsInd"][:nb].copy()
    shape = (2 * G, 2 * G)
    stages = []
    for (r, c, v), n in zip(coo, (go.n1, go.n2, go.n3)):
        if n < 0:
            stages.append(None)
            continue
        stages.append(spsp.csc_matrix(spsp.coo_matrix((v[:n], (r[:n].astype(np.int64), c[:n].astype(np.int64))),
                                                      shape=shape)))
    e2n = stages[0]
    e2n = stages[1].dot(e2n)
    if stages[2] is not None:
        e2n = stages[2].dot(e2n)
    out["edgeToNode"] = e2n
    return out
