"""Host grid geometry (grid_geom.cpp) against the reference's golden arrays."""
import numpy as np
import pytest

from conftest import golden

GRIDS = ["rect_24x20", "circle_32", "ellipse_40x24", "circle_128"]
ARRAYS = ["insidePoints", "insideEdges", "insideFaces", "Ds", "Dsi", "Dst", "Da", "Dai", "Dat", "Dati"]


def _grid(z):
    from openecloud_b200.grid import Grid
    nx, ny, lx, ly, bt = z["params"]
    return Grid(int(nx), int(ny), lx, ly, int(bt))


@pytest.mark.parametrize("name", GRIDS)
def test_geometry_arrays_bit_exact(name):
    z = golden(f"grid_{name}.npz")
    g = _grid(z)
    assert np.array_equal(g.getXMesh(), z["XMesh"]) and np.array_equal(g.getYMesh(), z["YMesh"])
    for a in ARRAYS:
        mine = np.asarray(getattr(g, "get" + a[0].upper() + a[1:])())
        assert mine.shape == z[a].shape, a
        assert np.array_equal(mine, z[a]), a
    if "boundaryPoints" in z:
        assert np.array_equal(g.getBoundaryPoints(), z["boundaryPoints"])
        assert np.array_equal(g.getBoundaryPointsInd(), z["boundaryPointsInd"])
        assert np.array_equal(g.getCutCellPointsInd(), z["cutCellPointsInd"])
        assert np.array_equal(g.getCutCellCenter(), z["cutCellCenter"])
        assert np.array_equal(g.getCutCellNormalVectors(), z["cutCellNormalVectors"])


@pytest.mark.parametrize("name", GRIDS)
def test_edge_to_node_matches(name):
    z = golden(f"grid_{name}.npz")
    g = _grid(z)
    e = g.getEdgeToNode().tocsr()
    e.sort_indices()
    ref = __import__("scipy.sparse", fromlist=["csr_matrix"]).csr_matrix(
        (z["e2n_data"], z["e2n_indices"], z["e2n_indptr"]), shape=e.shape)
    d = (e - ref)
    assert d.nnz == 0 or np.max(np.abs(d.data)) == 0.0


def test_user_boundfunc_matches_builtin_ellipse():
    """A Python boundFunc (boundType 3) gives the built-in ellipse geometry."""
    from openecloud_b200.grid import Grid
    a = Grid(40, 24, 0.09, 0.036, 1)
    ax, by = 4. / 0.09 ** 2, 4. / 0.036 ** 2
    b = Grid(40, 24, 0.09, 0.036, 3, boundFunc=lambda x, y: 1 if 1 > x ** 2 * ax + y ** 2 * by else 0)
    for k in ["insidePoints", "Ds", "BoundaryPoints", "CutCellNormalVectors"]:
        assert np.array_equal(getattr(a, "get" + k[0].upper() + k[1:])(), getattr(b, "get" + k[0].upper() + k[1:])())


def test_polygon_boundary():
    """boundType 4: a quadrant polygon (the circle's first quadrant)."""
    from openecloud_b200.grid import Grid
    t = np.linspace(0, np.pi / 2, 60)
    poly = np.stack([0.02 * np.cos(t), 0.02 * np.sin(t)], 1)
    poly = np.concatenate([[[0.0, 0.0]], poly, [[0.0, 0.0]]])
    g = Grid(32, 32, 0.04, 0.04, 4, boundFunc=poly)
    assert g.pointInPolygon(0.0, 0.0) == 1 and g.pointInPolygon(0.03, 0.0) == 0
    assert g.pointInPolygon(-0.01, -0.01) == 1
    ref = Grid(32, 32, 0.04, 0.04, 1)
    agree = np.mean(g.getInsidePoints() == ref.getInsidePoints())
    assert agree > 0.97
