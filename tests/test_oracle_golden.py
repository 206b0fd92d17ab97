"""The CPU oracle against golden vectors produced by the compiled reference."""
import numpy as np
import pytest

from conftest import golden
from oracle import oracle as O

GRIDS = ["rect_24x20", "circle_32", "ellipse_40x24"]
QE = -1.602176565e-19
QM = -1.602176565e-19 / 9.10938291e-31


def _grid(z):
    nx, ny, lx, ly, bt = z["params"]
    return O.GridGeom(nx, ny, lx, ly), int(bt)


@pytest.mark.parametrize("name", GRIDS)
def test_weights_deposit_gather_push(name):
    z = golden(f"grid_{name}.npz")
    g, _ = _grid(z)
    pd = z["pd_in"]
    inc, w = O.calc_grid_weights(pd, g)
    assert np.array_equal(inc, z["inCell"])
    for a, k in zip(w, ["w00", "w10", "w01", "w11"]):
        assert np.array_equal(a, z[k])
    assert np.array_equal(O.charge_to_grid(pd, g, QE), z["chargeOnGrid"])
    e = O.field_to_particles(pd, g, z["poisson_E"], 2)
    b = O.field_to_particles(pd, g, z["B_nodes"], 3)
    assert np.array_equal(e, z["eAtParticles"])
    assert np.array_equal(b, z["bAtParticles"])
    for tb in range(3):
        out = O.boris_push(pd, e, z["push_dt"], QM, tb, b_at=b, bconst=z["bconst"])
        assert np.array_equal(out, z[f"push{tb}"]), tb


@pytest.mark.parametrize("name", GRIDS)
def test_boundary_absorb_interaction_normals(name):
    z = golden(f"grid_{name}.npz")
    g, bt = _grid(z)
    geom = {k: z[k] for k in ["insideFaces", "boundaryPoints", "cutCellPointsInd", "cutCellNormalVectors"]
            if k in z}
    for tag in (["rect"] if bt == 0 else ["ell", "cc"]):
        kind = {"rect": 0, "ell": 1, "cc": 2}[tag]
        ins, moved = O.index_inside(z[f"{tag}_moved"], g, kind, geom)
        assert np.array_equal(ins, z[f"{tag}_isInside"])
        ab = O.save_absorbed(moved, ins)
        assert np.array_equal(ab, z[f"{tag}_absorbed"])
        assert 0 < len(ab) < len(moved)
        wall, nrm, miss = O.interaction(ab, g, kind, dt=z["bnd_dt"], geom=geom)
        assert miss == 0
        assert np.array_equal(wall, z[f"{tag}_wall"])
        assert np.array_equal(nrm, z[f"{tag}_normals"])


def test_clip_to_grid_edge_cases():
    pd = np.array([[1.0, -1.0, 0, 0, 0, 1], [0.0, 0.0, 0, 0, 0, 1], [-2.0, 3.0, 0, 0, 0, 1]], np.float64)
    lib = O.lib()
    import ctypes
    flag = lib.orc_clip_to_grid(pd.ctypes.data_as(ctypes.c_void_p), 3, 0.5, 0.25)
    assert flag == 1
    assert np.array_equal(pd[:, :2], [[0.5, -0.25], [0.0, 0.0], [-0.5, 0.25]])
