"""GPU Poisson solve (LU back-substitution + phiToE) against the reference.

phi: relative residual ||A phi - q|| / ||q|| <= 1e-8 on the inside nodes and
agreement with the reference's phi and E (golden vectors) to 1e-9 norm-wise.
"""
import numpy as np
import pytest

from conftest import golden, rel_err

GRIDS = ["rect_24x20", "circle_32", "ellipse_40x24", "circle_128"]


def _grid(z):
    from openecloud_b200.grid import Grid
    nx, ny, lx, ly, bt = z["params"]
    return Grid(int(nx), int(ny), lx, ly, int(bt))


@pytest.mark.gpu
@pytest.mark.parametrize("name", GRIDS)
@pytest.mark.parametrize("tail", [None, 0, 10 ** 9])
def test_lu_solve_matches_reference(gpu, name, tail):
    from openecloud_b200.poissonSolver import PoissonSolver
    z = golden(f"grid_{name}.npz")
    g = _grid(z)
    ps = PoissonSolver(g, tail=tail)
    q = z["poisson_q"]
    E = ps.solve(q)
    phi = ps.getPhi()
    ins = ps.insidePointsInd
    res = ps.systemMatrix.dot(phi[ins]) - q[ins]
    assert np.linalg.norm(res) / np.linalg.norm(q[ins]) <= 1e-8
    assert rel_err(phi, z["poisson_phi"]) <= 1e-9
    assert rel_err(E, z["poisson_E"]) <= 1e-9
    outside = np.setdiff1d(np.arange(g.getNpExt()), ins)
    assert np.all(phi[outside] == 0.0)


def test_trsv_levels_host():
    """oec_trsv_levels against a direct Python recurrence."""
    import scipy.sparse as spsp
    from openecloud_b200.poissonSolver import _levels
    rng = np.random.default_rng(3)
    n = 300
    A = spsp.random(n, n, density=0.02, random_state=4, format="csr") + spsp.eye(n)
    for lower in (True, False):
        T = (spsp.tril(A) if lower else spsp.triu(A)).tocsr()
        T.sort_indices()
        lev, nl = _levels(T, lower, n)
        ref = np.zeros(n, np.int64)
        order = range(n) if lower else range(n - 1, -1, -1)
        for r in order:
            cols = T.indices[T.indptr[r]:T.indptr[r + 1]]
            cols = cols[cols < r] if lower else cols[cols > r]
            ref[r] = 1 + (ref[cols].max() if len(cols) else 0)
        assert np.array_equal(lev, ref) and nl == ref.max()


@pytest.mark.gpu
@pytest.mark.parametrize("N,tail", [(128, 3072), (128, 2048), (128, 1024), (256, 8192), (256, 3072)])
def test_lu_head_paths_match_host_factor(gpu, N, tail):
    """Every way of running the head levels -- one CTA with the vector in
    shared memory (<= 28672 unknowns and <= 64 levels), one cooperative launch
    (<= 64 levels), one launch per level; a path that does not fit falls back
    -- agrees with the host solve of the same SuperLU factors.  128^2 has 12644
    unknowns (20 / 31 / 75 levels at tails 3072 / 2048 / 1024), 256^2 51040
    (37 / 114 levels at tails 8192 / 3072)."""
    from openecloud_b200.grid import Grid
    from openecloud_b200.poissonSolver import PoissonSolver
    g = Grid(N, N, 0.04, 0.04, 1)
    ps = PoissonSolver(g, tail=tail)
    ins = ps.insidePointsInd
    q = np.zeros(g.getNpExt())
    q[ins] = np.random.default_rng(N + tail).normal(size=ins.size) * 1e-9
    ref = ps.ludecom.solve(q[ins])
    for path in (1, 2, 3, 0):
        ps._lu_t.head_path = path
        ps.solve(q)
        phi = ps.getPhi()
        err = np.linalg.norm(phi[ins] - ref) / np.linalg.norm(ref)
        res = np.linalg.norm(ps.systemMatrix.dot(phi[ins]) - q[ins]) / np.linalg.norm(q[ins])
        assert err <= 1e-9 and res <= 1e-8, (path, ps.levels, err, res)


def test_lu_head_path_field_is_last():
    """oec_lu_t.head_path (C) sits after tu_inv, as the ctypes mirror has it."""
    from openecloud_b200.poissonSolver import LU_t
    assert LU_t._fields_[-1] == ("head_path", __import__("ctypes").c_int32)
    assert LU_t.head_path.offset == LU_t.tu_inv.offset + 8
