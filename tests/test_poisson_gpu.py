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
@pytest.mark.parametrize("N,tail", [(128, 3072), (128, 2048), (128, 1024), (256, 8192), (256, 3072), (512, 8192)])
def test_lu_head_paths_match_host_factor(gpu, N, tail):
    """Every way of running the head levels -- one CTA with the vector in
    shared memory (<= 28672 unknowns and <= 64 levels), one cooperative launch
    (<= 64 levels), one launch per level; a path that does not fit falls back
    -- agrees with the host solve of the same SuperLU factors.  128^2 has 12644
    unknowns (20 / 31 / 75 levels at tails 3072 / 2048 / 1024), 256^2 51040
    (37 / 114 levels at tails 8192 / 3072), 512^2 205012 (231 levels at tail
    8192: one-CTA runs between per-level launches)."""
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


@pytest.mark.gpu
def test_lu_invalid_head_path_is_rejected(gpu):
    """An unknown head_path is an argument error before any launch; the
    solver works again once it is valid."""
    from openecloud_b200 import _lib
    from openecloud_b200.poissonSolver import PoissonSolver
    z = golden("grid_circle_32.npz")
    ps = PoissonSolver(_grid(z))
    q = z["poisson_q"]
    ps._lu_t.head_path = 7
    with pytest.raises(_lib.OecError):
        ps.solve(q)
    ps._lu_t.head_path = 0
    ps.solve(q)
    assert rel_err(ps.getPhi(), z["poisson_phi"]) <= 1e-9


def test_lu_struct_tail_layout():
    """The last fields of oec_lu_t (C): tu_inv, head_path, l_level_lanes,
    u_level_lanes, at the offsets the ctypes mirror has."""
    import ctypes
    from openecloud_b200.poissonSolver import LU_t
    assert [f[0] for f in LU_t._fields_[-4:]] == ["tu_inv", "head_path", "l_level_lanes", "u_level_lanes"]
    assert LU_t.head_path.offset == LU_t.tu_inv.offset + 8
    assert LU_t.l_level_lanes.offset == LU_t.head_path.offset + 8  # int32 then 4 bytes of padding
    assert LU_t.u_level_lanes.offset == LU_t.l_level_lanes.offset + 8
    assert ctypes.sizeof(LU_t) == LU_t.u_level_lanes.offset + 8


def test_choose_tail_minimises_the_model():
    """choose_tail on the 128^2 circle's factors: among its candidates
    (at most n/4 rows and 16384), the tail with the lowest
    levels * 8 us + 2 m^2 * 8 B / 6000 GB/s, computed here from the level
    counts of oec_trsv_levels."""
    from scipy.sparse.linalg import splu
    from openecloud_b200.grid import Grid
    from openecloud_b200.poissonSolver import _levels, assemble, choose_tail
    a, _, _, _ = assemble(Grid(128, 128, 0.04, 0.04, 1))
    lu = splu(a, permc_spec="MMD_AT_PLUS_A", diag_pivot_thresh=0.1)
    n = lu.shape[0]
    Lc, Uc = lu.L.tocsr(), lu.U.tocsr()
    Lc.sort_indices()
    Uc.sort_indices()
    m = choose_tail(Lc, Uc, n)
    assert 0 < m <= min(n // 4, 16384)

    def model(t):
        h = n - t
        return ((_levels(Lc, True, h, nrows=h)[1] + _levels(Uc, False, h, nrows=h)[1]) * 8e-6 +
                2 * t * t * 8 / 6000e9)
    for t in (0, 1024, 2048, 3072):
        if t <= n // 4:
            assert model(m) <= model(t) + 1e-12, (m, t)
    assert m == 3072  # the measured optimum of this grid (0.15 ms; 2048: 0.18, 4096: 0.16)


def test_level_ordered_head_solve_host():
    """The setup's layout, replayed on the host: the strict-lower and
    strict-upper head rows of the 128^2 factors, reordered by dependency
    level, solved level by level through the reordered CSR (row w holds
    factor row rows[w]; L's first level skipped) equal the triangular solves
    of scipy on the head block."""
    import scipy.sparse as spsp
    from scipy.sparse.linalg import spsolve_triangular, splu
    from openecloud_b200.grid import Grid
    from openecloud_b200.poissonSolver import _level_lists, _levels, assemble
    a, _, _, _ = assemble(Grid(128, 128, 0.04, 0.04, 1))
    lu = splu(a, permc_spec="MMD_AT_PLUS_A", diag_pivot_thresh=0.1)
    n = lu.shape[0]
    h = n - 3072
    Lc, Uc = lu.L.tocsr(), lu.U.tocsr()
    rng = np.random.default_rng(5)
    for lower in (True, False):
        T = spsp.tril(Lc[:h, :h], k=-1, format="csr") if lower else spsp.triu(Uc[:h, :h], k=1, format="csr")
        T.sort_indices()
        diag = np.ones(h) if lower else Uc.diagonal()[:h]
        lev, nl = _levels(T, lower, h)
        rows, lptr = _level_lists(lev, nl)
        Tw = T[rows]  # level order
        dw = diag[rows]
        b = rng.normal(size=h)
        x = b.copy()
        first = 1 if lower else 0
        if lower:
            assert np.diff(Tw.indptr)[lptr[0]:lptr[1]].sum() == 0  # L's first level has no entries
        for l in range(first, nl):
            w = np.arange(lptr[l], lptr[l + 1])
            r = rows[w]
            sums = np.array([Tw.data[Tw.indptr[k]:Tw.indptr[k + 1]] @ x[Tw.indices[Tw.indptr[k]:Tw.indptr[k + 1]]]
                             for k in w])
            x[r] = (x[r] - sums) / dw[w]
        full = (T + spsp.diags(diag)).tocsr()
        ref = spsolve_triangular(full, b, lower=lower)
        assert np.linalg.norm(x - ref) <= 1e-12 * np.linalg.norm(ref), lower


def test_level_lanes_rule():
    """level_lanes: one pass of 1024 threads (rows * lanes <= 1024, lanes a
    power of two up to 32) and at most 16 loads per lane, else 0."""
    import scipy.sparse as spsp
    from openecloud_b200.poissonSolver import level_lanes
    # levels: 1 row of 40 entries, 3 rows of 2, 1500 rows of 1, 300 rows of 20, 20 rows of 600
    lens = [40] + [2] * 3 + [1] * 1500 + [20] * 300 + [600] * 20
    indptr = np.concatenate([[0], np.cumsum(lens)])
    csr = spsp.csr_matrix((np.ones(indptr[-1]), np.zeros(indptr[-1], np.int32), indptr), shape=(len(lens), 1))
    lptr = np.cumsum([0, 1, 3, 1500, 300, 20])
    assert level_lanes(csr, lptr).tolist() == [32, 32, 0, 2, 0]
