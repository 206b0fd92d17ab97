"""Iterative Poisson solve: the matrix-free operator and the PCG solve.

CPU: the edge-weight stencil (oec_stencil_t layout) reproduces the
reference's assembled system matrix A = S diag(meps) S^T
(poissonSolver.pyx:41-58) on rectangular, circular, elliptical and
polygon cut-cell grids.

GPU (through the C ABI): oec_stencil_apply equals A x in f64; oec_pcg_solve
reaches the f64 relative residual 1e-8 with and without the Jacobi
preconditioner and agrees with the LU solve (the judge) and with the
reference's phi; a warm start from a nearby solution cuts the iterations; an
iteration cap too small to converge makes solveDevice fall back to the LU
result.
"""
import numpy as np
import pytest

from conftest import golden, rel_err

HOST_GRIDS = [(64, 64, 0.04, 0.04, 1), (40, 30, 0.04, 0.03, 0), (48, 48, 0.09, 0.036, 1), (33, 47, 0.05, 0.07, 1)]


@pytest.mark.parametrize("args", HOST_GRIDS)
def test_stencil_equals_assembled_matrix(args):
    from openecloud_b200.grid import Grid
    from openecloud_b200.poissonSolver import assemble, stencil_apply_host
    g = Grid(*args)
    a, meps, _, ins = assemble(g)
    mask = np.asarray(g.getInsidePoints()) != 0
    x = np.random.default_rng(1).normal(size=g.getNpExt())
    y = stencil_apply_host(meps, mask, g.getNxExt(), x)
    ref = np.zeros(g.getNpExt())
    ref[ins] = a @ x[ins]
    assert np.max(np.abs(y - ref)) <= 1e-13 * np.max(np.abs(ref))
    assert np.all(y[~mask] == 0.0)


def test_stencil_on_polygon_cut_cell_grid():
    from openecloud_b200.grid import Grid
    from openecloud_b200.poissonSolver import assemble, stencil_apply_host
    poly = np.array([[-0.02, -0.015], [0.02, -0.015], [0.025, 0.0], [0.0, 0.02], [-0.025, 0.0]])
    g = Grid(48, 40, 0.06, 0.05, 4, boundFunc=poly) if _supports_polygon() else Grid(48, 40, 0.06, 0.05, 1)
    a, meps, _, ins = assemble(g)
    mask = np.asarray(g.getInsidePoints()) != 0
    x = np.random.default_rng(2).normal(size=g.getNpExt())
    y = stencil_apply_host(meps, mask, g.getNxExt(), x)
    ref = np.zeros(g.getNpExt())
    ref[ins] = a @ x[ins]
    assert np.max(np.abs(y - ref)) <= 1e-13 * np.max(np.abs(ref))


def _level_matrix(ex, ey, lk, inside, nx, ny):
    """Sparse operator of a multigrid level over all its nodes (rows and
    columns of outside nodes empty): leak + incident edge weights on the
    diagonal, -w between inside neighbours."""
    import scipy.sparse as spsp
    n = nx * ny
    ins = np.asarray(inside, bool)
    j, i = np.divmod(np.arange(n), nx)
    d = np.array(lk, dtype=float)
    rows, cols, vals = [], [], []
    for w, step, valid in ((ex, 1, i < nx - 1), (ey, nx, j < ny - 1)):
        a = np.nonzero(valid)[0]
        b = a + step
        d[a] += w[a]
        d[b] += w[a]
        both = ins[a] & ins[b]
        rows += [a[both], b[both]]
        cols += [b[both], a[both]]
        vals += [-w[a][both], -w[a][both]]
    d = np.where(ins, d, 0.0)
    rows.append(np.arange(n))
    cols.append(np.arange(n))
    vals.append(d)
    return spsp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n, n))


@pytest.mark.parametrize("args", HOST_GRIDS)
def test_mg_coarse_level_is_directional_galerkin_product(args):
    """Each coarse multigrid level splits by direction into
    P^T A_x P / fx + P^T A_y P / fy (piecewise-constant P over fx x fy
    aggregates; level 0 = the assembled matrix), three levels down; on the
    anisotropic ellipse the first steps coarsen along y only."""
    import scipy.sparse as spsp
    from openecloud_b200.grid import Grid
    from openecloud_b200.poissonSolver import assemble, mg_coarsen, mg_factors
    from oracle.mg_oracle import parent
    g = Grid(*args)
    a, meps, _, ins = assemble(g)
    nx, ny = g.getNxExt(), g.getNyExt()
    n = nx * ny
    mask = np.asarray(g.getInsidePoints()) != 0
    ex, ey, z = meps[:n], meps[n:], np.zeros(n)
    Ax, Ay = _level_matrix(ex, z, z, mask, nx, ny), _level_matrix(z, ey, z, mask, nx, ny)
    A = (Ax + Ay).tocsr()[ins][:, ins]
    assert abs(A - a).max() <= 1e-12 * abs(a).max()
    cur = (ex, ey, z, z, mask, nx, ny)
    factors = []
    for _ in range(3):
        fx, fy = mg_factors(cur[0], cur[1], cur[4], cur[5], cur[6])
        factors.append((fx, fy))
        nxt = mg_coarsen(*cur, fx, fy)
        NX, NY = nxt[5], nxt[6]
        P = spsp.csr_matrix((np.ones(cur[5] * cur[6]), (np.arange(cur[5] * cur[6]), parent(cur[5], cur[6], NX, NY))),
                            shape=(cur[5] * cur[6], NX * NY))
        Ax, Ay = (P.T @ Ax @ P) / fx, (P.T @ Ay @ P) / fy
        zc = np.zeros(NX * NY)
        for got, want in ((_level_matrix(nxt[0], zc, nxt[2], nxt[4], NX, NY, ), Ax),
                          (_level_matrix(zc, nxt[1], nxt[3], nxt[4], NX, NY), Ay)):
            assert abs(got - want).max() <= 1e-12 * abs(want).max()
        assert np.all(nxt[4] == (np.asarray(P.T @ cur[4].astype(float)) > 0))
        cur = nxt
    if args[2] / args[0] > 2 * args[3] / args[1]:  # cells wider than tall: strong y coupling
        assert factors[0] == (1, 2)
    elif args[0] == args[1] and args[2] == args[3]:
        assert factors == [(2, 2)] * 3


def test_mg_hierarchy_layout():
    """Level sizes halve (rounded up) down to at most 100 nodes; the block
    level is the first of at most MG_BLOCK_TOP nodes from which the coarser
    levels fit the one-CTA shared-memory solve (3 floats per node at least,
    226 KB), at most 8 levels."""
    from openecloud_b200.poissonSolver import mg_hierarchy, MG_BLOCK_SMEM, MG_BLOCK_TOP, MG_FLOATS_PER_NODE
    for nx, ny in ((1026, 1026), (130, 130), (66, 66), (26, 22), (515, 130)):
        yy, xx = np.mgrid[0:ny, 0:nx]
        inside = ((xx - nx / 2) / (nx / 2 - 1.5)) ** 2 + ((yy - ny / 2) / (ny / 2 - 1.5)) ** 2 < 1
        lv, block = mg_hierarchy(np.ones(nx * ny), np.ones(nx * ny), inside.ravel(), nx, ny)
        sizes = [(l[4], l[5]) for l in lv]
        for (a, b), (c, d) in zip(sizes, sizes[1:]):  # isotropic weights: both directions halve
            assert (c, d) == ((a + 1) // 2, (b + 1) // 2)
        assert sizes[-1][0] * sizes[-1][1] <= 100 and (len(sizes) == 1 or sizes[-2][0] * sizes[-2][1] > 100)
        smem = lambda k: 4 * MG_FLOATS_PER_NODE * sum(a * b for a, b in sizes[k:])  # noqa: E731
        top = lambda k: sizes[k][0] * sizes[k][1]  # noqa: E731
        assert smem(block) <= MG_BLOCK_SMEM and len(sizes) - block <= 8 and top(block) <= max(MG_BLOCK_TOP, 100)
        assert block == 0 or smem(block - 1) > MG_BLOCK_SMEM or len(sizes) - block + 1 > 8 or \
            top(block - 1) > MG_BLOCK_TOP


def _supports_polygon():
    import inspect
    from openecloud_b200.grid import Grid
    return "boundFunc" in inspect.signature(Grid.__init__).parameters


def _grid(z):
    from openecloud_b200.grid import Grid
    nx, ny, lx, ly, bt = z["params"]
    return Grid(int(nx), int(ny), lx, ly, int(bt))


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["rect_24x20", "circle_32", "ellipse_40x24", "circle_128"])
def test_stencil_apply_device(gpu, name):
    import torch
    from openecloud_b200 import device as D
    from openecloud_b200.poissonSolver import PoissonSolver
    z = golden(f"grid_{name}.npz")
    ps = PoissonSolver(_grid(z))
    x = np.random.default_rng(3).normal(size=ps.n_nodes)
    y = D.to_numpy(ps.applyOperator(D.to_device(x, torch.float64)))
    ins = ps.insidePointsInd
    ref = np.zeros(ps.n_nodes)
    ref[ins] = ps.systemMatrix @ x[ins]
    assert np.max(np.abs(y - ref)) <= 1e-13 * np.max(np.abs(ref))


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["rect_24x20", "circle_32", "ellipse_40x24", "circle_128"])
@pytest.mark.parametrize("precond", ["none", "jacobi", "mg"])
def test_pcg_matches_lu_and_reference(gpu, name, precond):
    from openecloud_b200.poissonSolver import PoissonSolver
    z = golden(f"grid_{name}.npz")
    q = z["poisson_q"]
    ps = PoissonSolver(_grid(z), method="pcg", precond=precond, pcgTol=1e-8, pcgMaxIter=20000)
    E = ps.solve(q)
    st = ps.lastStats
    assert st.converged == 1 and st.rel_residual <= 1e-8 and ps.nFallbacks == 0, (st.rel_residual, st.iterations)
    phi = ps.getPhi()
    ins = ps.insidePointsInd
    res = ps.systemMatrix.dot(phi[ins]) - q[ins]
    assert np.linalg.norm(res) / np.linalg.norm(q[ins]) <= 1.5e-8
    # the LU solve is the judge: phi within what a 1e-8 residual allows
    lu = PoissonSolver(_grid(z))
    lu.solve(q)
    assert rel_err(phi, lu.getPhi()) <= 1e-6
    assert rel_err(phi, z["poisson_phi"]) <= 1e-6
    assert rel_err(E, z["poisson_E"]) <= 1e-6


@pytest.mark.gpu
def test_pcg_warm_start_and_fallback(gpu):
    import torch
    from openecloud_b200 import device as D
    from openecloud_b200.poissonSolver import PoissonSolver
    z = golden("grid_circle_128.npz")
    q = z["poisson_q"]
    ps = PoissonSolver(_grid(z), method="pcg", precond="jacobi", pcgTol=1e-8, pcgMaxIter=20000)
    ps.solve(q)
    cold = ps.lastStats.iterations
    # a smooth 0.1 % change of the charge (as between time steps), solved
    # from the previous phi
    ins = ps.insidePointsInd
    x = np.linspace(0.0, 1.0, q.shape[0])
    q2 = q * (1.0 + 1e-3 * np.sin(2 * np.pi * x))
    ps.solve(q2)
    warm = ps.lastStats
    assert warm.converged == 1 and warm.iterations < cold, (warm.iterations, cold)
    assert warm.rel_residual0 < 0.01
    # cap the iterations: the solve misses tolerance and falls back to LU
    ps2 = PoissonSolver(_grid(z), method="pcg", precond="jacobi", pcgTol=1e-8, pcgMaxIter=3)
    E = ps2.solve(q)
    assert ps2.lastStats.converged == 0 and ps2.nFallbacks == 1
    lu = PoissonSolver(_grid(z))
    assert rel_err(E, lu.solve(q)) <= 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("cluster_top", [0, 4000, 1 << 30])
@pytest.mark.parametrize("name", ["rect_24x20", "ellipse_40x24", "circle_128"])
def test_mg_vcycle_matches_oracle(gpu, name, cluster_top):
    """oec_mg_apply (f32) equals the float64 restatement of the V-cycle on the
    device's own f32 level weights.  cluster_top 0: the small grids run every
    level in the one-CTA solve, the 128 circle its finest level in the tiled
    kernels; 4000: the coarse levels in the one-cluster solve; 2^30: every
    level in the one-cluster solve."""
    import ctypes
    import torch
    from openecloud_b200 import device as D
    from openecloud_b200.poissonSolver import PoissonSolver, _declare
    from oracle.mg_oracle import vcycle
    z = golden(f"grid_{name}.npz")
    ps = PoissonSolver(_grid(z), method="pcg", precond="mg")
    mg = ps._mg_setup(cluster_top=cluster_top)
    host = mg["host"]
    dinv = [D.to_numpy(k["dinv"]).astype(np.float64) for k in mg["keep"]]
    assert mg["nlevels"] >= 2 and host[-1][4] * host[-1][5] <= 100
    ins = host[0][3]
    r = np.where(ins, np.random.default_rng(5).normal(size=ins.size), 0.0).astype(np.float32)
    rd = D.to_device(r, torch.float32)
    zd = D.zeros(r.size, torch.float32)
    rc = _declare().oec_mg_apply(ctypes.byref(mg["c"]), rd.data_ptr(), zd.data_ptr(), D.stream())
    assert rc == 0
    got = D.to_numpy(zd).astype(np.float64)
    want = vcycle(host, r.astype(np.float64), omega=mg["c"].omega, scale=mg["c"].scale, dinv=dinv)
    assert np.all(got[~ins] == 0.0)
    assert np.max(np.abs(got - want)) <= 2e-4 * np.max(np.abs(want))


@pytest.mark.gpu
def test_mg_pcg_iterations(gpu):
    """One V-cycle per iteration cuts the iteration count of the 128x128
    circle by well over 5x against Jacobi, to the same 1e-8 residual; the
    V-cycle in one CTA (cluster_top 0) and wholly in one cluster (its CG dot
    products included) take the same iterations and solution."""
    from openecloud_b200.poissonSolver import PoissonSolver
    z = golden("grid_circle_128.npz")
    q = z["poisson_q"]
    its, phis = {}, {}
    for pc, ct in (("jacobi", None), ("mg", 0), ("mg", 1 << 30)):
        ps = PoissonSolver(_grid(z), method="pcg", precond=pc, pcgTol=1e-8, pcgMaxIter=20000)
        if ct is not None:
            ps._mg_setup(cluster_top=ct)
        ps.solve(q)
        assert ps.lastStats.converged == 1 and ps.nFallbacks == 0
        its[(pc, ct)] = ps.lastStats.iterations
        phis[(pc, ct)] = ps.getPhi()
    assert its[("mg", 0)] * 5 < its[("jacobi", None)], its
    assert abs(its[("mg", 0)] - its[("mg", 1 << 30)]) <= 1, its
    assert rel_err(phis[("mg", 0)], phis[("mg", 1 << 30)]) <= 1e-7


@pytest.mark.gpu
def test_warm_start_extrapolate_kernel(gpu):
    """oec_warm_start_extrapolate: phi <- 2 phi - prev and prev <- old phi,
    exactly (f64); with a history count, the first two calls keep phi."""
    import ctypes
    import torch
    from openecloud_b200 import device as D
    from openecloud_b200.poissonSolver import _declare
    rng = np.random.default_rng(12)
    a, b = rng.normal(size=100_003), rng.normal(size=100_003)
    phi, prev = D.to_device(a, torch.float64), D.to_device(b, torch.float64)
    L = _declare()
    assert L.oec_warm_start_extrapolate(phi.data_ptr(), prev.data_ptr(), a.size, None, D.stream()) == 0
    assert np.array_equal(D.to_numpy(phi), 2.0 * a - b) and np.array_equal(D.to_numpy(prev), a)
    assert L.oec_warm_start_extrapolate(None, prev.data_ptr(), 1, None, D.stream()) != 0
    hist = D.zeros(1, torch.int32)
    phi, prev = D.to_device(a, torch.float64), D.to_device(b, torch.float64)
    for k in range(3):
        assert L.oec_warm_start_extrapolate(phi.data_ptr(), prev.data_ptr(), a.size, hist.data_ptr(), D.stream()) == 0
        assert int(D.to_numpy(hist)[0]) == min(k + 1, 2)
        if k < 2:
            assert np.array_equal(D.to_numpy(phi), a) and np.array_equal(D.to_numpy(prev), a)
    assert np.array_equal(D.to_numpy(phi), a)  # 2a - a


@pytest.mark.gpu
def test_pcg_extrapolated_warm_start(gpu):
    """A charge that moves smoothly between solves (a Gaussian drifting by
    0.2 cell per solve): from the third solve on, the extrapolated guess
    2 phi_n-1 - phi_n-2 starts closer than the last phi, and both solves end
    at the LU solution."""
    from openecloud_b200.poissonSolver import PoissonSolver
    z = golden("grid_circle_128.npz")
    g = _grid(z)
    ins = np.asarray(g.getInsidePoints()) != 0
    nx = g.getNxExt()
    j, i = np.divmod(np.arange(g.getNpExt()), nx)

    def charge(t):
        q = np.exp(-((i - 50.0 - 0.2 * t) ** 2 + (j - 60.0) ** 2) / (2 * 8.0 ** 2)) * 1e-12
        return np.where(ins, q, 0.0)

    lu = PoissonSolver(g)
    res0 = {}
    for ws in ("previous", "extrapolate"):
        ps = PoissonSolver(g, method="pcg", precond="mg", warmStart=ws)
        r = []
        for t in range(6):
            E = ps.solve(charge(t))
            st = ps.lastStats
            assert st.converged == 1 and ps.nFallbacks == 0
            r.append(st.rel_residual0)
        assert rel_err(E, lu.solve(charge(5))) <= 1e-6
        res0[ws] = r
    for t in range(3, 6):
        assert res0["extrapolate"][t] < 0.5 * res0["previous"][t], res0


@pytest.mark.gpu
def test_pcg_synchronous_entry_point(gpu):
    """oec_pcg_solve (host statistics, one synchronisation) gives the
    asynchronous solve's result (solveDevice) to within the tolerance."""
    import ctypes
    import torch
    from openecloud_b200 import device as D
    from openecloud_b200.poissonSolver import PoissonSolver, PcgStats_t, PRECOND, _declare
    z = golden("grid_circle_128.npz")
    q = z["poisson_q"]
    ps = PoissonSolver(_grid(z), method="pcg", precond="mg", pcgTol=1e-8, pcgMaxIter=20000)
    ps.solve(q)
    a = ps.lastStats
    phi_async = ps.getPhi()
    qd = D.to_device(q, torch.float64)
    phi = D.zeros(ps.n_nodes, torch.float64)
    mg = ps._mg
    st = PcgStats_t()
    rc = _declare().oec_pcg_solve(ctypes.byref(ps._stencil), qd.data_ptr(), phi.data_ptr(), 1e-8, 20000,
                                  PRECOND["mg"], ctypes.cast(ctypes.pointer(mg["c"]), ctypes.c_void_p),
                                  ps._pcg_work.data_ptr(), ctypes.byref(st), D.stream())
    assert rc == 0
    # the dot products sum f64 atomics in arrival order: same algorithm, not
    # the same last bits
    assert st.converged == 1 and a.converged == 1 and st.rel_residual <= 1e-8
    assert abs(st.iterations - a.iterations) <= 2 and st.refinements == a.refinements
    assert np.abs(D.to_numpy(phi) - phi_async).max() <= 1e-7 * np.abs(phi_async).max()


@pytest.mark.gpu
@pytest.mark.parametrize("top,cluster_top", [(1280, 0), (9000, 0), (1280, 40000), (1280, 150000)])
def test_mg_vcycle_large_block_matches_tiled(gpu, top, cluster_top):
    """On the 512x512 ellipse (45 x 18 mm), a V-cycle whose one-CTA part
    starts at a larger level (129 x 65 nodes and coarser: the operator read
    from global memory, 3 floats per node in shared memory) equals the
    float64 restatement, as the default split does."""
    import ctypes
    import torch
    from openecloud_b200 import device as D
    from openecloud_b200.grid import Grid
    from openecloud_b200.poissonSolver import PoissonSolver, _declare
    from oracle.mg_oracle import vcycle
    ps = PoissonSolver(Grid(512, 512, 0.09, 0.036, 1), method="pcg", precond="mg")
    mg = ps._mg_setup(block_top=top, cluster_top=cluster_top)
    host = mg["host"]
    sizes = [h[4] * h[5] for h in host]
    block = mg["c"].block_level
    assert sizes[block] <= top and (top < 9000 or sizes[block] > 4608)
    dinv = [D.to_numpy(k["dinv"]).astype(np.float64) for k in mg["keep"]]
    ins = host[0][3]
    r = np.where(ins, np.random.default_rng(6).normal(size=ins.size), 0.0).astype(np.float32)
    rd = D.to_device(r, torch.float32)
    zd = D.zeros(r.size, torch.float32)
    assert _declare().oec_mg_apply(ctypes.byref(mg["c"]), rd.data_ptr(), zd.data_ptr(), D.stream()) == 0
    got = D.to_numpy(zd).astype(np.float64)
    want = vcycle(host, r.astype(np.float64), omega=mg["c"].omega, scale=mg["c"].scale, dinv=dinv)
    assert np.max(np.abs(got - want)) <= 2e-4 * np.max(np.abs(want))
