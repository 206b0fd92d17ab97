"""The oracle's particle loop against the compiled reference's, step by step.

The reference's loop (example01_basic.py:66-97: calcGridWeights,
eFieldToParticles, borisPush, indexInside, saveAbsorbed,
calculateInteractionPoint, calculateNormalVectors, generateSecondaries,
addAndRemoveParticles) in a fixed field on the 32x32 circle, 300 steps, with
and without the electrons' own field (chargeToGrid and PoissonSolver.solve
every step), made by make_golden.py --loop.  The oracle runs the same steps
from the same rows and the same MT seed: the same absorbed count, particle
count and array row count at every step (every placement rule of the refill
is taken on the way), and the same rows in the same slots, bit for bit
(checksums of every step, the rows at the end).
"""
import numpy as np
import pytest

from conftest import golden
from oracle import oracle as O
from oracle.poisson_oracle import from_golden

QE = -1.602176565e-19
QM = QE / 9.10938291e-31


def checksums(pd):
    i = np.arange(pd.shape[0], dtype=np.float64)
    return np.concatenate([pd.sum(0), [np.dot(i, pd[:, 0]), np.dot(i, pd[:, 2])]])


@pytest.mark.parametrize("fixture", ["loop_circle_32.npz", "loop_sc_circle_32.npz"])
def test_oracle_particle_loop_replays_reference(fixture):
    z = golden(fixture)
    solver = from_golden(golden("grid_circle_32.npz")) if int(z["space_charge"]) else None
    nx, ny, lx, ly, _ = z["params"]
    g = O.GridGeom(nx, ny, lx, ly)
    xm = -0.5 * g.lxExt + g.dx * np.arange(g.nx)
    ym = -0.5 * g.lyExt + g.dy * np.arange(g.ny)
    X, Y = np.meshgrid(xm, ym)
    k = float(z["k"])
    E = np.concatenate([(-k * X).reshape(-1), (-k * Y).reshape(-1)])
    f = O.furman("copper", float(z["sey"]))
    pd = z["pd0"].copy()
    array_len = pd.shape[0]
    O.seed(int(z["seed"]))
    rules = set()
    for s in range(z["counts"].shape[0]):
        field = E
        if solver is not None:
            field = solver.solve(O.charge_to_grid(pd, g, QE))[1] + E
        e = O.field_to_particles(pd, g, field, 2)
        pd = O.boris_push(pd, e, float(z["dt"]), QM, 0)
        inside, pd = O.index_inside(pd, g, 1)
        ab = O.save_absorbed(pd, inside)
        assert ab.shape[0] == z["absorbed"][s], s
        if ab.shape[0]:
            wall, normals, _ = O.interaction(ab, g, 1)
            sec = O.furman_emit(f, wall, normals, mode=0)
            n_keep = int(inside.sum())
            rules.add("remove" if not len(sec) else "new array" if n_keep + len(sec) > array_len
                      else "fill/append" if len(sec) >= ab.shape[0] else "shift")
            pd, array_len = O.add_and_remove(pd, sec, inside, array_len)
        assert pd.shape[0] == z["counts"][s], s
        assert array_len == z["array_len"][s], s
        assert np.array_equal(checksums(pd), z["checksums"][s]), s
    assert rules == {"remove", "new array", "fill/append", "shift"}, rules
    assert np.array_equal(pd, z["final"])


def test_oracle_replays_example01():
    """example01_basic.py's loop as written -- deposit, beam, solve, gather,
    push, boundary, Furman emission, refill and globalRandom every 50 steps,
    all on the one MT stream -- with 2000 macro-particles over its first
    1200 steps (the first bunch passage; make_golden.py --example01): the
    oracle replays the compiled reference bit for bit at every step."""
    z = golden("example01_circle_32.npz")
    solver = from_golden(golden("grid_circle_32.npz"))
    g = O.GridGeom(32, 32, 0.04, 0.04)
    f = O.furman("copper")
    target, dt = int(z["target"]), float(z["dt"])
    pd = z["pd0"].copy()
    array_len = pd.shape[0]
    O.seed(int(z["seed"]))
    for s in range(z["counts"].shape[0]):
        n = pd.shape[0]
        if s > 0 and s % 50 == 0 and (n > 1.05 * target or n < 0.95 * target):
            assert z["managed"][s], s
            pd = O.global_random(pd, target)
            if pd.shape[0] > n and pd.shape[0] > array_len:  # cloned rows in a new array
                array_len = int(pd.shape[0] * 1.1)
        else:
            assert not z["managed"][s], s
        q = O.charge_to_grid(pd, g, QE)
        if np.isfinite(z["beam_scale"][s]):
            q = q + z["beam_scale"][s] * z["profile"]
        e = O.field_to_particles(pd, g, solver.solve(q)[1], 2)
        pd = O.boris_push(pd, e, dt, QM, 0)
        inside, pd = O.index_inside(pd, g, 1)
        ab = O.save_absorbed(pd, inside)
        assert ab.shape[0] == z["absorbed"][s], s
        if ab.shape[0]:
            wall, normals, _ = O.interaction(ab, g, 1)
            pd, array_len = O.add_and_remove(pd, O.furman_emit(f, wall, normals, mode=0), inside, array_len)
        assert pd.shape[0] == z["counts"][s], s
        assert array_len == z["array_len"][s], s
        assert np.array_equal(checksums(pd), z["checksums"][s]), s
    assert z["managed"].sum() >= 3
    assert np.array_equal(pd, z["final"])
