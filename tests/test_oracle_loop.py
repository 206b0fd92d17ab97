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
