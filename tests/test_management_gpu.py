"""GPU particle management against the oracle / reference behaviour.

sortByColumn: the sorted weights equal the sorted FP32 weights exactly and
the rows move together.  globalRandom: exact counts, weights scaled by n/target,
survivors (or clones) are rows of the input.  localRandom: total weight
conserved (FP32 rounding), count moves towards the target like the
reference's, and the mean kinetic energy per weight stays within a few
percent of the reference's result.
"""
import numpy as np
import pytest

from conftest import golden
from oracle import oracle as O

pytestmark = pytest.mark.gpu
ME, QE = 9.10938291e-31, 1.602176565e-19


def _setup(pd, bt=1):
    from openecloud_b200.grid import Grid
    from openecloud_b200.particles import Particles
    from openecloud_b200.particleBoundary import AbsorbElliptical
    g = Grid(64, 64, 0.04, 0.04, bt)
    P = Particles("electrons", "variableWeight")
    P.setParticleData(pd)
    P._bind(g)
    return g, P, AbsorbElliptical(g, P)


def _rows_key(a):
    return a[np.lexsort(a.T[::-1])]


@pytest.mark.parametrize("col", [2, 5, 6])
def test_sort_by_column(gpu, col):
    z = golden("management.npz")
    g, P, bd = _setup(z["pd"])
    before = P.getParticleData()
    cells_before = P.soa()["cell"][:before.shape[0]].cpu().numpy()
    P.sortByColumn(col)
    after = P.getParticleData()
    assert np.array_equal(_rows_key(after), _rows_key(before))
    if col == 6:
        cells = P.soa()["cell"][:after.shape[0]].cpu().numpy()
        assert np.all(np.diff(cells) >= 0)
        # stable: equal cells keep their previous relative order
        order = np.argsort(cells_before, kind="stable")
        assert np.array_equal(after, before[order])
    else:
        assert np.all(np.diff(after[:, col]) >= 0)


@pytest.mark.parametrize("n", [4096, 300_001])
def test_sort_by_column_many_tiles_stable(gpu, n):
    """The radix sort over many 4096-key tiles (and a ragged last tile):
    sorting by cell keeps equal cells in their previous order, exactly as a
    stable host argsort; sorting by weight orders the FP32 weights."""
    from openecloud_b200.grid import Grid
    from openecloud_b200.particles import Particles
    rng = np.random.default_rng(n)
    g = Grid(64, 48, 0.04, 0.03, 0)
    pd = np.empty((n, 6))
    pd[:, 0] = rng.uniform(-0.0199, 0.0199, n)
    pd[:, 1] = rng.uniform(-0.0149, 0.0149, n)
    pd[:, 2:5] = rng.normal(0.0, 1e6, (n, 3))
    pd[:, 5] = rng.choice([0.5, 1.0, 1.5, 2.0], n)  # many equal weights
    P = Particles("electrons", "variableWeight")
    P.setParticleData(pd)
    P._bind(g)
    before = P.getParticleData()
    cells_before = P.soa()["cell"][:n].cpu().numpy()
    P.sortByColumn(6)
    after = P.getParticleData()
    assert np.array_equal(after, before[np.argsort(cells_before, kind="stable")])
    w_before = P.getParticleData()[:, 5].copy()
    rows = P.getParticleData()
    P.sortByColumn(5)
    after = P.getParticleData()
    assert np.array_equal(after, rows[np.argsort(w_before.astype(np.float32), kind="stable")])


@pytest.mark.parametrize("target", [3100, 5200, 800])
def test_global_random(gpu, target):
    from openecloud_b200.particleManagement import globalRandom
    z = golden("management.npz")
    g, P, bd = _setup(z["pd"])
    before = P.getParticleData()
    n = before.shape[0]
    globalRandom(g, P, target, seed=5)
    after = P.getParticleData()
    assert after.shape[0] == target
    scaled = before.copy()
    scaled[:, 5] = (before[:, 5].astype(np.float32).astype(np.float64) * (n / target)).astype(np.float32)
    # every row is one of the (weight-scaled) input rows
    ref_set = {tuple(r) for r in scaled}
    assert all(tuple(r) in ref_set for r in after)
    if target < n:
        assert len({tuple(r) for r in after}) == target  # no duplicates: drawn without replacement


@pytest.mark.parametrize("scheme", [0, 1])
@pytest.mark.parametrize("tag,target", [("down", 3000), ("up", 4600)])
def test_local_random_statistics(gpu, scheme, tag, target):
    from openecloud_b200.particleManagement import localRandom
    z = golden("management.npz")
    g, P, bd = _setup(z["pd"])
    before = P.getParticleData()
    localRandom(g, P, bd, target, mergeScheme=scheme, seed=3)
    after = P.getParticleData()
    ref = z[f"local{scheme}_{tag}"]
    # weight: conserved up to FP32 rounding of the merged sums
    assert abs(after[:, 5].sum() / before[:, 5].sum() - 1) < 1e-5
    # the count moves towards the target as the reference's does
    n0 = before.shape[0]
    assert (after.shape[0] - n0) * (ref.shape[0] - n0) >= 0
    assert abs(after.shape[0] - ref.shape[0]) <= 0.1 * n0

    def ekin(a):
        return 0.5 * ME / QE * np.sum(np.sum(a[:, 2:5] ** 2, 1) * a[:, 5]) / np.sum(a[:, 5])
    if scheme == 0:
        assert abs(ekin(after) / ekin(before) - 1) < 0.05


def _moments(pd):
    w = pd[:, 5]
    v = pd[:, 2:5]
    return np.array([pd.shape[0], w.sum(), *(w[:, None] * v).sum(0), (w * (v * v).sum(1)).sum()])


@pytest.mark.parametrize("scheme", [0, 1])
@pytest.mark.parametrize("t,target", [(0, 3000), (1, 4600)])
def test_local_random_ensemble_moments(gpu, scheme, t, target):
    """16 seeds of the device merge against 16 seeds of the reference's
    kd-tree merge (particleManagement.pyx:74-238) on the same 4000 rows: the
    ensemble means of the count, the total weight, the momentum (sum w v) and
    the energy (sum w |v|^2) agree within 4 combined standard errors plus a
    floor: 3 % of the count (the device pairs neighbours along a phase-space
    curve instead of searching a kd-tree, and its distance test passes
    2-3 % fewer pairs: measured 0.814 against 0.791 of the count at the
    3000 target), 5 % of the total momentum for a momentum component (the
    merged velocity is one of the pair's, so the momentum of a merge moves by
    a few percent of the total with the pairing; scheme 1's rescaling is not
    momentum-neutral either), 0.2 % for the weight and the energy."""
    from openecloud_b200.particleManagement import localRandom
    z = golden("management.npz")
    ref = golden("management_ensemble.npz")
    before = ref["before"]
    mine = []
    for k in range(16):
        g, P, bd = _setup(z["pd"])
        localRandom(g, P, bd, target, mergeScheme=scheme, seed=500 + k)
        mine.append(_moments(P.getParticleData()))
    mine = np.array(mine) / before
    theirs = ref["moments"][scheme, t] / before
    names = ["count", "weight", "px", "py", "pz", "energy"]
    if scheme == 1:
        # the reference's rescaling (particleManagement.pyx:200-236) scales the
        # kept velocity by a factor that depends on how alike the two paired
        # velocities are, so momentum and energy after it depend on the
        # pairing itself: both raise the energy (measured +2.8 % here against
        # +1.1 % for the kd-tree at the 3000 target), and the count and the
        # weight are compared as for scheme 0
        assert np.all(mine[:, 5] > 1.0) and np.all(ref["moments"][scheme, t][:, 5] / before[5] > 1.0)
        assert abs(mine[:, 5].mean() - (ref["moments"][scheme, t][:, 5] / before[5]).mean()) < 0.03
        names = names[:2]
    for i, name in enumerate(names):
        a, b = mine[:, i], theirs[:, i]
        se = np.sqrt(a.var(ddof=1) / len(a) + b.var(ddof=1) / len(b))
        floor = 0.03 if name == "count" else 0.002
        if name.startswith("p"):  # momentum components: relative to the total momentum magnitude
            floor = 0.05 * np.linalg.norm(before[2:5]) / abs(before[i])
        print(f"scheme {scheme} target {target} {name}: device {a.mean():.5f} +- {a.std():.5f}, "
              f"reference {b.mean():.5f} +- {b.std():.5f}")
        assert abs(a.mean() - b.mean()) <= 4 * se + floor, name
    if scheme == 0:
        assert np.all(np.abs(mine[:, 1] - 1) < 1e-5)  # every merge and split conserves the weight


def _search_sorted_ref(a, value):
    # particleManagement.pyx:244-262 as written
    n = a.shape[0]
    if a[n - 1] <= value:
        return n
    if a[0] >= value:
        return 0
    i0, i2 = 0, n - 1
    i1 = int((i2 + i0) * 0.5)
    while i1 != i0:
        if a[i1] > value:
            i2 = i1
        else:
            i0 = i1
        i1 = int((i2 + i0) * 0.5)
    return i1 + 1


def test_weight_thresholds_match_reference_search(gpu):
    import torch
    from openecloud_b200 import _lib
    from openecloud_b200 import device as D
    from openecloud_b200.grid import Grid
    from openecloud_b200.particles import Particles
    rng = np.random.default_rng(8)
    n = 5000
    pd = np.zeros((n, 6))
    pd[:, 0] = rng.uniform(-0.01, 0.01, n)
    pd[:, 1] = rng.uniform(-0.01, 0.01, n)
    pd[:, 5] = np.round(rng.uniform(0.5, 3.0, n), 2)  # ties
    P = Particles("electrons", "variableWeight")
    P.setParticleData(pd)
    P._bind(Grid(64, 64, 0.04, 0.04, 1))
    P.sortByColumn(5)
    w = D.to_numpy(P._soa["w"][:n]).astype(np.float64)
    thr = D.zeros(2, torch.int32)
    for lo, hi in [(1.0, 2.0), (0.1, 9.0), (w[0], w[-1]), (w[17], w[4000]), (1.5, 1.5), (-1.0, 0.4)]:
        _lib.call("oec_weight_thresholds", P.c_particles(), float(lo), float(hi), thr.data_ptr(), D.stream())
        got = tuple(int(x) for x in D.to_numpy(thr))
        assert got == (_search_sorted_ref(w, lo), _search_sorted_ref(w, hi)), (lo, hi, got)
