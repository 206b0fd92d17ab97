"""Oracle particle management against the compiled reference (same MT stream)."""
import numpy as np
import pytest

from conftest import golden
from oracle import oracle as O


def test_sort_by_column_replays_reference():
    z = golden("management.npz")
    assert np.array_equal(O.sort_by_column(z["pd"], 5, seed=11), z["sorted"])


@pytest.mark.parametrize("tag,target", [("kill", 3100), ("clone", 5200)])
def test_global_random_replays_reference(tag, target):
    z = golden("management.npz")
    out = O.global_random(z["pd"], target, seed=21)
    assert np.array_equal(out, z[f"global_{tag}"])
    # total weight is conserved in expectation only; count is exact
    assert out.shape[0] == target


@pytest.mark.parametrize("scheme", [0, 1])
@pytest.mark.parametrize("tag,target", [("down", 3000), ("up", 4600)])
def test_local_random_replays_reference(scheme, tag, target):
    z = golden("management.npz")
    g = O.GridGeom(64, 64, 0.04, 0.04)
    out = O.local_random(z["pd"], target, g, kind=1, seed=31 + scheme, scheme=scheme)
    ref = z[f"local{scheme}_{tag}"]
    assert out.shape == ref.shape
    assert np.array_equal(out, ref)
    # merging and halving conserve the total weight in scheme 0; the
    # reference's scheme 1 run on this input does not (its own output differs
    # by ~4e-4), which the replay reproduces
    if scheme == 0:
        assert np.isclose(out[:, 5].sum(), z["pd"][:, 5].sum(), rtol=1e-13)


def add_remove_rows(ids, rng):
    """Rows for the add/remove sequence: the id in the weight column, the
    rest arbitrary (placement moves whole rows)."""
    r = np.empty((ids.size, 6))
    r[:, :2] = rng.uniform(-0.019, 0.019, (ids.size, 2))
    r[:, 2:5] = rng.normal(0, 1e5, (ids.size, 3))
    r[:, 5] = ids
    return r


def test_add_and_remove_replays_reference():
    """Every placement rule of addAndRemoveParticles (remove only, in place
    with more and with fewer added rows than holes, a new larger array),
    slot by slot, against the compiled reference's id sequences."""
    z = golden("add_remove.npz")
    rng = np.random.default_rng(0)
    n0 = int(z["n0"])
    pd = add_remove_rows(np.arange(n0, dtype=np.float64), rng)
    array_len, next_id = n0, n0
    k = 0
    while f"ids{k}" in z.files:
        n, m = pd.shape[0], int(z[f"nadd{k}"])
        keep = np.unpackbits(z[f"keep{k}"])[:n].astype(np.uint16)
        add = add_remove_rows(np.arange(next_id, next_id + m, dtype=np.float64), rng)
        next_id += m
        pd, array_len = O.add_and_remove(pd, add, keep, array_len)
        assert np.array_equal(pd[:, 5].astype(np.int32), z[f"ids{k}"]), k
        assert array_len == int(z[f"len{k}"]), k
        k += 1
    assert k == 10
