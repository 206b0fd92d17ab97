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
