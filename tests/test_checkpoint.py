"""Checkpoint and reference-output files on the host (no GPU): the exact
store round trip, the configuration check and the reference's layouts
(example01_basic.py:76-78: (N, 6) float64 particleData.npy, uint0 count
histories)."""
import numpy as np
import pytest

from openecloud_b200 import checkpoint as C


def _store(n, rng):
    return {"cell": rng.integers(0, 1 << 20, n).astype(np.int32),
            **{k: rng.random(n, dtype=np.float32) for k in ("ox", "oy", "vx", "vy", "vz", "w")}}


def test_checkpoint_round_trip_is_exact(tmp_path):
    rng = np.random.default_rng(1)
    sig = {"grid": [128, 128, 0.04, 0.04, 1], "seed": 3}
    st = _store(5000, rng)
    arrays = {"rho_fix": rng.integers(-2 ** 40, 2 ** 40, 130 * 130), "wscale": np.array([2.0 ** 30]),
              "hist_w": rng.random(10), "phi_prev": None}
    C.write_checkpoint(str(tmp_path), sig, st, arrays, {"steps_done": 7})
    s2, a2, c2 = C.read_checkpoint(str(tmp_path), sig)
    for k in C.STORE_FIELDS:
        assert s2[k].dtype == st[k].dtype and np.array_equal(s2[k], st[k])
    assert set(a2) == {"rho_fix", "wscale", "hist_w"}
    assert np.array_equal(a2["rho_fix"], arrays["rho_fix"]) and a2["rho_fix"].dtype == np.int64
    assert c2 == {"steps_done": 7}
    with pytest.raises(C.CheckpointError):
        C.read_checkpoint(str(tmp_path), {"grid": [128, 128, 0.04, 0.04, 1], "seed": 4})


def test_checkpoint_rejects_ragged_store(tmp_path):
    rng = np.random.default_rng(2)
    st = _store(100, rng)
    st["vz"] = st["vz"][:99]
    with pytest.raises(C.CheckpointError):
        C.write_checkpoint(str(tmp_path), {}, st, {}, {})


def test_reference_outputs_layout(tmp_path):
    rows = np.random.default_rng(3).normal(size=(77, 6))
    C.write_reference_outputs(str(tmp_path), rows, [1.5e9, 2.5e9], [10000, 10200])
    back = C.read_particle_data(str(tmp_path))
    assert back.dtype == np.float64 and np.array_equal(back, rows)
    pc = np.load(tmp_path / C.PHYSICAL_COUNT)
    assert pc.dtype == np.uintp and list(pc) == [1500000000, 2500000000]
    np.save(tmp_path / "bad.npy", rows[:, :5])
    with pytest.raises(C.CheckpointError):
        C.read_particle_data(str(tmp_path / "bad.npy"))
    empty = np.zeros((0, 6))
    C.write_reference_outputs(str(tmp_path / "e"), empty, [], [])
    assert C.read_particle_data(str(tmp_path / "e")).shape == (0, 6)
