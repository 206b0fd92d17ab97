"""Batched buildup runs (one graph per batch step, runs on parallel branches).

GPU: a run advanced inside a batch reproduces the same run advanced alone bit
for bit with the LU solve (every kernel on its path is deterministic: the
fixed-point deposit is order-independent, the emission draws are keyed by
run seed, slot and step); a batch of uneven grids with the multigrid solve
converges in every run without a fallback; the autotuner's choices carry the
timings they were made from.
CPU: the autotuner keeps the fastest candidate and its record.
"""
import json

import numpy as np
import pytest

RUNS = [dict(nx=64, ny=64, lx=0.04, ly=0.04, boundType=1, n_init=2000, target=20000, seed=11, sey_max=1.6),
        dict(nx=64, ny=64, lx=0.04, ly=0.04, boundType=1, n_init=2000, target=20000, seed=12, sey_max=2.0,
             beam_particles=1.5e11),
        dict(nx=48, ny=48, lx=0.09, ly=0.036, boundType=1, n_init=2000, target=20000, seed=13, sey_max=1.8,
             type_b_field=1, b_const=(0.0, 8.33, 0.0)),
        dict(nx=48, ny=48, lx=0.09, ly=0.036, boundType=1, n_init=2000, target=20000, seed=14, sey_max=1.2,
             beam_particles=0.5e11)]


def test_autotuner_keeps_fastest_and_records(tmp_path):
    from openecloud_b200.autotune import Autotuner
    path = tmp_path / "tune.json"
    t = Autotuner(path=str(path))
    seen = []

    def trial(c):
        seen.append(c)
        return {1: 5.0, 4: 2.0, 16: 3.0}[c]
    assert t.branches("k", [1, 4, 16], trial) == 4 and seen == [1, 4, 16]
    assert t.branches("k", [1, 4, 16], trial) == 4 and seen == [1, 4, 16]  # remembered, no new trials
    rec = json.loads(path.read_text())["branches/k"]
    assert rec["choice"] == 4 and rec["ms_per_step"] == {"1": 5.0, "4": 2.0, "16": 3.0}
    assert Autotuner(path=str(path)).branches("k", [1], trial) == 4  # read back from the file


@pytest.mark.gpu
def test_batched_run_equals_standalone_run(gpu):
    from openecloud_b200.batch import BatchedBuildup
    from openecloud_b200.buildup import Buildup
    steps = 120
    runs = [dict(r, n_steps_table=steps + 1, management_every=50) for r in RUNS]
    batch = BatchedBuildup(runs, branches=4, poisson="lu")
    batch.run(steps)
    for cfg, (n_b, w_b) in zip(runs, batch.histories()):
        alone = Buildup(**cfg)
        alone.run(steps)
        n_a, w_a = alone.history()
        assert np.array_equal(n_a, n_b) and np.array_equal(w_a, w_b), cfg["seed"]
    for st in batch.status():
        assert st["n_capacity_drop"] == 0 and st["n_nonfinite"] == 0


@pytest.mark.gpu
def test_batched_multigrid_runs_and_autotuner(gpu):
    from openecloud_b200.autotune import Autotuner
    from openecloud_b200.batch import BatchedBuildup
    steps = 60
    runs = [dict(r, n_steps_table=steps + 1, management_every=50) for r in RUNS]
    tuner = Autotuner()
    batch = BatchedBuildup(runs, tuner=tuner)
    batch.run(steps, trial_steps=2)
    keys = sorted(tuner.choices)
    assert any(k.startswith("poisson/") for k in keys) and any(k.startswith("branches/") for k in keys)
    for k in keys:
        assert tuner.choices[k]["choice"] is not None
    assert batch.branches in (1, 4)
    for b in batch.runs:
        if b.ps.method == "pcg":
            assert b.ps.nFallbacks == 0 and b.ps.lastStats.converged == 1
        n, w = b.history()
        assert n[-1] > 0 and np.all(np.isfinite(w))
    mg = BatchedBuildup(runs, branches=4, poisson="mg")
    mg.run(steps)
    for b in mg.runs:
        assert b.ps.nFallbacks == 0 and b.ps.lastStats.converged == 1 and b.ps.lastStats.rel_residual <= 1e-8


def test_shard_runs_balances_and_covers():
    from openecloud_b200.batch import run_cost, scan_configs, shard_runs
    runs = scan_configs(64)
    for world in (1, 2, 3, 8):
        parts = [shard_runs(runs, r, world) for r in range(world)]
        assert sorted(i for p in parts for i in p) == list(range(64))
        loads = [sum(run_cost(runs[i]) for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(run_cost(r) for r in runs)


def _gather_worker(rank, world, port, runs, q):
    import os
    import torch.distributed as dist
    from openecloud_b200.batch import gather_histories, shard_runs
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    mine = shard_runs(runs, rank, world)
    hist = [(np.arange(5) + i, np.full(5, 10.0 * i)) for i in mine]  # stand-in histories
    out = gather_histories(mine, hist, len(runs))
    if rank == 0:
        q.put([(int(n[0]), float(w[0])) for n, w in out])
    dist.destroy_process_group()


def test_gather_histories_two_ranks_gloo():
    import socket
    import torch.multiprocessing as mp
    from openecloud_b200.batch import scan_configs
    runs = scan_configs(10)
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_gather_worker, args=(r, 2, port, runs, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert got == [(i, 10.0 * i) for i in range(10)]
