"""Sharded single run, host side (no GPU): the particle partition and the
exact deposit sum over ranks.

Two gloo ranks each take a contiguous slice of a cell-sorted store, compute
its fixed-point scale for the summed capacity, agree on the smallest scale
(reduce_scale), deposit their slice with the oracle's restatement of the
device deposit and sum the int64 grids (allreduce_deposit).  The summed grid
must equal the deposit of the whole store bit for bit (particles.pyx:336-351
is the deposit that is split)."""
import socket

import numpy as np
import pytest

from oracle import oracle as O


def test_particle_shard_covers_and_balances():
    from openecloud_b200.shard import particle_shard
    for n in (0, 1, 7, 1000, 1 << 20):
        for world in (1, 2, 3, 8):
            parts = [particle_shard(n, r, world) for r in range(world)]
            assert parts[0][0] == 0 and parts[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(parts, parts[1:]))
            sizes = [hi - lo for lo, hi in parts]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        particle_shard(10, 2, 2)


def _store(n, nx, seed):
    rng = np.random.default_rng(seed)
    cells = np.sort(rng.integers(nx + 1, nx * (nx - 2) - 2, n)).astype(np.int32)  # cell-sorted
    ox = rng.random(n, dtype=np.float32) * np.float32(0.99999994)
    oy = rng.random(n, dtype=np.float32) * np.float32(0.99999994)
    w = (rng.uniform(0.5, 1.5, n) * 1e4).astype(np.float32)
    w[rng.integers(0, n)] = np.float32(3.1e4)  # the largest weight sits in one shard
    return cells, ox, oy, w


def _worker(rank, world, port, n, nx, cap, q):
    import os
    import torch
    import torch.distributed as dist
    from openecloud_b200.shard import allreduce_deposit, particle_shard, reduce_scale
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        cells, ox, oy, w = _store(n, nx, 5)
        lo, hi = particle_shard(n, rank, world)
        scale = torch.tensor([O.deposit_scale(w[lo:hi], world * cap)], dtype=torch.float64)
        reduce_scale(scale)
        rho = torch.from_numpy(O.fixed_point_deposit(cells[lo:hi], ox[lo:hi], oy[lo:hi], w[lo:hi], nx, nx * nx,
                                                     float(scale[0])))
        allreduce_deposit(rho)
        if rank == 0:
            q.put((float(scale[0]), rho.numpy().tobytes()))
    finally:
        dist.destroy_process_group()


def _wait(q, procs, timeout=300):
    """The first result on q; fails at once when a rank exits with an error."""
    import queue
    import time
    t0 = time.time()
    while time.time() - t0 < timeout:
        try:
            return q.get(timeout=1)
        except queue.Empty:
            bad = [p.exitcode for p in procs if p.exitcode not in (None, 0)]
            if bad:
                for p in procs:
                    p.kill()
                pytest.fail(f"a rank exited with {bad}")
    for p in procs:
        p.kill()
    pytest.fail("no result from the ranks")


def test_sharded_deposit_sums_to_the_whole_store_gloo():
    import torch.multiprocessing as mp
    n, nx, world, cap = 200_000, 66, 2, 131072
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, n, nx, cap, q)) for r in range(world)]
    for p in procs:
        p.start()
    scale, raw = _wait(q, procs)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    cells, ox, oy, w = _store(n, nx, 5)
    whole_scale = O.deposit_scale(w, world * cap)
    assert scale == whole_scale
    whole = O.fixed_point_deposit(cells, ox, oy, w, nx, nx * nx, whole_scale)
    got = np.frombuffer(raw, dtype=np.int64)
    assert np.array_equal(got, whole)
    # exact conservation: the total is the sum of the quantised charges
    assert int(got.sum()) == int(np.rint(w.astype(np.float64) * whole_scale).astype(np.int64).sum())
