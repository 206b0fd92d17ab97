"""Sharded single run on the device.

* The device's int64 deposit equals the oracle's restatement of it bit for
  bit (the restatement the gloo test sums over ranks).
* A one-rank sharded run (NCCL, the all-reduce an identity) reproduces the
  plain run bit for bit, so the sharded step is the plain step plus the sum.
* Two ranks as two processes on this one GPU with gloo (host-side
  collectives; no kernel waits on another process): both ranks solve the
  same right-hand side, which is the deposit of the union of their
  particles, so their potentials are identical.
"""
import socket

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def test_device_deposit_equals_oracle_fixed_point(gpu):
    from openecloud_b200 import device as D
    from openecloud_b200.grid import Grid
    from openecloud_b200.particles import Particles
    rng = np.random.default_rng(8)
    n = 300_000
    g = Grid(128, 128, 0.04, 0.04, 0)
    pd = np.zeros((n, 6))
    pd[:, :2] = rng.uniform(-0.02, 0.02, (n, 2))
    pd[:, 5] = rng.uniform(0.5, 1.5, n) * 1e4
    P = Particles("electrons", "variableWeight")
    P.setParticleData(pd)
    P.chargeToGrid(g)
    fix, wscale = P.getChargeOnGridFixed()
    s = {k: D.to_numpy(v[:n]) for k, v in P.soa().items()}
    assert wscale == O.deposit_scale(s["w"], P._cap)
    ref = O.fixed_point_deposit(s["cell"], s["ox"], s["oy"], s["w"], g.getNxExt(), g.getNpExt(), wscale)
    assert np.array_equal(fix, ref)


def _init_pg(backend, rank, world, port):
    import datetime
    import os
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group(backend, rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))


def _port():
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        return so.getsockname()[1]


def test_one_rank_sharded_run_equals_plain_run(gpu):
    import torch.distributed as dist
    from openecloud_b200.buildup import Buildup
    from openecloud_b200.shard import ShardedBuildup
    kw = dict(seed=31, n_steps_table=121)
    plain = Buildup(**kw)
    plain.run(120)
    _init_pg("nccl", 0, 1, _port())
    try:
        sh = ShardedBuildup(0, 1, **kw)
        sh.run(120)
        hp, hs = plain.history(), sh.history()
        assert np.array_equal(hp[0], hs[0]) and np.array_equal(hp[1], hs[1])
        assert np.array_equal(plain.P.getParticleData(), sh.P.getParticleData())
    finally:
        dist.destroy_process_group()


def _two_rank_worker(rank, world, port, q):
    import torch
    import torch.distributed as dist
    from openecloud_b200 import device as D
    from openecloud_b200.shard import ShardedBuildup
    torch.cuda.set_device(0)
    _init_pg("gloo", rank, world, port)
    try:
        b = ShardedBuildup(rank, world, seed=40, n_init=20000, n_steps_table=81)
        wscale0 = float(D.to_numpy(b.P._wscale)[0])
        n0 = b.P.getMacroParticleCount()
        soa = {k: D.to_numpy(v[:n0]) for k, v in b.P.soa().items()}
        rho0 = b.P._rho_fix.clone()
        from openecloud_b200.shard import allreduce_deposit
        allreduce_deposit(rho0)
        parts = [None] * world
        dist.all_gather_object(parts, soa)
        b.run(80)
        phi = D.to_numpy(b.ps.phi)
        phis = [None] * world
        dist.all_gather_object(phis, phi)
        hist = b.history()
        if rank == 0:
            q.put(dict(parts=parts, rho0=D.to_numpy(rho0), wscale=wscale0,
                       nx=b.grid.getNxExt(), G=b.grid.getNpExt(), phis=phis, hist_n=hist[0], n0=n0))
    finally:
        dist.destroy_process_group()


def test_two_rank_sharded_run_shares_the_right_hand_side(gpu):
    import torch.multiprocessing as mp
    port = _port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_two_rank_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = q.get(timeout=600)
    for p in procs:
        p.join(timeout=300)
        assert p.exitcode == 0
    cat = {k: np.concatenate([p[k] for p in out["parts"]]) for k in out["parts"][0]}
    assert len(cat["cell"]) == 20000
    union = O.fixed_point_deposit(cat["cell"], cat["ox"], cat["oy"], cat["w"], out["nx"], out["G"], out["wscale"])
    assert np.array_equal(out["rho0"], union)
    assert np.array_equal(out["phis"][0], out["phis"][1])
    assert out["hist_n"][0] == 20000 and out["hist_n"][-1] > 0
