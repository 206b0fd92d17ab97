"""One buildup run sharded over GPUs: one process per GPU, particles
partitioned, the deposit summed.

The reference runs one store on one core; its per-step charge deposit
(chargeToGrid, particles.pyx:70-77, :336-351) is a sum over particles, so a
run's particles split over W stores deposit W partial grids whose sum is the
whole grid.  With the int64 fixed-point deposit that sum is exact and
independent of the order and the split, so the sharded run's right-hand
side equals the unsharded one bit for bit once every shard uses the same
scale.  Per step:

  1. each rank pushes, gathers, tests and deposits its own particles
     (oec_push_gather) and emits / compacts them (oec_add_remove);
  2. the int64 node grids are summed across ranks (one all-reduce of
     8 B per node: 8.4 MB at 1024^2, over NCCL on NVLink);
  3. every rank solves the same Poisson problem (the LU solve is
     deterministic, so all ranks hold the same E) and carries on.

Partitioning: the store is cell-sorted at setup, so contiguous slices of it
are spatial bins; particles that later cross bins stay on their rank (the
deposit does not care where a particle is stored).  The fixed-point scale is
taken for the summed capacity (oec_deposit_scale_capacity) and reduced to the
smallest over ranks, so no node of the summed grid can overflow.

Particle management (globalRandom) acts per shard with the target split in
proportion; the emission streams are keyed by a per-rank seed.  NCCL
collectives are not captured into the step graph here: a sharded run
launches its steps directly.
"""
import numpy as np
import torch

from . import _lib
from . import device as D
from .buildup import Buildup


def particle_shard(n, rank, world):
    """[lo, hi) of the rows of a cell-sorted store of n particles that
    `rank` of `world` holds: contiguous, sizes differing by at most one."""
    if world < 1 or not 0 <= rank < world or n < 0:
        raise ValueError("need 0 <= rank < world and n >= 0")
    base, extra = divmod(int(n), int(world))
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def reduce_scale(wscale, group=None):
    """The shards' common fixed-point scale: the smallest of their scales
    (the one of the largest weight), in place on every rank."""
    import torch.distributed as dist
    dist.all_reduce(wscale, op=dist.ReduceOp.MIN, group=group)
    return wscale


def allreduce_deposit(rho_fix, group=None):
    """Sums the int64 node grids of all ranks in place (exact)."""
    import torch.distributed as dist
    if rho_fix.dtype != torch.int64:
        raise TypeError("the fixed-point deposit is int64")
    dist.all_reduce(rho_fix, op=dist.ReduceOp.SUM, group=group)
    return rho_fix


class ShardedBuildup(Buildup):
    """A buildup run whose particles are split over the ranks of `group`
    (torch.distributed, one process per GPU).  Each rank loads its share of
    the initial electrons with its own seed, manages toward its share of the
    target and emits with its own stream; the deposit is all-reduced before
    every solve.  history() returns the summed (count, weight) history on
    every rank."""

    def __init__(self, rank, world, group=None, **kw):
        self.rank, self.world, self.group = int(rank), int(world), group
        n_init = int(kw.get("n_init", 10000))
        lo, hi = particle_shard(n_init, rank, world)
        t_lo, t_hi = particle_shard(int(kw.get("target", 100000)), rank, world)
        kw = dict(kw, n_init=max(hi - lo, 1), target=max(t_hi - t_lo, 1),
                  w_init=kw.get("w_init") if kw.get("w_init") is not None else 1e9 / n_init,
                  seed=int(kw.get("seed", 0)) + 7919 * rank)
        if kw.get("capacity") is None:
            kw["capacity"] = max(4 * kw["target"], 4 * kw["n_init"], 65536)
        self._total_capacity = None
        super().__init__(**kw)

    def _world_capacity(self):
        if self._total_capacity is None:
            import torch.distributed as dist
            c = torch.tensor([self.P._cap], dtype=torch.int64, device=D.device())
            dist.all_reduce(c, op=dist.ReduceOp.SUM, group=self.group)
            self._total_capacity = int(c.item())
        return self._total_capacity

    def _prepare_deposit(self):
        P, s = self.P, D.stream()
        self._total_capacity = None  # management may have grown a store
        _lib.call("oec_deposit_scale_capacity", P.c_particles(), self._world_capacity(), P._wscale.data_ptr(), s)
        reduce_scale(P._wscale, self.group)
        _lib.call("oec_deposit", self.grid.c_grid(), P.c_particles(), P._rho_fix.data_ptr(), P._wscale.data_ptr(),
                  1, P._status.data_ptr(), s)

    def _manage(self, step):
        """Management as Buildup._manage, per shard; the re-deposit that
        follows it (with its collectives) runs on every rank when any rank
        managed."""
        import torch.distributed as dist
        from .particleManagement import globalRandom, localRandom
        self._check_rows()
        n = self.P.getMacroParticleCount()
        do = step > 0 and step % self.management_every == 0 and \
            (n > 1.05 * self.target or n < 0.95 * self.target) and self.management in ("global", "local")
        if do and self.management == "global":
            globalRandom(self.grid, self.P, self.target, seed=self.seed + step, call=self.n_managed + 1)
        elif do:
            localRandom(self.grid, self.P, self.bd, self.target, seed=self.seed + step, call=self.n_managed + 1)
        flag = torch.tensor([1 if do else 0], dtype=torch.int32, device=D.device())
        dist.all_reduce(flag, op=dist.ReduceOp.MAX, group=self.group)
        if int(flag.item()):
            self._prepare_deposit()
            self.n_managed += 1
            return True
        return False

    def _launch_step(self):
        allreduce_deposit(self.P._rho_fix, self.group)
        super()._launch_step()

    def run(self, n_steps, use_graph=False):
        if use_graph and self.world > 1:
            raise ValueError("a sharded run launches its steps directly (no collectives in the step graph)")
        return super().run(n_steps, use_graph=use_graph)

    def history(self):
        import torch.distributed as dist
        n, w = super().history()
        t = torch.tensor(np.stack([n.astype(np.float64), w]), dtype=torch.float64, device=D.device())
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=self.group)
        t = t.cpu().numpy()
        return t[0].astype(np.int64), t[1]
