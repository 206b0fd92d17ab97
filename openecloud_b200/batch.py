"""Many independent buildup runs advanced together (SEY and intensity scans).

Each run is a `Buildup` with its own particles, beam, emitter and Poisson
state; runs on the same grid (size and chamber) share the Grid geometry and
the solver's factorisation / multigrid operators (`PoissonSolver.sibling`).
One time step of the whole batch is recorded once into one CUDA graph: the
runs' steps sit on parallel branches (streams forked from and joined to the
capturing stream), so the GPU interleaves the small kernels of many runs and
the host launches one graph per batch step.  A branch holds every k-th run;
the branch width, the Poisson solve of each grid and the multigrid block size
are chosen by `openecloud_b200.autotune.Autotuner` on the device.  The fused
particle kernel of every run is a persistent kernel; the iterative solve of a
run keeps its loops inside the graph (conditional nodes).

Management (roulette / merge) runs per run between graph replays at the runs'
common cadence; the batch graph is recaptured only when a device buffer of
some run has changed.

No reference counterpart: the reference runs one simulation per process.
"""
import concurrent.futures
import os

import numpy as np
import torch

from .autotune import Autotuner
from .buildup import Buildup
from .grid import Grid
from .lu_setup import factor
from .poissonSolver import PoissonSolver

GRID_KEYS = (("nx", 128), ("ny", 128), ("lx", 0.04), ("ly", 0.04), ("boundType", 1))


class BatchedBuildup:
    """runs: a list of keyword-argument dicts for `Buildup` (grid size,
    chamber, SEY, intensity, field, seed, ...); every run must use the same
    `management_every`.  branches: graph branch width (None: autotuned);
    poisson: 'lu', 'mg' or None (autotuned per grid); shard: (rank, world)
    to advance only this rank's share of the runs (one process per GPU, no
    exchange until `gather_histories`)."""

    def __init__(self, runs, branches=None, poisson=None, tuner=None, shard=None):
        if not runs:
            raise ValueError("no runs")
        # one GPU of several: this process's share of the runs (shard_runs),
        # their indices in `indices`; gather_histories collects them at the end
        self.n_total = len(runs)
        self.indices = list(range(len(runs))) if shard is None else shard_runs(runs, *shard)
        runs = [runs[i] for i in self.indices]
        if not runs:
            raise ValueError("no runs in this shard")
        self.tuner = tuner or Autotuner()
        every = {int(r.get("management_every", 50)) for r in runs}
        if len(every) != 1:
            raise ValueError("all runs of a batch need the same management_every")
        self.management_every = every.pop()
        self.shared = {}
        self.runs = []
        # the host setup of every distinct grid (geometry, assembly, SuperLU
        # factorisation: seconds each on the larger grids) in parallel
        # threads -- scipy's splu releases the GIL -- before the device setups
        keys = list(dict.fromkeys(tuple(cfg.get(k, d) for k, d in GRID_KEYS) for cfg in runs))
        grids = {key: Grid(*key) for key in keys}
        with concurrent.futures.ThreadPoolExecutor(max_workers=min(len(keys), os.cpu_count() or 1)) as ex:
            facts = dict(zip(keys, ex.map(lambda k: factor(grids[k]), keys)))
        for cfg in runs:
            key = tuple(cfg.get(k, d) for k, d in GRID_KEYS)
            if key not in self.shared:
                g = grids[key]
                ps = PoissonSolver(g, factors=facts.pop(key))
                if poisson is None:
                    self.tuner.poisson(ps)
                elif poisson == "mg":
                    ps.method, ps.precond = "pcg", "mg"
                    ps.prepare()
                else:
                    ps.method = "lu"
                self.shared[key] = (g, ps)
            g, ps = self.shared[key]
            self.runs.append(Buildup(grid=g, poisson=ps.sibling(), **cfg))
        self.branches = branches
        self.graph = None
        self._sig = None
        self._graph_branches = None
        self._main = torch.cuda.Stream()
        self._streams = []
        self.steps_done = 0

    # ------------------------------------------------------------ capture
    def _signature(self):
        return tuple(b._step_signature() for b in self.runs)

    def _capture(self, nb):
        for b in self.runs:
            b.ps.prepare()
        while len(self._streams) < nb:
            self._streams.append(torch.cuda.Stream())
        cur = torch.cuda.current_stream()
        main = self._main
        main.wait_stream(cur)
        self.graph = None
        g = torch.cuda.CUDAGraph()
        with torch.cuda.stream(main):
            g.capture_begin()
            try:
                fork = torch.cuda.Event()
                fork.record(main)
                joins = []
                for k in range(nb):
                    st = self._streams[k]
                    st.wait_event(fork)
                    with torch.cuda.stream(st):
                        for b in self.runs[k::nb]:
                            b._launch_step()
                    ev = torch.cuda.Event()
                    ev.record(st)
                    joins.append(ev)
                for ev in joins:
                    main.wait_event(ev)
            finally:
                g.capture_end()
        cur.wait_stream(main)
        self.graph = g
        self._sig = self._signature()
        self._graph_branches = nb

    def _replay(self, n, nb):
        if self.graph is None or self._graph_branches != nb or self._sig != self._signature():
            self._capture(nb)
        for _ in range(n):
            self.graph.replay()
        self.steps_done += n
        for b in self.runs:
            b.steps_done = self.steps_done

    # ---------------------------------------------------------------- run
    def _manage(self, step):
        if step % self.management_every == 0:
            for b in self.runs:
                b._manage(step)

    def _check_table(self, n):
        for b in self.runs:
            if self.steps_done + n > b._table_len:
                raise ValueError("beam table exhausted: increase n_steps_table")

    def run(self, n_steps, trial_steps=3):
        """Advance every run n_steps; returns device seconds (the branch
        width trials, when the width is autotuned, are part of the first
        steps and of the time)."""
        self._check_table(n_steps)
        s = torch.cuda.current_stream()
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record(s)
        k = 0
        if self.branches is None:
            cands = sorted({1, 4, 16, len(self.runs)} & set(range(1, len(self.runs) + 1)))
            budget = len(cands) * trial_steps
            if budget < n_steps and budget <= self.management_every - (self.steps_done % self.management_every):
                self._manage(self.steps_done)
                before = self.steps_done

                def trial(nb):
                    self._capture(nb)
                    return self._time_replays(trial_steps, nb)
                key = f"{len(self.runs)}runs_" + "_".join(sorted({Autotuner.grid_key(g) for g, _ in
                                                                  self.shared.values()}))
                self.branches = self.tuner.branches(key, cands, trial)
                k = self.steps_done - before  # steps the trials advanced (0 for a remembered choice)
            else:
                self.branches = len(self.runs)
        nb = self.branches
        while k < n_steps:
            step = self.steps_done
            self._manage(step)
            nxt = min(n_steps - k, self.management_every - (step % self.management_every))
            self._replay(nxt, nb)
            k += nxt
        t1.record(s)
        t1.synchronize()
        for b in self.runs:
            b._check_rows()
        return t0.elapsed_time(t1) * 1e-3

    def _time_replays(self, n, nb):
        s = torch.cuda.current_stream()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        self._replay(n, nb)
        e1.record(s)
        e1.synchronize()
        return e0.elapsed_time(e1) / n

    def histories(self):
        """(macro count, sum of weights) per run at the start of every step."""
        return [b.history() for b in self.runs]

    def status(self):
        return [b.status() for b in self.runs]


SCAN_GRIDS = (256, 512, 768, 1024)
CHAMBERS = {"circle": (0.04, 0.04), "ellipse": (0.09, 0.036)}  # R = 20 mm; half-axes 45 x 18 mm


def scan_configs(n=64, seed=4, cap=500_000, n_init=10_000, n_steps_table=2501, management_every=50):
    """The batched SEY / intensity scan: n runs drawn with `seed` from grids
    {256, 512, 768, 1024}^2 over circular (R = 20 mm) and elliptical
    (45 x 18 mm) chambers, delta_max ~ U(1.2, 2.0), bunch intensity
    ~ U(0.5e11, 1.5e11), dipole B_y ~ U(0, 8.33) T (a quarter of the runs
    field-free), each capped at `cap` macro-electrons by roulette."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        size = int(rng.choice(SCAN_GRIDS))
        chamber = str(rng.choice(sorted(CHAMBERS)))
        lx, ly = CHAMBERS[chamber]
        by = 0.0 if rng.random() < 0.25 else float(rng.uniform(0.0, 8.33))
        out.append(dict(nx=size, ny=size, lx=lx, ly=ly, boundType=1, n_init=n_init, target=cap,
                        sey_max=float(rng.uniform(1.2, 2.0)), beam_particles=float(rng.uniform(0.5e11, 1.5e11)),
                        type_b_field=1 if by > 0 else 0, b_const=(0.0, by, 0.0), seed=1000 + i,
                        n_steps_table=n_steps_table, management_every=management_every))
    return out


def run_cost(cfg):
    """Relative cost of one run's step: its grid nodes (the Poisson solve and
    the per-node kernels) plus its macro-electron cap (the particle kernels)."""
    nx, ny = cfg.get("nx", 128), cfg.get("ny", cfg.get("nx", 128))
    return (nx + 2) * (ny + 2) + int(cfg.get("target", 100000))


def shard_runs(runs, rank, world):
    """The indices of the runs of `rank` out of `world`: each run, costliest
    first, goes to the least loaded rank (ties to the lower rank), so every
    rank gets a similar share of the work without any data exchange during
    the runs."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must be in [0, world)")
    order = sorted(range(len(runs)), key=lambda i: (-run_cost(runs[i]), i))
    load = [0] * world
    mine = []
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        load[r] += run_cost(runs[i])
        if r == rank:
            mine.append(i)
    return sorted(mine)


def gather_histories(indices, histories, n_runs, group=None):
    """Rank 0 receives every run's (macro count, sum of weights) history in
    run order (other ranks get None): the one exchange of a sharded scan,
    after the runs (torch.distributed, any backend)."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    local = list(zip(indices, [(np.asarray(n), np.asarray(w)) for n, w in histories]))
    parts = [None] * world
    dist.all_gather_object(parts, local, group=group)
    if dist.get_rank(group) != 0:
        return None
    out = [None] * n_runs
    for part in parts:
        for i, h in part:
            out[i] = h
    if any(h is None for h in out):
        raise RuntimeError("a run's history is missing")
    return out
