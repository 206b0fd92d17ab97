"""Device autotuner for the buildup driver's tunable sizes.

Every choice is made by timing the candidates on the GPU the run uses (CUDA
events) on the run's own grid, and remembered per key for the process (and in
a JSON file when a path is given, so a scan of many runs measures each key
once):

* Poisson solve per grid: the LU back-substitution against the
  multigrid-preconditioned iterative solve at the solver's tolerance, timed
  warm-started as in a time step (the previous step's phi of a 0.1 %-different
  charge); a tie keeps LU (it is exact without iterating).
* Multigrid block size per grid: the largest level (nodes) handed to the
  one-CTA shared-memory solve of the V-cycle (a tile of the hierarchy): small
  blocks give the coarse levels to the tiled kernels (more launches), large
  ones leave one SM with more of the work.
* Branch width of a batched step graph (`openecloud_b200.batch`): how many
  graph branches (streams) the runs of a batch are spread over.

No reference counterpart: the reference has one solver and runs one
simulation at a time.
"""
import json
import os

import numpy as np
import torch

from . import device as D

MG_BLOCK_TOPS = (320, 1280, 4608, 9000)


def _time(fn, reps):
    """Mean device milliseconds of fn() after one warm-up call."""
    s = torch.cuda.current_stream()
    fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    for _ in range(reps):
        fn()
    e1.record(s)
    e1.synchronize()
    return e0.elapsed_time(e1) / reps


def test_charge(grid, seed=11, n=16):
    """A smooth charge per node inside the chamber (sum of Gaussians of
    sigma 2-8 % of the chamber size), scaled like a buildup's."""
    rng = np.random.default_rng(seed)
    nx, ny = grid.getNxExt(), grid.getNyExt()
    x = (np.arange(nx) - (nx - 1) / 2) * grid.getDx()
    y = (np.arange(ny) - (ny - 1) / 2) * grid.getDy()
    X, Y = np.meshgrid(x, y)
    rho = np.zeros_like(X)
    for _ in range(n):
        cx, cy = rng.uniform(-0.4, 0.4, 2) * np.array([x[-1], y[-1]])
        s = rng.uniform(0.02, 0.08) * min(x[-1], y[-1])
        rho += rng.uniform(0.5, 1.5) * np.exp(-((X - cx) ** 2 + (Y - cy) ** 2) / (2 * s * s))
    ins = np.asarray(grid.getInsidePoints()).reshape(ny, nx) != 0
    return (np.where(ins, rho, 0.0) * 1e-12).ravel()


class Autotuner:
    """Chooses sizes by measurement; `choices` holds every decision with the
    timings it was made from."""

    def __init__(self, path=None, reps=5):
        self.path = path
        self.reps = int(reps)
        self.choices = {}
        if path and os.path.exists(path):
            with open(path) as f:
                self.choices = json.load(f)

    def _save(self):
        if self.path:
            with open(self.path, "w") as f:
                json.dump(self.choices, f, indent=1, sort_keys=True)

    @staticmethod
    def grid_key(grid):
        return f"{grid.nx}x{grid.ny}_{grid.lx:g}x{grid.ly:g}_b{grid.boundType}"

    def mg_block_top(self, ps):
        """Largest multigrid level of the one-CTA solve for this solver's
        grid, by V-cycle time; builds the solver's hierarchy with it."""
        import ctypes
        from .poissonSolver import _declare
        key = "mg_block_top/" + self.grid_key(ps.gridObj)
        if key not in self.choices:
            G = ps.n_nodes
            r = D.to_device(np.where(D.to_numpy(ps._keep["inside"]) != 0,
                                     np.random.default_rng(0).normal(size=G), 0.0), torch.float32)
            z = D.zeros(G, torch.float32)
            L = _declare()
            times = {}
            for top in MG_BLOCK_TOPS:
                mg = ps._mg_setup(block_top=top)
                c = mg["c"]
                times[str(top)] = _time(lambda: L.oec_mg_apply(ctypes.byref(c), r.data_ptr(), z.data_ptr(),
                                                                D.stream()), 4 * self.reps)
            best = min(times, key=times.get)
            self.choices[key] = {"choice": int(best), "ms_per_vcycle": times}
            self._save()
        top = self.choices[key]["choice"]
        ps._mg_setup(block_top=top)
        return top

    def poisson(self, ps):
        """'lu' or 'mg' for this solver's grid (sets ps.method / ps.precond)."""
        key = "poisson/" + self.grid_key(ps.gridObj)
        self.mg_block_top(ps)
        if key not in self.choices:
            q = test_charge(ps.gridObj)
            qd = D.to_device(q, torch.float64)
            q2 = D.to_device(q * (1.0 + 1e-3 * np.sin(np.linspace(0, 2 * np.pi, q.size))), torch.float64)
            times = {}
            saved = (ps.method, ps.precond, ps.warmStart)
            ps.method = "lu"
            times["lu"] = _time(lambda: ps.solveDevice(qd), self.reps)
            ps.method, ps.precond, ps.warmStart = "pcg", "mg", "previous"

            def warm():
                ps.solveDevice(qd)
                ps.solveDevice(q2)
            times["mg"] = _time(warm, self.reps) / 2.0
            ps.method, ps.precond, ps.warmStart = saved
            best = "mg" if times["mg"] < times["lu"] else "lu"
            self.choices[key] = {"choice": best, "ms_per_solve": times}
            self._save()
        best = self.choices[key]["choice"]
        if best == "mg":
            ps.method, ps.precond = "pcg", "mg"
        else:
            ps.method = "lu"
        return best

    def branches(self, key, candidates, trial):
        """Fastest candidate by trial(c) -> ms (each trial does real work)."""
        key = "branches/" + key
        if key not in self.choices:
            times = {str(c): trial(c) for c in candidates}
            best = min(times, key=times.get)
            self.choices[key] = {"choice": int(best), "ms_per_step": times}
            self._save()
        return self.choices[key]["choice"]
