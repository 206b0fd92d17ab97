"""Device-resident electron-cloud buildup loop.

The reference's time loop (example01_basic.py:52-97) as one sequence of
liboec launches per step with every count kept on the device, so a step needs
no host synchronisation and can be captured once in a CUDA graph and
replayed.  Per step:

  1. Poisson right-hand side: fixed-point electron deposit (done by the
     previous step) + beam imprint table[step] * profile   (oec_rhs_with_beam)
  2. phi = A^-1 q, E = phiToE phi                          (oec_lu_solve, oec_spmv_csr)
  3. E -> cell corner table                                 (oec_field_prepare)
  4. gather + Boris push + move + wall test + deposit of the survivors
                                                            (oec_push_gather)
  5. absorbed indices, rows, wall point + normal            (oec_absorbed_index,
                                                             oec_save_absorbed,
                                                             oec_wall_interaction)
  6. Furman emission                                        (oec_furman_emit)
  7. refill in the reference's slot order (secondaries into
     holes, shift or append), deposit of the secondaries
     for the next step                                      (oec_add_remove)
  8. history (count, sum w) and ++step                      (oec_history, oec_step_advance)

Particle management (globalRandom / localRandom) runs between graph replays
at the reference's cadence; it re-deposits and refreshes the fixed-point
scale.

Particle order is physics here: the reference's Furman emitter gives a lone
secondary the elastic / rediffused / true-secondary split of the LAST
absorbed particle of the step (particleEmitter.pyx:245-246), so which particle
is last matters.  The refill puts every particle in the slot the reference's
array gives it (all three placement routines of particles.pyx, with the
array's row count tracked on the device), and the driver does not sort by
default.
Periodic cell sorting (`sort_every`) helps the deposit's warp aggregation but
is only order-neutral with the emitter's `compat` switch off.
"""
import time

import numpy as np
import torch

from . import _lib
from . import device as D
from .beam import LHCBeam, LHCBeamEndless
from .grid import Grid
from .particleBoundary import AbsorbElliptical, AbsorbRectangular, AbsorbArbitraryCutCell
from .particleEmitter import FurmanEmitter, SecElecEmitter, SimpleSecEmitter, homoLoader
from .particleManagement import globalRandom, localRandom
from .particles import Particles
from .poissonSolver import PoissonSolver, _declare as _poisson_declare


class Buildup:
    """A buildup run: grid, particles, boundary, emitter, Poisson solver, beam.

    Parameters mirror the configuration of example01_basic.py; `capacity`
    bounds the device particle store (the run reports a capacity drop in the
    status block instead of writing past it).  `b_multipoles` / `b_skew`
    (T/m^n) replace the constant field by the multipole field of
    magneticField.multipoleExpansion, gathered per particle (typeBField 2).
    `emitter` picks the secondary-emission model: 'furman' (FurmanEmitter,
    `material`, `sey_max`, `e_hat0`), 'secelec' (SecElecEmitter, stainless,
    `sey_max`) or 'simple' (SimpleSecEmitter).
    `poisson` reuses a
    PoissonSolver built for the same grid (its factorisation is the costly
    part of the setup on large grids; `PoissonSolver.sibling()` gives another
    run its own state over the same factors) and `grid` a Grid of the same
    parameters (read-only geometry, shareable between runs)."""

    def __init__(self, nx=128, ny=128, lx=0.04, ly=0.04, boundType=1, n_init=10000, w_init=None, dt=1e-11,
                 beam="endless", beam_particles=1.1e11, radius_sigma=0.002, bunch_length_sigma=0.25e-9 * 299792458.0,
                 material="copper", sey_max=1.6, e_hat0=300.0, type_b_field=0, b_const=(0., 0., 0.),
                 target=100000, management="global", management_every=50, capacity=None, seed=0,
                 n_steps_table=2500, sort_every=0, boundFunc=None, poisson=None, grid=None, b_multipoles=None,
                 b_skew=(), emitter="furman", abs_cap=None, metrics_log=None):
        if grid is not None and (grid.nx, grid.ny, grid.lx, grid.ly, grid.boundType) != (nx, ny, lx, ly, boundType):
            raise ValueError("grid: another grid than nx, ny, lx, ly, boundType describe")
        self.grid = grid if grid is not None else Grid(nx, ny, lx, ly, boundType, boundFunc=boundFunc)
        self.dt = float(dt)
        self.target = int(target)
        self.management = management
        self.management_every = int(management_every)
        self.sort_every = int(sort_every)
        self.seed = int(seed)
        self.type_b = int(type_b_field)
        cap = capacity or max(4 * self.target, 4 * n_init, 65536)
        self.P = Particles("electrons", "variableWeight", capacity=cap)
        self.P.setBConst(b_const)
        if boundType == 0:
            self.bd = AbsorbRectangular(self.grid, self.P)
        elif boundType == 1:
            self.bd = AbsorbElliptical(self.grid, self.P)
        else:
            self.bd = AbsorbArbitraryCutCell(self.grid, self.P)
        w_init = w_init if w_init is not None else 1e9 / n_init
        homoLoader(self.grid, self.P, self.bd, n_init, w_init, seed=seed)
        if emitter == "furman":
            self.em = FurmanEmitter(self.bd, self.P, material=material, seyMax=sey_max, seed=seed + 17)
            if e_hat0 is not None:
                self.em.setEHat0(e_hat0)
        elif emitter == "secelec":
            self.em = SecElecEmitter(self.bd, self.P, seyMax=sey_max, seed=seed + 17)
        elif emitter == "simple":
            self.em = SimpleSecEmitter(self.bd, self.P, seed=seed + 17)
        else:
            raise ValueError("emitter must be 'furman', 'secelec' or 'simple'")
        if poisson is not None and (poisson.gridObj.getNxExt(), poisson.gridObj.getNyExt()) != \
                (self.grid.getNxExt(), self.grid.getNyExt()):
            raise ValueError("poisson: a solver for another grid")
        self.ps = poisson if poisson is not None else PoissonSolver(self.grid)
        beam_cls = LHCBeamEndless if beam == "endless" else LHCBeam
        self.beam = beam_cls(self.grid, self.dt, nParticles=beam_particles, radiusSigma=radius_sigma,
                             bunchLengthSigma=bunch_length_sigma)
        self._table_len = int(n_steps_table)
        self.beam_profile = D.to_device(self.beam.getTransversalProfile(), torch.float64)
        self.beam_table = D.to_device(self.beam.scalarTable(self._table_len), torch.float64)
        G = self.grid.getNpExt()
        self.step_dev = D.zeros(1, torch.int32)
        self.rho = D.zeros(G, torch.float64)
        self.etab = D.zeros(8 * G, torch.float32)
        self.btab = None
        if b_multipoles is not None:
            # multipole field on the nodes (example04_multipole.py:45), gathered
            # per particle in the fused kernel (typeBField 2)
            from .magneticField import multipoleExpansionDevice
            b = multipoleExpansionDevice(self.grid, b_multipoles, b_skew)
            self.btab = self.P.fieldTable(self.grid, b, 3)
            self.type_b = 2
        self.hist_w = D.zeros(self._table_len, torch.float64)
        self.hist_n = D.zeros(self._table_len, torch.int32)
        self.scratch = D.zeros(256, torch.float64)  # oec_history's partial sums
        # absorbed rows per step: by default the store's capacity, so that no
        # step can absorb more (a bunch can sweep the whole cloud into the
        # wall at once); a smaller abs_cap saves memory, and a step that
        # absorbs more than it is counted on the device (status
        # n_rows_dropped) and run() raises
        self.abs_cap = int(abs_cap) if abs_cap is not None else max(4096, cap)
        self.bd.ensure_buffers(self.abs_cap)
        # the store does not grow inside a run: at most `cap` secondaries can be added per step
        self.em.out_cap = cap
        self.em.ensure_buffers(self.bd._rows.shape[0])
        self.P._deposit_buffers(self.grid)
        self.P._hole_buffers()
        self.P.c_scratch()  # allocated before any capture
        self._prepare_deposit()
        _lib.call("oec_history", self.P.c_particles(), self.step_dev.data_ptr(), self._table_len,
                  self.hist_w.data_ptr(), self.hist_n.data_ptr(), self.scratch.data_ptr(), D.stream())
        # what a checkpoint must match to be resumed by this run
        self._signature = {"grid": [int(nx), int(ny), float(lx), float(ly), int(boundType)], "dt": self.dt,
                           "seed": self.seed, "steps_table": self._table_len, "type_b": self.type_b,
                           "b_const": [float(b) for b in b_const], "emitter": emitter, "sey_max": float(sey_max),
                           "target": self.target, "management": management,
                           "management_every": self.management_every, "beam": beam,
                           "beam_particles": float(beam_particles)}
        self.metrics_log = metrics_log  # path: one JSON line per management interval
        self.graph = None
        self._rows_dropped = 0
        self.n_managed = 0       # management events (roulette / merge) so far
        self._graph_sig = None
        self._cap_stream = None
        self.steps_done = 0

    # ------------------------------------------------------------ pieces
    def _prepare_deposit(self):
        """Fixed-point scale from the current weights, then a full deposit."""
        P, s = self.P, D.stream()
        _lib.call("oec_deposit_scale", P.c_particles(), P._wscale.data_ptr(), s)
        _lib.call("oec_deposit", self.grid.c_grid(), P.c_particles(), P._rho_fix.data_ptr(), P._wscale.data_ptr(),
                  1, P._status.data_ptr(), s)

    def _launch_step(self):
        """All launches of one time step (no host synchronisation)."""
        P, g, bd, em, ps = self.P, self.grid, self.bd, self.em, self.ps
        s = D.stream()
        cg, cp, cb = g.c_grid(), P.c_particles(), bd.c_boundary()
        L = _lib.lib()
        _lib.call("oec_rhs_with_beam", cg, P._rho_fix.data_ptr(), P._wscale.data_ptr(), P.particleCharge,
                  self.beam_profile.data_ptr(), self.beam_table.data_ptr(), self.step_dev.data_ptr(),
                  self._table_len, self.rho.data_ptr(), s)
        ps.solveDevice(self.rho)
        _lib.call("oec_field_prepare", cg, ps.eAtGridPoints.data_ptr(), 2, self.etab.data_ptr(), s)
        _lib.call("oec_push_gather", cg, cp, self.etab.data_ptr(),
                  self.btab.data_ptr() if self.btab is not None else None, _lib.d3(P.bConst), self.dt,
                  P.particleCharge / P.particleMass, self.type_b, cb, P._mask.data_ptr(), P._rho_fix.data_ptr(),
                  P._wscale.data_ptr(), P._status.data_ptr(), s)
        _lib.call("oec_absorbed_index", cp, P._mask.data_ptr(), bd._index.data_ptr(), bd._index.shape[0],
                  bd._n_abs.data_ptr(), bd._scratch.data_ptr(), P._status.data_ptr(), s)
        cap = bd._rows.shape[0]
        _lib.call("oec_save_absorbed", cg, cp, bd._index.data_ptr(), bd._n_abs.data_ptr(), cap, bd._rows.data_ptr(),
                  s)
        _lib.call("oec_wall_interaction", cg, cb, self.dt, bd._rows.data_ptr(), bd._n_abs.data_ptr(), cap,
                  bd._normals.data_ptr(), P._status.data_ptr(), s)
        em._launch(cap, 0, self.step_dev, None)
        _lib.call("oec_add_remove", cg, cp, P.c_scratch(), P._mask.data_ptr(), bd._index.data_ptr(),
                  bd._n_abs.data_ptr(), bd._index.shape[0], em._out.data_ptr(), em._n_out.data_ptr(),
                  em._out.shape[0], P._array_len.data_ptr(), P._rho_fix.data_ptr(), P._wscale.data_ptr(),
                  P._status.data_ptr(), s)
        _lib.call("oec_step_advance", self.step_dev.data_ptr(), s)
        # state at the start of the next step, before its management
        # (example01_basic.py:56-57 records it there)
        _lib.call("oec_history", cp, self.step_dev.data_ptr(), self._table_len, self.hist_w.data_ptr(),
                  self.hist_n.data_ptr(), self.scratch.data_ptr(), s)
        del L

    def _log_metrics(self, step):
        """Appends one JSON line to metrics_log: the state at the start of
        `step` (macro count, sum of weights), the anomaly counters and the
        last iterative solve's statistics."""
        import json
        n = int(self.hist_n[step].item()) if step < self._table_len else None
        w = float(self.hist_w[step].item()) if step < self._table_len else None
        rec = {"step": step, "macro_particles": n, "sum_weights": w, "managed": self.n_managed,
               "status": {k: v for k, v in self.P.status().items() if v}}
        st = self.ps.lastStats
        if st is not None:
            rec["solve"] = {"iterations": st.iterations, "refinements": st.refinements, "converged": st.converged,
                            "rel_residual": st.rel_residual, "fallbacks": self.ps.nFallbacks}
        with open(self.metrics_log, "a") as f:
            f.write(json.dumps(rec) + "\n")

    def _check_rows(self):
        """Raises if a step absorbed more particles than the absorbed-row
        buffer holds: those particles were removed without a wall row and
        emitted no secondaries, so the run under-counts the build-up."""
        dropped = self.P.status()["n_rows_dropped"]
        if dropped > self._rows_dropped:
            self._rows_dropped = dropped
            raise RuntimeError(f"{dropped} absorbed particles exceeded the absorbed-row capacity ({self.abs_cap} rows "
                               "per step) and emitted nothing: build the run with a larger abs_cap")

    def _manage(self, step):
        self._check_rows()
        n = self.P.getMacroParticleCount()
        if step > 0 and step % self.management_every == 0 and (n > 1.05 * self.target or n < 0.95 * self.target):
            # draws keyed by the run's seed, the step and the run's own count
            # of management events: reproducible whatever else the process ran
            if self.management == "global":
                globalRandom(self.grid, self.P, self.target, seed=self.seed + step, call=self.n_managed + 1)
            elif self.management == "local":
                localRandom(self.grid, self.P, self.bd, self.target, seed=self.seed + step, call=self.n_managed + 1)
            else:
                return False
            self._prepare_deposit()
            self.n_managed += 1
            return True
        return False

    # -------------------------------------------------------------- run
    def run(self, n_steps, use_graph=True):
        """Advance n_steps; returns wall seconds on the device clock."""
        s = torch.cuda.current_stream()
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record(s)
        # emission draws are keyed by (seed, particle slot, device step
        # counter), so replays of one captured step draw fresh numbers
        k = 0
        while k < n_steps:
            step = self.steps_done + k
            if step >= self._table_len:
                raise ValueError("beam table exhausted: increase n_steps_table")
            if self.sort_every and step % self.sort_every == 0 and step > 0:
                self.P.sortByColumn(6)
            if step % self.management_every == 0:
                with torch.cuda.nvtx.range(f"management {step}"):
                    self._manage(step)
            # steps until the next management / sort point
            nxt = n_steps - k
            for every in (self.management_every, self.sort_every):
                if every:
                    nxt = min(nxt, every - (step % every))
            with torch.cuda.nvtx.range(f"buildup steps {step}..{step + nxt - 1}"):
                if use_graph:
                    self._replay(nxt)
                else:
                    for _ in range(nxt):
                        self._launch_step()
            k += nxt
            if self.metrics_log:
                self._log_metrics(step + nxt)
        t1.record(s)
        t1.synchronize()
        self.steps_done += n_steps
        self._check_rows()
        return t0.elapsed_time(t1) * 1e-3

    def _step_signature(self):
        """Everything a captured step bakes in: device buffers (a
        reallocation by management or sorting changes them) and the solver
        settings."""
        P, bd, em, ps = self.P, self.bd, self.em, self.ps
        bufs = (P._mask, P._rho_fix, P._wscale, P._status, P._array_len, bd._index, bd._rows, bd._normals,
                bd._n_abs, bd._scratch, em._work, em._out, em._n_out, self.btab)
        return (bytes(P.c_particles()), bytes(P.c_scratch()), tuple(0 if t is None else t.data_ptr() for t in bufs),
                bytes(em.c_params()),
                em.seed, ps.method, ps.precond, ps.warmStart, ps.pcgTol, ps.pcgMaxIter, id(ps.cnn))

    def _capture(self):
        """Records one time step into a CUDA graph (on a capture stream of its
        own; torch.cuda.graph's garbage collection per capture would cost
        more than the step)."""
        torch.cuda.nvtx.range_push("capture step graph")
        try:
            self._capture_step()
        finally:
            torch.cuda.nvtx.range_pop()

    def _capture_step(self):
        self.ps.prepare()
        if self._cap_stream is None:
            self._cap_stream = torch.cuda.Stream()
        cur = torch.cuda.current_stream()
        cs = self._cap_stream
        cs.wait_stream(cur)
        self.graph = None
        g = torch.cuda.CUDAGraph()
        with torch.cuda.stream(cs):
            g.capture_begin()
            try:
                self._launch_step()
            finally:
                g.capture_end()
        cur.wait_stream(cs)
        self.graph = g
        self._graph_sig = self._step_signature()

    def _replay(self, n):
        # A captured step holds raw device pointers: capture again when any
        # of them changed.
        if self.graph is None or self._graph_sig != self._step_signature():
            self._capture()
        for _ in range(n):
            self.graph.replay()

    # ------------------------------------------------------ checkpoints
    def save(self, directory):
        """Writes the reference's outputs (particleData.npy: (N, 6) float64
        rows; physicalParticleCount.npy and macroParticleCount.npy: the
        histories so far, example01_basic.py:76-78) and checkpoint.npz, the
        exact device state from which `load` resumes this run bit for bit."""
        from . import checkpoint as C
        P, ps = self.P, self.ps
        n = P.getMacroParticleCount()
        hist_n, hist_w = self.history()
        C.write_reference_outputs(directory, P.getParticleData(), hist_w[:-1], hist_n[:-1])
        store = {k: D.to_numpy(P.soa()[k][:n]) for k in C.STORE_FIELDS}
        arrays = {"rho_fix": D.to_numpy(P._rho_fix), "wscale": D.to_numpy(P._wscale),
                  "array_len": D.to_numpy(P._array_len),
                  "status": D.to_numpy(P._status), "step": D.to_numpy(self.step_dev),
                  "hist_n": D.to_numpy(self.hist_n), "hist_w": D.to_numpy(self.hist_w),
                  "phi": D.to_numpy(ps.phi),
                  "phi_prev": D.to_numpy(ps._phi_prev) if ps._phi_prev is not None else None,
                  "ws_hist": D.to_numpy(ps._ws_hist) if ps._ws_hist is not None else None}
        counters = {"steps_done": int(self.steps_done), "n_managed": int(self.n_managed),
                    "rows_dropped": int(self._rows_dropped)}
        C.write_checkpoint(directory, self._signature, store, arrays, counters)

    def load(self, directory):
        """Resumes the run saved by `save` into this one (built with the
        same configuration): the store, deposit, step counter, histories,
        warm-start state and counters are restored exactly."""
        from . import checkpoint as C
        store, arrays, counters = C.read_checkpoint(directory, self._signature)
        P, ps = self.P, self.ps
        n = store["cell"].shape[0]
        P.ensure_capacity(n)
        for k in C.STORE_FIELDS:
            P.soa()[k][:n].copy_(torch.from_numpy(store[k]))
        P._count.fill_(n)
        if "array_len" in arrays:
            P._array_len.copy_(torch.from_numpy(arrays["array_len"]))
        else:
            P._array_len.fill_(n)
        P._rho_fix.copy_(torch.from_numpy(arrays["rho_fix"]))
        P._wscale.copy_(torch.from_numpy(arrays["wscale"]))
        P._status.copy_(torch.from_numpy(arrays["status"]))
        self.step_dev.copy_(torch.from_numpy(arrays["step"]))
        self.hist_n.copy_(torch.from_numpy(arrays["hist_n"]))
        self.hist_w.copy_(torch.from_numpy(arrays["hist_w"]))
        ps.phi.copy_(torch.from_numpy(arrays["phi"]))
        if "phi_prev" in arrays:
            ps._phi_prev = D.to_device(arrays["phi_prev"], torch.float64)
            ps._ws_hist = D.to_device(arrays["ws_hist"], torch.int32)
        else:
            ps._phi_prev = ps._ws_hist = None
        self.steps_done = int(counters["steps_done"])
        self.n_managed = int(counters["n_managed"])
        self._rows_dropped = int(counters["rows_dropped"])
        self.graph = None  # the next replay captures again
        torch.cuda.synchronize()

    def loadParticleData(self, path):
        """Restarts from a particleData.npy of (N, 6) float64 rows, as the
        reference restarts through setParticleData (particles.pyx:126): the
        rows are converted to the FP32 store and deposited again."""
        from . import checkpoint as C
        self.P.setParticleData(C.read_particle_data(path))
        self._prepare_deposit()
        self.graph = None

    def history(self):
        """(macro count, sum of weights) at the start of every step so far."""
        n = self.steps_done + 1
        return D.to_numpy(self.hist_n[:n]), D.to_numpy(self.hist_w[:n])

    def status(self):
        return self.P.status()
