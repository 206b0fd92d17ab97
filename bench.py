"""Benchmark: particle-steps/s of the openECLOUD per-step particle kernels.

Workload (the kernel microbench configuration): 2^24 macro-electrons, uniform
inside a 512x512-node rectangular grid of 40x40 mm, Maxwellian velocities
(kT = 5 eV), uniform dipole B_y = 0.5 T (Boris type 1), E from a smooth
charge density (sum of 16 Gaussians, sigma 1-4 mm, seed 7), dt = 1e-11 s.
One step = gather E + Boris push + move + wall test + fixed-point deposit of
the survivors: the work of calcGridWeights + eFieldToParticles + borisPush
+ indexInside + chargeToGrid in the reference loop.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

At one GPU the line also carries "bunch_passage": seconds per bunch passage
of the c1 buildup (128x128 circular chamber, 2500 steps) on the device with
the LU, multigrid-PCG and Jacobi-PCG Poisson solves, next to the compiled
reference's passage on one host core (the other half of the headline
metric); and "production_passage": the 1024x1024 elliptical production
buildup sampled over 100 steps with the LU and multigrid-PCG solves, with
the single-solve comparison on that grid (LU against the iterative solve at
relative residual 1e-8); and "batched_scan": 64 independent runs of uneven
grids advanced in one graph per batch step, with the autotuner's choices.

N > 1 runs under torchrun, one rank per GPU; every rank advances its own
2^24 particles (independent shards, no collective on the data path:
weak scaling).  Rank 0 prints one JSON line.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

QE = 1.602176565e-19
ME = 9.10938291e-31
EPS0 = 8.85418781762e-12
METRIC = "particle-steps/s"

# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one launch of
# the fused kernel, by store size, from an ncu capture of
#   python bench.py --particles 8388608 --steps 2 --warmup 3 --e2e-steps 0 --no-cpu-baseline --no-passage
#       --no-production --no-batch --no-components
# (ncu --metrics dram__bytes_read.sum,dram__bytes_write.sum --clock-control none -k regex:k_push_gather -s 3 -c 1):
# the particle part scaled by 2 to 2^24 electrons, the grid part (E table and
# deposit grid, 12.7 MB) added once.
NCU_TRAFFIC_PER_LAUNCH = {1 << 24: 773544608}


# ------------------------------------------------------------- workload
def workload(n, nodes=512, seed=7):
    """Synthetic c2 inputs: particle rows (cell-sorted) and the node E field."""
    rng = np.random.default_rng(seed)
    lx = ly = 0.04
    dx = lx / (nodes - 1.)
    nx = nodes + 2
    lxh = (lx + 2 * dx) * 0.5
    pd = np.empty((n, 6), np.float64)
    pd[:, 0] = rng.uniform(-lx / 2, lx / 2, n)
    pd[:, 1] = rng.uniform(-ly / 2, ly / 2, n)
    sv = np.sqrt(5.0 * QE / ME)  # Maxwellian, kT = 5 eV, per component
    pd[:, 2:5] = rng.normal(0.0, sv, (n, 3))
    pd[:, 5] = 1e9 / n
    # cell-sorted order (the store keeps particles grouped by cell)
    ix = np.floor((pd[:, 0] + lxh) / dx).astype(np.int64)
    iy = np.floor((pd[:, 1] + lxh) / dx).astype(np.int64)
    pd = pd[np.argsort(ix + iy * nx, kind="stable")]
    # E of 16 Gaussian line-charge blobs (free-space closed form on the nodes)
    xm = np.linspace(-lxh, lxh, nx)
    X, Y = np.meshgrid(xm, xm)
    Ex = np.zeros_like(X)
    Ey = np.zeros_like(X)
    for _ in range(16):
        cx, cy = rng.uniform(-0.012, 0.012, 2)
        s = rng.uniform(1e-3, 4e-3)
        Q = rng.uniform(-1, 1) * 1e-9
        rx, ry = X - cx, Y - cy
        r2 = rx * rx + ry * ry + 1e-30
        f = Q / (2 * np.pi * EPS0) * (1 - np.exp(-r2 / (2 * s * s))) / r2
        Ex += f * rx
        Ey += f * ry
    E = np.concatenate([Ex.reshape(-1), Ey.reshape(-1)])
    return pd, E, (nodes, nodes, lx, ly)


# --------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.f = None

    def start(self):
        try:
            self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.gpu)], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": []}
        if self.proc is None:
            return out
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.flush()
        self.f.seek(0)
        rows = [l.strip().split(",") for l in self.f.read().splitlines() if l.strip()]
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
                for k, v in zip(names, r[5:9]):
                    if v.strip().lower() in ("active", "1"):
                        reasons.add(k)
            except Exception:
                continue
        if sm:
            out["sm_mhz"] = float(np.median(sm))
            out["sm_max_mhz"] = float(np.max(mx))
        out["reasons"] = sorted(reasons)
        out["samples"] = len(sm)
        return out


# ----------------------------------------------------------- CPU legs
def _ref_modules():
    ref = os.path.join(ROOT, "oracle", "_ref")
    if not os.path.exists(os.path.join(ref, "ref_compat.py")):
        return None
    sys.path.insert(0, ref)
    try:
        import ref_compat  # noqa: F401
        import grid as rgrid
        import particles as rparticles
        import particleBoundary as rboundary
        return rgrid, rparticles, rboundary
    except Exception:
        return None


def cpu_reference_steps(pd, E, geom, min_seconds, max_steps, min_steps=1, warm=0):
    """Time the compiled reference's own step (weights, deposit, gather, push,
    wall test) on the rows `pd` of the workload, after `warm` untimed steps;
    falls back to the C oracle port when the reference is not built."""
    n_sample = pd.shape[0]
    nx, ny, lx, ly = geom
    mods = _ref_modules()
    steps = 0
    if mods is not None:
        rgrid, rparticles, rboundary = mods
        g = rgrid.Grid(nx, ny, lx, ly, 0)
        P = rparticles.Particles("electrons", "variableWeight")
        P.setParticleData(pd.copy())
        P.setBConst(np.array([0.0, 0.5, 0.0]))
        bd = rboundary.AbsorbRectangular(g, P)
        kind = "reference"

        def step():
            P.calcGridWeights(g)
            P.chargeToGrid(g)
            P.eFieldToParticles(g, E)
            P.borisPush(1e-11, 1)
            bd.indexInside()
    else:
        from oracle import oracle as O
        og = O.GridGeom(nx, ny, lx, ly)
        state = {"pd": pd.copy()}
        kind = "port"
        qm = -QE / ME

        def step():
            p = state["pd"]
            O.charge_to_grid(p, og, -QE)
            e = O.field_to_particles(p, og, E, 2)
            state["pd"] = O.boris_push(p, e, 1e-11, qm, 1, bconst=[0.0, 0.5, 0.0])
            O.index_inside(state["pd"], og, 0)
    # Every timed step starts from the same in-grid rows: the reference
    # indexes its grid unchecked (particles.pyx:410-411), so particles may not
    # be left to drift out of the extended grid over many steps.
    def reload():
        if mods is not None:
            P.setParticleData(pd.copy())
        else:
            state["pd"] = pd.copy()
    for _ in range(warm):
        reload()
        step()
    dt = 0.0
    t_all = time.perf_counter()
    while steps < min_steps or (time.perf_counter() - t_all < min_seconds and steps < max_steps):
        reload()
        t0 = time.perf_counter()
        step()
        dt += time.perf_counter() - t0
        steps += 1
    return {"value": n_sample * steps / dt, "unit": METRIC, "cores": 1, "kind": kind, "steps": steps,
            "sample": f"the whole workload ({n_sample} particles) x {steps} steps, each from the same rows "
                      f"(512x512 rect, B_y=0.5 T), single thread ({dt:.1f} s)"}


def bench_config(n, nx, ny, world):
    """The workload description both arms print (one config for the ratio)."""
    return {"workload": "kernel microbench: 2^24 macro-electrons per GPU, 512x512 rect grid 40x40 mm, Maxwellian "
                        "5 eV, B_y=0.5 T, fused gather+Boris+move+wall test+int64 deposit, dt=1e-11 s",
            "particles_per_gpu": n, "grid_nodes": [nx + 2, ny + 2],
            "parallelism": f"{world} independent particle shards",
            "l2": "inputs 470 MB per step > 126 MB L2 (no flush needed)"}


def cpu_reference_c3(n_particles=2_000_000, solves=3):
    """The compiled reference on the production shapes, on one host core:
    SuperLU setup and back-substitution + E on the 512x512 and 1024x1024
    ellipses (45 x 18 mm half-axes), and one particle step of 2e6 electrons
    on the 1024x1024 ellipse at B_y = 8.33 T (weights, deposit, gather, Boris
    push, wall test); a production passage (5000 steps) is estimated as
    5000 x (solve + particle step).  None without oracle/_ref."""
    mods = _ref_modules()
    if mods is None:
        return None
    rgrid, rparticles, rboundary = mods
    import poissonSolver as rps
    out = {"cores": 1, "kind": "reference"}
    for nodes in (512, 1024):
        g = rgrid.Grid(nodes, nodes, 0.09, 0.036, 1)
        t0 = time.perf_counter()
        ps = rps.PoissonSolver(g)
        setup = time.perf_counter() - t0
        q = np.zeros(g.getNpExt())
        ins = np.asarray(g.getInsidePoints()) != 0
        q[ins] = np.random.default_rng(1).uniform(0, 1e-12, int(ins.sum()))
        ps.solve(q)
        t0 = time.perf_counter()
        for _ in range(solves):
            ps.solve(q)
        out[f"lu_solve_ms_{nodes}"] = (time.perf_counter() - t0) / solves * 1e3
        out[f"lu_setup_s_{nodes}"] = setup
    rng = np.random.default_rng(3)
    r = np.sqrt(rng.uniform(0, 1, n_particles)) * 0.99
    a = rng.uniform(0, 2 * np.pi, n_particles)
    pd = np.zeros((n_particles, 6))
    pd[:, 0], pd[:, 1] = r * np.cos(a) * 0.045, r * np.sin(a) * 0.018
    pd[:, 2:5] = rng.normal(0.0, np.sqrt(5.0 * QE / ME), (n_particles, 3))
    pd[:, 5] = 1e3
    P = rparticles.Particles("electrons", "variableWeight")
    P.setParticleData(pd)
    P.setBConst(np.array([0.0, 8.33, 0.0]))
    bd = rboundary.AbsorbElliptical(g, P)
    E = np.zeros(2 * g.getNpExt())

    def step():
        P.calcGridWeights(g)
        P.chargeToGrid(g)
        P.eFieldToParticles(g, E)
        P.borisPush(5e-12, 1)
        bd.indexInside()
    step()
    P.setParticleData(pd.copy())
    t0 = time.perf_counter()
    step()
    out["particle_step_ms_2e6"] = (time.perf_counter() - t0) * 1e3
    out["s_per_passage_estimate"] = 5000 * (out["lu_solve_ms_1024"] + out["particle_step_ms_2e6"]) * 1e-3
    out["sample"] = (f"{solves} solves per grid after one untimed; one particle step of {n_particles} electrons; "
                     "passage = 5000 x (1024^2 solve + particle step)")
    return out


def _ref_scan_worker(args):
    """One run of the batched scan on the compiled reference (its own loop,
    oracle/ref_buildup.py): seconds of `steps` steps after the setup."""
    cfg, steps = args
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_buildup
    t = {}
    ref_buildup.reference_buildup(int(cfg["seed"]), steps, nx=cfg["nx"], ny=cfg["ny"], lx=cfg["lx"], ly=cfg["ly"],
                                  boundType=cfg["boundType"], n_init=cfg["n_init"], target=cfg["target"], timing=t)
    return t["seconds"]


def cpu_reference_scan(n_runs=64, steps=50):
    """The batched scan on the host cores, process-parallel: K = nproc
    single-threaded processes of the compiled reference's loop, each on one
    run of the scan (the first K runs of the 64), `steps` steps each; the
    throughput is K * steps run-steps over the slowest process's time.  The
    reference's loop has no dipole field or SEY scan (c1's emitter and beam
    on each run's grid and chamber)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    try:
        import ref_buildup
    except Exception:
        return None
    if not ref_buildup.available():
        return None
    import multiprocessing as mp
    from openecloud_b200.batch import scan_configs
    k = os.cpu_count() or 1
    cfgs = scan_configs(n_runs)[:k]
    t0 = time.perf_counter()
    with mp.get_context("spawn").Pool(k) as pool:
        secs = pool.map(_ref_scan_worker, [(c, steps) for c in cfgs])
    wall = time.perf_counter() - t0
    return {"run_steps_per_s": k * steps / max(secs), "processes": k, "cores": k, "kind": "reference",
            "steps_per_run": steps, "slowest_run_s": max(secs), "wall_s_with_setup": wall,
            "grids": [f"{c['nx']}^2" for c in cfgs],
            "sample": f"{k} single-threaded processes (process-parallel), one scan run each, {steps} steps"}


PASSAGE = ("c1 buildup: 128x128 circular chamber R=20 mm, 1e4 initial electrons at rest, endless train "
           "1.1e11 p/bunch, sigma_r 2 mm, sigma_t 0.25 ns, 25 ns spacing, copper SEY deltaMax 1.6 (Emax 300 eV), "
           "roulette cap 1e5 every 50 steps, dt=1e-11 s; one bunch passage = 2500 steps")


def cpu_reference_passage():
    """Wall seconds of one bunch passage of the compiled reference's own loop
    (oracle/ref_buildup.py) on one host core; None without oracle/_ref."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    try:
        import ref_buildup
    except Exception:
        return None
    if not ref_buildup.available():
        return None
    t = {}
    ref_buildup.reference_buildup(100, 2500, timing=t)
    return {"s_per_passage": t["seconds"], "cores": 1, "kind": "reference",
            "sample": "one full passage (2500 steps) of the compiled reference's loop, seed 100"}


def gpu_passage():
    """Device seconds of one bunch passage of the buildup driver with each
    Poisson solve, every time step replayed from one captured graph: LU
    (f64, level-scheduled + dense tail), the multigrid-preconditioned
    iterative solve (f64 residual 1e-8, its loops inside the step graph, LU
    fallback on the device) over the whole passage, and the Jacobi-
    preconditioned one over its first 250 steps, scaled to 2500."""
    from openecloud_b200.buildup import Buildup
    Buildup(seed=999, n_steps_table=60).run(50)  # warm-up: module load, kernel attributes
    b = Buildup(seed=1000, n_steps_table=2501)
    s_lu = b.run(2500)
    nfin = int(b.history()[0][-1])
    out = {"workload": PASSAGE, "s_per_passage": s_lu, "solver": "LU (f64, level-scheduled + dense tail)",
           "final_macro_particles": nfin}
    m = Buildup(seed=1000, n_steps_table=2501)
    m.ps.method, m.ps.precond = "pcg", "mg"
    out["s_per_passage_pcg_mg"] = m.run(2500)
    out["pcg_mg_fallbacks"] = m.ps.nFallbacks
    out["pcg_mg_final_macro_particles"] = int(m.history()[0][-1])
    j = Buildup(seed=1000, n_steps_table=2501)
    j.ps.method, j.ps.precond = "pcg", "jacobi"
    out["s_per_passage_pcg_jacobi"] = j.run(250) * 10.0
    out["pcg_jacobi_sample"] = "first 250 steps x 10"
    out["pcg_jacobi_fallbacks"] = j.ps.nFallbacks
    out["timing"] = "device time (CUDA events) of the whole passage, state resident on the GPU, step graphs replayed"
    return out


PRODUCTION = ("production buildup (sampled): 1024x1024 grid over an elliptical chamber with half-axes 45x18 mm, "
              "dipole B_y=8.33 T, 25 ns train of 1.15e11 p/bunch (sigma_r 1 mm, sigma_t 0.25 ns), SEY deltaMax 1.8, "
              "2.2e6 initial macro-electrons, kd-tree merge (localRandom) toward 2e6 every 10 steps, dt=5e-12 s; "
              "one bunch passage = 5000 steps")


def _smooth_charge(grid, seed=11, n=16):
    """Charge per node from a sum of Gaussians (sigma 1-4 mm) inside the chamber."""
    rng = np.random.default_rng(seed)
    nx, ny = grid.getNxExt(), grid.getNyExt()
    x = (np.arange(nx) - (nx - 1) / 2) * grid.getDx()
    y = (np.arange(ny) - (ny - 1) / 2) * grid.getDy()
    X, Y = np.meshgrid(x, y)
    rho = np.zeros_like(X)
    for _ in range(n):
        cx, cy = rng.uniform(-0.5, 0.5, 2) * np.array([x[-1], y[-1]])
        s = rng.uniform(1e-3, 4e-3)
        rho += rng.uniform(0.5, 1.5) * np.exp(-((X - cx) ** 2 + (Y - cy) ** 2) / (2 * s * s))
    ins = np.asarray(grid.getInsidePoints()).reshape(ny, nx) != 0
    return (np.where(ins, rho, 0.0) * 1e-12).ravel()


def poisson_comparison(ps, reps=10):
    """Solve times on one grid: LU against the iterative solve (f64 residual
    1e-8) with the multigrid preconditioner (cold: zero start; warm: from
    the solution of a 0.1 % different charge, as between time steps) and
    with the Jacobi one (cold)."""
    import torch
    from openecloud_b200 import device as D
    q = _smooth_charge(ps.gridObj)
    qd = D.to_device(q, torch.float64)
    q2 = D.to_device(q * (1.0 + 1e-3 * np.sin(np.linspace(0, 2 * np.pi, q.size))), torch.float64)
    s = torch.cuda.current_stream()

    def timed(fn, n):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        for _ in range(n):
            fn()
        e1.record(s)
        e1.synchronize()
        return e0.elapsed_time(e1) / n

    out = {}
    saved = (ps.method, ps.precond, ps.warmStart)
    ps.method = "lu"
    out["lu_ms"] = timed(lambda: ps.solveDevice(qd), reps)
    phi_lu = D.to_numpy(ps.phi)
    fb0 = ps.nFallbacks
    ps.method, ps.precond, ps.warmStart = "pcg", "mg", "zero"
    out["mg_cold_ms"] = timed(lambda: ps.solveDevice(qd), reps)
    st = ps.lastStats
    out["mg_cold_iterations"], out["mg_cold_refinements"] = st.iterations, st.refinements
    out["mg_vs_lu_max_rel"] = float(np.abs(D.to_numpy(ps.phi) - phi_lu).max() / np.abs(phi_lu).max())
    ps.warmStart = "previous"

    def warm():
        ps.solveDevice(qd)
        ps.solveDevice(q2)
    out["mg_warm_ms"] = timed(warm, reps) / 2.0
    st = ps.lastStats
    out["mg_warm_iterations"], out["mg_warm_rel_residual0"] = st.iterations, st.rel_residual0
    ps.precond, ps.warmStart = "jacobi", "zero"
    out["jacobi_cold_ms"] = timed(lambda: ps.solveDevice(qd), 2)
    out["jacobi_cold_iterations"] = ps.lastStats.iterations
    out["fallbacks"] = ps.nFallbacks - fb0
    ps.method, ps.precond, ps.warmStart = saved
    out["tol"] = 1e-8
    out["timing"] = "device time (CUDA events) per solve, charge resident on the GPU"
    return out


def production_passage(steps=100, warm=10):
    """The production buildup (1024x1024 ellipse, 2e6 electrons, kd-tree
    merge every 10 steps) sampled over `steps` steps after `warm` untimed
    ones, with the LU and the multigrid-preconditioned iterative Poisson
    solve (one factorisation shared), scaled to a 5000-step passage; plus the
    solve comparison on the same 1024x1024 elliptical grid."""
    import torch
    from openecloud_b200.buildup import Buildup
    kw = dict(nx=1024, ny=1024, lx=0.09, ly=0.036, boundType=1, n_init=2_200_000, w_init=1e3, dt=5e-12,
              beam_particles=1.15e11, radius_sigma=1e-3, sey_max=1.8, type_b_field=1, b_const=(0., 8.33, 0.),
              target=2_000_000, management="local", management_every=10, n_steps_table=steps + warm + 25, seed=2000,
              abs_cap=4_400_000)
    t0 = time.perf_counter()
    lu = Buildup(**kw)
    setup = time.perf_counter() - t0
    out = {"workload": PRODUCTION, "steps_timed": steps, "setup_s": setup}
    out["poisson_solve"] = dict(workload="1024x1024 elliptical cut-cell grid 45x18 mm (the production grid), charge "
                                         "from 16 Gaussians (sigma 1-4 mm)", **poisson_comparison(lu.ps))
    lu.run(warm)  # first captures, first launches, the solver's one-time setup: not scaled to a passage
    t_lu = lu.run(steps)
    out["s_per_passage_lu"] = t_lu / steps * 5000
    out["final_macro_particles_lu"] = int(lu.history()[0][-1])
    out["management_events_lu"] = lu.n_managed
    def iterations(b, n=20):
        """Mean PCG iterations per solve over n more steps (one replay each)."""
        its = []
        for _ in range(n):
            b.run(1)
            its.append(b.ps.lastStats.iterations)
        return float(np.mean(its))

    lu.ps.resetHistory()
    m = Buildup(poisson=lu.ps, **kw)
    m.ps.method, m.ps.precond, m.ps.warmStart = "pcg", "mg", "extrapolate"
    fb0 = m.ps.nFallbacks
    m.run(warm)
    t_mg = m.run(steps)
    out["s_per_passage_pcg_mg"] = t_mg / steps * 5000
    out["pcg_mg_fallbacks"] = m.ps.nFallbacks - fb0
    out["final_macro_particles_pcg_mg"] = int(m.history()[0][-1])
    out["management_events_pcg_mg"] = m.n_managed
    out["pcg_mg_iterations_per_solve"] = iterations(m)
    from openecloud_b200.train_c5 import WEIGHTS
    if os.path.exists(WEIGHTS):
        # learned correction of the extrapolated warm start (the network
        # trained on pairs of this production run, openecloud_b200.train_c5)
        from openecloud_b200.cnn import PoissonCNN
        lu.ps.resetHistory()
        c = Buildup(poisson=lu.ps, **kw)
        c.ps.method, c.ps.precond, c.ps.warmStart = "pcg", "mg", "extrapolate+cnn"
        c.ps.cnn = PoissonCNN.for_solver(c.ps, weights=np.load(WEIGHTS).astype(np.float64), training=False)
        fb0 = c.ps.nFallbacks
        c.run(warm)
        t_c = c.run(steps)
        out["s_per_passage_pcg_mg_learned"] = t_c / steps * 5000
        out["pcg_mg_learned_fallbacks"] = c.ps.nFallbacks - fb0
        out["pcg_mg_learned_iterations_per_solve"] = iterations(c)
        out["final_macro_particles_pcg_mg_learned"] = int(c.history()[0][-1])
        x = torch.randn(c.ps.n_nodes, device="cuda", dtype=torch.float32)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        c.ps.cnn.forward(x)
        e0.record()
        for _ in range(10):
            c.ps.cnn.forward(x)
        e1.record()
        e1.synchronize()
        out["network_forward_ms"] = e0.elapsed_time(e1) / 10
        lu.ps.cnn = None
        lu.ps.warmStart = "extrapolate"
    out["timing"] = (f"device time (CUDA events) of {steps} steps after {warm} untimed ones (the management "
                     "events and graph captures of those steps included) x 5000/steps")
    return out


def component_rooflines(peak, n=1 << 24, n_merge=2_000_000):
    """Achieved HBM bandwidth of the per-step kernel groups beside the fused
    push/gather/deposit: (b) the standalone deposit, (c) the inside test, the
    absorbed-set scan, the wall rows and points, the Furman emission and the
    hole-refill / tail compaction, (d) the cell-binned merge (localRandom).
    The microbench store (2^24 electrons, cell-sorted) is pushed once with a
    20x longer step so that the electrons near the wall leave (about 2 %);
    algorithmic bytes per kernel / its CUDA-event time."""
    import torch
    from openecloud_b200 import _lib
    from openecloud_b200 import device as D
    from openecloud_b200.grid import Grid
    from openecloud_b200.particles import Particles
    from openecloud_b200.particleBoundary import AbsorbRectangular
    from openecloud_b200.particleEmitter import FurmanEmitter
    from openecloud_b200.particleManagement import localRandom
    s = torch.cuda.current_stream()
    sh = s.cuda_stream

    def timed(fn, reps=1, warm=1):
        for _ in range(warm):  # the first launch of a kernel also loads its module
            fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(s)
        for _ in range(reps):
            fn()
        b.record(s)
        b.synchronize()
        return a.elapsed_time(b) / reps

    def line(name, nbytes, ms, what):
        gbs = nbytes / (ms * 1e-3) / 1e9
        return {"kernel": name, "ms": ms, "alg_bytes": int(nbytes), "achieved_gbs": gbs, "frac": gbs / peak,
                "bytes": what}

    pd, E, (nx, ny, lx, ly) = workload(n, seed=7)
    g = Grid(nx, ny, lx, ly, 0)
    G = g.getNpExt()
    P = Particles("electrons", "variableWeight", capacity=n)
    P.setParticleData(pd)
    P.setBConst([0.0, 0.5, 0.0])
    bd = AbsorbRectangular(g, P)
    et = P.fieldTable(g, E, 2)
    P.pushGatherDeposit(g, et, 1e-11, 1, bd)
    P._hole_buffers()
    cg, cp, cb = g.c_grid(), P.c_particles(), bd.c_boundary()
    rho, wsc, st = P._rho_fix.data_ptr(), P._wscale.data_ptr(), P._status.data_ptr()
    out = []
    ms = timed(lambda: _lib.call("oec_deposit", cg, cp, rho, wsc, 1, st, sh), reps=5)
    out.append(line("deposit (oec_deposit)", 16 * n + 16 * G, ms, "cell, ox, oy, w per particle; grid clear + add"))
    # a long step: the electrons within ~2 cells of the wall leave
    P.pushGatherDeposit(g, et, 2e-10, 1, bd)
    ms = timed(lambda: _lib.call("oec_index_inside", cg, cp, cb, P._mask.data_ptr(), st, sh), reps=5)
    out.append(line("inside test (oec_index_inside)", 12.125 * n, ms, "cell, ox, oy per particle; absorbed bit"))
    bd.ensure_buffers(n // 8)
    L = _lib.lib()
    ms = timed(lambda: _lib.call("oec_absorbed_index", cp, P._mask.data_ptr(), bd._index.data_ptr(),
                                 bd._index.shape[0], bd._n_abs.data_ptr(), bd._scratch.data_ptr(), st, sh), reps=5)
    n_abs = int(D.to_numpy(bd._n_abs)[0])
    out.append(line("absorbed set (oec_absorbed_index)", n / 8 + 4 * n_abs, ms,
                    f"absorbed bits; {n_abs} indices"))
    cap = bd._rows.shape[0]
    ms = timed(lambda: _lib.call("oec_save_absorbed", cg, cp, bd._index.data_ptr(), bd._n_abs.data_ptr(), cap,
                                 bd._rows.data_ptr(), sh), reps=5)
    out.append(line("absorbed rows (oec_save_absorbed)", (4 + 28 + 48) * n_abs, ms,
                    "index, 7 fields gathered, one f64 row written per absorbed particle"))
    # the wall step moves the rows in place: its untimed first launch runs on copies
    rows_w, normals_w = bd._rows.clone(), bd._normals.clone()
    _lib.call("oec_wall_interaction", cg, cb, 2e-10, rows_w.data_ptr(), bd._n_abs.data_ptr(), cap,
              normals_w.data_ptr(), st, sh)
    del rows_w, normals_w
    ms = timed(lambda: _lib.call("oec_wall_interaction", cg, cb, 2e-10, bd._rows.data_ptr(), bd._n_abs.data_ptr(),
                                 cap, bd._normals.data_ptr(), st, sh), reps=1, warm=0)
    out.append(line("wall point and normal (oec_wall_interaction)", (48 + 48 + 16) * n_abs, ms,
                    "row read and written, normal written"))
    em = FurmanEmitter(bd, P, seyMax=1.6, seed=5)
    em.ensure_buffers(cap)
    ms = timed(lambda: em._launch(cap, 0, None, None), reps=3)
    n_sec = int(D.to_numpy(em._n_out)[0])
    out.append(line("Furman emission (oec_furman_emit)", (48 + 16) * n_abs + 48 * n_sec, ms,
                    f"row and normal per absorbed particle, row per secondary ({n_sec})"))
    # the placement rule the refill takes (decided on the device the same
    # way) and the kept particles it moves through the scratch store
    holes = D.to_numpy(bd._index[:min(n_abs, bd._index.shape[0])])
    if n_sec < n_abs:
        rule, moved = "in place, fewer rows than holes", n - int(holes[n_sec]) - (n_abs - n_sec)
    elif n - n_abs + n_sec > int(P._array_len.item()):
        rule, moved = "new array", n - n_abs
    else:
        rule, moved = "in place, rows fill the holes", 0
    # the refill changes the store, so it is timed once; a small store's
    # refill loads its kernels first
    W = Particles("electrons", "variableWeight")
    W.setParticleData(pd[:4096])
    W._bind(g)
    W.addAndRemoveParticles(pd[:16], (np.arange(4096) % 3 != 0).astype(np.uint16))
    tmp = P.c_scratch()  # the scratch store is allocated before the timed call
    ms = timed(lambda: _lib.call("oec_add_remove", cg, cp, tmp, P._mask.data_ptr(), bd._index.data_ptr(),
                                 bd._n_abs.data_ptr(), bd._index.shape[0], em._out.data_ptr(), em._n_out.data_ptr(),
                                 em._out.shape[0], P._array_len.data_ptr(), rho, wsc, st, sh), reps=1, warm=0)
    out.append(line("refill and compaction (oec_add_remove)", n / 8 + (48 + 28 + 16) * n_sec + 112 * moved, ms,
                    f"{rule}: absorbed bits; per secondary a row read, 7 fields written, its deposit; per moved "
                    f"particle ({moved}) 28 B read and 28 B written twice (through the scratch store)"))
    # (d) cell-binned merge of a 2e6-electron store over 10 % toward a 1.8e6 target
    pm, _, _ = workload(n_merge, seed=9)
    pm[:, 5] = np.random.default_rng(9).uniform(0.2, 2.0, n_merge) * 1e3
    Q = Particles("electrons", "variableWeight", capacity=2 * n_merge)
    Q.setParticleData(pm)
    bq = AbsorbRectangular(g, Q)
    Q._bind(g)
    localRandom(g, Q, bq, int(0.9 * n_merge), seed=3)  # first call: work buffers
    Q.setParticleData(pm)
    torch.cuda.synchronize()
    ms = timed(lambda: localRandom(g, Q, bq, int(0.9 * n_merge), seed=3), warm=0)
    out.append(line("merge (localRandom: weight sort, split, cell-binned merge, compaction)", 48 * 2 * n_merge, ms,
                    "rows read and written once per particle (48 B per particle and event); the whole call, "
                    "its host decisions included, after a first call that sized the work buffers"))
    return out


BATCH = ("batched scan: 64 independent buildup runs drawn with seed 4 from {256, 512, 768, 1024}^2 grids over "
         "circular (R=20 mm) and elliptical (45x18 mm) chambers, deltaMax U(1.2, 2.0), 0.5e11-1.5e11 p/bunch, "
         "B_y 0-8.33 T, 1e4 initial electrons each, roulette cap 5e5 every 50 steps, dt=1e-11 s")


def batched_scan(n_runs=64, steps=100, steady=50):
    """The batched scan in one graph per batch step (runs on parallel
    branches); the autotuner picks each grid's Poisson solve, the multigrid
    block size and the branch width (its trial steps are part of the first
    `steps`); then `steady` more steps at the chosen width."""
    import torch
    from openecloud_b200.autotune import Autotuner
    from openecloud_b200.batch import BatchedBuildup, scan_configs
    cfgs = scan_configs(n_runs, n_steps_table=steps + steady + 1)
    t0 = time.perf_counter()
    tuner = Autotuner()
    b = BatchedBuildup(cfgs, tuner=tuner)
    torch.cuda.synchronize()
    setup = time.perf_counter() - t0
    first = b.run(steps)
    sec = b.run(steady)
    steps_total = steps + steady
    psteps = sum(int(h[0][steps:steps_total].sum()) for h in b.histories())
    widths = next(v for k, v in tuner.choices.items() if k.startswith("branches/"))
    return {"workload": BATCH, "runs": n_runs, "setup_s": setup, "distinct_grids": len(b.shared),
            "branch_width": b.branches, "ms_per_batch_step_by_width": widths["ms_per_step"],
            "first_steps": steps, "first_steps_s": first, "steady_steps": steady,
            "ms_per_batch_step": sec / steady * 1e3, "run_steps_per_s": n_runs * steady / sec,
            "particle_steps_per_s": psteps / sec,
            "poisson_choice": {k.split("/", 1)[1]: v["choice"] for k, v in tuner.choices.items()
                               if k.startswith("poisson/")},
            "poisson_ms_per_solve": {k.split("/", 1)[1]: v["ms_per_solve"] for k, v in tuner.choices.items()
                                     if k.startswith("poisson/")},
            "mg_block_top": {k.split("/", 1)[1]: v["choice"] for k, v in tuner.choices.items()
                             if k.startswith("mg_block_top/")},
            "pcg_fallbacks": sum(r.ps.nFallbacks for r in b.runs if r.ps.method == "pcg"),
            "timing": "device time (CUDA events); steady = after the autotuner's trial steps"}


def run_reference(args, rank, world):
    """The compiled reference's own step on the host cores, on the same
    workload (2^24 electrons, seed 7) as the device arm: `warmup` untimed
    steps, then `steps` timed ones, each from the same rows."""
    if rank != 0:
        return
    t0 = time.perf_counter()
    n = args.particles
    pd, E, geom = workload(n, seed=7)
    res = cpu_reference_steps(pd, E, geom, min_seconds=0.0, max_steps=args.steps, min_steps=args.steps,
                              warm=args.warmup)
    ms = n / res["value"] * 1e3
    line = {"metric": METRIC, "value": res["value"], "unit": METRIC, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": bench_config(n, geom[0], geom[1], world),
            "impl": "reference", "cpu_baseline": {k: res[k] for k in ("kind", "cores", "sample", "value")},
            "e2e": {"value": res["value"], "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    cp = cpu_reference_passage()
    if cp is not None:
        line["bunch_passage"] = dict(workload=PASSAGE, **cp)
    line["wall_s"] = time.perf_counter() - t0
    print(json.dumps(line), flush=True)


# -------------------------------------------------------------- GPU arm
def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    from openecloud_b200 import _lib
    from openecloud_b200.grid import Grid
    from openecloud_b200.particles import Particles
    from openecloud_b200.particleBoundary import AbsorbRectangular

    torch.cuda.set_device(local_rank)
    n = args.particles
    pd, E, (nx, ny, lx, ly) = workload(n, seed=7 + rank)
    g = Grid(nx, ny, lx, ly, 0)
    P = Particles("electrons", "variableWeight", capacity=n)
    P.setParticleData(pd)
    P.setBConst([0.0, 0.5, 0.0])
    bd = AbsorbRectangular(g, P)
    et = P.fieldTable(g, E, 2)
    dt = 1e-11
    P.pushGatherDeposit(g, et, dt, 1, bd)  # computes the fixed-point scale once
    torch.cuda.synchronize()
    _log(f"setup done: {n} particles, capacity {P._cap}")

    cg, cp, cb = g.c_grid(), P.c_particles(), bd.c_boundary()
    bconst = _lib.d3([0.0, 0.5, 0.0])
    qm = P.particleCharge / P.particleMass
    stream = torch.cuda.current_stream()
    sh = stream.cuda_stream
    mask, rho, wsc, st = P._mask.data_ptr(), P._rho_fix.data_ptr(), P._wscale.data_ptr(), P._status.data_ptr()
    L = _lib.lib()

    def step():
        rc = L.oec_push_gather(cg, cp, et.data_ptr(), None, bconst, dt, qm, 1, cb, mask, rho, wsc, st, sh)
        if rc:
            raise _lib.OecError("oec_push_gather", rc)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = ClockSampler(local_rank)
    clocks.start()
    time.sleep(0.3)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    t_start.record(stream)
    for k in range(args.steps):
        ev[k][0].record(stream)
        step()
        ev[k][1].record(stream)
    t_end.record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    ms_total = t_start.elapsed_time(t_end)
    ms_kernel = float(np.mean([a.elapsed_time(b) for a, b in ev]))
    ms_step = ms_total / args.steps
    if world > 1:
        t = torch.tensor([ms_step, ms_kernel], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_step, ms_kernel = float(t[0]), float(t[1])
    status = P.status()
    _log(f"timed: {ms_step:.4f} ms/step, kernel {ms_kernel:.4f} ms, clocks {clk}")

    # ---------------------------------------------- end to end (host buffers)
    e2e = None
    if args.e2e_steps > 0:
        host = torch.from_numpy(pd).pin_memory()
        out = torch.empty_like(host).pin_memory()
        stage_rows = 1 << 22  # four 1M-row slots: large copies keep both PCIe directions busy
        staging = torch.empty((stage_rows, 6), dtype=torch.float64, device="cuda")
        hp, op_, sp = host.data_ptr(), out.data_ptr(), staging.data_ptr()

        def e2e_step():
            rc = L.oec_push_gather_host(cg, cp, hp, op_, n, sp, stage_rows, et.data_ptr(), None, bconst, dt, qm, 1,
                                        cb, mask, rho, wsc, st, sh)
            if rc:
                raise _lib.OecError("oec_push_gather_host", rc)

        e2e_step()
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(args.e2e_steps):
            e2e_step()
        b.record(stream)
        torch.cuda.synchronize()
        ms_e2e = a.elapsed_time(b) / args.e2e_steps
        if world > 1:
            t = torch.tensor([ms_e2e], device="cuda", dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms_e2e = float(t[0])
        # the copies alone, both directions at once: the floor of any
        # host-to-host step on this link
        dev_rows = torch.empty_like(host, device="cuda")
        side = torch.cuda.Stream()

        def copies():
            side.wait_stream(stream)
            with torch.cuda.stream(side):
                out.copy_(dev_rows, non_blocking=True)
            dev_rows.copy_(host, non_blocking=True)
            stream.wait_stream(side)
        copies()
        torch.cuda.synchronize()
        a.record(stream)
        copies()
        b.record(stream)
        torch.cuda.synchronize()
        ms_copy = a.elapsed_time(b)
        del dev_rows
        e2e = {"value": n * world / (ms_e2e * 1e-3), "unit": METRIC, "h2d_bytes_per_step": int(n * 48),
               "d2h_bytes_per_step": int(n * 48), "ms_per_step": ms_e2e,
               "copy_floor_ms": ms_copy, "frac_of_copy_floor": ms_copy / ms_e2e,
               "path": "oec_push_gather_host: (N,6) f64 rows in pinned host memory -> upload, fused kernel, "
                       "download in chunks with both copy directions overlapped (3 streams)"}

    # ----------------------------------------------------------- roofline
    # Algorithmic bytes of the hot-path step per launch: read and write
    # x, y, vx, vy, vz (40 B) and read w for the fused deposit (4 B) per
    # particle, E read once (2 f32 per node), the int64 deposit grid zeroed
    # and written once (2 x 8 B per node).
    G = (nx + 2) * (ny + 2)
    alg_bytes = 44 * n + 2 * 4 * G + 2 * 8 * G
    achieved = alg_bytes / (ms_kernel * 1e-3) / 1e9
    # The bytes this store layout moves: cell index, in-cell offsets and the
    # absorbed bit on top of the above, and the cell-centric E table.
    layout_bytes = (28 + 24 + 1.0 / 8) * n + 8 * 4 * G + 8 * G + 8 * G
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peak, peak_src = 6650.0, "fallback"
    if os.path.exists(peaks_path):
        try:
            peak = float(json.load(open(peaks_path))["hbm_gbs"])
            peak_src = "measured"
        except Exception:
            pass
    traffic = NCU_TRAFFIC_PER_LAUNCH.get(n)

    if e2e is not None:
        _log(f"e2e: {e2e['ms_per_step']:.3f} ms/step")
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_reference_steps(pd, E, (nx, ny, lx, ly), min_seconds=10.0, max_steps=30, min_steps=3, warm=1)
    passage = None
    if rank == 0 and world == 1 and not args.no_passage:
        passage = gpu_passage()
        _log(f"bunch passage: {passage['s_per_passage']:.3f} s (LU), {passage['s_per_passage_pcg_mg']:.3f} s "
             f"(MG-PCG), {passage['s_per_passage_pcg_jacobi']:.2f} s (Jacobi-PCG, est.)")
        if not args.no_cpu_baseline:
            cp = cpu_reference_passage()
            if cp is not None:
                passage["cpu_reference"] = cp
    production = None
    if rank == 0 and world == 1 and not args.no_production:
        production = production_passage()
        _log(f"production passage: {production['s_per_passage_lu']:.1f} s (LU), "
             f"{production['s_per_passage_pcg_mg']:.1f} s (MG-PCG); solve 1024^2: "
             f"{production['poisson_solve']['lu_ms']:.2f} ms LU, {production['poisson_solve']['mg_cold_ms']:.2f} ms "
             f"MG-PCG cold, {production['poisson_solve']['mg_warm_ms']:.2f} ms warm")

    cpu_c3 = cpu_scan = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and not args.no_production:
        cpu_c3 = cpu_reference_c3()
        if cpu_c3 is not None:
            _log(f"reference c3 shapes: LU 512^2 {cpu_c3['lu_solve_ms_512']:.0f} ms, 1024^2 "
                 f"{cpu_c3['lu_solve_ms_1024']:.0f} ms, particle step 2e6 {cpu_c3['particle_step_ms_2e6']:.0f} ms")
    if rank == 0 and world == 1 and not args.no_cpu_baseline and not args.no_batch:
        cpu_scan = cpu_reference_scan()
        if cpu_scan is not None:
            _log(f"reference scan, process-parallel: {cpu_scan['run_steps_per_s']:.1f} run-steps/s on "
                 f"{cpu_scan['processes']} processes")
    components = None
    if rank == 0 and world == 1 and not args.no_components:
        components = component_rooflines(peak)
        for c in components:
            _log(f"{c['kernel']}: {c['ms']:.3f} ms, {c['achieved_gbs']:.0f} GB/s ({c['frac']:.2f} of peak)")
    batch = None
    if rank == 0 and world == 1 and not args.no_batch:
        batch = batched_scan(steps=args.scan_steps)
        _log(f"batched scan: {batch['runs']} runs, {batch['ms_per_batch_step']:.1f} ms per batch step at width "
             f"{batch['branch_width']} ({batch['run_steps_per_s']:.0f} run-steps/s), setup {batch['setup_s']:.0f} s")

    if rank == 0:
        line = {"metric": METRIC, "value": n * world / (ms_step * 1e-3), "unit": METRIC, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32+i64", "data": "synthetic",
                "config": bench_config(n, nx, ny, world),
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": achieved / peak, "traffic": traffic,
                             "kernel": "k_push_gather<1,rect,deposit>", "kernel_ms": ms_kernel,
                             "alg_bytes_per_launch": alg_bytes,
                             "alg_bytes": "44 B per particle (x, y, vx, vy, vz read and written, w read) + "
                                          "E 2 x 4 B per node + int64 deposit grid 2 x 8 B per node",
                             "layout_bytes_per_launch": layout_bytes,
                             "layout_achieved": layout_bytes / (ms_kernel * 1e-3) / 1e9,
                             "layout_frac": layout_bytes / (ms_kernel * 1e-3) / 1e9 / peak,
                             "peak_source": peak_src},
                "clocks": clk, "e2e": e2e, "gpu_launches": 1 * args.steps,
                "status": {k: v for k, v in status.items() if v}}
        if cpu is not None:
            line["cpu_baseline"] = cpu
        if passage is not None:
            line["bunch_passage"] = passage
        if production is not None:
            line["production_passage"] = production
        if batch is not None:
            line["batched_scan"] = batch
            if cpu_scan is not None:
                batch["cpu_reference"] = cpu_scan
        if production is not None and cpu_c3 is not None:
            production["cpu_reference"] = cpu_c3
        if components is not None:
            line["component_rooflines"] = components
        print(json.dumps(line), flush=True)


def _log(msg):
    print(f"[bench] {msg}", file=sys.stderr, flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--particles", type=int, default=1 << 24)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-passage", action="store_true", help="skip the buildup bunch-passage timing")
    ap.add_argument("--no-production", action="store_true",
                    help="skip the 1024x1024 production passage sample and solve comparison")
    ap.add_argument("--no-batch", action="store_true", help="skip the 64-run batched scan")
    ap.add_argument("--scan-steps", type=int, default=100,
                    help="batch steps of the scan before its 50 steady ones (2450: a whole 2500-step passage)")
    ap.add_argument("--no-components", action="store_true",
                    help="skip the achieved bandwidth of the deposit, boundary, emission and merge kernels")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3) if args.impl == "ours" else args.warmup
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
