"""Generate golden fixtures by running the compiled openECLOUD reference.

Requires the reference modules built by ``python oracle/build_ref.py`` into
``oracle/_ref`` (which needs the reference source tree; it exists only where
the fixtures are generated).  Writes small ``.npz`` files next to this script;
the fixtures are committed, the reference is not.

Every array is produced by calling the reference's own public methods on
seeded inputs; the seeds and shapes are recorded in each file.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REF = os.path.join(REPO, "oracle", "_ref")


def _import_reference():
    if not os.path.isdir(REF):
        raise SystemExit("oracle/_ref missing: run python oracle/build_ref.py first")
    sys.path.insert(0, REF)
    import ref_compat  # noqa: F401  (scipy aliases used by beam.py)
    import grid, particles, particleBoundary, poissonSolver, randomGen  # noqa: E401
    return grid, particles, particleBoundary, poissonSolver, randomGen


GRIDS = {
    # name: (nx, ny, lx, ly, boundType)
    "rect_24x20": (24, 20, 0.03, 0.02, 0),
    "circle_32": (32, 32, 0.04, 0.04, 1),
    "ellipse_40x24": (40, 24, 0.09, 0.036, 1),
    "circle_128": (128, 128, 0.04, 0.04, 1),
}


def grid_arrays(g):
    out = {}
    for name in ["XMesh", "YMesh", "Ds", "Dst"]:
        out[name] = np.asarray(getattr(g, "get" + name)())
    out["Dsi"] = np.asarray(g.getDsi())
    out["Da"] = np.asarray(g.getDa())
    out["Dai"] = np.asarray(g.getDai())
    out["Dat"] = np.asarray(g.getDat())
    out["Dati"] = np.asarray(g.getDati())
    out["insidePoints"] = np.asarray(g.getInsidePoints())
    out["insideEdges"] = np.asarray(g.getInsideEdges())
    out["insideFaces"] = np.asarray(g.getInsideFaces())
    e2n = g.getEdgeToNode().tocsr()
    e2n.sort_indices()
    out["e2n_indptr"], out["e2n_indices"], out["e2n_data"] = e2n.indptr, e2n.indices, e2n.data
    for name in ["BoundaryPoints", "BoundaryPointsInd", "CutCellPointsInd", "CutCellNormalVectors",
                 "CutCellCenter"]:
        try:
            out[name[0].lower() + name[1:]] = np.asarray(getattr(g, "get" + name)())
        except Exception:
            pass
    return out


def random_inside(rng, n, lx, ly, kind):
    pts = []
    while sum(len(p) for p in pts) < n:
        x = (rng.random(4 * n) - 0.5) * lx
        y = (rng.random(4 * n) - 0.5) * ly
        if kind == 1:
            ok = x * x * 4 / lx ** 2 + y * y * 4 / ly ** 2 < 0.999
        else:
            ok = np.ones_like(x, bool)
        pts.append(np.stack([x[ok], y[ok]], 1))
    return np.concatenate(pts)[:n]


def make_particles(rng, n, lx, ly, kind, vscale):
    xy = random_inside(rng, n, lx, ly, kind)
    pd = np.empty((n, 6))
    pd[:, :2] = xy
    pd[:, 2:5] = rng.normal(0.0, vscale, (n, 3))
    pd[:, 5] = rng.uniform(0.5, 1.5, n) * 1e5
    return pd


def main():
    grid, particles, particleBoundary, poissonSolver, randomGen = _import_reference()
    rng = np.random.default_rng(20240611)
    for gname, (nx, ny, lx, ly, bt) in GRIDS.items():
        g = grid.Grid(nx, ny, lx, ly, bt)
        arrays = grid_arrays(g)
        arrays["params"] = np.array([nx, ny, lx, ly, bt], np.float64)
        # Poisson: random smooth charge, reference solve.
        ps = poissonSolver.PoissonSolver(g)
        xm, ym = arrays["XMesh"], arrays["YMesh"]
        X, Y = np.meshgrid(xm, ym)
        q = np.zeros_like(X)
        for _ in range(4):
            cx, cy = rng.uniform(-0.3, 0.3) * lx, rng.uniform(-0.3, 0.3) * ly
            s = rng.uniform(0.05, 0.15) * min(lx, ly)
            q += rng.uniform(-1, 1) * 1e-9 * np.exp(-((X - cx) ** 2 + (Y - cy) ** 2) / (2 * s * s))
        q = q.reshape(-1)
        E = np.asarray(ps.solve(q)).copy()
        arrays["poisson_q"] = q
        arrays["poisson_phi"] = np.asarray(ps.getPhi()).copy()
        arrays["poisson_E"] = E
        # Particle kernels on this grid.
        if gname != "circle_128":
            n = 600
            pd = make_particles(rng, n, lx, ly, bt, 2e6)
            P = particles.Particles("electrons", "variableWeight")
            P.setParticleData(pd.copy())
            P.calcGridWeights(g)
            arrays["pd_in"] = pd
            arrays["inCell"] = np.asarray(P.getInCell()).copy()
            arrays["w00"] = np.asarray(P.getWeightLowXLowY()).copy()
            arrays["w10"] = np.asarray(P.getWeightUpXLowY()).copy()
            arrays["w01"] = np.asarray(P.getWeightLowXUpY()).copy()
            arrays["w11"] = np.asarray(P.getWeightUpXUpY()).copy()
            P.chargeToGrid(g)
            arrays["chargeOnGrid"] = np.asarray(P.getChargeOnGrid()).copy()
            P.eFieldToParticles(g, E)
            arrays["eAtParticles"] = np.asarray(P.getEAtParticles()).copy()
            B = rng.normal(0, 0.3, 3 * g.getNpExt())
            P.bFieldToParticles(g, B)
            arrays["B_nodes"] = B
            arrays["bAtParticles"] = np.asarray(P.getBAtParticles())[:n].copy()
            dt = 2e-11
            for tb in (0, 1, 2):
                Q = particles.Particles("electrons", "variableWeight")
                Q.setParticleData(pd.copy())
                Q.setBConst(np.array([0.01, 0.5, -0.2]))
                Q.calcGridWeights(g)
                Q.eFieldToParticles(g, E)
                Q.bFieldToParticles(g, B)
                Q.borisPush(dt, tb)
                arrays[f"push{tb}"] = np.asarray(Q.getParticleData()).copy()
            arrays["push_dt"] = np.array(dt)
            arrays["bconst"] = np.array([0.01, 0.5, -0.2])
            # Boundary: particles near the wall moved outward by one push
            # (zero field), so about half cross the wall within one cell.
            dtb = 1e-11
            pb = make_particles(rng, n, lx, ly, bt, 1.0)
            scale = rng.uniform(0.95, 0.9995, n)
            if bt == 1:
                rho = np.sqrt(pb[:, 0] ** 2 * 4 / lx ** 2 + pb[:, 1] ** 2 * 4 / ly ** 2)
            else:
                rho = np.maximum(np.abs(pb[:, 0]) / (0.5 * lx), np.abs(pb[:, 1]) / (0.5 * ly))
            pb[:, 0] *= scale / np.maximum(rho, 1e-12)
            pb[:, 1] *= scale / np.maximum(rho, 1e-12)
            r = np.sqrt(pb[:, 0] ** 2 + pb[:, 1] ** 2) + 1e-30
            step = rng.uniform(0.2, 0.8, n) * min(lx / (nx - 1), ly / (ny - 1))
            ang = rng.uniform(-0.6, 0.6, n)
            ux, uy = pb[:, 0] / r, pb[:, 1] / r
            vx = (ux * np.cos(ang) - uy * np.sin(ang)) * step / dtb
            vy = (ux * np.sin(ang) + uy * np.cos(ang)) * step / dtb
            pb[:, 2], pb[:, 3] = vx, vy
            pb[:, 4] = rng.normal(0, 1e5, n)
            arrays["bnd_in"] = pb.copy()
            arrays["bnd_dt"] = np.array(dtb)
            zeroE = np.zeros(2 * g.getNpExt())
            kinds = [("rect", particleBoundary.AbsorbRectangular)] if bt == 0 else \
                [("ell", particleBoundary.AbsorbElliptical), ("cc", particleBoundary.AbsorbArbitraryCutCell)]
            for tag, cls in kinds:
                R = particles.Particles("electrons", "variableWeight")
                R.setParticleData(pb.copy())
                R.calcGridWeights(g)
                R.eFieldToParticles(g, zeroE)
                R.borisPush(dtb, 0)
                bd = cls(g, R)
                bd.indexInside()
                arrays[f"{tag}_moved"] = np.asarray(R.getParticleData()).copy()
                arrays[f"{tag}_isInside"] = np.asarray(R.getIsInside()).copy()
                bd.saveAbsorbed()
                arrays[f"{tag}_absorbed"] = np.asarray(bd.getAbsorbedParticles()).copy()
                if bd.getAbsorbedMacroParticleCount() > 0:
                    bd.calculateInteractionPoint()
                    bd.calculateNormalVectors()
                    arrays[f"{tag}_wall"] = np.asarray(bd.getAbsorbedParticles()).copy()
                    arrays[f"{tag}_normals"] = np.asarray(bd.getNormalVectors()).copy()
        path = os.path.join(HERE, f"grid_{gname}.npz")
        np.savez_compressed(path, **arrays)
        print("wrote", path, os.path.getsize(path))


if __name__ == "__main__" and not any(a.startswith("--") for a in sys.argv[1:]):
    main()


def _emission_absorbed():
    """The absorbed set of the emission fixtures: 16000 particles near the
    wall of a 64x64 circular chamber pushed across it (seed 4242)."""
    grid, particles, particleBoundary, poissonSolver, randomGen = _import_reference()
    rng = np.random.default_rng(4242)
    g = grid.Grid(64, 64, 0.04, 0.04, 1)
    n = 16000
    dtb = 1e-11
    lx = ly = 0.04
    pb = make_particles(rng, n, lx, ly, 1, 1.0)
    rho = np.sqrt(pb[:, 0] ** 2 * 4 / lx ** 2 + pb[:, 1] ** 2 * 4 / ly ** 2)
    scale = rng.uniform(0.97, 0.9999, n)
    pb[:, 0] *= scale / rho
    pb[:, 1] *= scale / rho
    # incident energies 0.1 eV .. 3 keV, directions within +-80 deg of outward
    energy = np.exp(rng.uniform(np.log(0.1), np.log(3000.), n))
    v = np.sqrt(2 * energy * 1.602176565e-19 / 9.10938291e-31)
    ang = rng.uniform(-1.4, 1.4, n)
    ux, uy = pb[:, 0] / np.hypot(pb[:, 0], pb[:, 1]), pb[:, 1] / np.hypot(pb[:, 0], pb[:, 1])
    vz_frac = rng.uniform(-0.3, 0.3, n)
    vp = v * np.sqrt(1 - vz_frac ** 2)
    pb[:, 2] = vp * (ux * np.cos(ang) - uy * np.sin(ang))
    pb[:, 3] = vp * (ux * np.sin(ang) + uy * np.cos(ang))
    pb[:, 4] = v * vz_frac
    # keep only particles that cross within one step (at most ~a cell)
    step_len = np.hypot(pb[:, 2], pb[:, 3]) * dtb
    pb[:, 2:5] *= np.minimum(1.0, 0.8 * (0.04 / 63) / np.maximum(step_len, 1e-30))[:, None]
    P = particles.Particles("electrons", "variableWeight")
    P.setParticleData(pb.copy())
    P.calcGridWeights(g)
    P.eFieldToParticles(g, np.zeros(2 * g.getNpExt()))
    P.borisPush(dtb, 0)
    bd = particleBoundary.AbsorbElliptical(g, P)
    bd.indexInside()
    bd.saveAbsorbed()
    bd.calculateInteractionPoint()
    bd.calculateNormalVectors()
    return P, bd


def emission_golden():
    """Reference Furman emission on absorbed sets, replayable by the oracle
    (same MT stream, same seed), plus special-function values."""
    grid, particles, particleBoundary, poissonSolver, randomGen = _import_reference()
    import particleEmitter
    import ref_probe
    out = {}
    P, bd = _emission_absorbed()
    out["abs_rows"] = np.asarray(bd.getAbsorbedParticles()).copy()
    out["abs_normals"] = np.asarray(bd.getNormalVectors()).copy()
    cases = [("copper", -1.0, None), ("copper", 1.6, 300.0), ("stainless", 1.8, None)]
    for k, (mat, sey, ehat) in enumerate(cases):
        em = particleEmitter.FurmanEmitter(bd, P, material=mat, seyMax=sey)
        if ehat is not None:
            em.setEHat0(ehat)
        randomGen.seed(1000 + k)
        sec = np.asarray(em.generateSecondaries()).copy()
        out[f"sec{k}"] = sec
        out[f"case{k}"] = np.array([0 if mat == "copper" else 1, sey, ehat if ehat is not None else -1.0, 1000 + k])
    # special functions of the reference (specFun.pyx) through the probe
    A, B, Pq = [], [], []
    for a in [0.3, 0.5, 0.9, 1.0, 1.5, 1.75, 2.5, 3.0, 7.5, 15.0, 34.5, 60.0]:
        for b in [0.4, 0.5, 1.0, 1.5, 3.0, 8.5, 11.5, 40.0]:
            for p in [1e-6, 0.003, 0.1, 0.37, 0.5, 0.81, 0.999]:
                A.append(a); B.append(b); Pq.append(p)
    A, B, Pq = np.array(A), np.array(B), np.array(Pq)
    out["bii_a"], out["bii_b"], out["bii_p"] = A, B, Pq
    out["bii"] = np.array([ref_probe.betaincinv(a, b, p) for a, b, p in zip(A, B, Pq)])
    GA, GP = np.meshgrid([0.2, 0.7, 1.0, 1.5, 2.5, 4.7, 12.0, 34.5, 115.0], [1e-8, 1e-3, 0.05, 0.4, 0.9, 0.999999])
    out["gii_a"], out["gii_p"] = GA.ravel(), GP.ravel()
    out["gii"] = np.array([ref_probe.gammaincinv(a, p) for a, p in zip(GA.ravel(), GP.ravel())])
    path = os.path.join(HERE, "emission.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "absorbed", len(out["abs_rows"]),
          "secondaries", [len(out[f"sec{k}"]) for k in range(3)])


if __name__ == "__main__" and "--emission" in sys.argv:
    emission_golden()


def management_golden():
    """Reference sortByColumn, globalRandom and localRandom on seeded inputs."""
    grid, particles, particleBoundary, poissonSolver, randomGen = _import_reference()
    import particleManagement
    rng = np.random.default_rng(99)
    g = grid.Grid(64, 64, 0.04, 0.04, 1)
    out = {}
    n = 4000
    pd = make_particles(rng, n, 0.04, 0.04, 1, 3e5)
    pd[:, 5] = np.exp(rng.normal(0, 0.8, n)) * 1e5
    out["pd"] = pd
    # sortByColumn(5)
    P = particles.Particles("electrons", "variableWeight")
    P.setParticleData(pd.copy())
    randomGen.seed(11)
    P.sortByColumn(5)
    out["sorted"] = np.asarray(P.getParticleData()).copy()
    # globalRandom: kill and clone
    for tag, target in [("kill", 3100), ("clone", 5200)]:
        P = particles.Particles("electrons", "variableWeight")
        P.setParticleData(pd.copy())
        randomGen.seed(21)
        particleManagement.globalRandom(g, P, target)
        out[f"global_{tag}"] = np.asarray(P.getParticleData()).copy()
    # localRandom (merge + split), ellipse boundary, both merge schemes
    for scheme in (0, 1):
        for tag, target in [("down", 3000), ("up", 4600)]:
            P = particles.Particles("electrons", "variableWeight")
            P.setParticleData(pd.copy())
            bd = particleBoundary.AbsorbElliptical(g, P)
            randomGen.seed(31 + scheme)
            particleManagement.localRandom(g, P, bd, target, mergeScheme=scheme)
            out[f"local{scheme}_{tag}"] = np.asarray(P.getParticleData()).copy()
    path = os.path.join(HERE, "management.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), {k: v.shape for k, v in out.items()})


if __name__ == "__main__" and "--management" in sys.argv:
    management_golden()


def management_moments(pd):
    """count, sum w, sum w v (3 components), sum w |v|^2 of (N, 6) rows."""
    w = pd[:, 5]
    v = pd[:, 2:5]
    return np.array([pd.shape[0], w.sum(), *(w[:, None] * v).sum(0), (w * (v * v).sum(1)).sum()])


def management_ensemble_golden(n_seeds=16):
    """The moments of the reference's localRandom output (both merge schemes,
    down to 3000 and up to 4600 from the 4000 rows of management.npz) over
    n_seeds seeds of its random stream."""
    grid, particles, particleBoundary, poissonSolver, randomGen = _import_reference()
    import particleManagement
    pd = np.load(os.path.join(HERE, "management.npz"))["pd"]
    g = grid.Grid(64, 64, 0.04, 0.04, 1)
    out = np.zeros((2, 2, n_seeds, 6))
    for scheme in (0, 1):
        for t, target in enumerate((3000, 4600)):
            for k in range(n_seeds):
                P = particles.Particles("electrons", "variableWeight")
                P.setParticleData(pd.copy())
                bd = particleBoundary.AbsorbElliptical(g, P)
                randomGen.seed(1000 + 31 * scheme + 7 * t + k)
                particleManagement.localRandom(g, P, bd, target, mergeScheme=scheme)
                out[scheme, t, k] = management_moments(np.asarray(P.getParticleData()))
    path = os.path.join(HERE, "management_ensemble.npz")
    np.savez_compressed(path, moments=out, before=management_moments(pd), targets=np.array([3000, 4600]))
    print("wrote", path, os.path.getsize(path))


if __name__ == "__main__" and "--management-ensemble" in sys.argv:
    management_ensemble_golden()


def reference_buildup(seed, n_steps, **kw):
    """oracle/ref_buildup.py: the reference's own loop on the c1 chamber."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import ref_buildup
    return ref_buildup.reference_buildup(seed, n_steps, **kw)


def buildup_golden(n_seeds=8, n_steps=2500):
    out = {}
    W, C = [], []
    for s in range(n_seeds):
        c, w = reference_buildup(100 + s, n_steps)
        W.append(w)
        C.append(c)
        print("seed", s, "final count", c[-1], "line density", w[-1])
    out["weight"] = np.array(W)[:, ::10]
    out["count"] = np.array(C)[:, ::10]
    out["every"] = np.array(10)
    path = os.path.join(HERE, "buildup_c1.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path))


if __name__ == "__main__" and "--buildup" in sys.argv:
    buildup_golden()


def _buildup20_seed(s):
    c, w = reference_buildup(200 + s, 20 * 2500)
    return c[::250], w[::250]


def buildup20_golden(n_seeds=8):
    """The c1 configuration over its full 20 bunch passages (50,000 steps),
    8 seeds of the reference's random stream (one process each), sampled
    every 250 steps."""
    import multiprocessing as mp
    with mp.get_context("spawn").Pool(n_seeds) as pool:
        res = pool.map(_buildup20_seed, range(n_seeds))
    out = {"count": np.array([r[0] for r in res]), "weight": np.array([r[1] for r in res]), "every": np.array(250)}
    path = os.path.join(HERE, "buildup_c1_20.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "final line density", out["weight"][:, -1])


if __name__ == "__main__" and "--buildup20" in sys.argv:
    buildup20_golden()


def beam_golden():
    grid, particles, particleBoundary, poissonSolver, randomGen = _import_reference()
    from beam import LHCBeam, LHCBeamEndless
    g = grid.Grid(64, 48, 0.04, 0.03, 1)
    e = LHCBeamEndless(g, 1e-11, nParticles=1.1e11)
    t = LHCBeam(g, 1e-11, nParticles=1.15e11)
    times = np.array([0.0, 1e-11, 3.3e-10, 1.0e-9, 1.7e-9, 2.5e-8 + 1.2e-9, 1.8e-6 + 4e-10, 2.05e-6 + 5e-10,
                      7.9e-6 + 1e-9, 3.0e-5 + 8e-10])
    as_arr = lambda v: np.zeros(g.getNpExt()) if np.isscalar(v) else np.asarray(v)  # noqa: E731
    out = {"times": times, "endless_profile": np.asarray(e.getTransversalProfile()),
           "train_profile": np.asarray(t.getTransversalProfile()),
           "endless_charge": np.array([as_arr(e.getCharge(x)) for x in times]),
           "train_charge": np.array([as_arr(t.getCharge(x)) for x in times])}
    path = os.path.join(HERE, "beam.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path))


if __name__ == "__main__" and "--beam" in sys.argv:
    beam_golden()


def extras_golden():
    """Reference multipoleExpansion on two grids and averageEnergy on a
    seeded particle set."""
    grid, particles, particleBoundary, poissonSolver, randomGen = _import_reference()
    import magneticField
    import util
    out = {}
    cases = [("circle_32", (32, 32, 0.04, 0.04, 1), [0., 5., 0., 0.01], []),
             ("ellipse_40x24", (40, 24, 0.09, 0.036, 1), [1.2, 0.5, 0.02, 0.003], [0.0, 0.2]),
             ("rect_24x20", (24, 20, 0.03, 0.02, 0), [0.3, -2.0], [0.1, 0.4, 7.0])]
    for name, gp, normal, skew in cases:
        g = grid.Grid(*gp)
        out[f"mp_{name}_params"] = np.array(gp, dtype=np.float64)
        out[f"mp_{name}_normal"] = np.array(normal, dtype=np.float64)
        out[f"mp_{name}_skew"] = np.array(skew, dtype=np.float64)
        out[f"mp_{name}_b"] = np.asarray(magneticField.multipoleExpansion(g, normal, skew)).copy()
    rng = np.random.default_rng(777)
    n = 2000
    pd = make_particles(rng, n, 0.04, 0.04, 1, 1.0)
    pd[:, 2:5] = rng.normal(0.0, 2e6, (n, 3))
    pd[:, 5] = rng.uniform(0.5, 1.5, n) * 1e5
    P = particles.Particles("electrons", "variableWeight")
    P.setParticleData(pd.copy())
    out["ae_particles"] = pd
    out["ae_energy"] = np.array([util.averageEnergy(P)])
    path = os.path.join(HERE, "extras.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path))


if __name__ == "__main__" and "--extras" in sys.argv:
    extras_golden()


def secelec_golden():
    """Reference SecElecEmitter (stainless, two settings) and SimpleSecEmitter
    on the emission fixtures' absorbed set, each after randomGen.seed (the
    oracle replays the same MT stream).  Needs the build recipe's integer
    cast of the secondary count (numpy rejects the reference's double)."""
    grid, particles, particleBoundary, poissonSolver, randomGen = _import_reference()
    import particleEmitter
    P, bd = _emission_absorbed()
    out = {"abs_rows": np.asarray(bd.getAbsorbedParticles()).copy(),
           "abs_normals": np.asarray(bd.getNormalVectors()).copy()}
    cases = [(0, -1.0, -1.0, 2000), (0, 1.8, 0.3, 2001), (1, -1.0, -1.0, 2002)]
    for k, (model, sey, reflec, seed) in enumerate(cases):
        cls = particleEmitter.SecElecEmitter if model == 0 else particleEmitter.SimpleSecEmitter
        em = cls(bd, P, seyMax=sey, reflec=reflec)
        randomGen.seed(seed)
        out[f"sec{k}"] = np.asarray(em.generateSecondaries()).copy()
        out[f"case{k}"] = np.array([model, sey, reflec, seed], dtype=np.float64)
    path = os.path.join(HERE, "secelec.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "absorbed", len(out["abs_rows"]),
          "secondaries", [len(out[f"sec{k}"]) for k in range(3)])


if __name__ == "__main__" and "--secelec" in sys.argv:
    secelec_golden()


CC_LX, CC_LY = 0.044, 0.036


def lhc_bound(x, y):
    """example05_arbitraryGeometry.py:35-39, as written there (its y test
    compares y^2 with 0.5 ly, so only the circle of radius lx/2 bounds)."""
    if x ** 2 + y ** 2 <= (0.5 * CC_LX) ** 2 and y ** 2 < 0.5 * CC_LY:
        return 1
    else:
        return 0


CC_RUN = dict(nx=44, ny=36, lx=CC_LX, ly=CC_LY, boundType=3, n_init=44 * 36 * 20, dt=2.155172413795e-11)


def buildup_cc_golden(n_seeds=8, n_steps=1160):
    """The reference loop on example05's chamber (cut-cell boundary from a
    user boundFunc, AbsorbArbitraryCutCell), c1's beam and emitter, one bunch
    passage at example05's time step, 8 seeds."""
    from ref_buildup import reference_buildup
    W, C = [], []
    for s in range(n_seeds):
        c, w = reference_buildup(300 + s, n_steps, boundFunc=lhc_bound, **CC_RUN)
        W.append(w)
        C.append(c)
        print("seed", s, "final count", c[-1], "line density", w[-1], flush=True)
    out = {"weight": np.array(W)[:, ::10], "count": np.array(C)[:, ::10], "every": np.array(10),
           "n_steps": np.array(n_steps)}
    path = os.path.join(HERE, "buildup_cc.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path))


if __name__ == "__main__" and "--buildup-cc" in sys.argv:
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    buildup_cc_golden()


# one reference Particles object through a sequence of addAndRemoveParticles
# calls that takes each of its placement rules: (label, keep fraction, rows added)
ADD_REMOVE_OPS = [
    ("remove", 0.8, 0),        # _removeParticles
    ("fill_append", 0.9, 500),  # in place, more rows than holes
    ("shift", 0.85, 100),      # in place, fewer rows than holes
    ("new_array", 0.95, 1500),  # above the array's rows: new array of 1.1 x count
    ("fill_append", 0.99, 120),  # in place inside the new array's room
    ("shift", 0.7, 50),
    ("nothing", 1.0, 0),
    ("remove", 0.6, 0),
    ("shift", 0.98, 1),
    ("new_array", 1.0, 3000),
]


def add_remove_golden(n0=3000):
    """Reference addAndRemoveParticles (particles.pyx:94-121, :201-269) over
    ADD_REMOVE_OPS.  Every row carries a unique id in its weight column
    (the initial rows 0..n0-1, then each call's added rows in turn), so the
    placement is recorded as the id sequence after each call, with the keep
    bits and the row count of the reference's array (getFullParticleData);
    the other columns play no part in the placement."""
    grid, particles, particleBoundary, poissonSolver, randomGen = _import_reference()
    rng = np.random.default_rng(123)
    next_id = [0]

    def rows(n):
        r = make_particles(rng, n, 0.04, 0.04, 1, 3e5) if n else np.zeros((0, 6))
        r[:, 5] = np.arange(next_id[0], next_id[0] + n, dtype=np.float64)
        next_id[0] += n
        return r

    P = particles.Particles("electrons", "variableWeight")
    pd0 = rows(n0)
    P.setParticleData(pd0.copy())
    out = {"n0": np.array(n0)}
    for k, (label, frac, n_add) in enumerate(ADD_REMOVE_OPS):
        n = P.getMacroParticleCount()
        keep = (rng.random(n) < frac).astype(np.uint16)
        add = rows(n_add)
        P.addAndRemoveParticles(add if n_add else np.zeros((0, 6)), keep)
        out[f"keep{k}"] = np.packbits(keep.astype(bool))
        out[f"nadd{k}"] = np.array(n_add)
        out[f"ids{k}"] = np.asarray(P.getParticleData())[:, 5].astype(np.int32)
        out[f"len{k}"] = np.array(np.asarray(P.getFullParticleData()).shape[0])
        print(label, n, "->", P.getMacroParticleCount(), "array rows", int(out[f"len{k}"]))
    path = os.path.join(HERE, "add_remove.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path))


if __name__ == "__main__" and "--add-remove" in sys.argv:
    add_remove_golden()


# a fixed inward field (the electrons are pushed outward) on the 32x32 circle:
# E = -k (x, y) at the nodes, so the wall sees impacts of up to ~2 keV and
# the refill takes every placement rule over the run
LOOP_RUN = dict(grid="circle_32", n0=800, k=1e7, dt=1e-11, steps=300, seed=5, sey=1.6)


def loop_field(xm, ym, k):
    X, Y = np.meshgrid(xm, ym)
    return np.concatenate([(-k * X).reshape(-1), (-k * Y).reshape(-1)])


def loop_checksums(pd):
    """Per-column sums and the slot-weighted sums of x and vx (which change
    when the same rows sit in other slots)."""
    i = np.arange(pd.shape[0], dtype=np.float64)
    return np.concatenate([pd.sum(0), [np.dot(i, pd[:, 0]), np.dot(i, pd[:, 2])]])


def loop_golden(space_charge=False):
    """The reference's particle loop (example01's calcGridWeights,
    eFieldToParticles, borisPush, indexInside, saveAbsorbed,
    calculateInteractionPoint, calculateNormalVectors, generateSecondaries,
    addAndRemoveParticles; example01_basic.py:66-97) in the fixed field of
    loop_field, LOOP_RUN['steps'] steps: per step the count, the row count of
    the particle array and the checksums, and the rows at the end.  With
    space_charge the electrons' own field is added every step (chargeToGrid,
    PoissonSolver.solve; example01_basic.py:71-81 without the beam) and
    their weights are 1e4 times larger, so that it matters."""
    grid, particles, particleBoundary, poissonSolver, randomGen = _import_reference()
    import particleEmitter
    r = LOOP_RUN
    nx, ny, lx, ly, bt = GRIDS[r["grid"]]
    g = grid.Grid(nx, ny, lx, ly, bt)
    E = loop_field(np.asarray(g.getXMesh()), np.asarray(g.getYMesh()), r["k"])
    rng = np.random.default_rng(77)
    pd0 = make_particles(rng, r["n0"], lx, ly, bt, 3e5)
    if space_charge:
        pd0[:, 5] *= 1e4
    P = particles.Particles("electrons", "variableWeight")
    P.setParticleData(pd0.copy())
    bd = particleBoundary.AbsorbElliptical(g, P)
    em = particleEmitter.FurmanEmitter(bd, P, seyMax=r["sey"])
    ps = poissonSolver.PoissonSolver(g)
    randomGen.seed(r["seed"])
    counts, lens, sums, absorbed = [], [], [], []
    for _ in range(r["steps"]):
        P.calcGridWeights(g)
        if space_charge:
            P.chargeToGrid(g)
            P.eFieldToParticles(g, np.asarray(ps.solve(np.asarray(P.getChargeOnGrid()))) + E)
        else:
            P.eFieldToParticles(g, E)
        P.borisPush(r["dt"], 0)
        bd.indexInside()
        bd.saveAbsorbed()
        na = bd.getAbsorbedMacroParticleCount()
        absorbed.append(na)
        if na > 0:
            bd.calculateInteractionPoint()
            bd.calculateNormalVectors()
            P.addAndRemoveParticles(em.generateSecondaries(), P.getIsInside())
        pd = np.asarray(P.getParticleData())
        counts.append(pd.shape[0])
        lens.append(np.asarray(P.getFullParticleData()).shape[0])
        sums.append(loop_checksums(pd))
    out = {"pd0": pd0, "counts": np.array(counts), "array_len": np.array(lens), "absorbed": np.array(absorbed),
           "checksums": np.array(sums), "final": np.asarray(P.getParticleData()).copy(),
           "params": np.array([nx, ny, lx, ly, bt], np.float64), "k": np.array(r["k"]), "dt": np.array(r["dt"]),
           "seed": np.array(r["seed"]), "sey": np.array(r["sey"]), "space_charge": np.array(int(space_charge))}
    path = os.path.join(HERE, "loop_sc_circle_32.npz" if space_charge else "loop_circle_32.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "final count", counts[-1], "absorbed", sum(absorbed))


if __name__ == "__main__" and "--loop" in sys.argv:
    loop_golden()
    loop_golden(space_charge=True)


def e2n_csc_golden():
    """Adds to each grid_*.npz the grid's edge-to-node matrix exactly as the
    reference returns it (CSC, its own index order: the order in which the
    phi -> E product sums), so that a restated solve gives the same E bit for
    bit; the CSR copy already stored is sorted."""
    grid, particles, particleBoundary, poissonSolver, randomGen = _import_reference()
    for gname, (nx, ny, lx, ly, bt) in GRIDS.items():
        path = os.path.join(HERE, f"grid_{gname}.npz")
        arrays = dict(np.load(path))
        e2n = grid.Grid(nx, ny, lx, ly, bt).getEdgeToNode().tocsc()
        arrays["e2n_csc_indptr"], arrays["e2n_csc_indices"], arrays["e2n_csc_data"] = \
            e2n.indptr.copy(), e2n.indices.copy(), e2n.data.copy()
        np.savez_compressed(path, **arrays)
        print("wrote", path, os.path.getsize(path))


if __name__ == "__main__" and "--e2n-csc" in sys.argv:
    e2n_csc_golden()


EXAMPLE01_RUN = dict(n_particles=2000, steps=1200, load_seed=3, seed=11)


def example01_golden():
    """example01_basic.py's loop as written (32x32 circle, LHCBeam, Furman
    emitter with its defaults, globalRandom every 50 steps outside +-5 %,
    dt = 2.155172413795e-11), with 2000 instead of 1e5 macro-particles, over
    its first 1200 steps (the first bunch passage).  The loaded rows are
    recorded and the MT stream re-seeded before the loop, so the oracle can
    start from them; the beam charge of each step is recorded as its scalar
    factor times the transverse profile (checked to be the reference's
    getCharge bit for bit).  Per step: count, array rows, absorbed count,
    whether globalRandom ran, checksums; the rows at the end."""
    grid, particles, particleBoundary, poissonSolver, randomGen = _import_reference()
    import particleEmitter
    import particleManagement
    from beam import LHCBeam
    r = EXAMPLE01_RUN
    N = r["n_particles"]
    g = grid.Grid(32, 32, 0.04, 0.04, 1)
    dt = 2.155172413795e-11
    beam = LHCBeam(g, dt)
    P = particles.Particles("electrons", "variableWeight")
    bd = particleBoundary.AbsorbElliptical(g, P)
    em = particleEmitter.FurmanEmitter(bd, P)
    ps = poissonSolver.PoissonSolver(g)
    randomGen.seed(r["load_seed"])
    particleEmitter.homoLoader(g, P, bd, N, 1.e9 / N)
    pd0 = np.asarray(P.getParticleData()).copy()
    profile = np.asarray(beam.getTransversalProfile()).copy()
    randomGen.seed(r["seed"])
    counts, lens, absorbed, managed, sums, beam_scale = [], [], [], [], [], []
    for ii in range(r["steps"]):
        n = P.getMacroParticleCount()
        man = ii > 0 and ii % 50 == 0 and (n > 1.05 * N or n < 0.95 * N)
        if man:
            particleManagement.globalRandom(g, P, N)
        managed.append(int(man))
        P.calcGridWeights(g)
        P.chargeToGrid(g)
        qb = beam.getCharge(ii * dt)
        saved, beam.qTransversalProfile = beam.qTransversalProfile, np.float64(1.0)
        scale = beam.getCharge(ii * dt)
        beam.qTransversalProfile = saved
        if np.isscalar(qb) and qb == 0:
            beam_scale.append(np.nan)  # no bunch: the reference adds the integer 0
        else:
            assert np.array_equal(float(scale) * profile, qb)
            beam_scale.append(float(scale))
        ps.solve(np.asarray(P.getChargeOnGrid()) + qb)
        P.eFieldToParticles(g, ps.getEAtGridPoints())
        P.borisPush(dt, 0)
        bd.indexInside()
        bd.saveAbsorbed()
        na = bd.getAbsorbedMacroParticleCount()
        absorbed.append(na)
        if na > 0:
            bd.calculateInteractionPoint()
            bd.calculateNormalVectors()
            P.addAndRemoveParticles(em.generateSecondaries(), P.getIsInside())
        pd = np.asarray(P.getParticleData())
        counts.append(pd.shape[0])
        lens.append(np.asarray(P.getFullParticleData()).shape[0])
        sums.append(loop_checksums(pd))
    out = {"pd0": pd0, "profile": profile, "beam_scale": np.array(beam_scale), "counts": np.array(counts),
           "array_len": np.array(lens), "absorbed": np.array(absorbed), "managed": np.array(managed),
           "checksums": np.array(sums), "final": np.asarray(P.getParticleData()).copy(), "dt": np.array(dt),
           "seed": np.array(r["seed"]), "target": np.array(N), "load_seed": np.array(r["load_seed"])}
    path = os.path.join(HERE, "example01_circle_32.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "final count", counts[-1], "absorbed", sum(absorbed),
          "management events", sum(managed), "beam steps", int(np.isfinite(out["beam_scale"]).sum()))


if __name__ == "__main__" and "--example01" in sys.argv:
    example01_golden()


# examples 02-05 as written, each with 1000 macro-particles over its first
# 600 steps (the first bunch and the start of the decay): what differs from
# example01 is the magnetic field, the management and the chamber
EXAMPLES = {
    "02": dict(grid=(32, 32, 0.04, 0.04, 1), type_b=1, bconst=(0., 0.1, 0.), management="global"),
    "03": dict(grid=(32, 32, 0.04, 0.04, 1), type_b=0, management="local"),
    "04": dict(grid=(32, 32, 0.04, 0.04, 1), type_b=2, multipole=(0., 5., 0., 0.01), management="local"),
    "05": dict(grid=(44, 36, CC_LX, CC_LY, 3), type_b=0, management="global_over_1.2"),
}
EXAMPLE_RUN = dict(n_particles=1000, steps=600, load_seed=3, seed=11)


def example_golden(name):
    """exampleNN's loop as written (the managements: globalRandom every 50
    steps outside +-5 % (02), localRandom with its kd-tree likewise (03,
    04), globalRandom whenever the count reaches 1.2x (05); B: constant
    (0, 0.1, 0) T (02), a quadrupole with an error from multipoleExpansion
    gathered per particle (04); chamber: example05's cut-cell boundary from
    its boundFunc) recorded like example01_golden; the grid arrays the
    oracle needs for the 44x36 chamber are stored with it."""
    grid, particles, particleBoundary, poissonSolver, randomGen = _import_reference()
    import particleEmitter
    import particleManagement
    import magneticField
    from beam import LHCBeam
    spec, r = EXAMPLES[name], EXAMPLE_RUN
    N = r["n_particles"]
    nx, ny, lx, ly, bt = spec["grid"]
    g = grid.Grid(nx, ny, lx, ly, bt, boundFunc=lhc_bound) if bt == 3 else grid.Grid(nx, ny, lx, ly, bt)
    dt = 2.155172413795e-11
    beam = LHCBeam(g, dt)
    P = particles.Particles("electrons", "variableWeight")
    bd = (particleBoundary.AbsorbArbitraryCutCell if bt == 3 else particleBoundary.AbsorbElliptical)(g, P)
    em = particleEmitter.FurmanEmitter(bd, P)
    ps = poissonSolver.PoissonSolver(g)
    randomGen.seed(r["load_seed"])
    particleEmitter.homoLoader(g, P, bd, N, 1.e9 / N)
    b_nodes = None
    if spec["type_b"] == 1:
        P.setBConst(np.array(spec["bconst"]))
    elif spec["type_b"] == 2:
        b_nodes = np.asarray(magneticField.multipoleExpansion(g, list(spec["multipole"]))).copy()
    out = {"pd0": np.asarray(P.getParticleData()).copy(), "params": np.array([nx, ny, lx, ly, bt], np.float64)}
    profile = np.asarray(beam.getTransversalProfile()).copy()
    randomGen.seed(r["seed"])
    counts, lens, absorbed, managed, sums, beam_scale = [], [], [], [], [], []
    for ii in range(r["steps"]):
        n = P.getMacroParticleCount()
        if spec["management"] == "global_over_1.2":
            man = ii > 0 and n >= 1.2 * N
        else:
            man = ii > 0 and ii % 50 == 0 and (n > 1.05 * N or n < 0.95 * N)
        if man and spec["management"] == "local":
            particleManagement.localRandom(g, P, bd, N)
        elif man:
            particleManagement.globalRandom(g, P, N)
        managed.append(int(man))
        P.calcGridWeights(g)
        P.chargeToGrid(g)
        qb = beam.getCharge(ii * dt)
        saved, beam.qTransversalProfile = beam.qTransversalProfile, np.float64(1.0)
        scale = beam.getCharge(ii * dt)
        beam.qTransversalProfile = saved
        if np.isscalar(qb) and qb == 0:
            beam_scale.append(np.nan)
        else:
            assert np.array_equal(float(scale) * profile, qb)
            beam_scale.append(float(scale))
        ps.solve(np.asarray(P.getChargeOnGrid()) + qb)
        P.eFieldToParticles(g, ps.getEAtGridPoints())
        if b_nodes is not None:
            P.bFieldToParticles(g, b_nodes)
        P.borisPush(dt, spec["type_b"])
        bd.indexInside()
        bd.saveAbsorbed()
        na = bd.getAbsorbedMacroParticleCount()
        absorbed.append(na)
        if na > 0:
            bd.calculateInteractionPoint()
            bd.calculateNormalVectors()
            P.addAndRemoveParticles(em.generateSecondaries(), P.getIsInside())
        pd = np.asarray(P.getParticleData())
        counts.append(pd.shape[0])
        lens.append(np.asarray(P.getFullParticleData()).shape[0])
        sums.append(loop_checksums(pd))
    out.update({"profile": profile, "beam_scale": np.array(beam_scale), "counts": np.array(counts),
                "array_len": np.array(lens), "absorbed": np.array(absorbed), "managed": np.array(managed),
                "checksums": np.array(sums), "final": np.asarray(P.getParticleData()).copy(), "dt": np.array(dt),
                "seed": np.array(r["seed"]), "target": np.array(N), "type_b": np.array(spec["type_b"]),
                "load_seed": np.array(r["load_seed"]),
                "bconst": np.array(spec.get("bconst", (0., 0., 0.))),
                "management": np.array(spec["management"])})
    if b_nodes is not None:
        out["b_nodes"] = b_nodes
    if bt == 3:
        arrays = grid_arrays(g)
        for k in ("insidePoints", "Dsi", "Dst", "insideFaces", "boundaryPoints", "cutCellPointsInd",
                  "cutCellNormalVectors"):
            out[k] = arrays[k]
        e2n = g.getEdgeToNode().tocsc()
        out["e2n_csc_indptr"], out["e2n_csc_indices"], out["e2n_csc_data"] = e2n.indptr, e2n.indices, e2n.data
    path = os.path.join(HERE, f"example{name}_loop.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "final count", counts[-1], "absorbed", sum(absorbed),
          "management events", sum(managed), "beam steps", int(np.isfinite(out["beam_scale"]).sum()))


if __name__ == "__main__" and "--examples" in sys.argv:
    for _name in EXAMPLES:
        example_golden(_name)
