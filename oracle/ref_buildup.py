"""Oracle (test infrastructure and CPU baseline only): the reference's own
buildup loop (example01_basic.py:52-97, Python 3, no plots) on the compiled
reference in oracle/_ref.  Used to make the buildup golden fixture and, in
bench.py's CPU baseline, to time one bunch passage on the host cores.
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.path.join(HERE, "_ref")


def available():
    return os.path.isdir(REF) and any(f.startswith("particles.") for f in os.listdir(REF))


def _import_reference():
    if not available():
        raise RuntimeError("oracle/_ref missing: run python oracle/build_ref.py first")
    if REF not in sys.path:
        sys.path.insert(0, REF)
    import ref_compat  # noqa: F401  (scipy aliases used by beam.py)
    import grid, particles, particleBoundary, poissonSolver, randomGen  # noqa: E401
    return grid, particles, particleBoundary, poissonSolver, randomGen


def reference_buildup(seed, n_steps, nx=128, lx=0.04, n_init=10000, dt=1e-11, target=100000, timing=None,
                      ny=None, ly=None, boundType=1, boundFunc=None, w_init=None):
    """The reference's own loop (example01_basic.py:52-97, Python 3, no plots);
    by default on the 128x128 circular chamber, else on Grid(nx, ny, lx, ly,
    boundType, boundFunc) with the matching absorber (rectangular,
    elliptical or cut-cell, particleBoundary.pyx); returns (macro counts, sum
    of weights).  With a dict `timing`, timing["seconds"] receives the wall
    time of the n_steps loop (setup excluded)."""
    grid, particles, particleBoundary, poissonSolver, randomGen = _import_reference()
    import particleEmitter
    import particleManagement
    from beam import LHCBeamEndless
    randomGen.seed(seed)
    ny = nx if ny is None else ny
    ly = lx if ly is None else ly
    g = grid.Grid(nx, ny, lx, ly, boundType, boundFunc=boundFunc) if boundFunc is not None else \
        grid.Grid(nx, ny, lx, ly, boundType)
    beam = LHCBeamEndless(g, dt, nParticles=1.1e11)
    beam.bunchLengthSigma = 0.25e-9 * 299792458.0          # sigma_t = 0.25 ns
    beam.tBunchLengthSigma = beam.bunchLengthSigma / beam.beamVelocity
    P = particles.Particles("electrons", "variableWeight")
    absorber = {0: particleBoundary.AbsorbRectangular, 1: particleBoundary.AbsorbElliptical}.get(
        boundType, particleBoundary.AbsorbArbitraryCutCell)
    bd = absorber(g, P)
    em = particleEmitter.FurmanEmitter(bd, P, seyMax=1.6)
    em.setEHat0(300.)
    ps = poissonSolver.PoissonSolver(g)
    particleEmitter.homoLoader(g, P, bd, n_init, 1e9 / n_init if w_init is None else w_init)
    counts = np.zeros(n_steps + 1, np.int64)
    weight = np.zeros(n_steps + 1)
    t0 = time.perf_counter()
    for ii in range(n_steps):
        weight[ii] = np.sum(np.asarray(P.getParticleData())[:, 5])
        counts[ii] = P.getMacroParticleCount()
        if ii > 0 and ii % 50 == 0 and (counts[ii] > 1.05 * target or counts[ii] < 0.95 * target):
            particleManagement.globalRandom(g, P, target)
        P.calcGridWeights(g)
        P.chargeToGrid(g)
        ps.solve(np.asarray(P.getChargeOnGrid()) + beam.getCharge(ii * dt))
        P.eFieldToParticles(g, ps.getEAtGridPoints())
        P.borisPush(dt, 0)
        bd.indexInside()
        bd.saveAbsorbed()
        if bd.getAbsorbedMacroParticleCount() > 0:
            bd.calculateInteractionPoint()
            bd.calculateNormalVectors()
            P.addAndRemoveParticles(em.generateSecondaries(), P.getIsInside())
    if timing is not None:
        timing["seconds"] = time.perf_counter() - t0
    weight[n_steps] = np.sum(np.asarray(P.getParticleData())[:, 5])
    counts[n_steps] = P.getMacroParticleCount()
    return counts, weight


