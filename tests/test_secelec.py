"""SecElecEmitter and SimpleSecEmitter (particleEmitter.pyx:316-597).

CPU: the C oracle, fed the reference's MT stream, reproduces the compiled
reference's secondaries bit for bit (two stainless settings and the simple
emitter; the fixture's reference build casts the secondary count to an
integer, which numpy >= 1.12 requires).
GPU: with injected uniforms the device emits exactly the oracle's counts and
rows within 1e-10 (device vs host libm); with its Philox draws the energy
spectrum and the count per absorbed particle pass two-sample KS tests against
the reference's; a buildup runs with either emitter.
"""
import numpy as np
import pytest

from conftest import golden, rel_err
from oracle import oracle as O

QE = 1.602176565e-19
ME = 9.10938291e-31


@pytest.mark.parametrize("case", [0, 1, 2])
def test_oracle_replays_reference(case):
    z = golden("secelec.npz")
    model, sey, reflec, seed = z[f"case{case}"]
    f = O.secelec(int(model), sey, reflec)
    out = O.secelec_emit(f, z["abs_rows"], z["abs_normals"], mode=0, seed=int(seed))
    ref = z[f"sec{case}"]
    assert out.shape == ref.shape and np.array_equal(out, ref)


def _setup(case, n_rep=1, seed=99):
    import torch
    from openecloud_b200.grid import Grid
    from openecloud_b200.particles import Particles
    from openecloud_b200.particleBoundary import AbsorbElliptical
    from openecloud_b200.particleEmitter import SecElecEmitter, SimpleSecEmitter
    z = golden("secelec.npz")
    model, sey, reflec, _ = z[f"case{case}"]
    g = Grid(64, 64, 0.04, 0.04, 1)
    P = Particles("electrons", "variableWeight")
    P.setParticleData(np.zeros((0, 6)))
    P._bind(g)
    bd = AbsorbElliptical(g, P)
    rows = np.tile(z["abs_rows"], (n_rep, 1))
    nv = np.tile(z["abs_normals"], (n_rep, 1))
    bd.ensure_buffers(len(rows))
    bd._rows[:len(rows)] = torch.as_tensor(rows, device="cuda")
    bd._normals[:len(rows)] = torch.as_tensor(nv, device="cuda")
    bd._n_abs.fill_(len(rows))
    bd._index = None  # row ids = row numbers
    bd._wall_done = True
    bd.absorbedMacroParticleCount = len(rows)
    em = (SecElecEmitter if model == 0 else SimpleSecEmitter)(bd, P, seyMax=float(sey), reflec=float(reflec),
                                                               seed=seed)
    return z, em, O.secelec(int(model), sey, reflec), rows, nv


@pytest.mark.gpu
@pytest.mark.parametrize("case", [0, 1, 2])
def test_replay_matches_oracle(gpu, case):
    import torch
    z, em, f, rows, nv = _setup(case)
    u = np.random.default_rng(40 + case).random((len(rows), 64))
    sec = em.generateSecondaries(replay=torch.as_tensor(u, device="cuda")).cpu().numpy()
    ref = O.secelec_emit(f, rows, nv, mode=1, uniforms=u)
    assert sec.shape == ref.shape
    assert np.array_equal(sec[:, [0, 1, 5]], ref[:, [0, 1, 5]])
    assert rel_err(sec[:, 2:5], ref[:, 2:5]) <= 1e-10


@pytest.mark.gpu
@pytest.mark.parametrize("case", [0, 1, 2])
def test_statistics_vs_reference(gpu, case):
    from scipy.stats import ks_2samp
    z, em, f, rows, nv = _setup(case, n_rep=20)
    sec = em.generateSecondaries().cpu().numpy()
    ref = z[f"sec{case}"]
    energy = lambda s: 0.5 * ME * np.sum(s[:, 2:5] ** 2, 1) / QE  # noqa: E731
    assert ks_2samp(energy(sec), energy(ref)).pvalue > 1e-3
    # secondaries per absorbed particle: the reference's mean within its
    # binomial spread of the device's
    mean_dev, mean_ref = len(sec) / len(rows), len(ref) / len(z["abs_rows"])
    assert abs(mean_dev - mean_ref) < 4 * np.sqrt(mean_ref / len(z["abs_rows"])), (mean_dev, mean_ref)
    assert np.all(np.isfinite(sec))


@pytest.mark.gpu
@pytest.mark.parametrize("emitter", ["secelec", "simple"])
def test_buildup_with_emitter(gpu, emitter):
    from openecloud_b200.buildup import Buildup
    b = Buildup(nx=48, ny=48, n_init=3000, target=30000, n_steps_table=301, emitter=emitter, seed=3)
    b.run(300)
    st = b.status()
    assert st["n_capacity_drop"] == 0
    n, w = b.history()
    assert n[-1] > 0 and np.all(np.isfinite(w))
