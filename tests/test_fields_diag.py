"""Multipole field (magneticField.pyx:23-59) and averageEnergy (util.pyx:8-20).

CPU: the numpy oracle reproduces the compiled reference's fields and mean
energy (golden fixtures made by tests/golden/make_golden.py --extras).
GPU: the device field equals the reference's to 1e-13 norm-wise (device
sin/cos/atan2 against the host libm); the device mean energy equals the
oracle's on the stored (FP32) particles to 1e-12 and the reference's on the
original FP64 rows to 1e-6; a buildup with a multipole field runs with the
gathered-B push.
"""
import numpy as np
import pytest

from conftest import golden, rel_err
from oracle import field_oracle as FO

CASES = ["circle_32", "ellipse_40x24", "rect_24x20"]


def _grid(z, name):
    from openecloud_b200.grid import Grid
    nx, ny, lx, ly, bt = z[f"mp_{name}_params"]
    return Grid(int(nx), int(ny), lx, ly, int(bt))


@pytest.mark.parametrize("name", CASES)
def test_multipole_oracle_matches_reference(name):
    z = golden("extras.npz")
    g = _grid(z, name)
    b = FO.multipole_expansion(g.getXMesh(), g.getYMesh(), z[f"mp_{name}_normal"], z[f"mp_{name}_skew"])
    assert rel_err(b, z[f"mp_{name}_b"]) <= 1e-14


def test_average_energy_oracle_matches_reference():
    z = golden("extras.npz")
    assert abs(FO.average_energy(z["ae_particles"]) / z["ae_energy"][0] - 1.0) <= 1e-14


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_multipole_device_matches_reference(gpu, name):
    from openecloud_b200.magneticField import multipoleExpansion
    z = golden("extras.npz")
    g = _grid(z, name)
    b = multipoleExpansion(g, z[f"mp_{name}_normal"], z[f"mp_{name}_skew"])
    assert b.shape == z[f"mp_{name}_b"].shape
    assert rel_err(b, z[f"mp_{name}_b"]) <= 1e-13
    assert np.all(b[2 * g.getNpExt():] == 0.0)


@pytest.mark.gpu
def test_average_energy_device(gpu):
    from openecloud_b200.grid import Grid
    from openecloud_b200.particles import Particles
    from openecloud_b200.util import averageEnergy
    z = golden("extras.npz")
    pd = z["ae_particles"]
    P = Particles("electrons", "variableWeight")
    P.setParticleData(pd)
    P._bind(Grid(64, 64, 0.04, 0.04, 1))
    e = averageEnergy(P)
    stored = P.getParticleData()
    assert abs(e / FO.average_energy(stored) - 1.0) <= 1e-12
    assert abs(e / z["ae_energy"][0] - 1.0) <= 1e-6


@pytest.mark.gpu
def test_buildup_with_multipole_field(gpu):
    """example04's quadrupole with an octupole error ([0, 5, 0, 0.01]) as the
    buildup's field: the step uses the gathered-B push and stays finite; the
    field bends the electrons, so the run differs from the field-free one."""
    from openecloud_b200.buildup import Buildup
    kw = dict(nx=32, ny=32, n_init=5000, target=50000, n_steps_table=201, seed=21)
    q = Buildup(b_multipoles=[0.0, 5.0, 0.0, 0.01], **kw)
    assert q.type_b == 2 and q.btab is not None
    q.run(200)
    free = Buildup(**kw)
    free.run(200)
    st = q.status()
    assert st["n_nonfinite"] == 0 and st["n_capacity_drop"] == 0
    nq, wq = q.history()
    nf, wf = free.history()
    assert np.all(np.isfinite(wq)) and nq[-1] > 0
    assert not np.array_equal(wq, wf)


@pytest.mark.gpu
def test_rhs_with_beam_matches_reference_charge(gpu):
    """oec_rhs_with_beam (the per-step Poisson right-hand side of the device
    loop: electron deposit + beam imprint, example01_basic.py:81) against the
    electron charge of the FP64 oracle plus the reference's own
    beam.getCharge(step * dt) (beam.py:68-78 train, :129-136 endless) at
    steps inside and between bunches."""
    import torch
    from conftest import golden
    from oracle import oracle as O
    from openecloud_b200 import _lib
    from openecloud_b200 import device as D
    from openecloud_b200.beam import LHCBeam, LHCBeamEndless
    from openecloud_b200.grid import Grid
    from openecloud_b200.particles import Particles
    z = golden("beam.npz")
    g = Grid(64, 48, 0.04, 0.03, 1)
    og = O.GridGeom(64, 48, 0.04, 0.03)
    rng = np.random.default_rng(4)
    n = 50000
    r = np.sqrt(rng.uniform(0, 1, n)) * 0.98
    a = rng.uniform(0, 2 * np.pi, n)
    pd = np.zeros((n, 6))
    pd[:, 0], pd[:, 1] = r * np.cos(a) * 0.02, r * np.sin(a) * 0.015
    pd[:, 5] = rng.uniform(0.5, 1.5, n) * 1e5
    P = Particles("electrons", "variableWeight")
    P.setParticleData(pd)
    P.chargeToGrid(g)
    q_e = O.charge_to_grid(P.getParticleData(), og, P.particleCharge)
    steps = [int(round(t / 1e-11)) for t in z["times"][:6]]
    G = g.getNpExt()
    for beam, key in ((LHCBeamEndless(g, 1e-11, nParticles=1.1e11), "endless_charge"),
                      (LHCBeam(g, 1e-11, nParticles=1.15e11), "train_charge")):
        table = D.to_device(beam.scalarTable(max(steps) + 1), torch.float64)
        profile = D.to_device(beam.getTransversalProfile(), torch.float64)
        for k, st in enumerate(steps):
            step_dev = D.to_device(np.array([st]), torch.int32)
            rho = D.zeros(G, torch.float64)
            _lib.call("oec_rhs_with_beam", g.c_grid(), P._rho_fix.data_ptr(), P._wscale.data_ptr(),
                      P.particleCharge, profile.data_ptr(), table.data_ptr(), step_dev.data_ptr(), table.shape[0],
                      rho.data_ptr(), D.stream())
            expect = q_e + z[key][k]
            err = np.max(np.abs(D.to_numpy(rho) - expect))
            assert err <= 1e-12 * np.max(np.abs(q_e)) + 1e-13 * np.max(np.abs(z[key][k])), (key, st, err)
