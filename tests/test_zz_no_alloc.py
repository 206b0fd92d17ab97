"""The deposit entry point that allocates nothing, against the regular path.

oec_deposit_charge_noalloc exists for callers that cannot call cudaMalloc
(hosts that own the whole device memory budget and forbid libraries from
allocating, or embeddings with a fixed memory plan).  It keeps its scratch in
file-scope device arrays.  This test calls it through the C ABI on two grids
in a row (and the first again, so the scratch left by an earlier call is
exercised) and compares each result with chargeToGrid's, which uses caller
buffers; the two paths run the same kernels, so the tolerance is the deposit
tolerance of the other tests (1e-12) and in practice the results are equal.
It also checks that a grid above the stated maximum is rejected.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _entry():
    from openecloud_b200 import _lib
    f = _lib.lib().oec_deposit_charge_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.POINTER(_lib.Grid_t), ctypes.POINTER(_lib.Particles_t), ctypes.c_double, ctypes.c_void_p,
                  ctypes.c_void_p]
    return f


def _case(nodes, n, seed):
    from openecloud_b200.grid import Grid
    from openecloud_b200.particles import Particles
    rng = np.random.default_rng(seed)
    g = Grid(nodes, nodes, 0.04, 0.04, 0)
    pd = np.empty((n, 6))
    pd[:, :2] = rng.uniform(-0.0199, 0.0199, (n, 2))
    pd[:, 2:5] = 0.0
    pd[:, 5] = rng.uniform(0.5, 1.5, n) * 1e4
    P = Particles("electrons", "variableWeight")
    P.setParticleData(pd)
    P._bind(g)
    return g, P


def test_noalloc_deposit_matches_regular_deposit(gpu):
    import torch
    from openecloud_b200 import device as D
    f = _entry()
    cases = [_case(128, 40000, 1), _case(512, 300000, 2)]
    for g, P in cases + cases[:1]:
        P.chargeToGrid(g)
        ref = P.getChargeOnGrid()
        out = torch.full((g.getNpExt(),), float("nan"), dtype=torch.float64, device="cuda")
        rc = f(g.c_grid(), P.c_particles(), P.particleCharge, out.data_ptr(), D.stream())
        assert rc == 0
        got = out.cpu().numpy()
        assert np.all(np.isfinite(got))
        err = np.max(np.abs(got - ref)) / np.max(np.abs(ref))
        assert err <= 1e-12, err


def test_noalloc_rejects_grid_above_maximum(gpu):
    import torch
    from openecloud_b200 import device as D
    f = _entry()
    g, P = _case(1100, 1000, 3)  # 1102^2 nodes > the 1,100,000-node scratch
    out = torch.zeros(g.getNpExt(), dtype=torch.float64, device="cuda")
    assert f(g.c_grid(), P.c_particles(), P.particleCharge, out.data_ptr(), D.stream()) == 3  # OEC_ERR_CAPACITY
