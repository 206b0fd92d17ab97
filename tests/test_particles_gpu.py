"""GPU parity of the particle kernels against the FP64 oracle and the
reference's golden vectors.

Tolerances (FP32 particle state against the FP64 oracle):
  * gather and push: norm-wise relative error <= 1e-6;
  * deposit: within 1e-12 (norm-wise) of the FP64 sum over the same stored
    particles, and the fixed-point total equals the sum of the quantised
    per-particle charges exactly;
  * inside test: bit-identical to the FP64 predicate on the stored positions.
"""
import numpy as np
import pytest

from conftest import golden, rel_err
from oracle import oracle as O

pytestmark = pytest.mark.gpu

QE = -1.602176565e-19
QM = -1.602176565e-19 / 9.10938291e-31
GRIDS = ["rect_24x20", "circle_32", "ellipse_40x24"]


def _setup(name, pd=None):
    from openecloud_b200.grid import Grid
    from openecloud_b200.particles import Particles
    z = golden(f"grid_{name}.npz")
    nx, ny, lx, ly, bt = z["params"]
    g = Grid(int(nx), int(ny), lx, ly, int(bt))
    P = Particles("electrons", "variableWeight")
    P.setParticleData(z["pd_in"] if pd is None else pd)
    return z, g, P, O.GridGeom(nx, ny, lx, ly)


@pytest.mark.parametrize("name", GRIDS)
def test_aos_roundtrip(gpu, name):
    z, g, P, og = _setup(name)
    P.calcGridWeights(g)
    back = P.getParticleData()
    pd = z["pd_in"]
    assert back.shape == pd.shape
    # positions: offset held in FP32 cell units -> error << 1e-6 cell
    assert np.max(np.abs(back[:, 0] - pd[:, 0])) < 1e-7 * og.dx
    assert np.max(np.abs(back[:, 1] - pd[:, 1])) < 1e-7 * og.dy
    assert rel_err(back[:, 2:], pd[:, 2:]) < 1e-7


@pytest.mark.parametrize("name", GRIDS)
def test_weights_match_reference(gpu, name):
    z, g, P, og = _setup(name)
    P.calcGridWeights(g)
    assert np.array_equal(P.getInCell(), z["inCell"])
    for get, k in [(P.getWeightLowXLowY, "w00"), (P.getWeightUpXLowY, "w10"), (P.getWeightLowXUpY, "w01"),
                   (P.getWeightUpXUpY, "w11")]:
        assert np.max(np.abs(get() - z[k])) < 1e-7


@pytest.mark.parametrize("name", GRIDS)
def test_gather_e_and_b(gpu, name):
    z, g, P, og = _setup(name)
    P.calcGridWeights(g)
    P.eFieldToParticles(g, z["poisson_E"])
    P.bFieldToParticles(g, z["B_nodes"])
    e = P.getEAtParticles()
    b = P.getBAtParticles()
    assert rel_err(e, z["eAtParticles"]) < 1e-6
    assert rel_err(b, z["bAtParticles"]) < 1e-6


@pytest.mark.parametrize("name", GRIDS)
@pytest.mark.parametrize("tb", [0, 1, 2])
def test_boris_push(gpu, name, tb):
    z, g, P, og = _setup(name)
    P.setBConst(z["bconst"])
    P.calcGridWeights(g)
    P.eFieldToParticles(g, z["poisson_E"])
    P.bFieldToParticles(g, z["B_nodes"])
    P.borisPush(float(z["push_dt"]), tb)
    out = P.getParticleData()
    ref = z[f"push{tb}"]
    for cols in ([0], [1], [2, 3, 4]):
        err = rel_err(out[:, cols], ref[:, cols])
        assert err < 1e-6, (cols, err)
    assert np.array_equal(out[:, 5], ref[:, 5].astype(np.float32).astype(np.float64))


def _quantised_total(w, wscale):
    return int(np.sum(np.rint(w.astype(np.float64) * wscale).astype(np.int64)))


@pytest.mark.parametrize("name", GRIDS)
def test_deposit_exact_and_within_1e12(gpu, name):
    z, g, P, og = _setup(name)
    P.chargeToGrid(g)
    q = P.getChargeOnGrid()
    fix, wscale = P.getChargeOnGridFixed()
    state = P.getParticleData()  # the FP32 state the GPU deposited, as f64 rows
    q_or = O.charge_to_grid(state, og, QE)
    err = rel_err(q, q_or)
    assert err <= 1e-12, err
    assert int(fix.sum()) == _quantised_total(state[:, 5], wscale)
    # and against the reference's own FP64 deposit of the unrounded inputs
    assert rel_err(q, z["chargeOnGrid"]) < 1e-6


def test_deposit_order_independent_and_large(gpu):
    from openecloud_b200.grid import Grid
    from openecloud_b200.particles import Particles
    rng = np.random.default_rng(5)
    g = Grid(256, 256, 0.04, 0.04, 0)
    n = 1 << 21
    pd = np.empty((n, 6))
    pd[:, 0] = rng.uniform(-0.02, 0.02, n)
    pd[:, 1] = rng.uniform(-0.02, 0.02, n)
    pd[:, 2:5] = 0.0
    pd[:, 5] = rng.uniform(0.5, 1.5, n) * 1e3
    A = Particles("electrons", "variableWeight")
    A.setParticleData(pd)
    A.chargeToGrid(g)
    fa, sa = A.getChargeOnGridFixed()
    B = Particles("electrons", "variableWeight")
    B.setParticleData(pd[rng.permutation(n)])
    B.chargeToGrid(g)
    fb, sb = B.getChargeOnGridFixed()
    assert sa == sb
    assert np.array_equal(fa, fb)  # bit-identical for any particle order
    state = A.getParticleData()
    assert int(fa.sum()) == _quantised_total(state[:, 5], sa)


@pytest.mark.parametrize("name", GRIDS)
def test_index_inside(gpu, name):
    from openecloud_b200 import particleBoundary as PB
    z = golden(f"grid_{name}.npz")
    bt = int(z["params"][4])
    for tag in (["rect"] if bt == 0 else ["ell"]):
        zz, g, P, og = _setup(name, pd=z[f"{tag}_moved"])
        cls = PB.AbsorbRectangular if tag == "rect" else PB.AbsorbElliptical
        bd = cls(g, P)
        bd.indexInside()
        ins = P.getIsInside()
        state = P.getParticleData()
        ins_or, _ = O.index_inside(state, og, 0 if tag == "rect" else 1)
        assert np.array_equal(ins, ins_or)
        # against the reference on its own f64 rows: same decision but for
        # points within FP32 rounding of the wall
        assert np.mean(ins == z[f"{tag}_isInside"]) > 0.99


@pytest.mark.parametrize("name", GRIDS)
@pytest.mark.parametrize("tb", [0, 1, 2])
def test_fused_push_gather_inside_deposit(gpu, name, tb):
    from openecloud_b200 import particleBoundary as PB
    z, g, P, og = _setup(name)
    bt = int(z["params"][4])
    P.setBConst(z["bconst"])
    P.calcGridWeights(g)
    before = P.getParticleData()
    bd = (PB.AbsorbRectangular if bt == 0 else PB.AbsorbElliptical)(g, P)
    et = P.fieldTable(g, z["poisson_E"], 2)
    btab = P.fieldTable(g, z["B_nodes"], 3) if tb == 2 else None
    dt = 4e-10  # large enough that a share of the particles leaves the domain
    P.pushGatherDeposit(g, et, dt, tb, bd, deposit=True, bCellTable=btab)
    after = P.getParticleData()
    # oracle: gather at the stored pre-push state, push in FP64
    e = O.field_to_particles(before, og, z["poisson_E"], 2)
    b = O.field_to_particles(before, og, z["B_nodes"], 3)
    ref = O.boris_push(before, e, dt, QM, tb, b_at=b, bconst=z["bconst"])
    for cols in ([0], [1], [2, 3, 4]):
        assert rel_err(after[:, cols], ref[:, cols]) < 1e-6, cols
    ins = P.getIsInside()
    ins_or, _ = O.index_inside(after, og, bt)
    assert np.array_equal(ins, ins_or)
    assert 0 < ins.sum() <= len(ins)
    # deposit of the survivors at their new position
    fix, wscale = P.getChargeOnGridFixed()
    q_gpu = fix.astype(np.float64) * (QE / wscale)
    q_or = O.charge_to_grid(after[ins == 1], og, QE)
    assert rel_err(q_gpu, q_or) <= 1e-12
    assert int(fix.sum()) == _quantised_total(after[ins == 1, 5], wscale)
    st = P.status()
    assert st["n_absorbed"] == int((ins == 0).sum())
    assert st["n_nonfinite"] == 0


def test_push_gather_host_equals_sequential_path(gpu):
    """oec_push_gather_host (host rows in, host rows out, copies overlapped
    over a ring of staging slots) gives the rows, deposit, absorbed bits and
    absorbed count of upload + fused kernel + download, bit for bit, over
    many chunks (300 000 particles through 16384-row slots, a shared output
    and an in-place call)."""
    import torch
    from openecloud_b200 import _lib
    from openecloud_b200 import device as D
    from openecloud_b200 import particleBoundary as PB
    from openecloud_b200.grid import Grid
    from openecloud_b200.particles import Particles
    rng = np.random.default_rng(12)
    n = 300_000
    g = Grid(128, 128, 0.04, 0.04, 0)
    pd = np.empty((n, 6))
    pd[:, 0] = rng.uniform(-0.0199, 0.0199, n)
    pd[:, 1] = rng.uniform(-0.0199, 0.0199, n)
    pd[:, 2:5] = rng.normal(0.0, 3e6, (n, 3))
    pd[:, 5] = rng.uniform(0.5, 1.5, n) * 1e4
    E = rng.normal(0.0, 2e4, 2 * g.getNpExt())
    dt = 2e-11

    def store():
        P = Particles("electrons", "variableWeight", capacity=n + 1024)
        P.setParticleData(pd)
        P.setBConst([0.0, 0.5, 0.0])
        bd = PB.AbsorbRectangular(g, P)
        et = P.fieldTable(g, E, 2)
        P.pushGatherDeposit(g, et, dt, 1, bd)  # deposit scale and buffers
        P.setParticleData(pd)
        torch.cuda.synchronize()
        return P, bd, et

    P, bd, et = store()
    P.pushGatherDeposit(g, et, dt, 1, bd)
    ref_rows = P.getParticleData()
    ref_rho = D.to_numpy(P._rho_fix).copy()
    ref_mask = D.to_numpy(P._mask).copy()
    ref_abs = P.status()["n_absorbed"]

    Q, bq, eq = store()
    L = _lib.lib()
    rows = 4 * 16384 + 1
    staging = torch.empty((rows, 6), dtype=torch.float64, device="cuda")
    host_in = torch.from_numpy(pd.copy()).pin_memory()
    host_out = torch.empty_like(host_in).pin_memory()
    for out in (host_out, host_in):  # a separate output, then in place
        Q.setParticleData(pd)
        host_in.copy_(torch.from_numpy(pd))
        rc = L.oec_push_gather_host(g.c_grid(), Q.c_particles(), host_in.data_ptr(), out.data_ptr(), n,
                                    staging.data_ptr(), rows, eq.data_ptr(), None, _lib.d3(Q.bConst), dt,
                                    Q.particleCharge / Q.particleMass, 1, bq.c_boundary(), Q._mask.data_ptr(),
                                    Q._rho_fix.data_ptr(), Q._wscale.data_ptr(), Q._status.data_ptr(),
                                    D.stream())
        assert rc == 0
        torch.cuda.synchronize()
        assert np.array_equal(out.numpy(), ref_rows)
        assert np.array_equal(D.to_numpy(Q._rho_fix), ref_rho)
        assert np.array_equal(D.to_numpy(Q._mask)[:ref_mask.size], ref_mask)
        assert Q.status()["n_absorbed"] == ref_abs and Q.getMacroParticleCount() == n
