"""Learned Poisson preconditioner: network kernels against the oracle.

CPU: the oracle's float64 gradients agree with central differences; the C
ABI's parameter layout is the oracle's.

GPU (through the C ABI): the forward pass and the parameter gradients of
oec_cnn_train_step match the oracle evaluated with the same bf16 rounding
points (the two differ only by f32 versus f64 accumulation); training on
(rho, phi) pairs of a 64x64 circular chamber lowers the loss; the trained
network as the PCG preconditioner needs fewer iterations than the Jacobi
preconditioner and than the untrained network, and the solve still meets
the f64 residual 1e-8.
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
from oracle import cnn_oracle  # noqa: E402


def test_oracle_gradient_finite_differences():
    assert cnn_oracle.finite_difference_check(ny=10, nx=13, n_probe=16, seed=1) <= 1e-5


def test_param_layout_matches_oracle():
    from openecloud_b200.cnn import param_layout, init_weights
    off, shapes = param_layout()
    assert off == cnn_oracle.layout()
    assert [(s[2], s[0]) for s in shapes[:7]] == cnn_oracle.SPECS
    assert init_weights(0).shape[0] == off[-1]
    assert np.array_equal(init_weights(3), cnn_oracle.init_weights(3))


def _case(ny=38, nx=45, seed=0):
    rng = np.random.default_rng(seed)
    inside = np.zeros((ny, nx), bool)
    inside[2:-2, 3:-3] = rng.random((ny - 4, nx - 6)) > 0.05
    x = rng.normal(size=(ny, nx))
    t = rng.normal(size=(ny, nx))
    w = cnn_oracle.bf16(cnn_oracle.init_weights(seed))
    return inside, x, t, w


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300))


KERNELS = ["mma.sync", "tcgen05"]


@pytest.mark.gpu
@pytest.mark.parametrize("kernel", KERNELS)
@pytest.mark.parametrize("shape", [(38, 45), (130, 257), (1026, 1026)])
def test_forward_matches_oracle(gpu, kernel, shape):
    """Forward pass through either tensor-core convolution kernel against the
    oracle, from a 38x45 grid to the production grid (1026^2 nodes: every
    level of the U-Net has several 128-pixel tiles per row and ragged
    tails)."""
    import torch
    from openecloud_b200 import device as D
    from openecloud_b200.cnn import PoissonCNN
    inside, x, t, w = _case(*shape)
    net = PoissonCNN(inside.shape[1], inside.shape[0], inside, weights=w, training=False, conv_kernel=kernel)
    z = D.to_numpy(net.forward(D.to_device(x.reshape(-1), torch.float32))).reshape(inside.shape)
    assert net.wait_timeouts() == 0
    zo, _ = cnn_oracle.forward(w, x, inside, bf=True)
    assert _rel(z, zo) <= 1e-2, _rel(z, zo)  # bf16 rounding-boundary flips, 7 layers
    assert np.all(z[~inside] == 0.0)


@pytest.mark.gpu
def test_tensor_core_kernels_agree(gpu):
    """The tcgen05 and mma.sync kernels compute the same sums in f32 (in
    another order): the forward passes agree far inside the bf16 rounding of
    the activations."""
    import torch
    from openecloud_b200 import device as D
    from openecloud_b200.cnn import PoissonCNN
    inside, x, t, w = _case(514, 514, seed=3)
    xd = D.to_device(x.reshape(-1), torch.float32)
    z = {k: D.to_numpy(PoissonCNN(514, 514, inside, weights=w, training=False, conv_kernel=k).forward(xd))
         for k in KERNELS}
    assert _rel(z["tcgen05"], z["mma.sync"]) <= 2e-2


@pytest.mark.gpu
@pytest.mark.parametrize("kernel", KERNELS)
@pytest.mark.parametrize("shape", [(38, 45), (70, 130)])
def test_gradients_match_oracle(gpu, shape, kernel):
    import torch
    from openecloud_b200 import device as D
    from openecloud_b200.cnn import PoissonCNN
    inside, x, t, w = _case(*shape, seed=2)
    net = PoissonCNN(shape[1], shape[0], inside, weights=w, conv_kernel=kernel)
    loss, g, z = net.loss_and_grad(D.to_device(x.reshape(-1), torch.float32), D.to_device(t.reshape(-1), torch.float32))
    assert net.wait_timeouts() == 0
    lo, go, zo = cnn_oracle.loss_and_grad(w, x, t, inside, bf=True)
    assert abs(loss - lo) <= 1e-3 * lo
    g = D.to_numpy(g).astype(np.float64)
    off = cnn_oracle.layout()
    for i in range(8):
        a, b = g[off[i]:off[i + 1]], go[off[i]:off[i + 1]]
        assert _rel(a, b) <= 2e-2, (i, _rel(a, b))


@pytest.mark.gpu
def test_residual_loss_gradients_match_oracle(gpu):
    import torch
    from openecloud_b200 import device as D
    from openecloud_b200.cnn import PoissonCNN
    from openecloud_b200.grid import Grid
    from openecloud_b200.poissonSolver import PoissonSolver, assemble, stencil_apply_host
    g = Grid(40, 30, 0.04, 0.03, 1)
    ps = PoissonSolver(g)
    ny, nx = g.getNyExt(), g.getNxExt()
    inside = (np.asarray(g.getInsidePoints()) != 0).reshape(ny, nx)
    _, meps, _, _ = assemble(g)
    s32 = ps._stencil.scale32
    # the f32 operator of the device: the f64 edge weights times scale32, rounded to f32
    m32 = (meps * s32).astype(np.float32).astype(np.float64)

    def apply_a(v):
        return stencil_apply_host(m32, inside.reshape(-1), nx, v.reshape(-1)).reshape(ny, nx)

    rng = np.random.default_rng(4)
    x = np.where(inside, rng.normal(size=(ny, nx)), 0.0)
    w = cnn_oracle.bf16(cnn_oracle.init_weights(6))
    net = PoissonCNN.for_solver(ps, weights=w)
    loss, gr, _ = net.loss_and_grad(D.to_device(x.reshape(-1), torch.float32), loss="residual")
    lo, go, _ = cnn_oracle.residual_loss_and_grad(w, x, inside, apply_a, bf=True)
    assert abs(loss - lo) <= 1e-3 * lo, (loss, lo)
    gr = D.to_numpy(gr).astype(np.float64)
    off = cnn_oracle.layout()
    for i in range(8):
        assert _rel(gr[off[i]:off[i + 1]], go[off[i]:off[i + 1]]) <= 2e-2, i


@pytest.mark.gpu
def test_training_and_warm_start(gpu):
    """Supervised training on (rho, phi) pairs of a 64x64 circular chamber: the
    trained network's warm start is much closer to the LU solution than the
    untrained network's or a zero start, and the iterative solve still reaches
    the f64 residual 1e-8 from it.  (Its bf16 noise is amplified by A, so it
    does not cut the Jacobi-PCG iteration count; the counts are printed.)"""
    from openecloud_b200.cnn import PoissonCNN, make_pairs
    from openecloud_b200.grid import Grid
    from openecloud_b200.poissonSolver import PoissonSolver
    ps = PoissonSolver(Grid(64, 64, 0.04, 0.04, 1), method="pcg", precond="jacobi", pcgMaxIter=20000)
    xs, ts = make_pairs(ps, 96, seed=5)
    test_x, test_t = make_pairs(ps, 6, seed=99)
    net = PoissonCNN.for_solver(ps, seed=1)
    ps.cnn = net

    def run(warm):
        ps.warmStart = warm
        it, err = [], []
        for k in range(len(test_x)):
            q = test_x[k].double() / ps._stencil.scale32
            phi_lu = test_t[k].double().cpu().numpy()  # A^-1 of the scaled charge q
            ps.phi.zero_()
            if warm == "cnn":
                net.warm_start(ps._stencil.scale32, q, ps.phi)
            err.append(np.linalg.norm(ps.phi.cpu().numpy() - phi_lu) / np.linalg.norm(phi_lu))
            ps.solveDevice(q)
            st = ps.lastStats
            assert st.converged == 1 and st.rel_residual <= 1e-8, (warm, st.rel_residual)
            it.append(st.iterations)
        return float(np.mean(it)), float(np.mean(err))

    zero = run("zero")
    untrained = run("cnn")
    losses = net.train(xs, ts, steps=3000, lr=3e-3, lr_final=1e-4, seed=0, loss="supervised")
    assert losses[-100:].mean() < 0.35 * losses[:50].mean(), (losses[:50].mean(), losses[-100:].mean())
    trained = run("cnn")
    print(f"Jacobi-PCG to 1e-8 (iterations, rel. error of the start vs LU): zero start {zero}, "
          f"untrained-network start {untrained}, trained-network start {trained}")
    assert trained[1] < 0.7 * zero[1] and trained[1] < 0.7 * untrained[1]


@pytest.mark.gpu
def test_learned_correction_on_the_production_chamber(gpu):
    """The network trained on 2e4 pairs of a production run
    (openecloud_b200/train_c5.py, weights in openecloud_b200/weights) as the
    correction of the extrapolated warm start, on another production run
    (1024x1024 ellipse 45 x 18 mm, 2.2e6 electrons, 8.33 T, merging every 10
    steps; seed 2000): over 40 steps after 20 warm-up ones, the multigrid-PCG
    solve at 1e-8 needs fewer iterations than from the extrapolation alone
    (measured 15.6 against 16.3 per solve), converges every time and never
    falls back to LU.  The corrected start has the LARGER initial residual
    (about 7x): the bf16 noise of the network's output sits in the highest
    spatial frequencies, which A amplifies and the first V-cycle removes,
    while the smooth error that costs CG its iterations is smaller.  Per step
    the correction costs one forward pass (0.3 ms at 1026^2), more than the
    iterations it saves (the passage times are in the benchmark)."""
    import os
    from openecloud_b200.buildup import Buildup
    from openecloud_b200.cnn import PoissonCNN
    from openecloud_b200.train_c5 import WEIGHTS, production_kwargs
    assert os.path.exists(WEIGHTS)
    w = np.load(WEIGHTS).astype(np.float64)
    kw = production_kwargs(seed=2000, steps=70)
    stats = {}
    ps = None
    for ws in ("extrapolate", "extrapolate+cnn"):
        b = Buildup(poisson=ps, **kw)
        ps = b.ps
        ps.resetHistory()
        ps.method, ps.precond, ps.warmStart = "pcg", "mg", ws
        ps.cnn = PoissonCNN.for_solver(ps, weights=w, training=False) if ws != "extrapolate" else None
        fb0 = ps.nFallbacks
        b.run(20)
        r0, it = [], []
        for _ in range(40):
            b.run(1)
            st = ps.lastStats
            assert st.converged == 1 and st.rel_residual <= 1e-8
            r0.append(st.rel_residual0)
            it.append(st.iterations)
        assert ps.nFallbacks == fb0
        if ps.cnn is not None:
            assert ps.cnn.wait_timeouts() == 0
        stats[ws] = (float(np.median(r0)), float(np.mean(it)))
    print(f"production chamber, MG-PCG to 1e-8 (median initial residual, mean iterations): extrapolation "
          f"{stats['extrapolate']}, with the learned correction {stats['extrapolate+cnn']}")
    assert stats["extrapolate+cnn"][1] < stats["extrapolate"][1]
