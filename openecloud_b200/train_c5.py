"""Training of the learned warm-start correction on the production chamber.

The network (openecloud_b200.cnn, a linear 4-level U-Net) learns what the
linear extrapolation of the Poisson solution in time misses: with q_n the
right-hand side of step n and phi_n its LU solution,

    A (phi_n - (2 phi_n-1 - phi_n-2)) = q_n - 2 q_n-1 + q_n-2,

so the input is the second difference d_n of the charge (normalised) and the
target the correction c_n = phi_n - 2 phi_n-1 + phi_n-2 (same scale).  The
pairs come from a production buildup run -- the 1024x1024 elliptical chamber
(45 x 18 mm), 2e6 macro-electrons, B_y = 8.33 T, 1.15e11 protons per bunch,
merging every 10 steps -- advanced with the FP64 LU solve; each step gives
one pair, on which the network takes one Adam step (the pairs are consumed
as the run produces them: 2e4 of them are 160 GB as stored arrays).  The
weights go to openecloud_b200/weights/poisson_c5_correction.npy.

    python -m openecloud_b200.train_c5 [--pairs 20000] [--seed 11]

Used as PoissonSolver(warmStart='extrapolate+cnn') with the network in
PoissonSolver.cnn (oec_cnn_correct).
"""
import argparse
import json
import os
import time

import numpy as np
import torch

from . import device as D
from .buildup import Buildup
from .cnn import PoissonCNN

WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "weights", "poisson_c5_correction.npy")


def production_kwargs(seed=2000, steps=5001, **over):
    """The production buildup of the benchmark (sampled passages)."""
    kw = dict(nx=1024, ny=1024, lx=0.09, ly=0.036, boundType=1, n_init=2_200_000, w_init=1e3, dt=5e-12,
              beam_particles=1.15e11, radius_sigma=1e-3, sey_max=1.8, type_b_field=1, b_const=(0., 8.33, 0.),
              target=2_000_000, management="local", management_every=10, n_steps_table=steps, seed=seed,
              abs_cap=4_400_000)  # the electrons released at rest cross the chamber together: bursts of > 1e6
                                  # absorbed in one step (half the store's capacity of rows)
    kw.update(over)
    return kw


class PairStream:
    """(x, t) pairs of a buildup run advanced with the LU solve: x = d/|d|,
    t = c/(s |d|) with d the second difference of the right-hand side, c the
    matching second difference of phi and s the f32 operator's scale (the
    network's output is in the units of the scaled inverse)."""

    def __init__(self, run):
        self.b = run
        ps = run.ps
        self.s32 = ps._stencil.scale32
        n = ps.n_nodes
        self.q = [D.zeros(n, torch.float64) for _ in range(2)]
        self.phi = [D.zeros(n, torch.float64) for _ in range(2)]
        self.seen = 0
        self.ins = torch.as_tensor(np.asarray(run.grid.getInsidePoints()) != 0, device=D.device())

    def next(self):
        """Advances the run one step; returns (x, t) once two earlier
        steps exist, else None."""
        b = self.b
        b.run(1)
        q, phi = b.rho, b.ps.phi
        out = None
        if self.seen >= 2:
            d = torch.where(self.ins, q - 2.0 * self.q[0] + self.q[1], 0.0)
            c = torch.where(self.ins, phi - 2.0 * self.phi[0] + self.phi[1], 0.0)
            nrm = float(torch.linalg.vector_norm(d)) * self.s32
            if nrm > 0:
                out = ((d * (self.s32 / nrm)).float(), (c / nrm).float())
        self.q[1].copy_(self.q[0])
        self.q[0].copy_(q)
        self.phi[1].copy_(self.phi[0])
        self.phi[0].copy_(phi)
        self.seen += 1
        return out


def train(pairs=20000, seed=11, lr=1e-3, lr_final=1e-4, log_every=1000, warm=20):
    """Trains on `pairs` consecutive steps of a production run (after `warm`
    steps) and returns (network, losses, seconds)."""
    b = Buildup(**production_kwargs(seed=seed, steps=pairs + warm + 8))
    b.run(warm)
    stream = PairStream(b)
    net = PoissonCNN.for_solver(b.ps, seed=seed)
    t0 = time.perf_counter()
    losses = []
    k = 0
    while k < pairs:
        p = stream.next()
        if p is None:
            continue
        x, t = p
        lr_k = lr * (lr_final / lr) ** (k / max(pairs - 1, 1))
        losses.append(net.train([x], [t], 1, lr=lr_k, lr_final=lr_k, seed=k)[0])
        k += 1
        if log_every and k % log_every == 0:
            print(f"[train_c5] pair {k}: loss {np.mean(losses[-log_every:]):.4e}", flush=True)
    return net, np.array(losses), time.perf_counter() - t0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--pairs", type=int, default=20000)
    ap.add_argument("--seed", type=int, default=11)
    ap.add_argument("--out", default=WEIGHTS)
    args = ap.parse_args()
    net, losses, secs = train(args.pairs, args.seed)
    os.makedirs(os.path.dirname(args.out), exist_ok=True)
    np.save(args.out, net.weights().astype(np.float32))
    k = max(1, len(losses) // 20)
    print(json.dumps({"pairs": args.pairs, "seconds": secs, "loss_first": float(np.mean(losses[:k])),
                      "loss_last": float(np.mean(losses[-k:])), "weights": args.out}), flush=True)


if __name__ == "__main__":
    main()
