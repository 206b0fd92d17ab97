"""Oracle (test infrastructure only): float64 numpy restatement of one
V-cycle of the aggregation multigrid preconditioner (oec_mg_apply in
``openecloud_b200/csrc/pcg.cu``).

The multigrid has no counterpart in the reference (it preconditions the
iterative solve that stands beside the reference's direct solve,
poissonSolver.pyx:83-88).  A level is given as (ex, ey, leak, inside, nx, ny)
with the operator (A x)_i = leak_i x_i + sum over the 4 grid edges of
w (x_i - x_j), x = 0 outside; level l+1 aggregates 2x2, 2x1 or 1x2 nodes of
level l (a direction whose size is kept is not aggregated).

Cycle (level 0 right-hand side r):
  down:  x1 = w D^-1 b;  x = x1 + w D^-1 (b - A x1);  b_c = P^T (b - A x)
  coarsest: x_c = A_c^-1 b_c (inside nodes)
  up:    t = x + s P x_c;  t' = t + w D^-1 (b - A t);  x = t' + w D^-1 (b - A t')
"""
import numpy as np


def apply_level(ex, ey, leak, inside, nx, x):
    n = ex.size
    ins = np.asarray(inside, bool)
    xm = np.where(ins, x, 0.0)
    col = np.arange(n) % nx
    y = leak * xm
    right = np.where(col + 1 < nx, np.roll(xm, -1), 0.0)
    left = np.where(col > 0, np.roll(xm, 1), 0.0)
    up = np.concatenate([xm[nx:], np.zeros(nx)])
    down = np.concatenate([np.zeros(nx), xm[:-nx]])
    ex_left = np.where(col > 0, np.roll(ex, 1), 0.0)
    ey_down = np.concatenate([np.zeros(nx), ey[:-nx]])
    y = y + ex * (xm - right) + ex_left * (xm - left) + ey * (xm - up) + ey_down * (xm - down)
    return np.where(ins, y, 0.0)


def diag_level(ex, ey, leak, inside, nx):
    """Diagonal of a level's operator (0 outside)."""
    n = ex.size
    col = np.arange(n) % nx
    d = leak + ex + ey + np.where(col > 0, np.roll(ex, 1), 0.0) + np.concatenate([np.zeros(nx), ey[:-nx]])
    return np.where(np.asarray(inside, bool), d, 0.0)


def parent(nx, ny, cnx=None, cny=None):
    """Coarse node of every fine node: aggregation by 2 along a direction
    whose size halves (rounded up), by 1 along one whose size is kept."""
    cnx = (nx + 1) // 2 if cnx is None else cnx
    cny = (ny + 1) // 2 if cny is None else cny
    fx = 1 if cnx == nx else 2
    fy = 1 if cny == ny else 2
    j, i = np.divmod(np.arange(nx * ny), nx)
    return (j // fy) * cnx + (i // fx)


def vcycle(levels, r, omega=0.8, scale=1.0, dinv=None):
    """levels: list of (ex, ey, leak, inside, nx, ny), finest first; dinv:
    optional per-level 1/diagonal (as stored on the device), else computed."""
    L = len(levels)
    if dinv is None:
        dinv = []
        for lv in levels:
            d = diag_level(*lv[:5])
            dinv.append(np.where(d != 0, 1.0 / np.where(d != 0, d, 1.0), 0.0))
    b = [None] * L
    x = [None] * L
    b[0] = np.asarray(r, np.float64)
    for k in range(L - 1):
        ex, ey, lk, ins, nx, ny = levels[k]
        A = lambda v: apply_level(ex, ey, lk, ins, nx, v)  # noqa: E731
        x1 = np.where(ins, omega * dinv[k] * b[k], 0.0)
        x[k] = np.where(ins, x1 + omega * dinv[k] * (b[k] - A(x1)), 0.0)
        res = np.where(ins, b[k] - A(x[k]), 0.0)
        nc = levels[k + 1][4] * levels[k + 1][5]
        b[k + 1] = np.bincount(parent(nx, ny, levels[k + 1][4], levels[k + 1][5]), weights=res, minlength=nc)
    ex, ey, lk, ins, nx, ny = levels[-1]
    idx = np.nonzero(ins)[0]
    M = np.empty((idx.size, idx.size))
    for c in range(idx.size):
        e = np.zeros(nx * ny)
        e[idx[c]] = 1.0
        M[:, c] = apply_level(ex, ey, lk, ins, nx, e)[idx]
    x[-1] = np.zeros(nx * ny)
    x[-1][idx] = np.linalg.solve(M, b[-1][idx])
    for k in range(L - 2, -1, -1):
        ex, ey, lk, ins, nx, ny = levels[k]
        A = lambda v: apply_level(ex, ey, lk, ins, nx, v)  # noqa: E731
        t = np.where(ins, x[k] + scale * x[k + 1][parent(nx, ny, levels[k + 1][4], levels[k + 1][5])], 0.0)
        t = np.where(ins, t + omega * dinv[k] * (b[k] - A(t)), 0.0)
        x[k] = np.where(ins, t + omega * dinv[k] * (b[k] - A(t)), 0.0)
    return x[0]
