"""PoissonSolver: finite-integration Poisson solve with the reference API.

Mirrors ``poissonSolver.PoissonSolver`` (poissonSolver.pyx:20-99).  Setup
(once per run, host): the system matrix A = S diag(eps0 dsi dst~) S^T over the
inside nodes and the gradient-to-node operator phiToE are assembled exactly as
the reference assembles them (poissonSolver.pyx:33-67) and A is factored by
SuperLU with the reference's options (``splu`` with MMD_AT_PLUS_A and
diag_pivot_thresh 0.1).  The y-derivative operator uses the signed offset
-nx that the reference intends (its unsigned offset wraps; poissonSolver.pyx:45).

Solve (every step, device): the FP64 LU back-substitution of
``oec_lu_solve`` (level-scheduled head rows + dense-inverse tail rows) and
the CSR product E = phiToE . phi (``oec_spmv_csr``).  With ``method='pcg'``
the solve is iterative instead (``oec_pcg_solve``: f64 residual refinement
around an f32 flexible PCG on the matrix-free 5-point operator, warm-started
by default from the linear extrapolation 2 phi_n-1 - phi_n-2 of the last two
solutions (``oec_warm_start_extrapolate``), Jacobi, multigrid or learned
preconditioner); the LU solve stays the fallback whenever the f64 relative
residual misses ``pcgTol``.
"""
import copy
import ctypes

import numpy as np
import scipy.sparse as spsp
import scipy.sparse.linalg as spspl
import torch

from . import _lib
from . import device as D
from .constants import epsilon_0
from .lu_setup import (LU_t, _level_lists, _levels, _np_ptr, assemble, choose_tail, factor,  # noqa: F401
                       level_lanes, lu_host_arrays, lu_struct)


class Stencil_t(ctypes.Structure):
    _P = ctypes.c_void_p
    _fields_ = [("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("ex64", _P), ("ey64", _P), ("ex32", _P),
                ("ey32", _P), ("dinv32", _P), ("inside", _P), ("scale32", ctypes.c_double)]


class PcgStats_t(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int32), ("refinements", ctypes.c_int32), ("converged", ctypes.c_int32),
                ("breakdown", ctypes.c_int32), ("rel_residual", ctypes.c_double),
                ("rel_residual0", ctypes.c_double)]


PRECOND = {"none": 0, "jacobi": 1, "cnn": 2, "mg": 3}


class MgLevel_t(ctypes.Structure):
    _P = ctypes.c_void_p
    _fields_ = [("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("ex", _P), ("ey", _P), ("leak", _P), ("dinv", _P),
                ("inside", _P), ("b", _P), ("x", _P), ("y", _P)]


class Mg_t(ctypes.Structure):
    _P = ctypes.c_void_p
    _fields_ = [("nlevels", ctypes.c_int32), ("levels", ctypes.POINTER(MgLevel_t)), ("block_level", ctypes.c_int32),
                ("ncoarse", ctypes.c_int32), ("coarse_idx", _P), ("coarse_inv", _P), ("omega", ctypes.c_float),
                ("scale", ctypes.c_float), ("cluster_top", ctypes.c_int32)]


MG_BLOCK_SMEM = 226 * 1024   # dynamic shared memory of the one-CTA coarse solve
MG_FLOATS_PER_NODE = 3       # b, x, y in shared memory (the operator moves there too when all 7 fit)
MG_CLUSTER_TOP = 0           # largest level given to the one-cluster coarse solve (0: the one-CTA solve)
MG_BLOCK_TOP = 1280          # largest level given to the one-CTA solve (one SM's issue rate bounds it)


def mg_coarsen(ex, ey, lkx, lky, inside, nx, ny, fx=2, fy=2):
    """Coarse level of the aggregation multigrid: aggregates of fx x fy nodes
    (fx, fy in {1, 2}; node (r, c) -> (r // fy, c // fx)) with the
    piecewise-constant P.  Per direction the coarse operator is the Galerkin
    product of that direction's part of A divided by the aggregation factor
    along it, A_c = P^T A_x P / fx + P^T A_y P / fy, which is what
    rediscretising the FIT operator on cells fx times wider and fy times
    taller gives (the weight of a face is its length over the distance across
    it): x-edges between inside nodes of different aggregates add w / fx to
    the coarse x-edge, y-edges w / fy to the coarse y-edge, edges from an
    inside node to the fixed outside and the leaks the same to the coarse
    leak of their direction; edges inside an aggregate cancel.  Keeping the
    directions apart is what lets a strongly anisotropic grid coarsen along
    one direction only.  Returns (ex, ey, lkx, lky, inside, nx, ny)."""
    NX, NY = (nx + fx - 1) // fx, (ny + fy - 1) // fy
    j, i = np.divmod(np.arange(nx * ny), nx)
    agg = (j // fy) * NX + (i // fx)
    inn = np.asarray(inside, bool)
    exc, eyc = np.zeros(NX * NY), np.zeros(NX * NY)
    lxc, lyc = np.zeros(NX * NY), np.zeros(NX * NY)
    ins = np.zeros(NX * NY, bool)
    ins[agg[inn]] = True
    np.add.at(lxc, agg[inn], lkx[inn] / fx)
    np.add.at(lyc, agg[inn], lky[inn] / fy)
    a_all = np.arange(nx * ny)
    for w, step, valid, tgt, lk, f in ((ex, 1, i < nx - 1, exc, lxc, fx), (ey, nx, j < ny - 1, eyc, lyc, fy)):
        a = a_all[valid]
        b = a + step
        wa = w[a] / f
        ia, ib = inn[a], inn[b]
        cross = ia & ib & (agg[a] != agg[b])
        np.add.at(tgt, agg[a][cross], wa[cross])
        la, lb = ia & ~ib, ib & ~ia
        np.add.at(lk, agg[a][la], wa[la])
        np.add.at(lk, agg[b][lb], wa[lb])
    return exc, eyc, lxc, lyc, ins, NX, NY


def mg_factors(ex, ey, inside, nx, ny, ratio=2.0):
    """Aggregation factors (fx, fy) of the next level: coarsen only along the
    strongly coupled direction while the mean inside-edge weights differ by
    more than `ratio`, else both ways."""
    ins = np.asarray(inside, bool)
    col = np.arange(nx * ny) % nx
    hx = ins & (col < nx - 1) & np.roll(ins, -1)
    vy = ins & np.concatenate([ins[nx:], np.zeros(nx, bool)])
    wx = ex[hx].mean() if hx.any() else 0.0
    wy = ey[vy].mean() if vy.any() else 0.0
    if wy > ratio * wx and ny > 1:
        return 1, 2
    if wx > ratio * wy and nx > 1:
        return 2, 1
    return 2, 2


def mg_hierarchy(ex, ey, inside, nx, ny, bottom=100, semi=True, block_top=None):
    """Levels (ex, ey, leak, inside, nx, ny) of the aggregation multigrid,
    finest first, coarsened until a level has at most `bottom` nodes, and the
    block level: the first level of at most MG_BLOCK_TOP nodes from which all
    coarser ones fit the one-CTA shared-memory solve."""
    z = np.zeros(nx * ny)
    cur = (np.asarray(ex, np.float64), np.asarray(ey, np.float64), z, z, np.asarray(inside, bool), nx, ny)
    lv = [cur[:2] + (z,) + cur[4:]]
    while cur[5] * cur[6] > bottom and max(cur[5], cur[6]) > 1:
        e, f, _, _, ins, X, Y = cur
        cur = mg_coarsen(*cur, *(mg_factors(e, f, ins, X, Y) if semi else (2, 2)))
        lv.append(cur[:2] + (cur[2] + cur[3],) + cur[4:])
    sizes = [l[4] * l[5] for l in lv]
    block = len(lv) - 1
    top = MG_BLOCK_TOP if block_top is None else block_top
    while block > 0 and len(lv) - (block - 1) <= 8 and sizes[block - 1] <= top and \
            4 * MG_FLOATS_PER_NODE * sum(sizes[block - 1:]) <= MG_BLOCK_SMEM:
        block -= 1
    return lv, block


def mg_apply_host(ex, ey, leak, inside, nx, x):
    """Host restatement of a multigrid level's operator (oec_mg_level_t)."""
    n = ex.size
    ins = np.asarray(inside, bool)
    xm = np.where(ins, x, 0.0)
    col = np.arange(n) % nx
    y = leak * xm
    right = np.where(col + 1 < nx, np.roll(xm, -1), 0.0)
    left = np.where(col > 0, np.roll(xm, 1), 0.0)
    up = np.concatenate([xm[nx:], np.zeros(nx)])
    down = np.concatenate([np.zeros(nx), xm[:-nx]])
    y = y + ex * (xm - right) + np.where(col > 0, np.roll(ex, 1), 0.0) * (xm - left)
    y = y + ey * (xm - up) + np.concatenate([np.zeros(nx), ey[:-nx]]) * (xm - down)
    return np.where(ins, y, 0.0)

_lib.OTHER_DECLARED.update({"oec_lu_solve", "oec_spmv_csr", "oec_trsv_levels", "oec_stencil_apply",
                            "oec_pcg_work_bytes", "oec_pcg_solve", "oec_mg_apply",
                            "oec_pcg_solve_async", "oec_warm_start_extrapolate"})


def _declare():
    L = _lib.lib()
    if not getattr(L, "_poisson_declared", False):
        P = ctypes.c_void_p
        L.oec_lu_solve.restype = ctypes.c_int
        L.oec_lu_solve.argtypes = [ctypes.POINTER(LU_t), P, P, P, P]
        L.oec_spmv_csr.restype = ctypes.c_int
        L.oec_spmv_csr.argtypes = [ctypes.c_int32, P, P, P, P, P, P]
        L.oec_trsv_levels.restype = ctypes.c_int
        L.oec_trsv_levels.argtypes = [ctypes.c_int32, P, P, ctypes.c_int32, ctypes.c_int32, P,
                                      ctypes.POINTER(ctypes.c_int32)]
        L.oec_stencil_apply.restype = ctypes.c_int
        L.oec_stencil_apply.argtypes = [ctypes.POINTER(Stencil_t), P, P, P]
        L.oec_pcg_work_bytes.restype = ctypes.c_int64
        L.oec_pcg_work_bytes.argtypes = [ctypes.c_int32, ctypes.c_int32]
        L.oec_pcg_solve.restype = ctypes.c_int
        L.oec_pcg_solve.argtypes = [ctypes.POINTER(Stencil_t), P, P, ctypes.c_double, ctypes.c_int32,
                                    ctypes.c_int32, P, P, ctypes.POINTER(PcgStats_t), P]
        L.oec_mg_apply.argtypes = [ctypes.POINTER(Mg_t), P, P, P]
        L.oec_pcg_solve_async.restype = ctypes.c_int
        L.oec_pcg_solve_async.argtypes = [ctypes.POINTER(Stencil_t), P, P, ctypes.c_double, ctypes.c_int32,
                                          ctypes.c_int32, P, P, P, ctypes.POINTER(LU_t), P, P, P]
        L.oec_warm_start_extrapolate.restype = ctypes.c_int
        L.oec_warm_start_extrapolate.argtypes = [P, P, ctypes.c_int64, P, P]
        L._poisson_declared = True
    return L



def stencil_apply_host(meps, inside_mask, nx, x):
    """Host restatement of oec_stencil_apply: (A x)_i = sum over the four edges
    of node i of meps * (x_i - x_j), x_j = 0 outside; 0 on outside nodes."""
    npn = inside_mask.shape[0]
    ex, ey = meps[:npn], meps[npn:]
    x = np.where(inside_mask, x, 0.0)
    y = np.zeros(npn)
    i = np.nonzero(inside_mask)[0]
    y[i] = (ex[i] * (x[i] - x[i + 1]) + ex[i - 1] * (x[i] - x[i - 1]) + ey[i] * (x[i] - x[i + nx]) +
            ey[i - nx] * (x[i] - x[i - nx]))
    return y


class PoissonSolver:
    """Reference: poissonSolver.pyx:33-67 (setup) and :83-98 (solve, getters)."""

    def __init__(self, gridObj, tail=None, method="lu", precond="jacobi", pcgTol=1e-8, pcgMaxIter=4000,
                 warmStart="extrapolate", factors=None):
        """factors: the result of lu_setup.factor(gridObj) when the host
        setup (assembly and SuperLU factorisation) was done beforehand, e.g.
        for several grids in parallel threads."""
        nx = gridObj.getNxExt()
        npn = gridObj.getNpExt()
        self.gridObj = gridObj
        a, meps, st, self.insidePointsInd, self.ludecom, self.phiToEAtGridPoints = \
            factors if factors is not None else factor(gridObj)
        self.systemMatrix = a
        self.n_nodes = npn
        self._device_setup(tail)
        self._stencil_setup(meps, nx, npn)
        self.phi = D.zeros(npn, torch.float64)
        self.eAtGridPoints = D.zeros(2 * npn, torch.float64)
        self.method = method
        self.precond = precond
        self.pcgTol = float(pcgTol)
        self.pcgMaxIter = int(pcgMaxIter)
        self.cnn = None          # a trained network (openecloud_b200.cnn) for precond='cnn' / warmStart='cnn'
        self._mg = None          # multigrid hierarchy for precond='mg' (built on first use)
        self.warmStart = warmStart  # 'previous' (last phi), 'extrapolate' (2 phi_n-1 - phi_n-2), 'zero' or 'cnn'
        self._phi_prev = None    # phi of the solve before the last ('extrapolate')
        self._ws_hist = None     # device count of the solutions seen, saturating at 2 ('extrapolate')
        self._q_hist = None      # the two previous charges ('extrapolate+cnn')
        self._q_count = None     # device count of the charges seen, saturating at 2
        self.nSolves = 0
        # statistics of the last iterative solve and the count of LU
        # fallbacks stay on the device (no host round trip per solve)
        self._stats_dev = D.zeros(ctypes.sizeof(PcgStats_t), torch.uint8)
        self._fb_count = D.zeros(1, torch.int32)
        self._pcg_used = False

    def _stencil_setup(self, meps, nx, npn):
        """Edge weights of A on the full extended grid (oec_stencil_t)."""
        ex = np.ascontiguousarray(meps[:npn], np.float64)
        ey = np.ascontiguousarray(meps[npn:], np.float64)
        inside = np.asarray(self.gridObj.getInsidePoints()).astype(np.uint8)
        diag = np.zeros(npn)
        i = np.nonzero(inside)[0]
        diag[i] = ex[i] + ex[i - 1] + ey[i] + ey[i - nx]
        scale = 1.0 / float(np.max(np.abs(meps))) if np.max(np.abs(meps)) > 0 else 1.0
        dinv = np.zeros(npn, np.float32)
        dinv[i] = (1.0 / (scale * diag[i])).astype(np.float32)
        k = self._keep
        k["ex64"], k["ey64"] = D.to_device(ex, torch.float64), D.to_device(ey, torch.float64)
        k["ex32"] = D.to_device((ex * scale).astype(np.float32), torch.float32)
        k["ey32"] = D.to_device((ey * scale).astype(np.float32), torch.float32)
        k["dinv32"] = D.to_device(dinv, torch.float32)
        k["inside"] = D.to_device(inside, torch.uint8)
        st = Stencil_t()
        st.nx, st.ny = nx, npn // nx
        for name in ("ex64", "ey64", "ex32", "ey32", "dinv32", "inside"):
            setattr(st, name, D.ptr(k[name]))
        st.scale32 = scale
        self._stencil = st
        self._pcg_work = D.empty(int(_declare().oec_pcg_work_bytes(st.nx, st.ny)), torch.uint8)

    def _mg_setup(self, omega=0.8, scale=1.0, bottom=100, block_top=None, cluster_top=None):
        """Aggregation multigrid hierarchy (oec_mg_t) on the scaled f32
        operator, down to at most `bottom` nodes, whose inside block is
        inverted densely (f64 on the host, stored in f32); levels of at most
        `block_top` nodes (default MG_BLOCK_TOP) go to the one-CTA solve, or
        with `cluster_top` > 0 (default MG_CLUSTER_TOP) the levels from the
        first one of at most `cluster_top` nodes go to the one-cluster solve.  The
        operators are shared with sibling solvers; the work vectors are this
        solver's.  The host copy of every level (ex, ey, leak, inside, nx, ny)
        is kept under "host"."""
        st = self._stencil
        k = self._keep
        ex = D.to_numpy(k["ex32"]).astype(np.float64)
        ey = D.to_numpy(k["ey32"]).astype(np.float64)
        inside = D.to_numpy(k["inside"]).astype(bool)
        lv, block = mg_hierarchy(ex, ey, inside, st.nx, st.ny, bottom,
                                 block_top=MG_BLOCK_TOP if block_top is None else block_top)
        e, f, lk, ins, X, Y = lv[-1]
        idx = np.nonzero(ins)[0]
        M = np.empty((idx.size, idx.size))
        for c in range(idx.size):
            v = np.zeros(X * Y)
            v[idx[c]] = 1.0
            M[:, c] = mg_apply_host(e, f, lk, ins, X, v)[idx]
        ops = []
        for n_, (e, f, lk, ins, X, Y) in enumerate(lv):
            i = np.nonzero(ins)[0]
            col = i % X
            d = lk[i] + e[i] + f[i] + np.where(col > 0, e[np.maximum(i - 1, 0)], 0.0) + \
                np.where(i >= X, f[np.maximum(i - X, 0)], 0.0)
            if np.any(d <= 0.0):
                raise ValueError("multigrid level with a non-positive diagonal")
            dinv = np.zeros(X * Y)
            dinv[i] = 1.0 / d
            t = {"nx": X, "ny": Y, "ex": D.to_device(e, torch.float32), "ey": D.to_device(f, torch.float32),
                 "leak": D.to_device(lk, torch.float32), "dinv": D.to_device(dinv, torch.float32),
                 "inside": D.to_device(ins.astype(np.uint8), torch.uint8)}
            if n_ == 0:  # the solver's own f32 operator and diagonal
                t["ex"], t["ey"], t["dinv"] = k["ex32"], k["ey32"], k["dinv32"]
            ops.append(t)
        shared = {"ops": ops, "cidx": D.to_device(idx.astype(np.int32), torch.int32),
                  "cinv": D.to_device(np.linalg.inv(M).astype(np.float32), torch.float32),
                  "block_level": block, "omega": omega, "scale": scale, "host": lv,
                  "cluster_top": MG_CLUSTER_TOP if cluster_top is None else int(cluster_top)}
        self._mg = self._mg_state(shared)
        return self._mg

    @staticmethod
    def _mg_state(shared):
        """This solver's multigrid work vectors and the oec_mg_t over them."""
        ops = shared["ops"]
        work = [{name: D.zeros(o["nx"] * o["ny"], torch.float32) for name in ("b", "x", "y")} for o in ops]
        levels = (MgLevel_t * len(ops))()
        for n_, (o, w) in enumerate(zip(ops, work)):
            levels[n_] = MgLevel_t(o["nx"], o["ny"], D.ptr(o["ex"]), D.ptr(o["ey"]), D.ptr(o["leak"]),
                                   D.ptr(o["dinv"]), D.ptr(o["inside"]), D.ptr(w["b"]), D.ptr(w["x"]),
                                   D.ptr(w["y"]))
        mg = Mg_t(len(ops), levels, shared["block_level"], shared["cidx"].shape[0], D.ptr(shared["cidx"]),
                  D.ptr(shared["cinv"]), shared["omega"], shared["scale"], shared.get("cluster_top", 0))
        keep = [dict(o, **w) for o, w in zip(ops, work)]
        return {"c": mg, "levels": levels, "work": work, "shared": shared, "keep": keep, "nlevels": len(ops),
                "block_level": shared["block_level"], "host": shared["host"]}

    def sibling(self):
        """A solver for another run on the same grid: shares the
        factorisation, the stencil, the field operator and the multigrid
        operators, and owns its phi, E, work areas and statistics, so
        siblings may solve at the same time (on different streams, or on the
        branches of one graph).  A trained network is not shared (its
        workspace is per network)."""
        s = copy.copy(self)
        npn = self.n_nodes
        s.phi = D.zeros(npn, torch.float64)
        s.eAtGridPoints = D.zeros(2 * npn, torch.float64)
        s._work = torch.zeros_like(self._work)
        s._pcg_work = torch.empty_like(self._pcg_work)
        s._stats_dev = torch.zeros_like(self._stats_dev)
        s._fb_count = torch.zeros_like(self._fb_count)
        s._phi_prev = s._ws_hist = None
        s._q_hist = s._q_count = None
        s._pcg_used = False
        s.nSolves = 0
        s.cnn = None
        s._mg = None if self._mg is None else PoissonSolver._mg_state(self._mg["shared"])
        return s

    def applyOperator(self, x):
        """A x on the inside nodes (device f64 [npExt] in and out)."""
        y = torch.empty_like(x)
        rc = _declare().oec_stencil_apply(ctypes.byref(self._stencil), x.data_ptr(), y.data_ptr(), D.stream())
        if rc:
            raise _lib.OecError("oec_stencil_apply", rc)
        return y

    # -------------------------------------------------------------- setup
    def _device_setup(self, tail):
        """Uploads the head/tail form of the factors (lu_setup.lu_host_arrays);
        the tail blocks are inverted on the device."""
        a = lu_host_arrays(self.ludecom, self.insidePointsInd, self.n_nodes, tail, inverses=False)
        self.tail = m = a["tail"]
        self._keep = {}
        k = self._keep
        for name in ("rhs_node", "sol_src", "sol_node", "l_rows", "l_ptr", "l_idx", "u_rows", "u_ptr", "u_idx",
                     "lc_ptr", "lc_idx"):
            if name in a:
                k[name] = D.to_device(a[name], torch.int32)
        for name in ("l_val", "u_val", "u_diag", "lc_val"):
            if name in a:
                k[name] = D.to_device(a[name], torch.float64)
        if m > 0:
            TL = D.to_device(a.pop("TL"), torch.float64)
            TU = D.to_device(a.pop("TU"), torch.float64)
            eye = torch.eye(m, dtype=torch.float64, device=D.device())
            k["tl_inv"] = torch.linalg.solve_triangular(TL, eye, upper=False, unitriangular=True).contiguous()
            k["tu_inv"] = torch.linalg.solve_triangular(TU, eye, upper=True).contiguous()
            del TL, TU, eye
        self._lu_host = a  # keeps the host level lists the solve reads
        self._l_level_ptr, self._u_level_ptr = a["l_level_ptr"], a["u_level_ptr"]
        self._l_level_lanes, self._u_level_lanes = a["l_level_lanes"], a["u_level_lanes"]
        self._lu_t = lu_struct(a, lambda name: D.ptr(k.get(name)))
        self._work = D.zeros(a["n"] + m + 1, torch.float64)
        E = self.phiToEAtGridPoints.tocsr()
        E.sort_indices()
        k["e_ptr"], k["e_idx"] = D.to_device(E.indptr, torch.int32), D.to_device(E.indices, torch.int32)
        k["e_val"] = D.to_device(E.data, torch.float64)
        self.levels = (a["l_nlevels"], a["u_nlevels"])

    # -------------------------------------------------------------- solve
    def _lu_solve(self, q):
        rc = _declare().oec_lu_solve(ctypes.byref(self._lu_t), q.data_ptr(), self.phi.data_ptr(),
                                     self._work.data_ptr(), D.stream())
        if rc:
            raise _lib.OecError("oec_lu_solve", rc)

    @property
    def lastStats(self):
        """PcgStats_t of the last iterative solve (None before the first)."""
        if not self._pcg_used:
            return None
        return PcgStats_t.from_buffer_copy(D.to_numpy(self._stats_dev).tobytes())

    @property
    def nFallbacks(self):
        """Iterative solves that missed pcgTol and were redone by LU."""
        return int(D.to_numpy(self._fb_count)[0])

    def resetHistory(self):
        """Forgets the earlier solutions and charges the warm starts use
        (when one solver object is handed from one run to the next)."""
        self._phi_prev = self._ws_hist = None
        self._q_hist = self._q_count = None
        self.phi.zero_()

    def prepare(self):
        """Builds what the configured iterative solve needs (the multigrid
        hierarchy) ahead of a CUDA graph capture that records the solve."""
        if self.method == "pcg" and self.precond == "mg" and self._mg is None:
            if torch.cuda.is_current_stream_capturing():
                raise RuntimeError("PoissonSolver.prepare() must run before the graph capture")
            self._mg_setup()
        if self.method == "pcg" and self.warmStart == "extrapolate+cnn" and self._q_hist is None:
            if torch.cuda.is_current_stream_capturing():
                raise RuntimeError("PoissonSolver.prepare() must run before the graph capture")
            self._q_hist = D.zeros(2 * self.n_nodes, torch.float64)
            self._q_count = D.zeros(1, torch.int32)
        if self.method == "pcg" and self.warmStart in ("extrapolate", "extrapolate+cnn") and self._phi_prev is None:
            if torch.cuda.is_current_stream_capturing():
                raise RuntimeError("PoissonSolver.prepare() must run before the graph capture")
            self._phi_prev = self.phi.clone()
            self._ws_hist = D.zeros(1, torch.int32)  # the first two solves start from phi itself

    def _pcg_solve(self, q):
        """Iterative solve warm-started from the current phi, with the LU
        solve run on the device when it misses pcgTol; enqueued without host
        synchronisation (and recorded whole when the stream is capturing)."""
        pc = PRECOND[self.precond]
        ctx = None
        if pc == PRECOND["mg"]:
            self.prepare()
            ctx = ctypes.cast(ctypes.pointer(self._mg["c"]), ctypes.c_void_p)
        elif pc == PRECOND["cnn"]:
            if self.cnn is None:
                raise ValueError("precond='cnn' needs a trained network in PoissonSolver.cnn")
            ctx = self.cnn.c_handle()
        if self.warmStart == "zero":
            self.phi.zero_()
        elif self.warmStart in ("extrapolate", "extrapolate+cnn"):
            self.prepare()
            rc = _declare().oec_warm_start_extrapolate(self.phi.data_ptr(), self._phi_prev.data_ptr(), self.n_nodes,
                                                       self._ws_hist.data_ptr(), D.stream())
            if rc:
                raise _lib.OecError("oec_warm_start_extrapolate", rc)
            if self.warmStart == "extrapolate+cnn":
                if self.cnn is None:
                    raise ValueError("warmStart='extrapolate+cnn' needs a trained network in PoissonSolver.cnn")
                self.cnn.correct(self._stencil.scale32, q, self._q_hist, self._q_count, self.phi)
        elif self.warmStart == "cnn":
            if self.cnn is None:
                raise ValueError("warmStart='cnn' needs a trained network in PoissonSolver.cnn")
            self.cnn.warm_start(self._stencil.scale32, q, self.phi)
        elif self.warmStart != "previous":
            raise ValueError("warmStart must be 'previous', 'extrapolate', 'extrapolate+cnn', 'zero' or 'cnn'")
        rc = _declare().oec_pcg_solve_async(ctypes.byref(self._stencil), q.data_ptr(), self.phi.data_ptr(),
                                            self.pcgTol, self.pcgMaxIter, pc, ctx, self._pcg_work.data_ptr(),
                                            self._stats_dev.data_ptr(), ctypes.byref(self._lu_t),
                                            self._work.data_ptr(), self._fb_count.data_ptr(), D.stream())
        if rc:
            raise _lib.OecError("oec_pcg_solve_async", rc)
        self._pcg_used = True

    def solveDevice(self, q, method=None):
        """q: device float64 [npExt] charge per node -> device E [2*npExt].

        method 'lu' (default of the instance: self.method) or 'pcg' (the
        device falls back to LU when the f64 relative residual misses
        pcgTol).  Enqueues work only: no host synchronisation, so a buildup
        step that contains it can be captured into a CUDA graph."""
        L = _declare()
        s = D.stream()
        method = method or self.method
        self.nSolves += 1
        if method == "pcg":
            self._pcg_solve(q)
        elif method == "lu":
            self._lu_solve(q)
        else:
            raise ValueError("method must be 'lu' or 'pcg'")
        k = self._keep
        rc = L.oec_spmv_csr(2 * self.n_nodes, k["e_ptr"].data_ptr(), k["e_idx"].data_ptr(), k["e_val"].data_ptr(),
                            self.phi.data_ptr(), self.eAtGridPoints.data_ptr(), s)
        if rc:
            raise _lib.OecError("oec_spmv_csr", rc)
        return self.eAtGridPoints

    def solve(self, q):
        """poissonSolver.pyx:83-88: charge per node (NOT density) -> E at nodes [Ex | Ey]."""
        qd = D.to_device(q, torch.float64).reshape(-1)
        if qd.shape[0] != self.n_nodes:
            raise ValueError("q must have npExt entries")
        self.solveDevice(qd)
        return D.to_numpy(self.eAtGridPoints)

    def getPhi(self):
        return D.to_numpy(self.phi)

    def getEAtGridPoints(self):
        return D.to_numpy(self.eAtGridPoints)

    def getPhiDevice(self):
        return self.phi

    def getEAtGridPointsDevice(self):
        return self.eAtGridPoints
