"""Host-side setup of the LU Poisson solve, without any GPU framework.

The reference assembles A = S diag(eps0 dsi dst~) S^T over the inside nodes
and factors it with SuperLU once per run (poissonSolver.pyx:33-67).  This
module does the same with scipy and lays the factors out for oec_lu_solve
(include/oec.h, oec_lu_t): head rows in level order with their level lists
and per-level lane counts, and the dense inverses of the tail blocks.  It
imports numpy, scipy and the library's ctypes binding only, so a host that
drives the library through its context/run handles needs nothing else.
"""
import ctypes

import numpy as np
import scipy.linalg.lapack as lapack
import scipy.sparse as spsp
import scipy.sparse.linalg as spspl

from . import _lib
from .constants import epsilon_0


class LU_t(ctypes.Structure):
    _P = ctypes.c_void_p
    _fields_ = [("n", ctypes.c_int32), ("head", ctypes.c_int32), ("n_nodes", ctypes.c_int32),
                ("rhs_node", _P), ("sol_src", _P), ("sol_node", _P),
                ("l_nlevels", ctypes.c_int32), ("l_level_ptr", _P), ("l_rows", _P),
                ("l_ptr", _P), ("l_idx", _P), ("l_val", _P), ("lc_ptr", _P), ("lc_idx", _P), ("lc_val", _P),
                ("tl_inv", _P), ("u_nlevels", ctypes.c_int32), ("u_level_ptr", _P), ("u_rows", _P),
                ("u_ptr", _P), ("u_idx", _P), ("u_val", _P), ("u_diag", _P), ("tu_inv", _P),
                ("head_path", ctypes.c_int32), ("l_level_lanes", _P), ("u_level_lanes", _P)]



def _declare_trsv():
    L = _lib.lib()
    if not getattr(L, "_trsv_declared", False):
        P = ctypes.c_void_p
        L.oec_trsv_levels.restype = ctypes.c_int
        L.oec_trsv_levels.argtypes = [ctypes.c_int32, P, P, ctypes.c_int32, ctypes.c_int32, P,
                                      ctypes.POINTER(ctypes.c_int32)]
        L._trsv_declared = True
    return L


def _np_ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _levels(csr, lower, ncols_dep, nrows=None):
    L = _declare_trsv()
    nrows = csr.shape[0] if nrows is None else nrows
    ptr = np.ascontiguousarray(csr.indptr[:nrows + 1], np.int32)
    idx = np.ascontiguousarray(csr.indices, np.int32)
    lev = np.zeros(max(nrows, 1), np.int32)
    nl = ctypes.c_int32(0)
    rc = L.oec_trsv_levels(nrows, _np_ptr(ptr), _np_ptr(idx), 1 if lower else 0, ncols_dep, _np_ptr(lev),
                           ctypes.byref(nl))
    if rc:
        raise _lib.OecError("oec_trsv_levels", rc)
    return lev[:nrows], nl.value


def _level_lists(lev, nlevels):
    order = np.argsort(lev, kind="stable").astype(np.int32)
    counts = np.bincount(lev, minlength=nlevels + 1)[1:]
    ptr = np.zeros(nlevels + 1, np.int32)
    np.cumsum(counts, out=ptr[1:])
    return order, ptr


def level_lanes(csr, level_ptr, threads=1024, max_per_lane=16):
    """Per head level (level-ordered CSR rows): the lanes per row with which
    one CTA of `threads` threads takes the level in one pass -- the largest
    power of two up to 32 with rows * lanes <= threads -- or 0 when the level
    is too wide for that or its longest row would need more than
    `max_per_lane` loads per lane (such a level keeps a launch of its own)."""
    level_ptr = np.asarray(level_ptr, np.int64)
    nl = level_ptr.size - 1
    lanes = np.zeros(max(nl, 1), np.int8)
    if nl <= 0:
        return lanes
    rows = np.diff(level_ptr)
    nnz = np.diff(np.asarray(csr.indptr, np.int64))
    longest = np.zeros(nl, np.int64)
    ne = rows > 0
    if nnz.size and ne.any():
        longest[ne] = np.maximum.reduceat(nnz, level_ptr[:-1][ne])
    for l in range(nl):
        r = int(rows[l])
        if r <= 0 or r > threads:
            continue
        g = 1
        while g < 32 and r * 2 * g <= threads:
            g *= 2
        if -(-int(longest[l]) // g) <= max_per_lane:
            lanes[l] = g
    return lanes


def choose_tail(Lcsr, Ucsr, n, launch_us=8.0, gbs=6000.0, max_tail=16384):
    """Rows handed to the dense tail: minimise the estimated solve time
    levels(head) * per-level cost + 2 * (m^2 * 8 B) / bandwidth over a few
    candidates.  The per-level cost (8 us) and the bandwidth of the dense
    products were measured on the B200 (128^2 to 1024^2); max_tail bounds the
    two dense inverses (2 * m^2 * 8 B: 4.3 GB at 16384), and the tail stays
    within a quarter of the unknowns: on a small grid a larger one streams
    more through L2 each step than it saves (a 128^2 buildup step ran slower
    with 6144 tail rows than with 3072 although the solve alone tied)."""
    best = (None, 0)
    for m in [0, 256, 512, 1024, 2048, 3072, 4096, 6144, 8192, 12288, 16384]:
        if m > min(n // 4, max_tail):
            continue
        h = n - m
        _, nl = _levels(Lcsr, True, h, nrows=h)
        _, nu = _levels(Ucsr, False, h, nrows=h)
        t = (nl + nu) * launch_us * 1e-6 + 2 * (m * m * 8) / (gbs * 1e9)
        if best[0] is None or t < best[0]:
            best = (t, m)
    return best[1]


def assemble(gridObj):
    """poissonSolver.pyx:41-58: A = S diag(meps) S^T over the inside nodes.

    Returns (A as CSC, meps [2*npExt] edge weights (x edges then y edges),
    S = [Px | Py] and the inside node indices)."""
    nx = gridObj.getNxExt()
    npn = gridObj.getNpExt()
    inside = np.nonzero(gridObj.getInsidePoints())[0]
    pxmt = spsp.identity(npn) - spsp.eye(npn, npn, -1)
    pymt = spsp.identity(npn) - spsp.eye(npn, npn, -int(nx))
    st = spsp.hstack([pxmt, pymt])
    meps = epsilon_0 * np.asarray(gridObj.getDsi()) * np.roll(gridObj.getDst(), npn)
    a = st.dot(spsp.diags(meps, 0).dot(st.transpose()))[:, inside].tocsc()[inside, :]
    return a, meps, st, inside


def factor(gridObj):
    """(A, meps, S, inside nodes, SuperLU factor of A with the reference's
    options, phiToEAtGridPoints) for a grid (poissonSolver.pyx:33-67)."""
    npn = gridObj.getNpExt()
    a, meps, st, inside = assemble(gridObj)
    lu = spspl.splu(a, permc_spec='MMD_AT_PLUS_A', diag_pivot_thresh=0.1)
    phi_to_e = gridObj.getEdgeToNode().dot(spsp.diags(gridObj.getDsi(), 0, (2 * npn, 2 * npn)).dot(st.transpose()))
    return a, meps, st, inside, lu, phi_to_e


def lu_host_arrays(lu, inside, n_nodes, tail=None, inverses=True):
    """The factors of `lu` (scipy SuperLU of A over the `inside` nodes) in
    oec_lu_t's layout as host arrays: the last m = `tail` rows (chosen by
    choose_tail when None) form the dense tail, the others are solved level
    by level.  With inverses=True the dense inverses of the tail's
    triangular blocks are computed here (LAPACK dtrtri); else "TL" / "TU"
    hold the blocks themselves for the caller to invert."""
    n = lu.shape[0]
    Lc = lu.L.tocsr()
    Uc = lu.U.tocsr()
    Lc.sort_indices()
    Uc.sort_indices()
    m = choose_tail(Lc, Uc, n) if tail is None else int(min(max(tail, 0), n))
    h = n - m
    ins = np.asarray(inside).astype(np.int32)
    inv_pr = np.empty(n, np.int64)
    inv_pr[lu.perm_r] = np.arange(n)
    a = {"n": n, "head": h, "tail": m, "n_nodes": int(n_nodes)}
    a["rhs_node"] = np.ascontiguousarray(ins[inv_pr], np.int32)
    a["sol_src"] = np.ascontiguousarray(lu.perm_c, np.int32)
    a["sol_node"] = np.ascontiguousarray(ins, np.int32)
    # strict lower L, head rows, in level order
    Lh = spsp.tril(Lc[:h, :], k=-1, format="csr")
    Lh.sort_indices()
    lev, nl = _levels(Lh, True, h)
    rows, lptr = _level_lists(lev, nl)
    Lh = Lh[rows]
    a.update(l_nlevels=nl, l_level_ptr=lptr, l_rows=rows, l_ptr=np.ascontiguousarray(Lh.indptr, np.int32),
             l_idx=np.ascontiguousarray(Lh.indices, np.int32), l_val=np.ascontiguousarray(Lh.data, np.float64),
             l_level_lanes=level_lanes(Lh, lptr))
    # strict upper U, head rows (all columns > row, tail columns included)
    Uh = spsp.triu(Uc[:h, :], k=1, format="csr")
    Uh.sort_indices()
    levu, nu = _levels(Uh, False, h)
    rowsu, uptr = _level_lists(levu, nu)
    Uh = Uh[rowsu]
    a.update(u_nlevels=nu, u_level_ptr=uptr, u_rows=rowsu, u_ptr=np.ascontiguousarray(Uh.indptr, np.int32),
             u_idx=np.ascontiguousarray(Uh.indices, np.int32), u_val=np.ascontiguousarray(Uh.data, np.float64),
             u_diag=np.ascontiguousarray(Uc.diagonal()[:h][rowsu] if h > 0 else np.zeros(1), np.float64),
             u_level_lanes=level_lanes(Uh, uptr))
    if m > 0:
        C = Lc[h:, :h].tocsr()
        C.sort_indices()
        a.update(lc_ptr=np.ascontiguousarray(C.indptr, np.int32), lc_idx=np.ascontiguousarray(C.indices, np.int32),
                 lc_val=np.ascontiguousarray(C.data, np.float64))
        TL = Lc[h:, h:].toarray()
        TU = Uc[h:, h:].toarray()
        if inverses:
            tl, info1 = lapack.dtrtri(TL, lower=1, unitdiag=1)
            tu, info2 = lapack.dtrtri(TU, lower=0, unitdiag=0)
            if info1 or info2:
                raise np.linalg.LinAlgError("singular tail block")
            a["tl_inv"] = np.ascontiguousarray(np.tril(tl, -1) + np.eye(m))
            a["tu_inv"] = np.ascontiguousarray(np.triu(tu))
        else:
            a["TL"], a["TU"] = TL, TU
    return a


def lu_struct(a, ptr):
    """An LU_t over the arrays of lu_host_arrays (host or device copies):
    `ptr(name)` gives the address of array `name` (None when absent); the
    level pointers and lane counts are always the host arrays of `a`."""
    s = LU_t()
    s.n, s.head, s.n_nodes = a["n"], a["head"], a["n_nodes"]
    for name in ("rhs_node", "sol_src", "sol_node", "l_rows", "l_ptr", "l_idx", "l_val", "lc_ptr", "lc_idx",
                 "lc_val", "tl_inv", "u_rows", "u_ptr", "u_idx", "u_val", "u_diag", "tu_inv"):
        setattr(s, name, ptr(name))
    s.l_nlevels, s.l_level_ptr = a["l_nlevels"], _np_ptr(a["l_level_ptr"]).value
    s.u_nlevels, s.u_level_ptr = a["u_nlevels"], _np_ptr(a["u_level_ptr"]).value
    s.l_level_lanes = _np_ptr(a["l_level_lanes"]).value
    s.u_level_lanes = _np_ptr(a["u_level_lanes"]).value
    return s
