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
the CSR product E = phiToE . phi (``oec_spmv_csr``).
"""
import ctypes

import numpy as np
import scipy.sparse as spsp
import scipy.sparse.linalg as spspl
import torch

from . import _lib
from . import device as D
from .constants import epsilon_0


class LU_t(ctypes.Structure):
    _P = ctypes.c_void_p
    _fields_ = [("n", ctypes.c_int32), ("head", ctypes.c_int32), ("n_nodes", ctypes.c_int32),
                ("rhs_node", _P), ("sol_src", _P), ("sol_node", _P),
                ("l_nlevels", ctypes.c_int32), ("l_level_ptr", _P), ("l_rows", _P),
                ("l_ptr", _P), ("l_idx", _P), ("l_val", _P), ("lc_ptr", _P), ("lc_idx", _P), ("lc_val", _P),
                ("tl_inv", _P), ("u_nlevels", ctypes.c_int32), ("u_level_ptr", _P), ("u_rows", _P),
                ("u_ptr", _P), ("u_idx", _P), ("u_val", _P), ("u_diag", _P), ("tu_inv", _P)]


_lib.OTHER_DECLARED.update({"oec_lu_solve", "oec_spmv_csr", "oec_trsv_levels"})


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
        L._poisson_declared = True
    return L


def _np_ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _levels(csr, lower, ncols_dep, nrows=None):
    L = _declare()
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


def choose_tail(Lcsr, Ucsr, n, launch_us=1.5, gbs=3000.0, max_tail=12288):
    """Rows handed to the dense tail: minimise the estimated solve time
    2*levels(head)*launch + 2*(m^2*8 B)/bandwidth over a few candidates."""
    best = (None, 0)
    for m in [0, 256, 512, 1024, 2048, 3072, 4096, 6144, 8192, 12288]:
        if m > min(n, max_tail):
            continue
        h = n - m
        _, nl = _levels(Lcsr, True, h, nrows=h)
        _, nu = _levels(Ucsr, False, h, nrows=h)
        t = (nl + nu) * launch_us * 1e-6 + 2 * (m * m * 8) / (gbs * 1e9)
        if best[0] is None or t < best[0]:
            best = (t, m)
    return best[1]


class PoissonSolver:
    """Reference: poissonSolver.pyx:33-67 (setup) and :83-98 (solve, getters)."""

    def __init__(self, gridObj, tail=None):
        nx = gridObj.getNxExt()
        npn = gridObj.getNpExt()
        self.gridObj = gridObj
        self.insidePointsInd = np.nonzero(gridObj.getInsidePoints())[0]
        pxmt = spsp.identity(npn) - spsp.eye(npn, npn, -1)
        pymt = spsp.identity(npn) - spsp.eye(npn, npn, -int(nx))
        st = spsp.hstack([pxmt, pymt])
        meps = epsilon_0 * np.asarray(gridObj.getDsi()) * np.roll(gridObj.getDst(), npn)
        a = st.dot(spsp.diags(meps, 0).dot(st.transpose()))[:, self.insidePointsInd].tocsc()[self.insidePointsInd, :]
        self.systemMatrix = a
        self.ludecom = spspl.splu(a, permc_spec='MMD_AT_PLUS_A', diag_pivot_thresh=0.1)
        self.phiToEAtGridPoints = gridObj.getEdgeToNode().dot(
            spsp.diags(gridObj.getDsi(), 0, (2 * npn, 2 * npn)).dot(st.transpose()))
        self.n_nodes = npn
        self._device_setup(tail)
        self.phi = D.zeros(npn, torch.float64)
        self.eAtGridPoints = D.zeros(2 * npn, torch.float64)

    # -------------------------------------------------------------- setup
    def _device_setup(self, tail):
        lu = self.ludecom
        n = lu.shape[0]
        Lc = lu.L.tocsr()
        Uc = lu.U.tocsr()
        Lc.sort_indices()
        Uc.sort_indices()
        m = choose_tail(Lc, Uc, n) if tail is None else int(min(max(tail, 0), n))
        h = n - m
        self.tail = m
        ins = self.insidePointsInd.astype(np.int32)
        inv_pr = np.empty(n, np.int64)
        inv_pr[lu.perm_r] = np.arange(n)
        dev = lambda a, dt=torch.int32: D.to_device(np.ascontiguousarray(a), dt)  # noqa: E731
        self._keep = {}
        k = self._keep
        k["rhs_node"] = dev(ins[inv_pr])
        k["sol_src"] = dev(lu.perm_c.astype(np.int32))
        k["sol_node"] = dev(ins)
        # strict lower L, head rows
        Lh = spsp.tril(Lc[:h, :], k=-1, format="csr")
        Lh.sort_indices()
        lev, nl = _levels(Lh, True, h)
        rows, lptr = _level_lists(lev, nl)
        k["l_rows"] = dev(rows)
        k["l_ptr"], k["l_idx"], k["l_val"] = dev(Lh.indptr), dev(Lh.indices), dev(Lh.data, torch.float64)
        self._l_level_ptr = lptr
        # strict upper U, head rows (all columns > row, tail columns included)
        Uh = spsp.triu(Uc[:h, :], k=1, format="csr")
        Uh.sort_indices()
        levu, nu = _levels(Uh, False, h)
        rowsu, uptr = _level_lists(levu, nu)
        k["u_rows"] = dev(rowsu)
        k["u_ptr"], k["u_idx"], k["u_val"] = dev(Uh.indptr), dev(Uh.indices), dev(Uh.data, torch.float64)
        k["u_diag"] = dev(Uc.diagonal()[:h], torch.float64) if h > 0 else D.zeros(1, torch.float64)
        self._u_level_ptr = uptr
        if m > 0:
            C = Lc[h:, :h].tocsr()
            C.sort_indices()
            k["lc_ptr"], k["lc_idx"], k["lc_val"] = dev(C.indptr), dev(C.indices), dev(C.data, torch.float64)
            TL = D.to_device(Lc[h:, h:].toarray(), torch.float64)
            TU = D.to_device(Uc[h:, h:].toarray(), torch.float64)
            eye = torch.eye(m, dtype=torch.float64, device=D.device())
            k["tl_inv"] = torch.linalg.solve_triangular(TL, eye, upper=False, unitriangular=True).contiguous()
            k["tu_inv"] = torch.linalg.solve_triangular(TU, eye, upper=True).contiguous()
            del TL, TU, eye
        else:
            for name in ("lc_ptr", "lc_idx", "lc_val", "tl_inv", "tu_inv"):
                k[name] = None
        s = LU_t()
        s.n, s.head, s.n_nodes = n, h, self.n_nodes
        for name in ("rhs_node", "sol_src", "sol_node", "l_rows", "l_ptr", "l_idx", "l_val", "lc_ptr", "lc_idx",
                     "lc_val", "tl_inv", "u_rows", "u_ptr", "u_idx", "u_val", "u_diag", "tu_inv"):
            setattr(s, name, D.ptr(k[name]))
        s.l_nlevels, s.l_level_ptr = nl, _np_ptr(self._l_level_ptr).value
        s.u_nlevels, s.u_level_ptr = nu, _np_ptr(self._u_level_ptr).value
        self._lu_t = s
        self._work = D.zeros(n + m + 1, torch.float64)
        E = self.phiToEAtGridPoints.tocsr()
        E.sort_indices()
        k["e_ptr"], k["e_idx"], k["e_val"] = dev(E.indptr), dev(E.indices), dev(E.data, torch.float64)
        self.levels = (nl, nu)

    # -------------------------------------------------------------- solve
    def solveDevice(self, q):
        """q: device float64 [npExt] charge per node -> device E [2*npExt]."""
        L = _declare()
        s = D.stream()
        rc = L.oec_lu_solve(ctypes.byref(self._lu_t), q.data_ptr(), self.phi.data_ptr(), self._work.data_ptr(), s)
        if rc:
            raise _lib.OecError("oec_lu_solve", rc)
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
