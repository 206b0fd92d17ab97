"""Learned preconditioner for the iterative Poisson solve.

A linear 4-level U-Net (16-32-64-64 channels, 3x3 convolutions, bf16 weights
and activations with f32 accumulation; kernels in ``csrc/cnn.cu``) that maps a
residual r on the extended grid to z ~ A32^-1 r, where A32 is the scaled FIT
operator of ``oec_pcg_solve``.  It is trained on the device by the project's
own forward and backward kernels (``oec_cnn_train_step``, Adam) on inputs of
the same grid: charges from the simulation's kind of sources (beam and cloud
blobs) and rough fields, with either the supervised loss
sum (N(x) - phi)^2 / sum phi^2 (phi from the LU solve) or the residual loss
sum (A N(x) - x)^2 / sum x^2, which weighs every spatial frequency of the
residuals that a preconditioner meets inside CG.  Plugged into
``PoissonSolver`` with ``precond='cnn'``.  No counterpart in the reference (its solve is SuperLU
only, poissonSolver.pyx:59, :85).
"""
import ctypes

import numpy as np
import torch

from . import _lib
from . import device as D


class Cnn_t(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("inside", ctypes.c_void_p),
                ("w16", ctypes.c_void_p), ("act", ctypes.c_void_p), ("conv_kernel", ctypes.c_int32)]


CONV_KERNELS = {"tcgen05": 0, "mma.sync": 1}  # OEC_CNN_CONV_TCGEN05, OEC_CNN_CONV_MMA_SYNC
CONV_KERNEL = "tcgen05"  # default kernel of the 3x3 convolutions (0.31 vs 0.40 ms per 1026^2 forward pass)


_lib.OTHER_DECLARED.update({"oec_cnn_num_params", "oec_cnn_param_layout", "oec_cnn_act_bytes", "oec_cnn_forward",
                            "oec_cnn_set_weights", "oec_cnn_train_step", "oec_cnn_warm_start_work_bytes",
                            "oec_cnn_warm_start", "oec_cnn_correct_work_bytes", "oec_cnn_correct",
                            "oec_cnn_status"})

SPECS = [(1, 16), (16, 32), (32, 64), (64, 64), (64, 32), (32, 16), (16, 16)]  # (in, out) of e0 e1 e2 e3 d2 d1 d0


def _declare():
    L = _lib.lib()
    if not getattr(L, "_cnn_declared", False):
        P = ctypes.c_void_p
        L.oec_cnn_num_params.restype = ctypes.c_int32
        L.oec_cnn_num_params.argtypes = []
        L.oec_cnn_param_layout.restype = ctypes.c_int
        L.oec_cnn_param_layout.argtypes = [P, P]
        L.oec_cnn_act_bytes.restype = ctypes.c_int64
        L.oec_cnn_act_bytes.argtypes = [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32]
        L.oec_cnn_forward.restype = ctypes.c_int
        L.oec_cnn_forward.argtypes = [ctypes.POINTER(Cnn_t), P, P, P]
        L.oec_cnn_status.restype = ctypes.c_int
        L.oec_cnn_status.argtypes = [ctypes.POINTER(Cnn_t), P, P]
        L.oec_cnn_set_weights.restype = ctypes.c_int
        L.oec_cnn_set_weights.argtypes = [ctypes.POINTER(Cnn_t), P, P]
        L.oec_cnn_warm_start_work_bytes.restype = ctypes.c_int64
        L.oec_cnn_warm_start_work_bytes.argtypes = [ctypes.c_int32, ctypes.c_int32]
        L.oec_cnn_warm_start.restype = ctypes.c_int
        L.oec_cnn_warm_start.argtypes = [ctypes.POINTER(Cnn_t), ctypes.c_double, P, P, P, P]
        L.oec_cnn_correct_work_bytes.restype = ctypes.c_int64
        L.oec_cnn_correct_work_bytes.argtypes = [ctypes.c_int32, ctypes.c_int32]
        L.oec_cnn_correct.restype = ctypes.c_int
        L.oec_cnn_correct.argtypes = [ctypes.POINTER(Cnn_t), ctypes.c_double, P, P, P, P, P, P]
        L.oec_cnn_train_step.restype = ctypes.c_int
        L.oec_cnn_train_step.argtypes = [ctypes.POINTER(Cnn_t), P, P, P, P, P, P, P, P, P, ctypes.c_float,
                                         ctypes.c_int32, ctypes.c_int32, P, P]
        L._cnn_declared = True
    return L


def param_layout():
    off = (ctypes.c_int32 * 9)()
    shp = (ctypes.c_int32 * 24)()
    rc = _declare().oec_cnn_param_layout(off, shp)
    if rc:
        raise _lib.OecError("oec_cnn_param_layout", rc)
    return list(off), [tuple(shp[3 * i:3 * i + 3]) for i in range(8)]


def init_weights(seed=0):
    """Variance-preserving random start: N(0, 1/(9 c_in)) per 3x3 layer."""
    rng = np.random.default_rng(seed)
    parts = [rng.normal(0.0, np.sqrt(1.0 / (9 * ci)), co * 9 * ci) for ci, co in SPECS]
    parts.append(rng.normal(0.0, np.sqrt(1.0 / 16), 16))
    return np.concatenate(parts)


class PoissonCNN:
    """The network on one extended grid (nx, ny) with its inside mask."""

    def __init__(self, nx, ny, inside, weights=None, seed=0, training=True, op=None, conv_kernel=None):
        L = _declare()
        kernel = CONV_KERNEL if conv_kernel is None else conv_kernel
        if kernel not in CONV_KERNELS:
            raise ValueError(f"conv_kernel must be one of {sorted(CONV_KERNELS)}")
        self.conv_kernel = kernel
        self.nx, self.ny = int(nx), int(ny)
        self.n = L.oec_cnn_num_params()
        self.inside = D.to_device(np.asarray(inside).astype(np.uint8).reshape(-1), torch.uint8)
        if self.inside.shape[0] != self.nx * self.ny:
            raise ValueError("inside must have nx*ny entries")
        w = init_weights(seed) if weights is None else np.asarray(weights, np.float64)
        if w.shape[0] != self.n:
            raise ValueError(f"expected {self.n} weights")
        self.w32 = D.to_device(w.astype(np.float32), torch.float32)
        self.w16 = D.zeros(self.n, torch.int16)
        self.training = bool(training)
        self.op = op  # oec_stencil_t of the scaled operator (residual loss), or None
        self.act = D.empty(int(L.oec_cnn_act_bytes(self.nx, self.ny, 1 if training else 0)), torch.uint8)
        self.c = Cnn_t(self.nx, self.ny, D.ptr(self.inside), D.ptr(self.w16), D.ptr(self.act),
                       CONV_KERNELS[kernel])
        self._check(L.oec_cnn_set_weights(ctypes.byref(self.c), self.w32.data_ptr(), D.stream()), "set_weights")
        if training:
            self.grad = D.zeros(self.n, torch.float32)
            self.m = D.zeros(self.n, torch.float32)
            self.v = D.zeros(self.n, torch.float32)
            self.wt16 = D.zeros(self.n, torch.int16)
            self.z = D.zeros(self.nx * self.ny, torch.float32)
            self.loss_dev = D.zeros(2, torch.float64)
            self.step = 0

    @staticmethod
    def _check(rc, what):
        if rc:
            raise _lib.OecError("oec_cnn_" + what, rc)

    @classmethod
    def for_solver(cls, ps, **kw):
        """The network on a PoissonSolver's extended grid and inside mask."""
        g = ps.gridObj
        return cls(g.getNxExt(), g.getNyExt(), np.asarray(g.getInsidePoints()) != 0, op=ps._stencil, **kw)

    def c_handle(self):
        return ctypes.cast(ctypes.pointer(self.c), ctypes.c_void_p)

    def wait_timeouts(self):
        """Bounded tensor-memory waits of the tcgen05 convolutions that gave
        up during the last forward pass or training step (0 on a healthy
        device)."""
        n = ctypes.c_int32(0)
        self._check(_declare().oec_cnn_status(ctypes.byref(self.c), ctypes.byref(n), D.stream()), "status")
        return int(n.value)

    def forward(self, x, out=None):
        """z = N(x) on the device (f32 [nx*ny])."""
        out = torch.empty_like(x) if out is None else out
        self._check(_declare().oec_cnn_forward(ctypes.byref(self.c), x.data_ptr(), out.data_ptr(), D.stream()),
                    "forward")
        return out

    def warm_start(self, scale32, q, phi):
        """phi <- |b| N(b/|b|), b = scale32 q (device f64 [nx*ny])."""
        L = _declare()
        if getattr(self, "_ws_work", None) is None:
            self._ws_work = D.empty(int(L.oec_cnn_warm_start_work_bytes(self.nx, self.ny)), torch.uint8)
        self._check(L.oec_cnn_warm_start(ctypes.byref(self.c), float(scale32), q.data_ptr(), phi.data_ptr(),
                                         self._ws_work.data_ptr(), D.stream()), "warm_start")
        return phi

    def correct(self, scale32, q, q_hist, count, phi):
        """phi += the network's estimate of A^-1 (q - 2 q1 + q2), the part of
        phi that the linear extrapolation in time misses (q_hist: device f64
        [2 * nx * ny] holding q1, q2; count: device int32, earlier charges
        seen, saturating at 2; both advanced here)."""
        L = _declare()
        if getattr(self, "_corr_work", None) is None:
            self._corr_work = D.empty(int(L.oec_cnn_correct_work_bytes(self.nx, self.ny)), torch.uint8)
        self._check(L.oec_cnn_correct(ctypes.byref(self.c), float(scale32), q.data_ptr(), q_hist.data_ptr(),
                                      count.data_ptr(), phi.data_ptr(), self._corr_work.data_ptr(), D.stream()),
                    "correct")
        return phi

    def _op_arg(self, loss):
        if loss == "residual":
            if self.op is None:
                raise ValueError("the residual loss needs the operator (PoissonCNN.for_solver)")
            return ctypes.byref(self.op)
        if loss != "supervised":
            raise ValueError("loss must be 'supervised' or 'residual'")
        return None

    def loss_and_grad(self, x, t=None, loss="supervised"):
        """(loss, gradient f32 [n], z) of one input without an update."""
        op = self._op_arg(loss)
        self._check(_declare().oec_cnn_train_step(ctypes.byref(self.c), op, x.data_ptr(), D.ptr(t),
                                                  self.z.data_ptr(), None, self.grad.data_ptr(), None, None,
                                                  self.wt16.data_ptr(), 0.0, 0, 0, self.loss_dev.data_ptr(),
                                                  D.stream()), "train_step")
        s = D.to_numpy(self.loss_dev)
        return s[0] / s[1], self.grad, self.z

    def train(self, xs, ts, steps, lr=1e-3, lr_final=None, seed=0, log_every=0, loss="supervised"):
        """Adam on inputs xs[i] (targets ts[i] for the supervised loss) drawn at
        random; returns the loss per step."""
        L = _declare()
        op = self._op_arg(loss)
        rng = np.random.default_rng(seed)
        losses = np.empty(steps)
        lr_final = lr if lr_final is None else lr_final
        hist = D.zeros((steps, 2), torch.float64)
        for k in range(steps):
            i = int(rng.integers(len(xs)))
            self.step += 1
            lr_k = lr * (lr_final / lr) ** (k / max(steps - 1, 1))
            t = None if ts is None else ts[i]
            self._check(L.oec_cnn_train_step(ctypes.byref(self.c), op, xs[i].data_ptr(), D.ptr(t),
                                             self.z.data_ptr(), self.w32.data_ptr(), self.grad.data_ptr(),
                                             self.m.data_ptr(), self.v.data_ptr(), self.wt16.data_ptr(), lr_k,
                                             self.step, 1, hist[k].data_ptr(), D.stream()), "train_step")
            if log_every and (k + 1) % log_every == 0:
                h = D.to_numpy(hist[k])
                print(f"[cnn] step {k + 1} loss {h[0] / h[1]:.4e}", flush=True)
        h = D.to_numpy(hist)
        losses[:] = h[:, 0] / h[:, 1]
        return losses

    def weights(self):
        return D.to_numpy(self.w32).astype(np.float64)


def make_pairs(ps, n, seed=0, blobs=(2, 12), rough=0.0):
    """Training pairs (x, t) on a PoissonSolver's grid: x = s q / |s q| with q a
    random charge per node (sums of Gaussian blobs of random width, sign and
    position inside the chamber, a beam-like blob at the centre half of the
    time; with probability `rough` instead white noise box-filtered over
    1, 2, 4 or 8 nodes), t = phi / |s q| with A phi = q from the LU solve
    (s = the scale of the f32 operator).  Returns device lists of f32 [npExt]
    tensors."""
    rng = np.random.default_rng(seed)
    g = ps.gridObj
    nx, ny = g.getNxExt(), g.getNyExt()
    X = np.tile(np.asarray(g.getXMesh()), ny)
    Y = np.repeat(np.asarray(g.getYMesh()), nx)
    inside = np.asarray(g.getInsidePoints()) != 0
    lx, ly = g.getLx(), g.getLy()
    xs, ts = [], []
    s32 = ps._stencil.scale32
    for _ in range(n):
        q = np.zeros(nx * ny)
        if rng.random() < rough:
            f = int(rng.choice([1, 2, 4, 8]))
            a = rng.normal(size=(ny // f + 1, nx // f + 1))
            q = np.repeat(np.repeat(a, f, 0), f, 1)[:ny, :nx].reshape(-1)
            q = np.where(inside, q, 0.0) * 1e-12
            qd = D.to_device(q, torch.float64)
            ps.solveDevice(qd, method="lu")
            nrm = float(np.linalg.norm(q)) * s32
            xs.append((qd * (s32 / nrm)).float())
            ts.append((ps.phi / nrm).float())
            continue
        for _ in range(int(rng.integers(blobs[0], blobs[1] + 1))):
            cx, cy = rng.uniform(-0.45, 0.45) * lx, rng.uniform(-0.45, 0.45) * ly
            sg = rng.uniform(0.01, 0.25) * min(lx, ly)
            q += rng.uniform(-1.0, 1.0) * np.exp(-((X - cx) ** 2 + (Y - cy) ** 2) / (2 * sg * sg))
        if rng.random() < 0.5:
            sg = rng.uniform(0.02, 0.06) * min(lx, ly)
            q += rng.uniform(1.0, 4.0) * np.exp(-(X ** 2 + Y ** 2) / (2 * sg * sg))
        q = np.where(inside, q, 0.0) * 1e-12
        qd = D.to_device(q, torch.float64)
        ps.solveDevice(qd, method="lu")
        phi = ps.phi.clone()
        nrm = float(np.linalg.norm(q)) * s32
        xs.append((qd * (s32 / nrm)).float())
        ts.append((phi / nrm).float())
    return xs, ts
