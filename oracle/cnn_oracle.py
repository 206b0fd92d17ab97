"""Oracle (test infrastructure only): numpy restatement of the learned
Poisson preconditioner of ``openecloud_b200/csrc/cnn.cu``.

The network has no counterpart in the reference; this file restates the
device network in float64 so that its forward pass, its loss and its
parameter gradients can be checked.  With ``bf16=True`` every value the
device stores in bf16 (inputs of each convolution, every activation and
activation gradient, the weights) is rounded to bf16 (round to nearest even)
at the same point, so the device and the oracle differ only by f32 versus f64
accumulation.  ``finite_difference_check`` validates the oracle's own
gradients in plain float64.

Network (extended grid of ny x nx nodes, level l has ceil(n / 2^l) per side):
  e0 = conv(x, 1->16); e1 = conv(pool e0, 16->32); e2 = conv(pool e1, 32->64);
  e3 = conv(pool e2, 64->64); u2 = up(e3) + e2; d2 = conv(u2, 64->32);
  u1 = up(d2) + e1; d1 = conv(u1, 32->16); u0 = up(d1) + e0;
  d0 = conv(u0, 16->16); z = inside * (d0 . w_out)
conv: 3x3, zero outside the image, weights [out][tap = 3 ty + tx][in];
pool: 0.25 * sum of the in-range 2x2 children; up: copy to the children.
"""
import numpy as np

SPECS = [(1, 16), (16, 32), (32, 64), (64, 64), (64, 32), (32, 16), (16, 16)]  # (in, out)


def layout():
    """Offsets of the 7 conv layers and the 1x1 output in the flat vector."""
    off = [0]
    for ci, co in SPECS:
        off.append(off[-1] + co * 9 * ci)
    off.append(off[-1] + 16)
    return off  # len 9: 7 conv starts, output start, total


def bf16(a):
    """Round float64 values to bf16 (via f32, round to nearest even), as float64."""
    f = np.asarray(a, np.float64).astype(np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def _unpack(w):
    off = layout()
    convs = [w[off[i]:off[i + 1]].reshape(co, 9, ci) for i, (ci, co) in enumerate(SPECS)]
    return convs, w[off[7]:off[8]]


def conv3(x, wk):
    """x [h, w, ci], wk [co, 9, ci] -> [h, w, co]."""
    h, wd, ci = x.shape
    xp = np.zeros((h + 2, wd + 2, ci))
    xp[1:-1, 1:-1] = x
    out = np.zeros((h, wd, wk.shape[0]))
    for tap in range(9):
        ty, tx = divmod(tap, 3)
        out += xp[ty:ty + h, tx:tx + wd] @ wk[:, tap, :].T
    return out


def conv3_back(x, wk, g):
    """Gradients of conv3(x, wk) given g = dL/dout: (dL/dx, dL/dwk)."""
    h, wd, ci = x.shape
    xp = np.zeros((h + 2, wd + 2, ci))
    xp[1:-1, 1:-1] = x
    gw = np.zeros_like(wk)
    gxp = np.zeros_like(xp)
    for tap in range(9):
        ty, tx = divmod(tap, 3)
        gw[:, tap, :] = np.einsum("hwo,hwi->oi", g, xp[ty:ty + h, tx:tx + wd])
        gxp[ty:ty + h, tx:tx + wd] += g @ wk[:, tap, :]
    return gxp[1:-1, 1:-1], gw


def pool(x):
    h, wd, c = x.shape
    H, W = (h + 1) // 2, (wd + 1) // 2
    xp = np.zeros((2 * H, 2 * W, c))
    xp[:h, :wd] = x
    return 0.25 * (xp[0::2, 0::2] + xp[1::2, 0::2] + xp[0::2, 1::2] + xp[1::2, 1::2])


def up(x, shape):
    return np.repeat(np.repeat(x, 2, axis=0), 2, axis=1)[:shape[0], :shape[1]]


def down_sum(g, coarse_shape):
    H, W = coarse_shape
    h, wd, c = g.shape
    gp = np.zeros((2 * H, 2 * W, c))
    gp[:h, :wd] = g
    return gp[0::2, 0::2] + gp[1::2, 0::2] + gp[0::2, 1::2] + gp[1::2, 1::2]


def forward(w, x, inside, bf=True):
    """x, inside: [ny, nx]; returns z [ny, nx] and the cache for backward."""
    R = bf16 if bf else (lambda a: np.asarray(a, np.float64))
    convs, wout = _unpack(R(w))
    x0 = R(np.where(inside, x, 0.0))[..., None]
    c = {"x0": x0, "convs": convs, "wout": wout}
    e0 = R(conv3(x0, convs[0]))
    p1 = R(pool(e0))
    e1 = R(conv3(p1, convs[1]))
    p2 = R(pool(e1))
    e2 = R(conv3(p2, convs[2]))
    p3 = R(pool(e2))
    e3 = R(conv3(p3, convs[3]))
    u2 = R(up(e3, e2.shape) + e2)
    d2 = R(conv3(u2, convs[4]))
    u1 = R(up(d2, e1.shape) + e1)
    d1 = R(conv3(u1, convs[5]))
    u0 = R(up(d1, e0.shape) + e0)
    d0 = R(conv3(u0, convs[6]))
    z = np.where(inside, d0 @ wout, 0.0)
    c.update(e0=e0, p1=p1, e1=e1, p2=p2, e2=e2, p3=p3, e3=e3, u2=u2, d2=d2, u1=u1, d1=d1, u0=u0, d0=d0,
             inside=inside, R=R)
    return z, c


def loss_and_grad(w, x, t, inside, bf=True):
    """loss = sum_inside (z - t)^2 / sum_inside t^2 and its gradient (flat)."""
    z, c = forward(w, x, inside, bf)
    tt = float(np.sum(np.where(inside, t, 0.0) ** 2))
    loss = float(np.sum(np.where(inside, z - t, 0.0) ** 2)) / tt
    gz = np.where(inside, 2.0 * (z - t) / tt, 0.0)
    return loss, backward(c, gz), z


def residual_loss_and_grad(w, x, inside, apply_a, bf=True):
    """Scale-free residual loss min_s |s A z - x|^2 / |x|^2 = 1 - (Az.x)^2 /
    (|Az|^2 |x|^2) (apply_a: the symmetric operator on [ny, nx] arrays) and
    its gradient (2 s / |x|^2) A (s A z - x), s = (Az.x) / |Az|^2."""
    z, c = forward(w, x, inside, bf)
    xm = np.where(inside, x, 0.0)
    y = apply_a(z)
    a, b, cc = float(np.sum(y * y)), float(np.sum(xm * xm)), float(np.sum(y * xm))
    s = cc / a
    loss = 1.0 - cc * cc / (a * b)
    gz = np.where(inside, (2.0 * s / b) * apply_a(s * y - xm), 0.0)
    return loss, backward(c, gz), z


def backward(c, gz):
    """Parameter gradient (flat) of the forward pass cached in c for dL/dz = gz."""
    R, convs = c["R"], c["convs"]
    gw = [None] * 7
    g_out = np.einsum("hw,hwc->c", gz, c["d0"])
    gd0 = R(gz[..., None] * c["wout"][None, None, :])
    gu0, gw[6] = conv3_back(c["u0"], convs[6], gd0)
    gu0 = R(gu0)
    gd1 = R(down_sum(gu0, c["d1"].shape[:2]))
    gu1, gw[5] = conv3_back(c["u1"], convs[5], gd1)
    gu1 = R(gu1)
    gd2 = R(down_sum(gu1, c["d2"].shape[:2]))
    gu2, gw[4] = conv3_back(c["u2"], convs[4], gd2)
    gu2 = R(gu2)
    ge3 = R(down_sum(gu2, c["e3"].shape[:2]))
    gp3, gw[3] = conv3_back(c["p3"], convs[3], ge3)
    gp3 = R(gp3)
    ge2 = R(gu2 + 0.25 * up(gp3, gu2.shape))
    gp2, gw[2] = conv3_back(c["p2"], convs[2], ge2)
    gp2 = R(gp2)
    ge1 = R(gu1 + 0.25 * up(gp2, gu1.shape))
    gp1, gw[1] = conv3_back(c["p1"], convs[1], ge1)
    gp1 = R(gp1)
    ge0 = R(gu0 + 0.25 * up(gp1, gu0.shape))
    _, gw[0] = conv3_back(c["x0"], convs[0], ge0)
    return np.concatenate([g.reshape(-1) for g in gw] + [g_out])


def finite_difference_check(ny=10, nx=13, n_probe=12, seed=0, h=1e-6):
    """Max relative difference between the oracle's float64 gradient and
    central differences of its loss, over random parameter indices."""
    rng = np.random.default_rng(seed)
    inside = rng.random((ny, nx)) > 0.2
    x = rng.normal(size=(ny, nx))
    t = rng.normal(size=(ny, nx))
    w = init_weights(seed)
    _, g, _ = loss_and_grad(w, x, t, inside, bf=False)
    worst = 0.0
    for i in rng.choice(w.size, n_probe, replace=False):
        wp, wm = w.copy(), w.copy()
        wp[i] += h
        wm[i] -= h
        fd = (loss_and_grad(wp, x, t, inside, bf=False)[0] - loss_and_grad(wm, x, t, inside, bf=False)[0]) / (2 * h)
        worst = max(worst, abs(fd - g[i]) / max(abs(g[i]), 1e-3 * np.max(np.abs(g))))
    return worst


def init_weights(seed=0):
    """Variance-preserving random start (the device module uses the same rule)."""
    rng = np.random.default_rng(seed)
    parts = [rng.normal(0.0, np.sqrt(1.0 / (9 * ci)), co * 9 * ci) for ci, co in SPECS]
    parts.append(rng.normal(0.0, np.sqrt(1.0 / 16), 16))
    return np.concatenate(parts)
