"""Oracle (test infrastructure only): float64 numpy restatements of the
multipole field and the mean-energy diagnostic.

* `multipole_expansion` follows magneticField.pyx:23-59: node (ii, jj) at
  (xMesh[ii], yMesh[jj]), r = sqrt(x^2 + y^2), phi = atan2(y, x) moved to
  [0, 2 pi), B_r = sum_k r^k (-skew_k cos((k+1) phi) + normal_k sin((k+1) phi)),
  B_phi = sum_k r^k (skew_k sin((k+1) phi) + normal_k cos((k+1) phi)),
  Bx = B_r cos phi - B_phi sin phi, By = B_r sin phi + B_phi cos phi, Bz = 0;
  a skew list shorter than the normal one is padded with zeros (:38-42), the
  order is the normal list's length (:50).
* `average_energy` follows util.pyx:8-20: sum (vx^2 + vy^2 + vz^2) w times
  m / (2 e) over sum w.
"""
import numpy as np

ELEMENTARY_CHARGE = 1.602176565e-19  # constants.pyx:3
ELECTRON_MASS = 9.10938291e-31       # constants.pyx:4


def multipole_expansion(xmesh, ymesh, normal, skew=()):
    normal = np.asarray(normal, np.float64)
    n = normal.size
    sk = np.zeros(n)
    s_in = np.asarray(skew, np.float64)
    sk[:min(n, s_in.size)] = s_in[:n]
    X, Y = np.meshgrid(np.asarray(xmesh, np.float64), np.asarray(ymesh, np.float64))
    r = np.sqrt(X ** 2 + Y ** 2)
    phi = np.arctan2(Y, X)
    phi = np.where(phi < 0, phi + 2 * np.pi, phi)
    br = np.zeros_like(r)
    bphi = np.zeros_like(r)
    for k in range(n):
        rk = r ** k
        br += rk * (-sk[k] * np.cos((k + 1) * phi) + normal[k] * np.sin((k + 1) * phi))
        bphi += rk * (sk[k] * np.sin((k + 1) * phi) + normal[k] * np.cos((k + 1) * phi))
    bx = br * np.cos(phi) - bphi * np.sin(phi)
    by = br * np.sin(phi) + bphi * np.cos(phi)
    return np.concatenate([bx.ravel(), by.ravel(), np.zeros(bx.size)])


def average_energy(pd, mass=ELECTRON_MASS):
    pd = np.asarray(pd, np.float64)
    e = np.sum((pd[:, 2] ** 2 + pd[:, 3] ** 2 + pd[:, 4] ** 2) * pd[:, 5])
    return e * mass * 0.5 / ELEMENTARY_CHARGE / np.sum(pd[:, 5])
