"""Statistical parity of the device buildup loop with the reference.

Configuration: 128x128 circular chamber R = 20 mm, 1e4 initial electrons,
endless bunch train (sigma_r 2 mm, sigma_t 0.25 ns, 1.1e11 protons, 25 ns),
copper SEY with delta_max 1.6 and E_max 300 eV, roulette cap 1e5 every 50
steps, dt = 1e-11 s, one bunch passage (2500 steps).  The golden file holds
the reference's line density for 8 seeds; the ensemble mean of 8 device runs
must stay within twice the reference's seed-to-seed spread (floor 0.2%).
"""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


def test_buildup_line_density_within_reference_spread(gpu):
    from openecloud_b200.buildup import Buildup
    z = golden("buildup_c1.npz")
    every = int(z["every"])
    ref = z["weight"]
    runs = []
    for s in range(8):
        b = Buildup(seed=1000 + s, n_steps_table=2501)
        b.run(2500)
        n, w = b.history()
        st = b.status()
        assert st["n_capacity_drop"] == 0 and st["n_nonfinite"] == 0
        runs.append(w[::every])
    gpu_w = np.array(runs)
    m_ref, s_ref = ref.mean(0), ref.std(0, ddof=1)
    m_gpu = gpu_w.mean(0)
    tol = 2 * np.maximum(s_ref, 0.002 * m_ref)
    bad = np.abs(m_gpu - m_ref) > tol
    assert not bad.any(), (np.nonzero(bad)[0][:10], m_gpu[bad][:5], m_ref[bad][:5])
    # the cloud builds up over the passage as in the reference
    assert m_gpu[-1] / m_gpu[0] > 1.2
