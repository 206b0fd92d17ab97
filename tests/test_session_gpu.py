"""A buildup run driven through the context and run handles of the C ABI
(oec_ctx_*, oec_run_*), from a process that never imports torch.

A child process sets the c1 run up with numpy and scipy only
(openecloud_b200.session), advances it through oec_run_steps (the step
graph, the LU solve and globalRandom owned by the library) and checks that
torch was never loaded; this process runs the same configuration through the
reference-API driver (Buildup) from the same initial rows.  The two launch
the same kernels in the same order with the same keys (emission: run seed,
particle slot, step; roulette: run seed + step, the run's count of
management events); they differ only in how the dense inverses of the LU
tail blocks are rounded (host LAPACK here, the device there), so the
histories agree exactly before the first management event and the particle
state to FP32 rounding; afterwards the counts and weights stay within a
fraction of a percent."""
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

CHILD = r"""
import sys
import numpy as np
sys.path.insert(0, {root!r})
from openecloud_b200.session import Context, Run
rows = np.load({rows!r})
with Context(0) as ctx:
    run = Run(ctx, rows, seed=77, n_steps_table=161)
    run.steps(40)
    rows40 = run.getParticleData()
    run.steps(110)
    c, w = run.history()
    st = ctx.status()
    run.close()
assert "torch" not in sys.modules, "torch was imported"
np.savez({out!r}, rows40=rows40, counts=c, weights=w, dropped=st["n_rows_dropped"])
print("child ok")
"""


def _rows(n=10000, seed=3):
    rng = np.random.default_rng(seed)
    r = np.sqrt(rng.uniform(0, 1, n)) * 0.0199
    a = rng.uniform(0, 2 * np.pi, n)
    rows = np.zeros((n, 6))
    rows[:, 0], rows[:, 1] = r * np.cos(a), r * np.sin(a)
    rows[:, 5] = 1e9 / n
    return rows


def test_run_handle_without_torch_matches_buildup(gpu, tmp_path):
    from openecloud_b200.buildup import Buildup
    rows = _rows()
    np.save(tmp_path / "rows.npy", rows)
    code = CHILD.format(root=ROOT, rows=str(tmp_path / "rows.npy"), out=str(tmp_path / "out.npz"))
    p = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600,
                       env=dict(os.environ))
    assert p.returncode == 0, p.stdout[-2000:] + p.stderr[-4000:]
    got = np.load(tmp_path / "out.npz")
    b = Buildup(seed=77, n_steps_table=161)
    b.P.setParticleData(rows)
    b._prepare_deposit()
    b.run(40)
    mine = b.P.getParticleData()
    rows40 = got["rows40"]
    assert rows40.shape == mine.shape
    scale = np.max(np.abs(mine), axis=0)
    assert np.all(np.max(np.abs(rows40 - mine), axis=0) <= 1e-6 * scale)
    b.run(110)
    n, w = b.history()
    assert np.array_equal(got["counts"][:41], n[:41])
    assert np.max(np.abs(got["weights"][:41] / w[:41] - 1)) <= 1e-12
    # the first roulette (step 50) clones up to the target of 1e5
    assert abs(got["counts"][51] / 1e5 - 1) < 0.01 and abs(n[51] / 1e5 - 1) < 0.01
    assert np.max(np.abs(got["counts"][51:].astype(float) / n[51:] - 1)) < 0.005
    assert np.max(np.abs(got["weights"][51:] / w[51:] - 1)) < 0.005
    assert int(got["dropped"]) == 0
