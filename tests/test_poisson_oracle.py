"""The oracle's Poisson solve (poissonSolver.pyx:33-88 restated) against the
compiled reference's phi and E on every grid fixture, bit for bit."""
import numpy as np
import pytest

from conftest import golden
from oracle.poisson_oracle import from_golden


@pytest.mark.parametrize("name", ["rect_24x20", "circle_32", "ellipse_40x24", "circle_128"])
def test_poisson_oracle_replays_reference(name):
    z = golden(f"grid_{name}.npz")
    phi, e = from_golden(z).solve(z["poisson_q"])
    assert np.array_equal(phi, z["poisson_phi"])
    assert np.array_equal(e, z["poisson_E"])
