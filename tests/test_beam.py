"""Beam imprint (host setup) against the reference's beam.py values."""
import numpy as np

from conftest import golden


def test_beam_profile_and_charge_match_reference():
    """Product beam (host setup) against the reference's beam.py values."""
    z = golden("beam.npz")
    from openecloud_b200.grid import Grid
    from openecloud_b200.beam import LHCBeam, LHCBeamEndless
    g = Grid(64, 48, 0.04, 0.03, 1)
    e = LHCBeamEndless(g, 1e-11, nParticles=1.1e11)
    t = LHCBeam(g, 1e-11, nParticles=1.15e11)
    assert np.max(np.abs(e.getTransversalProfile() - z["endless_profile"])) <= 1e-15
    assert np.max(np.abs(t.getTransversalProfile() - z["train_profile"])) <= 1e-15
    for k, tt in enumerate(z["times"]):
        ce = e.getCharge(tt)
        ct = t.getCharge(tt)
        ce = np.zeros(g.getNpExt()) if np.isscalar(ce) else ce
        ct = np.zeros(g.getNpExt()) if np.isscalar(ct) else ct
        assert np.allclose(ce, z["endless_charge"][k], rtol=1e-13, atol=0)
        assert np.allclose(ct, z["train_charge"][k], rtol=1e-13, atol=0)
