"""The direct lattice-sum oracle against the restated SPME (CPU): the reciprocal-space method
converges to the direct sum, which pins the restated torch-pme conventions physically."""
import os

import numpy as np

from oracle.reference_port import OracleFourierD3

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_spme_oracle_matches_direct_sum_648():
    d = np.load(os.path.join(GOLDEN, "direct_sio2_648.npz"))
    o = OracleFourierD3(d["numbers"], d["cell"], method="spme", mesh_spacing=1.2, interpolation_nodes=5,
                        c6tol=1.0, r_cut=6.0)
    e, f, s = o.calculate(d["positions"], d["cell"])
    e_ref = float(d["energy_ev"])
    assert abs(e - e_ref) <= 5e-6 * abs(e_ref)
    assert np.abs(f - d["forces"]).max() <= 2e-4
    assert np.abs(s - d["stress"]).max() <= 1e-6


def test_direct_sum_fixture_is_current():
    """Recompute the 648-atom direct sum and compare with the stored fixture."""
    from oracle.direct_d3 import direct_calculate

    d = np.load(os.path.join(GOLDEN, "direct_sio2_648.npz"))
    e, f, s = direct_calculate(d["numbers"], d["positions"], d["cell"], r_direct=float(d["r_direct"]),
                               c6tol=1.0, r_cut=6.0)
    assert abs(e - float(d["energy_ev"])) <= 1e-10 * abs(e)
    np.testing.assert_allclose(f, d["forces"], rtol=0, atol=1e-10)
