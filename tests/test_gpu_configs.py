"""GPU checks of the workload configurations beyond the reference fixtures.

* precision scaling: the plain float64 SPME and the mixed form against the direct pairwise
  D3 lattice sum (tests/golden/direct_sio2_*.npz) for the seeded SiO2 box and its 2x2x2
  replica -- the SPME discretisation error at the reference mesh, stated as tolerances;
* mixed chemistry: 12,000 H/C/N/O atoms in a triclinic cell, mesh spacing 1.0 A, spline
  order 6 -- mixed precision against plain float64 (energy 1e-6 relative, forces
  1e-4 eV/A, stress 1e-6 eV/A^3).
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
KW = dict(method="spme", mesh_spacing=1.2, interpolation_nodes=5, c6tol=1.0, r_cut=6.0)


@pytest.mark.parametrize("n", [648, 5184])
def test_spme_against_direct_lattice_sum(n, cuda_device):
    from fourierd3_b200 import D3Model

    path = os.path.join(GOLDEN, f"direct_sio2_{n}.npz")
    if not os.path.exists(path):
        pytest.skip("direct-sum fixture not generated")
    d = np.load(path)
    for prec in ("fp64", "mixed"):
        m = D3Model(d["numbers"], d["cell"], precision=prec, device=cuda_device, **KW)
        e, f, s = m(d["positions"], d["cell"])
        e_ref = float(d["energy_ev"])
        assert abs(float(e) - e_ref) <= 5e-6 * abs(e_ref), (prec, float(e), e_ref)
        assert np.abs(f.cpu().numpy() - d["forces"]).max() <= 2e-4
        assert np.abs(s.cpu().numpy() - d["stress"]).max() <= 1e-6


@pytest.mark.parametrize("seed", [0, 1])
def test_many_species_mixed_against_fp64(seed, cuda_device):
    """The mixed form keeps the C6 factors unscaled: float32 carries the same relative precision
    at any magnitude, and the factors (O(1-100) for Z up to 54) are far from float32 under- or
    overflow. Checked at the extreme of the batch workload: every element Z = 1..54 present
    (rank 8 of the C6 decomposition), dense (3 g/cm^3) and dilute (1 g/cm^3) triclinic boxes --
    energy 1e-6 relative, forces 1e-4 eV/A, stress 1e-6 eV/A^3 against plain float64."""
    from fourierd3_b200 import D3Model, structures

    density = (3.0, 3.0) if seed == 0 else (1.0, 1.0)
    pos, cell, nums = structures.random_box(seed=300 + seed, n_atoms=540, z_max=54, density=density,
                                            angles=(70.0, 110.0), d_min=1.0)
    nums = np.asarray(nums).copy()
    nums[:54] = np.arange(1, 55)              # every species present
    m64 = D3Model(nums, cell, precision="fp64", device=cuda_device, **KW)
    assert m64.setup.n_species == 54 and m64.setup.n_rank >= 8
    e64, f64, s64 = m64(pos, cell)
    e32, f32, s32 = D3Model(nums, cell, precision="mixed", device=cuda_device, **KW)(pos, cell)
    assert abs(float(e32) - float(e64)) <= 1e-6 * abs(float(e64)), (float(e32), float(e64))
    assert (f32 - f64).abs().max().item() <= 1e-4
    assert (s32 - s64).abs().max().item() <= 1e-6


def test_hcno_mixed_against_fp64(cuda_device):
    from fourierd3_b200 import D3Model, structures

    pos, cell, nums = structures.hcno_box(seed=0, n_atoms=12000)
    kw = dict(method="spme", mesh_spacing=1.0, interpolation_nodes=6, c6tol=1.0, r_cut=6.0)
    e64, f64, s64 = D3Model(nums, cell, precision="fp64", device=cuda_device, **kw)(pos, cell)
    e32, f32, s32 = D3Model(nums, cell, precision="mixed", device=cuda_device, **kw)(pos, cell)
    assert abs(float(e32) - float(e64)) <= 1e-6 * abs(float(e64))
    assert (f32 - f64).abs().max().item() <= 1e-4
    assert (s32 - s64).abs().max().item() <= 1e-6


@pytest.mark.parametrize("n", [648, 5184])
def test_gpu_direct_sum_matches_oracle(n, cuda_device):
    """The float64 direct pair sum on the device (pairs within 25 A + continuum tail, the plan's
    CN and C6 factors) against the CPU oracle's direct sum (oracle/direct_d3.py, fixtures made by
    tests/golden/make_direct.py): energy 1e-11 relative, forces 1e-9 eV/A, stress 1e-10 eV/A^3."""
    from fourierd3_b200 import D3Model

    d = np.load(os.path.join(os.path.dirname(__file__), "golden", f"direct_sio2_{n}.npz"))
    m = D3Model(d["numbers"], d["cell"], precision="fp64", device=cuda_device, **KW)
    e, f, s = m.direct(d["positions"], d["cell"], r_direct=float(d["r_direct"]))
    ref = float(d["energy_ev"])
    assert abs(float(e) - ref) <= 1e-11 * abs(ref), (float(e), ref)
    np.testing.assert_allclose(f.cpu().numpy(), d["forces"], rtol=0, atol=1e-9)
    np.testing.assert_allclose(s.cpu().numpy(), d["stress"], rtol=0, atol=1e-10)
    # the SPME float64 path converges to it (discretisation at h = 1.2 A, p = 5)
    e2, f2, _ = m(d["positions"], d["cell"])
    assert abs(float(e2) - ref) <= 5e-6 * abs(ref)
