"""Differentiation configuration: NVE velocity-Verlet on 20,736-atom SiO2 (the 648-atom box
replicated 4x4x2 with N(0, 0.05 A) jitter), dt = 1 fs, 300 K Maxwell-Boltzmann start, Verlet
list skin 0.5 A, float32 mesh (mixed form) forces from the adjoint kernels behind the
torch.autograd.Function. Every 10 steps the forces are checked against the plain float64
adjoints and against central finite differences (h = 1e-4 A) of the float64 energy; at step 0
also against the oracle's torch autograd forces (CPU).
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

KW = dict(method="spme", mesh_spacing=1.2, interpolation_nodes=5, c6tol=1.0)


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_md_graph_replay_matches_eager(dtype, cuda_device):
    """Each velocity-Verlet step captured as one CUDA graph (module forward + hand-written
    adjoints through autograd, both half kicks) replays bitwise equal to the same steps run
    eagerly, across Verlet-list rebuilds (a 0.1 A skin forces several re-captures); against the
    driver that cuts its list to r_cut before every call, positions agree to rounding."""
    from fourierd3_b200 import structures
    from fourierd3_b200.md import VelocityVerlet

    pos, cell, nums = structures.sio2_box(0)
    kw = dict(dt=1.0, temperature=600.0, seed=11, skin=0.1, dtype=dtype, device=cuda_device, **KW)
    eager = VelocityVerlet(nums, pos, cell, verlet_edges=True, **kw)
    graph = VelocityVerlet(nums, pos, cell, verlet_edges=True, graph=True, **kw)
    cut = VelocityVerlet(nums, pos, cell, **kw)
    for _ in range(30):
        a, b, c = eager.step(), graph.step(), cut.step()
    assert graph.rebuilds >= 2
    assert torch.equal(a.positions, b.positions) and torch.equal(a.forces, b.forces)
    assert torch.equal(a.velocities, b.velocities)
    assert (a.positions - c.positions).abs().max().item() < 1e-8
    assert abs(float(b.energy) - float(c.energy)) <= 1e-9 * abs(float(c.energy))


def test_md_nve_with_adjoint_checks(cuda_device):
    from fourierd3_b200 import FourierD3, structures
    from fourierd3_b200.geometry import HARTREE_TO_EV
    from fourierd3_b200.md import VelocityVerlet

    p0, c0, z0 = structures.sio2_box(0)
    pos, cell, nums = structures.replicate(p0, c0, z0, (4, 4, 2), jitter=0.05, seed=1)
    assert len(nums) == 20736
    md = VelocityVerlet(nums, pos, cell, dt=1.0, temperature=300.0, seed=7, skin=0.5, dtype=torch.float32,
                        device=cuda_device, **KW)
    ref = FourierD3(nums, cell, dtype=torch.float64, device=cuda_device, verbose=False, **KW)

    def energy64(x):
        ei, us = md._edges(x)
        ref._update_cell(md.cell_t)
        with torch.no_grad():
            return float(ref(x, ei, us @ md.cell_t)) * HARTREE_TO_EV

    # step 0: the oracle's autograd forces (CPU float64 restatement of the reference)
    from oracle.reference_port import OracleFourierD3

    e_or, f_or, s_or = OracleFourierD3(nums, cell, **KW).calculate(md.state.positions.cpu().numpy(), cell)
    assert np.abs(md.state.forces.cpu().numpy() - f_or).max() < 1e-4
    e_tot0 = md.state.energy + md.kinetic()
    rng = np.random.default_rng(3)
    h = 1e-4
    for step in range(1, 101):
        st = md.step()
        if step % 10:
            continue
        _, f64, _ = md.forces(st.positions, model=ref)
        assert (st.forces - f64).abs().max().item() < 1e-4, step
        for i in rng.choice(len(nums), 2, replace=False):
            for a in range(3):
                xp = st.positions.clone(); xp[i, a] += h
                xm = st.positions.clone(); xm[i, a] -= h
                fd = -(energy64(xp) - energy64(xm)) / (2 * h)
                assert abs(fd - f64[i, a].item()) < 1e-5, (step, i, a, fd, f64[i, a].item())
    drift = abs(md.state.energy + md.kinetic() - e_tot0) / len(nums)
    assert drift < 1e-5, drift
