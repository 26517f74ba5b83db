"""Hand-written adjoints against central finite differences (h = 1e-4 A) on the GPU."""
import numpy as np
import pytest

import golden_cases as gc

pytestmark = pytest.mark.gpu


def _energy(m, pos, cell):
    e, _, _ = m(pos, cell)
    return float(e)


@pytest.mark.parametrize("name", ["sio2_648_spme_p5", "hcno_240_spme_p6", "rand_96_pme_p6", "rand_96_ewald_k3_tol1e-2",
                                  "sio2_648_spme_p5_d4", "hcno_240_pme_p6_d4"])
def test_forces_and_stress_vs_central_differences(name, cuda_device):
    from fourierd3_b200 import D3Model

    rec = gc.load(name)
    m = D3Model(rec["numbers"], rec["cell"], precision="fp64", device=cuda_device, **gc.model_kwargs(rec["config"]))
    pos0, cell0 = rec["positions"].copy(), rec["cell"].copy()
    _, f, s = m(pos0, cell0)
    f = f.cpu().numpy()
    s = s.cpu().numpy()
    h = 1e-4
    rng = np.random.default_rng(0)
    for i in rng.choice(len(pos0), 4, replace=False):
        for a in range(3):
            p = pos0.copy(); p[i, a] += h
            q = pos0.copy(); q[i, a] -= h
            fd = -(_energy(m, p, cell0) - _energy(m, q, cell0)) / (2 * h)
            assert abs(fd - f[i, a]) < 1e-6, (i, a, fd, f[i, a])
    vol = abs(np.linalg.det(cell0))
    for a, b in [(0, 0), (1, 1), (0, 1), (2, 0)]:
        eps = np.zeros((3, 3)); eps[a, b] = h
        def strained(e):
            d = np.eye(3) + e
            return pos0 @ d.T, cell0 @ d.T
        pp, cp = strained(eps)
        pm, cm = strained(-eps)
        fd = (_energy(m, pp, cp) - _energy(m, pm, cm)) / (2 * h) / vol
        assert abs(fd - s[a, b]) < 1e-7, (a, b, fd, s[a, b])
