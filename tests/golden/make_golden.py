"""Generate the golden fixtures by running the REFERENCE's own code.

The reference package (src/fourierd3/) imports torch-pme, ase and matscipy,
none of which is installed; ``_shims/`` supplies minimal stand-ins whose
arithmetic is the oracle's restatement of those libraries. Its own C6^ref data
file is absent, so ``fourierd3.utils.load_c6ref`` is redirected to this
package's table (the seeded synthetic one unless FD3_C6REF is set). Everything
else -- CN, weights, C6 factors, self term, spreading, rfft, Green's function,
sinc deconvolution, Hermitian weights, Ewald sum, strain/autograd forces and
stress -- is the reference's code, executed unmodified.

Usage (needs the reference checkout; writes tests/golden/*.npz)::

    python tests/golden/make_golden.py <reference checkout>
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))


def _import_reference(ref_root: str):
    sys.path.insert(0, REPO)
    sys.path.insert(0, os.path.join(HERE, "_shims"))
    sys.path.insert(0, os.path.join(ref_root, "src"))
    import torch  # noqa: F401
    import fourierd3
    import fourierd3.utils as futils
    from fourierd3_b200 import tables

    futils.load_c6ref = lambda types: tables.c6ref_matrix(list(types))
    _repair_d4(fourierd3)
    return fourierd3


def _repair_d4(fourierd3):
    """The reference's D4 CN (cnfunc='d4') does not run as written: the mesh branch of
    compute_cn_d4 spreads with interpolation weights that forward only computes afterwards
    (src/fourierd3/core.py:514-516 vs :555), and the Ewald branch multiplies by
    self.one_hot_species, which is never defined (core.py:436). This wrapper supplies both --
    the weights at the positions passed in, and the (N, S) one-hot species matrix -- and then
    runs the reference's own compute_cn_d4 unchanged."""
    import torch

    core = fourierd3.core
    orig = core.FourierD3.compute_cn_d4

    def compute_cn_d4(self, positions, ex=None, nk=None):
        if self.method in ("pme", "spme"):
            self.mesh_interpolator.compute_weights(positions)
        else:
            self.one_hot_species = torch.nn.functional.one_hot(self.species, self.n_species).to(positions.dtype)
        return orig(self, positions, ex, nk)

    core.FourierD3.compute_cn_d4 = compute_cn_d4


def cases():
    from fourierd3_b200 import structures as st

    out = []
    p, c, z = st.sio2_box(0)
    base = dict(method="spme", mesh_spacing=1.2, interpolation_nodes=5, c6tol=1.0, k_cutoff=10.0, r_cut=6.0)
    out.append(("sio2_648_spme_p5", p, c, z, dict(base)))
    out.append(("sio2_648_pme_p5", p, c, z, dict(base, method="pme")))
    out.append(("sio2_648_ewald_k2", p, c, z, dict(base, method="ewald", k_cutoff=2.0)))
    ph, ch, zh = st.hcno_box(seed=3, n_atoms=240)
    out.append(("hcno_240_spme_p6", ph, ch, zh, dict(base, mesh_spacing=1.0, interpolation_nodes=6, c6tol=1e-2)))
    out.append(("hcno_240_spme_p4_tol1e-4", ph, ch, zh, dict(base, interpolation_nodes=4, c6tol=1e-4)))
    pr, cr, zr = st.random_box(seed=11, n_atoms=96, z_max=54, d_min=1.2)
    out.append(("rand_96_pme_p6", pr, cr, zr, dict(base, method="pme", interpolation_nodes=6, mesh_spacing=1.5)))
    out.append(("rand_96_ewald_k3_tol1e-2", pr, cr, zr, dict(base, method="ewald", k_cutoff=3.0, c6tol=1e-2)))
    # a cell narrower than the CN cutoff: periodic self-images are neighbours
    pt, ct, zt = st.random_box(seed=5, n_atoms=6, z_max=20, density=(1.5, 1.5), d_min=1.0)
    out.append(("tiny_6_spme_p4", pt, ct, zt, dict(base, interpolation_nodes=4, mesh_spacing=0.8)))
    # cncorr: the optional affine CN correction (core.py:383-384)
    out.append(("sio2_648_spme_p5_cncorr", p, c, z, dict(base, cncorr=[[0.05, 0.9], [-0.02, 1.1]])))
    # D4 coordination numbers in k-space (no neighbour list)
    out.append(("sio2_648_spme_p5_d4", p, c, z, dict(base, cnfunc="d4")))
    out.append(("hcno_240_pme_p6_d4", ph, ch, zh, dict(base, method="pme", mesh_spacing=1.0, interpolation_nodes=6,
                                                       c6tol=1e-2, cnfunc="d4")))
    out.append(("rand_96_ewald_k3_d4", pr, cr, zr, dict(base, method="ewald", k_cutoff=3.0, cnfunc="d4")))
    return out


def main(ref_root: str) -> None:
    fourierd3 = _import_reference(ref_root)
    import torch
    from ase import Atoms

    from fourierd3_b200 import tables

    for name, pos, cell, numbers, cfg in cases():
        cfg = dict(cfg)
        cncorr = cfg.pop("cncorr", None)
        calc = fourierd3.FourierD3ASECalculator(dtype=torch.float64, device=torch.device("cpu"), **cfg)
        atoms = Atoms(numbers, pos, cell)
        calc._build_model(atoms)
        if cncorr is not None:
            calc._model.cncorr = torch.tensor(cncorr, dtype=torch.float64)
        calc.calculate(atoms)
        model = calc._model
        edge_index, ushift = calc._build_graph(atoms)
        with torch.no_grad():
            a2b = float(model.angstrom_to_bohr)
            cell_t = torch.tensor(cell, dtype=torch.float64)
            model._update_cell(cell_t)
            pos_b = torch.tensor(pos) * a2b
            sh_b = torch.matmul(ushift, cell_t) * a2b
            if cfg.get("cnfunc") == "d4" and model.method == "ewald":
                arg = torch.matmul(model.kvectors, pos_b.T)             # core.py:519-523
                cn = model.compute_cn_d4(pos_b, torch.stack([torch.cos(arg), torch.sin(arg)], dim=0),
                                         arg.shape[0])
            elif cfg.get("cnfunc") == "d4":
                cn = model.compute_cn_d4(pos_b)
            else:
                cn = model.compute_cn_smooth(pos_b, edge_index, sh_b)
            w = model.compute_c6_weights(cn)
            c6 = torch.einsum("nk,nkr->nr", w, model.v_q_reshaped[model.species])
        rec = dict(
            positions=np.asarray(pos), cell=np.asarray(cell), numbers=np.asarray(numbers),
            energy_ev=np.float64(calc.results["energy"]), forces=calc.results["forces"],
            stress=calc.results["stress"], cn=cn.numpy(), c6=c6.numpy(), eigs=model.eigs.numpy(),
            n_edges=np.int64(edge_index.shape[1]),
            config=json.dumps(dict(cfg, cncorr=cncorr, c6_source=tables.c6_source(),
                                   mesh=[int(v) for v in getattr(model, "ns_mesh", [0, 0, 0])])),
        )
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **rec)
        print(f"{name}: N={len(numbers)} E={rec['energy_ev']:.12f} eV rank={model.n_rank} "
              f"edges={int(rec['n_edges'])}")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <reference checkout>")
    main(sys.argv[1])
