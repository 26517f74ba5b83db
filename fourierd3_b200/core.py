"""``FourierD3``: drop-in for the reference torch module (src/fourierd3/core.py:14-583).

Same constructor arguments, buffers the callers read (``volume``, ``cell``, ``species``,
``eigs``, ``eigvecs``, ``n_rank``, ``ns_mesh``, ``angstrom_to_bohr``), ``_update_cell``
and ``forward(positions [A], edge_index, shifts [A]) -> energy [Hartree]``. The energy is
differentiable with respect to positions, shifts and the cell given to ``_update_cell``,
so the reference's strain protocol (calculator.py:146-188) works unchanged -- but the
gradients come from the hand-written adjoint kernels of libfd3 behind a
``torch.autograd.Function``, not from autograd through torch ops.

Precision: ``dtype=torch.float64`` runs the plain float64 kernels (the reference's
float64 path to 1e-10); ``dtype=torch.float32`` (the reference default) runs the mixed
form -- float32 spreading / FFT / filter / gather with float64 energy and virial
accumulation, cell setup, self term and CN -- which is more accurate than an all-float32
evaluation. ``precision=`` overrides the mapping.
"""
from __future__ import annotations

from typing import List, Optional

import numpy as np
import torch

from fourierd3_b200 import engine as _engine
from fourierd3_b200 import geometry


def _det3(m: torch.Tensor) -> torch.Tensor:
    """Cofactor determinant (src/fourierd3/utils.py:130-139)."""
    c00 = m[1, 1] * m[2, 2] - m[1, 2] * m[2, 1]
    c10 = m[1, 2] * m[2, 0] - m[1, 0] * m[2, 2]
    c20 = m[1, 0] * m[2, 1] - m[1, 1] * m[2, 0]
    return m[0, 0] * c00 + m[0, 1] * c10 + m[0, 2] * c20


class _EdgeEnergy(torch.autograd.Function):
    """E(pos_b, shifts_b, cell_b) with gradients from the libfd3 adjoint kernels."""

    @staticmethod
    def forward(ctx, pos_b, shifts_b, cell_b, edge_index, eng):
        need = any(ctx.needs_input_grad[:3])
        e, gpos, gsh, gcell = eng.energy_edges(pos_b, cell_b, edge_index, shifts_b, need)
        if need:
            ctx.save_for_backward(gpos, gsh, gcell)
        return e

    @staticmethod
    def backward(ctx, grad_e):
        gpos, gsh, gcell = ctx.saved_tensors
        return (grad_e * gpos if ctx.needs_input_grad[0] else None,
                grad_e * gsh if ctx.needs_input_grad[1] else None,
                grad_e * gcell if ctx.needs_input_grad[2] else None, None, None)


class FourierD3(torch.nn.Module):
    def __init__(self, species: List, cell, pbc: Optional[torch.Tensor] = None, mesh_spacing: float = 1.2,
                 c6tol: float = 1, xcfunc: str = "pbe",
                 device=torch.device("cuda" if torch.cuda.is_available() else "cpu"),
                 dtype=torch.float32, method: str = "spme", params=None, cnfunc="smooth_cut",
                 interpolation_nodes: int = 5, k_cutoff: float = 10.0, r_cut: float = 6.0,
                 cncorr: Optional[torch.Tensor] = None, verbose=True, precision: Optional[str] = None) -> None:
        super().__init__()
        device = torch.device(device)
        if pbc is not None:
            assert bool(torch.as_tensor(pbc).all()), "particle-mesh only supports 3d pbc"   # core.py:96-97
        if verbose:
            print("Assuming 3D PBC are satisfied")
        if cnfunc not in ("smooth_cut", "d4"):
            raise ValueError(f"Unknown cnfunc '{cnfunc}'. Expected 'smooth_cut' or 'd4'.")
        if params is None:
            if xcfunc != "pbe":
                raise NotImplementedError                                                # core.py:169-170
            params = _engine.PBE_BJ
        params = [float(v) for v in (params.tolist() if torch.is_tensor(params) else params)]
        self.device = device
        self.dtype = dtype
        self.method = method
        self.mesh_spacing = mesh_spacing
        self.interpolation_nodes = interpolation_nodes
        self.k_cutoff = k_cutoff
        self.xcfunc = xcfunc
        self.cnfunc = cnfunc
        self.precision = precision or ("fp64" if dtype == torch.float64 else "mixed")
        a2b = geometry.ANGSTROM_TO_BOHR
        self.r_cut = r_cut * a2b
        self._r_cut_ang = float(r_cut)
        setup = _engine.species_setup(np.asarray(species), c6tol)
        self.n_species = setup.n_species
        self.n_rank = setup.n_rank
        self.register_buffer("species", torch.as_tensor(setup.species.astype(np.int64), device=device))
        self.register_buffer("angstrom_to_bohr", torch.tensor(a2b, dtype=torch.float64, device=device))
        cell_t = torch.as_tensor(np.asarray(cell, dtype=np.float64), dtype=torch.float64, device=device)
        self.register_buffer("cell", cell_t * self.angstrom_to_bohr)
        self.register_buffer("volume", torch.abs(_det3(self.cell)))
        self.register_buffer("eigs", torch.as_tensor(setup.eigs, device=device))
        self.register_buffer("eigvecs", torch.as_tensor(setup.eigvecs, device=device))
        self.register_buffer("v_q_reshaped", self.eigvecs.view(self.n_species, 7, self.n_rank))
        self.register_buffer("rcov", torch.as_tensor(setup.rcov, device=device))
        self.register_buffer("cnref", torch.as_tensor(setup.cnref, device=device))
        self.cncorr = None if cncorr is None else torch.as_tensor(cncorr, dtype=torch.float64)
        cell_b = cell_t.detach().cpu().numpy() * a2b
        if method in ("spme", "pme"):
            self.ns_mesh = torch.tensor(geometry.ns_mesh(cell_b, mesh_spacing * a2b))      # core.py:186
            if verbose:
                print("Using mesh size", self.ns_mesh)
            mesh, ens = tuple(int(v) for v in self.ns_mesh), (0, 0, 0)
        elif method == "ewald":
            self.ns = torch.tensor(geometry.ewald_ns(cell_b, k_cutoff))                    # core.py:228-230
            mesh, ens = (1, 1, 1), tuple(int(v) for v in self.ns)
        else:
            raise ValueError(f"unknown method {method!r}")
        self._eng = _engine.Engine(setup, method=method, order=interpolation_nodes, mesh=mesh, ewald_ns=ens,
                                   precision=self.precision, r_cut_bohr=self.r_cut, params=params,
                                   cncorr=None if cncorr is None else np.asarray(torch.as_tensor(cncorr).cpu()),
                                   cnfunc=cnfunc, device=device)

    def _update_cell(self, cell):
        """Set the (possibly strained, grad-carrying) cell in Angstrom (core.py:244-267)."""
        self.cell = torch.as_tensor(cell).to(device=self.device, dtype=torch.float64) * self.angstrom_to_bohr
        self.volume = torch.abs(_det3(self.cell))

    def forward(self, positions: torch.Tensor, edge_index: torch.Tensor = None,
                shifts: torch.Tensor = None) -> torch.Tensor:
        if positions.dim() != 2 or positions.shape[1] != 3 or positions.shape[0] != self.species.shape[0]:
            raise ValueError("positions must be (n_atoms, 3) for the species given at construction")
        if self.cnfunc == "d4":
            # k-space CN: no neighbour list; edges, if given, are not used (core.py:512-516)
            edge_index = torch.zeros((2, 0), dtype=torch.long, device=self.device)
            shifts = torch.zeros((0, 3), dtype=torch.float64, device=self.device)
        elif edge_index is None or shifts is None:
            raise ValueError("cnfunc='smooth_cut' needs edge_index and shifts")
        if edge_index.dim() != 2 or edge_index.shape[0] != 2 or shifts.shape != (edge_index.shape[1], 3):
            raise ValueError("edge_index must be (2, E) and shifts (E, 3)")
        # An edge index outside 0..n_atoms-1 is caught on the device (never dereferenced; the
        # energy and its gradients come back NaN), so the call makes no host synchronisation.
        pos_b = positions.to(torch.float64) * self.angstrom_to_bohr                         # core.py:505
        sh_b = shifts.to(torch.float64) * self.angstrom_to_bohr                             # core.py:507
        e = _EdgeEnergy.apply(pos_b, sh_b, self.cell, edge_index.to(self.device), self._eng)
        return e.to(self.dtype)
