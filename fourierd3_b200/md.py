"""NVE velocity-Verlet driver on the drop-in module (forces and stress from the adjoint kernels).

Units: eV, Angstrom, amu, fs. The neighbour list is a Verlet list of radius r_cut + skin,
rebuilt on the GPU when any atom has moved more than skin / 2 since the last build; before each
force call the list is cut back to the pairs closer than r_cut, so every step sees exactly the
pair set the reference's per-call matscipy build gives (the reference's smooth-cutoff CN is not
exactly zero beyond r_cut, src/fourierd3/core.py:357-364, so the skin pairs must not be kept).
Forces and stress come from ``FourierD3`` through the strain protocol of
src/fourierd3/calculator.py:146-188, i.e. torch.autograd calling the hand-written adjoints.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Optional

import numpy as np
import torch

from fourierd3_b200.core import FourierD3
from fourierd3_b200.engine import neighbour_list
from fourierd3_b200.geometry import ANGSTROM_TO_BOHR, HARTREE_TO_EV

KB_EV = 8.617333262e-5                 # eV / K
ACC = 9.6485332e-3                     # (eV / (A amu)) -> A / fs^2
MASS = {1: 1.008, 6: 12.011, 7: 14.007, 8: 15.999, 14: 28.085}


def masses_of(numbers) -> np.ndarray:
    from fourierd3_b200.structures import _MASS

    return np.array([MASS.get(int(z), float(_MASS[int(z)])) for z in numbers], dtype=np.float64)


def maxwell_boltzmann(masses: np.ndarray, temperature: float, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    v = rng.standard_normal((len(masses), 3)) * np.sqrt(KB_EV * temperature * ACC / masses)[:, None]
    v -= (masses[:, None] * v).sum(0) / masses.sum()          # zero total momentum
    return v


@dataclass
class MDState:
    step: int
    positions: torch.Tensor       # (N, 3) A, float64, device
    velocities: torch.Tensor      # (N, 3) A/fs
    forces: torch.Tensor          # (N, 3) eV/A
    energy: float                 # eV (potential)
    stress: np.ndarray            # (3, 3) eV/A^3


class VelocityVerlet:
    def __init__(self, numbers, positions, cell, *, dt: float = 1.0, temperature: float = 300.0, seed: int = 0,
                 skin: float = 0.5, r_cut: float = 6.0, dtype=torch.float32, device=None, **model_kw):
        self.device = torch.device(device) if device is not None else torch.device("cuda")
        self.numbers = np.asarray(numbers)
        self.cell = np.asarray(cell, dtype=np.float64)
        self.dt = float(dt)
        self.skin = float(skin)
        self.r_cut = float(r_cut)
        self.model = FourierD3(self.numbers, self.cell, dtype=dtype, device=self.device, verbose=False,
                               r_cut=r_cut, **model_kw)
        self.masses = torch.tensor(masses_of(self.numbers), dtype=torch.float64, device=self.device)
        self.cell_t = torch.tensor(self.cell, dtype=torch.float64, device=self.device)
        pos = torch.tensor(np.asarray(positions, dtype=np.float64), device=self.device)
        vel = torch.tensor(maxwell_boltzmann(masses_of(self.numbers), temperature, seed), device=self.device)
        self._ref_pos = None
        self.rebuilds = 0
        e, f, s = self.forces(pos)
        self.state = MDState(0, pos, vel, f, e, s)

    # -- neighbours --------------------------------------------------------------------------
    def _edges(self, pos: torch.Tensor):
        if self._ref_pos is None or (pos - self._ref_pos).norm(dim=1).max().item() > 0.5 * self.skin:
            i, j, S = neighbour_list(pos, self.cell, self.r_cut + self.skin)
            self._vi, self._vj, self._vS = i, j, S.to(torch.float64)
            self._ref_pos = pos.clone()
            self.rebuilds += 1
        d = pos[self._vj] - pos[self._vi] + self._vS @ self.cell_t
        keep = (d * d).sum(1) < self.r_cut * self.r_cut
        return torch.stack((self._vi[keep], self._vj[keep])), self._vS[keep]

    # -- forces through the module and its autograd.Function --------------------------------
    def forces(self, pos: torch.Tensor, model: Optional[FourierD3] = None):
        model = model or self.model
        edge_index, ushift = self._edges(pos)
        strain = torch.zeros(3, 3, dtype=torch.float64, device=self.device, requires_grad=True)
        scell = self.cell_t + torch.einsum("ab,Ab->Aa", strain, self.cell_t)
        model._update_cell(scell)
        p = pos.detach().clone().requires_grad_(True)
        sp = p + torch.einsum("ab,ib->ia", strain, p)
        energy = model(sp, edge_index, ushift @ scell).to(torch.float64) * HARTREE_TO_EV
        energy.backward()
        stress = (strain.grad / model.volume.detach() * ANGSTROM_TO_BOHR ** 3).cpu().numpy()
        return float(energy.detach()), -p.grad.detach(), stress

    def kinetic(self) -> float:
        v = self.state.velocities
        return float(0.5 * (self.masses[:, None] * v * v).sum() / ACC)

    def step(self) -> MDState:
        st = self.state
        a = st.forces * ACC / self.masses[:, None]
        v_half = st.velocities + 0.5 * self.dt * a
        pos = st.positions + self.dt * v_half
        e, f, s = self.forces(pos)
        v = v_half + 0.5 * self.dt * f * ACC / self.masses[:, None]
        self.state = MDState(st.step + 1, pos, v, f, e, s)
        return self.state
