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
    """``verlet_edges``: pass the Verlet list (r_cut + skin) unchanged between rebuilds and let
    the kernels drop the pairs beyond r_cut (fd3_plan_set_edge_cutoff) instead of cutting the
    list before every call; the edge count then stays fixed between rebuilds. ``graph``
    (needs ``verlet_edges``): each step -- half kick, drift, forces and stress through the
    module's autograd.Function, half kick -- is one CUDA-graph replay, re-captured after each
    list rebuild; the only host synchronisation per step is the rebuild test. In graph mode the
    state's energy and stress stay device tensors."""

    def __init__(self, numbers, positions, cell, *, dt: float = 1.0, temperature: float = 300.0, seed: int = 0,
                 skin: float = 0.5, r_cut: float = 6.0, dtype=torch.float32, device=None,
                 verlet_edges: bool = False, graph: bool = False, **model_kw):
        if graph and not verlet_edges:
            raise ValueError("graph=True needs verlet_edges=True (a fixed edge count between rebuilds)")
        self.device = torch.device(device) if device is not None else torch.device("cuda")
        self.numbers = np.asarray(numbers)
        self.cell = np.asarray(cell, dtype=np.float64)
        self.dt = float(dt)
        self.skin = float(skin)
        self.r_cut = float(r_cut)
        self.verlet_edges = bool(verlet_edges)
        self.use_graph = bool(graph)
        self._graph = None
        self.model = FourierD3(self.numbers, self.cell, dtype=dtype, device=self.device, verbose=False,
                               r_cut=r_cut, **model_kw)
        if self.verlet_edges:
            self.model._eng.set_edge_cutoff(True)
        self.masses = torch.tensor(masses_of(self.numbers), dtype=torch.float64, device=self.device)
        self.cell_t = torch.tensor(self.cell, dtype=torch.float64, device=self.device)
        pos = torch.tensor(np.asarray(positions, dtype=np.float64), device=self.device)
        vel = torch.tensor(maxwell_boltzmann(masses_of(self.numbers), temperature, seed), device=self.device)
        self._ref_pos = None
        self.rebuilds = 0
        e, f, s = self.forces(pos)
        self.state = MDState(0, pos, vel, f, e, s)

    # -- neighbours --------------------------------------------------------------------------
    def _needs_rebuild(self, pos: torch.Tensor) -> bool:
        return self._ref_pos is None or (pos - self._ref_pos).norm(dim=1).max().item() > 0.5 * self.skin

    def _rebuild(self, pos: torch.Tensor) -> None:
        i, j, S = neighbour_list(pos, self.cell, self.r_cut + self.skin)
        self._vi, self._vj, self._vS = i, j, S.to(torch.float64)
        self._ref_pos = pos.clone()
        self.rebuilds += 1

    def _edges(self, pos: torch.Tensor):
        if self._needs_rebuild(pos):
            self._rebuild(pos)
        if self.verlet_edges:
            return torch.stack((self._vi, self._vj)), self._vS
        d = pos[self._vj] - pos[self._vi] + self._vS @ self.cell_t
        keep = (d * d).sum(1) < self.r_cut * self.r_cut
        return torch.stack((self._vi[keep], self._vj[keep])), self._vS[keep]

    # -- forces through the module and its autograd.Function --------------------------------
    def forces(self, pos: torch.Tensor, model: Optional[FourierD3] = None):
        model = model or self.model
        edge_index, ushift = self._edges(pos)
        e, f, s = self._forces_device(pos, edge_index, ushift, model)
        return float(e), f, s.cpu().numpy()

    def _forces_device(self, pos, edge_index, ushift, model):
        """Energy [eV] (0-d), forces [eV/A] and stress [eV/A^3] on the device, by the strain protocol
        of src/fourierd3/calculator.py:146-188 (no host synchronisation)."""
        strain = torch.zeros(3, 3, dtype=torch.float64, device=self.device, requires_grad=True)
        scell = self.cell_t + torch.einsum("ab,Ab->Aa", strain, self.cell_t)
        model._update_cell(scell)
        p = pos.detach().clone().requires_grad_(True)
        sp = p + torch.einsum("ab,ib->ia", strain, p)
        energy = model(sp, edge_index, ushift @ scell).to(torch.float64) * HARTREE_TO_EV
        energy.backward()
        stress = strain.grad / model.volume.detach() * ANGSTROM_TO_BOHR ** 3
        return energy.detach(), -p.grad.detach(), stress.detach()

    def kinetic(self) -> float:
        v = self.state.velocities
        return float(0.5 * (self.masses[:, None] * v * v).sum() / ACC)

    def _drift(self, pos, vel, f):
        """Half kick and drift: (v(t + dt/2), x(t + dt))."""
        v_half = vel + 0.5 * self.dt * f * ACC / self.masses[:, None]
        return v_half, pos + self.dt * v_half

    def step(self) -> MDState:
        if self.use_graph:
            return self._graph_step()
        st = self.state
        v_half, pos = self._drift(st.positions, st.velocities, st.forces)
        if self.verlet_edges:
            if self._needs_rebuild(pos):
                self._rebuild(pos)
            e, f, s = self._forces_device(pos, torch.stack((self._vi, self._vj)), self._vS, self.model)
            e, s = float(e), s.cpu().numpy()
        else:
            e, f, s = self.forces(pos)
        v = v_half + 0.5 * self.dt * f * ACC / self.masses[:, None]
        self.state = MDState(st.step + 1, pos, v, f, e, s)
        return self.state

    # -- CUDA-graph steps ---------------------------------------------------------------------
    def _step_body(self) -> None:
        """One velocity-Verlet step on the static buffers (recorded into the graph)."""
        g = self._static
        v_half, pos = self._drift(g["pos"], g["vel"], g["f"])
        e, f, s = self._forces_device(pos, g["ei"], g["us"], self.model)
        g["vel"].copy_(v_half + 0.5 * self.dt * f * ACC / self.masses[:, None])
        g["pos"].copy_(pos)
        g["f"].copy_(f)
        g["e"].copy_(e)
        g["s"].copy_(s)

    def _capture(self) -> None:
        st = self.state
        self._static = {"pos": st.positions.clone(), "vel": st.velocities.clone(), "f": st.forces.clone(),
                        "e": torch.zeros((), dtype=torch.float64, device=self.device),
                        "s": torch.zeros((3, 3), dtype=torch.float64, device=self.device),
                        "ei": torch.stack((self._vi, self._vj)).contiguous(), "us": self._vS.contiguous()}
        # one eager step on a side stream warms the allocator and sizes the workspace for this
        # edge count; the state is restored before the capture
        keep = {k: self._static[k].clone() for k in ("pos", "vel", "f")}
        side = torch.cuda.Stream(self.device)
        side.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(side):
            self._step_body()
        torch.cuda.current_stream(self.device).wait_stream(side)
        for k, v in keep.items():
            self._static[k].copy_(v)
        self._graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self._graph):
            self._step_body()

    def _graph_step(self) -> MDState:
        st = self.state
        # the positions the step will evaluate forces at (the same ops the graph runs, so the
        # same values): the list is rebuilt there, exactly as the eager step does
        _, pos = self._drift(st.positions, st.velocities, st.forces)
        rebuild = self._needs_rebuild(pos)
        if rebuild:
            self._rebuild(pos)
        if rebuild or self._graph is None:
            self._capture()
        self._graph.replay()
        g = self._static
        self.state = MDState(st.step + 1, g["pos"].clone(), g["vel"].clone(), g["f"].clone(), g["e"].clone(),
                             g["s"].clone())
        return self.state
