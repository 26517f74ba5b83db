"""``FourierD3ASECalculator``: drop-in for src/fourierd3/calculator.py:10-192.

Same constructor arguments, ``implemented_properties``, ``_build_model``,
``_build_graph``, ``_update_cell`` and ``calculate`` contract (``results["energy"]`` eV
float, ``results["forces"]`` (N, 3) eV/A, ``results["stress"]`` full 3x3 eV/A^3).
``calculate`` runs the fused device path (GPU cell-list neighbour search instead of the
CPU matscipy build, hand-written adjoints instead of autograd). When ASE is installed the
class derives from ``ase.calculators.calculator.Calculator``; otherwise it provides the
same minimal ``results`` / ``calculate`` behaviour so non-ASE callers can use it with
any object exposing ``numbers``, ``positions``, ``cell`` and ``pbc``.
"""
from __future__ import annotations

import numpy as np
import torch

from fourierd3_b200 import engine as _engine
from fourierd3_b200.functional import D3Model
from fourierd3_b200.geometry import ANGSTROM_TO_BOHR, HARTREE_TO_EV

try:  # optional dependency, as in the reference
    from ase.calculators.calculator import Calculator, all_changes
except Exception:  # pragma: no cover - exercised when ase is absent
    all_changes = ["positions", "numbers", "cell", "pbc"]

    class Calculator:  # minimal stand-in with the ASE contract used here
        def __init__(self, **kwargs):
            self.results = {}
            self.atoms = None

        def calculate(self, atoms=None, properties=None, system_changes=all_changes):
            if atoms is not None:
                self.atoms = atoms
            self.results = {}

        def get_property(self, name, atoms=None):
            self.calculate(atoms)
            return self.results[name]


def _cell_array(atoms) -> np.ndarray:
    c = atoms.cell
    return np.asarray(getattr(c, "array", c), dtype=np.float64)


class FourierD3ASECalculator(Calculator):
    implemented_properties = ["energy", "forces", "stress"]

    def __init__(self, r_cut=6.0, method="spme",
                 device=torch.device("cuda" if torch.cuda.is_available() else "cpu"), verbose=False,
                 params=None, c6tol: float = 1, xcfunc: str = "pbe", cnfunc="smooth_cut",
                 k_cutoff: float = 10.0, mesh_spacing: float = 1.2, interpolation_nodes: int = 5,
                 dtype=torch.float32, precision=None, **kwargs):
        super().__init__(**kwargs)
        self.device = torch.device(device) if device is not None else torch.device("cuda")
        self.r_cut = float(r_cut)
        self.method = method
        self.verbose = verbose
        self.params = params
        self.angstrom_to_bohr = ANGSTROM_TO_BOHR
        self.HARTREE_TO_EV = HARTREE_TO_EV
        self.k_cutoff = k_cutoff
        self.xcfunc = xcfunc
        self.cnfunc = cnfunc
        self.c6tol = c6tol
        self.mesh_spacing = mesh_spacing
        self.interpolation_nodes = interpolation_nodes
        self.dtype = dtype
        self.precision = precision or ("fp64" if dtype == torch.float64 else "mixed")
        self._model = None
        self._cell = None

    def _build_model(self, atoms):
        if self.cnfunc not in ("smooth_cut", "d4"):
            raise ValueError(f"Unknown cnfunc '{self.cnfunc}'. Expected 'smooth_cut' or 'd4'.")   # calculator.py:174
        if self.params is None and self.xcfunc != "pbe":
            raise NotImplementedError
        self._model = D3Model(atoms.numbers, _cell_array(atoms), method=self.method,
                              mesh_spacing=self.mesh_spacing, interpolation_nodes=self.interpolation_nodes,
                              c6tol=self.c6tol, params=self.params, r_cut=self.r_cut, k_cutoff=self.k_cutoff,
                              precision=self.precision, cnfunc=self.cnfunc, device=self.device)
        if self.verbose:
            print(f"Using {self._model.setup.n_rank}-rank decomposition; mesh {self._model.mesh}")

    def _update_cell(self, cell):
        self._cell = np.asarray(cell.detach().cpu() if torch.is_tensor(cell) else cell, dtype=np.float64)

    def _build_graph(self, atoms, rcut=None):
        """(edge_index (2, E) int64, unit_shifts (E, 3)) on the device, from the GPU cell list."""
        pos = torch.as_tensor(np.asarray(atoms.positions), dtype=torch.float64, device=self.device)
        i, j, s = _engine.neighbour_list(pos, _cell_array(atoms), self.r_cut if rcut is None else rcut)
        return torch.stack((i, j)), s.to(self.dtype)

    def calculate(self, atoms=None, properties=None, system_changes=all_changes):
        super().calculate(atoms, properties, system_changes)
        atoms = atoms if atoms is not None else self.atoms
        if self._model is None:
            self._build_model(atoms)
        cell = self._cell if self._cell is not None else _cell_array(atoms)
        pos = torch.as_tensor(np.asarray(atoms.positions, dtype=np.float64))
        if self.device.type == "cuda":
            pos = pos.pin_memory().to(self.device, non_blocking=True)
        e, f, s = self._model(pos, cell)
        self.results["energy"] = float(e.item())
        self.results["forces"] = f.cpu().numpy()
        self.results["stress"] = s.cpu().numpy()
        self._cell = None
