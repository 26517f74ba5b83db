"""Functional surface ``forward(positions, cell, numbers) -> (energy, forces, stress)``.

One call runs the fused device path of libfd3: cell-list neighbour search, smooth-cutoff
CN and C6 factors, SPME/PME reciprocal sum and the hand-written adjoints; it returns the
quantities ``FourierD3ASECalculator.calculate`` produces (src/fourierd3/calculator.py:
177-192): energy [eV], forces [eV/A] (N, 3) and the full 3x3 stress [eV/A^3]
(= (dE/dstrain) / volume, the reference's sign).
"""
from __future__ import annotations

from typing import Optional

import numpy as np
import torch

from fourierd3_b200 import engine as _engine
from fourierd3_b200 import geometry


class D3Model:
    """Fixed species list, initial cell (for the mesh size) and options -> one engine."""

    def __init__(self, numbers, cell, *, method: str = "spme", mesh_spacing: float = 1.2,
                 interpolation_nodes: int = 5, c6tol: float = 1.0, params=None, r_cut: float = 6.0,
                 k_cutoff: float = 10.0, cncorr=None, precision: str = "fp64", cnfunc: str = "smooth_cut",
                 device: Optional[torch.device] = None):
        self.device = torch.device(device) if device is not None else torch.device("cuda")
        self.numbers = np.asarray(numbers)
        self.r_cut = float(r_cut)
        self.setup = _engine.species_setup(self.numbers, c6tol)
        cell_b = np.asarray(cell, dtype=np.float64) * geometry.ANGSTROM_TO_BOHR
        if method in ("spme", "pme"):
            mesh, ens = geometry.ns_mesh(cell_b, mesh_spacing * geometry.ANGSTROM_TO_BOHR), (0, 0, 0)
        else:
            mesh, ens = (1, 1, 1), geometry.ewald_ns(cell_b, k_cutoff)
        self.mesh = mesh
        self.engine = _engine.Engine(self.setup, method=method, order=interpolation_nodes, mesh=mesh,
                                     ewald_ns=ens, precision=precision,
                                     r_cut_bohr=self.r_cut * geometry.ANGSTROM_TO_BOHR,
                                     params=params if params is not None else _engine.PBE_BJ,
                                     cncorr=cncorr, cnfunc=cnfunc, device=self.device)

    def __call__(self, positions, cell, out=None):
        pos = torch.as_tensor(positions, dtype=torch.float64)
        if pos.device != self.device:
            pos = pos.to(self.device, non_blocking=True)
        pos = pos.contiguous()
        cell_h = np.asarray(cell.detach().cpu() if torch.is_tensor(cell) else cell, dtype=np.float64)
        return self.engine.energy_forces_stress(pos, cell_h, self.r_cut, out=out)

    def direct(self, positions, cell, r_direct: float = 25.0):
        """The direct pairwise lattice sum in float64 (pairs within ``r_direct`` A plus the
        continuum tail) with this model's CN, C6 factors and damping: the accuracy oracle the
        mesh methods converge to. Returns (E [eV], F [eV/A], stress [eV/A^3])."""
        pos = torch.as_tensor(positions, dtype=torch.float64).to(self.device).contiguous()
        cell_h = np.asarray(cell.detach().cpu() if torch.is_tensor(cell) else cell, dtype=np.float64)
        return self.engine.direct_energy_forces_stress(pos, cell_h, self.r_cut, r_direct)


_CACHE: dict = {}


def forward(positions, cell, numbers, **kwargs):
    """E [eV] (0-d), F [eV/A] (N, 3), stress [eV/A^3] (3, 3), all on the device.

    The model (decomposition, plan, cuFFT plans, workspace) is cached per species list,
    initial mesh and options, so repeated calls on the same system only run kernels.
    """
    cell_np = np.asarray(cell.detach().cpu() if torch.is_tensor(cell) else cell, dtype=np.float64)
    nums = np.asarray(numbers.cpu() if torch.is_tensor(numbers) else numbers)
    key = (nums.tobytes(), tuple(sorted(kwargs.items())))
    model = _CACHE.get(key)
    if model is None:
        model = D3Model(nums, cell_np, **kwargs)
        _CACHE[key] = model
    return model(positions, cell_np)


_BATCH_CACHE: dict = {}


def forward_batch(structures, *, graph: bool = True, lanes: int = 1, **kwargs):
    """Batched ``forward``: ``structures`` is a list of (positions, cell, numbers).

    Returns a list of (energy [eV] 0-d, forces [eV/A] (N_i, 3), stress [eV/A^3] (3, 3))
    device tensors, one per structure (views into the batch's output buffers, overwritten
    by the next call on the same batch). The batch (plans, workspaces and, with ``graph``,
    the captured CUDA graph) is cached per list of atomic numbers and cells, so repeated
    calls with new positions are a copy plus one graph replay.
    """
    from fourierd3_b200.batch import D3Batch

    host = []
    for pos, cell, numbers in structures:
        cell_np = np.asarray(cell.detach().cpu() if torch.is_tensor(cell) else cell, dtype=np.float64)
        nums = np.asarray(numbers.cpu() if torch.is_tensor(numbers) else numbers)
        host.append((pos, cell_np, nums))
    key = (tuple((n.tobytes(), c.tobytes()) for _, c, n in host), lanes, graph,
           tuple(sorted(kwargs.items())))
    batch = _BATCH_CACHE.get(key)
    if batch is None:
        first = [(np.asarray(p.detach().cpu() if torch.is_tensor(p) else p, dtype=np.float64), c, n)
                 for p, c, n in host]
        batch = D3Batch(first, lanes=lanes, **kwargs)
        if graph:
            batch.capture()
        _BATCH_CACHE[key] = batch
    e, f, s = batch([p for p, _, _ in host])
    fs = batch.split_forces(f)
    return [(e[i], fs[i], s[i]) for i in range(batch.n_struct)]
