"""Seeded synthetic periodic boxes used by the tests and the benchmark.

No public dataset is involved; every box is generated from a seed:

* ``sio2_box``: 216 Si + 432 O uniform in a cubic cell of edge 21.4 A
  (about 2.2 g/cm^3), rejection-sampled to a minimum periodic pair distance
  of 1.5 A.
* ``replicate``: an n1 x n2 x n3 supercell of a box, each position then
  jittered by N(0, sigma) from its own seed (648 -> 139,968 atoms at 6x6x6).
* ``hcno_box``: H:C:N:O = 50:30:10:10 in a triclinic cell (a=b=c, angles
  U(80, 100) degrees) at about 1.3 g/cm^3, minimum distance 0.9 A.
* ``random_box``: a triclinic cell of given atom count, element range and
  density, for ragged batches.
"""
from __future__ import annotations

import math
from typing import Sequence, Tuple

import numpy as np

AMU_G = 1.66053906660e-24
# standard atomic masses for Z = 1..54 (g/mol), used only to set box densities
_MASS = np.array([
    0.0, 1.008, 4.0026, 6.94, 9.0122, 10.81, 12.011, 14.007, 15.999, 18.998, 20.180,
    22.990, 24.305, 26.982, 28.085, 30.974, 32.06, 35.45, 39.948, 39.098, 40.078,
    44.956, 47.867, 50.942, 51.996, 54.938, 55.845, 58.933, 58.693, 63.546, 65.38,
    69.723, 72.630, 74.922, 78.971, 79.904, 83.798, 85.468, 87.62, 88.906, 91.224,
    92.906, 95.95, 97.0, 101.07, 102.91, 106.42, 107.87, 112.41, 114.82, 118.71,
    121.76, 127.60, 126.90, 131.29])


def cell_from_params(a: float, b: float, c: float, alpha: float, beta: float, gamma: float) -> np.ndarray:
    """Lattice vectors as rows, a along x, b in the xy-plane (angles in degrees)."""
    al, be, ga = (math.radians(v) for v in (alpha, beta, gamma))
    va = np.array([a, 0.0, 0.0])
    vb = np.array([b * math.cos(ga), b * math.sin(ga), 0.0])
    cx = c * math.cos(be)
    cy = c * (math.cos(al) - math.cos(be) * math.cos(ga)) / math.sin(ga)
    cz = math.sqrt(max(c * c - cx * cx - cy * cy, 1e-12))
    return np.stack([va, vb, np.array([cx, cy, cz])])


def _rsa(rng: np.random.Generator, cell: np.ndarray, n: int, d_min: float, max_tries: int = 2000) -> np.ndarray:
    """Random sequential addition with a wrapped-fractional minimum-image distance test."""
    frac = np.empty((n, 3))
    placed = 0
    d2 = d_min * d_min
    # bin placed atoms on a coarse fractional grid so each test touches few atoms
    nb = np.maximum(1, np.floor(1.0 / (d_min * np.linalg.norm(np.linalg.inv(cell), axis=0))).astype(int))
    bins: dict = {}
    while placed < n:
        for _ in range(max_tries):
            f = rng.random(3)
            b = tuple((f * nb).astype(int) % nb)
            ok = True
            cand = []
            for dx in (-1, 0, 1):
                for dy in (-1, 0, 1):
                    for dz in (-1, 0, 1):
                        cand.extend(bins.get(((b[0] + dx) % nb[0], (b[1] + dy) % nb[1], (b[2] + dz) % nb[2]), ()))
            if cand:
                df = frac[np.array(cand)] - f
                df -= np.round(df)
                dc = df @ cell
                if np.min(np.einsum("ij,ij->i", dc, dc)) < d2:
                    ok = False
            if ok:
                frac[placed] = f
                bins.setdefault(b, []).append(placed)
                placed += 1
                break
        else:
            raise RuntimeError("random sequential addition jammed; lower the density or d_min")
    return frac


def sio2_box(seed: int = 0, edge: float = 21.4, d_min: float = 1.5) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
    """(positions (648, 3) A, cell (3, 3) A, numbers (648,)) -- 216 Si then 432 O."""
    rng = np.random.default_rng(seed)
    cell = np.eye(3) * edge
    frac = _rsa(rng, cell, 648, d_min)
    numbers = np.array([14] * 216 + [8] * 432, dtype=np.int64)
    return frac @ cell, cell, numbers


def replicate(positions: np.ndarray, cell: np.ndarray, numbers: np.ndarray, reps: Sequence[int],
              jitter: float = 0.0, seed: int = 1):
    n1, n2, n3 = (int(v) for v in reps)
    shifts = np.array([[i, j, k] for i in range(n1) for j in range(n2) for k in range(n3)], dtype=np.float64)
    pos = (positions[None, :, :] + (shifts @ cell)[:, None, :]).reshape(-1, 3)
    nums = np.tile(numbers, len(shifts))
    sup = cell * np.array([n1, n2, n3], dtype=np.float64)[:, None]
    if jitter > 0:
        pos = pos + np.random.default_rng(seed).normal(0.0, jitter, pos.shape)
    return pos, sup, nums


def sio2_scaled(reps: int, seed: int = 0, jitter_seed: int = 1, jitter: float = 0.05):
    """The 648-atom SiO2 box replicated reps^3 times with N(0, jitter) noise (reps=6: 139,968 atoms)."""
    p, c, z = sio2_box(seed)
    return replicate(p, c, z, (reps, reps, reps), jitter=jitter, seed=jitter_seed)


def box_for_density(numbers: np.ndarray, density: float, angles: Tuple[float, float, float]) -> np.ndarray:
    mass = float(np.sum(_MASS[numbers])) * AMU_G
    vol = mass / density * 1e24                           # A^3
    unit = cell_from_params(1.0, 1.0, 1.0, *angles)
    a = (vol / abs(np.linalg.det(unit))) ** (1.0 / 3.0)
    return unit * a


def hcno_box(seed: int = 0, n_atoms: int = 12000, density: float = 1.3, d_min: float = 0.9):
    rng = np.random.default_rng(seed)
    counts = np.array([50, 30, 10, 10]) * n_atoms // 100
    counts[0] += n_atoms - counts.sum()
    numbers = np.repeat(np.array([1, 6, 7, 8]), counts)
    rng.shuffle(numbers)
    angles = tuple(rng.uniform(80.0, 100.0, 3))
    cell = box_for_density(numbers, density, angles)
    frac = _rsa(rng, cell, n_atoms, d_min)
    return frac @ cell, cell, numbers


def random_box(seed: int, n_atoms: int, z_max: int = 54, density: Tuple[float, float] = (1.0, 3.0),
               angles: Tuple[float, float] = (70.0, 110.0), d_min: float = 0.9):
    rng = np.random.default_rng(seed)
    numbers = rng.integers(1, z_max + 1, n_atoms)
    rho = rng.uniform(*density)
    ang = tuple(rng.uniform(*angles, 3))
    cell = box_for_density(numbers, rho, ang)
    frac = _rsa(rng, cell, n_atoms, d_min)
    return frac @ cell, cell, numbers


def batch_boxes(n_struct: int = 256, seed: int = 0, n_min: int = 32, n_max: int = 4096):
    """Ragged batch: atom counts log-uniform in [n_min, n_max], Z in 1..54, density U(1, 3)."""
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(math.log(n_min), math.log(n_max), n_struct)).astype(int)
    return [random_box(seed * 100003 + k, int(n)) for k, n in enumerate(sizes)]
