"""Stand-in for ase (not installed): an Atoms-like record and the Calculator base."""
import numpy as np


class _Cell:
    def __init__(self, array):
        self.array = np.asarray(array, dtype=np.float64)


class Atoms:
    def __init__(self, numbers, positions, cell, pbc=True):
        self.numbers = np.asarray(numbers)
        self.positions = np.asarray(positions, dtype=np.float64)
        self.cell = _Cell(cell)
        self.pbc = np.array([bool(pbc)] * 3) if np.ndim(pbc) == 0 else np.asarray(pbc)
