"""Host-side geometry conventions of the reference path (mesh size, SPME window).

* ``ns_mesh``: mesh points per axis, n_a = 2 ** ceil(log2(2 |a_a| / h + 1)) for the
  Bohr cell rows a_a and Bohr spacing h -- the torch-pme ``get_ns_mesh`` rule the
  reference calls at src/fourierd3/core.py:186.
* ``spme_window``: the SPME deconvolution window prod_a sinc(m_a / n_a)^(2p),
  clamped at 1e-10, built EXACTLY as src/fourierd3/pair_pot.py:184-202 builds it:
  the Miller indices come from ``torch.fft.fftfreq`` without a dtype, i.e. in
  torch's default float32, so the window is a float32 table even on the float64
  path. The GPU filter reads this table so that its G / window matches the
  reference bit for bit; the table is computed once per mesh on the host.
* ``ewald_ns``: the Ewald Miller-index box ceil(k_cut |a| / 2 pi) (core.py:228-230).
"""
from __future__ import annotations

import math

import numpy as np
import torch

ANGSTROM_TO_BOHR = 1 / 0.52917726      # src/fourierd3/core.py:120
HARTREE_TO_EV = 27.21138505            # src/fourierd3/calculator.py:54


def ns_mesh(cell_bohr: np.ndarray, spacing_bohr: float) -> tuple:
    norms = np.linalg.norm(np.asarray(cell_bohr, dtype=np.float64), axis=1)
    approx = 2.0 * norms / spacing_bohr + 1.0
    return tuple(int(2 ** math.ceil(math.log2(v))) for v in approx)


def spme_window(ns, order: int) -> np.ndarray:
    """float32 array (nx, ny, nz//2+1), the reference's cached ``_cached_sc``."""
    nx, ny, nz = (int(v) for v in ns)
    mx = torch.fft.fftfreq(nx, d=1.0 / nx, dtype=torch.float32)
    my = torch.fft.fftfreq(ny, d=1.0 / ny, dtype=torch.float32)
    mz = torch.fft.rfftfreq(nz, d=1.0 / nz, dtype=torch.float32)
    sc = (torch.sinc(mx / nx)[:, None, None] * torch.sinc(my / ny)[None, :, None]
          * torch.sinc(mz / nz)[None, None, :])
    sc = torch.pow(sc, 2 * int(order))
    sc = torch.where(sc < 1e-10, 1e-10, sc)
    return np.ascontiguousarray(sc.numpy(), dtype=np.float32)


def ewald_ns(cell_bohr: np.ndarray, k_cutoff: float) -> tuple:
    norms = np.linalg.norm(np.asarray(cell_bohr, dtype=np.float64), axis=1)
    return tuple(int(math.ceil(v)) for v in k_cutoff * norms / (2 * math.pi))
