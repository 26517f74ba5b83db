"""Per-element tables and the low-rank C6^ref decomposition (host-side setup).

Everything here runs once per model construction on the host, in float64, and
is not part of the timed path.

* ``load_tables`` returns the reference's element tables (``cnref`` (104, 7),
  ``rcov``, ``sqrtQz``, ``en``, ``rcov_cn`` (119,)), stored with their original
  float32/float64 precision (``src/fourierd3/utils.py:76-127``).
* ``c6ref_block(types)`` returns the (S, S, 7, 7) block of the C6^ref tensor for
  the species present (``src/fourierd3/utils.py:9-22``). The reference file
  ``data/reference-c6.pt`` is not distributed with the reference checkout this
  package was built against, so unless ``FD3_C6REF`` names a copy of it, a
  seeded SYNTHETIC table is used (``synthetic_c6ref_block``); every result
  produced with it is labelled ``c6_source == "synthetic"``.
* ``decomp`` is the rank search of ``src/fourierd3/utils.py:35-73``: Lanczos
  (``scipy.sparse.linalg.eigsh``) with a seeded start vector, raising the rank
  until the maximum relative error of V diag(lambda) V^T is below c6tol percent.
"""
from __future__ import annotations

import functools
import os
from typing import Sequence, Tuple

import numpy as np

_DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "d3_tables.npz")

N_REF = 7          # reference coordination environments per element
N_ELEM_C6 = 104    # element range of the C6^ref tensor


@functools.lru_cache(maxsize=1)
def load_tables() -> dict:
    with np.load(_DATA) as z:
        return {k: z[k].copy() for k in z.files}


def c6_source() -> str:
    """``"file:<path>"`` when FD3_C6REF points at reference-c6.pt, else ``"synthetic"``."""
    p = os.environ.get("FD3_C6REF", "")
    return f"file:{p}" if p and os.path.exists(p) else "synthetic"


@functools.lru_cache(maxsize=1)
def _synthetic_element_params():
    rng = np.random.default_rng(20240917)
    alpha0 = np.exp(rng.uniform(np.log(1.5), np.log(60.0), N_ELEM_C6))   # static polarisability
    omega0 = np.exp(rng.uniform(np.log(0.15), np.log(1.2), N_ELEM_C6))    # oscillator frequency, Ha
    a_slope = rng.uniform(0.03, 0.12, N_ELEM_C6)                          # CN dependence of alpha
    w_slope = rng.uniform(0.10, 0.45, N_ELEM_C6)                          # CN dependence of omega
    phase = rng.uniform(0.0, 2.0 * np.pi, (N_ELEM_C6, N_REF))             # symmetric ripple
    return alpha0, omega0, a_slope, w_slope, phase


def synthetic_c6ref_block(types: Sequence[int]) -> np.ndarray:
    """Seeded stand-in for ``reference-c6.pt[types][:, types]``, shape (S, S, 7, 7), float32.

    One Drude oscillator per (element, reference CN) slot, alpha(i w) = a / (1 + w^2/w0^2),
    combined by the Casimir-Polder integral: C6 = 1.5 a a' w0 w0' / (w0 + w0'), times a
    +-2 % symmetric ripple so that the matrix is not exactly positive semi-definite (the
    Lanczos search then also meets small negative eigenvalues, as with measured tables).
    Positive, symmetric under (Z_a, p) <-> (Z_b, q), zero wherever a slot is unused
    (cnref == -1). It is NOT the Grimme D3 table; results made with it say so.
    """
    t = load_tables()
    cnref = t["cnref"].astype(np.float64)
    alpha0, omega0, a_slope, w_slope, phase = _synthetic_element_params()
    types = np.asarray(types, dtype=np.int64)
    cr = cnref[types]                                    # (S, 7)
    valid = cr != -1
    crv = np.where(valid, cr, 0.0)
    a = alpha0[types][:, None] * (1.0 - a_slope[types][:, None] * crv)
    w = omega0[types][:, None] * (1.0 + w_slope[types][:, None] * crv)
    a = np.where(valid, a, 0.0).reshape(-1)              # (7S,)
    w = w.reshape(-1)
    ph = phase[types].reshape(-1)
    m = 1.5 * np.outer(a, a) * np.outer(w, w) / (w[:, None] + w[None, :])
    m = m * (1.0 + 0.02 * np.cos(ph[:, None] + ph[None, :]))
    s = len(types)
    return m.reshape(s, N_REF, s, N_REF).transpose(0, 2, 1, 3).astype(np.float32)


def c6ref_block(types: Sequence[int]) -> np.ndarray:
    """(S, S, 7, 7) C6^ref block for the sorted unique atomic numbers ``types``."""
    src = c6_source()
    if src == "synthetic":
        return synthetic_c6ref_block(types)
    import torch  # the real table is a torch-saved tensor

    full = torch.load(src[5:], weights_only=True)
    idx = torch.as_tensor(np.asarray(types, dtype=np.int64))
    return full[idx][:, idx].numpy()


def c6ref_matrix(types: Sequence[int]) -> np.ndarray:
    """Symmetric (7S, 7S) matrix M[(a,p),(b,q)] = C6^ref[Z_a, Z_b, p, q] (utils.py:22)."""
    blk = c6ref_block(types)
    s = len(types)
    return blk.transpose(0, 2, 1, 3).reshape(s * N_REF, s * N_REF)


def _maxrel_err(ref: np.ndarray, approx: np.ndarray) -> float:
    """Max |ref - approx| / |ref| over non-zero entries of ref (utils.py:25-32)."""
    safe = np.where(ref == 0, 1.0, ref)
    return float(np.max(np.abs(ref - approx) * np.where(ref == 0, 0.0, 1.0 / safe)))


def decomp(types: Sequence[int], c6tol: float, verbose: bool = False, seed: int = 42):
    """Low-rank eigendecomposition M ~ V diag(lam) V^T (utils.py:35-73).

    Returns (eigs (r,), eigvecs (7S, r)) in float64 and the achieved max relative error.
    """
    from scipy.sparse.linalg import eigsh

    m = c6ref_matrix(types).astype(np.float64)
    n = m.shape[0]
    max_rank = n - 1
    v0 = np.random.default_rng(seed).standard_normal(n).astype(np.float64)
    k = 1
    eigs, vecs = eigsh(m, k=k, v0=v0)
    while _maxrel_err(m, vecs @ np.diag(eigs) @ vecs.T) * 100 >= c6tol and k < max_rank:
        k += 1
        eigs, vecs = eigsh(m, k=k, v0=v0)
    err = _maxrel_err(m, vecs @ np.diag(eigs) @ vecs.T)
    if verbose:
        print(f"C6 decomposition: rank {k}, largest relative entry error {err * 100:.4g} %")
        if k == max_rank and err * 100 >= c6tol:
            print(f"C6 decomposition: tolerance {c6tol} % not met at the largest rank tried ({max_rank})")
    return eigs, vecs, err


@functools.lru_cache(maxsize=64)
def species_setup(types: Tuple[int, ...], c6tol: float):
    """Cached decomposition for a tuple of sorted unique atomic numbers."""
    eigs, vecs, err = decomp(list(types), c6tol)
    return eigs, vecs, err
