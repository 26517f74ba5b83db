"""ORACLE (test infrastructure only): brute-force periodic neighbour list.

Restates what the reference obtains from matscipy's ``neighbour_list("ijS",
cutoff=r_cut)`` (src/fourierd3/calculator.py:94-123): every directed pair
(i, j, S), S an integer lattice-shift vector, with

    |x_j - x_i + S . cell| < r_cut          (Angstrom, the caller's units)

in both directions, periodic self-images (i, i, S != 0) included and (i, i, 0)
excluded. matscipy (no version pinned, pyproject.toml:20) is not installed, so
its own rounding at the cutoff is UNPINNED; this module fixes the predicate's
float64 evaluation order exactly, and the GPU cell-list build evaluates the
identical expression (no fused multiply-add), so the two pair sets are equal
bit for bit:

    sh_a = (S_0 * cell[0,a] + S_1 * cell[1,a]) + S_2 * cell[2,a]
    d_a  = (x_j,a - x_i,a) + sh_a
    r2   = (d_0 * d_0 + d_1 * d_1) + d_2 * d_2 ;   pair iff r2 < r_cut * r_cut

Output is sorted by (i, j, S) lexicographically.
"""
from __future__ import annotations

import itertools
import math

import numpy as np


def image_range(cell: np.ndarray, r_cut: float) -> np.ndarray:
    """Per-axis number of lattice images that can hold a neighbour of a wrapped atom."""
    inv = np.linalg.inv(cell)
    heights = 1.0 / np.linalg.norm(inv, axis=0)          # perpendicular widths
    return np.array([int(math.ceil(r_cut / h)) + 1 for h in heights])


def neighbour_list(positions: np.ndarray, cell: np.ndarray, r_cut: float):
    x = np.asarray(positions, dtype=np.float64)
    c = np.asarray(cell, dtype=np.float64)
    n = x.shape[0]
    chunk = max(1, min(2048, 2_000_000 // max(n, 1)))
    # wrap into the cell so that a small image box suffices; S is corrected back below
    frac = x @ np.linalg.inv(c)
    off = np.floor(frac).astype(np.int64)                # x = wrapped + off . cell (approx.)
    rng = image_range(c, r_cut)
    rc2 = r_cut * r_cut
    out_i, out_j, out_s = [], [], []
    shifts = np.array(list(itertools.product(*[range(-m, m + 1) for m in rng])), dtype=np.int64)
    for i0 in range(0, n, chunk):
        i1 = min(n, i0 + chunk)
        ii = np.arange(i0, i1)
        for S in shifts:
            # S in the frame of the unwrapped input: S_true = S + off_i - off_j
            s_true = S[None, None, :] + off[ii][:, None, :] - off[None, :, :]   # (ni, n, 3)
            sh = ((s_true[..., 0:1] * c[0] + s_true[..., 1:2] * c[1]) + s_true[..., 2:3] * c[2])
            d = (x[None, :, :] - x[ii][:, None, :]) + sh
            r2 = (d[..., 0] * d[..., 0] + d[..., 1] * d[..., 1]) + d[..., 2] * d[..., 2]
            m = r2 < rc2
            self_pair = (ii[:, None] == np.arange(n)[None, :]) & np.all(s_true == 0, axis=-1)
            m &= ~self_pair
            a, b = np.nonzero(m)
            if a.size:
                out_i.append(ii[a])
                out_j.append(b)
                out_s.append(s_true[a, b])
    if not out_i:
        return (np.zeros(0, np.int64), np.zeros(0, np.int64), np.zeros((0, 3), np.int64))
    i = np.concatenate(out_i)
    j = np.concatenate(out_j)
    s = np.concatenate(out_s)
    # the wrapped image box may reach a pair twice only if it is the same (i, j, S): dedupe
    key = np.stack([i, j, s[:, 0], s[:, 1], s[:, 2]], axis=1)
    key = np.unique(key, axis=0)                         # sorted lexicographically
    return key[:, 0].copy(), key[:, 1].copy(), key[:, 2:].copy()


def neighbour_list_cells(positions: np.ndarray, cell: np.ndarray, r_cut: float):
    """Same pair set and order as ``neighbour_list`` via a numpy cell list (for large N).

    Candidate pairs come from bins at least r_cut high; every candidate is then tested
    with the exact predicate of the module docstring, so the result is identical.
    """
    x = np.asarray(positions, dtype=np.float64)
    c = np.asarray(cell, dtype=np.float64)
    inv = np.linalg.inv(c)
    heights = 1.0 / np.linalg.norm(inv, axis=0)
    nb = np.maximum(1, np.floor(heights / r_cut).astype(np.int64))
    if np.any(nb < 3):
        return neighbour_list(x, c, r_cut)
    frac = x @ inv
    off = np.floor(frac).astype(np.int64)
    b3 = np.minimum(((frac - off) * nb).astype(np.int64), nb - 1)
    bid = (b3[:, 0] * nb[1] + b3[:, 1]) * nb[2] + b3[:, 2]
    order = np.argsort(bid, kind="stable")
    counts = np.bincount(bid, minlength=int(np.prod(nb)))
    start = np.concatenate([[0], np.cumsum(counts)])
    rc2 = r_cut * r_cut
    out = []
    for d in itertools.product((-1, 0, 1), repeat=3):
        tb = b3 + np.array(d)
        S = np.floor_divide(tb, nb)
        tw = tb - S * nb
        tid = (tw[:, 0] * nb[1] + tw[:, 1]) * nb[2] + tw[:, 2]
        cnt = counts[tid]
        ii = np.repeat(np.arange(len(x)), cnt)
        base = np.repeat(start[tid], cnt)
        within = np.arange(len(ii)) - np.repeat(np.cumsum(cnt) - cnt, cnt)
        jj = order[base + within]
        s_true = np.repeat(S, cnt, axis=0) + off[ii] - off[jj]
        sh = ((s_true[:, 0:1] * c[0] + s_true[:, 1:2] * c[1]) + s_true[:, 2:3] * c[2])
        dv = (x[jj] - x[ii]) + sh
        r2 = (dv[:, 0] * dv[:, 0] + dv[:, 1] * dv[:, 1]) + dv[:, 2] * dv[:, 2]
        m = (r2 < rc2) & ~((ii == jj) & np.all(s_true == 0, axis=1))
        out.append(np.concatenate([ii[m, None], jj[m, None], s_true[m]], axis=1))
    key = np.unique(np.concatenate(out), axis=0)
    return key[:, 0].copy(), key[:, 1].copy(), key[:, 2:].copy()
