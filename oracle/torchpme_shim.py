"""ORACLE (test infrastructure only) -- restatement of the torch-pme routines the
reference calls. Parity for these conventions is UNPINNED: torch-pme (module
``torchpme``, no version pinned by the reference's pyproject.toml:19) is not
installed here and the reference has no tests fixing its behaviour. The
functions below restate torch-pme's documented algorithms in plain torch/numpy:

* ``get_ns_mesh`` (called at src/fourierd3/core.py:186): per axis
  n = 2 ** ceil(log2(2 * |a_i| / h + 1)).
* ``generate_kvectors`` (core.py:232,263; kspace_filter_d3.py:286):
  reciprocal cell B = 2 pi inv(cell)^T; k = m_x b_x + m_y b_y + m_z b_z with the
  FFT frequency orders m = fftfreq(n) * n on x and y, and on z either fftfreq
  (Ewald, full box, flattened) or rfftfreq (mesh, half box, grid shaped).
* ``mesh_weights`` (MeshInterpolator.compute_weights, core.py:555): fractional
  mesh coordinates u = n * (x @ inv(cell)); reference node round(u) for an odd
  number of nodes p and floor(u) for even p; node offsets
  1 - (p+1)//2 ... p//2; local coordinate x = u - ref (odd) or u - ref - 1/2
  (even); per-axis weights are the order-p cardinal B-spline (method "P3M")
  or the p-point Lagrange basis (method "Lagrange") evaluated at x.

Only tests/, the smoke check and bench.py's CPU baseline use this module.
"""
from __future__ import annotations

import math

import torch


def get_ns_mesh(cell: torch.Tensor, mesh_spacing: float) -> torch.Tensor:
    norms = torch.linalg.norm(cell, dim=1)
    approx = 2.0 * norms / mesh_spacing + 1.0
    return torch.tensor(2).pow(torch.ceil(torch.log2(approx)).long())


def _freq_orders(n: int, half: bool, like: torch.Tensor) -> torch.Tensor:
    if half:
        f = torch.fft.rfftfreq(n, device=like.device, dtype=like.dtype)
    else:
        f = torch.fft.fftfreq(n, device=like.device, dtype=like.dtype)
    return n * f


def generate_kvectors(cell: torch.Tensor, ns, for_ewald: bool) -> torch.Tensor:
    rec = 2.0 * math.pi * torch.linalg.inv(cell).T
    nx, ny, nz = (int(v) for v in ns)
    mx = _freq_orders(nx, False, cell).unsqueeze(-1) * rec[0]
    my = _freq_orders(ny, False, cell).unsqueeze(-1) * rec[1]
    mz = _freq_orders(nz, not for_ewald, cell).unsqueeze(-1) * rec[2]
    k = mx.view(-1, 1, 1, 3) + my.view(1, -1, 1, 3) + mz.view(1, 1, -1, 3)
    return k.reshape(-1, 3) if for_ewald else k


def bspline_weights(x: torch.Tensor, p: int) -> torch.Tensor:
    """Order-p cardinal B-spline at the p stencil nodes, shape (p, *x.shape).

    With alpha = 1/2 - x in [0, 1], node k has weight M_p(alpha + k), built by the
    Cox-de Boor recursion M_q(u) = [u M_{q-1}(u) + (q - u) M_{q-1}(u - 1)] / (q - 1).
    """
    a = 0.5 - x
    vals = [torch.ones_like(x)]                     # M_1(alpha + 0)
    for q in range(2, p + 1):
        new = []
        for j in range(q):
            u = a + j
            left = vals[j] if j < q - 1 else torch.zeros_like(x)
            right = vals[j - 1] if j >= 1 else torch.zeros_like(x)
            new.append((u * left + (q - u) * right) / (q - 1))
        vals = new
    return torch.stack(vals)


def lagrange_weights(x: torch.Tensor, p: int) -> torch.Tensor:
    """p-point Lagrange basis on equispaced nodes 0..p-1, charge at t = x + (p-1)/2."""
    t = x + 0.5 * (p - 1)
    out = []
    for k in range(p):
        w = torch.ones_like(x)
        for m in range(p):
            if m != k:
                w = w * (t - m) / (k - m)
        out.append(w)
    return torch.stack(out)


def mesh_weights(positions: torch.Tensor, inverse_cell: torch.Tensor, ns_mesh, p: int, method: str):
    """Return (weights (p, N, 3), base (N, 3) int64) -- base is the first stencil node
    (not yet wrapped); node k of axis a sits at (base[:, a] + k) mod n_a."""
    ns = torch.as_tensor([int(v) for v in ns_mesh], dtype=positions.dtype, device=positions.device)
    u = ns * torch.matmul(positions, inverse_cell)
    if p % 2 == 0:
        ref = torch.floor(u)
        x = u - (ref + 0.5)
    else:
        ref = torch.round(u)
        x = u - ref
    ref = ref.detach().long()
    if method == "P3M":
        w = bspline_weights(x, p)
    elif method == "Lagrange":
        w = lagrange_weights(x, p)
    else:
        raise ValueError(method)
    base = ref + (1 - (p + 1) // 2)
    return w, base
