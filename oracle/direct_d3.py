"""ORACLE (test infrastructure only): direct pairwise D3(BJ) lattice sum in float64.

The accuracy oracle for the reciprocal-space methods. With the same low-rank C6 the
reference uses (C6_ij = sum_r lambda_r c_ir c_jr, c from the smooth-cutoff CN and the
softmax interpolation, src/fourierd3/core.py:323-386, 449-543) the dispersion energy is

    E = -1/2 sum'_{i,j,n} C6_ij [ s6 / (r^6 + R0^6) + 3 s8 sqrt(Q_i Q_j) / (r^8 + R0^8) ],

the sum over all periodic images n except i = j at n = 0, r in Bohr, R0_XY =
a1 sqrt(3 sqrt(Q_X) sqrt(Q_Y)) + a2 (src/fourierd3/pair_pot.py:64). The reference evaluates
exactly this lattice sum in Fourier space (its k = 0 term included), so SPME/PME/Ewald
converge to it as the mesh is refined or the k cutoff raised.

Here the sum runs over all pairs closer than ``r_direct`` (Angstrom) and the remainder is the
continuum tail -(2 pi / Omega) sum_r lambda_r sum_XY A_X^r A_Y^r I_XY, A_X^r = sum_{i in X} c_ir,
I_XY = int_R^inf r^2 phi_XY(r) dr: the r^-6 part in closed form, the r^-8 part as a
series in (R0/R)^8; its virial is that of the stretched pairs beyond R,
(1/3) int r^3 phi'(r) dr = -R^3 phi(R)/3 - I. Forces and stress: analytic pair derivatives plus autograd through the CN
chain (strain convention of src/fourierd3/calculator.py:146-188).
"""
from __future__ import annotations

import itertools
import math

import numpy as np
import torch

from oracle.neighbours import neighbour_list_cells
from oracle.reference_port import ANGSTROM_TO_BOHR, HARTREE_TO_EV, OracleFourierD3


def _tail_integrals(R0: np.ndarray, qq: np.ndarray, s6: float, s8: float, Rc: float) -> np.ndarray:
    """I_XY = int_Rc^inf r^2 [s6/(r^6+R0^6) + 3 s8 qq/(r^8+R0^8)] dr (Bohr)."""
    a3 = R0 ** 3
    i6 = (math.pi / 2 - np.arctan(Rc ** 3 / a3)) / (3 * a3)
    # int r^2/(r^8+b^8) = sum_k (-1)^k b^(8k) Rc^-(5+8k) / (5+8k), |b/Rc| < 1
    t = (R0 / Rc) ** 8
    i8 = np.zeros_like(R0)
    term = Rc ** -5.0 * np.ones_like(R0)
    for k in range(12):
        i8 = i8 + ((-1) ** k) * term / (5 + 8 * k)
        term = term * t
    return s6 * i6 + 3 * s8 * qq * i8


def direct_calculate(numbers, positions, cell, r_direct: float = 20.0, chunk: int = 256, **model_kw):
    """(E [eV], F [eV/A] (N,3), stress [eV/A^3] (3,3)) of the direct lattice sum."""
    o = OracleFourierD3(numbers, cell, **model_kw)
    dt = torch.float64
    pos_np = np.asarray(positions, dtype=np.float64)
    cell_np = np.asarray(cell, dtype=np.float64)
    n = len(pos_np)
    # --- CN chain (differentiable w.r.t. positions and strain) ----------------------------
    i, j, S = neighbour_list_cells(pos_np, cell_np, o.r_cut_ang)
    cell_t = torch.tensor(cell_np, dtype=dt)
    strain = torch.zeros(3, 3, dtype=dt, requires_grad=True)
    scell = cell_t + torch.einsum("ab,Ab->Aa", strain, cell_t)
    pos = torch.tensor(pos_np, dtype=dt, requires_grad=True)
    spos = pos + torch.einsum("ab,ib->ia", strain, pos)
    sh = torch.matmul(torch.tensor(S, dtype=dt), scell)
    ei = torch.tensor(np.stack([i, j]))
    cn = o.cn(spos * o.a2b, ei, sh * o.a2b)
    c6 = o.c6_factors(cn)                                  # (N, R), differentiable
    c = c6.detach().numpy()
    lam = o.eigs.numpy()
    sp = o.species.numpy()
    g = o.green
    R0 = g.R.numpy()
    qq = g.qq.numpy()
    s6, s8 = float(o.params[0]), float(o.params[1])
    # --- pair sum within r_direct (Bohr) ---------------------------------------------------
    x = pos_np * ANGSTROM_TO_BOHR
    cb = cell_np * ANGSTROM_TO_BOHR
    rc = r_direct * ANGSTROM_TO_BOHR
    heights = 1.0 / np.linalg.norm(np.linalg.inv(cb), axis=0)
    nimg = [int(math.ceil(rc / h)) + 1 for h in heights]
    shifts = np.array(list(itertools.product(*[range(-m, m + 1) for m in nimg])), dtype=np.float64) @ cb
    e_pair = 0.0
    dEdc = np.zeros_like(c)
    grad = np.zeros_like(x)
    vir = np.zeros((3, 3))
    cl = c * lam[None, :]
    rc2 = rc * rc
    for i0 in range(0, n, chunk):
        i1 = min(n, i0 + chunk)
        ii = np.arange(i0, i1)
        C6 = cl[ii] @ c.T                                  # (ni, N)
        R0p = R0[sp[ii]][:, sp]
        qqp = qq[sp[ii]][:, sp]
        R06 = R0p ** 6
        R08 = R0p ** 8
        for sv in shifts:
            d = x[None, :, :] + sv[None, None, :] - x[ii][:, None, :]
            r2 = np.einsum("ijk,ijk->ij", d, d)
            m = (r2 < rc2) & (r2 > 1e-20)
            if not m.any():
                continue
            r2m = np.where(m, r2, 1.0)
            r6 = r2m ** 3
            r8 = r6 * r2m
            den6 = r6 + R06
            den8 = r8 + R08
            phi = s6 / den6 + 3 * s8 * qqp / den8
            # dphi/dr / r
            dphi_r = -s6 * 6 * r2m ** 2 / den6 ** 2 - 3 * s8 * qqp * 8 * r6 / den8 ** 2
            phi = np.where(m, phi, 0.0)
            dphi_r = np.where(m, dphi_r, 0.0)
            e_pair += -0.5 * np.sum(C6 * phi)
            # dE/dc_ir = -sum_j lambda_r c_jr phi_ij (both orderings of the pair)
            dEdc[ii] += -(phi @ c) * lam[None, :]
            # dE/dx_i = sum_j C6 phi'(r) d / r  (d = x_j + n - x_i)
            w = C6 * dphi_r
            grad[ii] += np.einsum("ij,ijk->ik", w, d)
            vir += -0.5 * np.einsum("ij,ija,ijb->ab", w, d, d)
    # --- continuum tail ----------------------------------------------------------------------
    vol = abs(np.linalg.det(cb))
    I = _tail_integrals(R0, qq, s6, s8, rc)
    S_sp = len(o.types)
    A = np.zeros((S_sp, c.shape[1]))
    np.add.at(A, sp, c)
    e_tail = -(2 * math.pi / vol) * float(np.einsum("r,xr,yr,xy->", lam, A, A, I))
    dEdc += -(4 * math.pi / vol) * lam[None, :] * (I[sp] @ A)
    # continuum virial of the pairs beyond R (each pair vector stretched by the strain):
    # (1/3) int r^3 phi' = -R^3 phi(R)/3 - I  ->  -E_tail + (2 pi R^3 / (3 Omega)) sum lam A A phi(R)
    phiR = s6 / (rc ** 6 + R0 ** 6) + 3 * s8 * qq / (rc ** 8 + R0 ** 8)
    surf = (2 * math.pi * rc ** 3 / (3 * vol)) * float(np.einsum("r,xr,yr,xy->", lam, A, A, phiR))
    vir += (-e_tail + surf) * np.eye(3)
    e_ha = e_pair + e_tail
    # --- chain to CN, positions and strain ----------------------------------------------------
    surrogate = torch.sum(torch.tensor(dEdc) * c6)
    surrogate.backward()
    g_pos = pos.grad.numpy() + grad * ANGSTROM_TO_BOHR    # dE/dx_A (Hartree/A)
    g_strain = strain.grad.numpy() + vir
    forces = -g_pos * HARTREE_TO_EV
    stress = g_strain * HARTREE_TO_EV / vol * (ANGSTROM_TO_BOHR ** 3)
    return e_ha * HARTREE_TO_EV, forces, stress
