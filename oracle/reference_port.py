"""ORACLE (test infrastructure only): CPU float64 restatement of the reference's
FourierD3 energy and of its ASE strain/autograd protocol for forces and stress.

Header: this module is the checker, never the product. Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py`` (CPU baseline / reference arm) may
import it. Parity status: PINNED for everything written in the reference
package itself -- tests/golden/make_golden.py runs the reference's own modules
(src/fourierd3/{core,pair_pot,kspace_filter_d3,mesh_interpolator_d3,utils,
calculator}.py) and this restatement is checked against those fixtures.
UNPINNED for the torch-pme and matscipy conventions (see torchpme_shim.py and
neighbours.py), which the fixture run has to shim as well.

Each step cites the reference line it follows.
"""
from __future__ import annotations

import math
from typing import Optional, Sequence

import numpy as np
import torch

from fourierd3_b200 import tables
from oracle import torchpme_shim as pme
from oracle.neighbours import neighbour_list_cells as neighbour_list

ANGSTROM_TO_BOHR = 1 / 0.52917726      # core.py:120
HARTREE_TO_EV = 27.21138505            # calculator.py:54
PBE_BJ = (1.0, 0.7875, 0.4289, 4.4407) # core.py:168


def det3(m):
    """Cofactor determinant (utils.py:130-139)."""
    c00 = m[1, 1] * m[2, 2] - m[1, 2] * m[2, 1]
    c10 = m[1, 2] * m[2, 0] - m[1, 0] * m[2, 2]
    c20 = m[1, 0] * m[2, 1] - m[1, 1] * m[2, 0]
    return m[0, 0] * c00 + m[0, 1] * c10 + m[0, 2] * c20


def inv3(m):
    """Adjugate / determinant inverse (utils.py:142-167)."""
    c00 = m[1, 1] * m[2, 2] - m[1, 2] * m[2, 1]
    c01 = m[0, 2] * m[2, 1] - m[0, 1] * m[2, 2]
    c02 = m[0, 1] * m[1, 2] - m[0, 2] * m[1, 1]
    c10 = m[1, 2] * m[2, 0] - m[1, 0] * m[2, 2]
    c11 = m[0, 0] * m[2, 2] - m[0, 2] * m[2, 0]
    c12 = m[0, 2] * m[1, 0] - m[0, 0] * m[1, 2]
    c20 = m[1, 0] * m[2, 1] - m[1, 1] * m[2, 0]
    c21 = m[0, 1] * m[2, 0] - m[0, 0] * m[2, 1]
    c22 = m[0, 0] * m[1, 1] - m[0, 1] * m[1, 0]
    adj = torch.stack([torch.stack([c00, c01, c02]), torch.stack([c10, c11, c12]),
                       torch.stack([c20, c21, c22])])
    det = m[0, 0] * c00 + m[0, 1] * c10 + m[0, 2] * c20
    return adj / det


class GreenD3:
    """G_XY(|k|) of the BJ-damped r^-6 / r^-8 pair potential (pair_pot.py:35-228)."""

    def __init__(self, sqrtq: torch.Tensor, params: torch.Tensor):
        self.params = params
        qq = torch.outer(sqrtq, sqrtq)                               # pair_pot.py:55
        self.qq = qq
        self.R = params[2] * torch.sqrt(3 * qq) + params[3]          # pair_pot.py:64
        R = self.R
        self.pi = torch.tensor(math.pi, dtype=R.dtype)
        self.sq3 = torch.sqrt(torch.tensor(3.0, dtype=R.dtype))
        self.sq2 = torch.sqrt(torch.tensor(2.0, dtype=R.dtype))
        self.sin8 = torch.sin(self.pi / 8)
        self.cos8 = torch.cos(self.pi / 8)
        R2, R3 = R ** 2, R ** 3
        R4 = R * R3
        R5 = R * R4
        R6 = R3 ** 2
        R8 = R3 * R5
        pi2 = self.pi ** 2
        self.selfcont = params[0] / torch.diagonal(R6) + 3 * params[1] * torch.diagonal(qq) / torch.diagonal(R8)  # :84-89
        self.c6_s1 = (2 * pi2) / (3 * R3)                           # :95
        self.c6_s2 = (2 * pi2 * R) / 9                              # :96
        self.c6_pre = (2 * pi2) / (3 * R4)                          # :98
        self.c8_s1 = (pi2 * self.sq2 * self.sin8) / R5              # :102
        self.c8_s2 = self.c8_s1 * R2 / 6                            # :103
        self.c8_pre = -pi2 / R6                                     # :105

    def __call__(self, k: torch.Tensor) -> torch.Tensor:
        """k: |k| of any shape -> G of shape (S, S, *k.shape) (pair_pot.py:142-178)."""
        ex = (slice(None), slice(None)) + (None,) * k.dim()
        R = self.R[ex]
        kk = k.unsqueeze(0).unsqueeze(0)
        ksq = kk * kk
        small = kk * R < 1e-15
        ks = torch.where(small, torch.ones_like(kk), kk)
        u = ks * R
        f6s = self.c6_s1[ex] - self.c6_s2[ex] * ksq
        n6 = torch.exp(-u) - 2 * torch.exp(-u / 2) * torch.cos(self.pi / 3 + u * self.sq3 / 2)
        f6 = self.params[0] * torch.where(small, f6s, self.c6_pre[ex] / ks * n6)
        f8s = self.c8_s1[ex] - self.c8_s2[ex] * ksq
        n8 = (torch.exp(-u * self.sin8) * torch.cos(self.pi / 4 + u * self.cos8)
              + torch.exp(-u * self.cos8) * torch.cos(3 * self.pi / 4 + u * self.sin8))
        f8 = 3 * self.params[1] * torch.where(small, f8s, self.c8_pre[ex] / ks * n8)
        return f6 + self.qq[ex] * f8


class CNPotentialD4:
    """Fourier transform of the D4 CN pair function f_AB(r) = delta_AB / 2 erfc(k0 (r - r0_AB) / r0_AB)
    (pair_pot.py:235-406): r0_AB = rcov_cn_A + rcov_cn_B, delta_AB = k1 exp(-(|EN_A - EN_B| + k2)^2 / k3),
    closed form for k r0 >= 1e-3 and a k^2 Taylor branch below; self term delta_AA / 2 erfc(-k0)."""

    K0, K1, K2, K3 = 7.5, 4.10451, 19.08857, 2 * 11.28174 ** 2      # pair_pot.py:275-278

    def __init__(self, types, dtype=torch.float64):
        t = tables.load_tables()
        idx = torch.as_tensor(list(types))
        rc = torch.tensor(t["rcov_cn"])[idx].to(dtype)               # pair_pot.py:294-297
        self.r0 = rc.unsqueeze(0) + rc.unsqueeze(1)
        en = torch.tensor(t["en"])[idx].to(dtype)                    # pair_pot.py:301-305
        ed = torch.abs(en.unsqueeze(0) - en.unsqueeze(1))
        self.delta = self.K1 * torch.exp(-torch.square(ed + self.K2) / self.K3)
        k0 = torch.tensor(self.K0, dtype=dtype)
        self.k0sq = k0 * k0
        self.pi = torch.tensor(math.pi, dtype=dtype)
        A = 1.0 / 3.0 + 1.0 / (2.0 * self.K0 ** 2)                   # pair_pot.py:321-324
        B = 1.0 / 30.0 + 1.0 / (6.0 * self.K0 ** 2) + 1.0 / (8.0 * self.K0 ** 4)
        r0sq = self.r0 * self.r0
        self.c0 = 4.0 * self.pi * self.delta * r0sq * self.r0 * A
        self.c2 = 4.0 * self.pi * self.delta * r0sq * r0sq * self.r0 * B
        self.selfcont = (torch.diagonal(self.delta) / 2.0 * torch.erfc(-k0)).view(-1)   # pair_pot.py:330-331

    def __call__(self, k: torch.Tensor) -> torch.Tensor:
        """|k| of any shape -> hat f of shape (S, S, *k.shape) (pair_pot.py:336-376)."""
        ex = (slice(None), slice(None)) + (None,) * k.dim()
        r0, delta = self.r0[ex], self.delta[ex]
        kk = k.unsqueeze(0).unsqueeze(0)
        small = kk * r0 < 1e-3
        ks = torch.where(small, torch.ones_like(kk), kk)
        kr0 = ks * r0
        gauss = torch.exp(-kr0 * kr0 / (4.0 * self.k0sq))
        s, c = torch.sin(kr0), torch.cos(kr0)
        term1 = (s - kr0 * c) / (ks * ks * ks)
        term2 = r0 * r0 * s / (2.0 * self.k0sq * ks)
        large = 4.0 * self.pi * delta * gauss * (term1 + term2)
        return torch.where(small, self.c0[ex] - self.c2[ex] * kk * kk, large)


def sinc_window(ns, order: int) -> torch.Tensor:
    """prod_a sinc(m_a / n_a)^(2p), clamped at 1e-10, on the rfft half grid (pair_pot.py:184-207).

    The reference builds the Miller indices with ``torch.fft.fftfreq`` without a dtype,
    i.e. in torch's default float32, so the whole window is float32 even on the float64
    path; G / window then promotes to float64. Restated exactly, float32 included.
    """
    nx, ny, nz = (int(v) for v in ns)
    dtype = torch.float32
    mx = torch.fft.fftfreq(nx, d=1.0 / nx, dtype=dtype)
    my = torch.fft.fftfreq(ny, d=1.0 / ny, dtype=dtype)
    mz = torch.fft.rfftfreq(nz, d=1.0 / nz, dtype=dtype)
    sc = (torch.sinc(mx / nx)[:, None, None] * torch.sinc(my / ny)[None, :, None]
          * torch.sinc(mz / nz)[None, None, :])
    sc = torch.pow(sc, 2 * order)
    return torch.where(sc < 1e-10, 1e-10, sc)


def hermitian_weights(nzh: int, dtype=torch.float64) -> torch.Tensor:
    """1 at the first and last rfft z-plane, 2 elsewhere (pair_pot.py:213-218)."""
    w = torch.full((nzh,), 2.0, dtype=dtype)
    w[0] = 1.0
    w[-1] = 1.0
    return w


class OracleFourierD3:
    """Float64 CPU restatement of ``FourierD3`` (core.py:50-583), cnfunc='smooth_cut'."""

    def __init__(self, numbers: Sequence[int], cell, mesh_spacing: float = 1.2, c6tol: float = 1.0,
                 method: str = "spme", params=None, interpolation_nodes: int = 5,
                 k_cutoff: float = 10.0, r_cut: float = 6.0, cncorr: Optional[np.ndarray] = None,
                 cnfunc: str = "smooth_cut"):
        dt = torch.float64
        self.dtype = dt
        if cnfunc not in ("smooth_cut", "d4"):
            raise ValueError(f"Unknown cnfunc '{cnfunc}'")                # calculator.py:174
        self.cnfunc = cnfunc
        self.method = method
        self.order = int(interpolation_nodes)
        numbers = np.asarray(numbers)
        uniq = np.unique(numbers)                                    # core.py:104-114
        remap = {int(z): i for i, z in enumerate(uniq)}
        self.types = [int(z) for z in uniq]
        self.species = torch.tensor([remap[int(z)] for z in numbers], dtype=torch.long)
        self.n_species = len(uniq)
        self.a2b = torch.tensor(ANGSTROM_TO_BOHR, dtype=dt)         # core.py:120-125
        self.r_cut = r_cut * ANGSTROM_TO_BOHR
        self.r_cut_ang = float(r_cut)
        cell_b = torch.as_tensor(np.asarray(cell), dtype=dt) * self.a2b
        eigs, vecs, _ = tables.species_setup(tuple(self.types), float(c6tol))   # core.py:139
        self.eigs = torch.tensor(eigs, dtype=dt)
        self.n_rank = self.eigs.shape[0]
        self.vq = torch.tensor(vecs, dtype=dt).view(self.n_species, 7, self.n_rank)  # core.py:148
        t = tables.load_tables()
        self.rcov = torch.tensor(t["rcov"])[uniq].to(dt)             # core.py:152
        self.cnref = torch.tensor(t["cnref"])[uniq, :].to(dt)        # core.py:155
        sqrtq = torch.tensor(t["sqrtQz"])[uniq].to(dt)               # pair_pot.py:53
        p = params if params is not None else PBE_BJ
        self.params = torch.tensor(p, dtype=dt)
        self.green = GreenD3(sqrtq, self.params)
        self.cnpot = CNPotentialD4(self.types, dt) if cnfunc == "d4" else None   # core.py:177-179
        self.cncorr = None if cncorr is None else torch.as_tensor(np.asarray(cncorr), dtype=dt)
        if method in ("spme", "pme"):
            self.ns_mesh = pme.get_ns_mesh(cell_b, mesh_spacing * ANGSTROM_TO_BOHR)   # core.py:186
        elif method == "ewald":
            norms = torch.linalg.norm(cell_b, dim=1)                 # core.py:228-230
            self.ns = torch.ceil(k_cutoff * norms / (2 * math.pi)).long()
        else:
            raise ValueError(method)

    # --- core.py:323-386 -------------------------------------------------
    def cn(self, pos_b, edge_index, shifts_b):
        src, dst = edge_index[0], edge_index[1]
        vec = pos_b[dst] - pos_b[src] + shifts_b
        r = torch.linalg.norm(vec, dim=-1)
        rs = torch.clamp(r, min=1e-6)
        rcs = self.rcov[self.species[src]] + self.rcov[self.species[dst]]
        r1 = 0.5 * rcs + 0.5 * self.r_cut
        coeff = torch.where(rs > r1, rs, r1)
        denom = (self.r_cut - coeff).pow(2) + 1e-6
        kcn = 16.0 + (coeff - r1) ** 2 / denom
        arg = -kcn * ((4.0 / 3.0) * rcs * (1.0 / rs) - 1.0)
        contrib = torch.sigmoid(-arg)
        contrib = torch.where(r > 1e-6, contrib, torch.zeros((), dtype=self.dtype))
        cn = torch.zeros(pos_b.shape[0], dtype=self.dtype).index_add(0, src, contrib)
        if self.cncorr is not None:
            cn = self.cncorr[self.species, 1] * cn + self.cncorr[self.species, 0]
        return cn

    # --- core.py:449-478, 525-543 -----------------------------------------
    def c6_factors(self, cn):
        refs = self.cnref[self.species]
        logits = -4.0 * torch.square(cn.unsqueeze(1) - refs)
        logits = logits.masked_fill(refs == -1, float("-inf"))
        w = torch.softmax(logits, dim=1)
        return torch.einsum("nk,nkr->nr", w, self.vq[self.species])

    def _stencil(self, pos_b, cell_b):
        """Per-atom stencil weights (N, p^3) and flat mesh indices (N p^3,) of the torch-pme
        interpolator (MeshInterpolator.compute_weights, core.py:555)."""
        n_atoms = pos_b.shape[0]
        nx, ny, nz = (int(v) for v in self.ns_mesh)
        p = self.order
        w, base = pme.mesh_weights(pos_b, inv3(cell_b), self.ns_mesh, p,
                                   "P3M" if self.method == "spme" else "Lagrange")
        sh = torch.arange(p)
        ix = (base[:, 0][:, None] + sh[None, :]) % nx                # (N, p)
        iy = (base[:, 1][:, None] + sh[None, :]) % ny
        iz = (base[:, 2][:, None] + sh[None, :]) % nz
        wx, wy, wz = w[:, :, 0].T, w[:, :, 1].T, w[:, :, 2].T        # (N, p)
        wgeo = (wx[:, :, None, None] * wy[:, None, :, None] * wz[:, None, None, :]).reshape(n_atoms, -1)
        lin = (iz[:, None, None, :] + nz * (iy[:, None, :, None] + ny * ix[:, :, None, None])).reshape(-1)
        return wgeo, lin

    # --- core.py:388-447: D4 CN in k-space (no neighbour list) -----------------------
    def cn_d4(self, pos_b, cell_b, volume):
        """CN_i = phi_{X_i}(r_i) / volume - f_{X_i X_i}(0), phi_X = sum_Y G^CN_XY * rho_Y with rho the
        one-hot species density. The mesh branch spreads with the interpolation weights of the
        current positions and the Ewald branch uses the (N, S) one-hot species matrix: the
        reference's own code reads weights only computed later in forward (core.py:514 vs 555)
        and an attribute it never defines (core.py:436); this is the algorithm with both repaired."""
        n_atoms = pos_b.shape[0]
        S = self.n_species
        if self.method in ("spme", "pme"):
            nx, ny, nz = (int(v) for v in self.ns_mesh)
            wgeo, lin = self._stencil(pos_b, cell_b)
            onehot = torch.zeros(n_atoms, S, dtype=self.dtype)
            onehot[torch.arange(n_atoms), self.species] = 1.0            # core.py:417-418
            vals = (onehot.unsqueeze(1) * wgeo.unsqueeze(2)).flatten(0, 1)
            rho = torch.zeros(nx * ny * nz, S, dtype=self.dtype).index_add(0, lin, vals)
            rho = rho.t().contiguous().view(S, nx, ny, nz)
            hat = torch.fft.rfftn(rho, norm="backward", dim=(1, 2, 3))   # kspace_filter_d3.py:142
            kvec = pme.generate_kvectors(cell_b, self.ns_mesh, for_ewald=False)
            G = self.cnpot(torch.linalg.norm(kvec, dim=-1))              # (S, S, nx, ny, nzh)
            if self.method == "spme":
                G = G / sinc_window(self.ns_mesh, self.order)           # pair_pot.py:378-399
            Gf = G.flatten(2).permute(2, 0, 1).to(torch.complex128)     # (nk, S, S)
            interm = torch.einsum("kab,bk->ak", Gf, hat.flatten(1))     # kspace_filter_d3.py:148
            phi = torch.fft.irfftn(interm.view(hat.shape), norm="forward", s=(nx, ny, nz), dim=(1, 2, 3))
            flat = phi.reshape(S, -1).t()                                # (M, S)
            g = flat[lin, :].view(n_atoms, -1, S)
            phi_atoms = (wgeo.unsqueeze(2) * g).sum(dim=1)              # mesh_interpolator_d3.py:140-189
        else:
            kvec = pme.generate_kvectors(cell_b, self.ns, for_ewald=True)
            G = self.cnpot(torch.linalg.norm(kvec, dim=1))               # (S, S, nk)
            arg = torch.matmul(kvec, pos_b.T)
            ex = torch.stack([torch.cos(arg), torch.sin(arg)], dim=0)   # (2, nk, N)
            nk = ex.shape[1]
            onehot = torch.nn.functional.one_hot(self.species, S).to(self.dtype)
            Sf = torch.mm(ex.reshape(2 * nk, n_atoms), onehot).view(2, nk, S)   # core.py:436
            F = torch.einsum("tkj,kij->tki", Sf, G.permute(2, 0, 1))
            phi_atoms = torch.einsum("tka,tki->ai", ex, F)
        cn_raw = phi_atoms[torch.arange(n_atoms), self.species]
        return cn_raw / volume - self.cnpot.selfcont[self.species]      # core.py:444-446

    def kspace_mesh(self, pos_b, c6, cell_b):
        """SPME/PME k-space sum (core.py:553-561, mesh_interpolator_d3.py:74-138,
        kspace_filter_d3.py:29-70)."""
        n_atoms = pos_b.shape[0]
        S, R = self.n_species, self.n_rank
        nx, ny, nz = (int(v) for v in self.ns_mesh)
        p = self.order
        wgeo, lin = self._stencil(pos_b, cell_b)
        onehot = torch.zeros(n_atoms, S, R, dtype=self.dtype).index_put(
            (torch.arange(n_atoms), self.species), c6)               # core.py:537-543
        vals = (onehot.reshape(n_atoms, S * R).unsqueeze(1) * wgeo.unsqueeze(2)).flatten(0, 1)
        rho = torch.zeros(nx * ny * nz, S * R, dtype=self.dtype).index_add(0, lin, vals)
        rho = rho.t().contiguous().view(S, R, nx, ny, nz)
        sk = torch.fft.rfftn(rho, norm="backward", dim=(2, 3, 4))   # kspace_filter_d3.py:55
        kvec = pme.generate_kvectors(cell_b, self.ns_mesh, for_ewald=False)
        knorm = torch.linalg.norm(kvec, dim=-1)
        G = self.green(knorm)                                         # (S, S, nx, ny, nzh)
        if self.method == "spme":
            G = G / sinc_window(self.ns_mesh, p)
        G = G * hermitian_weights(G.shape[-1])
        Gf = G.flatten(2).permute(2, 0, 1).to(torch.complex128)     # (nk, S, S)
        skf = sk.flatten(2).permute(2, 0, 1)                          # (nk, S, R)
        interm = torch.bmm(Gf, skf.conj())
        per_rank = (skf * interm).real.sum(dim=(0, 1))                # (R,)
        return torch.dot(self.eigs, per_rank)

    def kspace_ewald(self, pos_b, c6, cell_b):
        """Direct Ewald k-sum (core.py:225-242, 563-577), including the |lambda| weighting."""
        n_atoms = pos_b.shape[0]
        kvec = pme.generate_kvectors(cell_b, self.ns, for_ewald=True)
        knorm = torch.linalg.norm(kvec, dim=1)
        G = self.green(knorm)                                         # (S, S, nk)
        arg = torch.matmul(kvec, pos_b.T)
        ex = torch.stack([torch.cos(arg), torch.sin(arg)], dim=0)     # (2, nk, N)
        onehot = torch.zeros(n_atoms, self.n_species, self.n_rank, dtype=self.dtype).index_put(
            (torch.arange(n_atoms), self.species), c6)
        sc = torch.einsum("izr,pki->rzpk", onehot, ex)
        sc = sc * torch.sqrt(torch.abs(self.eigs)).view(-1, 1, 1, 1)
        return torch.sum(torch.einsum("ijk,ripk,rjpk->jk", G, sc, sc))

    def energy(self, pos_ang, edge_index, shifts_ang, cell_ang):
        """Energy in Hartree; differentiable w.r.t. positions, shifts and cell (core.py:480-583)."""
        cell_b = cell_ang * self.a2b                                 # core.py:254
        volume = torch.abs(det3(cell_b))                             # core.py:255
        pos_b = pos_ang * self.a2b                                   # core.py:505
        shifts_b = shifts_ang * self.a2b                             # core.py:507
        if self.cnfunc == "d4":
            cn = self.cn_d4(pos_b, cell_b, volume)                   # core.py:517-524
        else:
            cn = self.cn(pos_b, edge_index, shifts_b)
        c6 = self.c6_factors(cn)
        tmp = torch.sum(torch.square(c6) * self.green.selfcont[self.species].unsqueeze(1), dim=0)
        vself = torch.dot(self.eigs, tmp)                            # core.py:547-550
        if self.method == "ewald":
            ek = self.kspace_ewald(pos_b, c6, cell_b)
        else:
            ek = self.kspace_mesh(pos_b, c6, cell_b)
        return ek / (-2 * volume) + vself / 2, volume                # core.py:581

    def calculate(self, positions: np.ndarray, cell: np.ndarray, edges=None):
        """E [eV], F [eV/A] (N,3), stress [eV/A^3] (3,3) by the strain protocol of
        calculator.py:146-192. ``edges`` = (edge_index (2,E), unit_shifts (E,3)) or None
        to build them with the oracle neighbour list."""
        dt = self.dtype
        cell_t = torch.as_tensor(np.asarray(cell), dtype=dt)
        strain = torch.zeros(3, 3, dtype=dt, requires_grad=True)
        scell = cell_t + torch.einsum("ab,Ab->Aa", strain, cell_t)
        pos = torch.tensor(np.asarray(positions), dtype=dt, requires_grad=True)
        spos = pos + torch.einsum("ab,ib->ia", strain, pos)
        if self.cnfunc == "d4":                                       # calculator.py:171-173
            edge_index = torch.zeros((2, 0), dtype=torch.long)
            ushift = torch.zeros((0, 3), dtype=dt)
        elif edges is None:
            i, j, S = neighbour_list(np.asarray(positions, dtype=np.float64),
                                     np.asarray(cell, dtype=np.float64), self.r_cut_ang)
            edge_index = torch.tensor(np.stack((i, j)), dtype=torch.long)
            ushift = torch.tensor(S, dtype=dt)
        else:
            edge_index = torch.as_tensor(edges[0], dtype=torch.long)
            ushift = torch.as_tensor(edges[1], dtype=dt)
        sshift = torch.matmul(ushift, scell)
        e, volume = self.energy(spos, edge_index, sshift, scell)
        e_ev = e * HARTREE_TO_EV
        e_ev.backward()
        forces = -pos.grad
        stress = strain.grad / volume.detach() * (ANGSTROM_TO_BOHR ** 3)
        return float(e_ev.detach()), forces.numpy(), stress.numpy()
