"""Plan + workspace owner around the C ABI (one per model / structure shape).

``Engine`` holds one ``fd3_plan`` (per-species tables, cuFFT plans) and a cached
device workspace allocated through PyTorch's caching allocator; it exposes the two
compute entry points of include/fd3.h:

* ``energy_edges``  -- the reference module surface: energy and its gradients with
  respect to Bohr positions, Bohr shift vectors and the Bohr cell, from a
  caller-supplied edge list (src/fourierd3/core.py:480-583);
* ``energy_forces_stress`` -- the fused calculator path: device cell-list neighbour
  search + CN + C6 factors + SPME/PME + adjoints, returning eV, eV/A, eV/A^3
  (src/fourierd3/calculator.py:125-192).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np
import torch

from fourierd3_b200 import _native, geometry, tables

PBE_BJ = (1.0, 0.7875, 0.4289, 4.4407)   # src/fourierd3/core.py:168


@dataclass
class SpeciesSetup:
    """Species remapping and per-species tables (src/fourierd3/core.py:102-161)."""

    types: tuple           # sorted unique atomic numbers
    species: np.ndarray    # compact ids (N,) int32
    eigs: np.ndarray       # (r,)
    eigvecs: np.ndarray    # (S*7, r)
    rcov: np.ndarray       # (S,) Bohr, float32 values widened (core.py:152)
    cnref: np.ndarray      # (S, 7)
    sqrtq: np.ndarray      # (S,)
    c6_err: float
    rcov_cn: np.ndarray = None   # (S,) D4 CN covalent radii, float32 values widened (pair_pot.py:294)
    en: np.ndarray = None        # (S,) electronegativities (pair_pot.py:301)

    @property
    def n_species(self) -> int:
        return len(self.types)

    @property
    def n_rank(self) -> int:
        return int(self.eigs.shape[0])


def species_setup(numbers: Sequence[int], c6tol: float) -> SpeciesSetup:
    numbers = np.asarray(numbers).astype(np.int64)
    uniq = np.unique(numbers)
    remap = {int(z): i for i, z in enumerate(uniq)}
    species = np.array([remap[int(z)] for z in numbers], dtype=np.int32)
    eigs, vecs, err = tables.species_setup(tuple(int(z) for z in uniq), float(c6tol))
    t = tables.load_tables()
    return SpeciesSetup(
        types=tuple(int(z) for z in uniq), species=species,
        eigs=np.ascontiguousarray(eigs, dtype=np.float64),
        eigvecs=np.ascontiguousarray(vecs, dtype=np.float64),
        rcov=t["rcov"][uniq].astype(np.float64), cnref=t["cnref"][uniq].astype(np.float64),
        sqrtq=t["sqrtQz"][uniq].astype(np.float64), c6_err=float(err),
        rcov_cn=t["rcov_cn"][uniq].astype(np.float64), en=t["en"][uniq].astype(np.float64))


def _stream_ptr(device: torch.device) -> int:
    return torch.cuda.current_stream(device).cuda_stream


class Engine:
    """One fd3 plan for a fixed species set, method, mesh and precision."""

    def __init__(self, setup: SpeciesSetup, *, method: str, order: int, mesh: Sequence[int],
                 ewald_ns: Sequence[int] = (0, 0, 0), precision: str = "fp64", r_cut_bohr: float,
                 params: Sequence[float] = PBE_BJ, cncorr: Optional[np.ndarray] = None,
                 cnfunc: str = "smooth_cut", device: torch.device):
        if device.type != "cuda":
            raise RuntimeError("fourierd3_b200 computes on CUDA devices only (B200, sm_100a)")
        if method not in _native.METHODS:
            raise ValueError(f"unknown method {method!r}; expected 'spme', 'pme' or 'ewald'")
        if precision not in ("fp64", "mixed"):
            raise ValueError("precision must be 'fp64' or 'mixed'")
        if cnfunc not in _native.CNFUNCS:
            raise ValueError(f"Unknown cnfunc '{cnfunc}'. Expected 'smooth_cut' or 'd4'.")
        if cnfunc == "d4" and (method == "ewald" or setup.n_species > 8):
            raise NotImplementedError(
                "cnfunc='d4' is built for the mesh methods ('spme', 'pme') with at most 8 species; the reference's "
                "own Ewald branch of the D4 CN reads an attribute it never defines (src/fourierd3/core.py:436)")
        self.cnfunc = cnfunc
        self.setup = setup
        self.method = method
        self.order = int(order)
        self.mesh = tuple(int(v) for v in mesh)
        self.precision = precision
        self.device = device
        self._keep = []  # numpy arrays referenced by the descriptor until create returns
        d = _native.PlanDesc()
        d.n_species = setup.n_species
        d.n_rank = setup.n_rank
        d.method = _native.METHODS[method]
        d.order = self.order
        for a in range(3):
            d.mesh[a] = self.mesh[a]
            d.ewald_ns[a] = int(ewald_ns[a])
        d.precision = _native.PREC_FP64 if precision == "fp64" else _native.PREC_MIXED
        d.r_cut = float(r_cut_bohr)
        for k in range(4):
            d.params[k] = float(params[k])

        def keep(a, dt=np.float64):
            a = np.ascontiguousarray(a, dtype=dt)
            self._keep.append(a)
            return a

        d.rcov = _native.dptr(keep(setup.rcov))
        d.cnref = _native.dptr(keep(setup.cnref))
        d.eigvecs = _native.dptr(keep(setup.eigvecs))
        d.eigs = _native.dptr(keep(setup.eigs))
        d.sqrtq = _native.dptr(keep(setup.sqrtq))
        if cncorr is not None:
            d.has_cncorr = 1
            d.cncorr = _native.dptr(keep(np.asarray(cncorr, dtype=np.float64).reshape(-1, 2)))
        d.cnfunc = _native.CNFUNCS[cnfunc]
        if cnfunc == "d4":
            d.rcov_cn = _native.dptr(keep(setup.rcov_cn))
            d.en = _native.dptr(keep(setup.en))
        if method == "spme":
            win = keep(geometry.spme_window(self.mesh, self.order), np.float32)
            d.deconv = win.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
        self._plan = ctypes.c_void_p()
        lib = _native.lib()
        with torch.cuda.device(device):
            _native.check(lib.fd3_plan_create(ctypes.byref(d), ctypes.byref(self._plan)), "fd3_plan_create")
        self._keep = []
        self._work = None
        self._species_dev = None

    def __del__(self):
        plan = getattr(self, "_plan", None)
        if plan is not None and plan.value:
            try:
                _native.lib().fd3_plan_destroy(plan)
            except Exception:
                pass

    # ------------------------------------------------------------------ helpers
    def species_tensor(self) -> torch.Tensor:
        if self._species_dev is None:
            self._species_dev = torch.as_tensor(self.setup.species, dtype=torch.int32, device=self.device)
        return self._species_dev

    def workspace(self, n_atoms: int, n_bins: int) -> torch.Tensor:
        nbytes = ctypes.c_size_t()
        _native.check(_native.lib().fd3_workspace_size(self._plan, n_atoms, n_bins, ctypes.byref(nbytes)),
                      "fd3_workspace_size")
        if self._work is None or self._work.numel() < nbytes.value:
            self._work = torch.empty(int(nbytes.value), dtype=torch.uint8, device=self.device)
        return self._work

    def edge_workspace(self, n_atoms: int, n_edges: int) -> torch.Tensor:
        """Workspace of the edge-list entry point (grown, never shrunk, so a fixed edge count
        keeps every pointer fixed, e.g. across CUDA-graph replays)."""
        nbytes = ctypes.c_size_t()
        _native.check(_native.lib().fd3_edge_workspace_size(self._plan, n_atoms, n_edges, ctypes.byref(nbytes)),
                      "fd3_edge_workspace_size")
        if self._work is None or self._work.numel() < nbytes.value:
            self._work = torch.empty(int(nbytes.value), dtype=torch.uint8, device=self.device)
        return self._work

    def workspace_bytes(self, n_atoms: int, cell_ang: np.ndarray, r_cut_ang: float) -> int:
        """Bytes of device workspace one fused call on this structure shape needs."""
        nb, _ = self.cell_grid(cell_ang, r_cut_ang)
        nbytes = ctypes.c_size_t()
        _native.check(_native.lib().fd3_workspace_size(self._plan, n_atoms, nb[0] * nb[1] * nb[2],
                                                       ctypes.byref(nbytes)), "fd3_workspace_size")
        return int(nbytes.value)

    @staticmethod
    def cell_grid(cell_ang: np.ndarray, r_cut_ang: float):
        c = np.ascontiguousarray(cell_ang, dtype=np.float64).reshape(9)
        nb = (ctypes.c_int32 * 3)()
        rr = (ctypes.c_int32 * 3)()
        _native.check(_native.lib().fd3_cell_grid(_native.dptr(c), float(r_cut_ang), nb, rr), "fd3_cell_grid")
        return tuple(nb), tuple(rr)

    _KNOBS = {"filter_kt": _native.TUNE_FILTER_KT, "spread_zc": _native.TUNE_SPREAD_ZC,
              "spread_cap": _native.TUNE_SPREAD_CAP, "fft_x": _native.TUNE_FFT_X,
              "xpencil": _native.TUNE_XPENCIL, "xq": _native.TUNE_XQ, "xranks": _native.TUNE_XRANKS,
              "filter_mma": _native.TUNE_FILTER_MMA, "gather_tile": _native.TUNE_GATHER_TILE,
              "fft_yz": _native.TUNE_FFT_YZ}

    def set_tuning(self, filter_kt: Optional[int] = None, spread_zc: Optional[int] = None,
                   spread_cap: Optional[int] = None, fft_x: Optional[int] = None,
                   xpencil: Optional[int] = None, xq: Optional[int] = None,
                   xranks: Optional[int] = None, filter_mma: Optional[int] = None,
                   gather_tile: Optional[int] = None, fft_yz: Optional[int] = None) -> None:
        """Launch-shape knobs (results agree to rounding): ``filter_kt`` = k-points per filter
        tile, ``spread_zc`` = z-tiles per column chunk of the spread, ``spread_cap`` = staged
        atoms per chunk at most, ``fft_x`` = 0 (3D cuFFT around the filter), 1 (2D cuFFT and the
        x FFT / filter / inverse x FFT in one kernel, pencils of ``xpencil`` = 1, 2 or 4 kz values
        of every channel) or 2 (the same with TMA-moved units of ``xq`` = 4, 8, 16 or 32
        flattened (y, kz) values of ``xranks`` = 1, 2 or 4 ranks, mixed precision),
        ``filter_mma`` = 1 (mixed precision: the per-k-point species products of the separate
        filter on the tensor cores) or 0 (CUDA cores), ``gather_tile`` = 1 (one CTA per mesh
        tile and species stages the tile's potential box once by TMA) or 0 (warp per atom reading
        the mesh directly), ``fft_yz`` = 1 or 2 (mixed precision, x-pass paths, ny = nz = 256:
        the (y, z) plane transforms by this library's cluster kernels, one pass each way, the
        forward on clusters of 2 or 4 CTAs; the default) or 0 (cuFFT); -1 (0 for the cap)
        restores a default."""
        for name, val in (("filter_kt", filter_kt), ("spread_zc", spread_zc), ("spread_cap", spread_cap),
                          ("fft_x", fft_x), ("xpencil", xpencil), ("xq", xq), ("xranks", xranks),
                          ("filter_mma", filter_mma), ("gather_tile", gather_tile), ("fft_yz", fft_yz)):
            if val is not None:
                _native.check(_native.lib().fd3_plan_set_tuning(self._plan, self._KNOBS[name], int(val)),
                              "fd3_plan_set_tuning")

    def tuning(self) -> dict:
        out = {}
        for name, knob in self._KNOBS.items():
            v = ctypes.c_int32()
            _native.check(_native.lib().fd3_plan_get_tuning(self._plan, knob, ctypes.byref(v)), "fd3_plan_get_tuning")
            out[name] = int(v.value)
        return out

    def set_edge_cutoff(self, on: bool) -> None:
        """Edge-list path: edges at or beyond the CN cutoff contribute nothing (a Verlet list
        with a skin can then be passed unchanged between rebuilds)."""
        _native.check(_native.lib().fd3_plan_set_edge_cutoff(self._plan, 1 if on else 0), "fd3_plan_set_edge_cutoff")

    def atom_terms(self, n_atoms: int,cell_ang: Optional[np.ndarray] = None, r_cut_ang: float = 0.0,
                   work: Optional[torch.Tensor] = None):
        """Per-atom CN (after cncorr) and rank-r C6 factors (n_atoms, r) of the last call that used
        this engine's workspace (or ``work``): the fused call when ``cell_ang`` is given, the
        edge-list call otherwise (src/fourierd3/core.py:323-386, 449-478, 525-532)."""
        nbins = 0
        if cell_ang is not None:
            nb, _ = self.cell_grid(cell_ang, r_cut_ang)
            nbins = nb[0] * nb[1] * nb[2]
        work = self._work if work is None else work
        if work is None:
            raise RuntimeError("atom_terms: no compute call has used this engine's workspace yet")
        cn = torch.empty(n_atoms, dtype=torch.float64, device=self.device)
        c6 = torch.empty((n_atoms, self.setup.n_rank), dtype=torch.float64, device=self.device)
        _native.check(_native.lib().fd3_atom_terms(self._plan, n_atoms, nbins, ctypes.c_void_p(work.data_ptr()),
                                                   work.numel(), ctypes.c_void_p(cn.data_ptr()),
                                                   ctypes.c_void_p(c6.data_ptr()),
                                                   ctypes.c_void_p(_stream_ptr(self.device))), "fd3_atom_terms")
        return cn, c6

    def profile(self, on: bool = True) -> None:
        """Record CUDA events between pipeline stages of the following calls."""
        _native.check(_native.lib().fd3_profile_enable(self._plan, 1 if on else 0), "fd3_profile_enable")

    def stage_times(self) -> dict:
        """{stage name: milliseconds} of the last call (waits for its last event)."""
        ms = (ctypes.c_double * 24)()
        names = ctypes.create_string_buffer(512)
        n = ctypes.c_int32()
        _native.check(_native.lib().fd3_profile_read(self._plan, ms, 24, names, 512, ctypes.byref(n)),
                      "fd3_profile_read")
        keys = names.value.decode().split(",") if n.value else []
        out: dict = {}
        for k, v in zip(keys, list(ms)[: n.value]):
            out[k] = out.get(k, 0.0) + v
        return out

    # ------------------------------------------------------------------ entry points
    def energy_edges(self, pos_b: torch.Tensor, cell_b: torch.Tensor, edge_index: torch.Tensor,
                     shifts_b: torch.Tensor, need_grad: bool):
        """Returns (energy [Ha], dE/dpos, dE/dshift, dE/dcell) -- gradients None if not need_grad."""
        n = pos_b.shape[0]
        e = edge_index.shape[1]
        pos = pos_b.detach().to(torch.float64).contiguous()
        cell = cell_b.detach().to(torch.float64).contiguous()
        sh = shifts_b.detach().to(torch.float64).contiguous()
        ei = edge_index.to(torch.int64).contiguous()
        src, dst = ei[0], ei[1]
        work = self.edge_workspace(n, e)
        # torch.ops.fd3.energy_edges: the operator layer over fd3_energy_edges (current stream)
        energy, gpos, gsh, gcell = _native.ops().energy_edges(
            _native.handle(self._plan), pos, self.species_tensor(), cell, src.contiguous(), dst.contiguous(), sh,
            bool(need_grad), work)
        if not need_grad:
            return energy, None, None, None
        return energy, gpos, gsh, gcell

    def energy_forces_stress(self, pos_ang: torch.Tensor, cell_ang: np.ndarray, r_cut_ang: float,
                             cell_dev: Optional[torch.Tensor] = None, out=None,
                             species: Optional[torch.Tensor] = None, work: Optional[torch.Tensor] = None):
        """Fused path. Returns (energy [eV], forces [eV/A], stress [eV/A^3] 3x3).

        ``species`` (int32 compact ids on the device) and ``work`` (a uint8 device buffer of
        at least ``workspace_bytes``) let a caller that owns its buffers -- the batch runner,
        a captured CUDA graph -- keep every pointer fixed; by default the engine's own are used.
        """
        n = pos_ang.shape[0]
        cell_h = np.ascontiguousarray(cell_ang, dtype=np.float64).reshape(9)
        if work is None:
            (nb, _) = self.cell_grid(cell_h, r_cut_ang)
            work = self.workspace(n, nb[0] * nb[1] * nb[2])
        if species is None:
            species = self.species_tensor()
        if out is None:
            # torch.ops.fd3.energy_forces_stress: the operator layer over fd3_energy_forces_stress
            return _native.ops().energy_forces_stress(
                _native.handle(self._plan), pos_ang, species, torch.from_numpy(cell_h.reshape(3, 3).copy()),
                float(r_cut_ang), work, cell_dev)
        # caller-owned outputs (the batch runner's packed buffers, fixed across graph replays):
        # the C ABI directly
        if cell_dev is None:
            cell_dev = torch.as_tensor(cell_h, dtype=torch.float64).to(self.device, non_blocking=False)
        energy, forces, stress = out
        rc = _native.lib().fd3_energy_forces_stress(
            self._plan, n, ctypes.c_void_p(pos_ang.data_ptr()), ctypes.c_void_p(species.data_ptr()),
            _native.dptr(cell_h), ctypes.c_void_p(cell_dev.data_ptr()), float(r_cut_ang),
            ctypes.c_void_p(work.data_ptr()), work.numel(), ctypes.c_void_p(energy.data_ptr()),
            ctypes.c_void_p(forces.data_ptr()), ctypes.c_void_p(stress.data_ptr()),
            ctypes.c_void_p(_stream_ptr(self.device)))
        _native.check(rc, "fd3_energy_forces_stress")
        return energy, forces, stress

    def direct_energy_forces_stress(self, pos_ang: torch.Tensor, cell_ang: np.ndarray, r_cut_ang: float,
                                    r_direct_ang: float = 25.0):
        """Direct pairwise D3(BJ) lattice sum in float64 (the accuracy oracle of the mesh methods,
        on the device): every image pair closer than ``r_direct_ang`` plus the continuum tail,
        with this plan's CN and C6 factors. Returns (energy [eV], forces [eV/A], stress [eV/A^3])."""
        n = pos_ang.shape[0]
        cell_h = np.ascontiguousarray(cell_ang, dtype=np.float64).reshape(9)
        nbytes = ctypes.c_size_t()
        _native.check(_native.lib().fd3_direct_workspace_size(self._plan, n, _native.dptr(cell_h), float(r_cut_ang),
                                                              float(r_direct_ang), ctypes.byref(nbytes)),
                      "fd3_direct_workspace_size")
        work = torch.empty(int(nbytes.value), dtype=torch.uint8, device=self.device)
        species = self.species_tensor()
        cell_dev = torch.as_tensor(cell_h, dtype=torch.float64).to(self.device)
        energy = torch.empty((), dtype=torch.float64, device=self.device)
        forces = torch.empty((n, 3), dtype=torch.float64, device=self.device)
        stress = torch.empty((3, 3), dtype=torch.float64, device=self.device)
        pos = pos_ang.to(device=self.device, dtype=torch.float64).contiguous()
        rc = _native.lib().fd3_direct_energy_forces_stress(
            self._plan, n, ctypes.c_void_p(pos.data_ptr()), ctypes.c_void_p(species.data_ptr()),
            _native.dptr(cell_h), ctypes.c_void_p(cell_dev.data_ptr()), float(r_cut_ang), float(r_direct_ang),
            ctypes.c_void_p(work.data_ptr()), work.numel(), ctypes.c_void_p(energy.data_ptr()),
            ctypes.c_void_p(forces.data_ptr()), ctypes.c_void_p(stress.data_ptr()),
            ctypes.c_void_p(_stream_ptr(self.device)))
        _native.check(rc, "fd3_direct_energy_forces_stress")
        return energy, forces, stress


def neighbour_list(positions: torch.Tensor, cell_ang: np.ndarray, r_cut: float):
    """GPU replacement of matscipy ``neighbour_list("ijS")`` (calculator.py:94-123).

    Returns (i, j, S) device tensors (int64, int64, int32 (E, 3)), rows sorted by i.
    """
    if positions.device.type != "cuda":
        raise RuntimeError("neighbour_list runs on CUDA devices only")
    lib = _native.lib()
    pos = positions.detach().to(torch.float64).contiguous()
    n = pos.shape[0]
    cell_h = np.ascontiguousarray(cell_ang, dtype=np.float64).reshape(9)
    nbytes = ctypes.c_size_t()
    _native.check(lib.fd3_neighbor_workspace_size(n, _native.dptr(cell_h), float(r_cut), ctypes.byref(nbytes)),
                  "fd3_neighbor_workspace_size")
    work = torch.empty(int(nbytes.value), dtype=torch.uint8, device=pos.device)
    stream = ctypes.c_void_p(_stream_ptr(pos.device))
    count = ctypes.c_int64()
    _native.check(lib.fd3_neighbor_count(n, ctypes.c_void_p(pos.data_ptr()), _native.dptr(cell_h), float(r_cut),
                                         ctypes.c_void_p(work.data_ptr()), work.numel(), ctypes.byref(count), stream),
                  "fd3_neighbor_count")
    cap = int(count.value)
    src = torch.empty(max(cap, 1), dtype=torch.int64, device=pos.device)
    dst = torch.empty(max(cap, 1), dtype=torch.int64, device=pos.device)
    sh = torch.empty((max(cap, 1), 3), dtype=torch.int32, device=pos.device)
    _native.check(lib.fd3_neighbor_fill(n, ctypes.c_void_p(pos.data_ptr()), _native.dptr(cell_h), float(r_cut),
                                        ctypes.c_void_p(work.data_ptr()), work.numel(), cap,
                                        ctypes.c_void_p(src.data_ptr()), ctypes.c_void_p(dst.data_ptr()),
                                        ctypes.c_void_p(sh.data_ptr()), ctypes.byref(count), stream),
                  "fd3_neighbor_fill")
    m = int(count.value)
    return src[:m], dst[:m], sh[:m]
