"""Batched evaluation of many independent periodic structures, optionally as one CUDA graph.

``D3Batch`` takes a list of structures (positions [A], cell [A], atomic numbers) of uneven
atom counts, cells and mesh sizes and evaluates energy, forces and stress for all of them
in one call -- the batched form of ``FourierD3ASECalculator.calculate``
(src/fourierd3/calculator.py:125-192) applied to each structure independently.

Layout on the device:

* one packed positions buffer (sum N, 3) float64 and packed compact species ids; the
  caller updates positions in place (``positions_view`` / ``set_positions``) between calls;
* packed outputs: energy (B,), forces (sum N, 3), stress (B, 3, 3);
* structures are split over ``lanes`` CUDA streams by a longest-processing-time rule on
  the cost model N + M * S * r (atoms + mesh points x channels); each lane owns ONE
  workspace buffer sized for the largest structure on that lane and runs its structures
  back to back, so the device memory held is the sum over lanes of the lane maxima, not
  the sum over all structures (with 54 species the mesh channels of a 256-structure batch
  add up to hundreds of GB);
* plans (species tables, cuFFT plans) are shared by structures with the same species
  set, method, mesh and Ewald box.

``capture()`` records every lane's launches into one ``torch.cuda.CUDAGraph`` (fork/join
over the lane streams), after which a call is a single graph replay. The cells are fixed
for the life of a capture (they set the cell-list grid and the mesh).

From host memory to host memory: ``run_host`` replays one graph with the copy of the
positions in and of the results out inside it (one evaluation at a time);
``host_pipeline()`` keeps two evaluations in flight, each slot with its own pinned and
device buffers and graph, so the copies of one run on copy streams beside the other's compute.

``autotune_filter`` and ``autotune_spread`` time the filter k-tile and the spread z-chunk on
the heaviest structures; ``autotune_lanes`` times candidate lane counts under graph replay and
caches the winner in a JSON file keyed by the batch's shape signature.
"""
from __future__ import annotations

import gc
import hashlib
import json
import os
import time
from typing import List, Optional, Sequence, Tuple

import numpy as np
import torch

from fourierd3_b200 import engine as _engine
from fourierd3_b200 import geometry

_ALIGN = 256


def _mesh_and_box(cell_ang, method: str, mesh_spacing: float, k_cutoff: float):
    cell_b = np.asarray(cell_ang, dtype=np.float64) * geometry.ANGSTROM_TO_BOHR
    if method in ("spme", "pme"):
        return geometry.ns_mesh(cell_b, mesh_spacing * geometry.ANGSTROM_TO_BOHR), (0, 0, 0)
    return (1, 1, 1), geometry.ewald_ns(cell_b, k_cutoff)


def structure_cost(numbers, cell_ang, *, method: str = "spme", mesh_spacing: float = 1.2,
                   k_cutoff: float = 10.0, c6tol: float = 1.0) -> float:
    """Cost model N + M * S * r used to balance lanes and ranks."""
    setup = _engine.species_setup(np.asarray(numbers), c6tol)
    mesh, ens = _mesh_and_box(cell_ang, method, mesh_spacing, k_cutoff)
    m = mesh[0] * mesh[1] * mesh[2] if method in ("spme", "pme") else ens[0] * ens[1] * ens[2]
    return float(len(numbers) + m * setup.n_species * setup.n_rank)


def lpt_split(costs: Sequence[float], parts: int) -> List[List[int]]:
    """Longest-processing-time assignment of items to ``parts`` bins (heaviest first)."""
    bins: List[List[int]] = [[] for _ in range(parts)]
    load = [0.0] * parts
    for i in sorted(range(len(costs)), key=lambda k: (-costs[k], k)):
        b = min(range(parts), key=lambda q: (load[q], q))
        bins[b].append(i)
        load[b] += costs[i]
    return bins


def shard(structures: Sequence, rank: int, world: int, **cost_kw) -> List[int]:
    """Indices of the structures rank ``rank`` of ``world`` evaluates (LPT on the cost model)."""
    if not 0 <= rank < world:
        raise ValueError("rank must be in [0, world)")
    costs = [structure_cost(z, c, **cost_kw) for (_, c, z) in structures]
    return sorted(lpt_split(costs, world)[rank])


class D3Batch:
    """Energy, forces and stress of B independent structures per call."""

    def __init__(self, structures: Sequence[Tuple[np.ndarray, np.ndarray, np.ndarray]], *,
                 method: str = "spme", mesh_spacing: float = 1.2, interpolation_nodes: int = 5,
                 c6tol: float = 1.0, params=None, r_cut: float = 6.0, k_cutoff: float = 10.0,
                 precision: str = "mixed", lanes: int = 1, device: Optional[torch.device] = None):
        if len(structures) == 0:
            raise ValueError("empty batch")
        self.device = torch.device(device) if device is not None else torch.device("cuda")
        if self.device.type != "cuda":
            raise RuntimeError("fourierd3_b200 computes on CUDA devices only (B200, sm_100a)")
        if self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        self.r_cut = float(r_cut)
        self.method = method
        self.precision = precision
        self.n_struct = len(structures)
        self._engines: dict = {}
        self._graph = None
        self._graph_host = None
        self._pipe = None
        counts, cells, species, setups, keys, costs = [], [], [], [], [], []
        for pos, cell, numbers in structures:
            pos = np.asarray(pos, dtype=np.float64)
            numbers = np.asarray(numbers)
            cell = np.asarray(cell, dtype=np.float64)
            if pos.ndim != 2 or pos.shape[1] != 3 or pos.shape[0] != numbers.shape[0] or pos.shape[0] < 1:
                raise ValueError("each structure needs positions (N, 3) and N atomic numbers, N >= 1")
            if cell.shape != (3, 3):
                raise ValueError("each cell must be 3x3")
            setup = _engine.species_setup(numbers, c6tol)
            mesh, ens = _mesh_and_box(cell, method, mesh_spacing, k_cutoff)
            key = (setup.types, mesh, ens)
            if key not in self._engines:
                self._engines[key] = _engine.Engine(
                    setup, method=method, order=interpolation_nodes, mesh=mesh, ewald_ns=ens,
                    precision=precision, r_cut_bohr=self.r_cut * geometry.ANGSTROM_TO_BOHR,
                    params=params if params is not None else _engine.PBE_BJ, device=self.device)
            counts.append(pos.shape[0])
            cells.append(cell)
            species.append(setup.species)
            setups.append(setup)
            keys.append(key)
            m = mesh[0] * mesh[1] * mesh[2] if method in ("spme", "pme") else ens[0] * ens[1] * ens[2]
            costs.append(float(pos.shape[0] + m * setup.n_species * setup.n_rank))
        self.counts = counts
        self.costs = costs
        self.offsets = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
        total = int(self.offsets[-1])
        dev = self.device
        self.positions = torch.empty((total, 3), dtype=torch.float64, device=dev)
        self.positions.copy_(torch.from_numpy(np.concatenate([np.asarray(p, dtype=np.float64)
                                                              for p, _, _ in structures])))
        self.species = torch.from_numpy(np.concatenate(species).astype(np.int32)).to(dev)
        self.cells_host = np.stack(cells)
        self.cells = torch.from_numpy(self.cells_host.reshape(-1, 9).copy()).to(dev)
        # one flat output buffer [energy (B) | stress (B, 3, 3) | forces (N, 3)] so that a host
        # read of every result is a single copy
        B = self.n_struct
        self._out = torch.zeros(10 * B + 3 * total, dtype=torch.float64, device=dev)
        self.energy = self._out[:B]
        self.stress = self._out[B:10 * B].view(B, 3, 3)
        self.forces = self._out[10 * B:].view(total, 3)
        self._host = None   # pinned host buffers of the host-I/O graph (positions, outputs)
        self._keys = keys
        self._need = [self._engines[k].workspace_bytes(counts[i], cells[i], self.r_cut)
                      for i, k in enumerate(keys)]
        self.lanes = 0
        self.set_lanes(lanes)

    # ------------------------------------------------------------------ lanes
    def set_lanes(self, lanes: int) -> None:
        """Split the structures over ``lanes`` streams, each with one workspace (drops a capture)."""
        lanes = max(1, min(int(lanes), self.n_struct))
        if lanes == self.lanes:
            return
        self.drop_captures()
        self._work = None
        torch.cuda.synchronize(self.device)
        split = lpt_split(self.costs, lanes)
        self.lane_of = np.zeros(self.n_struct, dtype=np.int64)
        for q, items in enumerate(split):
            self.lane_of[items] = q
        sizes = [max(self._need[i] for i in items) if items else 0 for items in split]
        self.workspace_bytes = int(sum(-(-s // _ALIGN) * _ALIGN for s in sizes))
        self._work = torch.empty(max(self.workspace_bytes, 1), dtype=torch.uint8, device=self.device)
        self._streams = [torch.cuda.Stream(self.device) for _ in range(lanes)]
        self._lane_items = []
        base = 0
        for q, items in enumerate(split):
            wsl = self._work[base: base + sizes[q]]
            base += -(-sizes[q] // _ALIGN) * _ALIGN
            # heaviest first inside a lane as well: the long mesh stages start early
            self._lane_items.append((sorted(items, key=lambda k: (-self.costs[k], k)), wsl))
        self._lane_calls = self._make_lane_calls(self.positions, self._out)
        self._pipe = None
        self.lanes = lanes

    def _make_lane_calls(self, positions: torch.Tensor, out: torch.Tensor) -> list:
        """Per lane, the engine calls of its structures reading ``positions`` (sum N, 3) and
        writing the packed result buffer ``out`` [energy (B) | stress (B, 3, 3) | forces (sum N, 3)]."""
        B = self.n_struct
        energy, stress = out[:B], out[B:10 * B].view(B, 3, 3)
        forces = out[10 * B:].view(-1, 3)
        lane_calls = []
        for items, wsl in self._lane_items:
            calls = []
            for i in items:
                a, b = int(self.offsets[i]), int(self.offsets[i + 1])
                calls.append((self._engines[self._keys[i]], positions[a:b], self.cells_host[i],
                              self.cells[i], (energy[i], forces[a:b], stress[i]),
                              self.species[a:b], wsl))
            lane_calls.append(calls)
        return lane_calls

    def _launch_all(self, lane_calls: Optional[list] = None) -> None:
        main = torch.cuda.current_stream(self.device)
        fork = torch.cuda.Event()
        fork.record(main)
        joins = []
        for st, calls in zip(self._streams, self._lane_calls if lane_calls is None else lane_calls):
            st.wait_event(fork)
            with torch.cuda.stream(st):
                for eng, pos, cell_h, cell_d, out, spc, wsl in calls:
                    eng.energy_forces_stress(pos, cell_h, self.r_cut, cell_dev=cell_d, out=out,
                                             species=spc, work=wsl)
                ev = torch.cuda.Event()
                ev.record(st)
            joins.append(ev)
        for ev in joins:
            main.wait_event(ev)

    # ------------------------------------------------------------------ graph
    def capture(self, host_io: bool = False) -> None:
        """Record the whole batch (all lanes) as one CUDA graph; later calls replay it.

        host_io: record a second graph (replayed by ``run_host``) that also copies the positions in from the pinned host buffer of
        ``host_buffers()`` and every result out to it (one copy each way), so that one replay
        (``run_host``) is a whole evaluation from host memory to host memory."""
        if host_io:
            self.host_buffers()
            g = self._record(None, copy_in=(self.positions, self._host["pos"]),
                             copy_out=(self._host["out"], self._out))
            self._graph_host = g
        else:
            self._graph = self._record(None)

    def _record(self, lane_calls: Optional[list], copy_in=None, copy_out=None) -> torch.cuda.CUDAGraph:
        """One CUDA graph of ``lane_calls`` (default: the batch's own buffers), optionally with a
        copy (dst, src) before and after the launches."""
        side = torch.cuda.Stream(self.device)
        side.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(side):
            self._launch_all(lane_calls)  # warm-up outside the capture: cuFFT and module loading
        torch.cuda.current_stream(self.device).wait_stream(side)
        torch.cuda.synchronize(self.device)
        # a graph that dies in an unreachable cycle must not be freed by the cycle collector while
        # this capture runs (destroying a graph during a capture invalidates the capture)
        gc.collect()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            if copy_in is not None:
                copy_in[0].copy_(copy_in[1], non_blocking=True)
            self._launch_all(lane_calls)
            if copy_out is not None:
                copy_out[0].copy_(copy_out[1], non_blocking=True)
        torch.cuda.synchronize(self.device)
        return g

    def host_buffers(self) -> dict:
        """Pinned host buffers for host-to-host evaluation: ``positions`` (sum N, 3) read by the
        host-I/O graph, and ``energy`` (B,), ``stress`` (B, 3, 3), ``forces`` (sum N, 3) that it
        writes (views of one pinned buffer)."""
        if self._host is None:
            self._host = self._pinned_io()
        return self._host

    def _pinned_io(self) -> dict:
        pos = torch.empty(tuple(self.positions.shape), dtype=torch.float64).pin_memory()
        pos.copy_(self.positions.cpu())
        out = torch.zeros(self._out.shape, dtype=torch.float64).pin_memory()
        B, total = self.n_struct, int(self.positions.shape[0])
        return {"pos": pos, "out": out, "positions": pos, "energy": out[:B],
                "stress": out[B:10 * B].view(B, 3, 3), "forces": out[10 * B:].view(total, 3)}

    def run_host(self):
        """One evaluation from the pinned host positions to the pinned host results (a single
        graph replay with both copies inside; captures with host_io=True first if needed). The
        results are valid once the current stream has been synchronised. Returns the host
        (energy, forces, stress) views."""
        if getattr(self, "_graph_host", None) is None:
            self.capture(host_io=True)
        self._graph_host.replay()
        h = self._host
        return h["energy"], h["forces"], h["stress"]

    def host_pipeline(self) -> "HostPipeline":
        """The batch's two-slot host-to-host pipeline (created on first use; see ``HostPipeline``)."""
        if self._pipe is None:
            self._pipe = HostPipeline(self)
        return self._pipe

    def drop_captures(self) -> None:
        """Forget every captured graph (after a change of lanes or launch knobs)."""
        self._graph = None
        self._graph_host = None
        self._pipe = None

    @property
    def captured(self) -> bool:
        return self._graph is not None

    # ------------------------------------------------------------------ calls
    def positions_view(self, i: int) -> torch.Tensor:
        a, b = int(self.offsets[i]), int(self.offsets[i + 1])
        return self.positions[a:b]

    def set_positions(self, positions) -> None:
        """Copy new positions in: a packed (sum N, 3) tensor or a list of (N_i, 3) arrays."""
        if isinstance(positions, (list, tuple)):
            if len(positions) != self.n_struct:
                raise ValueError("one positions array per structure expected")
            for i, p in enumerate(positions):
                t = torch.as_tensor(p, dtype=torch.float64)
                if tuple(t.shape) != (self.counts[i], 3):
                    raise ValueError(f"structure {i}: positions must be ({self.counts[i]}, 3)")
                self.positions_view(i).copy_(t, non_blocking=True)
        else:
            t = torch.as_tensor(positions, dtype=torch.float64)
            if tuple(t.shape) != tuple(self.positions.shape):
                raise ValueError(f"packed positions must be {tuple(self.positions.shape)}")
            self.positions.copy_(t, non_blocking=True)

    def __call__(self, positions=None):
        """(energy [eV] (B,), forces [eV/A] (sum N, 3), stress [eV/A^3] (B, 3, 3)) on the device.

        The returned tensors are the batch's static output buffers: the next call overwrites them.
        """
        if positions is not None:
            self.set_positions(positions)
        if self._graph is not None:
            self._graph.replay()
        else:
            self._launch_all()
        return self.energy, self.forces, self.stress

    def split_forces(self, forces: Optional[torch.Tensor] = None) -> List[torch.Tensor]:
        f = self.forces if forces is None else forces
        return [f[int(self.offsets[i]): int(self.offsets[i + 1])] for i in range(self.n_struct)]

    # ------------------------------------------------------------------ autotuning
    def signature(self) -> str:
        h = hashlib.sha1()
        h.update(json.dumps([self.method, self.precision, self.r_cut]).encode())
        for i in range(self.n_struct):
            k = self._keys[i]
            h.update(json.dumps([self.counts[i], list(k[0]), list(k[1]), list(k[2])]).encode())
        dev = torch.cuda.get_device_properties(self.device)
        h.update(f"{dev.name}:{dev.multi_processor_count}".encode())
        return h.hexdigest()[:20]

    def time_replays(self, reps: int = 3) -> float:
        """Milliseconds per graph replay (captures first if needed), median of ``reps``."""
        if self._graph is None:
            self.capture()
        st = torch.cuda.current_stream(self.device)
        times = []
        for _ in range(reps):
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(st)
            self._graph.replay()
            b.record(st)
            b.synchronize()
            times.append(a.elapsed_time(b))
        return float(np.median(times))


class HostPipeline:
    """Host-to-host evaluations of a ``D3Batch`` with two in flight, so that the PCIe copies of
    one evaluation overlap the compute of the other (the copy engines and the SMs work at once).

    Slot s (0 or 1) owns pinned host buffers ``host[s]`` (``positions`` (sum N, 3) read;
    ``energy`` (B,), ``stress`` (B, 3, 3), ``forces`` (sum N, 3) written), device copies of the
    positions and of the packed results, and a CUDA graph of the whole batch on those device
    buffers. Both graphs share the batch's workspace, so the evaluations themselves run one after
    another on the submitting stream; only the copies run beside them, on two copy streams.

    ``submit(s)`` enqueues the host-to-device copy of slot s's positions, the slot's graph and the
    device-to-host copy of its results, and returns at once. ``wait(s)`` blocks until the results
    of slot s's last submission are in host memory; after it the caller may read them and write
    the slot's next positions. A stream of evaluations alternates the slots::

        for k, positions in enumerate(stream):
            s = k % 2
            pipe.wait(s)             # results of evaluation k - 2 are now in pipe.host[s]
            pipe.host[s]["positions"].copy_(positions)
            pipe.submit(s)

    Cells, species, lanes and launch knobs are the batch's; changing any of them drops the
    pipeline with the batch's other captures.
    """

    def __init__(self, batch: D3Batch):
        # no reference back to the batch: a batch <-> pipeline cycle would leave the graphs to
        # the cycle collector, which may free them in the middle of a later capture
        self.device = dev = batch.device
        # ... but the memory its graphs read stays alive with the pipeline: the workspace, the
        # species and cells, and the plans (none of them refers to the batch)
        self._keep = (batch._work, batch.species, batch.cells, dict(batch._engines))
        self.host = [batch._pinned_io() for _ in range(2)]
        self.dev_pos = [batch.positions.clone() for _ in range(2)]
        self.dev_out = [torch.zeros_like(batch._out) for _ in range(2)]
        self.h2d_bytes = int(batch.positions.numel()) * 8
        self.d2h_bytes = int(batch._out.numel()) * 8
        self.graphs = [batch._record(batch._make_lane_calls(self.dev_pos[s], self.dev_out[s]))
                       for s in range(2)]
        self.h2d = torch.cuda.Stream(dev)
        self.d2h = torch.cuda.Stream(dev)
        self._in_done = [torch.cuda.Event() for _ in range(2)]
        self._computed = [torch.cuda.Event() for _ in range(2)]
        self._out_done = [torch.cuda.Event() for _ in range(2)]

    def submit(self, s: int) -> None:
        """Enqueue one evaluation of slot ``s`` from ``host[s]["positions"]`` to ``host[s]``'s results."""
        if s not in (0, 1):
            raise ValueError("slot must be 0 or 1")
        main = torch.cuda.current_stream(self.device)
        # the slot's device positions are rewritten only once its previous evaluation has read them
        self.h2d.wait_event(self._computed[s])
        with torch.cuda.stream(self.h2d):
            self.dev_pos[s].copy_(self.host[s]["pos"], non_blocking=True)
        self._in_done[s].record(self.h2d)
        main.wait_event(self._in_done[s])
        # ... and its device results only once the previous copy out of them has finished
        main.wait_event(self._out_done[s])
        self.graphs[s].replay()
        self._computed[s].record(main)
        self.d2h.wait_event(self._computed[s])
        with torch.cuda.stream(self.d2h):
            self.host[s]["out"].copy_(self.dev_out[s], non_blocking=True)
        self._out_done[s].record(self.d2h)

    def wait(self, s: int) -> dict:
        """Block until slot ``s``'s last results are in host memory; returns ``host[s]``."""
        if s not in (0, 1):
            raise ValueError("slot must be 0 or 1")
        self._out_done[s].synchronize()
        return self.host[s]

    def fence(self) -> None:
        """Order both copy streams after the work enqueued so far on the current stream (for
        instance a timing event recorded before the first ``submit``)."""
        main = torch.cuda.current_stream(self.device)
        self.h2d.wait_stream(main)
        self.d2h.wait_stream(main)

    def join(self) -> None:
        """Order the current stream after every copy enqueued so far (for instance before a timing
        event recorded after the last ``submit``)."""
        main = torch.cuda.current_stream(self.device)
        main.wait_stream(self.h2d)
        main.wait_stream(self.d2h)


def _profiled_stage(batch: "D3Batch", i: int, stage, reps: int = 2) -> float:
    """Milliseconds of one pipeline stage of structure ``i``, or the summed milliseconds of a
    tuple of stages (eager, profiled calls; the fastest of ``reps`` after one warm-up call)."""
    stages = (stage,) if isinstance(stage, str) else tuple(stage)
    q = int(batch.lane_of[i])
    for call in batch._lane_calls[q]:
        eng, pos, cell_h, cell_d, out, spc, wsl = call
        if pos.data_ptr() == batch.positions_view(i).data_ptr():
            eng.profile(True)
            best = float("inf")
            for _ in range(reps + 1):
                eng.energy_forces_stress(pos, cell_h, batch.r_cut, cell_dev=cell_d, out=out, species=spc, work=wsl)
                t = eng.stage_times()
                best = min(best, sum(t.get(s, float("inf")) for s in stages))
            eng.profile(False)
            return best
    raise KeyError(i)


def autotune_filter(batch: "D3Batch", candidates: Sequence = (0, 1, 2, 4, 8, 16, "tc"), reps: int = 2) -> dict:
    """Pick the filter per species-count class from the heaviest structure of each class: a
    CUDA-core k-tile width (0 = per-thread register kernel) or "tc" (mixed precision: the
    tensor-core filter, where it applies).

    Classes: up to 8 species, 9-24, 25-64. Each class is timed on its heaviest structure
    (profiled eager calls) and its best choice is set on every engine of that class where it
    is valid. Returns {class: (choice, {choice: ms})}. Drops a captured graph.
    """
    batch.drop_captures()
    classes: dict = {}
    for i, key in enumerate(batch._keys):
        s = len(key[0])
        c = 0 if s <= 8 else (1 if s <= 24 else 2)
        if c not in classes or batch.costs[i] > batch.costs[classes[c]]:
            classes[c] = i

    def apply(e, choice) -> bool:
        try:
            if choice == "tc":
                e.set_tuning(filter_kt=-1, filter_mma=1)
                return e.tuning()["filter_mma"] == 1
            e.set_tuning(filter_mma=0, filter_kt=choice)
            return True
        except ValueError:
            return False

    out = {}
    for c, i in sorted(classes.items()):
        eng = batch._engines[batch._keys[i]]
        times = {}
        for choice in candidates:
            if apply(eng, choice):
                times[choice] = _profiled_stage(batch, i, "filter", reps)
        best = min(times, key=times.get)
        for key, e in batch._engines.items():
            s = len(key[0])
            if (0 if s <= 8 else (1 if s <= 24 else 2)) == c and not apply(e, best):
                e.set_tuning(filter_kt=-1, filter_mma=-1)
        out[c] = (best, times)
    return out


def autotune_spread(batch: "D3Batch", candidates: Sequence[int] = (0, 2, 4, 8, 15), reps: int = 2) -> dict:
    """Pick the spread's z-chunk length (0 = per-tile kernel) from the heaviest structure of each
    plan: every candidate is timed (profiled eager calls) and the fastest is set on that plan.
    Returns {plan index: (chunk, {chunk: ms})}. Drops a captured graph."""
    batch.drop_captures()
    heaviest: dict = {}
    for i, key in enumerate(batch._keys):
        if key not in heaviest or batch.costs[i] > batch.costs[heaviest[key]]:
            heaviest[key] = i
    out = {}
    for n, (key, i) in enumerate(heaviest.items()):
        eng = batch._engines[key]
        times = {}
        for zc in candidates:
            eng.set_tuning(spread_zc=zc)
            if eng.tuning()["spread_zc"] != zc and zc != 0:
                continue   # capped by the mesh: the same as a smaller chunk
            times[zc] = _profiled_stage(batch, i, "spread", reps)
        best = min(times, key=times.get)
        eng.set_tuning(spread_zc=best)
        out[n] = (best, times)
    return out


def autotune_fft_x(batch: "D3Batch", pencils: Sequence[int] = (1, 2, 4), reps: int = 2,
                   tma_units: Sequence[tuple] = ((16, 1), (8, 2), (8, 4), (4, 4))) -> dict:
    """Choose per plan between the 3D cuFFT transforms around the separate filter ("0") and the
    (y, z) 2D cuFFT transforms around a fused x-FFT / filter / inverse x-FFT kernel: pencils of
    ``pencils`` kz values of every channel ("1/<kz>"), or TMA-moved units of (q values, ranks)
    from ``tma_units`` ("2/<q>/<ranks>", mixed precision), by the summed time of the forward
    transform, filter and inverse transform stages of the plan's heaviest structure. Plans where
    no fused path applies keep "0". On an x-pass path with 256 x 256 (y, z) planes it then times
    the (y, z) transforms as cluster kernels on pairs (the default), with the forward on quads
    ("<choice>/yz2") and by cuFFT ("<choice>/yz0"), and keeps the fastest. Returns
    {plan index: (choice, {choice: ms})}. Drops a captured graph."""
    batch.drop_captures()
    heaviest: dict = {}
    for i, key in enumerate(batch._keys):
        if key not in heaviest or batch.costs[i] > batch.costs[heaviest[key]]:
            heaviest[key] = i
    out = {}
    stages = ("fft_r2c", "filter", "fft_c2r")
    for n, (key, i) in enumerate(heaviest.items()):
        eng = batch._engines[key]
        eng.set_tuning(fft_x=0, xpencil=-1)
        times = {"0": _profiled_stage(batch, i, stages, reps)}
        for kz in pencils:
            eng.set_tuning(fft_x=1, xpencil=kz)
            t = eng.tuning()
            if t["fft_x"] != 1 or t["xpencil"] != kz:
                continue   # no fused kernel for this mesh, species or rank count, or too wide
            times[f"1/{kz}"] = _profiled_stage(batch, i, stages, reps)
        for xq, xr in tma_units:
            eng.set_tuning(fft_x=2, xq=xq, xranks=xr)
            t = eng.tuning()
            if t["fft_x"] != 2 or (t["xq"], t["xranks"]) != (xq, xr):
                continue   # float64 plan, or the unit does not apply to this mesh / rank count
            times[f"2/{xq}/{xr}"] = _profiled_stage(batch, i, stages, reps)
        best = min(times, key=times.get)
        parts = best.split("/")
        if best == "0":
            eng.set_tuning(fft_x=0, xpencil=-1)
        elif parts[0] == "1":
            eng.set_tuning(fft_x=1, xpencil=int(parts[1]))
        else:
            eng.set_tuning(fft_x=2, xq=int(parts[1]), xranks=int(parts[2]))
        if best != "0" and eng.tuning()["fft_yz"] > 0:
            # the (y, z) transforms of the chosen x-pass path: cluster kernels (pairs, the
            # default; the forward on quads) or cuFFT
            yz_times = {1: times[best]}
            for v in (2, 0):
                eng.set_tuning(fft_yz=v)
                yz_times[v] = _profiled_stage(batch, i, stages, reps)
                times[f"{best}/yz{v}"] = yz_times[v]
            eng.set_tuning(fft_yz=min(yz_times, key=yz_times.get))
        out[n] = (best, times)
    return out


def autotune_lanes(batch: D3Batch, candidates: Sequence[int] = (1, 2, 4, 8), *,
                   cache: Optional[str] = None, reps: int = 3, mem_fraction: float = 0.6) -> int:
    """Choose the lane count with the fastest graph replay; cache it per batch signature.

    Candidates whose lane workspaces would exceed ``mem_fraction`` of the free device
    memory are skipped. With ``cache`` (a JSON path) a known signature is not re-timed.
    """
    sig = batch.signature()
    table = {}
    if cache and os.path.exists(cache):
        with open(cache) as f:
            table = json.load(f)
        if sig in table:
            batch.set_lanes(int(table[sig]["lanes"]))
            return batch.lanes
    results = {}
    for q in candidates:
        split = lpt_split(batch.costs, max(1, min(q, batch.n_struct)))
        need = sum(max(batch._need[i] for i in items) for items in split if items)
        free, _ = torch.cuda.mem_get_info(batch.device)
        if need > mem_fraction * (free + batch.workspace_bytes):
            continue
        batch.set_lanes(q)
        results[batch.lanes] = batch.time_replays(reps)
    best = min(results, key=results.get)
    batch.set_lanes(best)
    if cache:
        table[sig] = {"lanes": best, "ms": results, "when": time.strftime("%Y-%m-%d %H:%M:%S")}
        tmp = cache + ".tmp"
        with open(tmp, "w") as f:
            json.dump(table, f, indent=1, sort_keys=True)
        os.replace(tmp, cache)
    return best
