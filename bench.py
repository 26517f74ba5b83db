#!/usr/bin/env python
"""E+F+stress throughput of the FourierD3 dispersion path on B200.

Workload: the seeded 648-atom SiO2 box (216 Si + 432 O, L = 21.4 A) replicated 6x6x6 with
N(0, 0.05 A) jitter = 139,968 atoms; PBE-BJ, CN cutoff 6 A, SPME order 5, mesh spacing
1.2 A (256^3 mesh), default c6tol. One step = device cell-list neighbour search + CN + C6
factors + spread + FFT + filter + inverse FFT + gather + CN adjoint: energy, forces and
stress all produced. Synthetic inputs; the C6^ref table is the seeded synthetic stand-in
unless FD3_C6REF points at the real file.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl fd3|reference]

With N > 1 (torchrun, one rank per GPU) each rank runs an independent replica of the box
(the path does not shard a single box): value = N * atoms / max-over-ranks step time.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np
import torch

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "E+F+stress atoms/s, 140k-atom SiO2: mixed/batched vs plain FP64, same B200"
WORKLOAD = "sio2_139968_spme_p5_h1.2_E+F+stress"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="fd3", choices=["fd3", "reference", "reference-gpu"],
                    help="'reference-gpu': only the reference package's float64 torch path on this GPU "
                         "(the headline run starts it as a child process for the plain_fp64_reference_gpu block)")
    ap.add_argument("--no-reference-gpu", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the ragged-batch block of the headline line")
    ap.add_argument("--reps", type=int, default=6)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--precision", default="both", choices=["both", "mixed", "fp64"],
                    help="'both' times plain fp64 and mixed (headline); one value restricts the run")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--workload", default="sio2", choices=["sio2", "batch", "accuracy"],
                    help="'sio2': the 139,968-atom box (headline); 'batch': 256 structures, 32-4,096 atoms, "
                         "Z 1-54, graph-captured lanes vs per-structure launches")
    ap.add_argument("--batch-size", type=int, default=256)
    ap.add_argument("--tuning", default=None,
                    help="fixed launch knobs instead of the autotuners, e.g. 'spread_zc=4,fft_x=1,xpencil=4' "
                         "(names of D3Engine.set_tuning; for profiling one configuration)")
    return ap.parse_args()


def dist_setup(args):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime

        import torch.distributed as dist

        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if torch.cuda.is_available():
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    elif torch.cuda.is_available():
        torch.cuda.set_device(0)
    return ws, rank, local


def gpu_local_cpus(dev_idx: int):
    """The host CPUs NVML reports as closest to the GPU (its NUMA node), or None."""
    try:
        import pynvml

        pynvml.nvmlInit()
        try:
            pr = torch.cuda.get_device_properties(dev_idx)
            h = pynvml.nvmlDeviceGetHandleByPciBusId(
                f"{pr.pci_domain_id:08x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0")
        except Exception:
            h = pynvml.nvmlDeviceGetHandleByIndex(dev_idx)
        ncpu = os.cpu_count() or 1
        words = pynvml.nvmlDeviceGetCpuAffinity(h, (ncpu + 63) // 64)
        cpus = {64 * w + b for w, m in enumerate(words) for b in range(64) if (int(m) >> b) & 1}
        cpus &= set(range(ncpu))
        return cpus or None
    except Exception:
        return None


def on_local_cpus(fn):
    """fn() run by this thread bound to the GPU's NUMA-local CPUs (so that pinned pages it
    allocates and first writes sit next to the GPU); returns (fn's result, cpus or None)."""
    cpus = gpu_local_cpus(torch.cuda.current_device())
    old = os.sched_getaffinity(0) if hasattr(os, "sched_getaffinity") else None
    bound = False
    if cpus and old is not None and (cpus & old):
        try:
            os.sched_setaffinity(0, cpus & old)
            bound = True
        except OSError:
            bound = False
    try:
        r = fn()
    finally:
        if bound:
            os.sched_setaffinity(0, old)
    return r, (cpus & old if bound else None)


def host_buffers_local(batch):
    """batch.host_buffers() on the GPU's NUMA-local CPUs; returns (buffers, cpus or None)."""
    def make():
        h = batch.host_buffers()
        h["out"].zero_()
        h["positions"].copy_(batch.positions.cpu())
        return h
    return on_local_cpus(make)


def time_pipeline(pipe, steps, warmup, ws, device):
    """Milliseconds per evaluation of a two-slot host pipeline (HostPipeline): W untimed
    submissions, then K bracketed by a barrier and a device synchronisation on both sides; the
    events sit on the submitting stream, the first before the first host-to-device copy (the copy
    streams are ordered after it) and the last after the last device-to-host copy."""
    for k in range(warmup):
        pipe.wait(k % 2)
        pipe.submit(k % 2)
    pipe.wait(0)
    pipe.wait(1)
    barrier(ws)
    torch.cuda.synchronize(device)
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record()
    pipe.fence()
    for k in range(steps):
        pipe.wait(k % 2)
        pipe.submit(k % 2)
    pipe.join()
    b.record()
    torch.cuda.synchronize(device)
    barrier(ws)
    return a.elapsed_time(b) / steps


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(x: float, ws: int, device) -> float:
    if ws == 1:
        return x
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


class ClockSampler:
    """SM clocks and clock-event (throttle) reasons of this process's GPU, read through NVML every
    5 ms by a background thread during the timed region (a region of tens of milliseconds still
    gets several samples); falls back to `nvidia-smi -lms 200` when NVML is unavailable. Only
    reads the GPU's state."""

    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"))
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.sm, self.mx, self.reasons = [], [], set()
        self._stop = None
        self._thread = None
        self.proc = None
        self.path = None

    def _nvml_handle(self):
        import pynvml

        pynvml.nvmlInit()
        try:
            pr = torch.cuda.get_device_properties(self.idx)
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(
                f"{pr.pci_domain_id:08x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0")
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.idx)

    def __enter__(self):
        import threading

        try:
            nv, h = self._nvml_handle()
            get_reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                nv.nvmlDeviceGetCurrentClocksThrottleReasons
            bits = [(name, getattr(nv, const)) for name, const in self.REASONS]
            max_sm = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            self._stop = threading.Event()

            def poll():
                while True:
                    try:
                        self.sm.append(float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)))
                        self.mx.append(max_sm)
                        r = get_reasons(h)
                        self.reasons.update(name for name, b in bits if r & b)
                    except Exception:
                        pass
                    if self._stop.wait(0.005):
                        break

            self._thread = threading.Thread(target=poll, daemon=True)
            self._thread.start()
        except Exception:
            self._thread = None
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            try:
                self.proc = subprocess.Popen(
                    ["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.FIELDS}",
                     "--format=csv,noheader,nounits", "-lms", "200"],
                    stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            except Exception:
                self.proc = None
        return self

    def __exit__(self, *exc):
        if self._thread is not None:
            self._stop.set()
            self._thread.join(timeout=5)
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def _read_smi(self):
        names = [name for name, _ in self.REASONS]
        try:
            for line in open(self.path):
                f = [v.strip() for v in line.split(",")]
                if len(f) < 9:
                    continue
                try:
                    self.sm.append(float(f[1]))
                    self.mx.append(float(f[2]))
                except ValueError:
                    continue
                for k, v in zip(names, f[5:9]):
                    if v.lower() == "active":
                        self.reasons.add(k)
        except Exception:
            pass
        finally:
            try:
                os.remove(self.path)
            except Exception:
                pass

    def summary(self):
        if self.path is not None:
            self._read_smi()
        if not self.sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        return {"sm_mhz": float(np.median(self.sm)), "sm_max_mhz": float(max(self.mx)),
                "reasons": sorted(self.reasons), "samples": len(self.sm),
                "source": "nvml" if self.path is None else "nvidia-smi"}


def measured_peaks():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def touched_mesh_values(pos, cell, numbers, mesh, order: int, R: int) -> int:
    """Mesh values (species plane points x R ranks) that some atom's p^3 stencil reaches: what the
    gather must read at least once (SPME stencil centring: round for odd p, floor for even p)."""
    n = np.asarray(mesh)
    u = (np.asarray(pos) @ np.linalg.inv(np.asarray(cell))) * n
    ref = np.round(u).astype(np.int64) if order % 2 else np.floor(u).astype(np.int64)
    offs = np.arange(order) - (order // 2 if order % 2 else order // 2 - 1)
    total = 0
    z = np.asarray(numbers)
    for sp in np.unique(z):
        r = ref[z == sp]
        X = (r[:, 0, None] + offs) % n[0]
        Y = (r[:, 1, None] + offs) % n[1]
        Z = (r[:, 2, None] + offs) % n[2]
        lin = (X[:, :, None, None] * (n[1] * n[2]) + Y[:, None, :, None] * n[2] + Z[:, None, None, :]).reshape(-1)
        total += np.unique(lin).size
    return int(total) * R


def stage_bytes(stage: str, n: int, mesh, C: int, R: int, b: int, touched: int = 0) -> float:
    """Algorithmic HBM bytes of one launch of a pipeline stage: mesh terms per mesh point and
    channel (b bytes real, 2b complex), atom terms per atom. The gather reads only the mesh
    values the atoms' stencils reach (``touched``, when given)."""
    M = mesh[0] * mesh[1] * mesh[2]
    Mh = mesh[0] * mesh[1] * (mesh[2] // 2 + 1)
    if stage == "spread":
        return C * M * b + n * (24 + 4 + 8 * R)
    if stage == "filter":
        # float64: the float32 SPME window table is read per k-point; the mixed form multiplies
        # three per-axis factors (L1-resident) instead
        return 2 * C * Mh * 2 * b + (Mh * 4 if b == 8 else 0)
    if stage == "gather":
        return (touched if touched else C * M) * b + n * (24 + 4 + 16 * R + 8 + 24)
    if stage in ("fft_r2c", "fft_c2r"):
        return C * M * b + C * Mh * 2 * b
    if stage == "cn_c6":
        return n * (32 + 16 + 8 + 16 * R)
    if stage == "cn_adjoint":
        return n * (32 + 16 + 8 + 24 + 24)
    if stage == "cell_list":
        return n * (24 + 4 + 16 + 32 + 16 + 4 * 4)
    return 0.0


def cpu_baseline_port(threads: int, reps_list=(1, 2, 3)):
    """The oracle (CPU float64 restatement of the reference, neighbour search included) timed on
    the host cores at the 1x1x1, 2x2x2 and 3x3x3 replicas of the SiO2 box (648, 5,184 and
    17,496 atoms): one warm-up and one timed E+F+stress evaluation each."""
    from fourierd3_b200 import structures as st
    from oracle.reference_port import OracleFourierD3

    torch.set_num_threads(threads)
    out = {}
    for reps in reps_list:
        p, c, z = st.sio2_scaled(reps)
        o = OracleFourierD3(z, c, method="spme", mesh_spacing=1.2, interpolation_nodes=5, c6tol=1.0, r_cut=6.0)
        o.calculate(p, c)                      # warm-up (decomposition cache, allocator)
        t0 = time.perf_counter()
        o.calculate(p, c)
        dt = time.perf_counter() - t0
        out[len(z)] = (len(z) / dt, dt)
    return out


REF_SAMPLE_WORKLOAD = "sio2_5184_spme_p5_h1.2_E+F+stress"


def run_reference(args, ws, rank):
    """Reference arm: the reference algorithm's CPU path on the host cores. The reference's own
    dependencies (torch-pme, ase, matscipy) are not installable offline, so the arm times the
    oracle -- the float64 CPU restatement of the reference, neighbour search included -- with
    every host thread, on a bounded sample: the 5,184-atom 2x2x2 replica of the benchmarked
    SiO2 box (the 139,968-atom box takes about a minute per evaluation on the host)."""
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    from fourierd3_b200 import structures as st
    from oracle.reference_port import OracleFourierD3

    torch.set_num_threads(threads)
    p, c, z = st.sio2_scaled(2)
    o = OracleFourierD3(z, c, method="spme", mesh_spacing=1.2, interpolation_nodes=5, c6tol=1.0, r_cut=6.0)
    for _ in range(args.warmup):
        o.calculate(p, c)
    per = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        o.calculate(p, c)
        per.append(time.perf_counter() - t0)
    dt = float(np.median(per))
    val = len(z) / dt
    sample = ("one E+F+stress evaluation per step of the 5,184-atom 2x2x2 replica of the benchmarked SiO2 box "
              "(128^3 mesh), neighbour search included; median of the timed steps")
    line = {
        "metric": METRIC, "value": val, "unit": "atoms/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
        "config": {"workload": REF_SAMPLE_WORKLOAD, "sample_of": WORKLOAD, "n_atoms": len(z), "method": "spme",
                   "order": 5},
        "cpu_baseline": {"value": val, "unit": "atoms/s", "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": val, "unit": "atoms/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_reference_gpu(args, local):
    """The metric's denominator, "plain FP64 on the same B200": the reference package's own
    float64 torch path on this GPU. The package (installed unmodified in baseline/_ref) is driven
    through its ASE calculator, FourierD3ASECalculator.calculate (calculator.py:125-192: strain,
    _update_cell, forward, autograd backward, results copied to the host), in float64 at the
    benchmarked box. Its third-party imports are satisfied by the committed stand-ins in
    tests/golden/_shims (torch-pme's mesh size, k-vectors and spline weights restated in plain
    torch; not installable offline), and its table loaders, which read data files the package
    does not ship, return this repository's copies of the same tables (the C6^ref table being the
    synthetic stand-in the kernels use). The neighbour list is built once, outside the timed
    region, as the reference's own timing script does (papercode/get_scaling.py:69); it is the
    same pair set matscipy returns. Prints one JSON line."""
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    ref_root = os.path.join(REPO, "baseline", "_ref")
    out = {"impl": "reference-gpu-fp64"}
    if not os.path.exists(os.path.join(ref_root, "fourierd3", "core.py")):
        out["unavailable"] = "the reference package is not installed in baseline/_ref"
        print(json.dumps(out), flush=True)
        return
    sys.path[:0] = [ref_root, os.path.join(REPO, "tests", "golden", "_shims")]
    import fourierd3
    import fourierd3.core as rcore
    import fourierd3.pair_pot as rpp
    import fourierd3.utils as rutils
    from ase import Atoms

    from fourierd3_b200 import structures as st
    from fourierd3_b200 import tables
    from fourierd3_b200.engine import neighbour_list

    t = tables.load_tables()
    rutils.load_c6ref = lambda types: tables.c6ref_matrix(list(types))
    rcore.load_rcov = lambda: torch.from_numpy(t["rcov"].copy())
    rcore.load_cnref = lambda: torch.from_numpy(t["cnref"].copy())
    rpp.load_sqrtQz = lambda types, device, dtype=torch.float32: \
        torch.from_numpy(t["sqrtQz"].copy())[types].to(device=device, dtype=dtype)
    rpp.load_en = lambda: torch.from_numpy(t["en"].copy())
    rpp.load_rcov_cn = lambda: torch.from_numpy(t["rcov_cn"].copy())

    pos, cell, nums = st.sio2_scaled(args.reps)
    t0 = time.perf_counter()
    calc = fourierd3.FourierD3ASECalculator(dtype=torch.float64, device=device, method="spme", mesh_spacing=1.2,
                                            interpolation_nodes=5, c6tol=1.0, r_cut=6.0)
    atoms = Atoms(nums, pos, cell)
    calc._build_model(atoms)
    i, j, S = neighbour_list(torch.tensor(pos, dtype=torch.float64, device=device), cell, 6.0)
    edges = (torch.stack([i, j]), S.to(torch.float64))
    calc._build_graph = lambda atoms_, rcut=None: edges
    setup_s = time.perf_counter() - t0
    torch.cuda.reset_peak_memory_stats(device)
    ms_med, ms_mean = time_steps_stats(lambda: calc.calculate(atoms), args.steps, args.warmup, 1, device)
    out.update({
        "value": len(nums) / (ms_med * 1e-3), "unit": "atoms/s", "ms_per_step": ms_med, "mean_ms": ms_mean,
        "steps": args.steps, "warmup": args.warmup, "n_atoms": len(nums), "dtype": "f64",
        "mesh": [int(v) for v in calc._model.ns_mesh], "c6_rank": int(calc._model.n_rank),
        "energy_ev": float(calc.results["energy"]), "setup_s": setup_s,
        "peak_mem_gb": torch.cuda.max_memory_allocated(device) / 1e9,
        "step": "FourierD3ASECalculator.calculate with the neighbour list prebuilt (papercode/get_scaling.py:69)",
        "third_party": "torch-pme / ase / matscipy stand-ins from tests/golden/_shims",
        "c6_source": tables.c6_source()})
    print(json.dumps(out), flush=True)


def child_json(cmd, local, label, timeout_s):
    """Runs a bench leg in a child process (its memory is released when it exits, and a failure
    there cannot end the headline run); returns the last JSON line it prints."""
    env = dict(os.environ, LOCAL_RANK=str(local), WORLD_SIZE="1", RANK="0")
    try:
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout_s, env=env)
    except subprocess.TimeoutExpired:
        return {"leg": label, "unavailable": f"did not finish within {timeout_s} s"}
    for line in reversed(r.stdout.splitlines()):
        if line.startswith("{"):
            try:
                return json.loads(line)
            except ValueError:
                break
    tail = (r.stderr or r.stdout).strip().splitlines()[-3:]
    return {"leg": label, "unavailable": f"exit {r.returncode}: " + " | ".join(tail)}


def reference_gpu_subprocess(args, local, timeout_s=900):
    """run_reference_gpu in a child process; returns its JSON record."""
    cmd = [sys.executable, os.path.join(REPO, "bench.py"), "--impl", "reference-gpu", "--reps", str(args.reps),
           "--steps", str(max(3, min(args.steps, 5))), "--warmup", "1"]
    return child_json(cmd, local, "reference-gpu-fp64", timeout_s)


def batch_subprocess(args, local, timeout_s=900):
    """The ragged-batch workload (256 structures, 32-4,096 atoms, Z 1-54) in a child process, 3
    timed graph replays after 3 warm-up replays; returns its JSON record (value, ms per batch,
    heaviest structure's stages, clocks)."""
    cmd = [sys.executable, os.path.join(REPO, "bench.py"), "--workload", "batch", "--steps", "3", "--warmup", "3"]
    return child_json(cmd, local, "batch", timeout_s)


BATCH_WORKLOAD = "batch256_N32-4096_Z1-54_spme_p5_h1.2_E+F+stress"


def run_accuracy(args, ws, rank, local):
    """Precision scaling: the seeded SiO2 box replicated 1^3..6^3 (648..139,968 atoms, jitter
    N(0, 0.05 A)); plain float64 SPME, the mixed form (3D transforms) and the mixed form as the
    headline runs it (TMA x-pass) against the float64 direct pairwise D3 lattice sum computed on
    the device at every size (pairs within 25 A + continuum tail), against the CPU oracle's direct
    sum where a fixture exists (648, 5,184 atoms), and the mixed forms against float64 SPME. One
    JSON line per size; energies in eV, forces eV/A, stress eV/A^3."""
    if rank != 0:
        return
    from fourierd3_b200 import structures as st
    from fourierd3_b200.functional import D3Model

    device = torch.device("cuda", local)
    kw = dict(method="spme", mesh_spacing=1.2, interpolation_nodes=5, c6tol=1.0, r_cut=6.0)
    golden = os.path.join(REPO, "tests", "golden")

    def diff(a, b):
        return {"energy_rel": abs(a[0] - b[0]) / abs(b[0]), "force_max_ev_a": float(np.abs(a[1] - b[1]).max()),
                "stress_max_ev_a3": float(np.abs(a[2] - b[2]).max())}

    for reps in range(1, 7):
        pos, cell, nums = st.sio2_scaled(reps)
        path = os.path.join(golden, f"direct_sio2_{len(nums)}.npz")
        d = np.load(path) if os.path.exists(path) else None
        if d is not None:   # the direct-sum fixture's own structure (648: the box before jitter)
            pos, cell, nums = d["positions"], d["cell"], d["numbers"]
        res = {}
        for prec in ("fp64", "mixed"):
            m = D3Model(nums, cell, precision=prec, device=device, **kw)
            e, f, s = m(pos, cell)
            res[prec] = (float(e), f.cpu().numpy(), s.cpu().numpy())
            if prec == "fp64":
                torch.cuda.synchronize(device)
                t0 = time.perf_counter()
                e, f, s = m.direct(pos, cell, r_direct=25.0)
                torch.cuda.synchronize(device)
                res["direct_gpu_s"] = time.perf_counter() - t0
                res["direct_gpu"] = (float(e), f.cpu().numpy(), s.cpu().numpy())
            else:
                # the mixed form as the headline runs it: TMA x-pass where it applies
                m.engine.set_tuning(fft_x=2, xq=4, xranks=4)
                if m.engine.tuning()["fft_x"] == 2:
                    e, f, s = m(pos, cell)
                    res["mixed_tma"] = (float(e), f.cpu().numpy(), s.cpu().numpy())
            del m
            torch.cuda.empty_cache()
        line = {"workload": "accuracy_sio2_scaling", "n_atoms": len(nums), "reps": reps,
                "energy_ev_fp64": res["fp64"][0], "energy_ev_direct": res["direct_gpu"][0],
                "direct_gpu_s": res["direct_gpu_s"]}
        for form in ("mixed", "mixed_tma"):
            if form in res:
                line[f"{form}_vs_fp64"] = diff(res[form], res["fp64"])
        for form in ("fp64", "mixed", "mixed_tma"):
            if form in res:
                line[f"{form}_vs_direct_gpu"] = diff(res[form], res["direct_gpu"])
        if d is not None:
            ref = (float(d["energy_ev"]), d["forces"], d["stress"])
            line["direct_gpu_vs_direct_cpu_oracle"] = diff(res["direct_gpu"], ref)
            for form in ("fp64", "mixed", "mixed_tma"):
                if form in res:
                    line[f"{form}_vs_direct_cpu_oracle"] = diff(res[form], ref)
        print(json.dumps(line), flush=True)


def run_batch(args, ws, rank, local):
    """Batch workload: structures sharded over ranks (LPT on N + M*S*r), one graph per rank."""
    from fourierd3_b200 import _native, structures as st
    from fourierd3_b200.batch import D3Batch, autotune_filter, autotune_lanes, lpt_split

    device = torch.device("cuda", local)
    structs = st.batch_boxes(args.batch_size, seed=0)
    kw = dict(method="spme", mesh_spacing=1.2, interpolation_nodes=5, c6tol=1.0, r_cut=6.0)
    t0 = time.perf_counter()
    # one D3Batch over every structure only to read the cost model; ranks then keep their share
    costs = []
    from fourierd3_b200.batch import structure_cost
    for p, c, z in structs:
        costs.append(structure_cost(z, c, method="spme", mesh_spacing=1.2))
    mine = sorted(lpt_split(costs, ws)[rank]) if ws > 1 else list(range(len(structs)))
    sub = [structs[i] for i in mine]
    n_local = int(sum(len(structs[i][2]) for i in mine))
    n_total = int(sum(len(z) for _, _, z in structs))
    res = {}
    plain = D3Batch(sub, precision="mixed", lanes=1, device=device, **kw)
    setup_s = time.perf_counter() - t0
    steps = max(1, min(args.steps, 5))
    warm = max(3, min(args.warmup, 3))
    # per-structure launches, default tiles: the untuned eager baseline
    res["mixed_eager_1lane"] = max_over_ranks(time_steps(lambda: plain(), steps, warm, ws, device), ws, device)
    del plain
    torch.cuda.empty_cache()
    b = D3Batch(sub, precision="mixed", lanes=1, device=device, **kw)
    ftune = autotune_filter(b, reps=1)
    lanes = autotune_lanes(b, (1, 2, 4), reps=2)
    if not b.captured:
        b.capture()
    with ClockSampler(torch.cuda.current_device()) as cs:
        ms = max_over_ranks(time_steps(lambda: b(), steps, warm, ws, device), ws, device)
    clocks = cs.summary()
    res["mixed_graph"] = ms
    # the kernel count per replay: count one eager pass over the same lanes
    l0 = _native.launch_count()
    b._launch_all()
    torch.cuda.synchronize(device)
    per_batch = _native.launch_count() - l0
    # stage times of the heaviest structure (profiled eager call)
    big = int(np.argmax(b.costs))
    eng = b._lane_calls[int(b.lane_of[big])][0][0]
    stages = {}
    for call in b._lane_calls[int(b.lane_of[big])]:
        if call[0] is eng:
            e_, pos_, ch_, cd_, out_, spc_, wsl_ = call
            eng.profile(True)
            eng.energy_forces_stress(pos_, ch_, b.r_cut, cell_dev=cd_, out=out_, species=spc_, work=wsl_)
            stages = eng.stage_times()
            eng.profile(False)
            break
    # end to end: one graph replay that copies the host positions in and E/F/stress out
    host_buffers_local(b)

    def e2e():
        b.run_host()

    e2e_ms = max_over_ranks(time_steps(e2e, steps, warm, ws, device), ws, device)
    mesh_pts = sum(int(np.prod(b._keys[i][1])) * len(b._keys[i][0]) * b._engines[b._keys[i]].setup.n_rank
                   for i in range(b.n_struct))
    line = {
        "metric": "E+F+stress atoms/s, ragged batch of 256 periodic structures", "value": n_total / (ms * 1e-3),
        "unit": "atoms/s", "n_gpus": ws, "steps": steps, "warmup": warm, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32-mesh+f64-accum",
        "data": "synthetic",
        "config": {"workload": BATCH_WORKLOAD, "n_structures": len(structs), "n_atoms": n_total,
                   "n_atoms_rank0": n_local, "lanes": lanes, "mesh_channel_points_rank0": mesh_pts,
                   "l2": "inputs larger than L2", "parallelism": f"shard{ws}", "setup_s": setup_s,
                   "filter_tile_by_species_class": {str(k): v[0] for k, v in ftune.items()},
                   "filter_tile_ms": {str(k): v[1] for k, v in ftune.items()}},
        "per_structure_eager": {"value": n_total / (res["mixed_eager_1lane"] * 1e-3),
                                "ms_per_step": res["mixed_eager_1lane"]},
        "graph_over_eager": res["mixed_eager_1lane"] / ms,
        "stages_ms_heaviest": stages,
        "e2e": {"value": n_total / (e2e_ms * 1e-3), "unit": "atoms/s", "ms_per_step": e2e_ms,
                "h2d_bytes_per_step": int(b.positions.numel() * 8),
                "d2h_bytes_per_step": int((b.energy.numel() + b.forces.numel() + b.stress.numel()) * 8)},
        "gpu_launches": int(per_batch) * steps,
        "clocks": clocks,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)


def time_steps_stats(fn, steps, warmup, ws, device):
    """W untimed steps, then K steps bracketed by a barrier and a device synchronisation on both
    sides, with a CUDA event on the launching stream before every step and after the last:
    returns (median, mean) milliseconds per step."""
    for _ in range(warmup):
        fn()
    barrier(ws)
    torch.cuda.synchronize(device)
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(steps + 1)]
    evs[0].record()
    for k in range(steps):
        fn()
        evs[k + 1].record()
    torch.cuda.synchronize(device)
    barrier(ws)
    per = [evs[k].elapsed_time(evs[k + 1]) for k in range(steps)]
    return float(np.median(per)), evs[0].elapsed_time(evs[-1]) / steps


def time_steps(fn, steps, warmup, ws, device):
    return time_steps_stats(fn, steps, warmup, ws, device)[0]


def main():
    args = parse()
    ws, rank, local = dist_setup(args)
    if args.impl == "reference-gpu":
        run_reference_gpu(args, local)
        return
    if args.impl == "reference":
        run_reference(args, ws, rank)
        if ws > 1:
            import torch.distributed as dist

            dist.destroy_process_group()
        return
    if args.workload == "accuracy":
        run_accuracy(args, ws, rank, local)
        if ws > 1:
            import torch.distributed as dist

            dist.destroy_process_group()
        return
    if args.workload == "batch":
        run_batch(args, ws, rank, local)
        if ws > 1:
            import torch.distributed as dist

            dist.destroy_process_group()
        return
    from fourierd3_b200 import _native, tables, structures as st
    from fourierd3_b200.functional import D3Model

    device = torch.device("cuda", local)
    pos, cell, nums = st.sio2_scaled(args.reps)
    n = len(nums)
    precs = ("fp64", "mixed") if args.precision == "both" else (args.precision,)
    head = "mixed" if "mixed" in precs else "fp64"
    models = {prec: D3Model(nums, cell, precision=prec, device=device, method="spme", mesh_spacing=1.2,
                            interpolation_nodes=5, c6tol=1.0, r_cut=6.0) for prec in precs}
    mesh = models[head].mesh
    R = models[head].setup.n_rank
    S = models[head].setup.n_species
    C = S * R
    pos_dev = torch.tensor(pos, dtype=torch.float64, device=device)
    cell_dev = torch.tensor(cell, dtype=torch.float64, device=device)
    outs = {k: (torch.empty((), dtype=torch.float64, device=device),
                torch.empty((n, 3), dtype=torch.float64, device=device),
                torch.empty((3, 3), dtype=torch.float64, device=device)) for k in models}

    def step(prec):
        models[prec].engine.energy_forces_stress(pos_dev, cell, 6.0, cell_dev=cell_dev, out=outs[prec])

    # the production form: the whole step captured as one CUDA graph (D3Batch of one box); a
    # replay relaunches every kernel and cuFFT pass, so nothing is cached between steps
    from fourierd3_b200.batch import D3Batch

    from fourierd3_b200.batch import autotune_fft_x, autotune_spread

    graphs, tuned = {}, {}
    for prec in precs:
        b = D3Batch([(pos, cell, nums)], precision=prec, lanes=1, device=device, method="spme", mesh_spacing=1.2,
                    interpolation_nodes=5, c6tol=1.0, r_cut=6.0)
        # launch shapes chosen by timing (results agree to rounding); the same plan settings
        # are copied to the eager model so both forms run the same kernels
        eng = next(iter(b._engines.values()))
        if args.tuning:
            eng.set_tuning(**{k: int(v) for k, v in (kv.split("=") for kv in args.tuning.split(","))})
            tuned[prec] = eng.tuning()
        else:
            sp = autotune_spread(b, reps=2)
            fx = autotune_fft_x(b, reps=2)
            tuned[prec] = eng.tuning()
            tuned[prec]["spread_ms"] = {str(k): round(v, 4) for k, v in sp[0][1].items()}
            tuned[prec]["fft_filter_ms"] = {str(k): round(v, 4) for k, v in fx[0][1].items()}
        models[prec].engine.set_tuning(spread_zc=tuned[prec]["spread_zc"], fft_x=tuned[prec]["fft_x"],
                                       xpencil=tuned[prec]["xpencil"] if tuned[prec]["fft_x"] == 1 else -1,
                                       xq=tuned[prec]["xq"] if tuned[prec]["fft_x"] == 2 else -1,
                                       xranks=tuned[prec]["xranks"] if tuned[prec]["fft_x"] == 2 else -1,
                                       fft_yz=tuned[prec]["fft_yz"])
        b.capture()
        graphs[prec] = b

    res, eager = {}, {}
    clocks = None
    for prec in precs:
        l0 = _native.launch_count()
        step(prec)
        torch.cuda.synchronize(device)
        per_step = _native.launch_count() - l0
        if prec == head:
            launches = per_step
            with ClockSampler(torch.cuda.current_device()) as cs:
                ms, ms_mean = time_steps_stats(lambda: graphs[prec](), args.steps, args.warmup, ws, device)
            clocks = cs.summary()
            head_mean = max_over_ranks(ms_mean, ws, device)
        else:
            ms = time_steps(lambda: graphs[prec](), args.steps, args.warmup, ws, device)
        res[prec] = max_over_ranks(ms, ws, device)
        eager[prec] = max_over_ranks(time_steps(lambda: step(prec), args.steps, args.warmup, ws, device), ws, device)

    # per-stage CUDA-event times on the launching stream (separate, profiled steps)
    stages = {}
    for prec in precs:
        eng = models[prec].engine
        eng.profile(True)
        acc: dict = {}
        nprof = max(3, min(args.steps, 10))
        for _ in range(nprof):
            step(prec)
            for k, v in eng.stage_times().items():
                acc[k] = acc.get(k, 0.0) + v / nprof
        eng.profile(False)
        stages[prec] = acc

    # end-to-end through the public API with host buffers: D3Batch.run_host replays one graph
    # that copies the positions in from pinned host memory, evaluates, and copies energy, stress
    # and forces back out (one copy each way)
    gb = graphs[head]
    # the pinned host buffers on the GPU's own NUMA node (allocated and first written by a thread
    # bound to the CPUs NVML lists for the GPU; the binding is undone afterwards)
    hbuf, local_cpus = host_buffers_local(gb)
    hbuf["positions"].copy_(torch.tensor(pos, dtype=torch.float64))
    h2d_bytes = int(hbuf["pos"].numel() * 8)
    d2h_bytes = int(hbuf["out"].numel() * 8)

    def e2e_step():
        gb.run_host()

    # the same evaluations through the two-slot pipeline (HostPipeline): each evaluation still
    # copies its positions in and its results out, on copy streams, beside the other's compute
    def make_pipe():
        pp = gb.host_pipeline()
        for h in pp.host:
            h["out"].zero_()
            h["positions"].copy_(torch.tensor(pos, dtype=torch.float64))
        return pp

    e2e_ms = e2e_seq_ms = None
    if not args.no_e2e:
        e2e_seq_ms = max_over_ranks(time_steps(e2e_step, args.steps, args.warmup, ws, device), ws, device)
        pipe, _ = on_local_cpus(make_pipe)
        assert pipe.h2d_bytes == h2d_bytes and pipe.d2h_bytes == d2h_bytes
        e2e_ms = max_over_ranks(time_pipeline(pipe, args.steps, args.warmup, ws, device), ws, device)

    b = 4 if head == "mixed" else 8
    st_mixed = stages[head]
    # this library's stages: the (y, z) transform stages count when the fused cluster kernels run
    # them (otherwise they are cuFFT's)
    yz_own = int(models[head].engine.tuning().get("fft_yz", 0)) > 0
    ours = {k: v for k, v in st_mixed.items() if yz_own or not k.startswith("fft")}
    dom = max(ours, key=ours.get)
    peak, peak_kind = measured_peaks()
    touched = touched_mesh_values(pos, cell, nums, mesh, 5, R)
    dom_bytes = stage_bytes(dom, n, mesh, C, R, b, touched)
    achieved = dom_bytes / (ours[dom] * 1e-3) / 1e9
    # every own stage against the same peak (algorithmic bytes / CUDA-event stage time)
    stage_roof = {}
    for k, ms in ours.items():
        by = stage_bytes(k, n, mesh, C, R, b, touched)
        if by > 0 and ms > 0:
            stage_roof[k] = {"bytes": by, "ms": ms, "gbs": by / (ms * 1e-3) / 1e9,
                             "frac": by / (ms * 1e-3) / 1e9 / peak}
    # DRAM bytes (read + write) per launch from one-kernel ncu captures on this 256^3 x 8-channel mixed
    # mesh (the mesh-side traffic does not depend on N), for the filter kernel the tuner picked:
    # 3D-path filter, the cp.async pencil x-pass (fft_x 1) or the TMA x-pass (fft_x 2, 4 q x 4 ranks)
    fx = int(tuned.get(head, {}).get("fft_x", 0))
    filter_traffic = {0: 541.3e6 + 481.7e6, 1: 547.0e6 + 492.3e6, 2: 541.2e6 + 488.1e6}[fx]
    if fx == 2 and (tuned[head].get("xq"), tuned[head].get("xranks")) != (4, 4):
        filter_traffic = None
    traffic_by_stage = {"filter": filter_traffic, "spread": (20.3e6 + 492.5e6),
                        "fft_r2c": (545.1e6 + 488.7e6) if yz_own else None,
                        "fft_c2r": (566.8e6 + 493.5e6) if yz_own else None}
    kernel_names = {"filter": {0: "k_filter", 1: "k_xfilter", 2: "k_xpass"}[fx], "spread": "k_spread_col",
                    "gather": "k_gather_z", "fft_r2c": "k_yz_forward", "fft_c2r": "k_yz_inverse",
                    "cn_c6": "k_cn_bins + k_c6_atoms", "cn_adjoint": "k_cn_adjoint_hits"}
    mesh_match = tuple(mesh) == (256, 256, 256) and C == 8 and head == "mixed"
    roof = {"bound": "hbm", "kernel": dom, "kernel_name": kernel_names.get(dom), "achieved": achieved,
            "peak": peak, "peak_kind": peak_kind,
            "unit": "GB/s", "frac": achieved / peak,
            "traffic": traffic_by_stage.get(dom) if mesh_match else None,
            "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum, 256^3 x 8 channels, mixed"
                              if mesh_match and dom in traffic_by_stage else None,
            "bytes_per_launch": dom_bytes, "ms_per_launch": ours[dom], "stages": stage_roof}
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        sizes = cpu_baseline_port(threads)
        big = max(sizes)
        cpu = {"value": sizes[big][0], "unit": "atoms/s", "cores": threads, "kind": "port",
               "sample": f"oracle (CPU float64 restatement, neighbour search included): one E+F+stress of the "
                         f"{big}-atom 3x3x3 replica of the benchmarked box, {sizes[big][1]:.1f} s; "
                         f"also 648 and 5,184 atoms (by_size)",
               "by_size": {str(k): {"atoms_per_s": v, "s": t} for k, (v, t) in sorted(sizes.items())}}

    # the metric's denominator: the reference package's float64 torch path on this GPU
    ref_gpu = None
    if rank == 0 and ws == 1 and not args.no_reference_gpu:
        ref_gpu = reference_gpu_subprocess(args, local)
    # the batched form of the metric ("mixed/batched"): the ragged 256-structure batch
    batch = None
    if rank == 0 and ws == 1 and not args.no_batch:
        batch = batch_subprocess(args, local)

    ms = res[head]
    line = {
        "metric": METRIC, "value": ws * n / (ms * 1e-3), "unit": "atoms/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32-mesh+f64-accum" if head == "mixed" else "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "n_atoms": n, "mesh": list(mesh), "method": "spme", "order": 5,
                   "species": S, "c6_rank": R, "precision": head, "parallelism": f"replicas{ws}",
                   "execution": "one CUDA graph per step (fourierd3_b200.batch.D3Batch.capture)",
                   "autotuned": tuned.get(head),
                   "l2": "inputs larger than L2 (mesh channels %.2f GB)" % (C * mesh[0] * mesh[1] * mesh[2] * 4 / 1e9),
                   "c6_source": tables.c6_source()},
        "plain_fp64": ({"value": ws * n / (res["fp64"] * 1e-3), "ms_per_step": res["fp64"],
                        "eager_ms_per_step": eager["fp64"], "stages_ms": stages["fp64"]} if "fp64" in res else None),
        "eager": {"value": ws * n / (eager[head] * 1e-3), "ms_per_step": eager[head],
                  "note": "the same step launched from the host without graph capture"},
        "mixed_over_fp64": res["fp64"] / ms if "fp64" in res and head == "mixed" else None,
        "plain_fp64_reference_gpu": ref_gpu,
        "batch": batch,
        "mixed_over_reference_fp64_gpu": (ref_gpu["ms_per_step"] / ms
                                          if ref_gpu and "ms_per_step" in ref_gpu else None),
        "fp64_over_reference_fp64_gpu": (ref_gpu["ms_per_step"] / res["fp64"]
                                         if ref_gpu and "ms_per_step" in ref_gpu and "fp64" in res else None),
        "timing": {"statistic": "median of the timed steps (CUDA events per step on the launching stream)",
                   "mean_ms_per_step": head_mean},
        "stages_ms": stages[head],
        "roofline": roof,
        "cpu_baseline": cpu,
        "e2e": ({"value": ws * n / (e2e_ms * 1e-3), "unit": "atoms/s", "ms_per_step": e2e_ms,
                 "h2d_bytes_per_step": h2d_bytes, "d2h_bytes_per_step": d2h_bytes,
                 "path": "D3Batch.host_pipeline: every evaluation copies the pinned host positions in "
                         "and energy, stress and forces out to pinned host memory, on copy streams, "
                         "two evaluations in flight (K evaluations timed from the first copy in to "
                         "the last copy out)",
                 "sequential": {"value": ws * n / (e2e_seq_ms * 1e-3), "ms_per_step": e2e_seq_ms,
                                "path": "D3Batch.run_host: one graph replay with both copies inside, "
                                        "one evaluation at a time (median step)"},
                 "host_buffers": ("pinned on the GPU's NUMA node (allocated from a thread bound to the "
                                  f"{len(local_cpus)} CPUs NVML lists for the GPU)" if local_cpus
                                  else "pinned (NVML CPU affinity unavailable)")}
                if e2e_ms is not None else None),
        "gpu_launches": int(launches) * args.steps,
        "clocks": clocks,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


if __name__ == "__main__":
    main()
