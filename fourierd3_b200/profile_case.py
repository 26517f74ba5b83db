"""One configuration of the fused E+F+stress call, run a few times eagerly: the command that
per-kernel profiles (Nsight Compute) and launch lists are taken on.

    python -m fourierd3_b200.profile_case --case sio2 --reps 4 --precision fp64 --calls 3
    python -m fourierd3_b200.profile_case --case batch-heaviest --precision mixed --calls 2
    python -m fourierd3_b200.profile_case --case sio2 --reps 1 --method ewald --calls 2

Cases: ``sio2`` (the 648-atom SiO2 box replicated ``reps`` times per axis), ``hcno`` (the
12,000-atom triclinic HCNO box, p = 6, h = 1.0), ``batch-heaviest`` (the costliest structure of
the 256-structure ragged batch: 54 species, rank 8). Each call is launched from the host
without a CUDA graph so that every kernel appears as its own launch; the script prints the
energy, the launch knobs in effect and the stage times of one profiled call.
"""
from __future__ import annotations

import argparse
import json

import numpy as np
import torch

from . import structures as st
from .functional import D3Model


def build_case(case: str, reps: int):
    """(positions, cell, numbers, model keyword arguments) of a named configuration."""
    kw = dict(method="spme", mesh_spacing=1.2, interpolation_nodes=5, c6tol=1.0, r_cut=6.0)
    if case == "sio2":
        pos, cell, nums = st.sio2_scaled(reps)
    elif case == "hcno":
        pos, cell, nums = st.hcno_box()
        kw.update(mesh_spacing=1.0, interpolation_nodes=6)
    elif case == "batch-heaviest":
        from .batch import structure_cost

        structs = st.batch_boxes(256, seed=0)
        costs = [structure_cost(z, c, method="spme", mesh_spacing=1.2) for _, c, z in structs]
        pos, cell, nums = structs[int(np.argmax(costs))]
    else:
        raise ValueError(f"unknown case {case!r}")
    return pos, cell, nums, kw


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--case", default="sio2", choices=["sio2", "hcno", "batch-heaviest"])
    ap.add_argument("--reps", type=int, default=4, help="replicas per axis of the 648-atom SiO2 box")
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--method", default=None, choices=["spme", "pme", "ewald"])
    ap.add_argument("--cnfunc", default="smooth_cut", choices=["smooth_cut", "d4"])
    ap.add_argument("--calls", type=int, default=3)
    ap.add_argument("--tuning", default=None, help="launch knobs, e.g. 'spread_zc=4,fft_x=2,xq=4,xranks=4'")
    args = ap.parse_args(argv)

    pos, cell, nums, kw = build_case(args.case, args.reps)
    if args.method:
        kw["method"] = args.method
    kw["cnfunc"] = args.cnfunc
    dev = torch.device("cuda", 0)
    m = D3Model(nums, cell, precision=args.precision, device=dev, **kw)
    if args.tuning:
        m.engine.set_tuning(**{k: int(v) for k, v in (t.split("=") for t in args.tuning.split(","))})
    p = torch.tensor(pos, dtype=torch.float64, device=dev)
    for _ in range(args.calls):
        e, f, s = m.engine.energy_forces_stress(p, cell, kw["r_cut"])
    torch.cuda.synchronize(dev)
    m.engine.profile(True)
    m.engine.energy_forces_stress(p, cell, kw["r_cut"])
    stages = m.engine.stage_times()
    m.engine.profile(False)
    print(json.dumps({"case": args.case, "n_atoms": len(nums), "n_species": int(len(np.unique(nums))),
                      "precision": args.precision, "method": kw["method"], "energy_ev": float(e),
                      "tuning": m.engine.tuning(), "stages_ms": stages}))


if __name__ == "__main__":
    main()
