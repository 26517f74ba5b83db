"""Loader for the golden fixtures in tests/golden/ (made by tests/golden/make_golden.py)."""
import glob
import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def names():
    """Fixtures produced by the reference's own code (make_golden.py); direct_* are oracle sums."""
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz"))
                  if not os.path.basename(p).startswith("direct_"))


def load(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    rec = {k: z[k] for k in z.files}
    rec["config"] = json.loads(str(rec["config"]))
    return rec


def model_kwargs(cfg):
    kw = dict(method=cfg["method"], mesh_spacing=cfg["mesh_spacing"], interpolation_nodes=cfg["interpolation_nodes"],
              c6tol=cfg["c6tol"], k_cutoff=cfg["k_cutoff"], r_cut=cfg["r_cut"])
    if cfg.get("cncorr") is not None:
        kw["cncorr"] = np.asarray(cfg["cncorr"], dtype=np.float64)
    if cfg.get("cnfunc", "smooth_cut") != "smooth_cut":
        kw["cnfunc"] = cfg["cnfunc"]
    return kw


def is_d4(name):
    """Fixtures with the k-space D4 coordination number (no edge list)."""
    return load(name)["config"].get("cnfunc") == "d4"


def skip_unbuilt(name):
    """pytest.skip for a fixture whose configuration the device path does not build: the D4 CN
    with the Ewald method (the reference's own branch for it reads an attribute it never
    defines, src/fourierd3/core.py:436; the fixture comes from the repaired code and pins the
    oracle only)."""
    import pytest

    cfg = load(name)["config"]
    if cfg.get("cnfunc") == "d4" and cfg["method"] == "ewald":
        pytest.skip("D4 CN with the Ewald method is not built on the device")
