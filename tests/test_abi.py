"""libfd3.so loads and exports every symbol include/fd3.h declares (CPU, no compute)."""
import ctypes
import os
import re

from fourierd3_b200 import _native

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    txt = open(os.path.join(REPO, "include", "fd3.h")).read()
    return sorted(set(re.findall(r"FD3_API\s+[\w\s\*]+?\b(fd3_\w+)\s*\(", txt)))


def test_header_and_binding_agree():
    assert declared_symbols() == sorted(_native.EXPORTED)


def test_library_loads_and_exports_all_symbols():
    lib = _native.lib()
    for name in declared_symbols():
        assert hasattr(lib, name), name
    assert isinstance(_native.launch_count(), int)
    assert lib.fd3_last_error() is not None


def test_plan_desc_layout_matches_header():
    # int32 x 12 (n_species..has_cncorr with two int[3]) then doubles and pointers
    d = _native.PlanDesc
    assert d.r_cut.offset == 48 and d.params.offset == 56 and d.rcov.offset == 88
    assert ctypes.sizeof(d) == 88 + 7 * 8


def test_cell_grid_host_geometry():
    import numpy as np

    from fourierd3_b200.engine import Engine

    nb, reach = Engine.cell_grid(np.eye(3) * 21.4, 6.0)
    assert nb == (3, 3, 3) and reach == (1, 1, 1)
    nb, reach = Engine.cell_grid(np.eye(3) * 5.0, 6.0)       # cell narrower than the cutoff
    assert nb == (1, 1, 1) and reach == (2, 2, 2)
