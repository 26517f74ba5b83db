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
    # cnfunc (int32, padded) and the two D4 table pointers follow the original seven pointers
    assert d.cnfunc.offset == 88 + 7 * 8 and d.rcov_cn.offset == 152 and d.en.offset == 160
    assert ctypes.sizeof(d) == 168


def test_cell_grid_host_geometry():
    import numpy as np

    from fourierd3_b200.engine import Engine

    nb, reach = Engine.cell_grid(np.eye(3) * 21.4, 6.0)
    assert nb == (3, 3, 3) and reach == (1, 1, 1)
    nb, reach = Engine.cell_grid(np.eye(3) * 5.0, 6.0)       # cell narrower than the cutoff
    assert nb == (1, 1, 1) and reach == (2, 2, 2)


def test_invalid_arguments_return_status_codes():
    """Argument checks happen on the host before any device work: bad descriptors, null plans
    and degenerate cells come back as FD3_EINVAL (and a readable fd3_last_error), never a crash."""
    import numpy as np

    lib = _native.lib()
    plan = ctypes.c_void_p()

    def desc(**kw):
        d = _native.PlanDesc()
        d.n_species, d.n_rank, d.method, d.order, d.precision = 2, 4, 0, 5, 0
        for a in range(3):
            d.mesh[a] = 32
            d.ewald_ns[a] = 2
        d.r_cut = 11.3
        for k, v in kw.items():
            setattr(d, k, v)
        return d

    for bad in (dict(n_species=0), dict(n_species=65), dict(n_rank=0), dict(n_rank=33), dict(method=7),
                dict(precision=3), dict(order=0), dict(order=9)):
        assert lib.fd3_plan_create(ctypes.byref(desc(**bad)), ctypes.byref(plan)) == _native.FD3_EINVAL, bad
        assert not plan.value
    d = desc()
    d.mesh[1] = 0
    assert lib.fd3_plan_create(ctypes.byref(d), ctypes.byref(plan)) == _native.FD3_EINVAL
    d = desc(method=2)
    d.ewald_ns[2] = 0
    assert lib.fd3_plan_create(ctypes.byref(d), ctypes.byref(plan)) == _native.FD3_EINVAL
    assert lib.fd3_last_error()

    nbytes = ctypes.c_size_t()
    assert lib.fd3_workspace_size(None, 10, 0, ctypes.byref(nbytes)) == _native.FD3_EINVAL
    cell = np.eye(3).reshape(9) * 20.0
    assert lib.fd3_energy_forces_stress(None, 10, None, None, _native.dptr(cell), None, 6.0, None, 0, None, None,
                                        None, None) == _native.FD3_EINVAL
    assert lib.fd3_energy_edges(None, 10, None, None, None, 0, None, None, None, 0, None, 0, None, None, None, None,
                                None) == _native.FD3_EINVAL
    assert lib.fd3_plan_set_tuning(None, _native.TUNE_FILTER_KT, 4) == _native.FD3_EINVAL
    v = ctypes.c_int32()
    assert lib.fd3_plan_get_tuning(None, _native.TUNE_FILTER_KT, ctypes.byref(v)) == _native.FD3_EINVAL
    assert lib.fd3_plan_set_tuning(None, _native.TUNE_XPENCIL, 4) == _native.FD3_EINVAL
    # degenerate cell, non-positive cutoff
    nb = (ctypes.c_int32 * 3)()
    rr = (ctypes.c_int32 * 3)()
    flat = np.zeros(9)
    assert lib.fd3_cell_grid(_native.dptr(flat), 6.0, nb, rr) == _native.FD3_EINVAL
    assert lib.fd3_cell_grid(_native.dptr(cell), 0.0, nb, rr) == _native.FD3_EINVAL
    assert lib.fd3_neighbor_workspace_size(10, _native.dptr(flat), 6.0, ctypes.byref(nbytes)) == _native.FD3_EINVAL
    # a null cell or an empty box is an argument error, not a host crash
    assert lib.fd3_cell_grid(None, 6.0, nb, rr) == _native.FD3_EINVAL
    assert lib.fd3_neighbor_workspace_size(10, None, 6.0, ctypes.byref(nbytes)) == _native.FD3_EINVAL
    assert lib.fd3_neighbor_workspace_size(0, _native.dptr(cell), 6.0, ctypes.byref(nbytes)) == _native.FD3_EINVAL
    count = ctypes.c_int64()
    assert lib.fd3_neighbor_fill_static(10, None, None, 6.0, 16, None, None, None, ctypes.byref(count),
                                        None) == _native.FD3_EINVAL
    assert lib.fd3_energy_forces_stress(None, 10, None, None, None, None, 6.0, None, 0, None, None, None,
                                        None) == _native.FD3_EINVAL
