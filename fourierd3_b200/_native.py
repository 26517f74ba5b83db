"""ctypes binding of libfd3.so (the C ABI declared in include/fd3.h).

The library is built in-tree by ``python -m fourierd3_b200.build``. There is no
fallback: if the shared object is missing or fails to load, every compute call
raises, so a GPU run can never silently take a CPU or pure-PyTorch path.
"""
from __future__ import annotations

import ctypes
import os
import threading

_LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_lib", "libfd3.so")

FD3_OK, FD3_EINVAL, FD3_ECAPACITY, FD3_ECUDA, FD3_ECUFFT, FD3_ENOMEM = range(6)
METHODS = {"spme": 0, "pme": 1, "ewald": 2}
PREC_FP64, PREC_MIXED = 0, 1
TUNE_FILTER_KT = 0
TUNE_SPREAD_ZC = 1
TUNE_SPREAD_CAP = 2
TUNE_FFT_X = 3
TUNE_XPENCIL = 4
TUNE_XQ = 5
TUNE_XRANKS = 6
TUNE_FILTER_MMA = 7
TUNE_GATHER_TILE = 8
TUNE_FFT_YZ = 9

_c_int32 = ctypes.c_int32
_c_int64 = ctypes.c_int64
_c_double = ctypes.c_double
_vp = ctypes.c_void_p
_dp = ctypes.POINTER(ctypes.c_double)


class PlanDesc(ctypes.Structure):
    _fields_ = [
        ("n_species", _c_int32), ("n_rank", _c_int32), ("method", _c_int32), ("order", _c_int32),
        ("mesh", _c_int32 * 3), ("ewald_ns", _c_int32 * 3), ("precision", _c_int32),
        ("has_cncorr", _c_int32), ("r_cut", _c_double), ("params", _c_double * 4),
        ("rcov", _dp), ("cnref", _dp), ("eigvecs", _dp), ("eigs", _dp), ("sqrtq", _dp),
        ("cncorr", _dp), ("deconv", ctypes.POINTER(ctypes.c_float)),
        ("cnfunc", _c_int32), ("rcov_cn", _dp), ("en", _dp),
    ]


CN_SMOOTH, CN_D4 = 0, 1
CNFUNCS = {"smooth_cut": CN_SMOOTH, "d4": CN_D4}


# symbol -> (restype, argtypes); mirrors include/fd3.h
_SIGS = {
    "fd3_plan_create": (ctypes.c_int, [ctypes.POINTER(PlanDesc), ctypes.POINTER(_vp)]),
    "fd3_plan_destroy": (ctypes.c_int, [_vp]),
    "fd3_plan_set_tuning": (ctypes.c_int, [_vp, _c_int32, _c_int32]),
    "fd3_plan_set_edge_cutoff": (ctypes.c_int, [_vp, _c_int32]),
    "fd3_plan_get_tuning":(ctypes.c_int, [_vp, _c_int32, ctypes.POINTER(_c_int32)]),
    "fd3_workspace_size": (ctypes.c_int, [_vp, _c_int64, _c_int64, ctypes.POINTER(ctypes.c_size_t)]),
    "fd3_edge_workspace_size": (ctypes.c_int, [_vp, _c_int64, _c_int64, ctypes.POINTER(ctypes.c_size_t)]),
    "fd3_cell_grid":(ctypes.c_int, [_dp, _c_double, ctypes.POINTER(_c_int32), ctypes.POINTER(_c_int32)]),
    "fd3_energy_edges": (ctypes.c_int, [_vp, _c_int64, _vp, _vp, _vp, _c_int64, _vp, _vp, _vp, _c_int32, _vp,
                                        ctypes.c_size_t, _vp, _vp, _vp, _vp, _vp]),
    "fd3_energy_forces_stress": (ctypes.c_int, [_vp, _c_int64, _vp, _vp, _dp, _vp, _c_double, _vp,
                                                ctypes.c_size_t, _vp, _vp, _vp, _vp]),
    "fd3_atom_terms": (ctypes.c_int, [_vp, _c_int64, _c_int64, _vp, ctypes.c_size_t, _vp, _vp, _vp]),
    "fd3_direct_workspace_size": (ctypes.c_int, [_vp, _c_int64, _dp, _c_double, _c_double,
                                                 ctypes.POINTER(ctypes.c_size_t)]),
    "fd3_direct_energy_forces_stress": (ctypes.c_int, [_vp, _c_int64, _vp, _vp, _dp, _vp, _c_double, _c_double,
                                                       _vp, ctypes.c_size_t, _vp, _vp, _vp, _vp]),
    "fd3_neighbor_workspace_size":(ctypes.c_int, [_c_int64, _dp, _c_double, ctypes.POINTER(ctypes.c_size_t)]),
    "fd3_neighbor_count": (ctypes.c_int, [_c_int64, _vp, _dp, _c_double, _vp, ctypes.c_size_t,
                                          ctypes.POINTER(_c_int64), _vp]),
    "fd3_neighbor_fill": (ctypes.c_int, [_c_int64, _vp, _dp, _c_double, _vp, ctypes.c_size_t, _c_int64, _vp, _vp,
                                         _vp, ctypes.POINTER(_c_int64), _vp]),
    "fd3_neighbor_fill_static": (ctypes.c_int, [_c_int64, _vp, _dp, _c_double, _c_int64, _vp, _vp, _vp,
                                                ctypes.POINTER(_c_int64), _vp]),
    "fd3_profile_enable": (ctypes.c_int, [_vp, _c_int32]),
    "fd3_profile_read": (ctypes.c_int, [_vp, _dp, _c_int32, ctypes.c_char_p, _c_int32, ctypes.POINTER(_c_int32)]),
    "fd3_last_error": (ctypes.c_char_p, []),
    "fd3_launch_count": (_c_int64, []),
}
EXPORTED = tuple(_SIGS)

_lock = threading.Lock()
_lib = None


def lib_path() -> str:
    return _LIB_PATH


_TORCH_LIB_PATH = os.path.join(os.path.dirname(_LIB_PATH), "libfd3_torch.so")
_ops_loaded = False


def ops():
    """``torch.ops.fd3``: the thin operator library over the C ABI (energy_forces_stress,
    energy_edges; CUDA kernels call libfd3 on the current stream, Meta kernels give shapes).
    Loaded once, after libfd3.so itself; raises if it has not been built."""
    global _ops_loaded
    if not _ops_loaded:
        lib()
        with _lock:
            if not _ops_loaded:
                if not os.path.exists(_TORCH_LIB_PATH):
                    raise RuntimeError(f"{_TORCH_LIB_PATH} is missing: build it with `python -m fourierd3_b200.build`")
                import torch

                torch.ops.load_library(_TORCH_LIB_PATH)
                _ops_loaded = True
    import torch

    return torch.ops.fd3


def handle(p: ctypes.c_void_p) -> int:
    """A plan pointer as the integer the operator library takes."""
    return int(p.value or 0)


def lib() -> ctypes.CDLL:
    """Load libfd3.so once; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(_LIB_PATH):
                raise RuntimeError(f"{_LIB_PATH} is missing: build it with `python -m fourierd3_b200.build`")
            h = ctypes.CDLL(_LIB_PATH)
            for name, (res, args) in _SIGS.items():
                f = getattr(h, name)
                f.restype = res
                f.argtypes = args
            _lib = h
    return _lib


def check(rc: int, what: str) -> None:
    if rc == FD3_OK:
        return
    msg = lib().fd3_last_error().decode(errors="replace")
    text = f"{what} failed with status {rc}: {msg}"
    if rc in (FD3_EINVAL, FD3_ECAPACITY, FD3_ENOMEM):
        raise ValueError(text)
    raise RuntimeError(text)


def launch_count() -> int:
    return int(lib().fd3_launch_count())


def dptr(arr) -> _dp:
    """ctypes double* to a C-contiguous float64 numpy array (host)."""
    return arr.ctypes.data_as(_dp)
