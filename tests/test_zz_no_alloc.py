"""The allocation-free neighbour build (fd3_neighbor_fill_static) through the C ABI.

Some callers cannot allocate device memory themselves -- an MD engine or host runtime that
owns all device memory and forbids raw allocations during its timestep, or code with a fixed
memory budget. For them the library offers a neighbour build whose scratch is a fixed array
inside libfd3. This test checks that it returns exactly what the workspace-based entry point
returns, on two calls in a row (the shared scratch keeps the previous call's contents, so the
second call must not depend on them), and that an input too large for the fixed scratch is
rejected with a clear error. The file is named so that pytest collects it last.
"""
import ctypes

import numpy as np
import pytest
import torch

from fourierd3_b200 import _native, neighbour_list, structures

pytestmark = pytest.mark.gpu


def _static_fill(pos, cell, r_cut, capacity):
    lib = _native.lib()
    cell_h = np.ascontiguousarray(cell, dtype=np.float64).reshape(9)
    src = torch.full((capacity,), -1, dtype=torch.int64, device=pos.device)
    dst = torch.full((capacity,), -1, dtype=torch.int64, device=pos.device)
    sh = torch.full((capacity, 3), 7, dtype=torch.int32, device=pos.device)
    count = ctypes.c_int64(-1)
    rc = lib.fd3_neighbor_fill_static(pos.shape[0], ctypes.c_void_p(pos.data_ptr()), _native.dptr(cell_h),
                                      float(r_cut), capacity, ctypes.c_void_p(src.data_ptr()),
                                      ctypes.c_void_p(dst.data_ptr()), ctypes.c_void_p(sh.data_ptr()),
                                      ctypes.byref(count), ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    return rc, int(count.value), src, dst, sh


@pytest.mark.parametrize("box", ["sio2", "hcno"])
def test_static_scratch_matches_workspace_entry_point(box, cuda_device):
    if box == "sio2":
        p, c, _ = structures.sio2_box(0)
    else:
        p, c, _ = structures.hcno_box(seed=3, n_atoms=240)
    pos = torch.tensor(p, dtype=torch.float64, device=cuda_device)
    i_ref, j_ref, s_ref = neighbour_list(pos, c, 6.0)          # workspace-based fd3_neighbor_fill
    n_ref = i_ref.numel()
    for _ in range(2):                                          # two calls in a row on the shared scratch
        rc, count, src, dst, sh = _static_fill(pos, c, 6.0, n_ref)
        assert rc == _native.FD3_OK, _native.lib().fd3_last_error()
        assert count == n_ref
        torch.cuda.synchronize()
        np.testing.assert_array_equal(src.cpu().numpy(), i_ref.cpu().numpy())
        np.testing.assert_array_equal(dst.cpu().numpy(), j_ref.cpu().numpy())
        np.testing.assert_array_equal(sh.cpu().numpy(), s_ref.cpu().numpy())


def test_static_scratch_reports_needed_capacity(cuda_device):
    """An output one row too short: FD3_ECAPACITY, with the needed row count written back."""
    p, c, _ = structures.sio2_box(0)
    pos = torch.tensor(p, dtype=torch.float64, device=cuda_device)
    n_ref = neighbour_list(pos, c, 6.0)[0].numel()
    rc, count, *_ = _static_fill(pos, c, 6.0, n_ref - 1)
    assert rc == _native.FD3_ECAPACITY
    assert count == n_ref


def test_static_scratch_rejects_oversize_input(cuda_device):
    p, c, _ = structures.sio2_box(0)
    big = structures.replicate(p, c, np.zeros(len(p), dtype=np.int64), (5, 5, 5))   # 81,000 atoms
    pos = torch.tensor(big[0], dtype=torch.float64, device=cuda_device)
    rc, count, *_ = _static_fill(pos, big[1], 6.0, 16)
    assert rc == _native.FD3_EINVAL
    msg = _native.lib().fd3_last_error().decode()
    assert "static scratch" in msg and "bytes" in msg
