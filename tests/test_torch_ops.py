"""The operator layer over the C ABI (torch.ops.fd3, fourierd3_b200/_lib/libfd3_torch.so): it
loads, registers both operators with their schemas, and its Meta kernels give the output shapes
(what torch.compile / export trace with). No GPU: nothing is computed."""
import os

import pytest
import torch

from fourierd3_b200 import _native

pytestmark = pytest.mark.skipif(not os.path.exists(_native._TORCH_LIB_PATH), reason="operator library not built")


def test_ops_register_with_schemas():
    ops = _native.ops()
    s1 = str(ops.energy_forces_stress.default._schema)
    s2 = str(ops.energy_edges.default._schema)
    assert "Tensor? cell_dev=None" in s1 and s1.endswith("-> (Tensor, Tensor, Tensor)")
    assert "bool need_grad" in s2 and s2.endswith("-> (Tensor, Tensor, Tensor, Tensor)")


def test_meta_kernels_give_shapes():
    ops = _native.ops()
    meta = dict(device="meta")
    pos = torch.empty(17, 3, dtype=torch.float64, **meta)
    sp = torch.empty(17, dtype=torch.int32, **meta)
    work = torch.empty(64, dtype=torch.uint8, **meta)
    e, f, s = ops.energy_forces_stress(0, pos, sp, torch.eye(3, dtype=torch.float64), 6.0, work)
    assert e.shape == () and f.shape == (17, 3) and s.shape == (3, 3) and f.dtype == torch.float64
    ei = torch.empty(40, dtype=torch.int64, **meta)
    e, gp, gs, gc = ops.energy_edges(0, pos, sp, torch.empty(3, 3, dtype=torch.float64, **meta), ei, ei,
                                     torch.empty(40, 3, dtype=torch.float64, **meta), True, work)
    assert gp.shape == (17, 3) and gs.shape == (40, 3) and gc.shape == (3, 3)
