"""Element tables, the synthetic C6 stand-in and the rank search (CPU)."""
import numpy as np

from fourierd3_b200 import tables


def test_tables_shapes_and_dtypes():
    t = tables.load_tables()
    assert t["cnref"].shape == (104, 7) and t["cnref"].dtype == np.float32
    for k in ("rcov", "sqrtQz", "rcov_cn"):
        assert t[k].shape == (119,) and t[k].dtype == np.float32
    assert t["en"].dtype == np.float64


def test_synthetic_c6_properties():
    types = [1, 6, 8, 14, 26]
    blk = tables.synthetic_c6ref_block(types)
    assert blk.shape == (5, 5, 7, 7) and blk.dtype == np.float32
    m = tables.c6ref_matrix(types)
    np.testing.assert_array_equal(m, m.T)                       # symmetric under (Za,p) <-> (Zb,q)
    cnref = tables.load_tables()["cnref"][types]
    valid = (cnref != -1).reshape(-1)
    assert np.all(m[valid][:, valid] > 0)                       # positive where both slots used
    assert np.all(m[~valid] == 0) and np.all(m[:, ~valid] == 0)  # zero where a slot is unused


def test_decomp_meets_tolerance_and_is_deterministic():
    for tol in (1.0, 1e-2):
        e1, v1, err = tables.decomp([8, 14], tol)
        e2, v2, _ = tables.decomp([8, 14], tol)
        assert err * 100 < tol
        np.testing.assert_array_equal(e1, e2)
        np.testing.assert_array_equal(v1, v2)
    # tighter tolerance -> at least as many ranks
    assert len(tables.decomp([8, 14], 1e-4)[0]) >= len(tables.decomp([8, 14], 1.0)[0])


def test_c6_source_label_default_synthetic(monkeypatch):
    monkeypatch.delenv("FD3_C6REF", raising=False)
    assert tables.c6_source() == "synthetic"
