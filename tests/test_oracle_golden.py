"""The oracle restatement against fixtures produced by the reference's own code (CPU)."""
import functools

import numpy as np
import pytest

import golden_cases as gc
from oracle.neighbours import neighbour_list_cells as neighbour_list
from oracle.reference_port import OracleFourierD3


@functools.lru_cache(maxsize=8)
def _edges(key):
    rec = gc.load(key)
    i, j, S = neighbour_list(rec["positions"], rec["cell"], rec["config"]["r_cut"])
    return np.stack([i, j]), S


def _edge_key(name):
    # fixtures that share a structure share one neighbour build
    rec = gc.load(name)
    for other in gc.names():
        o = gc.load(other)
        if o["positions"].shape == rec["positions"].shape and np.array_equal(o["positions"], rec["positions"]):
            return other
    return name


@pytest.mark.parametrize("name", gc.names())
def test_oracle_matches_reference_fixture(name):
    rec = gc.load(name)
    cfg = rec["config"]
    kw = gc.model_kwargs(cfg)
    o = OracleFourierD3(rec["numbers"], rec["cell"], **kw)
    ei, S = _edges(_edge_key(name))
    assert ei.shape[1] == int(rec["n_edges"])
    e, f, s = o.calculate(rec["positions"], rec["cell"], edges=(ei, S))
    assert abs(e - float(rec["energy_ev"])) <= 1e-12 * abs(float(rec["energy_ev"]))
    np.testing.assert_allclose(f, rec["forces"], rtol=0, atol=1e-11)
    np.testing.assert_allclose(s, rec["stress"], rtol=0, atol=1e-13)
    assert np.array_equal(o.eigs.numpy(), rec["eigs"])
