"""Host-side helpers of bench.py that its roofline figures rest on: the count of mesh values the
atoms' stencils touch (the gather's algorithmic bytes) against a brute-force set of stencil
points, and the per-stage algorithmic byte formulas on a hand-checked case."""
import itertools
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))


def _brute_touched(pos, cell, numbers, mesh, order):
    n = np.asarray(mesh)
    u = (np.asarray(pos) @ np.linalg.inv(np.asarray(cell))) * n
    pts = set()
    for ui, z in zip(u, numbers):
        # SPME centring: nearest point for odd orders, the point below for even ones
        ref = np.round(ui).astype(int) if order % 2 else np.floor(ui).astype(int)
        lo = -(order // 2) if order % 2 else -(order // 2 - 1)
        for d in itertools.product(range(lo, lo + order), repeat=3):
            pts.add((int(z), *((ref + np.array(d)) % n).tolist()))
    return len(pts)


def test_touched_mesh_values_match_a_brute_force_count():
    import bench

    rng = np.random.default_rng(4)
    cell = np.array([[9.0, 0.0, 0.0], [1.5, 8.0, 0.0], [0.5, -1.0, 10.0]])
    for n_atoms, mesh, order in ((5, (8, 8, 8), 5), (12, (10, 12, 9), 4), (30, (6, 7, 8), 6)):
        pos = rng.uniform(0, 1, (n_atoms, 3)) @ cell
        numbers = rng.choice([8, 14, 1], n_atoms)
        for R in (1, 3):
            want = _brute_touched(pos, cell, numbers, mesh, order) * R
            assert bench.touched_mesh_values(pos, cell, numbers, mesh, order, R) == want


def test_stage_bytes_formulas():
    import bench

    mesh, C, n, R = (4, 6, 8), 6, 10, 3
    M, Mh = 4 * 6 * 8, 4 * 6 * 5
    for b in (4, 8):
        assert bench.stage_bytes("fft_r2c", n, mesh, C, R, b) == C * M * b + C * Mh * 2 * b
        assert bench.stage_bytes("fft_c2r", n, mesh, C, R, b) == C * M * b + C * Mh * 2 * b
        assert bench.stage_bytes("spread", n, mesh, C, R, b) == C * M * b + n * (28 + 8 * R)
    # the float64 filter also reads the float32 window table once per k-point
    assert bench.stage_bytes("filter", n, mesh, C, R, 8) == 2 * C * Mh * 16 + Mh * 4
    assert bench.stage_bytes("filter", n, mesh, C, R, 4) == 2 * C * Mh * 8
    # the gather reads the touched values when they are given, else the whole mesh
    assert bench.stage_bytes("gather", n, mesh, C, R, 4, touched=100) == 400 + n * (60 + 16 * R)
    assert bench.stage_bytes("gather", n, mesh, C, R, 4) == C * M * 4 + n * (60 + 16 * R)
    assert bench.stage_bytes("unknown", n, mesh, C, R, 4) == 0.0
