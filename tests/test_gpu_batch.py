"""GPU checks of the batch runner (fourierd3_b200.batch.D3Batch).

* eager and graph-replayed batch results equal the per-structure ``D3Model`` results bit
  for bit (the fused path is deterministic: segment-sorted cell lists and mesh tiles,
  tile-owned spreading, fixed-order block reductions), for 1 and several lanes;
* one structure of the batch matches the float64 oracle (energy 1e-10 relative, forces
  1e-8 eV/A, stress 1e-10 eV/A^3), so the batch path inherits the drop-in parity;
* positions updated in place are picked up by a graph replay;
* the host-I/O graph (run_host: positions copied in and results out inside one replay) equals
  the device path bit for bit, and so does every evaluation of the two-slot host pipeline;
* the lane autotuner picks one of its candidates and writes its cache.
"""
import json

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _structures(n=12, seed=7, n_max=384):
    from fourierd3_b200 import structures as st

    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(24), np.log(n_max), n)).astype(int)
    out = []
    for k, m in enumerate(sizes):
        # a handful of elements per structure keeps the oracle check fast
        pos, cell, z = st.random_box(seed * 1000 + k, int(m), z_max=18 if k % 2 else 54)
        out.append((pos, cell, z))
    return out


KW = dict(method="spme", mesh_spacing=1.2, interpolation_nodes=5, c6tol=1.0, r_cut=6.0)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_equals_single_structure_calls(precision, cuda_device):
    from fourierd3_b200 import D3Model
    from fourierd3_b200.batch import D3Batch

    structs = _structures()
    singles = []
    for pos, cell, z in structs:
        e, f, s = D3Model(z, cell, precision=precision, device=cuda_device, **KW)(pos, cell)
        singles.append((e.clone(), f.clone(), s.clone()))
    for lanes in (1, 3):
        b = D3Batch(structs, precision=precision, lanes=lanes, device=cuda_device, **KW)
        for mode in ("eager", "graph"):
            if mode == "graph":
                b.capture()
            e, f, s = b()
            torch.cuda.synchronize()
            fs = b.split_forces(f)
            for i, (e1, f1, s1) in enumerate(singles):
                assert torch.equal(e[i], e1), (lanes, mode, i, float(e[i]), float(e1))
                assert torch.equal(fs[i], f1), (lanes, mode, i)
                assert torch.equal(s[i], s1), (lanes, mode, i)


def test_batch_member_matches_oracle(cuda_device):
    from fourierd3_b200.batch import D3Batch
    from oracle.reference_port import OracleFourierD3

    structs = _structures(n=5)
    b = D3Batch(structs, precision="fp64", lanes=2, device=cuda_device, **KW)
    b.capture()
    e, f, s = b()
    k = 1   # a z_max=18 structure: few species, quick on the CPU
    pos, cell, z = structs[k]
    e_ref, f_ref, s_ref = OracleFourierD3(z, cell, **KW).calculate(pos, cell)
    assert abs(float(e[k]) - e_ref) <= 1e-10 * abs(e_ref)
    assert np.abs(b.split_forces()[k].cpu().numpy() - f_ref).max() <= 1e-8
    assert np.abs(s[k].cpu().numpy() - s_ref).max() <= 1e-10


def test_replay_sees_new_positions(cuda_device):
    from fourierd3_b200 import D3Model
    from fourierd3_b200.batch import D3Batch

    structs = _structures(n=6)
    b = D3Batch(structs, precision="mixed", lanes=2, device=cuda_device, **KW)
    b.capture()
    rng = np.random.default_rng(3)
    moved = [(p + rng.normal(0.0, 0.02, p.shape), c, z) for p, c, z in structs]
    e, f, s = b([torch.from_numpy(p) for p, _, _ in moved])
    torch.cuda.synchronize()
    for i, (pos, cell, z) in enumerate(moved):
        e1, f1, s1 = D3Model(z, cell, precision="mixed", device=cuda_device, **KW)(pos, cell)
        assert torch.equal(e[i], e1)
        assert torch.equal(b.split_forces()[i], f1)
        assert torch.equal(s[i], s1)


def test_run_host_matches_device_call(cuda_device):
    """run_host (one graph replay with the host positions copied in and every result copied out)
    gives the device-path results bit for bit, picks up new host positions, and leaves the
    device-I/O graph (__call__) reading the device positions."""
    from fourierd3_b200.batch import D3Batch

    structs = _structures(n=5)
    b = D3Batch(structs, precision="mixed", lanes=2, device=cuda_device, **KW)
    b.capture()
    e0, f0, s0 = (t.clone() for t in b())
    h = b.host_buffers()
    assert h["positions"].is_pinned() and h["forces"].is_pinned()
    e, f, s = b.run_host()
    torch.cuda.synchronize()
    assert torch.equal(e, e0.cpu()) and torch.equal(f, f0.cpu()) and torch.equal(s, s0.cpu())
    rng = np.random.default_rng(5)
    moved = np.concatenate([p + rng.normal(0.0, 0.02, p.shape) for p, _, _ in structs])
    h["positions"].copy_(torch.from_numpy(moved))
    e2, f2, s2 = b.run_host()
    torch.cuda.synchronize()
    ed, fd, sd = (t.cpu() for t in b(torch.from_numpy(moved)))
    torch.cuda.synchronize()
    assert torch.equal(e2, ed) and torch.equal(f2, fd) and torch.equal(s2, sd)
    assert not torch.equal(e2, e0.cpu())
    # the device-I/O graph still follows the device positions
    back = torch.from_numpy(np.concatenate([p for p, _, _ in structs]))
    e3, _, _ = b(back)
    torch.cuda.synchronize()
    assert torch.equal(e3, e0)


def test_host_pipeline_matches_device_calls(cuda_device):
    """The two-slot host pipeline (copies of one evaluation beside the other's compute) gives,
    for every evaluation of a stream of different positions, the device-path results bit for
    bit, each in its own slot's host buffers."""
    from fourierd3_b200.batch import D3Batch

    structs = _structures(n=5)
    b = D3Batch(structs, precision="mixed", lanes=2, device=cuda_device, **KW)
    b.capture()
    rng = np.random.default_rng(11)
    base = np.concatenate([p for p, _, _ in structs])
    stream = [base + rng.normal(0.0, 0.02, base.shape) for _ in range(5)]
    expect = []
    for p in stream:
        e, f, s = b(torch.from_numpy(p))
        expect.append((e.cpu(), f.cpu(), s.cpu()))
    torch.cuda.synchronize()
    pipe = b.host_pipeline()
    assert pipe.host[0]["positions"].is_pinned() and pipe.host[1]["forces"].is_pinned()
    got = [None] * len(stream)

    def collect(k):
        h = pipe.wait(k % 2)
        got[k] = (h["energy"].clone(), h["forces"].clone(), h["stress"].clone())

    for k, p in enumerate(stream):
        s = k % 2
        if k >= 2:
            collect(k - 2)
        else:
            pipe.wait(s)
        pipe.host[s]["positions"].copy_(torch.from_numpy(p))
        pipe.submit(s)
    collect(len(stream) - 2)
    collect(len(stream) - 1)
    for (e, f, s), (ed, fd, sd) in zip(got, expect):
        assert torch.equal(e, ed) and torch.equal(f, fd) and torch.equal(s, sd)
    assert not torch.equal(got[0][0], got[1][0])
    # the batch's own graph still reads the batch's device positions
    e3, _, _ = b(torch.from_numpy(stream[2]))
    torch.cuda.synchronize()
    assert torch.equal(e3.cpu(), expect[2][0])


def test_autotune_lanes_caches(tmp_path, cuda_device):
    from fourierd3_b200.batch import D3Batch, autotune_lanes

    structs = _structures(n=8)
    b = D3Batch(structs, precision="mixed", device=cuda_device, **KW)
    cache = str(tmp_path / "tune.json")
    best = autotune_lanes(b, (1, 2, 4), cache=cache, reps=2)
    assert best in (1, 2, 4)
    table = json.load(open(cache))
    assert table[b.signature()]["lanes"] == best
    b2 = D3Batch(structs, precision="mixed", device=cuda_device, **KW)
    assert autotune_lanes(b2, (1, 2, 4), cache=cache) == best


def test_forward_batch_surface(cuda_device):
    from fourierd3_b200 import D3Model, forward_batch

    structs = _structures(n=4)
    res = forward_batch([(torch.from_numpy(p), c, z) for p, c, z in structs], precision="fp64",
                        device=cuda_device, **KW)
    for (pos, cell, z), (e, f, s) in zip(structs, res):
        e1, f1, s1 = D3Model(z, cell, precision="fp64", device=cuda_device, **KW)(pos, cell)
        assert torch.equal(e, e1) and torch.equal(f, f1) and torch.equal(s, s1)
