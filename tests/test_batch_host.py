"""Host-side logic of the batch runner: LPT lane/rank split and the cost model, plus the
two-rank shard exchange over ``gloo`` (the multi-GPU batch path shards structures across
ranks with no data-path collective; only the result indices are gathered)."""
import os
import socket

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def test_lpt_split_is_a_balanced_partition():
    from fourierd3_b200.batch import lpt_split

    rng = np.random.default_rng(0)
    costs = list(np.exp(rng.uniform(0, 6, 97)))
    for parts in (1, 2, 3, 8):
        bins = lpt_split(costs, parts)
        flat = sorted(i for b in bins for i in b)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[i] for i in b) for b in bins]
        # LPT bound: makespan <= 4/3 OPT, and OPT >= max(mean load, largest item)
        opt_lb = max(sum(costs) / parts, max(costs))
        assert max(loads) <= 4.0 / 3.0 * opt_lb + 1e-9


def test_cost_model_counts_mesh_channels():
    from fourierd3_b200 import structures as st
    from fourierd3_b200.batch import structure_cost

    pos, cell, z = st.sio2_box(0)
    c = structure_cost(z, cell)
    # 648 atoms, 64^3 mesh, two species times the C6 rank
    from fourierd3_b200 import engine

    setup = engine.species_setup(z, 1.0)
    assert c == 648 + 64 ** 3 * 2 * setup.n_rank


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, costs, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from fourierd3_b200.batch import lpt_split

    mine = sorted(lpt_split(costs, world)[rank])
    t = torch.full((len(costs),), -1, dtype=torch.int64)
    t[: len(mine)] = torch.tensor(mine, dtype=torch.int64)
    parts = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(parts, t)
    if rank == 0:
        q.put([p[p >= 0].tolist() for p in parts])
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_shards_cover_the_batch():
    rng = np.random.default_rng(1)
    costs = [float(v) for v in np.exp(rng.uniform(0, 5, 40))]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, costs, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert sorted(got[0] + got[1]) == list(range(40))
    assert not set(got[0]) & set(got[1])


def test_lpt_split_more_parts_than_items_and_ties():
    from fourierd3_b200.batch import lpt_split

    bins = lpt_split([3.0, 1.0], 4)
    assert bins == [[0], [1], [], []]
    # equal costs: heaviest-first order breaks ties by index, bins by their own index
    assert lpt_split([1.0, 1.0, 1.0, 1.0], 2) == [[0, 2], [1, 3]]


def test_shard_covers_the_batch_and_checks_the_rank():
    import pytest

    from fourierd3_b200 import structures as st
    from fourierd3_b200.batch import shard

    structs = [st.random_box(k, 24 + 8 * k, z_max=18) for k in range(7)]
    for world in (1, 2, 3):
        parts = [shard(structs, r, world) for r in range(world)]
        assert sorted(i for p in parts for i in p) == list(range(len(structs)))
        assert all(p == sorted(p) for p in parts)
    for bad in (-1, 3):
        with pytest.raises(ValueError):
            shard(structs, bad, 3)


def test_batch_refuses_empty_input_and_non_cuda_devices():
    import pytest

    from fourierd3_b200 import structures as st
    from fourierd3_b200.batch import D3Batch

    with pytest.raises(ValueError):
        D3Batch([])
    with pytest.raises(RuntimeError):
        D3Batch([st.random_box(0, 24, z_max=18)], device="cpu")
