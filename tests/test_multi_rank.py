"""Multi-rank host logic on CPU (gloo, world size 2): every rank computes the
same planet assignment, every planet is owned exactly once, and the job time
is the maximum over ranks."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

from conftest import PKG

import ggb_shard


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, costs, out):
    sys.path.insert(0, PKG)
    import datetime

    import torch
    import torch.distributed as dist

    import ggb_shard as S
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    owned, loads = S.assign(costs, world)
    mine = owned[rank]
    # each rank "times" its own planets: the job time is the max over ranks
    t_local = float(sum(costs[i] for i in mine))
    t_max = S.max_over_ranks(t_local, dist)
    gathered = [None] * world
    dist.all_gather_object(gathered, owned)
    out[rank] = (mine, t_local, t_max, gathered)
    dist.barrier()
    dist.destroy_process_group()


def test_assignment_is_a_partition_and_balanced():
    costs = [ggb_shard.planet_cost(N, p, R) for N, p, R in
             [(64, 100_000, 512), (128, 500_000, 1024), (256, 1_000_000, 1024), (64, 300_000, 512),
              (256, 700_000, 512), (128, 100_000, 512), (512, 1_000_000, 1024)]]
    for world in (1, 2, 3, 8):
        owned, loads = ggb_shard.assign(costs, world)
        flat = sorted(i for o in owned for i in o)
        assert flat == list(range(len(costs)))
        assert max(loads) <= sum(costs) / world + max(costs)


def test_two_gloo_ranks_agree():
    costs = [float(c) for c in (5, 3, 8, 1, 9, 2, 7)]
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    manager = ctx.Manager()
    out = manager.dict()
    procs = [ctx.Process(target=_rank, args=(r, world, port, costs, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    owned0 = out[0][3]
    assert out[1][3] == owned0                    # identical plans on every rank
    assert sorted(out[0][0] + out[1][0]) == list(range(len(costs)))
    tmax = max(out[0][1], out[1][1])
    assert out[0][2] == tmax and out[1][2] == tmax


def test_batch_workload_is_deterministic_and_sharded():
    """The batched workload's 64 planets (bench.batch_specs) are the same on
    every call and rank, drawn from the stated ranges, and every planet goes
    to exactly one rank."""
    import importlib.util
    root = os.path.dirname(PKG)
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(root, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    a, b = bench.batch_specs(), bench.batch_specs()
    assert a == b and len(a) == 64
    assert {p["N"] for p in a} <= {64, 128, 256} and {p["R"] for p in a} <= {512, 1024}
    assert all(100_000 <= p["particles"] <= 1_000_000 and p["bands"] in (4, 8, 12) for p in a)
    assert all(2.0 <= p["noise_scale"] <= 5.0 for p in a) and len({p["seed"] for p in a}) == 64
    costs = [ggb_shard.planet_cost(p["N"], p["particles"], p["R"]) for p in a]
    for world in (1, 2, 4, 8):
        owned, loads = ggb_shard.assign(costs, world)
        assert sorted(i for o in owned for i in o) == list(range(64))
        assert max(loads) <= sum(costs) / world + max(costs)
