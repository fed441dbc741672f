"""Host-side planning of batched streams (CPU): the per-stream cost model,
the longest-first assignment of streams to GPUs, and that every rank of a
multi-GPU job derives the same assignment (gloo, world size 2)."""
import os
import socket

import numpy as np
import pytest


def lpt(costs, ranks):
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * ranks
    out = [0] * len(costs)
    for i in order:
        r = min(range(ranks), key=lambda q: (load[q], q))
        out[i] = r
        load[r] += costs[i]
    return out


def test_stream_cost_orders_workloads(of):
    c1, c2 = of.CONFIGS["c1"], of.CONFIGS["c2"]
    assert of.stream_cost(c2) > of.stream_cost(c1) > 0
    cs = of.c4_configs(count=64)
    assert len({(c.width, c.resolution) for c in cs}) >= 6
    for c in cs:
        assert c.width in (160, 320, 640) and c.resolution in (128, 256, 512)
        assert 2000.0 <= c.size_mm <= 3000.0


def test_shard_is_longest_first_greedy(of):
    rng = np.random.default_rng(3)
    for ranks in (1, 2, 3, 8):
        costs = [float(x) for x in rng.integers(1, 1000, 37)]
        plan = of.shard(costs, ranks)
        assert plan == lpt(costs, ranks)
        load = np.zeros(ranks)
        for i, r in enumerate(plan):
            assert 0 <= r < ranks
            load[r] += costs[i]
        assert load.max() <= sum(costs) / ranks + max(costs)
    assert of.shard([], 4) == []


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import torch.distributed as dist
    import torch
    import openfusion_b200 as of
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    try:
        cs = of.c4_configs(count=64)
        plan = of.shard([of.stream_cost(c) for c in cs], world)
        mine = [i for i, r in enumerate(plan) if r == rank]
        got = [None] * world
        dist.all_gather_object(got, (plan, mine))
        q.put((rank, got))
    finally:
        dist.destroy_process_group()


def test_every_rank_derives_the_same_shard_plan():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    world = 2
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for _, got in results:
        plans = [g[0] for g in got]
        assert plans[0] == plans[1]
        shares = [g[1] for g in got]
        assert sorted(shares[0] + shares[1]) == list(range(64))
        assert shares[0] and shares[1]
