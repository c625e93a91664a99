"""The multi-GPU host logic on CPU: two gloo ranks (world size 2) split a
batch by estimated cost and check, through collectives, that the ranges are
disjoint, cover the batch and are balanced; that weak-scaling ranks generate
distinct batches; and that the max-over-ranks reduction bench.py uses for its
timed interval returns the slowest rank's time."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from lmie_b200 import shard, workloads


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        cases = workloads.batched_uneven(64)
        a, b = shard.strong_slice(cases, rank, world)
        got = [None] * world
        dist.all_gather_object(got, (a, b))
        costs = [shard.case_cost(c) for c in cases]
        loads = [sum(costs[x:y]) for x, y in got]
        own = workloads.batched_uneven(4, seed=shard.weak_seed(workloads.SEED, rank))
        firsts = [None] * world
        dist.all_gather_object(firsts, (own[0].lam, own[0].a1))
        t = torch.tensor([0.5 + rank], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        q.put((rank, got, loads, firsts, float(t.item())))
    finally:
        dist.destroy_process_group()


def test_two_ranks_split_and_reduce():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, got, loads, firsts, tmax in res:
        (a0, b0), (a1, b1) = got
        assert a0 == 0 and b0 == a1 and b1 == 64          # disjoint and covering, in order
        assert max(loads) <= 1.5 * (sum(loads) / world)    # balanced within the largest case
        assert firsts[0] != firsts[1]                      # weak scaling: distinct batches
        assert tmax == 1.5                                 # the slowest rank's time


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_balanced_ranges_properties(world):
    rng = np.random.default_rng(world)
    costs = list(rng.uniform(1, 100, 50) ** 2)
    r = shard.balanced_ranges(costs, world)
    assert r[0][0] == 0 and r[-1][1] == 50
    assert all(r[i][1] == r[i + 1][0] for i in range(world - 1))
    assert all(b > a for a, b in r)
    loads = [sum(costs[a:b]) for a, b in r]
    assert max(loads) <= sum(costs) / world + max(costs)
