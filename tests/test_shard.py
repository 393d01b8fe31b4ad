"""Sharding of batched problems over ranks (the N>1 path of the batched workload):
every rank computes the same longest-processing-time assignment on its own, the shards
partition the problems, and the load is balanced.  Runs as world_size-2 gloo ranks on CPU."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from cytnx_b200.batch import shard_problems
from cytnx_b200 import workloads as W


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, result_q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        dims = W.hubbard_batch_dims(256, seed=0)
        costs = [float(d) ** 3 for d in dims]
        mine = shard_problems(costs, world)[rank]
        # every rank reports its shard; rank 0 checks the union
        sizes = [None] * world
        dist.all_gather_object(sizes, mine)
        load = torch.tensor([sum(costs[i] for i in mine)], dtype=torch.float64)
        loads = [torch.zeros(1, dtype=torch.float64) for _ in range(world)]
        dist.all_gather(loads, load)
        if rank == 0:
            result_q.put((sizes, [float(x.item()) for x in loads], sum(costs), max(costs)))
    finally:
        dist.destroy_process_group()


def test_lpt_shards_partition_and_balance():
    costs = [float(d) ** 3 for d in W.hubbard_batch_dims(256, seed=0)]
    for n in (1, 2, 3, 4, 8):
        sh = shard_problems(costs, n)
        flat = sorted(i for s in sh for i in s)
        assert flat == list(range(256))
        loads = [sum(costs[i] for i in s) for s in sh]
        # LPT bound: max load <= mean + largest item
        assert max(loads) <= sum(costs) / n + max(costs) + 1e-6
        assert sh == shard_problems(costs, n)  # deterministic
    with pytest.raises(Exception):
        shard_problems(costs, 0)


def test_two_gloo_ranks_agree_on_shards():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    try:
        shards, loads, total, biggest = q.get(timeout=120)
    finally:
        for p in procs:
            p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    assert sorted(shards[0] + shards[1]) == list(range(256))
    assert not set(shards[0]) & set(shards[1])
    assert abs(sum(loads) - total) <= 1e-6 * total
    assert max(loads) - min(loads) <= biggest
