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


def _rank_matvecs(rank, world, port, result_q):
    """Each rank takes its LPT shard (flop cost model) of a small Hubbard batch, computes its
    problems' matvecs (the oracle stands in for the device path on CPU) and the results are
    gathered by problem index."""
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta

    import numpy as np
    from cytnx_b200.batch import problem_flops
    from oracle import workloads as OW

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        dims = [40, 96, 17, 64, 128, 33]
        costs = [problem_flops(p) for p in W.hubbard_batch(dims)]
        mine = shard_problems(costs, world)[rank]
        local = {i: OW.heff_matvec(OW.hubbard_two_site(dims[i], 100 + i)) for i in mine}
        gathered = [None] * world
        dist.all_gather_object(gathered, local)
        if rank == 0:
            merged = {}
            for g in gathered:
                merged.update(g)
            result_q.put(({i: v.tolist() for i, v in merged.items()}, costs))
    finally:
        dist.destroy_process_group()


def test_sharded_matvecs_gather_to_the_single_rank_result():
    import numpy as np
    from oracle import workloads as OW

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_matvecs, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    try:
        merged, costs = q.get(timeout=180)
    finally:
        for p in procs:
            p.join(timeout=180)
    assert all(p.exitcode == 0 for p in procs)
    dims = [40, 96, 17, 64, 128, 33]
    assert sorted(merged) == list(range(len(dims)))
    for i, D in enumerate(dims):
        ref = OW.heff_matvec(OW.hubbard_two_site(D, 100 + i))
        assert np.array_equal(np.asarray(merged[i]), ref)
    # the cost model is the algorithmic flop count: larger problems cost more
    assert costs[4] > costs[1] > costs[0] > costs[2]
