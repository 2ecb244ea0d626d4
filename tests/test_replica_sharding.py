"""Replicas across ranks (one process per GPU, no collective on the step
path): whole replicas go to ranks, balanced by cost. Run here as two `gloo`
ranks on the CPU: each rank computes its own shard of the same seeded
replica set, the ranks exchange them, and the shards must partition the set
with the costs balanced; the timing reduction (the max over ranks) is checked
the same way."""

import os
import socket

import pytest
import torch.multiprocessing as mp


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def worker(rank, world, port, out):
    import datetime
    import sys

    import torch
    import torch.distributed as dist

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, os.path.join(root, "virial-engine_b200"))
    import virial_lj as vl

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    reps = vl.uneven_replicas(64, 2024, sizes=(500, 2000))
    mine = vl.shard_replicas(reps, world)[rank]
    shards = [None] * world
    dist.all_gather_object(shards, mine)
    loads = [sum(vl.replica_cost(reps[i]) for i in s) for s in shards]
    # each rank's own step time, reduced to the slowest rank
    t = torch.tensor([1.0 + rank], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    if rank == 0:
        out.put((shards, loads, max(vl.replica_cost(r) for r in reps), float(t.item())))
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2])
def test_shards_partition_and_balance_across_gloo_ranks(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    shards, loads, biggest, slowest = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    every = sorted(i for s in shards for i in s)
    assert every == list(range(64))
    # longest-first greedy: no rank exceeds another by more than one replica
    assert max(loads) - min(loads) <= biggest
    assert slowest == float(world)


def test_one_rank_takes_everything():
    import virial_lj as vl
    reps = vl.uneven_replicas(8, 7, sizes=(500, 1000))
    assert vl.shard_replicas(reps, 1) == [list(range(8))]
    with pytest.raises(ValueError):
        vl.shard_replicas(reps, 0)
