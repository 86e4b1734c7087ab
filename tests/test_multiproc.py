"""Multi-process (world size 2, gloo on CPU) coverage of the N>1 paths: the ensemble is
sharded across ranks with no exchange while stepping, replicas report the max time over
ranks, and per-member diagnostics are gathered on the host."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import datetime
    import torch
    import torch.distributed as dist
    import tarang_b200 as tb
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    members = tb.ensemble_members()
    mine = tb.shard_members(members, rank, world)
    # gather every rank's shard and a per-member diagnostic (here: the member's cost)
    shards = [None] * world
    dist.all_gather_object(shards, mine)
    load = torch.tensor([float(sum(members[i][0] ** 3 for i in mine))])
    loads = [torch.zeros(1) for _ in range(world)]
    dist.all_gather(loads, load)
    # replica timing: the reported time is the max over ranks
    t = torch.tensor([1.0 + rank])
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    if rank == 0:
        q.put((shards, [float(x) for x in loads], float(t)))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_ensemble_sharding_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    shards, loads, tmax = q.get(timeout=100)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    allidx = sorted(shards[0] + shards[1])
    assert allidx == list(range(64))            # every member on exactly one rank
    assert not set(shards[0]) & set(shards[1])
    assert abs(loads[0] - loads[1]) / max(loads) < 0.05   # N^3 cost balanced
    assert tmax == 2.0
