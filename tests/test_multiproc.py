"""Multi-process (world size 2, gloo on CPU) coverage of the N>1 paths: the ensemble is
sharded across ranks with no exchange while stepping, replicas report the max time over
ranks, and per-member diagnostics are gathered on the host."""
import os
import socket

import numpy as np
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


def _step_worker(rank, world, port, q):
    """Each rank advances its shard of a small RBC ensemble two steps (the FP64 oracle on
    the CPU stands in for the GPU kernels, so the path runs here without a GPU) and the
    ranks gather the per-member Nusselt numbers on the host."""
    import datetime
    import math
    import sys
    import torch.distributed as dist
    import tarang_b200 as tb
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    from oracle import tarang_ref as R
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    members = [(16, 2e4 * (1 + k), 1.0) if k % 2 else (32, 1e4 * (1 + k), 1.0) for k in range(6)]
    mine = tb.shard_members(members, rank, world)
    kf = (math.pi, 2 * math.pi, 2 * math.pi)
    nu = {}
    for i in mine:
        N, Ra, Pr = members[i]
        g = R.Grid((N, N, N), kf, "SFF")
        cfg = R.RBCConfig(g, Ra=Ra, Pr=Pr, dt=1e-3)
        U = np.zeros((3,) + g.shape, complex)
        T = R.rbc_temperature_ic(g, 1e-3, 4.0, 3 + i)
        for _ in range(2):
            U, T = R.rbc_rk4_step(cfg, U, T)
        nu[i] = R.nusselt(cfg, U, T)
    gathered = [None] * world
    dist.all_gather_object(gathered, nu)
    if rank == 0:
        q.put((members, gathered))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.timeout(240)
def test_sharded_ensemble_steps_and_gathers_two_ranks():
    """Two gloo ranks each step their shard (no exchange while stepping) and gather the
    per-member Nusselt numbers: every member once, equal bit for bit to stepping it alone."""
    import math
    from oracle import tarang_ref as R
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_step_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    members, gathered = q.get(timeout=220)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert not set(gathered[0]) & set(gathered[1])
    merged = {**gathered[0], **gathered[1]}
    assert sorted(merged) == list(range(len(members)))
    kf = (math.pi, 2 * math.pi, 2 * math.pi)
    for i in (0, 5):
        N, Ra, Pr = members[i]
        g = R.Grid((N, N, N), kf, "SFF")
        cfg = R.RBCConfig(g, Ra=Ra, Pr=Pr, dt=1e-3)
        U = np.zeros((3,) + g.shape, complex)
        T = R.rbc_temperature_ic(g, 1e-3, 4.0, 3 + i)
        for _ in range(2):
            U, T = R.rbc_rk4_step(cfg, U, T)
        assert merged[i] == R.nusselt(cfg, U, T)
        assert math.isfinite(merged[i]) and merged[i] > 0.99
