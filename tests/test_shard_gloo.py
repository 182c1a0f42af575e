"""Sharding of the batched runs across ranks with no data-path collective,
checked with two gloo ranks on CPU (the oracle does each rank's work)."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from hit3d_b200.batch import batched_runs, run_cost, shard_runs


def test_shard_assignment_covers_every_run_once():
    ps = batched_runs()
    assert len(ps) == 96
    costs = [run_cost(p) for p in ps]
    for world in (1, 2, 4, 8):
        shards = shard_runs(costs, world)
        flat = sorted(i for s in shards for i in s)
        assert flat == list(range(96))
        loads = [sum(costs[i] for i in s) for s in shards]
        assert max(loads) <= 1.6 * (sum(costs) / world)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import oracle
    from hit3d_b200.batch import run_sharded, run_seed
    sizes = [16, 24, 16, 32, 16]
    costs = [n ** 3 for n in sizes]

    def work(runs):
        out = {}
        for r in runs:
            o = oracle.Oracle(sizes[r], flow_type=1, nu=1.0 / 100.0, dt=0.005)
            o.init_velocity(run_seed(r), isp_type=2, peak_wavenum=4.0, ir_exp=2.0)
            o.dealias_all()
            o.step(2)
            out[r] = o.stats()[1]["energy"]
        return out

    def gather(d):
        parts = [None] * world
        dist.all_gather_object(parts, d)
        return parts

    res = run_sharded(rank, world, costs, work, gather)
    if rank == 0:
        q.put(res)
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_match_serial():
    import oracle
    from hit3d_b200.batch import run_seed
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    sizes = [16, 24, 16, 32, 16]
    for r, n in enumerate(sizes):
        o = oracle.Oracle(n, flow_type=1, nu=1.0 / 100.0, dt=0.005)
        o.init_velocity(run_seed(r), isp_type=2, peak_wavenum=4.0, ir_exp=2.0)
        o.dealias_all()
        o.step(2)
        assert res[r] == o.stats()[1]["energy"]
