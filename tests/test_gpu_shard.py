"""The batched form sharded over two processes (one per rank, gloo for the one
gather of small results, no collective on the data path), each driving its
own device contexts: every run ends as in one process stepping all runs.
Both ranks use cuda:0 here (one GPU); their kernels never wait on each other."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu

SIZES = [32, 48, 32, 64, 32, 48]


def _params():
    from hit3d_b200 import Params
    return [Params(nx=n, flow_type=1, kfmax=2, nu=1.0 / (300.0 + 40.0 * r), dt=0.004 * 32.0 / n)
            for r, n in enumerate(SIZES)]


def _step_runs(runs):
    """Step the given runs as one batch; per run the energy and the fields."""
    from hit3d_b200.batch import Batch, run_seed
    ps = _params()
    b = Batch([ps[r] for r in runs])
    for c, r in zip(b.contexts, runs):
        c.init_velocity(run_seed(r), 2, 4.0, 2.0)
        c.dealias_all()
    b.step(8, graph_steps=3)
    out = {r: (c.stats()[1]["energy"], c.download_fields()) for c, r in zip(b.contexts, runs)}
    b.close()
    return out


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    import torch
    torch.cuda.set_device(0)
    from hit3d_b200.batch import run_cost, run_sharded

    def gather(d):
        parts = [None] * world
        dist.all_gather_object(parts, d)
        return parts

    res = run_sharded(rank, world, [run_cost(p) for p in _params()], _step_runs, gather)
    if rank == 0:
        q.put({r: (e, f.tobytes()) for r, (e, f) in res.items()})
    dist.barrier()
    dist.destroy_process_group()


def test_two_processes_match_one():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = q.get(timeout=600)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    ref = _step_runs(list(range(len(SIZES))))
    assert sorted(res) == list(range(len(SIZES)))
    for r, (e, f) in ref.items():
        assert res[r][0] == e, r
        assert res[r][1] == f.tobytes(), r
