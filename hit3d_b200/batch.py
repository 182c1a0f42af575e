"""Batched form: many independent runs of uneven sizes on one GPU, and their
sharding across GPUs (one process per GPU, no collective on the data path).

The reference runs one simulation per MPI job; this module has no reference
counterpart.  A Batch owns one device context per run (hit3d_batch_* in the
C-ABI); Batch.step advances all runs, replaying a CUDA graph that holds a chunk
of steps of every run.  Training data for a learned closure come from
Context.sgs_fields (filtered velocity, exact subgrid stress, filtered gradients).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import replace
from typing import Callable, List, Sequence

import numpy as np

from .gpu import Context, Params, _check, _Params, lib

RN1 = 67748937.0


def batched_runs(seed: int = 2026, kind: str = "training") -> List[Params]:
    """The batched workload: 96 forced runs, 32 x 32^3, 32 x 48^3, 28 x 64^3 and
    4 x 128^3, per-run seeds, Re uniform in [200, 800], 2/3 rule, FP64."""
    rng = np.random.default_rng(seed)
    sizes = [32] * 32 + [48] * 32 + [64] * 28 + [128] * 4
    out = []
    for n in sizes:
        re = float(rng.uniform(200.0, 800.0))
        # dt scaled with the grid so that the Courant number stays below ~0.4
        dt = 0.004 * 64.0 / n
        out.append(Params(nx=n, dealias=0, flow_type=1, force_type=1, kfmax=2, famp=0.5, nu=1.0 / re, dt=dt))
    return out


def run_seed(r: int) -> float:
    return RN1 + 7919.0 * r


def shard_runs(costs: Sequence[float], world: int) -> List[List[int]]:
    """Longest-processing-time assignment of runs to ranks (deterministic)."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * world
    shards: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        shards[r].append(i)
        load[r] += costs[i]
    return [sorted(s) for s in shards]


def run_cost(p: Params) -> float:
    """Relative cost of one step: N^3 log N."""
    return float(p.nx) ** 3 * np.log2(p.nx)


class Batch:
    """Many runs advanced together on one device."""

    def __init__(self, params: Sequence[Params]):
        arr = (_Params * len(params))(*[p.to_c() for p in params])
        h = C.c_void_p()
        _check(lib().hit3d_batch_create(arr, len(params), C.byref(h)), "hit3d_batch_create")
        self._h = h
        self.params = list(params)
        self.contexts: List[Context] = []
        for r, p in enumerate(params):
            ch = C.c_void_p()
            _check(lib().hit3d_batch_context(h, r, C.byref(ch)), "hit3d_batch_context")
            self.contexts.append(Context(replace(p), _handle=ch))

    def init(self, isp_type: int = 2, peak: float = 4.0, ir_exp: float = 2.0):
        for r, c in enumerate(self.contexts):
            c.init_velocity(run_seed(r), isp_type, peak, ir_exp)
            c.dealias_all()

    def step(self, nsteps: int, graph_steps: int = 10):
        _check(lib().hit3d_batch_step(self._h, int(nsteps), int(graph_steps)), "hit3d_batch_step")

    @property
    def graph_launches(self) -> int:
        return int(lib().hit3d_batch_graph_launches(self._h))

    @property
    def nclasses(self) -> int:
        """Size classes: runs of one grid size, precision and forcing stepped by
        batched launches."""
        return int(lib().hit3d_batch_nclasses(self._h))

    def autotune(self):
        """Per size class, pick the fused x-pass launch shape (variants 8-14) and
        the column-tile shape of the strided passes by timing them on the class's
        buffers.  Returns [(variant, tile, ms of the 7 variants, ms of the 4 tiles)]."""
        k = self.nclasses
        choice = (C.c_int32 * (2 * max(k, 1)))()
        ms = np.zeros(11 * max(k, 1))
        _check(lib().hit3d_batch_autotune(self._h, choice, ms.ctypes.data_as(C.POINTER(C.c_double))),
               "hit3d_batch_autotune")
        return [(int(choice[2 * q]), int(choice[2 * q + 1]), ms[11 * q:11 * q + 7].tolist(),
                 ms[11 * q + 7:11 * q + 11].tolist()) for q in range(k)]

    def close(self):
        if getattr(self, "_h", None):
            for c in self.contexts:
                c.close()
            lib().hit3d_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def run_sharded(rank: int, world: int, costs: Sequence[float], work: Callable[[List[int]], dict], gather) -> dict:
    """Run this rank's shard and gather every rank's results (dict run -> result).

    `gather` is a callable taking this rank's dict and returning the list of all
    ranks' dicts (torch.distributed.all_gather_object in practice); there is no
    collective on the data path, only this one exchange of small results."""
    mine = shard_runs(costs, world)[rank]
    res = work(mine)
    merged: dict = {}
    for part in gather(res):
        merged.update(part)
    return merged
