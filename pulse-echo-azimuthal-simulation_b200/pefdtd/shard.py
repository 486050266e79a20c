"""Independent solves dealt to ranks (one process per GPU).

A single solve does not shard: its grids (at most 10.5 M cells, 0.44 GB) fit
one GPU many times over, so several GPUs run replicas. What shards is a
batch of independent solves, the azimuths of a sweep or the specimens of a
campaign: each rank advances its share with no exchange while the solves
run, and the traces (a few kB per solve) are gathered once at the end. The
reference has no counterpart: it runs its sweep as one sequential loop on
one GPU (sim/pipeline/sweep_runner.py:322-390).

The process group is the caller's (``torch.distributed``, NCCL between GPUs,
gloo on CPU); every rank takes the same collective steps in the same order.
"""
from __future__ import annotations

import numpy as np


def assign(costs, world):
    """Deal items to ``world`` ranks, heaviest first, each to the least
    loaded rank (ties to the lower rank): deterministic, so every rank
    computes the same shares. Returns one sorted index list per rank."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    loads = [0.0] * world
    shares = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (loads[k], k))
        shares[r].append(i)
        loads[r] += float(costs[i])
    return [sorted(s) for s in shares]


def solve_cost(setup):
    """Cell updates of one sweep setup (``sweep.azimuth_setup``) or workload
    problem (``workloads.make_problem``): cells x steps."""
    if "spec" in setup:
        return float(np.prod(setup["spec"]["mats"].shape)) * float(setup["nt"])
    return float(np.prod(setup["lab"].shape)) * float(setup["nt"])


def _group_info(group):
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        return 0, 1
    return dist.get_rank(group), dist.get_world_size(group)


def run_sharded(items, solver, costs=None, group=None):
    """Solve ``items`` across the ranks of ``group`` (the default group when
    initialised, else this process alone). ``solver(list_of_items)`` returns
    one trace per item; each rank calls it on its share only. Returns the
    traces of all items, in input order, on every rank."""
    rank, world = _group_info(group)
    if costs is None:
        costs = [1.0] * len(items)
    shares = assign(costs, world)
    mine = shares[rank]
    traces = list(solver([items[i] for i in mine])) if mine else []
    if len(traces) != len(mine):
        raise RuntimeError(f"solver returned {len(traces)} traces for {len(mine)} items")
    if world == 1:
        return traces
    import torch.distributed as dist
    parts = [None] * world
    dist.all_gather_object(parts, [(i, np.asarray(t)) for i, t in zip(mine, traces)], group=group)
    out = [None] * len(items)
    for part in parts:
        for i, t in part:
            out[i] = t
    return out
