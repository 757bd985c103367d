"""Multi-GPU plumbing: one process per GPU (torch.distributed), ensemble
members sharded across ranks with balanced work and no data-path collective;
only results are gathered and device times are max-reduced.

A single simulation fits one B200 (the largest configuration holds ~12 GB),
so a single instance is never split across GPUs; several GPUs run several
instances (ensembles, or independent replicas in bench.py).
"""
from __future__ import annotations

import heapq
from typing import Callable, Sequence


def partition_work(weights: Sequence[float], world: int) -> list[list[int]]:
    """Longest-processing-time-first assignment of items (weights = work,
    e.g. nz * nvz * steps) to `world` ranks; deterministic; each rank's list
    is in increasing item order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(weights)), key=lambda i: (-weights[i], i))
    heap = [(0.0, r) for r in range(world)]
    parts: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + weights[i], r))
    return [sorted(p) for p in parts]


def imbalance(weights: Sequence[float], parts: list[list[int]]) -> float:
    """max rank load / mean rank load."""
    loads = [sum(weights[i] for i in p) for p in parts]
    mean = sum(loads) / len(loads)
    return max(loads) / mean if mean > 0 else 1.0


def run_sharded(items: Sequence, weights: Sequence[float], work: Callable[[list], list],
                dist=None):
    """Runs `work` on this rank's share of `items` and gathers every item's
    result to all ranks, in item order.  `dist` is torch.distributed (already
    initialised) or None for a single process."""
    if dist is None or not dist.is_initialized():
        return list(work(list(items)))
    world, rank = dist.get_world_size(), dist.get_rank()
    parts = partition_work(weights, world)
    mine = parts[rank]
    res = work([items[i] for i in mine])
    gathered = [None] * world
    dist.all_gather_object(gathered, (mine, list(res)))
    out = [None] * len(items)
    for idx, vals in gathered:
        for i, v in zip(idx, vals):
            out[i] = v
    return out


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """Slowest rank's time (device-measured seconds or milliseconds)."""
    if dist is None or not dist.is_initialized():
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_ensemble_sharded(instances: Sequence, dist=None, runner: Callable | None = None,
                         reduce_device=None, **runner_kw):
    """The ensemble workload over all ranks: this rank's share of `instances`
    (balanced by nz * nvz * steps, partition_work) runs as one batched
    ensemble (`runner`, default ensemble.run_on_gpu); every member's result
    comes back to every rank in instance order and the run time is the
    slowest rank's.  Returns (results, seconds, this rank's share).  The
    reference's counterpart is one process per configuration
    (manage.py:361-428); here the only exchange is the final gather."""
    if runner is None:
        from .ensemble import run_on_gpu as runner
    weights = [x.cells * x.nsteps for x in instances]
    world = dist.get_world_size() if dist is not None and dist.is_initialized() else 1
    rank = dist.get_rank() if world > 1 else 0
    share = partition_work(weights, world)[rank]
    timing = {"seconds": 0.0}

    def work(chunk):
        if not chunk:
            return []
        res, secs = runner(list(chunk), **runner_kw)[:2]
        timing["seconds"] = secs
        return res

    results = run_sharded(instances, weights, work, dist)
    seconds = max_over_ranks(timing["seconds"], dist, reduce_device)
    return results, seconds, share
