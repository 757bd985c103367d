"""Sharding of ensembles across ranks (world size 2, gloo, on CPU): the
partition covers every member once with balanced work, results come back in
member order on every rank, and times are max-reduced."""
import os
import socket

import numpy as np
import pytest

from cosenu_b200.distributed import imbalance, partition_work


def test_partition_is_complete_and_balanced():
    from cosenu_b200.ensemble import ensemble_instances
    xs = ensemble_instances(256)
    w = [x.cells * x.nsteps for x in xs]
    for world in (1, 2, 4, 8):
        parts = partition_work(w, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(256))
        assert imbalance(w, parts) < 1.05
    assert partition_work(w, 4) == partition_work(w, 4)  # deterministic


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    from cosenu_b200.distributed import max_over_ranks, partition_work, run_sharded
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        items = list(range(37))
        weights = [((i * 7919) % 13) + 1 for i in items]
        seen = []

        def work(chunk):
            seen.extend(chunk)
            return [i * i + 0.5 for i in chunk]

        out = run_sharded(items, weights, work, dist)
        t = max_over_ranks(1.0 + rank, dist)
        q.put((rank, seen, out, t, partition_work(weights, world)[rank]))
    finally:
        dist.destroy_process_group()


def test_sharded_run_gloo_world2():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    seen = [r[1] for r in res]
    assert sorted(seen[0] + seen[1]) == list(range(37))      # each item computed once
    assert not set(seen[0]) & set(seen[1])
    for r in res:
        assert r[2] == [i * i + 0.5 for i in range(37)]      # every rank has all, in order
        assert r[3] == 2.0                                    # slowest rank's time
        assert sorted(r[1]) == r[4]
