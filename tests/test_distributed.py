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


def _tiny_instances():
    from cosenu_b200.ensemble import Instance
    rng = np.random.default_rng(5)
    out = []
    for i, (nz, nvz) in enumerate([(32, 8), (64, 8), (48, 6), (32, 4), (64, 10), (40, 8),
                                   (56, 6)]):
        out.append(Instance(nz=nz, nvz=nvz, alpha=float(rng.uniform(0.6, 1.2)),
                            sig_nu=float(rng.uniform(0.4, 0.8)),
                            sig_nubar=float(rng.uniform(0.3, 0.7)),
                            mu=float(rng.uniform(0.5, 2.0)), seed=500 + i,
                            nsteps=int(rng.integers(2, 9)), z0=-nz / 2, z1=nz / 2, index=i))
    return out


def _oracle_runner(chunk):
    """CPU stand-in for the batched GPU ensemble at the member boundary: every
    member of the chunk evolved by the oracle from the same seeded initial
    condition; 'seconds' is the number of members (so the max over ranks is
    checkable)."""
    from oracle.oracle import Case, Oracle
    o = Oracle()
    res = []
    for x in chunk:
        case = Case(nz=x.nz, nvz=x.nvz, gz=4, z0=x.z0, z1=x.z1, cfl=x.cfl, omega=0.0, mu=x.mu,
                    scheme="fv")
        G, bG, st0 = o.init_seeded(case, seed=x.seed, instance=x.index, sig_nu=x.sig_nu,
                                   sig_nubar=x.sig_nubar, alpha=x.alpha)
        st = o.step(case, st0, x.nsteps)
        res.append(o.analyse(case, st, G, bG, st0))
    return res, float(len(chunk))


def _ens_worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    from cosenu_b200.distributed import run_ensemble_sharded
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        res, secs, share = run_ensemble_sharded(_tiny_instances(), dist, runner=_oracle_runner)
        q.put((rank, res, secs, share))
    finally:
        dist.destroy_process_group()


def test_sharded_ensemble_gloo_world2():
    """The ensemble workload's sharded path (partition, per-rank ensemble,
    gather, max-reduced time) with the per-rank ensemble replaced by the
    oracle: every rank ends with every member's result, in member order,
    equal to one process running all members."""
    import torch.multiprocessing as mp
    from cosenu_b200.distributed import partition_work, run_ensemble_sharded
    xs = _tiny_instances()
    want, _, share1 = run_ensemble_sharded(xs, None, runner=_oracle_runner)
    assert share1 == list(range(len(xs)))
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_ens_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted([q.get(timeout=300) for _ in procs], key=lambda r: r[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    parts = partition_work([x.cells * x.nsteps for x in xs], 2)
    assert sorted(res[0][3] + res[1][3]) == list(range(len(xs)))
    for rank, got, secs, share in res:
        assert share == parts[rank]
        assert secs == float(max(len(p) for p in parts))   # the slowest rank's time
        assert len(got) == len(xs)
        for g, w in zip(got, want):
            assert g == w                                    # bitwise: same oracle, same seed
