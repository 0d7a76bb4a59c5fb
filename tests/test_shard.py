"""Scan sharding over ranks: LPT partition and the gather to rank 0, world_size 2 on gloo.

The per-rank propagation is replaced by a deterministic stand-in (CPU only); the GPU path
itself is the single-GPU scan tested elsewhere.
"""
import os
import socket

import numpy as np
import pytest

from heomtest import load_pkg


def test_lpt_partition_balances_and_covers():
    import importlib

    load_pkg()
    shard = importlib.import_module("eto_heom_b200.shard")
    work = [901 + 37 * (i % 53) for i in range(1024)]
    parts = shard.lpt_partition(work, 4)
    assert sorted(i for p in parts for i in p) == list(range(1024))
    loads = [sum(work[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(work)


def test_partition_keeps_groups_whole_and_balances():
    import importlib
    import sys

    heom = load_pkg()
    shard = importlib.import_module("eto_heom_b200.shard")
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
    from make_fixtures import scan_points
    pts = heom.make_points([(a, b, c, d) for a, b, c, d, _ in scan_points()])
    groups = shard.scan_groups(pts)
    assert len(groups) == 127 and sum(len(g) for g in groups) == 1024   # t1 = 0: R and NR coincide
    for world in (2, 4, 8):
        parts = shard.partition_groups(pts, world)
        assert sorted(i for p in parts for i in p) == list(range(1024))
        owner = {i: r for r, p in enumerate(parts) for i in p}
        for g in groups:   # every group on one rank
            assert len({owner[i] for i in g}) == 1
        w = [shard.group_work(pts, g) for g in groups]
        loads = [sum(w[gi] for gi, g in enumerate(groups) if owner[g[0]] == r) for r in range(world)]
        assert max(loads) - min(loads) <= max(w)


def _points(n):
    heom = load_pkg()
    rows = [(50.0, 50.0 + 5 * i, 60.0 + 5 * i, 100.0 + 7 * (i % 11)) for i in range(n)]
    return heom.make_points(rows)


def _fake_run(sub):
    # deterministic per-point "P(t)": counts = 3 + (i % 4) values encoding tau2 and the index
    out = []
    for p in sub:
        k = int(round((p["tau2"] - 50.0) / 5))
        c = 3 + k % 4
        out.append(np.arange(c) + 1j * k)
    return np.concatenate(out) if out else np.zeros(0, np.complex128)


def _worker(rank, world, port, n, q):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import sys
        sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
        load_pkg()
        shard = __import__("eto_heom_b200.shard", fromlist=["x"])
        pts = _points(n)
        counts = np.array([3 + i % 4 for i in range(n)], dtype=np.int64)
        full = shard.sharded_scan(_fake_run, pts, counts, rank, world)
        if rank == 0:
            q.put(full)
    finally:
        dist.destroy_process_group()


def test_sharded_scan_gathers_in_point_order_gloo():
    import multiprocessing as mp

    n, world = 37, 2
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, n, q)) for r in range(world)]
    for p in procs:
        p.start()
    full = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    expect = _fake_run(_points(n))
    assert np.array_equal(full, expect)
