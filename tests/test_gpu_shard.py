"""The sharded scan with the real staged plan: world size 2 over gloo, both ranks on the
one GPU of the call (their kernels never wait on each other: each rank's staged scan is
one self-contained launch sequence on its own plan).

Each rank runs whole (tau1, tau2) groups of a 128-point slice of the c2 scan through its
own FP64 plan; the gather brings every point's P(t) to rank 0 in the caller's order,
compared against one rank running every point.  Pairing of groups inside a job can
change where the staged scan jumps over pulse-free gaps, which changes rounding only:
the bar is 1e-12 relative per point.
"""
import os
import socket
import sys

import numpy as np
import pytest

from heomtest import key, load_pkg, rel_err

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


def _rows():
    sys.path.insert(0, os.path.join(HERE, "golden"))
    from make_fixtures import scan_points
    grid = [(a, b, c, d) for a, b, c, d, _ in scan_points()]
    return grid[::8]   # 128 points: every t2 and kind, t1 every 40 fs


def _worker(rank, world, port, q):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        sys.path.insert(0, HERE)
        heom = load_pkg()
        shard = __import__("eto_heom_b200.shard", fromlist=["x"])
        prob = heom.Problem.from_key(key("c0_dimer.key"))
        prob.prepare_sample()
        pts = heom.make_points(_rows())
        plan = heom.Plan(prob, "fp64", max_points=len(pts))
        _, _, counts, _ = plan.scan_layout(pts)
        full = shard.sharded_scan(lambda sub: plan.run_scan(sub).P, pts, counts, rank, world)
        mine = len(shard.partition_groups(pts, world)[rank])
        q.put((rank, mine, full))
    finally:
        dist.destroy_process_group()


def test_sharded_staged_scan_matches_one_rank():
    import multiprocessing as mp

    heom = load_pkg()
    prob = heom.Problem.from_key(key("c0_dimer.key"))
    prob.prepare_sample()
    pts = heom.make_points(_rows())
    one = heom.Plan(prob, "fp64", max_points=len(pts)).run_scan(pts)
    world = 2
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = [q.get(timeout=300) for _ in range(world)]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    shares = {r: m for r, m, _ in got}
    full = next(f for r, _, f in got if r == 0)
    assert sum(shares.values()) == len(pts) and min(shares.values()) > 0
    errs = [rel_err(full[one.offsets[i]:one.offsets[i] + one.counts[i]], one.point(i)) for i in range(len(pts))]
    print(f"\nsharded (2 ranks: {shares[0]} + {shares[1]} points) vs one rank: max {max(errs):.2e}")
    assert max(errs) <= 1e-12
