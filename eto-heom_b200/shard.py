"""Sharding a 2DES delay scan over several GPUs (one process per GPU).

Scan points are independent, so a scan shards with no exchange during propagation: each
rank takes a longest-processing-time-first share of the points (by RK4 step count, the
work measure of a point), runs it through its own plan, and one gather brings the P(t)
buffers to rank 0, which reassembles them in the caller's point order.

The propagation of a single point is not sharded (replicas only): it would need a halo
exchange of neighbour-ADO rows/columns every RK4 stage, and every BASELINE point fits one
GPU with room to spare.
"""
from __future__ import annotations

import heapq

import numpy as np


def steps_of(t_end: float, t_start: float = 0.0, dt: float = 0.5) -> int:
    """RK4 steps of a point ending at t_end (float time, as dynamics.cpp:344-347)."""
    nstep = np.float32((np.float32(t_end) - np.float32(t_start)) / np.float32(dt))
    return int(nstep) + 1 if nstep >= 0 else 0


def lpt_partition(work: list[int], world: int) -> list[list[int]]:
    """Indices of each rank's points: longest first onto the least-loaded rank."""
    heap = [(0, r) for r in range(world)]
    heapq.heapify(heap)
    out = [[] for _ in range(world)]
    for i in sorted(range(len(work)), key=lambda k: (-work[k], k)):
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + work[i], r))
    return [sorted(ix) for ix in out]


def sharded_scan(run_points, points: np.ndarray, counts: np.ndarray, rank: int, world: int,
                 t_start: float = 0.0, dt: float = 0.5, device=None):
    """Run this rank's share of `points` and gather every point's P(t) on rank 0.

    run_points(sub_points) -> concatenated complex P of those points (their own layout
    order); counts[i] = recorded points of point i (heom_scan_layout).  Returns the full
    concatenated P (caller's point order) on rank 0, None elsewhere.  Uses
    torch.distributed (NCCL with CUDA tensors, gloo with CPU tensors)."""
    import torch
    import torch.distributed as dist

    work = [steps_of(float(p["t_end"]), t_start, dt) for p in points]
    share = lpt_partition(work, world)
    mine = share[rank]
    local = run_points(points[mine]) if mine else np.zeros(0, dtype=np.complex128)
    n_max = max(int(sum(counts[i] for i in s)) for s in share)
    buf = np.zeros((n_max, 2), dtype=np.float64)
    buf[:len(local), 0] = local.real
    buf[:len(local), 1] = local.imag
    t = torch.from_numpy(buf)
    if device is not None:
        t = t.to(device)
    gathered = [torch.zeros_like(t) for _ in range(world)] if rank == 0 else None
    dist.gather(t, gather_list=gathered, dst=0)
    if rank != 0:
        return None
    offsets = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    full = np.zeros(int(offsets[-1]), dtype=np.complex128)
    for r in range(world):
        g = gathered[r].cpu().numpy()
        pos = 0
        for i in share[r]:
            c = int(counts[i])
            full[offsets[i]:offsets[i] + c] = g[pos:pos + c, 0] + 1j * g[pos:pos + c, 1]
            pos += c
    return full
