"""Sharding a 2DES delay scan over several GPUs (one process per GPU).

Scan points are independent, so a scan shards with no exchange during propagation: each
rank takes a share of the points, runs it through its own plan, and one gather brings the
P(t) buffers to rank 0, which reassembles them in the caller's point order.  This is the
batched form of the reference's one-process-per-key job model
(script/cpu-script/submit_jobs.sh:49-67).

The staged scan shares work inside a (tau1, tau2) group: the points of a group have the
same first two pulses, so their R and D2 components are propagated once for the group up
to the members' pulse-3 windows.  The partition therefore hands out whole groups,
longest-processing-time first, weighted by the group's staged work: the shared stage
(until the later of the first two pulses has ended) plus each member's pulse-3 window
and pulse-free tail.  Splitting a group would repeat its shared stage on every rank that
holds a member.

The propagation of a single point is not sharded (replicas only): it would need a halo
exchange of neighbour-ADO rows/columns every RK4 stage, and every configured point fits
one GPU with room to spare.
"""
from __future__ import annotations

import heapq

import numpy as np


def steps_of(t_end: float, t_start: float = 0.0, dt: float = 0.5) -> int:
    """RK4 steps of a point ending at t_end (float time, as dynamics.cpp:344-347)."""
    nstep = np.float32((np.float32(t_end) - np.float32(t_start)) / np.float32(dt))
    return int(nstep) + 1 if nstep >= 0 else 0


def lpt_partition(work: list[float], world: int) -> list[list[int]]:
    """Indices of each rank's items: largest first onto the least-loaded rank."""
    heap = [(0.0, r) for r in range(world)]
    heapq.heapify(heap)
    out = [[] for _ in range(world)]
    for i in sorted(range(len(work)), key=lambda k: (-work[k], k)):
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + work[i], r))
    return [sorted(ix) for ix in out]


def scan_groups(points: np.ndarray) -> list[list[int]]:
    """Point indices of each (tau1, tau2) group, in order of first appearance."""
    index: dict[tuple[float, float], int] = {}
    groups: list[list[int]] = []
    for i, p in enumerate(points):
        k = (float(p["tau1"]), float(p["tau2"]))
        if k not in index:
            index[k] = len(groups)
            groups.append([])
        groups[index[k]].append(i)
    return groups


def group_work(points: np.ndarray, members: list[int], taup: float = 20.0, t_start: float = 0.0,
               dt: float = 0.5) -> float:
    """Staged work of one group in component-steps: R and D2 until the first two pulses
    are over, then for every member its pulse-3 window (two components; four while pulse 2
    is still on) and its pulse-free tail, which costs a few per cent of a stepped
    component.  A load-balancing weight: it follows the staged planner's stages, not its
    exact counts."""
    p0 = points[members[0]]
    t12 = max(float(p0["tau1"]), float(p0["tau2"])) + 2 * taup
    w = 2.0 * steps_of(t12, t_start, dt)
    win = 4 * taup / dt + 1
    for i in members:
        p = points[i]
        tau3 = float(p["tau3"])
        four = tau3 - 2 * taup < t12
        w += (4.0 if four else 2.0) * win
        w += 0.05 * max(0, steps_of(float(p["t_end"]), t_start, dt) - steps_of(tau3 + 2 * taup, t_start, dt))
    return w


def partition_groups(points: np.ndarray, world: int, taup: float = 20.0, t_start: float = 0.0,
                     dt: float = 0.5) -> list[list[int]]:
    """Point indices of each rank: whole (tau1, tau2) groups, LPT by staged work."""
    groups = scan_groups(points)
    w = [group_work(points, g, taup, t_start, dt) for g in groups]
    return [sorted(i for gi in share for i in groups[gi]) for share in lpt_partition(w, world)]


def gather_to_rank0(local: np.ndarray, rank: int, world: int, device=None) -> list[np.ndarray] | None:
    """Every rank's complex vector on rank 0 (one torch.distributed gather: NCCL with CUDA
    tensors, gloo with CPU tensors); None on the other ranks."""
    import torch
    import torch.distributed as dist

    n = torch.tensor([len(local)], dtype=torch.int64)
    if device is not None:
        n = n.to(device)
    sizes = [torch.zeros_like(n) for _ in range(world)]
    dist.all_gather(sizes, n)
    n_max = max(int(s.item()) for s in sizes)
    buf = np.zeros((max(n_max, 1), 2), dtype=np.float64)
    buf[:len(local), 0] = local.real
    buf[:len(local), 1] = local.imag
    t = torch.from_numpy(buf)
    if device is not None:
        t = t.to(device)
    gathered = [torch.zeros_like(t) for _ in range(world)] if rank == 0 else None
    dist.gather(t, gather_list=gathered, dst=0)
    if rank != 0:
        return None
    out = []
    for r in range(world):
        g = gathered[r].cpu().numpy()[:int(sizes[r].item())]
        out.append(g[:, 0] + 1j * g[:, 1])
    return out


def sharded_scan(run_points, points: np.ndarray, counts: np.ndarray, rank: int, world: int,
                 t_start: float = 0.0, dt: float = 0.5, taup: float = 20.0, device=None):
    """Run this rank's share of `points` (whole (tau1, tau2) groups) and gather every
    point's P(t) on rank 0.

    run_points(sub_points) -> concatenated complex P of those points (their own layout
    order); counts[i] = recorded points of point i (heom_scan_layout).  Returns the full
    concatenated P (caller's point order) on rank 0, None elsewhere."""
    share = partition_groups(points, world, taup, t_start, dt)
    mine = share[rank]
    local = run_points(points[mine]) if mine else np.zeros(0, dtype=np.complex128)
    parts = gather_to_rank0(np.asarray(local, dtype=np.complex128), rank, world, device)
    if rank != 0:
        return None
    offsets = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    full = np.zeros(int(offsets[-1]), dtype=np.complex128)
    for r in range(world):
        g = parts[r]
        pos = 0
        for i in share[r]:
            c = int(counts[i])
            full[offsets[i]:offsets[i] + c] = g[pos:pos + c]
            pos += c
    return full
