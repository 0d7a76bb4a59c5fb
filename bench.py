"""Benchmark: 2DES propagations/sec on the 1024-point dimer delay scan.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (one "step" = one pass over the whole scan): the dimer of the c0 fixture
(N = 4 levels, 70 ADOs) scanned over 64 t1 delays (0-315 fs) x 8 waiting times
(0-700 fs) x {rephasing, non-rephasing} = 1024 independent 2DES points, t3 = 400 fs,
dt = 0.5 fs (901-2931 RK4 steps per point).  One propagation = one point = the three
mask trajectories 111, 110, 101 combined, as one CPU_2DES run of one key file.

value: propagations/s of the chosen path (staged FP32-bulk scan, inputs resident on the
device, CUDA-event time of the scan per step, L2 flushed between steps).
e2e:   the same through the public C ABI with host buffers (heom_run_scan: H2D of the
points, D2H of every P(t) into a page-locked output array), wall time of the
synchronous call.
Also reported: the plain FP64 path (bit-exact, one point at a time) on a sample of
points, the FP32-bulk error against the FP64 scan, the roofline of the scan kernel,
GPU clocks during the timed region and the reference CPU build on a bounded sample.

Multi-GPU (torchrun): every rank runs its own 1024-point scan of a different disorder /
orientation sample (weak scaling), no collective on the data path; value = all points /
max-over-ranks time.  After the timed region one gather (eto-heom_b200/shard.py, NCCL)
brings the ranks' P(t) to rank 0, which forms the disorder average as CPU_2DES does.
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "tests"))
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))

METRIC = "2DES propagations/sec, chosen vs plain FP64 on 1 B200 at ≤1e-6 P(t) err"
UNIT = "propagations/s"
KEY = os.path.join(ROOT, "tests", "golden", "keys", "c0_dimer.key")
# dram__bytes_read.sum + dram__bytes_write.sum of one scan_slots launch of the bench's own
# 1024-point scan (the second run of a plan, T0 powers cached), from one ncu capture of
# `bench.py --profile-run fp32-bulk-full` (profiles/scan_slots_dram_dimer_scan.md):
# 27,223,040 B read (mostly the FP64 jump powers, read cold: ncu and the bench's L2 flush
# both start the launch with an empty L2) + 5,175,552 B written (snapshots, P records).
DRAM_BYTES_PER_SCAN = 29598208.0 + 6949888.0
TEMPLATE = os.path.join(ROOT, "tests", "golden", "keys", "c2_dimer_scan.key-tmpl")


def scan_rows():
    from make_fixtures import scan_points
    return [(a, b, c, d) for a, b, c, d, _ in scan_points()]


def flops_per_traj_step(N: int, n_ado: int, links: int) -> float:
    """Algorithmic real flops of one RK4 step of one trajectory: four stages of the
    dense commutator (16 N^3), damping + stage axpys (24 N^2) per ADO and one-hot
    row/column neighbour updates (16 N per link)."""
    return 4.0 * (n_ado * (16 * N ** 3 + 24 * N ** 2) + 16 * N * links)


def steps_of(t_end: float, t_start: float = 0.0, dt: float = 0.5) -> int:
    nstep = np.float32((np.float32(t_end) - np.float32(t_start)) / np.float32(dt))
    return int(nstep) + 1 if nstep >= 0 else 0


class Clocks:
    """nvidia-smi sampler for the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        if shutil.which("nvidia-smi"):
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.path)
        busy = [s for s in sm if mx and s > 0.5 * mx] or sm
        return {"sm_mhz": statistics.median(busy) if busy else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def measured_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return {}


def fp32_peak_tflops(heom, device: int) -> float:
    """FP32 FMA throughput of this GPU, measured now by the library's FMA-loop kernel
    (best of three); the scan kernel runs on these pipes, not on the tensor cores."""
    return max(heom.fma_peak_tflops(device, fp64=False) for _ in range(3))


# ------------------------------------------------------------------ reference arm
def reference_cpu(rows, n_points: int, cores: int):
    """Run the reference's own CPU build (oracle/_ref/CPU_2DES, one process per key file,
    `cores` at a time -- the reference's process-per-key model) on n_points points."""
    exe = os.path.join(ROOT, "oracle", "_ref", "CPU_2DES")
    kind = "reference"
    if not os.path.exists(exe):
        exe = os.path.join(ROOT, "oracle", "heom_oracle")
        kind = "port"
        if not os.path.exists(exe):
            subprocess.check_call(["make", "-C", os.path.join(ROOT, "oracle"), "all"])
    tmpl = open(TEMPLATE).read()
    # stratified sample: spread over the scan
    idx = np.linspace(0, len(rows) - 1, n_points).round().astype(int)
    d = tempfile.mkdtemp()
    keys = []
    for j, i in enumerate(idx):
        r = rows[i]
        t = (tmpl.replace("TAU1", repr(r[0])).replace("TAU2", repr(r[1])).replace("TAU3", repr(r[2]))
             .replace("T_END", repr(r[3])))
        p = os.path.join(d, f"key_{j}.key")
        open(p, "w").write(t)
        keys.append(p)
    t0 = time.perf_counter()
    procs = []
    for p in keys:
        while len([q for q in procs if q.poll() is None]) >= cores:
            time.sleep(0.005)
        procs.append(subprocess.Popen([exe, p] + (["--structured"] if kind == "port" else []),
                                      stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL))
    for q in procs:
        q.wait()
    wall = time.perf_counter() - t0
    shutil.rmtree(d, ignore_errors=True)
    steps = sum(steps_of(rows[i][3]) for i in idx)
    return len(keys) / wall, kind, wall, steps


def run_reference_arm(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    rows = scan_rows()
    cores = os.cpu_count() or 1
    per_step = max(cores, 1)
    vals = []
    kind = "reference"
    wall_total = 0.0
    for s in range(a.warmup + a.steps):
        v, kind, wall, _ = reference_cpu(rows, per_step, cores)
        if s >= a.warmup:
            vals.append(v)
            wall_total += wall
    value = float(np.mean(vals))
    sample = (f"{per_step} stratified scan points per step, one CPU_2DES process per key file, "
              f"{cores} concurrent (the reference's process-per-key model)")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": a.gpus,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 * wall_total / max(a.steps, 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": {"workload": "c2 dimer 2DES delay scan (1024 points), reference CPU build",
                                        "points_per_step": per_step},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "cpu_model": cpu_model(), "kind": kind,
                         "sample": sample + "; the rate over this sample stands for the whole 1024-point scan "
                                            "(an extrapolation: the sample is stratified over the scan's "
                                            "point lengths)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


# ------------------------------------------------------------------ our arm
C1_KEY = os.path.join(ROOT, "tests", "golden", "keys", "c1_fmo.key")


def c3_record(heom, device: int) -> dict:
    """Config 3, the precision study: the 12-site chain (single-excitation manifold, N = 13,
    2925 ADOs), linear response (pulse 3 only) over 6001 RK4 steps, FP32-bulk contractions
    on FP64 state against the bit-exact FP64 path and the FP64 staged path."""
    from heomtest import rel_err

    k = os.path.join(ROOT, "tests", "golden", "keys", "c3_chain.key")
    out = {}
    P = {}
    for prec in ("fp64-exact", "fp64", "fp32-bulk"):
        prob = heom.Problem.from_key(k, single_manifold=True)
        prob.prepare_sample()
        plan = heom.Plan(prob, prec, device=device)
        plan.run_traj(0, 0, 1)
        t0 = time.perf_counter()
        P[prec] = plan.run_traj(0, 0, 1)
        out[prec.replace("-", "_") + "_ms_per_step"] = 1e3 * (time.perf_counter() - t0) / 6001
    inf = heom.Problem.from_key(k, single_manifold=True).info
    out.update({"workload": f"c3 chain: N={inf.sys_size}, {inf.n_ado} ADOs, 6001 RK4 steps, linear response",
                "fp32_bulk_vs_fp64_exact_max_rel_err": rel_err(P["fp32-bulk"], P["fp64-exact"]),
                "fp32_bulk_vs_fp64_staged_max_rel_err": rel_err(P["fp32-bulk"], P["fp64"]),
                "fp64_staged_vs_fp64_exact_max_rel_err": rel_err(P["fp64"], P["fp64-exact"])})
    return out


def large_n_record(heom, device: int, fp32_peak: float) -> dict:
    """The FMO aggregate (N = 29 with the two-exciton manifold, K = 14, L = 3, 680 ADOs):
    one 2DES point, pulses at 50/150/250 fs, propagated to 300 fs (601 RK4 steps), on
    the plain bit-exact FP64 path (three trajectories, one stage launch per RK4 stage)
    and on the FP32-bulk general-size path (the mixed-difference basis, four components).
    Rates are algorithmic flops (4 [n_ado (16 N^3 + 24 N^2) + 16 N links] per
    trajectory-step) over host wall time of run_2des (graph replays + read-back)."""
    from heomtest import rel_err

    text = open(C1_KEY).read()
    assert "TIME\n0 2000 0.5 0.5" in text
    d = tempfile.mkdtemp()
    k = os.path.join(d, "c1_300fs.key")
    with open(k, "w") as f:
        f.write(text.replace("TIME\n0 2000 0.5 0.5", "TIME\n0 300 0.5 0.5"))
    prob = heom.Problem.from_key(k)
    prob.prepare_sample()
    shutil.rmtree(d, ignore_errors=True)
    inf = prob.info
    depth = prob.ado().astype(int).sum(axis=1)
    links = 2 * int((depth < inf.L).sum() * inf.K * inf.K_m)
    F = flops_per_traj_step(inf.sys_size, inf.n_ado, links)
    steps = steps_of(300.0)

    def timed(plan, **kw):
        plan.run_2des(**kw)
        t0 = time.perf_counter()
        P, _ = plan.run_2des(**kw)
        return P, time.perf_counter() - t0

    fp64_peak = max(heom.fma_peak_tflops(device, fp64=True) for _ in range(3))
    px = heom.Plan(prob, "fp64-exact", device=device)
    Px, tx = timed(px)
    pb = heom.Plan(prob, "fp32-bulk", device=device)
    Pb, tb = timed(pb, trajectories=False)
    p64 = heom.Plan(prob, "fp64", device=device)
    P64, t64 = timed(p64, trajectories=False)
    # the binary128 truth of this point (the same key as tests/golden/keys/c1_fmo_300fs.key)
    truth_c1 = np.load(os.path.join(ROOT, "tests", "golden", "ref", "truth_c1_fmo_300fs.npz"))["combined"]
    ax = F * 3 * steps / tx / 1e12
    ab = F * 4 * steps / tb / 1e12
    return {
        "workload": f"c1 FMO 2DES point: N={inf.sys_size}, {inf.n_ado} ADOs, {links} links, {steps} RK4 steps",
        "flop_per_trajectory_step": F,
        "fp64_exact": {"ms_per_step": tx / steps * 1e3, "tflops": ax, "peak_fp64_fma_tflops": fp64_peak,
                       "frac": ax / fp64_peak, "rel_err_vs_truth": rel_err(Px, truth_c1),
                       "note": "three trajectories per step; its output is the reference build's, bit for bit, so "
                               "rel_err_vs_truth is the reference's own rounding noise; bit-exact arithmetic uses no "
                               "FMA, so its ceiling is half the FMA peak; launch: " + px.describe()},
        "fp32_bulk": {"ms_per_step": tb / steps * 1e3, "tflops": ab, "peak_fp32_fma_tflops": fp32_peak,
                      "frac": ab / fp32_peak, "rel_err_vs_exact": rel_err(Pb, Px),
                      "rel_err_vs_fp64_staged": rel_err(Pb, P64), "rel_err_vs_truth": rel_err(Pb, truth_c1),
                      "note": "four mixed-difference components per step (general-size staged path)"},
        "fp64_staged": {"ms_per_step": t64 / steps * 1e3, "tflops": F * 4 * steps / t64 / 1e12,
                        "peak_fp64_fma_tflops": fp64_peak, "frac": F * 4 * steps / t64 / 1e12 / fp64_peak,
                        "fp32_bulk_speedup": t64 / tb, "rel_err_vs_truth": rel_err(P64, truth_c1),
                        "note": "the same four components with FP64 contractions"},
    }


def adjoint_record(heom, device: int) -> dict:
    """Config 4 at its stated size: the trimer (N = 7, 210 ADOs) rephasing P(t1, t3) on
    32 t1 x 128 t3 at t2 = 200 fs, L2 loss against the target of the Hamiltonian
    parameters perturbed by 2 %, gradient of the 12 parameters by the checkpointed
    adjoint (heom_adjoint_scan).  Wall time of one FP64 forward scan and of one gradient
    (forward with checkpoints, recomputed segments and the adjoint sweep)."""
    import importlib
    import math

    from make_fixtures import c4_fit_rows

    ag = importlib.import_module("eto_heom_b200.autograd")
    prob = heom.Problem.from_key(os.path.join(ROOT, "tests", "golden", "keys", "c4_trimer_fit.key"))
    prob.prepare_sample()
    params = ag.ScanParameters(prob)
    rows = c4_fit_rows()
    pts = heom.make_points(rows)
    th0 = params.theta0.copy()
    th_t = th0.copy()
    th_t[:params.n_h] *= 1.02
    params.apply(th_t)
    target = heom.Plan(prob, "fp64", device=device, max_points=len(pts)).run_scan(pts).P
    params.apply(th0)
    plan = heom.Plan(prob, "fp64", device=device, max_points=len(pts))
    plan.run_scan(pts)
    t0 = time.perf_counter()
    P = plan.run_scan(pts).P
    t_fwd = time.perf_counter() - t0
    g = 2.0 * (P - target)
    plan.adjoint_scan(pts, g)
    t0 = time.perf_counter()
    _, grad = plan.adjoint_scan(pts, g)
    t_adj = time.perf_counter() - t0
    steps = max(steps_of(r[3]) for r in rows)
    return {"workload": "c4 trimer fit: N=7, 210 ADOs, rephasing 32 t1 x 128 t3 at t2 = 200 fs, 12 parameters",
            "records": int(len(P)), "max_rk4_steps": steps, "checkpoint_interval": int(math.ceil(math.sqrt(steps))),
            "forward_ms": 1e3 * t_fwd, "gradient_ms": 1e3 * t_adj, "loss": float(np.sum(np.abs(g / 2) ** 2)),
            "grad_norm": float(np.linalg.norm(grad)),
            "note": "FP64 mixed-difference basis; checked against Richardson-extrapolated central "
                    "differences (h = 1e-4 relative) in tests/test_gpu_adjoint_c4.py"}


def run_ours(a):
    import torch

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))  # rank 0 runs the extra records while the others wait

    from heomtest import load_pkg, rel_err

    heom = load_pkg()
    prob = heom.Problem.from_key(KEY)
    for _ in range(rank + 1):  # each rank: its own disorder/orientation sample
        prob.prepare_sample()
    rows = scan_rows()
    n = len(rows)
    pts = heom.make_points(rows)
    plan = heom.Plan(prob, "fp32-bulk", device=local, max_points=n, autotune=True)
    pts, off, cnt, tot = plan.scan_layout(pts)

    # device-resident inputs
    d_pts = torch.from_numpy(pts.view(np.uint8).copy()).cuda()
    d_off = torch.from_numpy(off.copy()).cuda()
    d_P = torch.zeros(2 * tot, dtype=torch.float64, device="cuda")
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")  # > 126 MB L2
    stream = torch.cuda.current_stream()

    def one_scan():
        plan.run_scan_device(d_pts.data_ptr(), n, d_P.data_ptr(), d_off.data_ptr())

    # The plan runs on its own stream; bracket every scan with events on that stream by
    # synchronising around it (the scan is ~0.1 s, the host gap is negligible).
    for _ in range(a.warmup):
        one_scan()
        torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = plan.launches
    times, host_ms = [], []
    with Clocks(local) as clk:
        for _ in range(a.steps):
            flush.fill_(1.0)
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            h0 = time.perf_counter()
            one_scan()  # returns once queued: the point read-back, the host planning, the launches
            host_ms.append(1e3 * (time.perf_counter() - h0))
            torch.cuda.synchronize()
            e1.record(stream)
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
    launches = plan.launches - launches0
    work = plan.scan_work  # component-steps of the last (timed) scan; 0 for a single pass
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ms = float(np.mean(times))
    if dist:
        t = torch.tensor([ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = world * n / (ms / 1e3)
    averaged = None
    if dist:
        # the disorder average of the ranks' samples (CPU_2DES.cpp:83-89) on rank 0: one
        # gather of every rank's P(t) through the shard module (NCCL), outside the timed region
        import importlib
        shard = importlib.import_module("eto_heom_b200.shard")
        torch.cuda.synchronize()
        mine = d_P.cpu().numpy().view(np.complex128).copy()
        parts = shard.gather_to_rank0(mine, rank, world, device=torch.device("cuda", local))
        if rank == 0:
            avg = np.mean(np.stack(parts), axis=0)
            averaged = {"samples": world, "records": int(len(avg)), "finite": bool(np.isfinite(avg).all())}

    # kernel-only duration (CUDA events around the scan kernel alone are the same
    # graph; the order kernel is ~10 us), roofline of the scan kernel
    inf = prob.info
    depth = prob.ado().astype(int).sum(axis=1)
    up_links = int((depth < inf.L).sum() * inf.K * inf.K_m)  # down links are equal in number
    F = flops_per_traj_step(inf.sys_size, inf.n_ado, 2 * up_links)
    traj_steps = 3 * sum(steps_of(r[3]) for r in rows)
    # The staged scan propagates `work` component-steps (one RK4 step of one n_ado x N x N
    # state each, the cost of one reference trajectory step); the reference runs 3
    # trajectories x all steps.  The roofline uses the executed work; the reference-
    # equivalent rate is reported beside it.
    exec_steps = work if work > 0 else 4 * sum(steps_of(r[3]) for r in rows)
    achieved = F * exec_steps / (ms / 1e3) / 1e12
    ref_equiv = F * traj_steps / (ms / 1e3) / 1e12
    peak = fp32_peak_tflops(heom, local)
    # Mixed-pipe bound of the FP32-bulk kernel: the 24 N^2 per-ADO stage work (damping,
    # site-energy diagonal, Horner update) runs in FP64, the rest in FP32.
    peak64 = max(heom.fma_peak_tflops(local, fp64=True) for _ in range(3))
    F64 = 4.0 * inf.n_ado * 24 * inf.sys_size ** 2
    t_bound = exec_steps * ((F - F64) / (peak * 1e12) + F64 / (peak64 * 1e12))

    out = None
    if rank == 0:
        # e2e through the host-buffer C ABI
        e2e_t = []
        # the caller's output, page-locked (heom_host_alloc) and reused across scans: P is
        # copied into it by DMA and checked for Inf/NaN on the device
        host_out = heom.pinned_empty(max(tot, 1))
        for s in range(max(2, min(a.steps, 5))):
            t0 = time.perf_counter()
            r32 = plan.run_scan(pts, (pts, off, cnt, tot), out=host_out)
            e2e_t.append(time.perf_counter() - t0)
        r32 = heom.ScanResult(r32.P.copy(), r32.offsets, r32.counts)
        e2e_val = n / float(np.mean(e2e_t[1:] if len(e2e_t) > 1 else e2e_t))
        # accuracy gate: FP32-bulk vs the FP64 scan path on the full scan
        r64 = heom.Plan(prob, "fp64", device=local, max_points=n).run_scan(pts, (pts, off, cnt, tot))
        errs = [rel_err(r32.point(i), r64.point(i)) for i in range(n)]
        # against the binary128 truth of the reference's scheme on a stratified 48-point
        # subset of this scan (tests/golden/ref/truth_c2.npz, the first sample of the key)
        truth_acc = None
        if world == 1:
            from heomtest import truth
            t_rows, t_want, t_ref, t_gidx = truth("c2")
            if all(tuple(rows[int(g)]) == tuple(r) for g, r in zip(t_gidx, t_rows)):
                truth_acc = {"points": len(t_want),
                             "fp32_bulk_max_rel_err": max(rel_err(r32.point(int(g)), w) for g, w in zip(t_gidx, t_want)),
                             "fp64_staged_max_rel_err": max(rel_err(r64.point(int(g)), w) for g, w in zip(t_gidx, t_want)),
                             "reference_build_max_rel_err": max(rel_err(r, w) for r, w in zip(t_ref, t_want)),
                             "reference_build_median_rel_err": float(np.median([rel_err(r, w) for r, w in zip(t_ref, t_want)]))}
        # plain FP64 path (bit-exact, one point at a time) on a stratified sample
        tmpl = open(TEMPLATE).read()
        sample_idx = np.linspace(0, n - 1, 8).round().astype(int)
        plain_t, plain_steps = 0.0, 0
        tmpd = tempfile.mkdtemp()
        for i in sample_idx:
            r = rows[i]
            k = os.path.join(tmpd, "p.key")
            open(k, "w").write(tmpl.replace("TAU1", repr(r[0])).replace("TAU2", repr(r[1]))
                               .replace("TAU3", repr(r[2])).replace("T_END", repr(r[3])))
            pp = heom.Problem.from_key(k)
            pp.prepare_sample()
            pl = heom.Plan(pp, "fp64-exact", device=local)
            pl.run_2des()  # warm
            t0 = time.perf_counter()
            pl.run_2des()
            plain_t += time.perf_counter() - t0
            plain_steps += steps_of(r[3])
            pl.close()
        shutil.rmtree(tmpd, ignore_errors=True)
        # scale the sample to the whole scan by step count
        full_steps = sum(steps_of(r[3]) for r in rows)
        plain_val = n / (plain_t * full_steps / plain_steps)
        # CPU baseline: the reference build on a bounded sample
        cores = os.cpu_count() or 1
        cpu_val, kind, wall, _ = reference_cpu(rows, cores, cores)
        clocks = clk.summary()
        large_n = large_n_record(heom, local, peak)
        precision_c3 = c3_record(heom, local)
        adjoint = adjoint_record(heom, local)
        # cold-sample e2e: a new disorder/orientation sample before every scan
        # (heom_problem_prepare_sample + heom_plan_update + heom_run_scan), so the per-sample
        # set-up -- T0 and its squares on the GPU, the dual tail rows on the host -- falls
        # inside the timed region.  Run last: it moves the problem to new samples.
        cold_t = []
        for _ in range(3):
            t0 = time.perf_counter()
            prob.prepare_sample()
            plan.update()
            plan.run_scan(pts, (pts, off, cnt, tot), out=host_out)
            cold_t.append(time.perf_counter() - t0)
        warm_s = float(np.mean(e2e_t[1:] if len(e2e_t) > 1 else e2e_t))
        e2e_cold = {"value": n / float(np.mean(cold_t)), "unit": UNIT,
                    "h2d_bytes_per_step": int(pts.nbytes + off.nbytes), "d2h_bytes_per_step": int(16 * tot),
                    "setup_ms_per_sample": 1e3 * (float(np.mean(cold_t)) - warm_s),
                    "note": "a new disorder/orientation sample every step: prepare_sample + plan.update + "
                            "run_scan through the host-buffer C ABI; setup = cold minus warm e2e time"}
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 contractions / f64 state", "data": "synthetic",
            "config": {"workload": "c2: 1024-point dimer 2DES delay scan (64 t1 x 8 t2 x R/NR, t3 400 fs, "
                                   "dt 0.5 fs, N=4, 70 ADOs), batched FP32-bulk scan kernel",
                       "points_per_gpu": n, "rk4_steps_per_point": [min(steps_of(r[3]) for r in rows),
                                                                    max(steps_of(r[3]) for r in rows)],
                       "l2": "flushed (256 MB write) between timed steps; state is shared-memory resident",
                       "launch": plan.describe(), "parallelism": f"dp{world} (independent scans)"},
            "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": int(pts.nbytes + off.nbytes),
                    "d2h_bytes_per_step": int(16 * tot),
                    "note": "heom_run_scan with host buffers: points and offsets staged through the plan's "
                            "page-locked buffer, P copied into the caller's page-locked output array"},
            "e2e_cold": e2e_cold,
            "gpu_launches": int(launches),
            "host_ms_per_step": float(np.median(host_ms)),
            "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak,
                         "frac_mixed": t_bound / (ms / 1e3),
                         "peak_fp64": peak64,
                         "traffic": DRAM_BYTES_PER_SCAN if n == 1024 else None,
                         "executed_component_steps": int(exec_steps), "reference_trajectory_steps": int(traj_steps),
                         "reference_equivalent_tflops": ref_equiv,
                         "note": (f"algorithmic flops = {F:.0f} flop per component-step (4 stages: 16N^3 + 24N^2 "
                                  "per ADO, 16N per link) x the component-steps the staged scan propagates; "
                                  "reference_equivalent counts the reference's 3 trajectories x all steps; "
                                  "peak = FP32 FMA throughput measured in this run by the library's "
                                  "FMA-loop kernel (MEASURED_PEAKS.json holds only HBM and bf16 tensor peaks); "
                                  "frac_mixed = the time the FP32 work (16N^3 + links) needs at the FP32 peak "
                                  "plus the time the FP64 work (24N^2 per ADO and stage) needs at the measured "
                                  "FP64 FMA peak, over the measured time")},
            "accuracy": {"fp32_bulk_vs_fp64_max_rel_err": float(max(errs)),
                         "fp32_bulk_vs_fp64_median_rel_err": float(np.median(errs)), "points_checked": n,
                         "vs_binary128_truth": truth_acc},
            "plain_fp64": {"value": plain_val, "unit": UNIT, "sample": f"{len(sample_idx)} points, one at a time, "
                           "bit-exact FP64 path, scaled to the scan by RK4 step count",
                           "speedup_of_chosen": value / plain_val},
            "cpu_baseline": {"value": cpu_val, "unit": UNIT, "cores": cores, "cpu_model": cpu_model(), "kind": kind,
                             "sample": f"{cores} stratified scan points, one CPU_2DES process each, "
                                       f"{cores} concurrent ({wall:.1f} s); extrapolated to the 1024-point "
                                       "scan as points per second over the sample"},
            "clocks": clocks,
            "large_n": large_n,
            "precision_c3": precision_c3,
            "adjoint_c4": adjoint,
        }
        if averaged:
            out["disorder_average"] = averaged
        print(json.dumps(out), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return out


def profile_run(precision: str):
    """A small case of a kernel for profiler captures.

    fp32-bulk / fp64: the first 148 points of the dimer scan (one per SM) with t3
    shortened to 50 fs, default launch shape, one run of the scan kernel.
    fp32-bulk-tails: all 1024 points with t3 = 100 fs (the tail kernel's full grid).
    fp32-bulk-full: the bench's 1024-point scan, run twice (the second run is the bench's
    steady state: T0 and its powers are cached on the plan).
    c1-*: one 2DES point of the FMO key (N = 8, 680 ADOs) with the pulses at 10, 20 and
    30 fs (5 fs wide) and the end at 40 fs -- 81 RK4 steps of the general-size staged
    path (c1-fp32-bulk, c1-fp64) or of the bit-exact path (c1-fp64-exact)."""
    import torch

    from heomtest import load_pkg

    heom = load_pkg()
    if precision.startswith("c1-"):
        with open(os.path.join(ROOT, "tests", "golden", "keys", "c1_fmo.key")) as f:
            text = f.read()
        pulses = "PULSE\n3\n0.5308 50 20 12500\n0.5308 150 20 12500\n0.5308 250 20 12500"
        assert pulses in text and "TIME\n0 2000 0.5 0.5" in text
        text = text.replace(pulses, "PULSE\n3\n0.5308 10 5 12500\n0.5308 20 5 12500\n0.5308 30 5 12500")
        text = text.replace("TIME\n0 2000 0.5 0.5", "TIME\n0 40 0.5 0.5")
        d = tempfile.mkdtemp()
        path = os.path.join(d, "c1_small.key")
        with open(path, "w") as f:
            f.write(text)
        prob = heom.Problem.from_key(path)
        prob.prepare_sample()
        plan = heom.Plan(prob, precision[3:])
        t0 = time.perf_counter()
        P, _ = plan.run_2des(trajectories=False)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        shutil.rmtree(d, ignore_errors=True)
        print(f"profile run: FMO 2DES point, {len(P)} P values, {wall * 1e3:.1f} ms wall, {plan.describe()}")
        return
    prob = heom.Problem.from_key(KEY)
    prob.prepare_sample()
    if precision == "fp32-bulk-full":  # the bench's own 1024-point scan, run twice (T0 powers cached)
        plan = heom.Plan(prob, "fp32-bulk", max_points=1024)
        pts = heom.make_points(scan_rows())
        for _ in range(2):
            r = plan.run_scan(pts)
        torch.cuda.synchronize()
        print(f"profile run: 1024 points, {len(r.P)} P values, {plan.describe()}")
        return
    if precision == "fp32-bulk-tails":  # every point, t3 = 100 fs: the tail kernel's full grid
        rows = [(a, b, c, c + 100.0) for a, b, c, _ in scan_rows()]
        precision = "fp32-bulk"
    else:
        rows = [(a, b, c, c + 50.0) for a, b, c, _ in scan_rows()[:148]]
    plan = heom.Plan(prob, precision, max_points=len(rows))
    r = plan.run_scan(heom.make_points(rows))
    torch.cuda.synchronize()
    print(f"profile run: {len(rows)} points, {len(r.P)} P values, {plan.describe()}")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--profile-run", default=None, choices=["fp32-bulk", "fp64", "fp32-bulk-tails", "fp32-bulk-full", "c1-fp32-bulk", "c1-fp64",
                             "c1-fp64-exact"],
                    help="run only a small scan of that precision (for profiler captures)")
    a = ap.parse_args()
    if a.profile_run:
        profile_run(a.profile_run)
    elif a.impl == "reference":
        run_reference_arm(a)
    else:
        run_ours(a)


if __name__ == "__main__":
    main()
