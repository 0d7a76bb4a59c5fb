"""GPU checks of the batched delay-scan path (HEOM_FP64 / HEOM_FP32_BULK).

Accuracy gates (max_t |P - P_ref| / max_t |P_ref| per scan point, combined output):
  * FP32-bulk vs the FP64 scan path: <= 1e-6 (the FP32-bulk target);
  * FP64 scan vs the reference's own arithmetic (bit-exact path): the reference's
    combined output is a residue of per-trajectory values ~9 orders larger, so it
    carries its own rounding noise, measured per point against the binary128 truth
    (tests/golden/ref/truth_scan_short.npz).  The FP64 scan must lie within that noise
    plus 1e-10; its own error against the truth is gated in test_gpu_truth.py.
"""
import numpy as np
import pytest

from heomtest import key, load_pkg, rel_err, truth

pytestmark = pytest.mark.gpu

FP32_TOL = 1e-6


def scan_geometry(t0=50.0, t1s=(0.0, 35.0, 80.0, 155.0), t2s=(0.0, 100.0, 300.0), t3=150.0):
    rows = []
    for t2 in t2s:
        for t1 in t1s:
            rows.append((t0, t0 + t1, t0 + t1 + t2, t0 + t1 + t2 + t3))   # rephasing
            rows.append((t0 + t1, t0, t0 + t1 + t2, t0 + t1 + t2 + t3))   # non-rephasing
    return rows


@pytest.fixture(scope="module")
def setup():
    heom = load_pkg()
    prob = heom.Problem.from_key(key("c0_dimer.key"))
    prob.prepare_sample()
    return heom, prob


def exact_point(heom, prob, row, tmp_path_factory):
    # The bit-exact path on a key file with this point's pulse times.
    text = open(key("c2_dimer_scan.key-tmpl")).read()
    text = (text.replace("TAU1", repr(row[0])).replace("TAU2", repr(row[1])).replace("TAU3", repr(row[2]))
            .replace("T_END", repr(row[3])))
    d = tmp_path_factory.mktemp("pt")
    k = d / "p.key"
    k.write_text(text)
    p = heom.Problem.from_key(str(k))
    p.prepare_sample()
    P, _ = heom.Plan(p, "fp64-exact").run_2des()
    return P


def test_scan_fp32_vs_fp64(setup):
    heom, prob = setup
    rows = scan_geometry()
    pts = heom.make_points(rows)
    r64 = heom.Plan(prob, "fp64", max_points=len(rows)).run_scan(pts)
    r32 = heom.Plan(prob, "fp32-bulk", max_points=len(rows), autotune=True).run_scan(pts)
    assert np.array_equal(r64.counts, r32.counts)
    errs = [rel_err(r32.point(i), r64.point(i)) for i in range(len(rows))]
    print("fp32-bulk vs fp64 per point:", ["%.2e" % e for e in errs])
    assert max(errs) <= FP32_TOL


def test_scan_fp64_vs_reference_arithmetic(setup, tmp_path_factory):
    heom, prob = setup
    rows = scan_geometry()[:6]
    t_rows, t_want, _, _ = truth("scan_short")
    assert np.array_equal(t_rows[:6], np.array(rows))
    pts = heom.make_points(rows)
    r64 = heom.Plan(prob, "fp64", max_points=len(rows)).run_scan(pts)
    errs, noise = [], []
    for i, row in enumerate(rows):
        ref = exact_point(heom, prob, row, tmp_path_factory)
        assert len(ref) == r64.counts[i]
        errs.append(rel_err(r64.point(i), ref))
        noise.append(rel_err(ref, t_want[i]))
    print("fp64 scan vs reference arithmetic per point:", ["%.2e" % e for e in errs])
    print("reference arithmetic vs truth per point:   ", ["%.2e" % e for e in noise])
    for e, n in zip(errs, noise):
        assert e <= n * (1 + 1e-3) + 1e-10


def test_scan_point_order_does_not_matter(setup):
    heom, prob = setup
    rows = scan_geometry()
    pts = heom.make_points(rows)
    plan = heom.Plan(prob, "fp32-bulk", max_points=len(rows))
    a = plan.run_scan(pts)
    perm = np.random.default_rng(0).permutation(len(rows))
    b = plan.run_scan(pts[perm])
    for j, i in enumerate(perm):
        assert np.array_equal(a.point(i), b.point(j))


def test_scan_device_entry_matches_host_entry(setup):
    import torch
    heom, prob = setup
    rows = scan_geometry()
    plan = heom.Plan(prob, "fp32-bulk", max_points=len(rows))
    pts, off, cnt, tot = plan.scan_layout(heom.make_points(rows))
    host = plan.run_scan(pts, (pts, off, cnt, tot))
    d_pts = torch.from_numpy(pts.view(np.uint8).copy()).cuda()
    d_off = torch.from_numpy(off).cuda()
    d_P = torch.zeros(2 * tot, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    plan.run_scan_device(d_pts.data_ptr(), len(pts), d_P.data_ptr(), d_off.data_ptr())
    # the plan runs on its own stream; a device-wide sync orders the read-back
    torch.cuda.synchronize()
    dev = d_P.cpu().numpy().view(np.complex128)
    assert np.array_equal(dev, host.P)


@pytest.mark.parametrize("precision,tol", [("fp32-bulk", FP32_TOL), ("fp64", 1e-11)])
def test_staged_scan_matches_single_pass(setup, precision, tol):
    """The staged scan (shared R/D2 per (tau1, tau2), per-point pulse-3 windows, tails
    D = Q - R four per CTA) against the single pass.  Up to each point's pulse-3 window
    end it performs the single-pass operations on the same values; the tail propagates
    Q - R instead of Q and R, which changes rounding only.  Includes points that cannot
    be staged: pulse 3 before pulse 2, pulse 3 outside the point, an end time inside
    pulse 3's window."""
    heom, prob = setup
    rows = scan_geometry() + [(50.0, 150.0, 90.0, 260.0), (50.0, 80.0, 400.0, 300.0), (50.0, 70.0, 120.0, 130.0)]
    pts = heom.make_points(rows)
    staged = heom.Plan(prob, precision, max_points=len(rows))
    single = heom.Plan(prob, precision, max_points=len(rows), single_pass=True)
    a, b = staged.run_scan(pts), single.run_scan(pts)
    assert np.array_equal(a.counts, b.counts)
    errs = [rel_err(a.point(i), b.point(i)) for i in range(len(rows))]
    print(f"{precision} staged vs single pass: max {max(errs):.2e}")
    assert max(errs) <= tol
    # the device entry plans the same stages from the points it reads back
    import torch
    lay = staged.scan_layout(pts)
    d_pts = torch.from_numpy(lay[0].view(np.uint8).copy()).cuda()
    d_off = torch.from_numpy(lay[1].copy()).cuda()
    d_P = torch.zeros(2 * lay[3], dtype=torch.float64, device="cuda")
    staged.run_scan_device(d_pts.data_ptr(), len(rows), d_P.data_ptr(), d_off.data_ptr())
    torch.cuda.synchronize()
    Pd = d_P.cpu().numpy().view(np.complex128)
    assert np.array_equal(Pd, a.P[:lay[3]])


def test_staged_jump_chains_match_single_pass(setup):
    """Whole t2 columns of the delay grid (8 delays 100 fs apart) for a few t1: each
    (tau1, tau2) group's jump job carries D2 through seven members, and every 200-step
    leg between consecutive delays is one product with the prepared leg T0^200.  The
    FP64 staged scan against the FP64 single pass, which steps every point."""
    heom, prob = setup
    rows = []
    for t1 in (0.0, 45.0, 160.0):
        for t2 in [100.0 * k for k in range(8)]:
            rows.append((50.0, 50.0 + t1, 50.0 + t1 + t2, 50.0 + t1 + t2 + 400.0))  # rephasing
            rows.append((50.0 + t1, 50.0, 50.0 + t1 + t2, 50.0 + t1 + t2 + 400.0))  # non-rephasing
    pts = heom.make_points(rows)
    staged = heom.Plan(prob, "fp64", max_points=len(rows))
    single = heom.Plan(prob, "fp64", max_points=len(rows), single_pass=True)
    a, b = staged.run_scan(pts), single.run_scan(pts)
    assert np.array_equal(a.counts, b.counts)
    errs = [rel_err(a.point(i), b.point(i)) for i in range(len(rows))]
    print(f"jump chains, fp64 staged vs single pass: max {max(errs):.2e}")
    assert max(errs) <= 1e-11


@pytest.mark.parametrize("precision", ["fp32-bulk", "fp64"])
def test_scan_edge_cases(setup, precision):
    """An empty scan, and a staged scan mixing ordinary points with points that record
    nothing (end before pulse 3) and a point that ends inside pulse 3's window: the
    empty points get no output and leave the others unchanged."""
    heom, prob = setup
    plan = heom.Plan(prob, precision, max_points=16)
    empty = plan.run_scan(heom.make_points([]))
    assert len(empty.P) == 0
    base = scan_geometry()[:4]
    odd = [(50.0, 100.0, 300.0, 250.0),   # ends before pulse 3: no record
           (50.0, 60.0, 200.0, 210.0),    # ends inside pulse 3's window
           (60.0, 50.0, 400.0, 120.0)]    # ends before pulse 2
    mixed = base[:2] + odd + base[2:]
    r = plan.run_scan(heom.make_points(mixed))
    alone = plan.run_scan(heom.make_points(base))
    assert r.counts[2] == 0 and r.counts[4] == 0 and r.counts[3] > 0
    for j, i in enumerate([0, 1, 5, 6]):
        assert rel_err(r.point(i), alone.point(j)) <= (1e-6 if precision == "fp32-bulk" else 1e-11)
    assert np.isfinite(r.P).all()


def test_staged_replay_matches_planned_run():
    """A repeated staged scan skips the host planning and replays the last plan, also for
    a new sample of the same structure (plan.update), whose T0 powers and dual rows are
    formed again.  Both give the bits of a freshly planned run."""
    heom = load_pkg()
    rows = scan_geometry()
    pts = heom.make_points(rows)
    pa = heom.Problem.from_key(key("c0_dimer.key"))
    pa.prepare_sample()
    plan = heom.Plan(pa, "fp32-bulk", max_points=len(rows))
    first = plan.run_scan(pts)
    work = plan.scan_work
    again = plan.run_scan(pts)                    # replayed: captured into a CUDA graph
    thrice = plan.run_scan(pts)                   # the graph launched again
    assert np.array_equal(first.P, again.P) and np.array_equal(first.P, thrice.P) and plan.scan_work == work
    pa.prepare_sample()
    plan.update()
    second = plan.run_scan(pts)                   # replayed on the new sample (new dual rows: no graph)
    assert np.array_equal(plan.run_scan(pts).P, second.P)   # and as a graph again
    pb = heom.Problem.from_key(key("c0_dimer.key"))
    pb.prepare_sample()
    pb.prepare_sample()
    fresh = heom.Plan(pb, "fp32-bulk", max_points=len(rows)).run_scan(pts)
    assert np.array_equal(second.P, fresh.P)
    assert not np.array_equal(second.P, first.P)


def test_scan_into_caller_buffer(setup):
    heom, prob = setup
    rows = scan_geometry()[:6]
    plan = heom.Plan(prob, "fp32-bulk", max_points=len(rows))
    lay = plan.scan_layout(heom.make_points(rows))
    want = plan.run_scan(lay[0], lay)
    buf = np.full(lay[3] + 5, np.nan, dtype=np.complex128)
    got = plan.run_scan(lay[0], lay, out=buf)
    assert np.shares_memory(got.P, buf) and np.array_equal(got.P, want.P)
    with pytest.raises(ValueError):
        plan.run_scan(lay[0], lay, out=np.zeros(lay[3] - 1, dtype=np.complex128))


def test_scan_into_page_locked_buffer(setup):
    """An output array from heom_host_alloc receives P by DMA with the Inf/NaN check on
    the device (one extra launch); the result equals the staged copy-out bit for bit,
    also at an offset that ends exactly at the buffer's end, and when the buffer is
    reused."""
    heom, prob = setup
    rows = scan_geometry()[:6]
    plan = heom.Plan(prob, "fp32-bulk", max_points=len(rows))
    lay = plan.scan_layout(heom.make_points(rows))
    want = plan.run_scan(lay[0], lay)
    pinned = heom.pinned_empty(lay[3] + 8)
    for start in (0, 8, 0):
        view = pinned[start:start + lay[3]]
        before = plan.launches
        got = plan.run_scan(lay[0], lay, out=view)
        assert np.shares_memory(got.P, pinned) and np.array_equal(got.P, want.P)
        assert plan.launches - before >= 1
