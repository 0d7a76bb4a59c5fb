"""Bounded device-side waits of the staged scan, and deferred error reporting.

The staged scan's jobs wait for their producers' flags with a limit on %globaltimer
(scan_slots).  The reference has no such waits; its errors exit the process
(etoheom-gpu/lib/HEOM_utilize.h:23-38).  Here a wait that expires sets an error word
that the host reads, and the context stays usable.  The test makes one wait expire by
the plan's test hook: one consumer job waits for a flag value that no producer sets,
with a 0.5 s limit.  Every access stays in bounds and every wait ends.
"""
import numpy as np
import pytest

from heomtest import key, load_pkg
from test_gpu_scan import scan_geometry

pytestmark = pytest.mark.gpu

WAIT_NS = 500_000_000   # 0.5 s: far above every legitimate wait of this small scan


@pytest.fixture(scope="module")
def setup():
    heom = load_pkg()
    prob = heom.Problem.from_key(key("c0_dimer.key"))
    prob.prepare_sample()
    rows = scan_geometry()
    return heom, prob, rows


def test_expired_wait_is_reported_by_the_host_entry(setup):
    heom, prob, rows = setup
    plan = heom.Plan(prob, "fp32-bulk", max_points=len(rows))
    pts = heom.make_points(rows)
    good = plan.run_scan(pts)
    plan.inject_wait_fault(WAIT_NS)
    with pytest.raises(heom.HeomError) as ei:
        plan.run_scan(pts)
    assert ei.value.code == -9, str(ei.value)
    # the next run on the same plan is unaffected
    again = plan.run_scan(pts)
    assert np.array_equal(again.P, good.P)


def test_expired_wait_is_deferred_to_sync_on_the_device_entry(setup):
    import torch
    heom, prob, rows = setup
    plan = heom.Plan(prob, "fp32-bulk", max_points=len(rows))
    pts, off, cnt, tot = plan.scan_layout(heom.make_points(rows))
    good = plan.run_scan(pts, (pts, off, cnt, tot))
    d_pts = torch.from_numpy(pts.view(np.uint8).copy()).cuda()
    d_off = torch.from_numpy(off).cuda()
    d_P = torch.zeros(2 * tot, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    plan.inject_wait_fault(WAIT_NS)
    plan.run_scan_device(d_pts.data_ptr(), len(pts), d_P.data_ptr(), d_off.data_ptr())   # returns at once
    with pytest.raises(heom.HeomError) as ei:
        plan.sync()
    assert ei.value.code == -9, str(ei.value)
    P = d_P.cpu().numpy().view(np.complex128)
    assert np.isnan(P).any(), "the job whose wait expired must leave NaN in its records"
    plan.sync()   # the status was consumed
    # a clean device-entry run afterwards
    d_P.zero_()
    torch.cuda.synchronize()
    plan.run_scan_device(d_pts.data_ptr(), len(pts), d_P.data_ptr(), d_off.data_ptr())
    plan.sync()
    assert np.array_equal(d_P.cpu().numpy().view(np.complex128), good.P)


def test_inject_hook_rejects_bad_limits(setup):
    heom, prob, rows = setup
    plan = heom.Plan(prob, "fp32-bulk", max_points=len(rows))
    for bad in (0, 61_000_000_000):
        with pytest.raises(heom.HeomError):
            plan.inject_wait_fault(bad)
