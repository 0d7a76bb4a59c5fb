"""GPU check of heom_run_scan_noalloc, the delay-scan entry point that allocates nothing.

It exists for callers that cannot let a library allocate device memory (their whole
budget is reserved up front by their own pool or a framework's caching allocator, or
allocation is allowed only during initialisation).  Its scratch lives in a fixed
file-scope device array, so this test calls it twice in a row through the C ABI -- the
second call reuses the first call's scratch contents -- and compares both outputs with
the plan-based entry point's (heom_run_scan) on the same inputs, and that the second call
leaves the device's free memory unchanged.  The file sorts last so that a run stopping
at the first failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

from heomtest import key, load_pkg, rel_err

pytestmark = pytest.mark.gpu

FP32_TOL = 1e-6  # the FP32-bulk tolerance used by the scan tests


def _rows():
    rows = []
    for t2 in (0.0, 100.0):
        for t1 in (0.0, 25.0, 60.0):
            rows.append((50.0, 50.0 + t1, 50.0 + t1 + t2, 50.0 + t1 + t2 + 120.0))
            rows.append((50.0 + t1, 50.0, 50.0 + t1 + t2, 50.0 + t1 + t2 + 120.0))
    return rows


def test_noalloc_scan_matches_plan_entry_twice():
    import torch

    heom = load_pkg()
    prob = heom.Problem.from_key(key("c0_dimer.key"))
    prob.prepare_sample()
    rows = _rows()
    plan = heom.Plan(prob, "fp32-bulk", max_points=len(rows))
    pts, off, cnt, tot = plan.scan_layout(heom.make_points(rows))
    ref = plan.run_scan(pts, (pts, off, cnt, tot))

    d_pts = torch.from_numpy(pts.view(np.uint8).copy()).cuda()
    d_off = torch.from_numpy(off.copy()).cuda()
    stream = torch.cuda.current_stream().cuda_stream
    L = heom.lib()
    d_P = torch.empty((2 * tot,), dtype=torch.float64, device="cuda")
    h_P = torch.empty((2 * tot,), dtype=torch.float64, pin_memory=True)
    free_after_first = None
    for call in range(2):
        d_P.fill_(float("nan"))
        torch.cuda.synchronize()
        rc = L.heom_run_scan_noalloc(prob._h, heom.FP32_BULK, ctypes.c_void_p(d_pts.data_ptr()), len(rows),
                                     ctypes.c_void_p(d_P.data_ptr()), ctypes.c_void_p(d_off.data_ptr()),
                                     ctypes.c_void_p(stream))
        assert rc == 0, L.heom_last_error().decode()
        torch.cuda.synchronize()
        # the property the entry point exists for: after the first call (which may load
        # the module's static array) no call changes the device's free memory
        free = torch.cuda.mem_get_info()[0]
        if call == 0:
            free_after_first = free
        else:
            assert free == free_after_first, f"device free memory moved by {free_after_first - free} bytes"
        h_P.copy_(d_P)
        out = h_P.numpy().view(np.complex128)
        assert np.isfinite(out).all(), f"call {call}: output not fully written"
        errs = [rel_err(out[off[i]:off[i] + cnt[i]], ref.point(i)) for i in range(len(rows))]
        assert max(errs) <= FP32_TOL, f"call {call}: max rel err {max(errs):.3e}"


def test_noalloc_rejects_sizes_beyond_its_scratch():
    heom = load_pkg()
    prob = heom.Problem.from_key(key("c0_dimer.key"))
    prob.prepare_sample()
    L = heom.lib()
    rc = L.heom_run_scan_noalloc(prob._h, heom.FP32_BULK, ctypes.c_void_p(16), 65537, ctypes.c_void_p(16),
                                 ctypes.c_void_p(16), None)
    assert rc == -6 and "65536" in L.heom_last_error().decode()
