"""The heom_scan driver end to end on the GPU: the replacement of gen_2d_data.sh +
submit_jobs.sh + one CPU_2DES process per key.

fp64-exact: every out_{tau}_{T}.out is byte-identical to the reference CPU_2DES output
of the same key file (tests/golden/ref/scan, generated by make_fixtures.py --golden).
fp64 (batched, mixed-difference basis) and fp32-bulk, printed at full precision: within
1e-10 and 1e-6 of the binary128 truth of each file (tests/golden/ref/truth_scan_driver.npz,
disorder-averaged over the key's two samples).  The reference's own file departs from
the truth by its 7 printed digits plus its rounding noise, which is printed.
"""
import os
import subprocess

import numpy as np
import pytest

from heomtest import REF
from test_scan_driver import EXE, _template_args

pytestmark = pytest.mark.gpu

GOLD = os.path.join(REF, "scan")


def _run(tmp_path, tag, *extra):
    out = tmp_path / tag
    r = subprocess.run(_template_args(tmp_path / "in", out) + list(extra), capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return out


def _load(path):
    v = np.loadtxt(path, ndmin=2)
    return v[:, 0] + 1j * v[:, 1]


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def test_scan_driver_exact_is_byte_identical(tmp_path):
    out = _run(tmp_path, "exact", "--precision", "fp64-exact")
    names = sorted(os.listdir(GOLD))
    assert sorted(os.listdir(out)) == names and len(names) == 10
    for n in names:
        assert (out / n).read_bytes() == open(os.path.join(GOLD, n), "rb").read(), n


def test_scan_driver_batched_precisions(tmp_path):
    o64 = _run(tmp_path, "f64", "--precision", "fp64", "--full-precision")
    o32 = _run(tmp_path, "f32", "--precision", "fp32-bulk", "--full-precision")
    t = np.load(os.path.join(REF, "truth_scan_driver.npz"))
    truth = {str(n): t["truth"][t["offsets"][i]:t["offsets"][i + 1]] for i, n in enumerate(t["names"])}
    e64, e32, eref = [], [], []
    for n in sorted(os.listdir(GOLD)):
        ref, p64, p32 = _load(os.path.join(GOLD, n)), _load(o64 / n), _load(o32 / n)
        assert len(p64) == len(ref) == len(p32) == len(truth[n])
        e64.append(_rel(p64, truth[n]))
        e32.append(_rel(p32, truth[n]))
        eref.append(_rel(ref, truth[n]))
    print(f"vs truth: fp64 batched max {max(e64):.2e}; fp32-bulk max {max(e32):.2e}; "
          f"CPU_2DES (7 digits) max {max(eref):.2e}")
    assert max(e64) <= 1e-10 and max(e32) <= 1e-6
