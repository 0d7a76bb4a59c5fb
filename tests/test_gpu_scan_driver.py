"""The heom_scan driver end to end on the GPU (SURVEY 8f.1 replacement of
gen_2d_data.sh + submit_jobs.sh + one CPU_2DES process per key).

fp64-exact: every out_{tau}_{T}.out is byte-identical to the reference CPU_2DES output
of the same key file (tests/golden/ref/scan, generated by make_fixtures.py --golden).
fp64 (batched, mixed-difference basis): within 1e-4 of the reference's combined output,
whose own rounding noise is of that order.  fp32-bulk: within 2e-6 of fp64 (1e-6 FP32
contraction tolerance plus the printed 17-digit values).
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
    e64, e32 = [], []
    for n in sorted(os.listdir(GOLD)):
        ref, p64, p32 = _load(os.path.join(GOLD, n)), _load(o64 / n), _load(o32 / n)
        assert len(p64) == len(ref) == len(p32)
        e64.append(_rel(p64, ref))
        e32.append(_rel(p32, p64))
    print(f"fp64 batched vs CPU_2DES max {max(e64):.2e}; fp32-bulk vs fp64 max {max(e32):.2e}")
    assert max(e64) <= 1e-4 and max(e32) <= 2e-6
