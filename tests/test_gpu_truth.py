"""The scan paths against the true result of the reference's scheme, on the c2 scan.

The truth is the reference's discrete scheme (dynamics.cpp:298-432, CPU_2DES.cpp:65-79)
on its own double-precision problem data, propagated and combined in IEEE binary128
(oracle heom_oracle --quad; fixtures from tests/golden/make_fixtures.py --truth).  The
combined output p111 - p110 - p101 cancels up to ~9 orders of magnitude, so the
reference's own double result carries rounding noise far above 1e-10 of it; the truth
does not (~1e-24).  Gates, max_t |P - P_true| / max_t |P_true| per point:
  * FP64 scan (staged and single pass): <= 1e-10;
  * FP32-bulk scan (staged and single pass): <= 1e-6;
  * the bit-exact FP64 path reproduces the reference's own noise, which is printed.
The c2 subset is 48 points stratified over rephasing / non-rephasing, all 8 waiting
times and coherence times 0-315 fs, at full length (t3 = 400 fs), taken out of one run
of the full 1024-point scan.
"""
import os
import sys

import numpy as np
import pytest

from heomtest import key, load_pkg, rel_err, truth

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
from make_fixtures import scan_key_text, scan_points  # noqa: E402

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-10
FP32_TOL = 1e-6


@pytest.fixture(scope="module")
def dimer():
    heom = load_pkg()
    prob = heom.Problem.from_key(key("c0_dimer.key"))
    prob.prepare_sample()
    return heom, prob


def errors(result, idx, want):
    return np.array([rel_err(result.point(g), w) for g, w in zip(idx, want)])


@pytest.mark.parametrize("precision,tol", [("fp64", FP64_TOL), ("fp32-bulk", FP32_TOL)])
@pytest.mark.parametrize("single_pass", [False, True], ids=["staged", "single-pass"])
def test_c2_scan_vs_truth(dimer, precision, tol, single_pass):
    heom, prob = dimer
    rows, want, ref, gidx = truth("c2")
    grid = [(a, b, c, d) for a, b, c, d, _ in scan_points()]
    assert all(tuple(grid[g]) == tuple(r) for g, r in zip(gidx, rows))
    plan = heom.Plan(prob, precision, max_points=len(grid), single_pass=single_pass)
    res = plan.run_scan(heom.make_points(grid))
    for g, w in zip(gidx, want):
        assert res.counts[g] == len(w)
    e = errors(res, gidx, want)
    e_ref = np.array([rel_err(r, w) for r, w in zip(ref, want)])
    print(f"\n{precision} {'single pass' if single_pass else 'staged'} vs truth over {len(e)} c2 points: "
          f"max {e.max():.2e} median {np.median(e):.2e}; reference build vs truth: max {e_ref.max():.2e} "
          f"median {np.median(e_ref):.2e}")
    assert e.max() <= tol


def test_exact_path_carries_the_reference_noise(dimer, tmp_path):
    """The bit-exact path reproduces the reference build on c2 points, noise included:
    its error against the truth equals the reference's own, bit for bit."""
    heom, _ = dimer
    rows, want, ref, _ = truth("c2")
    picks = [0, len(rows) // 2 + 1, len(rows) - 1]   # shortest, a middle and the longest point
    for j in picks:
        k = tmp_path / f"p{j}.key"
        k.write_text(scan_key_text(rows[j]))
        p = heom.Problem.from_key(str(k))
        p.prepare_sample()
        P, _ = heom.Plan(p, "fp64-exact").run_2des()
        assert np.array_equal(P, ref[j])
        print(f"point {tuple(float(v) for v in rows[j])}: exact path (= reference build) vs truth "
              f"{rel_err(P, want[j]):.2e}")


@pytest.mark.parametrize("precision,tol", [("fp64", FP64_TOL), ("fp32-bulk", FP32_TOL)])
def test_short_scan_vs_truth(dimer, precision, tol):
    """The shortened 24-point scan of the scan tests (t3 = 150 fs), staged."""
    heom, prob = dimer
    rows, want, _, _ = truth("scan_short")
    plan = heom.Plan(prob, precision, max_points=len(rows))
    res = plan.run_scan(heom.make_points([tuple(r) for r in rows]))
    e = errors(res, range(len(rows)), want)
    print(f"\n{precision} vs truth, short scan: max {e.max():.2e}")
    assert e.max() <= tol
