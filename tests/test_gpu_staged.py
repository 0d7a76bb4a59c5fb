"""GPU checks of the general-size staged path (HEOM_FP64 / HEOM_FP32_BULK for any N).

Per trajectory the FP64 staged path differs from the reference only by operation order
(fused multiply-adds, Horner form of RK4), so it must agree with the bit-exact path to
~1e-12 relative; FP32-bulk must stay within 1e-6 of FP64.  The c3 test is the precision
study of the single-excitation chain (N = 13, 2925 ADOs, 6000 RK4 steps, linear
response): the FP32-bulk error against the FP64 reference arithmetic is printed and
bounded.
"""
import os

import numpy as np
import pytest

from heomtest import REF, golden, key, load_pkg, rel_err

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
FP32_TOL = 1e-6


def _plan(heom, name, precision, single=False):
    prob = heom.Problem.from_key(key(name), single_manifold=single)
    prob.prepare_sample()
    return prob, heom.Plan(prob, precision)


@pytest.mark.parametrize("name,mask", [("c4_trimer_short.key", (1, 1, 1)), ("c4_trimer_short.key", (0, 1, 0)),
                                       ("c1_fmo_short.key", (1, 1, 1)), ("c3_chain_short.key", (0, 0, 1))])
def test_staged_trajectory_matches_exact(name, mask):
    heom = load_pkg()
    single = name.startswith("c3")
    _, exact = _plan(heom, name, "fp64-exact", single)
    _, f64 = _plan(heom, name, "fp64", single)
    _, f32 = _plan(heom, name, "fp32-bulk", single)
    ref = exact.run_traj(*mask)
    p64 = f64.run_traj(*mask)
    p32 = f32.run_traj(*mask)
    e64, e32 = rel_err(p64, ref), rel_err(p32, p64)
    print(f"{name} {mask}: fp64 staged vs exact {e64:.2e}, fp32-bulk vs fp64 {e32:.2e}")
    assert len(p64) == len(ref) and e64 <= FP64_TOL and e32 <= FP32_TOL


def test_staged_2des_point_matches_reference():
    heom = load_pkg()
    traj_ref, comb_ref = golden("c4_trimer_short.key")
    _, f64 = _plan(heom, "c4_trimer_short.key", "fp64")
    P, tr = f64.run_2des()
    for t in range(3):
        assert rel_err(tr[t], traj_ref[0, t]) <= FP64_TOL
    # the combined output against the binary128 truth of the reference's scheme; the
    # reference's own combined output departs from it by its rounding noise
    true = np.load(os.path.join(REF, "truth_c4_trimer_short.npz"))["combined"]
    e, noise = rel_err(P, true), rel_err(comb_ref, true)
    print(f"trimer combined vs truth: fp64 mixed-difference basis {e:.2e}, reference arithmetic {noise:.2e}")
    assert e <= 1e-10
    _, f32 = _plan(heom, "c4_trimer_short.key", "fp32-bulk")
    P32, _ = f32.run_2des()
    assert rel_err(P32, true) <= FP32_TOL


def test_trimer_scan_runs_on_staged_path():
    heom = load_pkg()
    prob = heom.Problem.from_key(key("c4_trimer.key"))
    prob.prepare_sample()
    rows = [(50.0, 50.0 + t1, 250.0 + t1, 330.0 + t1) for t1 in (0.0, 20.0, 45.0)]
    pts = heom.make_points(rows)
    r64 = heom.Plan(prob, "fp64", max_points=len(rows)).run_scan(pts)
    plan32 = heom.Plan(prob, "fp32-bulk", max_points=len(rows))
    assert "unsupported" in plan32.describe()  # does not fit one CTA: staged path serves it
    r32 = plan32.run_scan(pts)
    for i in range(len(rows)):
        assert rel_err(r32.point(i), r64.point(i)) <= FP32_TOL


def test_c3_chain_precision_study():
    heom = load_pkg()
    _, exact = _plan(heom, "c3_chain.key", "fp64-exact", True)
    _, f64 = _plan(heom, "c3_chain.key", "fp64", True)
    _, f32 = _plan(heom, "c3_chain.key", "fp32-bulk", True)
    ref = exact.run_traj(0, 0, 1)
    p64 = f64.run_traj(0, 0, 1)
    p32 = f32.run_traj(0, 0, 1)
    assert len(ref) == 5901
    e64, e32, e32x = rel_err(p64, ref), rel_err(p32, p64), rel_err(p32, ref)
    print(f"c3 chain (N=13, 2925 ADOs, 6001 steps): fp64 staged vs exact {e64:.2e}; "
          f"fp32-bulk vs fp64 {e32:.2e}; fp32-bulk vs exact {e32x:.2e}")
    assert e64 <= 1e-10 and e32x <= 1e-5


@pytest.mark.parametrize("precision", ["fp64-exact", "fp64", "fp32-bulk"])
def test_run_with_no_records(tmp_path, precision):
    """A key whose end time precedes pulse 3 records nothing (the reference prints no line)."""
    heom = load_pkg()
    with open(key("c4_trimer_short.key")) as f:
        text = f.read()
    assert "TIME\n0 160 0.5 0.5" in text
    k = tmp_path / "early_end.key"
    k.write_text(text.replace("TIME\n0 160 0.5 0.5", "TIME\n0 40 0.5 0.5"))
    prob = heom.Problem.from_key(str(k))
    prob.prepare_sample()
    assert prob.info.n_record == 0
    P, tr = heom.Plan(prob, precision).run_2des()
    assert len(P) == 0 and all(len(t) == 0 for t in tr)


def test_trimer_full_2des_vs_truth():
    """The config-4 trimer (N = 7, 210 ADOs) over 0-1000 fs (2001 steps, pulses at 50,
    150 and 350 fs) on the general-size staged path, against the binary128 truth; the
    reference build's own combined output is printed beside it."""
    heom = load_pkg()
    true = np.load(os.path.join(REF, "truth_c4_trimer.npz"))["combined"]
    _, comb_ref = golden("c4_trimer.key")
    errs = {}
    for prec, tol in (("fp64", 1e-10), ("fp32-bulk", FP32_TOL)):
        _, plan = _plan(heom, "c4_trimer.key", prec)
        P, _ = plan.run_2des(trajectories=False)
        errs[prec] = rel_err(P, true)
        assert len(P) == len(true) and errs[prec] <= tol
    print(f"\ntrimer 0-1000 fs vs truth: fp64 staged {errs['fp64']:.2e}, fp32-bulk {errs['fp32-bulk']:.2e}, "
          f"reference build {rel_err(comb_ref, true):.2e}")


def test_fmo_2des_vs_truth():
    """The FMO aggregate (N = 29, 680 ADOs) through all three pulse windows (601 steps) on
    the general-size staged path, against the binary128 truth (three trajectories run
    separately and combined exactly); the reference build's own output is printed."""
    heom = load_pkg()
    true = np.load(os.path.join(REF, "truth_c1_fmo_300fs.npz"))["combined"]
    _, comb_ref = golden("c1_fmo_300fs.key")
    errs = {}
    for prec, tol in (("fp64", 1e-10), ("fp32-bulk", FP32_TOL)):
        _, plan = _plan(heom, "c1_fmo_300fs.key", prec)
        P, _ = plan.run_2des(trajectories=False)
        errs[prec] = rel_err(P, true)
        assert len(P) == len(true) and errs[prec] <= tol
    print(f"\nFMO 0-300 fs vs truth: fp64 staged {errs['fp64']:.2e}, fp32-bulk {errs['fp32-bulk']:.2e}, "
          f"reference build {rel_err(comb_ref, true):.2e}")
