"""Pin the binary128 truth oracle (ho_2des_q) and its fixtures, CPU only.

ho_2des_q runs the reference's scheme on the reference's own double-precision data
with the propagation and the combination p111 - p110 - p101 in binary128.  Its
trajectories must agree with the reference build's (golden vectors from oracle/_ref)
to the reference's double rounding, ~1e-15; its combined output is the true one, from
which the reference build departs by the rounding noise that the cancellation
amplifies.  The committed truth fixtures are checked the same way.
"""
import numpy as np
import pytest

from heomtest import golden, key, oracle, rel_err, truth


@pytest.mark.parametrize("name", ["t_strong.key", "t_disorder.key"])
def test_truth_trajectories_match_reference_build(name):
    traj_ref, comb_ref = golden(name)
    comb, traj = oracle().load(key(name)).run_2des_truth()
    assert traj.shape == traj_ref.shape
    e = max(rel_err(traj[s, m], traj_ref[s, m]) for s in range(traj.shape[0]) for m in range(3))
    print(f"\n{name}: trajectories vs reference build {e:.2e}; reference combined vs truth "
          f"{rel_err(comb_ref, comb):.2e}")
    assert e <= 1e-14


def test_truth_fixture_matches_reference_build():
    d = np.load(__import__("os").path.join(__import__("heomtest").REF, "truth_c0_dimer_short.npz"))
    traj_ref, comb_ref = golden("c0_dimer_short.key")
    assert d["traj"].shape == traj_ref.shape
    e = max(rel_err(d["traj"][0, m], traj_ref[0, m]) for m in range(3))
    assert e <= 1e-14
    # the reference's combined output carries its rounding noise, well above 1e-10 here
    noise = rel_err(comb_ref, d["combined"])
    print(f"\nc0 short point: reference combined vs truth {noise:.2e}")
    assert 1e-10 < noise < 1e-4


def test_c2_truth_fixture():
    rows, want, ref, gidx = truth("c2")
    assert len(rows) == 48 and len(set(gidx.tolist())) == 48
    # both kinds and all 8 waiting times, t3 = 400 fs
    t2 = {round(r[2] - max(r[0], r[1])) for r in rows}
    assert t2 == {0, 100, 200, 300, 400, 500, 600, 700}
    assert all(abs(r[3] - r[2] - 400.0) < 1e-9 for r in rows)
    assert any(r[0] < r[1] for r in rows) and any(r[0] > r[1] for r in rows)
    e = np.array([rel_err(r, w) for r, w in zip(ref, want)])
    print(f"\nreference build vs truth over the c2 subset: max {e.max():.2e} median {np.median(e):.2e} "
          f"min {e.min():.2e}")
    assert all(np.isfinite(w).all() and np.abs(w).max() > 0 for w in want)
    assert e.max() < 0.1


def test_split_trajectories_combine_to_the_truth():
    """heom_oracle --quad-mask runs one binary128 trajectory and prints (hi, lo) pairs; the
    three masks combined exactly reproduce ho_2des_q's combined output bit for bit."""
    import os
    import subprocess
    import sys
    from heomtest import ROOT
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    from make_fixtures import _split_values
    exe = os.path.join(ROOT, "oracle", "heom_oracle")
    if not os.path.exists(exe):
        subprocess.check_call(["make", "-C", os.path.join(ROOT, "oracle"), "heom_oracle"])
    outs = [_split_values(subprocess.run([exe, key("t_strong.key"), "--quad-mask", m], check=True,
                                         capture_output=True, text=True).stdout) for m in ("111", "110", "101")]
    comb = np.array([complex(float(a[0] - b[0] - c[0]), float(a[1] - b[1] - c[1])) for a, b, c in zip(*outs)])
    want, _ = oracle().load(key("t_strong.key")).run_2des_truth()
    assert np.array_equal(comb, want)


@pytest.mark.parametrize("name", ["c4_trimer.key", "c1_fmo_300fs.key"])
def test_large_key_truth_fixture(name):
    """The binary128 truth of the config-4 trimer (0-1000 fs) and of the FMO aggregate
    through its three pulse windows (0-300 fs): one combined value per reference record,
    departing from the reference build's combined output by its rounding noise only."""
    import os
    from heomtest import REF
    want = np.load(os.path.join(REF, "truth_" + name.replace(".key", ".npz")))["combined"]
    _, comb_ref = golden(name)
    assert want.shape == comb_ref.shape and np.isfinite(want).all() and np.abs(want).max() > 0
    noise = rel_err(comb_ref, want)
    print(f"\n{name}: reference combined vs truth {noise:.2e}")
    assert 1e-12 < noise < 1e-5
