"""Pin the CPU oracle against the reference's own code (golden vectors), CPU only.

The golden vectors were produced by the reference's etoheom-cpu sources compiled
unmodified (oracle/_ref, see tests/golden/make_fixtures.py).  The oracle must match
them bit for bit -- per trajectory and on the combined output -- in both its dense
(reference-shaped) and structured (one-hot S as row/column ops) forms.
"""
import math

import numpy as np
import pytest

from heomtest import golden, key, oracle

GOLDEN_KEYS = ["c0_dimer_short.key", "t_disorder.key", "t_ref_example.key", "t_strong.key",
               "c4_trimer_short.key", "c1_fmo_short.key"]


@pytest.mark.parametrize("name", GOLDEN_KEYS)
@pytest.mark.parametrize("mode", [0, 1])
def test_oracle_bit_exact_vs_reference(name, mode):
    if mode == 0 and name.startswith("c1"):
        pytest.skip("dense N=29 form is minutes of CPU; the structured form covers it")
    traj_ref, comb_ref = golden(name)
    p = oracle().load(key(name))
    comb, traj = p.run_2des(mode=mode)
    assert comb.shape == comb_ref.shape
    assert np.array_equal(traj, traj_ref), "per-trajectory P(t) differs from the reference build"
    assert np.array_equal(comb, comb_ref), "combined P(t) differs from the reference build"


@pytest.mark.slow
def test_oracle_full_dimer_bit_exact():
    traj_ref, comb_ref = golden("c0_dimer.key")
    comb, traj = oracle().load(key("c0_dimer.key")).run_2des(mode=1)
    assert np.array_equal(comb, comb_ref) and np.array_equal(traj, traj_ref)


@pytest.mark.parametrize("name", ["c0_dimer.key", "c1_fmo.key", "c3_chain.key", "c4_trimer.key",
                                  "t_ref_example.key"])
def test_ado_count_is_binomial(name):
    p = oracle().load(key(name), single_manifold=name.startswith("c3"))
    M = p.K * p.K_m
    assert p.n_ado == math.comb(M + p.L, p.L)
    expected = {"c0_dimer.key": 70, "c1_fmo.key": 680, "c3_chain.key": 2925, "c4_trimer.key": 210}
    if name in expected:
        assert p.n_ado == expected[name]
    ado = p.ado()
    assert (ado.sum(axis=1) <= p.L).all()
    assert (ado[0] == 0).all()
    # lexicographic order, as the recursion in Build_ADO produces (utilize.cpp:3-18)
    rows = [tuple(r) for r in ado]
    assert rows == sorted(rows)
    assert len(set(rows)) == len(rows)


@pytest.mark.parametrize("name", ["t_ref_example.key", "t_strong.key", "c4_trimer_short.key"])
def test_dense_and_structured_rhs_identical(name):
    p = oracle().load(key(name))
    p.prepare_sample()
    rng = np.random.default_rng(3)
    N = p.N
    V = rng.normal(size=(N, N)) + 1j * rng.normal(size=(N, N))
    rho = rng.normal(size=(p.n_ado, N, N)) + 1j * rng.normal(size=(p.n_ado, N, N))
    a = p.rhs(V, rho, mode=0)
    b = p.rhs(V, rho, mode=1)
    assert np.array_equal(a, b)


def test_no_pulses_keeps_ground_state(tmp_path):
    # Zero field amplitude: rho stays |0><0| exactly and P(t) is exactly zero.
    text = open(key("c0_dimer_short.key")).read().replace("0.5308 ", "0 ")
    k = tmp_path / "nofield.key"
    k.write_text(text)
    comb, traj = oracle().load(str(k)).run_2des(mode=1)
    assert np.all(comb == 0) and np.all(traj == 0)


def test_linear_response_scales_with_field(tmp_path):
    # Pulse-3-only trajectory (mask 001): P is first order in E0 to high accuracy.
    base = open(key("c0_dimer_short.key")).read()
    out = []
    for scale in (1.0, 2.0):
        k = tmp_path / f"lin{scale}.key"
        k.write_text(base.replace("0.5308 ", f"{0.5308 * scale!r} "))
        p = oracle().load(str(k))
        p.prepare_sample()
        out.append(p.traj((0, 0, 1)))
    r = np.abs(out[1] - 2 * out[0]).max() / np.abs(out[1]).max()
    assert r < 1e-6
