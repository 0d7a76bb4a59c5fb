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


def _static_field_key(tmp_path, name, heom_line, dt, t_end=20):
    """The short dimer with time-independent pulses (carrier 0, width 1e9 fs, all three
    centred at t = 0, so P is recorded from the first step): V(t) = H - E0 (X0 + X1^T + X2^T)
    is constant and the step map is the RK4 polynomial of one fixed Liouvillian."""
    text = open(key("c0_dimer_short.key")).read()
    lines = text.split("\n")
    i = lines.index("PULSE")
    for q in range(3):
        lines[i + 2 + q] = "0.5308 0 1e9 0"
    j = lines.index("TIME")
    lines[j + 1] = f"0 {t_end} {dt!r} 0.5"
    if heom_line is not None:
        h = lines.index("HEOM")
        lines[h + 1] = heom_line
    k = tmp_path / name
    k.write_text("\n".join(lines))
    return str(k)


def test_rk4_global_error_is_fourth_order(tmp_path):
    """Halving dt divides the global error of P(t) by ~16 (autonomous linear system)."""
    P = []
    for dt in (0.125, 0.0625, 0.03125):
        p = oracle().load(_static_field_key(tmp_path, f"rk{dt}.key", None, dt))
        p.prepare_sample()
        P.append(p.traj((1, 1, 1)))
    assert len(P[0]) == len(P[1]) == len(P[2]) == 41
    e1 = np.abs(P[0] - P[1]).max()
    e2 = np.abs(P[1] - P[2]).max()
    ratio = e1 / e2
    print(f"RK4 error ratio for dt halving: {ratio:.2f}")
    assert 14.0 < ratio < 18.0


def test_single_ado_matches_step_polynomial_and_expm(tmp_path):
    """L = 0: one ADO, no bath couplings, drho/dt = -i[V, rho] with constant V.  The RK4
    step is exactly T4(hL) = sum_k (hL)^k / k! for k <= 4 (checked to rounding), and
    its result approaches expm(-i[V, .] t) with error O(h^4)."""
    from scipy.linalg import expm

    dt = 0.0625
    p = oracle().load(_static_field_key(tmp_path, "l0.key", "2 0", dt))
    p.prepare_sample()
    assert p.n_ado == 1
    N = p.N
    E0 = 0.5308 / 5308.0
    V = p.matrix(0) - E0 * (p.matrix(1) + p.matrix(2).T + p.matrix(3).T)
    X3 = p.matrix(4)
    # Liouvillian as an N^2 x N^2 matrix, column k = rhs(e_k)
    Lm = np.zeros((N * N, N * N), dtype=np.complex128)
    for k in range(N * N):
        e = np.zeros((1, N, N), dtype=np.complex128)
        e.flat[k] = 1.0
        Lm[:, k] = p.rhs(V, e).reshape(-1)
    # row-major vec: vec(V rho) = (V x I) vec(rho), vec(rho V) = (I x V^T) vec(rho)
    assert np.allclose(Lm, -1j * (np.kron(V, np.eye(N)) - np.kron(np.eye(N), V.T)), rtol=0, atol=1e-14)
    hL = dt * Lm
    T4 = np.eye(N * N) + hL + hL @ hL / 2 + hL @ hL @ hL / 6 + hL @ hL @ hL @ hL / 24
    U = expm(hL)
    rho_p = np.zeros(N * N, dtype=np.complex128)
    rho_p[0] = 1.0
    rho_e = rho_p.copy()
    Pp, Pe = [], []
    P = p.traj((1, 1, 1))
    stride = int(0.5 / dt)
    for i in range(len(P) * stride):
        if i % stride == 0:
            Pp.append(np.trace(rho_p.reshape(N, N) @ X3))
            Pe.append(np.trace(rho_e.reshape(N, N) @ X3))
        rho_p = T4 @ rho_p
        rho_e = U @ rho_e
    Pp, Pe = np.array(Pp), np.array(Pe)
    e_poly = np.abs(P - Pp).max() / np.abs(Pp).max()
    e_expm = np.abs(P - Pe).max() / np.abs(Pe).max()
    print(f"L=0: oracle vs RK4 polynomial {e_poly:.2e}, vs expm {e_expm:.2e}")
    assert e_poly < 1e-11
    assert e_expm < 1e-3 and e_expm > 10 * e_poly
