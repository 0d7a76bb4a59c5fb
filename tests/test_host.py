"""Host-side set-up of libheom.so against the oracle, CPU only (no kernel launches).

Key-file parsing, the ADO hierarchy, construct_Hal (disorder draws + diagonal sort +
two-exciton block), the orientational rotation and X[0..3] must match the oracle bit for
bit, sample after sample (the RNG stream is shared between disorder and rotation).
"""
import os
import re

import numpy as np
import pytest

from heomtest import ROOT, cuda_available, key, load_pkg, oracle

KEYS = ["c0_dimer.key", "c1_fmo.key", "c3_chain.key", "c4_trimer.key", "t_disorder.key", "t_ref_example.key",
        "t_strong.key"]


@pytest.fixture(scope="module")
def heom():
    return load_pkg()


@pytest.mark.parametrize("name", KEYS)
def test_setup_matches_oracle(heom, name):
    single = name.startswith("c3")
    prob = heom.Problem.from_key(key(name))
    ref = oracle().load(key(name), single_manifold=single)
    inf = prob.info
    assert (inf.single_size, inf.sys_size, inf.K, inf.K_m, inf.L, inf.n_ado, inf.n_sample) == (
        ref.single_size, ref.N, ref.K, ref.K_m, ref.L, ref.n_ado, ref.n_sample)
    assert inf.n_steps == ref.n_steps and inf.print_stride == ref.stride
    assert np.array_equal(prob.ado(), ref.ado())
    assert np.array_equal(prob.matrix(heom.MAT_HKEY), ref.matrix(5))
    for s in range(min(inf.n_sample, 3)):
        prob.prepare_sample()
        ref.prepare_sample()
        assert np.array_equal(prob.matrix(heom.MAT_H), ref.matrix(0)), f"H differs at sample {s}"
        for q in range(4):
            assert np.array_equal(prob.matrix(heom.MAT_X0 + q), ref.matrix(1 + q)), f"X{q} differs at sample {s}"


def test_identity_preparation(heom):
    prob = heom.Problem.from_key(key("t_disorder.key"))
    ref = oracle().load(key("t_disorder.key"))
    prob.prepare_identity()
    ref.prepare_identity()
    assert np.array_equal(prob.matrix(heom.MAT_H), ref.matrix(0))
    assert np.array_equal(prob.matrix(heom.MAT_X0), ref.matrix(1))
    # the diagonal sort leaves H[0][0] = 0 and sorts the single-excitation energies
    d = np.real(np.diag(prob.matrix(heom.MAT_H)))[1:3]
    assert d[0] <= d[1]


def test_rng_reset_repeats_samples(heom):
    prob = heom.Problem.from_key(key("t_disorder.key"))
    prob.prepare_sample()
    h1 = prob.matrix(heom.MAT_H)
    prob.prepare_sample()
    h2 = prob.matrix(heom.MAT_H)
    assert not np.array_equal(h1, h2)
    prob.reset_rng()
    prob.prepare_sample()
    assert np.array_equal(prob.matrix(heom.MAT_H), h1)


def _write(tmp_path, text, name="k.key"):
    p = tmp_path / name
    p.write_text(text)
    return str(p)


def test_missing_file_is_io_error(heom):
    with pytest.raises(heom.HeomError) as e:
        heom.Problem.from_key("/nonexistent/dir/x.key")
    assert e.value.code == -2


@pytest.mark.parametrize("drop", ["PULSE", "POLARIZATION", "DISORDER", "DIPOLE", "BATH"])
def test_missing_section_is_parse_error(heom, tmp_path, drop):
    # The reference crashes or exits on these (polar.cpp:75-78, CPU_2DES.cpp:83,
    # dynamics.cpp:15); the library reports a parse error instead.
    text = open(key("c0_dimer_short.key")).read().replace(f"\n{drop}\n", "\nIGNORED_SECTION\n")
    with pytest.raises(heom.HeomError) as e:
        heom.Problem.from_key(_write(tmp_path, text))
    assert e.value.code == -3


def test_pulse_count_must_be_three(heom, tmp_path):
    text = open(key("c0_dimer_short.key")).read().replace("PULSE\n3\n", "PULSE\n2\n")
    with pytest.raises(heom.HeomError) as e:
        heom.Problem.from_key(_write(tmp_path, text))
    assert e.value.code == -3 and "3 pulses" in str(e.value)


def test_bath_before_hamiltonian_rejected(heom, tmp_path):
    text = open(key("c0_dimer_short.key")).read()
    ham = text.index("HAMILTONIAN")
    dis = text.index("DISORDER")
    bath = text.index("BATH")
    dip = text.index("DIPOLE")
    reordered = text[:ham] + text[bath:dip] + text[ham:bath] + text[dip:]
    with pytest.raises(heom.HeomError):
        heom.Problem.from_key(_write(tmp_path, reordered))
    assert dis > ham


def test_unknown_keywords_and_comments_ignored(heom, tmp_path):
    text = open(key("c0_dimer_short.key")).read()
    text = "# leading comment\nBATHTYPE\nartificial\n\n" + text
    prob = heom.Problem.from_key(_write(tmp_path, text))
    ref = heom.Problem.from_key(key("c0_dimer_short.key"))
    assert prob.info.n_ado == ref.info.n_ado
    assert np.array_equal(prob.matrix(heom.MAT_HKEY), ref.matrix(heom.MAT_HKEY))


def test_record_count_matches_schedule(heom):
    prob = heom.Problem.from_key(key("c0_dimer.key"))
    inf = prob.info
    # float time loop of dynamics.cpp:344-367
    t = np.float32(inf.t_start)
    nstep = np.float32((np.float32(inf.t_end) - np.float32(inf.t_start)) / np.float32(inf.step_size))
    c = 0
    i = 0
    while i <= nstep:
        if float(t) >= inf.tau[2] and i % inf.print_stride == 0:
            c += 1
        t = np.float32(t + np.float32(inf.step_size))
        i += 1
    assert inf.n_record == c == 1501 and inf.n_steps == 2001


# ------------------------------------------------------------------ ABI
def _declared_functions():
    hdr = open(os.path.join(ROOT, "include", "heom.h")).read()
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    return sorted(set(re.findall(r"\b(heom_[a-z0-9_]+)\s*\(", hdr)))


def test_library_exports_every_declared_symbol(heom):
    L = heom.lib()
    names = _declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, f"libheom.so lacks {missing}"
    assert L.heom_abi_version() == 1


@pytest.mark.skipif(cuda_available(), reason="checks the no-device error path")
def test_plan_without_device_fails_loudly(heom):
    prob = heom.Problem.from_key(key("c0_dimer_short.key"))
    with pytest.raises(heom.HeomError) as e:
        heom.Plan(prob)
    assert e.value.code == -4


def test_host_free_rejects_foreign_pointers(heom):
    """heom_host_free frees only buffers of heom_host_alloc: NULL is a no-op, any other
    pointer is HEOM_ERR_ARG (checked before any CUDA call)."""
    import ctypes
    L = heom.lib()
    assert L.heom_host_free(None) == 0
    foreign = np.zeros(4)
    assert L.heom_host_free(ctypes.c_void_p(foreign.ctypes.data)) == -1
    assert L.heom_host_alloc(16, None) == -1
