"""Population-dynamics keys on the host (no GPU): the param_dynamics restatement.

param::param_dynamics (etoheom-cpu/lib/param.cpp:250-348) reads SIZE levels that are all
sites (no ground state, no two-exciton block), divides H by hbar and adds the bath's
reorganisation energy to the first K diagonal elements.  construct_ADO_set is the same
as for 2DES keys.
"""
import numpy as np
import pytest

from heomtest import key, load_pkg

HBAR = 5308.0  # etoheom-cpu/lib/constant.cpp


@pytest.mark.parametrize("name,size,K,L,n_ado", [("d_dimer.key", 2, 2, 3, 35), ("d_trimer.key", 3, 3, 3, 1330)])
def test_dynamics_key_parse(name, size, K, L, n_ado):
    heom = load_pkg()
    prob = heom.Problem.from_key(key(name), dynamics=True)
    inf = prob.info
    assert (inf.single_size, inf.sys_size, inf.K, inf.L, inf.n_ado) == (size, size, K, L, n_ado)
    text = open(key(name)).read().split("\n")
    h0 = text.index("HAMILTONIAN")
    Hkey = np.array([[float(x) for x in text[h0 + 1 + i].split()] for i in range(size)])
    lam = float(text[text.index("BATH") + 1])
    want = Hkey / HBAR + np.diag([lam] * K + [0.0] * (size - K))
    H = prob.matrix(heom.MAT_H)
    assert np.array_equal(H.real, want) and not H.imag.any()
    prob.prepare_sample()  # draws nothing: CPU_dynamics has no disorder or orientation
    assert np.array_equal(prob.matrix(heom.MAT_H), H)
    # records: every print_step from t_start, (t_end - t_start) / print_step + 1 of them
    assert inf.n_record == int(round((inf.t_end - inf.t_start) / inf.print_step)) + 1


def test_dynamics_flag_matters():
    heom = load_pkg()
    with pytest.raises(heom.HeomError):  # a population key lacks the 2DES blocks
        heom.Problem.from_key(key("d_dimer.key"))
