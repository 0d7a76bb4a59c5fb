"""Population dynamics on the GPU: the dynamics_solver / CPU_dynamics replacement.

The bit-exact FP64 path runs the reference's RK4 and right-hand side
(total_ADO_dynamics, dynamics.cpp:52-115, which is total_ADO_dynamics_Ht with the static
H and S_j on level j); populations must equal the reference build's full-precision
values bit for bit (tests/golden/ref/d_*.npz, from oracle/_ref/ref_dynamics), and the
heom_dynamics executable's stdout must equal CPU_dynamics' byte for byte.  d_dimer runs
in shared memory, d_trimer (1330 ADOs) on the staged global-memory form.
"""
import os
import subprocess

import numpy as np
import pytest

from heomtest import KEYS, PKG_DIR, REF, key, load_pkg

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["d_dimer.key", "d_trimer.key"])
def test_populations_bit_exact(name):
    heom = load_pkg()
    prob = heom.Problem.from_key(key(name), dynamics=True)
    plan = heom.Plan(prob, "fp64-exact")
    pops = plan.run_populations((1, 2))
    ref = np.load(os.path.join(REF, name.replace(".key", ".npz")))["population"]
    n = pops.shape[1]
    assert n <= ref.shape[1] and not ref[:, n:].any()
    assert np.array_equal(pops, ref[:, :n]), np.max(np.abs(pops - ref[:, :n]))
    # trace of the reduced density matrix stays 1 to rounding when every level is listed
    if prob.info.sys_size == 2:
        assert np.allclose(pops.sum(axis=0), 1.0, atol=1e-12)


@pytest.mark.parametrize("name", ["d_dimer.key", "d_trimer.key"])
def test_heom_dynamics_cli_byte_identical(name):
    out = subprocess.run([os.path.join(PKG_DIR, "heom_dynamics"), name], cwd=KEYS, capture_output=True)
    assert out.returncode == 0, out.stderr.decode()
    assert out.stdout == open(os.path.join(REF, name.replace(".key", ".out")), "rb").read()


def test_dynamics_plan_rejects_batched_paths():
    heom = load_pkg()
    prob = heom.Problem.from_key(key("d_dimer.key"), dynamics=True)
    with pytest.raises(heom.HeomError):
        heom.Plan(prob, "fp32-bulk")
    plan = heom.Plan(prob, "fp64-exact")
    with pytest.raises(heom.HeomError):
        plan.run_populations((0,))  # sites are 1-based (dynamics.cpp:211-215)
