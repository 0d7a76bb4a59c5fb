"""Precision study for a tensor-core commutator on the large systems (N = 7, 13, 29).

The general-size FP32-bulk path contracts the commutator [A, w] of every ADO block in
FP32 on the CUDA cores.  On tcgen05 tensor cores the 32-bit operand kind is TF32 (10-bit
mantissa), so a tensor-core commutator would either round both factors to TF32
(1xTF32) or split each factor into two TF32 parts and accumulate three products
(3xTF32, dropping lo x lo).  HEOM_SG_CONTRACTION=tf32 | tf32x3 makes the FP32-bulk stage
kernel round its commutator products exactly that way (cvt.rna.tf32.f32 on each factor,
exact products, FP32 accumulation), which measures what either form would do to P(t)
against the 1e-6 gate before any tensor-core kernel is written.  The reference for each
case is the FP64 staged path (mixed-difference basis), within ~1e-13 of the truth where
the truth is available.  The bath couplings and the FP64 state are unchanged.
"""
import os

import numpy as np
import pytest

from heomtest import key, load_pkg, rel_err

pytestmark = pytest.mark.gpu

CASES = [
    ("c1_fmo_300fs.key", False, None),       # FMO aggregate, N = 29, 680 ADOs, 2DES point
    ("c4_trimer_short.key", False, None),    # trimer, N = 7, 210 ADOs, 2DES point
    ("c3_chain.key", True, (0, 0, 1)),       # chain, N = 13, 2925 ADOs, linear response
]


def _run(heom, name, single, mask, precision, contraction=None):
    # the variable is read when the plan sets up its general-size state, on its first run
    if contraction:
        os.environ["HEOM_SG_CONTRACTION"] = contraction
    try:
        prob = heom.Problem.from_key(key(name), single_manifold=single)
        prob.prepare_sample()
        plan = heom.Plan(prob, precision)
        if mask:
            return plan.run_traj(*mask)
        P, _ = plan.run_2des(trajectories=False)
        return P
    finally:
        os.environ.pop("HEOM_SG_CONTRACTION", None)


@pytest.mark.parametrize("name,single,mask", CASES, ids=[c[0].split(".")[0] for c in CASES])
def test_tf32_contraction_error(name, single, mask):
    heom = load_pkg()
    ref = _run(heom, name, single, mask, "fp64")
    errs = {c: rel_err(_run(heom, name, single, mask, "fp32-bulk", c), ref) for c in ("fp32", "tf32x3", "tf32")}
    print(f"\n{name}: FP32-bulk contraction error vs FP64 -- FP32 {errs['fp32']:.2e}, "
          f"3xTF32 {errs['tf32x3']:.2e}, 1xTF32 {errs['tf32']:.2e} (gate 1e-6)")
    assert errs["fp32"] <= 1e-6
    assert all(np.isfinite(v) for v in errs.values())
    # the emulation is live: TF32 rounding must move the result
    assert errs["tf32"] > errs["fp32"]
