"""The config-4 gradient at its stated size: trimer 2DES fit on a 32 x 128 grid.

Trimer (N = 1 + 3 + 3 = 7 levels, 210 ADOs), rephasing P(t1, t3) with t1 = 0..155 fs in
5 fs steps at t2 = 200 fs and 128 t3 samples every 2 fs (tests/golden/keys/
c4_trimer_fit.key, make_fixtures.c4_fit_rows).  The target comes from the six Hamiltonian
parameters (3 site energies, 3 couplings) perturbed by +2 %.  Objective
L = sum over the 4096 records of |P - P_target|^2; gradient with respect to the 12
parameters (plus the 6 bath amplitude scales) from the checkpointed adjoint
(heom_adjoint_scan, checkpoints every ceil(sqrt(steps)) steps).

Check: central finite differences of the FP64 forward with h = 1e-4 relative.  For the
site energies (~12,400 cm^-1) a 1e-4 relative step shifts the phase by ~0.15 rad over the
longest point, so the plain difference carries ~4e-3 relative truncation error; the
differences at h, h/2 and h/4 are Richardson-extrapolated to O(h^6) and the adjoint must
match that limit to 1e-6 relative.  Couplings and bath scales must also meet 1e-6
against the plain h = 1e-4 difference.  The forward it differentiates is the
reference's scheme (dynamics.cpp:298-432); the reference has no gradients.
"""
import math
import os
import sys
import time

import numpy as np
import pytest

from heomtest import key, load_pkg

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
from make_fixtures import c4_fit_rows  # noqa: E402

pytestmark = pytest.mark.gpu

REL_TOL = 1e-6


def test_c4_adjoint_full_grid():
    import importlib
    heom = load_pkg()
    ag = importlib.import_module("eto_heom_b200.autograd")
    prob = heom.Problem.from_key(key("c4_trimer_fit.key"))
    prob.prepare_sample()
    params = ag.ScanParameters(prob)
    rows = c4_fit_rows()
    pts = heom.make_points(rows)
    th0 = params.theta0.copy()
    assert len(th0) == 12 and params.n_h == 6

    def forward(th):
        params.apply(th)
        plan = heom.Plan(params.problem, "fp64", max_points=len(pts))
        r = plan.run_scan(pts)
        return r

    r0 = forward(th0)
    assert len(r0.P) == 32 * 128 and all(c == 128 for c in r0.counts)
    th_t = th0.copy()
    th_t[:6] *= 1.02
    target = forward(th_t).P
    P0 = r0.P
    params.apply(th0)
    plan = heom.Plan(params.problem, "fp64", max_points=len(pts))
    plan.adjoint_scan(pts, 2.0 * (P0 - target))   # warm
    t0 = time.perf_counter()
    r, grad = plan.adjoint_scan(pts, 2.0 * (P0 - target))
    t_adj = time.perf_counter() - t0
    assert np.allclose(r.P, P0, rtol=0, atol=1e-12 * np.abs(P0).max())

    def loss(th):
        return float(np.sum(np.abs(forward(th).P - target) ** 2))

    def central(i, h):
        d = h * abs(th0[i])
        tp, tm = th0.copy(), th0.copy()
        tp[i] += d
        tm[i] -= d
        return (loss(tp) - loss(tm)) / (2 * d)

    t0 = time.perf_counter()
    fd1 = np.array([central(i, 1e-4) for i in range(12)])
    t_fd = time.perf_counter() - t0
    fd2 = np.array([central(i, 5e-5) for i in range(12)])
    fd4 = np.array([central(i, 2.5e-5) for i in range(12)])
    r1 = (4 * fd2 - fd1) / 3          # O(h^4)
    r2 = (4 * fd4 - fd2) / 3
    rich = (16 * r2 - r1) / 15        # O(h^6)
    steps = max(int(np.float32(rw[3]) / np.float32(0.5)) + 1 for rw in rows)
    print(f"\nc4 grid: 32 x 128 records, {steps} RK4 steps at most, checkpoints every "
          f"{math.ceil(math.sqrt(steps))} steps; adjoint {t_adj * 1e3:.1f} ms per gradient, "
          f"one FD gradient (24 forwards) {t_fd:.2f} s")
    for i in range(12):
        print(f"param {i:2d}: adjoint {grad[i]: .10e}  fd(1e-4) {fd1[i]: .10e} rel {abs(grad[i] - fd1[i]) / abs(fd1[i]):.2e}"
              f"  extrapolated rel {abs(grad[i] - rich[i]) / abs(rich[i]):.2e}")
    scale = np.abs(rich).max()
    assert np.all(np.abs(grad - rich) <= REL_TOL * np.abs(rich) + 1e-10 * scale)
    assert np.all(np.abs(grad[3:] - fd1[3:]) <= REL_TOL * np.abs(fd1[3:]) + 1e-10 * scale)
