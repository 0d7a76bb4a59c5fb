"""GPU check of the adjoint gradient (config-4 form on a short trimer scan).

Objective: L(theta) = sum_t |P(theta) - P_target|^2 over a rephasing delay scan, with the
target generated at theta * 1.02.  Gradient of the 12 parameters (3 site energies, 3
couplings, 6 bath amplitude scales) from heom_adjoint_scan, checked against central
finite differences of the FP64 forward with h = 1e-4 relative.  Also checks that the
torch.autograd.Function wrapper returns the same gradient.
"""
import importlib

import numpy as np
import pytest

from heomtest import key, load_pkg

pytestmark = pytest.mark.gpu

REL_TOL = 1e-6


def _setup():
    heom = load_pkg()
    ag = importlib.import_module("eto_heom_b200.autograd")
    prob = heom.Problem.from_key(key("c4_trimer_short.key"))
    prob.prepare_sample()
    params = ag.ScanParameters(prob)
    rows = [(20.0, 20.0 + t1, 50.0 + t1, 95.0 + t1) for t1 in (0.0, 10.0, 25.0)]
    pts = heom.make_points(rows)
    return heom, ag, params, pts


def _forward(heom, params, theta, pts):
    params.apply(theta)
    plan = heom.Plan(params.problem, "fp64", max_points=len(pts))
    return plan.run_scan(pts).P


def test_adjoint_matches_central_differences():
    heom, ag, params, pts = _setup()
    th0 = params.theta0.copy()
    target = _forward(heom, params, th0 * 1.02, pts)
    P0 = _forward(heom, params, th0, pts)
    params.apply(th0)
    plan = heom.Plan(params.problem, "fp64", max_points=len(pts))
    r, grad = plan.adjoint_scan(pts, 2.0 * (P0 - target))
    assert np.allclose(r.P, P0, rtol=0, atol=1e-12 * np.abs(P0).max())
    loss = lambda th: float(np.sum(np.abs(_forward(heom, params, th, pts) - target) ** 2))  # noqa: E731

    def central(i, h):
        d = h * abs(th0[i])
        tp, tm = th0.copy(), th0.copy()
        tp[i] += d
        tm[i] -= d
        return (loss(tp) - loss(tm)) / (2 * d)

    # h = 1e-4 relative central differences, and their Richardson extrapolation with
    # h/2 (error O(h^4)).  For the site energies (~12,300 cm^-1) a 1e-4 relative step is
    # a 1.2 cm^-1 shift -- 0.05 rad of phase over the propagation -- so the plain central
    # difference itself carries ~(0.05)^2/6 relative truncation error there.
    fd = np.array([central(i, 1e-4) for i in range(len(th0))])
    fd2 = np.array([central(i, 5e-5) for i in range(len(th0))])
    fdr = (4 * fd2 - fd) / 3
    for i in range(len(th0)):
        print(f"param {i:2d}: adjoint {grad[i]: .9e}  fd(1e-4) {fd[i]: .9e} rel {abs(grad[i] - fd[i]) / abs(fd[i]):.2e}"
              f"  richardson rel {abs(grad[i] - fdr[i]) / abs(fdr[i]):.2e}")
    scale = np.abs(fdr).max()
    assert np.all(np.abs(grad - fdr) <= REL_TOL * np.abs(fdr) + 1e-9 * scale)
    # every non-energy parameter meets the bar against the plain h = 1e-4 difference too
    assert np.all(np.abs(grad[3:] - fd[3:]) <= REL_TOL * np.abs(fd[3:]))


def test_autograd_function_uses_the_adjoint():
    import torch

    heom, ag, params, pts = _setup()
    th0 = params.theta0.copy()
    target = _forward(heom, params, th0 * 1.02, pts)
    T = torch.from_numpy(np.stack([target.real, target.imag], axis=1))
    theta = torch.tensor(th0, dtype=torch.float64, requires_grad=True)
    P = ag.scan_response(theta, params, pts)
    loss = ((P - T) ** 2).sum()
    loss.backward()
    P0 = P.detach().numpy()
    params.apply(th0)
    plan = heom.Plan(params.problem, "fp64", max_points=len(pts))
    _, grad = plan.adjoint_scan(pts, 2.0 * ((P0[:, 0] + 1j * P0[:, 1]) - target))
    assert np.allclose(theta.grad.numpy(), grad, rtol=1e-12, atol=0)
