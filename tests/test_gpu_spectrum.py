"""GPU check of the differentiable spectral loss (the trimer fit's objective).

theta (3 site energies, 3 couplings, 6 bath amplitude scales) -> P(t) of a short
rephasing + non-rephasing delay scan on the FP64 path (autograd.scan_response) -> the
2D spectrum of gen-2d-spectrum/gen_2d_spectrum.py:63-102 (spectrum.spectrum_2d) -> L2
loss against the spectrum at theta * 1.02.  theta.grad comes from torch's backward
through the spectrum and heom_adjoint_scan; it is checked against Richardson-extrapolated
central differences of the same loss evaluated with plain forward scans.
"""
import importlib

import numpy as np
import pytest
import torch

from heomtest import key, load_pkg

pytestmark = pytest.mark.gpu

REL_TOL = 1e-6
T1 = (0.0, 10.0, 20.0)


def _setup():
    heom = load_pkg()
    ag = importlib.import_module("eto_heom_b200.autograd")
    sp = importlib.import_module("eto_heom_b200.spectrum")
    prob = heom.Problem.from_key(key("c4_trimer_short.key"))
    prob.prepare_sample()
    params = ag.ScanParameters(prob)
    # the script's delay layout: rephasing tau = t1 (pulse 1 first), non-rephasing
    # tau = -t1 (pulse 2 first); tau3 = t0 + t1 + T, t_end = tau3 + 45 fs
    rows = [(20.0, 20.0 + t, 50.0 + t, 95.0 + t) for t in T1]
    rows += [(20.0 + t, 20.0, 50.0 + t, 95.0 + t) for t in T1[1:]]
    return heom, ag, sp, params, heom.make_points(rows)


def _spectrum(sp, cols):
    """cols: signals of R(0), R(10), R(20), NR(-10), NR(-20)."""
    R = sp.assemble(cols[:3], size1=96)
    NR = sp.assemble([cols[4], cols[3], cols[0]], size1=96)
    S, _, _ = sp.spectrum_2d(R, NR, len(cols[4]), 3, sigma=(8, 0.8), interp_factor=2,
                             time=45.0, t_step=0.5, tau_end=20.0, tau_step=10.0)
    return S


def _loss_plain(heom, sp, params, theta, pts, target):
    params.apply(theta)
    r = heom.Plan(params.problem, "fp64", max_points=len(pts)).run_scan(pts)
    cols = [torch.from_numpy(1j * r.point(i)) for i in range(len(pts))]
    return float(sp.spectral_loss(_spectrum(sp, cols), target))


def test_spectral_loss_gradient_matches_central_differences():
    heom, ag, sp, params, pts = _setup()
    th0 = params.theta0.copy()
    layout = heom.Plan(params.problem, "fp64", max_points=len(pts)).scan_layout(pts)
    _, off, cnt, _ = layout
    with torch.no_grad():
        Pt = ag.scan_response(torch.tensor(th0 * 1.02, dtype=torch.float64), params, pts)
        target = _spectrum(sp, sp.signal_columns(Pt, off, cnt))
    theta = torch.tensor(th0, dtype=torch.float64, requires_grad=True)
    P = ag.scan_response(theta, params, pts)
    loss = sp.spectral_loss(_spectrum(sp, sp.signal_columns(P, off, cnt)), target)
    loss.backward()
    grad = theta.grad.numpy()
    lv = float(loss.detach())
    assert abs(lv - _loss_plain(heom, sp, params, th0, pts, target)) <= 1e-12 * lv

    def central(i, h):
        d = h * abs(th0[i])
        tp, tm = th0.copy(), th0.copy()
        tp[i] += d
        tm[i] -= d
        return (_loss_plain(heom, sp, params, tp, pts, target) - _loss_plain(heom, sp, params, tm, pts, target)) / (2 * d)

    fd = np.array([central(i, 1e-4) for i in range(len(th0))])
    fd2 = np.array([central(i, 5e-5) for i in range(len(th0))])
    fdr = (4 * fd2 - fd) / 3
    for i in range(len(th0)):
        print(f"param {i:2d}: backward {grad[i]: .9e}  richardson {fdr[i]: .9e}  "
              f"rel {abs(grad[i] - fdr[i]) / abs(fdr[i]):.2e}")
    scale = np.abs(fdr).max()
    assert np.all(np.abs(grad - fdr) <= REL_TOL * np.abs(fdr) + 1e-9 * scale)
