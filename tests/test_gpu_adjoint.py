"""GPU check of the adjoint gradient (config-4 form on a short trimer scan).

Objective: L(theta) = sum_t |P(theta) - P_target|^2 over a rephasing delay scan, with the
target generated at theta * 1.02.  Gradient of the 12 parameters (3 site energies, 3
couplings, 6 bath amplitude scales) from heom_adjoint_scan, checked against central
finite differences of the FP64 forward with h = 1e-4 relative.  Also checks that the
torch.autograd.Function wrapper returns the same gradient.
"""
import importlib
import os
import subprocess

import numpy as np
import pytest

from heomtest import ROOT, key, load_pkg

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


REF_DRIVER = os.path.join(ROOT, "oracle", "_ref", "ref_driver")


def _key_text(base: str, row, eps_d=None, j_d=None, bath_d=None) -> str:
    """The trimer key with the point's pulse times and end, and optional perturbations of
    a HAMILTONIAN diagonal entry (eps_d = (a, h)), a coupling pair (j_d = (a, b, h)) or
    the amplitude of one BATH line (bath_d = (k, factor): alpha and, through it,
    conj(alpha) scale together, as heom_problem_set_bath_scale does for every site)."""
    lines = base.split("\n")
    h0 = lines.index("HAMILTONIAN") + 1
    H = [[float(x) for x in lines[h0 + r].split()] for r in range(4)]
    if eps_d:
        H[eps_d[0]][eps_d[0]] += eps_d[1]
    if j_d:
        H[j_d[0]][j_d[1]] += j_d[2]
        H[j_d[1]][j_d[0]] += j_d[2]
    for r in range(4):
        lines[h0 + r] = " ".join(repr(v) for v in H[r])
    if bath_d:
        b0 = lines.index("BATH") + 3 + bath_d[0]
        v = [float(x) for x in lines[b0].split()]
        v[0] *= bath_d[1]
        v[1] *= bath_d[1]
        lines[b0] = " ".join(repr(x) for x in v)
    p0 = lines.index("PULSE") + 2
    for q in range(3):
        f = lines[p0 + q].split()
        f[1] = repr(row[q])
        lines[p0 + q] = " ".join(f)
    t0 = lines.index("TIME") + 1
    f = lines[t0].split()
    f[1] = repr(row[3])
    lines[t0] = " ".join(f)
    return "\n".join(lines)


def _ref_combined(path: str) -> np.ndarray:
    out = subprocess.run([REF_DRIVER, path], capture_output=True, text=True, check=True).stdout.split("\n")
    i = next(k for k, l in enumerate(out) if l.startswith("#combined"))
    n = int(out[i].split()[1])
    v = np.array([[float(x) for x in out[i + 1 + j].split()] for j in range(n)])
    return v[:, 0] + 1j * v[:, 1]


@pytest.mark.skipif(not os.path.exists(REF_DRIVER), reason="the reference build (oracle/_ref) is not built")
def test_adjoint_matches_reference_build_differences(tmp_path):
    """Finite differences of the reference CPU build itself (oracle/_ref/ref_driver: the
    reference's unmodified library, full-precision output) through its own inputs: the
    key file's HAMILTONIAN entries (3 site energies, 3 couplings, step 0.05 cm^-1) and
    BATH line amplitudes (each line scaled for all sites at once, step 2.5e-4), against
    the adjoint gradient (the bath-line derivative is the sum over sites).  The
    reference's combined P = p111 - p110 - p101 cancels ~7 orders of magnitude, so its
    rounding noise is ~1e-9..1e-8 of P; over a 0.05 cm^-1 step that limits the
    differences to ~1e-4 relative -- the tolerance is 2e-3."""
    from concurrent.futures import ThreadPoolExecutor

    heom, ag, params, pts = _setup()
    th0 = params.theta0.copy()
    rows = [(20.0, 20.0 + t1, 50.0 + t1, 95.0 + t1) for t1 in (0.0, 25.0)]
    pts = heom.make_points(rows)
    target = _forward(heom, params, th0 * 1.02, pts)
    P0 = _forward(heom, params, th0, pts)
    params.apply(th0)
    plan = heom.Plan(params.problem, "fp64", max_points=len(pts))
    layout = plan.scan_layout(pts)
    _, off, cnt, _ = layout
    _, grad = plan.adjoint_scan(pts, 2.0 * (P0 - target))
    base = open(key("c4_trimer_short.key")).read()
    K, Km = params.K, params.K_m
    cases = [("eps", (a, 1)) for a in (1, 2, 3)] + [("J", ab) for ab in ((1, 2), (1, 3), (2, 3))]
    cases += [("bath", (k,)) for k in range(Km)]

    def loss_of(tag, kw):
        jobs = []
        for i, r in enumerate(rows):
            p = tmp_path / f"{tag}_{i}.key"
            p.write_text(_key_text(base, r, **kw))
            jobs.append(str(p))
        with ThreadPoolExecutor(max_workers=len(jobs)) as ex:
            Ps = list(ex.map(_ref_combined, jobs))
        return sum(float(np.sum(np.abs(Ps[i] - target[off[i]:off[i] + cnt[i]]) ** 2)) for i in range(len(rows)))

    specs = []
    for name, arg in cases:
        if name == "eps":
            h = 0.05
            specs.append((f"eps{arg[0]}", h, {"eps_d": (arg[0], h)}, {"eps_d": (arg[0], -h)}))
        elif name == "J":
            h = 0.05
            specs.append((f"J{arg[0]}{arg[1]}", h, {"j_d": (arg[0], arg[1], h)}, {"j_d": (arg[0], arg[1], -h)}))
        else:
            h = 2.5e-4
            specs.append((f"bath{arg[0]}", h, {"bath_d": (arg[0], 1 + h)}, {"bath_d": (arg[0], 1 - h)}))
    with ThreadPoolExecutor(max_workers=4) as ex:
        plus = list(ex.map(lambda s: loss_of(s[0] + "p", s[2]), specs))
        minus = list(ex.map(lambda s: loss_of(s[0] + "m", s[3]), specs))
    fd = np.array([(lp - lm) / (2 * s[1]) for s, lp, lm in zip(specs, plus, minus)])
    n_h = params.n_h
    adj = np.concatenate([grad[:n_h], [sum(grad[n_h + j * Km + k] for j in range(K)) for k in range(Km)]])
    scale = np.abs(fd).max()
    for s, g, f in zip(specs, adj, fd):
        print(f"{s[0]:6s}: adjoint {g: .9e}  reference-build fd {f: .9e}  rel {abs(g - f) / abs(f):.2e}")
    assert np.all(np.abs(adj - fd) <= 2e-3 * np.abs(fd) + 1e-5 * scale)
