"""torch.autograd.Function over the C ABI: P(t1, t3) of a delay scan as a differentiable
function of the Hamiltonian and bath parameters.

    params = ScanParameters(problem)              # theta0 = current eps, J, bath scales
    P = scan_response(theta, params, points)      # (total, 2) real tensor: Re, Im of P
    loss = ((P - target) ** 2).sum(); loss.backward()   # theta.grad via the adjoint kernels

Forward runs the FP64 staged/scan path at theta; backward runs heom_adjoint_scan with the
incoming gradient dL/dP (complex convention dL/dRe + i dL/dIm), which re-propagates forward
with checkpoints and returns dL/dtheta.  theta lives on the CPU (12 scalars for the
config-4 trimer); the propagation itself always runs on the GPU.
"""
from __future__ import annotations

import numpy as np
import torch

from . import MAT_H, Plan, Problem


class ScanParameters:
    """Maps a parameter vector theta onto a problem: H = H0 + sum_i (theta_i - theta0_i) dH_i
    for site energies and couplings (exact: H is linear in them), bath scales set directly."""

    def __init__(self, problem: Problem):
        self.problem = problem
        inf = problem.info
        self.n = problem.param_count()
        self.n_bath = inf.K * inf.K_m
        self.n_h = self.n - self.n_bath
        self.H0 = problem.matrix(MAT_H)
        self.dH = [problem.param_dH(i) for i in range(self.n_h)]
        Hk = problem.matrix(5)  # the key's Hamiltonian (cm^-1 / hbar, lambda added)
        s = inf.single_size
        eps = [np.real(Hk[a, a]) for a in range(1, s)]
        J = [np.real(Hk[a, b]) for a in range(1, s) for b in range(a + 1, s)]
        hbar = 5308.0
        self.theta0 = np.array([e * hbar for e in eps] + [j * hbar for j in J] + [1.0] * self.n_bath)
        self.K, self.K_m = inf.K, inf.K_m

    def apply(self, theta: np.ndarray) -> None:
        d = np.asarray(theta, dtype=np.float64) - self.theta0
        H = self.H0.copy()
        for i in range(self.n_h):
            if d[i] != 0.0:
                H = H + d[i] * self.dH[i]
        self.problem.set_matrix(MAT_H, H)
        for j in range(self.K):
            for k in range(self.K_m):
                self.problem.set_bath_scale(j, k, float(theta[self.n_h + j * self.K_m + k]))


class _ScanResponse(torch.autograd.Function):
    @staticmethod
    def forward(ctx, theta: torch.Tensor, params: ScanParameters, points: np.ndarray):
        th = theta.detach().cpu().double().numpy()
        params.apply(th)
        plan = Plan(params.problem, "fp64", max_points=len(points))
        layout = plan.scan_layout(points)
        r = plan.run_scan(points, layout)
        ctx.params, ctx.points, ctx.theta = params, points, th
        out = torch.from_numpy(np.stack([r.P.real, r.P.imag], axis=1).copy())
        return out.to(theta.dtype)

    @staticmethod
    def backward(ctx, grad_out: torch.Tensor):
        g = grad_out.detach().cpu().double().numpy()
        dLdP = g[:, 0] + 1j * g[:, 1]
        ctx.params.apply(ctx.theta)
        plan = Plan(ctx.params.problem, "fp64", max_points=len(ctx.points))
        _, grad = plan.adjoint_scan(ctx.points, dLdP)
        return torch.from_numpy(grad), None, None


def scan_response(theta: torch.Tensor, params: ScanParameters, points: np.ndarray) -> torch.Tensor:
    """Differentiable P of a delay scan: (total, 2) tensor of (Re P, Im P)."""
    return _ScanResponse.apply(theta, params, points)
