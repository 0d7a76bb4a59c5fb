"""The torch spectrum pipeline (eto-heom_b200/spectrum.py) against scipy's functions,
which gen-2d-spectrum/gen_2d_spectrum.py:63-109 calls, on seeded synthetic scans of the
script's shapes (1000 rows x 61 delay columns), plus its gradient.

The script itself needs matplotlib, which is not installed, so its scipy calls are made
here directly on the same arrays: fft2 + fftshift (:64-66), gaussian_filter with
sigma (8, 0.8) (:70), RegularGridInterpolator on the doubled grid (:80-102) and the
fftfreq axes (:105-109).
"""
import importlib

import numpy as np
import pytest
import torch
from scipy.fft import fft2, fftfreq, fftshift
from scipy.interpolate import RegularGridInterpolator
from scipy.ndimage import gaussian_filter

from heomtest import load_pkg

TOL = 1e-12  # float64 throughout; only the summation order differs


@pytest.fixture(scope="module")
def sp():
    load_pkg()
    return importlib.import_module("eto_heom_b200.spectrum")


def _scan(rng, size1=1000, n=61, lines=801):
    """Synthetic columns: decaying oscillations with the scan's record length."""
    t = np.arange(lines) * 0.5
    cols = []
    for _ in range(n):
        w, g, a = rng.uniform(0.05, 0.5), rng.uniform(0.002, 0.02), rng.normal(size=2)
        cols.append(1e-4 * (a[0] + 1j * a[1]) * np.exp((1j * w - g) * t))
    return cols


def _rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / np.max(np.abs(np.asarray(b))))


def test_spectrum_matches_scipy(sp):
    rng = np.random.default_rng(7)
    R = np.zeros((1000, 61), np.complex128)
    NR = np.zeros((1000, 61), np.complex128)
    for i, c in enumerate(_scan(rng)):
        R[: len(c), i] = c
    for i, c in enumerate(_scan(rng)):
        NR[: len(c), i] = c
    ref = fftshift(fft2(NR)).real + fftshift(fft2(R)).real
    S = sp.spectrum(torch.from_numpy(R), torch.from_numpy(NR))
    assert _rel(S.numpy(), ref) < TOL
    ref_f = gaussian_filter(ref, sigma=(8, 0.8))
    Sf = sp.gaussian_filter(torch.from_numpy(ref), (8, 0.8))
    assert _rel(Sf.numpy(), ref_f) < TOL
    x, y = np.arange(ref_f.shape[0]), np.arange(ref_f.shape[1])
    nx, ny = np.linspace(0, x[-1], 2 * len(x)), np.linspace(0, y[-1], 2 * len(y))
    g = np.meshgrid(nx, ny, indexing="ij")
    ref_u = RegularGridInterpolator((x, y), ref_f)(np.array([g[0].ravel(), g[1].ravel()]).T).reshape(len(nx), len(ny))
    Su = sp.upsample_linear(torch.from_numpy(ref_f), 2)
    assert Su.shape == (2000, 122) and _rel(Su.numpy(), ref_u) < TOL
    S2, w_t, w_tau = sp.spectrum_2d(torch.from_numpy(R), torch.from_numpy(NR), 801, 61)
    assert _rel(S2.numpy(), ref_u) < TOL
    t = np.linspace(0, 1000 + (2000 - 801) * 10, 2000)
    tau = np.linspace(0, 600 + (122 - 61) * 10, 122)
    assert np.allclose(w_t, 5308 * 2 * np.pi * fftshift(fftfreq(len(t), t[1] - t[0])), rtol=0, atol=1e-9)
    assert np.allclose(w_tau, 5308 * 2 * np.pi * fftshift(fftfreq(len(tau), tau[1] - tau[0])), rtol=0, atol=1e-9)


@pytest.mark.parametrize("shape,sigma", [((40, 7), (8, 0.8)), ((5, 3), (4.0, 2.5)), ((64, 16), 1.3), ((9, 4), (0, 1))])
def test_gaussian_filter_boundaries(sp, shape, sigma):
    """Radii beyond the axis length reflect repeatedly, as scipy's 'reflect' mode does."""
    x = np.random.default_rng(3).normal(size=shape)
    assert _rel(sp.gaussian_filter(torch.from_numpy(x), sigma).numpy(), gaussian_filter(x, sigma)) < TOL


def test_load_scan_reads_cpu_2des_files(sp, tmp_path):
    """out_{tau}_{T}.out files in CPU_2DES's "%.6e %.6e" form, read into the script's
    column layout: signal * i, zero-padded to size1 rows, cut beyond it."""
    rng = np.random.default_rng(11)
    taus = np.arange(-30, 31, 10)
    data = {}
    for tau in taus:
        n = int(rng.integers(5, 14))
        z = rng.normal(size=n) + 1j * rng.normal(size=n)
        data[int(tau)] = z
        with open(tmp_path / f"out_{tau}_0.out", "w") as f:
            for v in z:
                f.write(f"{v.real:.6e} {v.imag:.6e}\n")
    R, NR, t_size, tau_size = sp.load_scan(str(tmp_path), 0, -30, 30, 10, size1=10)
    assert R.shape == (10, 4) and NR.shape == (10, 4)
    assert t_size == len(data[-30]) and tau_size == 4
    for i, tau in enumerate(range(0, 31, 10)):
        z = np.array([float(f"{v.real:.6e}") + 1j * float(f"{v.imag:.6e}") for v in data[tau]])[:10]
        col = np.zeros(10, np.complex128)
        col[: len(z)] = 1j * z
        assert np.array_equal(R[:, i].numpy(), col)
    for i, tau in enumerate(range(-30, 1, 10)):
        z = np.array([float(f"{v.real:.6e}") + 1j * float(f"{v.imag:.6e}") for v in data[tau]])[:10]
        col = np.zeros(10, np.complex128)
        col[: len(z)] = 1j * z
        assert np.array_equal(NR[:, i].numpy(), col)


def test_spectral_loss_gradient(sp):
    """The pipeline is differentiable in the P(t) values: gradcheck on a small scan."""
    rng = np.random.default_rng(5)
    counts, total = [6, 4, 7], 17
    offsets = [0, 6, 10]
    P = torch.tensor(rng.normal(size=(total, 2)), dtype=torch.float64, requires_grad=True)
    target = torch.tensor(rng.normal(size=(16, 6)), dtype=torch.float64)

    def f(P):
        cols = sp.signal_columns(P, offsets, counts)
        R = sp.assemble(cols, size1=8)
        NR = sp.assemble(cols[::-1], size1=8)
        S, _, _ = sp.spectrum_2d(R, NR, 6, 3, sigma=(1.5, 0.8), interp_factor=2, time=10.0, t_step=1.0,
                                 tau_end=6.0, tau_step=1.0)
        return sp.spectral_loss(S, target)

    assert torch.autograd.gradcheck(f, (P,), eps=1e-6, atol=1e-7, rtol=1e-6)
