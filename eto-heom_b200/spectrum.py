"""2D spectrum from a delay scan's P(t), in torch and differentiable.

Restates the numerical part of gen-2d-spectrum/gen_2d_spectrum.py (lines 8-109):

    reph, nonreph, t_size, tau_size = load_scan("2d-output", T=0)    # :21-61
    S = spectrum(reph, nonreph)                                        # :63-66
    S = gaussian_filter(S, (8, 0.8))                                   # :70
    S = upsample_linear(S, 2)                                          # :80-102
    w_t, w_tau = frequency_axes(S.shape, t_size, tau_size)             # :105-109

or all of it as spectrum_2d(...).  The plotting tail of that script (the cubic griddata
resampling for the contour map, :111-141) produces a picture, not a number, and is not
restated; normalise() is its line 126.

Every step is a torch operation (complex FFT, a separable convolution with scipy's
'reflect' boundary, linear interpolation), so a loss on the spectrum back-propagates to
the P(t) columns and, through eto_heom_b200.autograd.scan_response, to the Hamiltonian
and bath parameters: the L2 spectral loss of the trimer fit.

Column layout (gen_2d_spectrum.py:26-61): column i of the non-rephasing block holds the
point with tau = tau_start + i*tau_step (tau_start..0, both ends included), column i of
the rephasing block tau = i*tau_step (0..tau_end); row j is P at the j-th recorded step
times i, zero-padded (or cut) to `size1` rows.
"""
from __future__ import annotations

import os
from typing import Sequence

import numpy as np
import torch

HBAR = 5308.0  # cm^-1 fs, the script's conversion factor (gen_2d_spectrum.py:108)


def read_out(path: str) -> np.ndarray:
    """One CPU_2DES output file ("re im" per line) as i*(re + i im)
    (gen_2d_spectrum.py:31-35)."""
    a = np.loadtxt(path, dtype=np.float64, ndmin=2)
    if a.size == 0:
        return np.zeros(0, dtype=np.complex128)
    return 1j * (a[:, 0] + 1j * a[:, 1])


def taus(start: float, end: float, step: float) -> np.ndarray:
    """np.arange(start, end + 1, step): the script's delay columns, end included."""
    return np.arange(start, end + 1, step)


def assemble(columns: Sequence, size1: int = 1000) -> torch.Tensor:
    """Stack per-delay signals (1-D complex, already multiplied by i) as the columns of a
    (size1, n) complex128 tensor, zero-padded or cut to size1 rows
    (gen_2d_spectrum.py:36-38).  Tensors keep their autograd graph."""
    cols = []
    for c in columns:
        c = torch.as_tensor(c)
        if not c.is_complex():
            raise ValueError("assemble: columns must be complex")
        c = c.to(torch.complex128)[:size1]
        if c.shape[0] < size1:
            c = torch.cat([c, c.new_zeros(size1 - c.shape[0])])
        cols.append(c)
    return torch.stack(cols, dim=1)


def load_scan(out_dir: str, T=0, tau_start: int = -600, tau_end: int = 600, tau_step: int = 10,
              size1: int = 1000):
    """Read out_{tau}_{T}.out of a delay scan (gen_2d_spectrum.py:21-61).

    Returns (rephasing, nonrephasing, t_size, tau_size): two (size1, n) complex128 tensors,
    the line count of the first non-rephasing file and the number of non-rephasing
    columns (the script's t_size and tau_size, used by frequency_axes)."""
    def block(a, b):
        return [read_out(os.path.join(out_dir, f"out_{tau}_{T}.out")) for tau in taus(a, b, tau_step)]

    nr = block(tau_start, 0)
    re = block(0, tau_end)
    return assemble(re, size1), assemble(nr, size1), len(nr[0]), len(nr)


def spectrum(rephasing: torch.Tensor, nonrephasing: torch.Tensor) -> torch.Tensor:
    """Re fftshift(fft2(R)) + Re fftshift(fft2(NR)) (gen_2d_spectrum.py:64-66)."""
    def one(x):
        return torch.fft.fftshift(torch.fft.fft2(x), dim=(-2, -1)).real

    return one(rephasing) + one(nonrephasing)


def _gauss_weights(sigma: float, truncate: float, dtype, device) -> torch.Tensor:
    r = int(truncate * float(sigma) + 0.5)
    x = torch.arange(-r, r + 1, dtype=dtype, device=device)
    w = torch.exp(-0.5 * (x / float(sigma)) ** 2)
    return w / w.sum()


def _reflect_index(n: int, r: int, device) -> torch.Tensor:
    """Indices of an axis of length n extended by r on both sides with the half-sample
    symmetric boundary (d c b a | a b c d | d c b a), repeated as often as r needs."""
    i = torch.arange(-r, n + r, device=device) % (2 * n)
    return torch.where(i >= n, 2 * n - 1 - i, i)


def _filter_axis(x: torch.Tensor, w: torch.Tensor, dim: int) -> torch.Tensor:
    r = (w.numel() - 1) // 2
    if r == 0:
        return x * w[0]
    n = x.shape[dim]
    xe = x.index_select(dim, _reflect_index(n, r, x.device))
    win = xe.unfold(dim, 2 * r + 1, 1)  # window along a new last axis
    return (win * w).sum(-1)


def gaussian_filter(x: torch.Tensor, sigma=(8.0, 0.8), truncate: float = 4.0) -> torch.Tensor:
    """scipy.ndimage.gaussian_filter(x, sigma) with its defaults (mode 'reflect',
    truncate 4) for a real 2-D tensor: a normalised Gaussian of radius
    int(truncate*sigma + 0.5) per axis, applied axis by axis (gen_2d_spectrum.py:70)."""
    if x.dim() != 2:
        raise ValueError("gaussian_filter: 2-D input expected")
    s = (sigma, sigma) if np.isscalar(sigma) else tuple(sigma)
    for d in range(2):
        if s[d] > 0:
            x = _filter_axis(x, _gauss_weights(s[d], truncate, x.dtype, x.device), d)
    return x


def _linear_axis(x: torch.Tensor, factor: int, dim: int) -> torch.Tensor:
    n = x.shape[dim]
    m = n * factor
    pos = torch.linspace(0, n - 1, m, dtype=torch.float64, device=x.device)
    lo = torch.clamp(torch.floor(pos).long(), 0, max(n - 2, 0))
    hi = torch.clamp(lo + 1, max=n - 1)
    f = (pos - lo.to(torch.float64)).to(x.dtype)
    shape = [1] * x.dim()
    shape[dim] = m
    f = f.view(shape)
    return x.index_select(dim, lo) * (1 - f) + x.index_select(dim, hi) * f


def upsample_linear(x: torch.Tensor, factor: int = 2) -> torch.Tensor:
    """Bilinear resampling of a 2-D grid onto linspace(0, n-1, n*factor) per axis, as
    RegularGridInterpolator((arange(n0), arange(n1)), x) evaluated on that grid does
    (gen_2d_spectrum.py:80-102)."""
    for d in range(2):
        x = _linear_axis(x, factor, d)
    return x


def frequency_axes(shape, t_size: int, tau_size: int, time: float = 1000.0, t_step: float = 10.0,
                   tau_end: float = 600.0, tau_step: float = 10.0):
    """The script's axes in cm^-1 (gen_2d_spectrum.py:105-109): w_t for the rows, w_tau
    for the columns of the resampled spectrum."""
    n1, n2 = shape
    t = np.linspace(0, time + (n1 - t_size) * t_step, n1)
    tau = np.linspace(0, tau_end + (n2 - tau_size) * tau_step, n2)
    w_t = HBAR * 2 * np.pi * np.fft.fftshift(np.fft.fftfreq(len(t), t[1] - t[0]))
    w_tau = HBAR * 2 * np.pi * np.fft.fftshift(np.fft.fftfreq(len(tau), tau[1] - tau[0]))
    return w_t, w_tau


def normalise(x: torch.Tensor) -> torch.Tensor:
    """x / max|x| (gen_2d_spectrum.py:126)."""
    return x / x.abs().max()


def spectrum_2d(rephasing: torch.Tensor, nonrephasing: torch.Tensor, t_size: int, tau_size: int,
                sigma=(8.0, 0.8), interp_factor: int = 2, **axes):
    """The whole numerical pipeline: (S, w_t, w_tau) with S the filtered, resampled
    spectrum (gen_2d_spectrum.py:63-109).  `axes` passes time, t_step, tau_end and
    tau_step to frequency_axes."""
    S = upsample_linear(gaussian_filter(spectrum(rephasing, nonrephasing), sigma), interp_factor)
    w_t, w_tau = frequency_axes(tuple(S.shape), t_size, tau_size, **axes)
    return S, w_t, w_tau


def spectral_loss(S: torch.Tensor, target: torch.Tensor) -> torch.Tensor:
    """Sum of squared differences of two spectra on the same grid."""
    return ((S - target) ** 2).sum()


def signal_columns(P: torch.Tensor, offsets: Sequence[int], counts: Sequence[int]):
    """Split the (total, 2) output of autograd.scan_response into per-point signals
    i*P (the script's d * 1j), keeping the autograd graph."""
    z = torch.complex(P[:, 0].to(torch.float64), P[:, 1].to(torch.float64)) * 1j
    return [z[o:o + c] for o, c in zip(offsets, counts)]


__all__ = ["HBAR", "read_out", "taus", "assemble", "load_scan", "spectrum", "gaussian_filter",
           "upsample_linear", "frequency_axes", "normalise", "spectrum_2d", "spectral_loss",
           "signal_columns"]

