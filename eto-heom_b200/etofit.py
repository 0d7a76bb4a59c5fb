"""Effective-thermal-oscillator (ETO) bath fitting: the BATH block of a key file.

Restates the fitting procedure of the reference's ``etom/ohmic_ETOM.py:17-106,172-191``,
``etom/superohmic_ETOM.py`` and ``etom/debye_lorentz_ETOM.py`` without plotting or
rewriting a template in place:

* the bath correlation function C(t) = (1/pi) Int_0^inf J(w) [cos(wt) coth(beta hbar w/2)
  - i sin(wt)] dw is sampled on ``t = linspace(0, t_max, n_t)`` fs;
* Re C(t) is fitted to ``sum_j a_j cos(w_j t) exp(-g_j t)`` (``curve_fit``, every initial
  parameter equal to ``init_guess``);
* Im C(t) is fitted to ``sum_j b_j cos(w_j t) exp(-g_j t)`` with the (g_j, w_j) of the
  real fit held fixed;
* each oscillator becomes two BATH lines ``a/2 b/2 g w`` and ``a/2 b/2 g -w`` (amplitudes
  times the coupling strength), preceded by the reorganisation line and the line count.

Units: frequencies and rates in fs^-1, ``hbar = 5308`` cm^-1 fs, ``kT`` in cm^-1 (the
reference multiplies ``beta * w * hbar``).  The fitted numbers depend on the scipy
version, which is why the test fixtures freeze them into key files.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

HBAR = 5308.0          # cm^-1 fs   (reference constant.cpp:9, ohmic_ETOM.py:7)
BOLTZ_K = 0.695        # cm^-1 / K  (reference constant.cpp:8)


@dataclass
class BathFit:
    """One fitted bath: the reorganisation line and the per-line (a/2, b/2, g, w)."""

    reorganisation: float
    lines: list  # list of (alpha_re, alpha_im, gamma_re, gamma_im)

    def key_block(self) -> str:
        """The text that follows the ``BATH`` keyword in a key file."""
        out = [repr(float(self.reorganisation)), str(len(self.lines))]
        out += [f"{a:.8f} {b:.8f} {g:.8f} {w:.8f}" for a, b, g, w in self.lines]
        return "\n".join(out) + "\n"


def _correlation(J, beta_hbar, t_values):
    from scipy.integrate import quad

    def re(t):
        v, _ = quad(lambda w: J(w) * np.cos(w * t) / np.tanh(0.5 * beta_hbar * w), 0, np.inf,
                    epsabs=1e-10, epsrel=1e-10, limit=10_000_000)
        return v / np.pi

    def im(t):
        v, _ = quad(lambda w: -J(w) * np.sin(w * t), 0, np.inf,
                    epsabs=1e-10, epsrel=1e-10, limit=10_000_000)
        return v / np.pi

    return (np.array([re(t) for t in t_values]), np.array([im(t) for t in t_values]))


def _fit(t_values, y_re, y_im, n_osc, init_guess, bounded_imag=False):
    from scipy.optimize import curve_fit

    def f_re(t, *p):
        r = 0.0
        for j in range(n_osc):
            r = r + p[3 * j] * np.cos(p[3 * j + 2] * t) * np.exp(-p[3 * j + 1] * t)
        return r

    p_re, _ = curve_fit(f_re, t_values, y_re, p0=[init_guess] * (3 * n_osc), maxfev=1_000_000_000)
    g = p_re[1::3]
    w = p_re[2::3]

    def f_im(t, *b):
        r = 0.0
        for j in range(n_osc):
            r = r + b[j] * np.cos(w[j] * t) * np.exp(-g[j] * t)
        return r

    kw = {"bounds": (-np.inf, np.inf)} if bounded_imag else {}
    p_im, _ = curve_fit(f_im, t_values, y_im, p0=[init_guess] * n_osc, maxfev=1_000_000_000, **kw)
    return p_re, p_im


def _lines(p_re, p_im, n_osc, scale):
    out = []
    for j in range(n_osc):
        a, g, w = p_re[3 * j], p_re[3 * j + 1], p_re[3 * j + 2]
        b = p_im[j]
        out.append((scale * a / 2, scale * b / 2, g, w))
        out.append((scale * a / 2, scale * b / 2, g, -w))
    return out


def ohmic(reorg_cm: float, wc_cm: float, temperature_k: float, n_osc: int = 1,
          t_max: float = 1000.0, n_t: int = 1000, init_guess: float = 0.1) -> BathFit:
    """Ohmic J(w) = eta w exp(-w/wc); eta fixed by lambda = eta wc / pi (ohmic_ETOM.py:176)."""
    wc = wc_cm / HBAR
    eta = (reorg_cm / HBAR) * math.pi / wc
    kt = temperature_k * BOLTZ_K
    t = np.linspace(0, t_max, n_t)
    y_re, y_im = _correlation(lambda w: w * np.exp(-w / wc), HBAR / kt, t)
    p_re, p_im = _fit(t, y_re, y_im, n_osc, init_guess)
    return BathFit(eta * wc / math.pi, _lines(p_re, p_im, n_osc, eta))


def superohmic(reorg_cm: float, wc_cm: float, temperature_k: float, n_osc: int = 1,
               t_max: float = 500.0, n_t: int = 1000, init_guess: float = 0.01) -> BathFit:
    """Super-ohmic J(w) = eta w^3/wc^2 exp(-w/wc); lambda line = 6 eta wc / pi
    (superohmic_ETOM.py:22,177)."""
    wc = wc_cm / HBAR
    eta = (reorg_cm / HBAR) * math.pi / (6.0 * wc)
    kt = temperature_k * BOLTZ_K
    t = np.linspace(0, t_max, n_t)
    y_re, y_im = _correlation(lambda w: w ** 3 / wc ** 2 * np.exp(-w / wc), HBAR / kt, t)
    p_re, p_im = _fit(t, y_re, y_im, n_osc, init_guess, bounded_imag=True)
    return BathFit(6.0 * eta * wc / math.pi, _lines(p_re, p_im, n_osc, eta))


def debye_lorentz(reorg_cm: float, gamma_cm: float, temperature_k: float, n_osc: int = 2,
                  n_matsubara: int = 100, t_max: float = 1000.0, n_t: int = 1000,
                  init_guess: float = 0.001) -> BathFit:
    """Drude-Lorentz bath through its Matsubara series (debye_lorentz_ETOM.py:17-40)."""
    gam = gamma_cm / HBAR
    lam = reorg_cm / HBAR
    beta_hbar = HBAR / (temperature_k * BOLTZ_K)
    t = np.linspace(0, t_max, n_t)
    y_re = gam * lam / np.tan(beta_hbar * gam / 2) * np.exp(-gam * t)
    for i in range(n_matsubara):
        nu = 2 * np.pi * (i + 1) / beta_hbar
        y_re = y_re + 4 * lam * gam / beta_hbar * nu / (nu ** 2 - gam ** 2) * np.exp(-nu * t)
    y_im = gam * lam * np.exp(-gam * t)
    p_re, p_im = _fit(t, y_re, y_im, n_osc, init_guess)
    return BathFit(lam, _lines(p_re, p_im, n_osc, 1.0))
