"""CPU restatement (numpy) of the reference's power-spectrum observables — TEST INFRASTRUCTURE.

Only the tests use it, as the checker of the device observables.  Each function follows the
reference file and lines it names (``src/discoeb/perturbations.py``, ``src/discoeb/util.py``).
Parity pins: there are no golden vectors for these functions in the reference's tests; the
restatement is pinned by known answers in ``tests/test_observables_oracle.py`` (the FFTLog xi_0 of
a Gaussian P(k) against its closed form, the multipoles against a Gauss-Legendre projection of
the Kaiser spectrum, the Savitzky-Golay filter reproducing cubics).
"""
from __future__ import annotations

import numpy as np

from .cmb_oracle import lngamma_complex


def get_power(k, y, idx, A_s, n_s, k_p):
    """perturbations.py:1445-1468"""
    return 2 * np.pi**2 * A_s * (k / k_p) ** (n_s - 1) * k ** (-3) * y[..., idx] ** 2


def savgol_filter(y, window_length, polyorder):
    """util.py:291-327: least-squares polynomial coefficients, convolved with mode 'same'"""
    halflen, rem = divmod(window_length, 2)
    pos = halflen - 0.5 if rem == 0 else halflen
    x = np.arange(-pos, window_length - pos, dtype=float)[::-1]
    A = x ** np.arange(polyorder + 1).reshape(-1, 1)
    Y = np.zeros(polyorder + 1)
    Y[0] = 1.0
    coeffs = np.linalg.lstsq(A, Y, rcond=None)[0]
    return np.convolve(y, coeffs, mode="same")


def get_power_smoothed(k, y, dlogk, idx, A_s, n_s, k_p):
    """perturbations.py:1471-1493"""
    wl = round(dlogk / (np.log(k[1]) - np.log(k[0])))
    wl += (wl + 1) % 2
    Pm = get_power(k, y, idx, A_s, n_s, k_p)
    Pms = np.exp(savgol_filter(np.log(Pm), wl, 3))
    Pms[: wl // 2] = Pm[: wl // 2]
    Pms[-wl // 2:] = Pm[-wl // 2:]
    return Pms


def amplitudes(k, y, A_s, n_s, k_p):
    """delta_m and theta_m amplitudes of power_Kaiser / power_multipoles (perturbations.py:1515-1516)"""
    fac = 2 * np.pi**2 * A_s
    s = np.sqrt(fac * (k / k_p) ** (n_s - 1) * k ** (-3))
    return s * y[:, 4], s * y[:, 5]


def power_Kaiser(y, k, bias, nmu, A_s, n_s, k_p, mu_sampling=True, smooth_dlogk=None):
    """perturbations.py:1495-1524"""
    mu = np.linspace(-1, 1, nmu) if mu_sampling else np.cos(np.linspace(0, np.pi, nmu))
    if smooth_dlogk is None:
        deltam, thetam = amplitudes(k, y, A_s, n_s, k_p)
    else:
        deltam = np.sqrt(get_power_smoothed(k, y, smooth_dlogk, 4, A_s, n_s, k_p))
        thetam = -np.sqrt(get_power_smoothed(k, y, smooth_dlogk, 5, A_s, n_s, k_p))
    return (bias * deltam[:, None] - mu[None, :] ** 2 * thetam[:, None]) ** 2, mu


def power_multipoles(y, k, b, A_s, n_s, k_p):
    """perturbations.py:1528-1564"""
    deltam, thetam = amplitudes(k, y, A_s, n_s, k_p)
    P0 = b**2 * deltam**2 - 2 * b / 3 * deltam * thetam + 1 / 5 * thetam**2
    P2 = -4 * b / 3 * deltam * thetam + 4 / 7 * thetam**2
    P4 = 8 / 35 * thetam**2
    return P0, P2, P4


def get_xi_from_P(k, Pk, ell=0):
    """perturbations.py:1409-1442 (FFTLog, Talman 1978, Hamilton 2000)"""
    N = len(k)
    L = np.log(k[N - 1] / k[0])
    fPk = np.fft.rfft(Pk * k**1.5)
    ki = np.pi * np.arange(N // 2 + 1) / L
    zp = (1.5 + ell) / 2 + 1j * ki
    theta = lngamma_complex(zp).imag
    fPk = fPk * np.exp(2j * (theta - np.log(np.pi) * ki))
    r = 2 * np.pi / k
    xi = np.real(1j**ell * np.fft.irfft(fPk) / (2 * np.pi * r) ** 1.5)
    return xi[::-1], r[::-1]
