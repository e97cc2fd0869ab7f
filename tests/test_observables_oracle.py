"""Known-answer pins of the observables' CPU restatement (oracle/observables_oracle.py), which the
GPU tests use as their checker, and the host pieces of discoeb_b200.observables (CPU)."""
import math

import numpy as np
import pytest

from oracle import observables_oracle as OB


@pytest.mark.parametrize("ell", [0, 2, 4])
def test_fftlog_xi_of_gaussian_spectrum_matches_closed_form(ell):
    # P(k) = k^l exp(-a k^2): int k^2 P(k) j_l(k r) dk = sqrt(pi) r^l exp(-r^2/4a) / (2^(l+2) a^(l+3/2)),
    # and xi_l = i^l / (2 pi^2) times that (the reference's convention, with the i^l factor).  The
    # reference's FFTLog (a periodic transform in log k without end-point weights) is accurate to
    # ~1e-3 of the peak at 4096 points over 8 decades, and the error halves on a grid of twice the
    # points over 9 decades.
    a = 50.0
    errs = []
    for n, lo in ((4096, 1e-5), (8192, 1e-6)):
        k = np.geomspace(lo, 1e3, n)
        xi, r = OB.get_xi_from_P(k, k**ell * np.exp(-a * k**2), ell=ell)
        exact = (1j**ell).real / (2 * math.pi**2) * math.sqrt(math.pi) * r**ell * np.exp(-r**2 / (4 * a)) \
            / (2 ** (ell + 2) * a ** (ell + 1.5))
        sel = (r > 2.0) & (r < 40.0)
        errs.append(np.abs(xi[sel] - exact[sel]).max() / np.abs(exact[sel]).max())
        assert np.all(np.diff(r) > 0)
    assert errs[0] < 2e-3, errs
    assert errs[1] < 0.6 * errs[0], errs


def test_multipoles_are_legendre_projections_of_kaiser():
    rng = np.random.default_rng(1)
    K = 16
    k = np.geomspace(1e-3, 1.0, K)
    y = np.zeros((K, 20))
    y[:, 4] = rng.uniform(1.0, 3.0, K) * 1e2
    y[:, 5] = -rng.uniform(0.2, 1.0, K) * 1e2
    A_s, n_s, k_p, b = 2.1e-9, 0.965, 0.05, 1.7
    P0, P2, P4 = OB.power_multipoles(y, k, b, A_s, n_s, k_p)
    x, w = np.polynomial.legendre.leggauss(16)
    d, t = OB.amplitudes(k, y, A_s, n_s, k_p)
    Pkmu = (b * d[:, None] - x[None, :] ** 2 * t[:, None]) ** 2
    for ell, P in ((0, P0), (2, P2), (4, P4)):
        Lx = np.polynomial.legendre.Legendre.basis(ell)(x)
        proj = (2 * ell + 1) / 2 * (Pkmu * (w * Lx)[None, :]).sum(1)
        np.testing.assert_allclose(P, proj, rtol=1e-12, atol=1e-12 * np.abs(P0).max())
    Pk, mu = OB.power_Kaiser(y, k, b, 7, A_s, n_s, k_p)
    np.testing.assert_allclose(Pk, (b * d[:, None] - mu[None, :] ** 2 * t[:, None]) ** 2, rtol=1e-15)


def test_savgol_smoothing_keeps_power_laws():
    # log P linear in log k is reproduced by a cubic Savitzky-Golay filter away from the ends
    k = np.geomspace(1e-3, 1.0, 200)
    y = np.zeros((200, 20))
    y[:, 4] = k**-0.3
    Ps = OB.get_power_smoothed(k, y, 0.5, 4, 2.1e-9, 0.965, 0.05)
    P = OB.get_power(k, y, 4, 2.1e-9, 0.965, 0.05)
    np.testing.assert_allclose(Ps, P, rtol=1e-11)
    # and a cubic in the sample index is reproduced exactly by the filter itself
    i = np.arange(50, dtype=float)
    cub = 0.1 * i**3 - 2 * i**2 + i - 5
    out = OB.savgol_filter(cub, 9, 3)
    np.testing.assert_allclose(out[4:-4], cub[4:-4], rtol=1e-10, atol=1e-9)


def test_host_savgol_coefficients_match_oracle_filter():
    from discoeb_b200.observables import savgol_coeffs
    c = savgol_coeffs(11, 3)
    assert abs(c.sum() - 1.0) < 1e-12
    y = np.random.default_rng(0).normal(size=40)
    np.testing.assert_allclose(np.convolve(y, c, mode="same"), OB.savgol_filter(y, 11, 3), rtol=0, atol=1e-14)
