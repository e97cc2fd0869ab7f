"""The FFTLog coefficient helpers of the line of sight compiled for the host: complex digamma
against scipy, and the derivative of M_l(p) along the grid spacing against difference quotients
of the same function (CPU)."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT


@pytest.fixture(scope="module")
def lib(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("fftlog") / "fftlog_shim.so")
    subprocess.run(["g++", "-O2", "-fPIC", "-shared", "-std=c++17", "-I", os.path.join(ROOT, "disco-eb_b200", "csrc"),
                    "-o", out, os.path.join(ROOT, "tests", "cpu_model", "fftlog_shim.cpp")], check=True)
    L = ctypes.CDLL(out)
    d, dp = ctypes.c_double, ctypes.POINTER(ctypes.c_double)
    L.shim_lngamma.argtypes = [d, d, dp]
    L.shim_digamma.argtypes = [d, d, dp]
    L.shim_mcoef.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, d, d, d, dp, dp]
    L.shim_mcoef_run.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, d, d, d, dp, dp]
    return L


def _call(f, *args):
    out = np.zeros(2)
    f(*args, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    return complex(out[0], out[1])


def test_digamma_matches_scipy_on_both_branches(lib):
    scipy_special = pytest.importorskip("scipy.special")
    rng = np.random.default_rng(3)
    # the arguments the line of sight meets: (l - 0.1)/2 + i eta/2 and (3.1 + l)/2 - i eta/2,
    # l up to a few thousand, |eta| up to ~1e4, plus the reflection region Re z <= 0.5
    zs = [complex(r, i) for r, i in zip(rng.uniform(-0.45, 1500.0, 200), rng.uniform(-3000.0, 3000.0, 200))]
    zs += [complex(-0.05, 0.0), complex(0.45, 0.0), complex(-0.05, 37.0), complex(0.45, -250.0), complex(2.0, 1e-3)]
    for z in zs:
        got = _call(lib.shim_digamma, z.real, z.imag)
        ref = complex(scipy_special.psi(z))
        assert abs(got - ref) <= 1e-11 * max(1.0, abs(ref)), (z, got, ref)


def test_mcoef_tangent_is_the_derivative_of_the_coefficient(lib):
    dp = ctypes.POINTER(ctypes.c_double)
    n_fft, bias = 16384, -1.1
    for dl in (8.2e-4, 2.4e-3):
        for l in (0, 1, 2, 30, 700, 2500):
            for q in (0, 1, 17, 900, 4000, 8192):
                b, bd = np.zeros(2), np.zeros(2)
                lib.shim_mcoef(l, q, n_fft, bias, dl, 1.0, b.ctypes.data_as(dp), bd.ctypes.data_as(dp))
                # fourth-order quotient: the phase of M_l turns fast with the spacing at large q
                h = 1e-6 * dl
                fd, tmp = np.zeros(2), np.zeros(2)
                for m, w in ((2, -1.0 / 12), (1, 8.0 / 12), (-1, -8.0 / 12), (-2, 1.0 / 12)):
                    bm = np.zeros(2)
                    lib.shim_mcoef(l, q, n_fft, bias, dl + m * h, 0.0, bm.ctypes.data_as(dp), tmp.ctypes.data_as(dp))
                    fd += w * bm / h
                scale = max(np.abs(fd).max(), np.abs(b).max() / dl, 1e-300)
                # the quotient's own rounding: ln M is a difference of two log-Gammas of size ~l ln l
                eta = 2 * np.pi * q / (n_fft * dl)
                big = sum(abs(_call(lib.shim_lngamma, a.real, a.imag)) for a in
                          (complex((1 + l + bias) / 2, eta / 2), complex((2 + l - bias) / 2, -eta / 2)))
                if not np.isfinite(big):  # the reference's log-Gamma overflows: M and M' are zero
                    assert np.all(b == 0.0) and np.all(bd == 0.0), (dl, l, q, b, bd)
                    continue
                noise = 4e-16 * (big + 10.0) * np.abs(b).max() / h
                assert np.abs(bd - fd).max() <= 1e-7 * scale + noise, (dl, l, q, bd, fd, noise)


def test_mcoef_recurrence_in_l_matches_the_direct_evaluation(lib):
    """the table kernel evaluates log-Gamma at every 16th l of a parity and steps
    M_{l+2} = M_l (1 + l + p)/(2 + l - p) (and d ln M/dp by psi(z + 1) = psi(z) + 1/z) in between.
    Agreement to the direct evaluation's own rounding: its phase is the difference of two
    log-Gammas of size ~|z ln z| (~1e4 at the largest frequencies), so eps times those moves M by
    up to ~1e-12 of |M| there, in the reference's direct evaluation as well"""
    dp = ctypes.POINTER(ctypes.c_double)
    n_fft, bias, count = 16384, -1.1, 16
    for dl in (8.2e-4, 2.4e-3):
        for l0 in (2, 3, 34, 1001, 2466):
            for q in (0, 1, 17, 900, 4000, 8192):
                run, run_d = np.zeros(2 * count), np.zeros(2 * count)
                lib.shim_mcoef_run(l0, count, q, n_fft, bias, dl, 0.7, run.ctypes.data_as(dp), run_d.ctypes.data_as(dp))
                eta = 2 * np.pi * q / (n_fft * dl)
                for i in range(count):
                    l = l0 + 2 * i
                    b, bd = np.zeros(2), np.zeros(2)
                    lib.shim_mcoef(l, q, n_fft, bias, dl, 0.7, b.ctypes.data_as(dp), bd.ctypes.data_as(dp))
                    big = sum(abs(_call(lib.shim_lngamma, a.real, a.imag)) for a in
                              (complex((1 + l + bias) / 2, eta / 2), complex((2 + l - bias) / 2, -eta / 2)))
                    tol = (1e-13 + 4e-16 * big) * np.abs(b).max()
                    assert np.abs(run[2 * i:2 * i + 2] - b).max() <= tol, (dl, l0, q, i)
                    assert np.abs(run_d[2 * i:2 * i + 2] - bd).max() <= (1e-12 + 4e-16 * big) * np.abs(bd).max() + \
                        tol * (0.7 / dl) * eta, (dl, l0, q, i)
