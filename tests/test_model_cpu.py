"""The device model and stepper sources, compiled for one host thread, against the oracle (CPU).

The CUDA kernels instantiate the same headers with a 32-lane warp team; this harness
checks their algebra (RHS, Jacobian, structured W solve, full adaptive solve) before any
GPU run.
"""
import ctypes

import numpy as np
import pytest

from conftest import background
from discoeb_b200 import _abi
from oracle import pyoracle as O

dp = ctypes.POINTER(ctypes.c_double)
CP = ctypes.POINTER(_abi.DiscoebCosmo)
L = dict(lmaxg=12, lmaxgp=12, lmaxr=17, lmaxnu=17, nqmax=5)


def ptr(a):
    return a.ctypes.data_as(dp)


@pytest.fixture(scope="module")
def setup():
    bg = background("disco_notebook", 512)
    keep = []
    C = _abi.make_cosmo(bg, de_guard_eps=0.0, table_ptrs=_abi.host_table_ptrs(bg, keep), **L)
    OP = O.OracleProblem(bg, **L)
    return bg, C, OP, keep


def _states(bg, OP, k):
    ts = 0.99 * OP.start_time(k)
    tout = bg["tau_of_a_spline"].evaluate(np.array([1e-4, 1e-3, 0.01, 0.3, 1.0]))
    ys, st = OP.solve([k], ts, OP.ics(ts, k), tout, rtol=1e-6, atol=1e-8, max_steps=100000)
    return tout, ys[0]


@pytest.mark.parametrize("k", [1e-4, 3e-3, 0.05, 0.3, 2.0, 10.0])
def test_rhs_jacobian_and_wsolve_match_oracle(shim, setup, k):
    bg, C, OP, _ = setup
    n = OP.n
    rng = np.random.default_rng(1)
    tout, ys = _states(bg, OP, k)
    for tau, ybase in zip(tout, ys):
        y = ybase * (1 + 0.01 * rng.standard_normal(n))
        for regime in (-1, 0, 1, 2):
            f_o = OP.rhs(tau, y, k, regime)
            f_s, c0 = np.zeros(n), np.zeros(n)
            shim.shim_rhs(ctypes.byref(C), tau, ptr(y), k, regime, ptr(f_s), ptr(c0))
            np.testing.assert_allclose(f_s, f_o, rtol=0, atol=1e-12 * np.abs(f_o).max())
            Jo, dTo = OP.jacobian(tau, y, k, regime)
            Js, dTs = np.zeros((n, n)), np.zeros(n)
            shim.shim_jacobian(ctypes.byref(C), tau, ptr(y), k, regime, ptr(Js), ptr(dTs))
            assert np.max(np.abs(Js - Jo) / (np.abs(Jo).max(axis=0) + 1e-300)) < 1e-12
            np.testing.assert_allclose(dTs, dTo, rtol=0, atol=1e-14 * (np.abs(dTo).max() + 1e-300))
            if regime == 1 and tau < 100.0:
                continue  # RSA forced deep in the tightly coupled era is not a regime the solver visits
            h = 0.05 * tau
            W = np.eye(n) / (0.19 * h) - Jo
            r = rng.standard_normal(n)
            x_o = np.linalg.solve(W, r)
            x_s = np.zeros(n)
            rc = shim.shim_wsolve(ctypes.byref(C), tau, ptr(y), k, regime, h, ptr(r), ptr(x_s))
            assert rc == 0
            np.testing.assert_allclose(x_s, x_o, rtol=0, atol=1e-10 * np.abs(x_o).max())


@pytest.mark.parametrize("k", [1e-4, 1e-2, 0.1, 1.0, 10.0])
def test_adaptive_solve_matches_oracle(shim, setup, k):
    bg, C, OP, _ = setup
    n = OP.n
    ctrl = _abi.DiscoebControl(1e-5, 1e-8, 0.25, 0.8, 0.0, 20.0, 0.3, 100000, 0, 0, 0)
    tout = bg["tau_of_a_spline"].evaluate(np.array([1 / 3, 0.5, 2 / 3, 1.0]))
    ts = 0.99 * min(tout.min(), OP.start_time(k))
    y0 = OP.ics(ts, k)
    sw = OP.switch_times(k)
    yo, st = OP.solve([k], ts, y0, tout, rtol=1e-5, atol=1e-8, max_steps=100000)
    ys = np.zeros((4, n))
    stats = (ctypes.c_int * 3)()
    shim.shim_solve_mode(ctypes.byref(C), ctypes.byref(ctrl), k, ts, ptr(y0), ptr(sw), 4, ptr(tout), ptr(ys), stats)
    assert stats[0] == 0
    assert abs(stats[1] - st.steps) <= max(2, 0.01 * st.steps)  # same step sequence up to rounding flips
    for v in (0, 2, 3, 5):
        np.testing.assert_allclose(ys[:, v], yo[0][:, v], rtol=1e-6)


@pytest.mark.parametrize("k", [1e-4, 0.05, 2.0, 10.0])
def test_mixed_precision_wsolve_matches_oracle(shim, setup, k):
    """The mixed-precision W solve (FP32 chain factors, one FP64 refinement of every chain solve)
    against the dense FP64 solve of the oracle's W, at the bar of the FP64 structured solve."""
    bg, C, OP, _ = setup
    n = OP.n
    rng = np.random.default_rng(2)
    tout, ys = _states(bg, OP, k)
    worst = 0.0
    for tau, ybase in zip(tout, ys):
        y = ybase * (1 + 0.01 * rng.standard_normal(n))
        for regime in (-1, 0, 2):
            Jo, _ = OP.jacobian(tau, y, k, regime)
            for h in (0.05 * tau, 1e-3 * tau):
                W = np.eye(n) / (0.19 * h) - Jo
                r = rng.standard_normal(n)
                x_o = np.linalg.solve(W, r)
                x_m, x_d = np.zeros(n), np.zeros(n)
                assert shim.shim_wsolve_mixed(ctypes.byref(C), tau, ptr(y), k, regime, h, ptr(r), ptr(x_m)) == 0
                assert shim.shim_wsolve(ctypes.byref(C), tau, ptr(y), k, regime, h, ptr(r), ptr(x_d)) == 0
                np.testing.assert_allclose(x_m, x_o, rtol=0, atol=1e-10 * np.abs(x_o).max())
                worst = max(worst, float(np.abs(x_m - x_d).max() / np.abs(x_d).max()))
    assert worst > 0.0  # the FP32 factors do change the rounding
    print("mixed vs FP64 structured solve:", worst)


@pytest.mark.parametrize("k", [1e-3, 0.1, 10.0])
def test_mixed_precision_adaptive_solve_matches_fp64(shim, setup, k):
    bg, C, OP, _ = setup
    n = OP.n
    ctrl = _abi.DiscoebControl(1e-5, 1e-8, 0.25, 0.8, 0.0, 20.0, 0.3, 100000, 0, 0, 0)
    tout = bg["tau_of_a_spline"].evaluate(np.array([1 / 3, 0.5, 2 / 3, 1.0]))
    ts = 0.99 * min(tout.min(), OP.start_time(k))
    y0 = OP.ics(ts, k)
    sw = OP.switch_times(k)
    ys, ym = np.zeros((4, n)), np.zeros((4, n))
    st_d, st_m = (ctypes.c_int * 3)(), (ctypes.c_int * 3)()
    shim.shim_solve_mode(ctypes.byref(C), ctypes.byref(ctrl), k, ts, ptr(y0), ptr(sw), 4, ptr(tout), ptr(ys), st_d)
    shim.shim_solve_mode_mixed(ctypes.byref(C), ctypes.byref(ctrl), k, ts, ptr(y0), ptr(sw), 4, ptr(tout), ptr(ym),
                               st_m)
    assert st_d[0] == 0 and st_m[0] == 0
    assert abs(st_m[1] - st_d[1]) <= max(2, 0.01 * st_d[1])
    # the refined solves differ from the FP64 ones by ~1e-12 (the test above), which the error
    # control turns into different step sizes: the solutions then agree to well inside rtol
    for v in (0, 2, 3, 5):
        np.testing.assert_allclose(ym[:, v], ys[:, v], rtol=1e-6)
