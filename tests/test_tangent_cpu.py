"""Forward-mode derivatives, checked on the CPU.

* The tangent stepper (stepper.cuh, compiled for one host thread) against central finite
  differences of the same discrete solve with its accepted step sequence replayed: the tangent
  is the exact derivative of the Rodas5 solution at a fixed step sequence, so the two agree to
  finite-difference accuracy.
* The host tangents of gradients.background_tangents (complex step through the background with
  the Recfast step sequence replayed) against central finite differences of the same replayed
  background.
"""
import ctypes
import warnings

import numpy as np
import pytest

from conftest import background
from discoeb_b200 import _abi
from discoeb_b200.background import evolve_background
from discoeb_b200.gradients import background_tangents, theta_to_params
from discoeb_b200.spline import spline_interpolation
from oracle import pyoracle as O

dp = ctypes.POINTER(ctypes.c_double)
L = dict(lmaxg=8, lmaxgp=8, lmaxr=8, lmaxnu=6, nqmax=3)
SCALARS = ("grhom", "Omegam", "Omegab", "OmegaDE", "amnu", "w0", "wa", "H0")
TABLES = {"xe": "xe_of_loga_spline", "cs2a": "cs2a_of_loga_spline", "logrhonu": "logrhonu_of_loga_spline",
          "logpnu": "logpnu_of_loga_spline"}


def ptr(a):
    return a.ctypes.data_as(dp)


@pytest.fixture(scope="module")
def prob():
    bg = background("disco_notebook", 256)
    return bg, O.OracleProblem(bg, **L)


def _cosmo(bg, keep, scalar=None, eps=0.0, table=None, dtab=None):
    """DiscoebCosmo of bg with one scalar moved by eps or one table's y moved by eps*dtab."""
    bgp = dict(bg)
    if table is not None:
        s0 = bg[TABLES[table]]
        s1 = spline_interpolation.__new__(spline_interpolation)
        s1.__dict__.update(s0.__dict__)
        s1.y = s0.y + eps * dtab
        bgp[TABLES[table]] = s1
    C = _abi.make_cosmo(bgp, de_guard_eps=0.0, table_ptrs=_abi.host_table_ptrs(bgp, keep), **L)
    if scalar is not None:
        setattr(C, scalar, getattr(C, scalar) + eps)
    return C


@pytest.mark.parametrize("k", [0.01, 0.3])
@pytest.mark.parametrize("case", ["y0", "grhom", "Omegab", "amnu", "w0", "H0", "xe", "cs2a", "logrhonu"])
def test_tangent_is_derivative_of_discrete_solve(shim, prob, k, case):
    bg, OP = prob
    n = OP.n
    keep = []
    rng = np.random.default_rng(7)
    C = _cosmo(bg, keep)
    ctrl = _abi.DiscoebControl(1e-5, 1e-8, 0.25, 0.8, 0.0, 20.0, 0.3, 100000, 0, 0, 0)
    tout = np.array([bg["tau_of_a_spline"].evaluate(1.0)])
    ts = 0.99 * OP.start_time(k)
    y0 = OP.ics(ts, k)
    sw = OP.switch_times(k)
    tn = _abi.DiscoebTangent()
    yd0 = np.zeros(n)
    dtab = None
    if case == "y0":
        yd0 = y0 * 0.3 * rng.standard_normal(n)
    elif case in TABLES:
        yt = bg[TABLES[case]].y
        dtab = 1e-3 * rng.standard_normal(yt.size) * np.abs(yt)
        keep.append(dtab)
        setattr(tn, case + "_y", dtab.ctypes.data)
    else:
        setattr(tn, case, 1.0)
    yo, ydo = np.zeros((1, n)), np.zeros((1, n))
    stats = (ctypes.c_int * 3)()
    tlog = np.zeros(100000)
    shim.shim_solve_mode_tangent(ctypes.byref(C), ctypes.byref(tn), ctypes.byref(ctrl), k, ts, ptr(y0), ptr(yd0),
                                 ptr(sw), 1, ptr(tout), ptr(yo), ptr(ydo), stats, ptr(tlog), tlog.size)
    assert stats[0] == 0
    tsteps = tlog[:stats[2]].copy()
    assert tsteps[-1] == tout[0]

    def run(eps):
        if case == "y0":
            Cx, yy0 = C, y0 + eps * yd0
        elif case in TABLES:
            Cx, yy0 = _cosmo(bg, keep, table=case, eps=eps, dtab=dtab), y0
        else:
            Cx, yy0 = _cosmo(bg, keep, scalar=case, eps=eps), y0
        ye = np.zeros(n)
        shim.shim_replay(ctypes.byref(Cx), k, ts, ptr(yy0.copy()), ptr(sw), len(tsteps), ptr(tsteps), ptr(ye))
        return ye

    # table moves are eps * 1e-3 relative: eps = 0.1 keeps them well above round-off
    eps = 1e-6 if case == "y0" else 0.1 if case in TABLES else 1e-6 * abs(getattr(C, case))
    yp, ym = run(eps), run(-eps)
    np.testing.assert_allclose(run(0.0), yo[0], rtol=1e-12, atol=1e-300)  # the replay reproduces the solve
    fd = (yp - ym) / (2 * eps)
    for v in (0, 2, 3, 5, 6):  # a, eta, delta_c, delta_b, theta_b
        noise = 1e-12 * abs(yo[0][v]) / eps  # round-off of the difference quotient
        assert abs(ydo[0][v] - fd[v]) <= 1e-5 * abs(fd[v]) + noise, (v, ydo[0][v], fd[v], noise)


@pytest.mark.parametrize("case", ["y", "grhom", "Omegam", "Omegab", "OmegaDE", "amnu", "w0", "wa", "H0", "logrhonu",
                                  "logpnu", "xe", "cs2a"])
def test_output_and_projection_tangents(shim, prob, case):
    """output_vars and the RSA projection in dual numbers against central differences."""
    bg, OP = prob
    n = OP.n
    keep = []
    rng = np.random.default_rng(3)
    k = 0.3
    tau = bg["tau_of_a_spline"].evaluate(0.5)
    ts = 0.99 * OP.start_time(k)
    ys, _ = OP.solve([k], ts, OP.ics(ts, k), np.array([tau]), rtol=1e-6, atol=1e-9, max_steps=100000)
    y = ys[0][0]
    tn = _abi.DiscoebTangent()
    yd = np.zeros(n)
    dtab = None
    if case == "y":
        yd = y * rng.standard_normal(n)
    elif case in TABLES:
        yt = bg[TABLES[case]].y
        dtab = rng.standard_normal(yt.size) * np.abs(yt)
        keep.append(dtab)
        setattr(tn, case + "_y", dtab.ctypes.data)
    else:
        setattr(tn, case, 1.0)
    C = _cosmo(bg, keep)
    o, od, r, rd = np.zeros(20), np.zeros(20), np.zeros(4), np.zeros(4)
    shim.shim_output_tangent(ctypes.byref(C), ctypes.byref(tn), k, tau, ptr(y), ptr(yd), ptr(o), ptr(od), ptr(r),
                             ptr(rd))

    def at(eps):
        if case == "y":
            Cx, yy = C, y + eps * yd
        elif case in TABLES:
            Cx, yy = _cosmo(bg, keep, table=case, eps=eps, dtab=dtab), y
        else:
            Cx, yy = _cosmo(bg, keep, scalar=case, eps=eps), y
        oo, ood, rr, rrd = np.zeros(20), np.zeros(20), np.zeros(4), np.zeros(4)
        shim.shim_output_tangent(ctypes.byref(Cx), None, k, tau, ptr(yy.copy()), ptr(np.zeros(n)), ptr(oo),
                                 ptr(ood), ptr(rr), ptr(rrd))
        return np.concatenate([oo, rr])

    eps = 1e-6 if case == "y" or case in TABLES else 1e-6 * (abs(getattr(C, case)) or 1.0)
    fd = (at(eps) - at(-eps)) / (2 * eps)
    got = np.concatenate([od, rd])
    val = np.concatenate([o, r])
    tol = 1e-6 * np.abs(fd) + 1e-12 * np.abs(val) / eps  # truncation + round-off
    assert np.all(np.abs(got - fd) <= tol + 1e-12 * np.abs(fd).max()), np.abs(got - fd) / (np.abs(fd) + 1e-300)


@pytest.mark.parametrize("k", [1e-3, 0.05, 1.0])
def test_tangent_replayed_from_step_records_equals_combined_solve(shim, prob, k):
    """The per-mode block kernel of discoeb_jvp solves the forward once, records every accepted
    step (start state, stages, factorisation of W) and carries each direction's tangent through
    the records afterwards: the same arithmetic as the tangent interleaved with the forward
    stages, so the results agree exactly."""
    bg, OP = prob
    n = OP.n
    keep = []
    C = _cosmo(bg, keep)
    ctrl = _abi.DiscoebControl(1e-5, 1e-8, 0.25, 0.8, 0.0, 20.0, 0.3, 100000, 0, 0, 0)
    tout = bg["tau_of_a_spline"].evaluate(np.array([0.25, 0.5, 1.0]))
    ts = 0.99 * min(tout.min(), OP.start_time(k))
    y0, sw = OP.ics(ts, k), OP.switch_times(k)
    yd0 = y0 * np.random.default_rng(5).standard_normal(n) * 0.1
    tn = _abi.DiscoebTangent()
    tn.Omegab, tn.amnu, tn.w0 = 1.0, 0.2, 0.5
    ya, yda, yb_d = np.zeros((3, n)), np.zeros((3, n)), np.zeros((3, n))
    s1, s2 = (ctypes.c_int * 3)(), (ctypes.c_int * 3)()
    shim.shim_solve_mode_tangent(ctypes.byref(C), ctypes.byref(tn), ctypes.byref(ctrl), k, ts, ptr(y0.copy()),
                                 ptr(yd0.copy()), ptr(sw), 3, ptr(tout), ptr(ya), ptr(yda), s1, ptr(np.zeros(1)), 0)
    shim.shim_solve_mode_tangent_records(ctypes.byref(C), ctypes.byref(tn), ctypes.byref(ctrl), k, ts, ptr(y0.copy()),
                                         ptr(yd0.copy()), ptr(sw), 3, ptr(tout), ptr(yb_d), s2)
    assert s1[0] == s2[0] == 0 and s1[1] == s2[1] and s1[2] == s2[2]
    np.testing.assert_array_equal(yb_d, yda)


def _fd_background(theta, name, trace, eps):
    side = []
    for sgn in (1, -1):
        th = dict(theta)
        th[name] += sgn * eps
        side.append(evolve_background(param=theta_to_params(th), replay=trace))
    return side


@pytest.mark.parametrize("name", ["omega_c", "omega_b", "h", "w0", "wa", "m_nu"])
def test_host_tangents_match_replayed_fd(name):
    """Complex-step tangents vs central differences of the replayed background.

    The Recfast right-hand side selects formulas by the values of x_H, x_He and the Compton
    time (jnp.where in the reference): forward-mode AD, like the complex step, differentiates
    the branch taken, while a difference quotient that straddles a switch sees its jump.
    Table knots are compared where two step sizes give consistent quotients (a smooth point).
    """
    from discoeb_b200.perturbations import adiabatic_ics
    theta = dict(omega_c=0.12, omega_b=0.0224, h=0.674, n_s=0.965, ln10As=np.log(21.0), w0=-0.9, wa=0.05, m_nu=0.06)
    ks, aout, ts = np.array([0.01, 0.2]), np.array([0.5, 1.0]), np.array([0.5, 0.1])
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        trace = {}
        bg = evolve_background(param=theta_to_params(theta), trace=trace)
        d = background_tangents(theta, bg, trace, (name,), aexp_out=aout, tau_start=ts, kmodes=ks, L=L)[0]
        eps = 1e-4 * abs(theta[name])
        side = _fd_background(theta, name, trace, eps)
        side2 = _fd_background(theta, name, trace, 4 * eps)
    fd_tau = (side[0]["tau_of_a_spline"].evaluate(aout) - side[1]["tau_of_a_spline"].evaluate(aout)) / (2 * eps)
    np.testing.assert_allclose(d["tau_out"], fd_tau, rtol=1e-6)
    for key, field in (("grhom", "grhom"), ("OmegaDE", "OmegaDE"), ("amnu", "amnu"), ("H0", "H0")):
        fd = (side[0][key] - side[1][key]) / (2 * eps)
        assert abs(d["scalars"][field] - fd) <= 1e-6 * abs(fd) + 1e-12, (field, d["scalars"][field], fd)
    for short, key in TABLES.items():
        fd = (side[0][key].y - side[1][key].y) / (2 * eps)
        fd2 = (side2[0][key].y - side2[1][key].y) / (8 * eps)
        # truncation (local) + round-off; switches move with theta, so a knot downstream of a
        # moved switch has a difference quotient that depends on eps: those are left out (for h
        # a switch near z = 2000 moves, which leaves about 40% of the xe knots comparable)
        tol = 1e-4 * np.abs(fd) + 1e-12 * np.abs(bg[key].y) / eps + 1e-9 * np.abs(fd).max()
        smooth = np.abs(fd - fd2) <= tol
        assert smooth.mean() > 0.3, (short, smooth.mean())
        yy, _ = d["tables"][short]
        assert np.all((np.abs(yy - fd) <= tol)[smooth]), short
    y0p = adiabatic_ics(tau=ts, param=side[0], kmode=ks, **L)
    y0m = adiabatic_ics(tau=ts, param=side[1], kmode=ks, **L)
    fd = (y0p - y0m) / (2 * eps)
    y0 = adiabatic_ics(tau=ts, param=bg, kmode=ks, **L)
    # per mode: the derivative of each initial field, to the scale of that mode's state
    tol = 1e-6 * np.abs(fd).max(axis=1, keepdims=True) + 1e-12 * np.abs(y0).max(axis=1, keepdims=True) / eps
    assert np.all(np.abs(d["y0"] - fd) <= 1e-5 * np.abs(fd) + tol)
