"""The discrete adjoint (adjoint.cuh, compiled for one host thread), checked on the CPU against the
forward-mode tangent of the same discrete solve.

* One Rodas5 step: the reverse sweep is the transpose of the tangent step, so for any tangent
  (state, parameter and table-knot directions) and any cotangent lambda of the result,
  lambda . dy_1 = ybar_0 . dy_0 + pbar . dp + tbar . dtables  to rounding.
* A whole mode: record the forward solve (step end times and checkpoints), run the reverse sweep
  from a cotangent of the 20 output fields at every output time, and compare with the
  forward-mode tangent of the same solve along a random direction (state, parameters, tables and
  output times), through the output layer.
"""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, background
from discoeb_b200 import _abi
from oracle import pyoracle as O

dp = ctypes.POINTER(ctypes.c_double)
CP = ctypes.POINTER(_abi.DiscoebCosmo)
CT = ctypes.POINTER(_abi.DiscoebControl)
L = dict(lmaxg=8, lmaxgp=8, lmaxr=8, lmaxnu=6, nqmax=3)
SCALARS = ("grhom", "Omegam", "Omegab", "OmegaDE", "amnu", "w0", "wa", "H0")
TABLES = {"xe": "xe_of_loga_spline", "cs2a": "cs2a_of_loga_spline", "logrhonu": "logrhonu_of_loga_spline",
          "logpnu": "logpnu_of_loga_spline"}


def ptr(a):
    return a.ctypes.data_as(dp)


@pytest.fixture(scope="module")
def adj(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("adj") / "adjoint_shim.so")
    subprocess.run(["g++", "-O2", "-fPIC", "-shared", "-std=c++17", "-I", os.path.join(ROOT, "include"),
                    "-I", os.path.join(ROOT, "disco-eb_b200", "csrc"), "-o", out,
                    os.path.join(ROOT, "tests", "cpu_model", "adjoint_shim.cpp")], check=True)
    A = ctypes.CDLL(out)
    i, d, vp = ctypes.c_int, ctypes.c_double, ctypes.c_void_p
    A.shim_adjoint_step.argtypes = [CP, vp, d, d, d, i, dp, dp, dp, dp, dp, dp, dp, dp, i]
    A.shim_fwd_record.argtypes = [CP, CT, d, d, dp, dp, i, dp, i, i, dp, dp, dp, ctypes.POINTER(i)]
    A.shim_bwd_mode.argtypes = [CP, d, d, dp, i, dp, dp, dp, i, i, dp, dp, dp, dp, dp, i]
    return A


@pytest.fixture(scope="module")
def setup():
    bg = background("disco_notebook", 256)
    OP = O.OracleProblem(bg, **L)
    keep = []
    C = _abi.make_cosmo(bg, de_guard_eps=0.0, table_ptrs=_abi.host_table_ptrs(bg, keep), **L)
    nk = max(bg[v].n for v in TABLES.values())
    return bg, OP, C, keep, nk


def _random_tangent(bg, C, rng, keep, parts=("scalars", "tables")):
    tn = _abi.DiscoebTangent()
    tabs = {}
    if "scalars" in parts:
        for f in SCALARS:
            setattr(tn, f, getattr(C, f) * rng.standard_normal())
    if "tables" in parts:
        for short, key in TABLES.items():
            sp = bg[key]
            dy = rng.standard_normal(sp.n) * np.abs(sp.y) * 1e-2
            dS = rng.standard_normal(sp.n) * np.abs(sp.S) * 1e-2
            keep += [dy, dS]
            tabs[short] = (dy, dS)
            setattr(tn, short + "_y", dy.ctypes.data)
            setattr(tn, short + "_S", dS.ctypes.data)
    return tn, tabs


def _pair(tn, tabs, pbar, tbar):
    """pbar . d(parameters) + tbar . d(tables) for the direction tn."""
    s = sum(pbar[i] * getattr(tn, f) for i, f in enumerate(SCALARS))
    for ti, short in enumerate(TABLES):
        if short in tabs:
            dy, dS = tabs[short]
            s += tbar[2 * ti, :dy.size] @ dy + tbar[2 * ti + 1, :dS.size] @ dS
    return s


@pytest.mark.parametrize("k,a_at,regime", [(0.05, 1e-4, 0), (0.05, 2e-3, 0), (0.3, 0.01, 1), (0.01, 0.01, 2),
                                           (1.0, 0.5, 1)])
def test_adjoint_step_is_the_transpose_of_the_tangent_step(adj, setup, k, a_at, regime):
    bg, OP, C, keep, nk = setup
    n = OP.n
    rng = np.random.default_rng(int(1e4 * k) + regime)
    tau = float(bg["tau_of_a_spline"].evaluate(np.array([a_at]))[0])
    ts = 0.99 * OP.start_time(k)
    ys, _ = OP.solve([k], ts, OP.ics(ts, k), np.array([tau]), rtol=1e-6, atol=1e-9, max_steps=100000)
    y = ys[0, 0].copy()
    tn, tabs = _random_tangent(bg, C, rng, keep)
    yd = y * rng.standard_normal(n) * 0.3 + 1e-3 * rng.standard_normal(n) * np.abs(y).max()
    lam1 = rng.standard_normal(n)
    y1, yd1, lam0, pbar, tbar = np.zeros(n), np.zeros(n), np.zeros(n), np.zeros(16), np.zeros((8, nk))
    rc = adj.shim_adjoint_step(ctypes.byref(C), ctypes.addressof(tn), k, tau, 0.01 * tau, regime, ptr(y), ptr(yd),
                               ptr(lam1), ptr(y1), ptr(yd1), ptr(lam0), ptr(pbar), ptr(tbar), nk)
    assert rc == 0
    lhs = lam1 @ yd1
    rhs = lam0 @ yd + _pair(tn, tabs, pbar[1:9], tbar)
    assert abs(lhs - rhs) <= 1e-12 * np.abs(lam1 * yd1).sum(), (lhs, rhs)


@pytest.mark.parametrize("k", [2e-3, 0.05, 0.5])
@pytest.mark.parametrize("every", [1, 7])
def test_adjoint_mode_equals_forward_mode_tangent(adj, shim, setup, k, every):
    bg, OP, C, keep, nk = setup
    n = OP.n
    rng = np.random.default_rng(int(1e3 * k) + every)
    aout = np.array([0.05, 0.3, 1.0])
    tout = bg["tau_of_a_spline"].evaluate(aout)
    nout = tout.size
    ts = 0.99 * min(tout.min(), OP.start_time(k))
    y0 = OP.ics(ts, k)
    sw = OP.switch_times(k)
    ctrl = _abi.DiscoebControl(1e-5, 1e-8, 0.25, 0.8, 0.0, 20.0, 0.3, 100000, 0, 0, 0)
    cap = 20000
    tlog = np.zeros(cap)
    ckpt = np.zeros(((cap + every - 1) // every, n))
    y20 = np.zeros((nout, 20))
    st = (ctypes.c_int * 3)()
    assert adj.shim_fwd_record(ctypes.byref(C), ctypes.byref(ctrl), k, ts, ptr(y0), ptr(sw), nout, ptr(tout), cap,
                               every, ptr(tlog), ptr(ckpt), ptr(y20), st) == 0
    nacc = st[2]
    ob = rng.standard_normal((nout, 20)) / (np.abs(y20) + 1e-30)
    y0bar, toutbar, pbar, tbar = np.zeros(n), np.zeros(nout), np.zeros(8), np.zeros((8, nk))
    adj.shim_bwd_mode(ctypes.byref(C), k, ts, ptr(sw), nout, ptr(tout), ptr(tlog), ptr(ckpt), every, nacc, ptr(ob),
                      ptr(y0bar), ptr(toutbar), ptr(pbar), ptr(tbar), nk)
    # forward mode along a random direction of every input
    tn, tabs = _random_tangent(bg, C, rng, keep)
    yd0 = y0 * 0.1 * rng.standard_normal(n)
    tdot = tout * 1e-3 * rng.standard_normal(nout)
    yo, ydo = np.zeros((nout, n)), np.zeros((nout, n))
    stats = (ctypes.c_int * 3)()
    shim.shim_solve_mode_tangent(ctypes.byref(C), ctypes.addressof(tn), ctypes.byref(ctrl), k, ts, ptr(y0), ptr(yd0),
                                 ptr(sw), nout, ptr(tout), ptr(yo), ptr(ydo), stats, None, 0)
    assert stats[0] == 0 and stats[2] == nacc
    lhs = 0.0
    for j in range(nout):
        regime = (1 if C.use_rsa and tout[j] >= sw[0] else (2 if C.use_ufa and tout[j] >= sw[1] else 0))
        f, c0 = np.zeros(n), np.zeros(n)
        shim.shim_rhs(ctypes.byref(C), tout[j], ptr(yo[j]), k, regime, ptr(f), ptr(c0))
        ydm = ydo[j] + f * tdot[j]
        o, od = np.zeros(20), np.zeros(20)
        shim.shim_projected_output_tangent(ctypes.byref(C), ctypes.addressof(tn), k, tout[j], ptr(yo[j]), ptr(ydm),
                                           ptr(o), ptr(od))
        np.testing.assert_allclose(o, y20[j], rtol=1e-13, atol=1e-300)
        lhs += ob[j] @ od
    rhs = y0bar @ yd0 + toutbar @ tdot + _pair(tn, tabs, pbar, tbar)
    assert abs(lhs - rhs) <= 1e-10 * abs(lhs), (lhs, rhs)
