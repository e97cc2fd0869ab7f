"""ctypes driver of the C oracle: TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline legs of ``bench.py``
import this module, and only as the checker / the timed CPU restatement.  It runs
the reference's per-mode algorithm (``evolve_one_mode``, src/discoeb/perturbations.py:882-949,
and the batched ``evolve_modes_batched``, :1002-1120) on the CPU in float64.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import threading
from concurrent.futures import ThreadPoolExecutor

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")
MAX_NQ = 64


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


class Spline(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int), ("uniform", ctypes.c_int),
                ("x", ctypes.POINTER(ctypes.c_double)), ("y", ctypes.POINTER(ctypes.c_double)),
                ("S", ctypes.POINTER(ctypes.c_double))]


class Problem(ctypes.Structure):
    _fields_ = ([(f, ctypes.c_int) for f in ("n", "lmaxg", "lmaxgp", "lmaxr", "lmaxnu", "nqmax",
                                              "use_tca", "use_rsa", "use_ufa")]
                + [(f, ctypes.c_double) for f in ("tca_tau_c_over_tau_h", "tca_tau_c_over_tau_k",
                                                   "rsa_tau_c_over_tau", "rsa_tau_over_tau_k", "ufa_tau_over_tau_k",
                                                   "grhom", "grhog", "grhor", "Omegam", "Omegab", "OmegaDE", "Omegak",
                                                   "Neff", "Nmnu", "amnu", "w0", "wa", "cs2_DE", "YHe", "H0", "taumin",
                                                   "de_guard_eps")]
                + [("q", ctypes.c_double * MAX_NQ), ("w", ctypes.c_double * MAX_NQ)]
                + [(f, Spline) for f in ("xe_loga", "cs2a_loga", "logrhonu_loga", "logpnu_loga",
                                         "a_of_tau", "xe_of_tau", "tau_of_a")])


class Control(ctypes.Structure):
    _fields_ = ([(f, ctypes.c_double) for f in ("rtol", "atol", "pcoeff", "icoeff", "dcoeff", "factormax", "factormin")]
                + [("max_steps", ctypes.c_int), ("linear_interp", ctypes.c_int), ("literal_regime", ctypes.c_int)])


class Stats(ctypes.Structure):
    _fields_ = [("steps", ctypes.c_int), ("accepted", ctypes.c_int), ("rejected", ctypes.c_int), ("status", ctypes.c_int)]


_lib = None
_lock = threading.Lock()
_dp = ctypes.POINTER(ctypes.c_double)


def lib():
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                build()
            L = ctypes.CDLL(LIB_PATH)
            P = ctypes.POINTER(Problem)
            L.oracle_nvar.argtypes = [P]
            L.oracle_rhs.argtypes = [P, ctypes.c_double, _dp, ctypes.c_double, _dp, ctypes.c_int]
            L.oracle_jacobian.argtypes = [P, ctypes.c_double, _dp, ctypes.c_double, _dp, _dp, ctypes.c_int]
            L.oracle_start_time.argtypes = [P, ctypes.c_double]
            L.oracle_start_time.restype = ctypes.c_double
            L.oracle_ics.argtypes = [P, ctypes.c_double, ctypes.c_double, _dp]
            L.oracle_rsa_project.argtypes = [P, ctypes.c_double, ctypes.c_double, _dp, _dp]
            L.oracle_output_vars.argtypes = [P, ctypes.c_double, _dp, _dp]
            L.oracle_switch_times.argtypes = [P, ctypes.c_double, _dp]
            L.oracle_regime.argtypes = [P, ctypes.c_double, _dp]
            L.oracle_solve.argtypes = [P, ctypes.POINTER(Control), ctypes.c_int, _dp, ctypes.c_double, _dp,
                                       ctypes.c_int, _dp, _dp, _dp, ctypes.POINTER(Stats)]
            _lib = L
    return _lib


def _ptr(a):
    return a.ctypes.data_as(_dp)


def _c(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class OracleProblem:
    """Holds an ``OracleProblem`` struct and the arrays it points to."""

    def __init__(self, param, *, lmaxg, lmaxgp, lmaxr, lmaxnu, nqmax, de_guard_eps=0.0):
        from discoeb_b200.background import get_neutrino_momentum_bins
        self.keep = []
        P = Problem()
        P.lmaxg, P.lmaxgp, P.lmaxr, P.lmaxnu, P.nqmax = lmaxg, lmaxgp, lmaxr, lmaxnu, nqmax
        P.n = 7 + (lmaxg + 1) + (lmaxgp + 1) + (lmaxr + 1) + nqmax * (lmaxnu + 1) + 2
        P.use_tca = int(bool(param.get("use_tca", False)))
        P.tca_tau_c_over_tau_h = param.get("tca_tau_c_over_tau_h_trigger", 0.015)
        P.tca_tau_c_over_tau_k = param.get("tca_tau_c_over_tau_k_trigger", 0.010)
        P.use_rsa = int(bool(param.get("use_rsa", True)))
        P.rsa_tau_c_over_tau = param.get("rsa_tau_c_over_tau_trigger", 10.0)
        P.rsa_tau_over_tau_k = param.get("rsa_tau_over_tau_k_trigger", 80.0)
        P.use_ufa = int(bool(param.get("use_ur_fluid", True)))
        P.ufa_tau_over_tau_k = param.get("ur_fluid_tau_over_tau_k_trigger", 120.0)
        for f in ("grhom", "grhog", "grhor", "Omegam", "Omegab", "OmegaDE", "Omegak", "Neff", "Nmnu", "amnu",
                  "cs2_DE", "YHe", "H0", "taumin"):
            setattr(P, f, float(param[f]))
        P.w0 = float(param["w_DE_0"])
        P.wa = float(param["w_DE_a"])
        P.de_guard_eps = de_guard_eps
        q, w = get_neutrino_momentum_bins(nqmax)
        for i in range(nqmax):
            P.q[i] = q[i]
            P.w[i] = w[i]
        for name, key in (("xe_loga", "xe_of_loga_spline"), ("cs2a_loga", "cs2a_of_loga_spline"),
                          ("logrhonu_loga", "logrhonu_of_loga_spline"), ("logpnu_loga", "logpnu_of_loga_spline"),
                          ("a_of_tau", "a_of_tau_spline"), ("xe_of_tau", "xe_of_tau_spline"),
                          ("tau_of_a", "tau_of_a_spline")):
            s = param[key]
            x, y, S = _c(s.x), _c(s.y), _c(s.S)
            self.keep += [x, y, S]
            setattr(P, name, Spline(s.n, int(s.uniform), _ptr(x), _ptr(y), _ptr(S)))
        self.P = P
        self.n = P.n
        self.param = param

    @property
    def ref(self):
        return ctypes.byref(self.P)

    def rhs(self, tau, y, k, regime=-1):
        y = _c(y)
        f = np.zeros(self.n)
        lib().oracle_rhs(self.ref, tau, _ptr(y), k, _ptr(f), regime)
        return f

    def jacobian(self, tau, y, k, regime=-1):
        y = _c(y)
        J = np.zeros((self.n, self.n))
        dT = np.zeros(self.n)
        lib().oracle_jacobian(self.ref, tau, _ptr(y), k, _ptr(J), _ptr(dT), regime)
        return J, dT

    def start_time(self, k):
        return lib().oracle_start_time(self.ref, float(k))

    def ics(self, tau, k):
        y = np.zeros(self.n)
        lib().oracle_ics(self.ref, float(tau), float(k), _ptr(y))
        return y

    def switch_times(self, k):
        sw = np.zeros(3)
        lib().oracle_switch_times(self.ref, float(k), _ptr(sw))
        return sw

    def rsa_project(self, tau, k, y):
        y = _c(y)
        o = np.zeros(self.n)
        lib().oracle_rsa_project(self.ref, float(tau), float(k), _ptr(y), _ptr(o))
        return o

    def output_vars(self, k, y):
        y = _c(y)
        o = np.zeros(20)
        lib().oracle_output_vars(self.ref, float(k), _ptr(y), _ptr(o))
        return o

    def solve(self, ks, t0, y0, tout, *, rtol, atol, pcoeff=0.25, icoeff=0.80, dcoeff=0.0, factormax=20.0,
              factormin=0.3, max_steps=2048, linear_interp=False, literal_regime=False, sw=None):
        ks = _c(np.atleast_1d(ks))
        nb = ks.shape[0]
        y0 = _c(y0).reshape(nb, self.n)
        tout = _c(np.atleast_1d(tout))
        if sw is None:
            sw = np.array([self.switch_times(k) for k in ks])
        sw = _c(sw).reshape(nb, 3)
        C = Control(rtol, atol, pcoeff, icoeff, dcoeff, factormax, factormin, int(max_steps),
                    int(linear_interp), int(literal_regime))
        yout = np.zeros((nb, tout.shape[0], self.n))
        st = Stats()
        lib().oracle_solve(self.ref, ctypes.byref(C), nb, _ptr(ks), float(t0), _ptr(y0), tout.shape[0], _ptr(tout),
                           _ptr(sw), _ptr(yout), ctypes.byref(st))
        return yout, st


def k_sampling(param, kmin, kmax, num_k, method):
    """k grid of evolve_perturbations (src/discoeb/perturbations.py:1177-1199)."""
    if method == "log":
        return np.geomspace(kmin, kmax, num_k)
    if method == "linear":
        return np.linspace(kmin, kmax, num_k)
    if method == "camb":
        taurst = param["tau_maxvis"]
        q1, q2 = 8.0 / taurst, 30.0 / taurst
        n1, n2 = int(num_k * 0.2), int(num_k * 0.4)
        n3 = num_k - n1 - n2
        return np.concatenate([np.geomspace(kmin, q1, n1, endpoint=False), np.linspace(q1, q2, n2, endpoint=False),
                               np.geomspace(q2, kmax, n3)])
    raise ValueError(f"Unknown k_sampling_method: {method}")


def evolve_perturbations(*, param, aexp_out, kmin, kmax, num_k, lmaxg=11, lmaxgp=11, lmaxr=11, lmaxnu=8, nqmax=3,
                         rtol=1e-4, atol=1e-4, pcoeff=0.25, icoeff=0.80, dcoeff=0.0, factormax=20.0, factormin=0.3,
                         max_steps=2048, return_full=False, k_sampling_method="camb", mode="clip",
                         de_guard_eps=0.0, threads=None, kmodes=None, batch_size=None):
    """Oracle forward solve with the reference's call surface.

    mode='reference': diffrax semantics (linear interpolation to tau_out, switches
    evaluated per RHS call), per mode or batched (``batch_size``) like the reference.
    mode='clip': steps end exactly on every tau_out and approximation switch time and
    the switches hold per step (the semantics the device kernels implement).
    Returns (y, kmodes, stats) with y[num_k, nout, 20] or [num_k, nout, n] (return_full).
    """
    OP = OracleProblem(param, lmaxg=lmaxg, lmaxgp=lmaxgp, lmaxr=lmaxr, lmaxnu=lmaxnu, nqmax=nqmax,
                       de_guard_eps=de_guard_eps)
    if kmodes is None:
        kmodes = k_sampling(param, kmin, kmax, num_k, k_sampling_method)
    kmodes = np.asarray(kmodes, dtype=np.float64)
    aexp_out = np.atleast_1d(np.asarray(aexp_out, dtype=np.float64))
    tau_out = param["tau_of_a_spline"].evaluate(aexp_out)
    nout = tau_out.shape[0]
    literal = mode == "reference"
    kw = dict(rtol=rtol, atol=atol, pcoeff=pcoeff, icoeff=icoeff, dcoeff=dcoeff, factormax=factormax,
              factormin=factormin, max_steps=max_steps, linear_interp=literal, literal_regime=literal)
    groups = ([np.arange(i, i + batch_size) for i in range(0, len(kmodes), batch_size)] if batch_size
              else [np.array([i]) for i in range(len(kmodes))])

    def run(idx):
        ks = kmodes[idx]
        ts = np.array([0.99 * min(tau_out.min(), OP.start_time(k)) for k in ks])
        t0 = ts.min()
        y0 = np.stack([OP.ics(t0, k) for k in ks])
        ys, st = OP.solve(ks, t0, y0, tau_out, **kw)
        return idx, ys, st

    nthreads = threads or os.cpu_count() or 1
    ys_all = np.zeros((len(kmodes), nout, OP.n))
    stats = [None] * len(groups)
    with ThreadPoolExecutor(max_workers=nthreads) as ex:
        for gi, (idx, ys, st) in enumerate(ex.map(run, groups)):
            ys_all[idx] = ys
            stats[gi] = (st.steps, st.accepted, st.rejected, st.status)
    proj = np.zeros_like(ys_all)
    for i, k in enumerate(kmodes):
        for j in range(nout):
            proj[i, j] = OP.rsa_project(tau_out[j], k, ys_all[i, j])
    if return_full:
        return proj, kmodes, stats
    out = np.zeros((len(kmodes), nout, 20))
    for i, k in enumerate(kmodes):
        for j in range(nout):
            out[i, j] = OP.output_vars(k, proj[i, j])
    return out, kmodes, stats


def output_fields_fixed(param, kmodes, aexp_out, tau_start, switch_tau, *, lmaxg, lmaxgp, lmaxr, lmaxnu, nqmax, rtol,
                        atol, max_steps=400000, de_guard_eps=1e-9, threads=None):
    """Output fields [K, nout, 20] of the clip-mode solve with the start times ``tau_start`` [K] and
    approximation switch times ``switch_tau`` [K, 3] given (held at a base point's values when the
    parameters move, the convention of forward-mode AD through the reference), and status [K]."""
    OP = OracleProblem(param, lmaxg=lmaxg, lmaxgp=lmaxgp, lmaxr=lmaxr, lmaxnu=lmaxnu, nqmax=nqmax,
                       de_guard_eps=de_guard_eps)
    kmodes = np.asarray(kmodes, dtype=np.float64)
    tau_out = param["tau_of_a_spline"].evaluate(np.atleast_1d(np.asarray(aexp_out, dtype=np.float64)))
    nout = tau_out.shape[0]

    def run(i):
        k, t0 = float(kmodes[i]), float(tau_start[i])
        ys, st = OP.solve([k], t0, OP.ics(t0, k), tau_out, rtol=rtol, atol=atol, max_steps=max_steps,
                          sw=np.asarray(switch_tau[i], dtype=np.float64))
        out = np.array([OP.output_vars(k, OP.rsa_project(tau_out[j], k, ys[0, j])) for j in range(nout)])
        return i, out, st.status

    out = np.zeros((kmodes.shape[0], nout, 20))
    status = np.zeros(kmodes.shape[0], dtype=np.int32)
    with ThreadPoolExecutor(max_workers=threads or os.cpu_count() or 1) as ex:
        for i, o, s in ex.map(run, range(kmodes.shape[0])):
            out[i], status[i] = o, s
    return out, status
