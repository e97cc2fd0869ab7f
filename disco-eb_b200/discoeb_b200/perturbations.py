"""Linear perturbations: the reference's call surface over the sm_100a solver.

Mirrors ``src/discoeb/perturbations.py`` of the reference:

* ``evolve_perturbations`` / ``evolve_perturbations_batched`` (perturbations.py:1124-1337)
  take the same keyword arguments and return ``(y, kmodes, param)`` with
  ``y[num_k, nout, 20]`` output fields (or ``[num_k, nout, nvar]`` with ``return_full``).
* ``get_power`` (perturbations.py:1446-1468) and ``compute_time_derivatives``
  (perturbations.py:1339-1406).

The host computes the k grid, the output times, the start times and the adiabatic
initial conditions (vectorised numpy restatements of perturbations.py:680-835), then one
call of the C ABI ``discoeb_fwd`` integrates every mode on the GPU.  Inputs and outputs
are numpy arrays (``torch`` tensors on a CUDA device are accepted for ``aexp_out``); the
GPU is required - there is no CPU path.

Documented differences from the reference (all within the solver tolerance):
steps end exactly on the output times (the reference interpolates linearly between
accepted steps, so its intermediate outputs carry O(h^2) error) and on the times where
the radiation-streaming / ultra-relativistic-fluid approximations switch on; each mode
chooses its own step sizes (``batch_size`` is accepted for call compatibility).
At w = -1 exactly the reference's dark-energy fluid equations divide by 1 + w = 0
(NaN); ``de_guard_eps`` (default 1e-9) holds the dark-energy perturbations fixed where
|1 + w| < de_guard_eps, which is the cosmological-constant limit.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np

from . import _abi
from .background import get_aprimeoa, get_neutrino_momentum_bins

AKTHOM_RHS = 2.3038921003709498e-9
AKTHOM_START = 2.3048e-9  # the start-time criterion uses this rounder constant (perturbations.py:802)


def nvar_of(lmaxg, lmaxgp, lmaxr, lmaxnu, nqmax):
    return 7 + (lmaxg + 1) + (lmaxgp + 1) + (lmaxr + 1) + nqmax * (lmaxnu + 1) + 2


def k_sampling(param, kmin, kmax, num_k, k_sampling_method):
    """k grid (perturbations.py:1177-1199)."""
    if k_sampling_method == "log":
        return np.geomspace(kmin, kmax, num_k)
    if k_sampling_method == "linear":
        return np.linspace(kmin, kmax, num_k)
    if k_sampling_method == "camb":
        if "tau_maxvis" not in param:
            raise ValueError("param dictionary must contain 'tau_maxvis' for 'camb' k-sampling.")
        taurst = param["tau_maxvis"]
        q1, q2 = 8.0 / taurst, 30.0 / taurst
        n1, n2 = int(num_k * 0.2), int(num_k * 0.4)
        n3 = num_k - n1 - n2
        return np.concatenate([np.geomspace(kmin, q1, n1, endpoint=False), np.linspace(q1, q2, n2, endpoint=False),
                               np.geomspace(q2, kmax, n3)])
    raise ValueError(f"Unknown k_sampling_method: {k_sampling_method}")


def determine_starting_time(*, param, k):
    """CLASS-style start time, vectorised over k (perturbations.py:784-835, util.py:249-280)."""
    k = np.atleast_1d(np.asarray(k, dtype=np.float64))
    x0 = math.log(param["taumin"])
    x1 = math.log(float(param["tau_of_a_spline"].evaluate(0.1)))

    def tau_H(logtau):
        a = param["a_of_tau_spline"].evaluate(np.exp(logtau))
        return 1.0 / get_aprimeoa(param=param, aexp=a)

    def cond_large(logtau):
        return tau_H(logtau) * k / 0.07 - 1.0

    def cond_small(logtau):
        tau = np.exp(logtau)
        akthom = AKTHOM_START * (1.0 - param["YHe"]) * param["Omegab"] * param["H0"] ** 2
        xe = param["xe_of_tau_spline"].evaluate(tau)
        a = param["a_of_tau_spline"].evaluate(tau)
        opac = xe * akthom / a**2
        return (1.0 / opac) / tau_H(logtau) / 0.0004 - 1.0

    def bisect(func, shape):
        left = np.full(shape, x0)
        right = np.full(shape, x1)
        for _ in range(7):
            mid = 0.5 * (left + right)
            same = func(mid) * func(left) > 0
            left = np.where(same, mid, left)
            right = np.where(same, right, mid)
        return 0.5 * (left + right)

    lt_large = bisect(cond_large, k.shape)
    lt_small = bisect(cond_small, ())
    return np.exp(np.minimum(lt_small, lt_large))


def adiabatic_ics(*, tau, param, kmode, lmaxg, lmaxgp, lmaxr, lmaxnu, nqmax):
    """Adiabatic initial conditions for many modes (perturbations.py:680-781).

    ``tau`` and ``kmode`` broadcast; returns ``y[len, nvar]``.
    """
    tau = np.atleast_1d(np.asarray(tau, dtype=np.float64))
    k = np.atleast_1d(np.asarray(kmode, dtype=np.float64))
    tau, k = np.broadcast_arrays(tau, k)
    n = nvar_of(lmaxg, lmaxgp, lmaxr, lmaxnu, nqmax)
    iq0 = 10 + lmaxg + lmaxgp + lmaxr
    a = param["a_of_tau_spline"].evaluate(tau)
    y = np.zeros(tau.shape + (n,), dtype=np.result_type(a.dtype, np.asarray(param["grhom"]).dtype, np.float64))
    rhonu_bg = np.exp(param["logrhonu_of_loga_spline"].evaluate(np.log(a)))
    rhom = param["grhom"] * param["Omegam"] / a**3
    rhor = (param["grhog"] + param["grhor"] * (param["Neff"] + param["Nmnu"] * rhonu_bg)) / a**4
    rhonu = param["grhor"] * (param["Neff"] + param["Nmnu"] * rhonu_bg) / a**4
    fracb = param["Omegab"] / param["Omegam"]
    fracnu = rhonu / rhor
    om = a * rhom / np.sqrt(rhor)
    ci, s2 = -1.0, 1.0
    kt = k * tau
    deltag = -(kt**2) / 3 * (1 - om * tau / 5) * ci * s2
    thetag = -(kt**3) / tau / 36 * (1 - 3 * (1 + 5 * fracb - fracnu) / 20 / (1 - fracnu) * om * tau) * ci * s2
    deltar = deltag
    thetar = (-(kt**4) / tau / 36 / (4 * fracnu + 15)
              * (4 * fracnu + 11 + 12 - 3 * (8 * fracnu**2 + 50 * fracnu + 275) / 20 / (2 * fracnu + 15) * tau * om) * ci)
    shearr = kt**2 / (45 + 12 * fracnu) * (3 * s2 - 1) * (1 + (4 * fracnu - 5) / 4 / (2 * fracnu + 15) * tau * om) * ci
    cs2_Q = param["cs2_DE"]
    w_Q = param["w_DE_0"] + param["w_DE_a"] * (1.0 - a)
    deltaq = kt**2 / 4 * (1 + w_Q) * (4 - 3 * cs2_Q) / (4 - 6 * w_Q + 3 * cs2_Q) * ci * s2
    thetaq = kt**4 / tau / 4 * cs2_Q / (4 - 6 * w_Q + 3 * cs2_Q) * ci * s2
    eta = ci * (1 - kt**2 / 12 / (15 + 4 * fracnu)
                * (5 + 4 * s2 * fracnu - (16 * fracnu**2 + 280 * fracnu + 325) / 10 / (2 * fracnu + 15) * tau * om))
    y[..., 0] = a
    y[..., 2] = eta
    y[..., 3] = 0.75 * deltag
    y[..., 5] = 0.75 * deltag
    y[..., 6] = thetag
    y[..., 7] = deltag
    y[..., 8] = thetag
    y[..., 9 + lmaxg + lmaxgp] = deltar
    y[..., 10 + lmaxg + lmaxgp] = thetar
    y[..., 11 + lmaxg + lmaxgp] = shearr * 2.0
    q, _ = get_neutrino_momentum_bins(nqmax)
    aq = a[..., None] * param["amnu"] / q
    v = 1 / np.sqrt(1 + aq**2)
    dlfdlq = -q / (1.0 + np.exp(-q))
    y[..., iq0:iq0 + nqmax] = -0.25 * dlfdlq * deltar[..., None]
    y[..., iq0 + nqmax:iq0 + 2 * nqmax] = -dlfdlq * thetar[..., None] / v / k[..., None] / 3.0
    y[..., iq0 + 2 * nqmax:iq0 + 3 * nqmax] = -0.5 * dlfdlq * shearr[..., None]
    y[..., -2] = deltaq
    y[..., -1] = thetaq
    return y


def _tauc_over_tau_crossing(param, trigger):
    """First tau where tau_c(a(tau))/tau exceeds ``trigger`` (monotone in tau), by bisection."""
    akthom = AKTHOM_RHS * (1.0 - param["YHe"]) * param["Omegab"] * param["H0"] ** 2
    spl = param["a_of_tau_spline"]
    lo, hi = math.log(spl.x[0]), math.log(spl.x[-1])

    def g(lt):
        tau = math.exp(lt)
        a = float(spl.evaluate(tau))
        xe = float(param["xe_of_loga_spline"].evaluate(math.log(a)))
        opac = xe * akthom / a**2
        return 1.0 / max(opac, 1e-30) / tau - trigger

    if g(lo) > 0:
        return math.exp(lo)
    if g(hi) <= 0:
        return math.inf
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if g(mid) > 0:
            hi = mid
        else:
            lo = mid
        if hi - lo < 1e-15:
            break
    return math.exp(hi)


def approximation_switch_times(param, kmodes):
    """``[K, 3]`` times where RSA starts, the UR-fluid approximation starts and TCA ends.

    The triggers (approximations.py:50-75) depend on (tau, k, tau_c) only; tau_c/tau
    grows monotonically, so each switch happens once.  The solver ends a step exactly
    there and holds the regime fixed inside each step.
    """
    s = _abi.approximation_settings(param)
    k = np.asarray(kmodes, dtype=np.float64)
    sw = np.full((k.shape[0], 3), np.inf)
    if s["use_rsa"]:
        tc = _tauc_over_tau_crossing(param, s["tau_c_over_tau_trigger"])
        sw[:, 0] = np.maximum(tc, s["tau_over_tau_k_trigger"] / k)
    if s["use_ur_fluid"]:
        sw[:, 1] = s["ur_fluid_tau_over_tau_k_trigger"] / k
    if s["use_tca"]:
        raise NotImplementedError("use_tca=True is not supported by the GPU solver (the reference default is False)")
    return sw


class DeviceCosmo:
    """Device copies of one cosmology's tables plus its ``DiscoebCosmo`` struct."""

    def __init__(self, param, *, lmaxg, lmaxgp, lmaxr, lmaxnu, nqmax, de_guard_eps, device):
        import torch
        self.tensors = []
        ptrs = {}
        for key in ("xe_of_loga_spline", "cs2a_of_loga_spline", "logrhonu_of_loga_spline", "logpnu_of_loga_spline"):
            s = param[key]
            t = torch.from_numpy(np.ascontiguousarray(s.table())).to(device, non_blocking=True)
            self.tensors.append(t)
            base = t.data_ptr()
            ptrs[key] = (s.n, int(s.uniform), base, base + 8 * s.n, base + 16 * s.n)
        xe, cs = param["xe_of_loga_spline"], param["cs2a_of_loga_spline"]
        if xe.n == cs.n and np.array_equal(xe.x, cs.x):
            n_, u_, _, yp, sp = ptrs["cs2a_of_loga_spline"]
            ptrs["cs2a_of_loga_spline"] = (n_, u_, ptrs["xe_of_loga_spline"][2], yp, sp)
        rn, rp = param["logrhonu_of_loga_spline"], param["logpnu_of_loga_spline"]
        if rn.n == rp.n and np.array_equal(rn.x, rp.x):
            n_, u_, _, yp, sp = ptrs["logpnu_of_loga_spline"]
            ptrs["logpnu_of_loga_spline"] = (n_, u_, ptrs["logrhonu_of_loga_spline"][2], yp, sp)
        self.host = _abi.make_cosmo(param, lmaxg=lmaxg, lmaxgp=lmaxgp, lmaxr=lmaxr, lmaxnu=lmaxnu, nqmax=nqmax,
                                    de_guard_eps=de_guard_eps, table_ptrs=ptrs)
        raw = bytes(ctypes.string_at(ctypes.addressof(self.host), ctypes.sizeof(self.host)))
        self.struct = torch.frombuffer(bytearray(raw), dtype=torch.uint8).to(device, non_blocking=True)


def _check_status(status, nsteps, kmodes, on_failure):
    bad = np.nonzero(status != 0)[0]
    if bad.size and on_failure == "raise":
        i = bad[0]
        raise RuntimeError(f"{bad.size} k-mode(s) failed; first: k={kmodes[i]:.6g} status="
                           f"{_abi.STATUS_NAMES.get(int(status[i]), status[i])} after {nsteps[i]} steps "
                           "(increase max_steps or loosen rtol/atol)")


def solve_modes(*, param, kmodes, tau_out, lmaxg, lmaxgp, lmaxr, lmaxnu, nqmax, rtol, atol, pcoeff, icoeff, dcoeff,
                factormax, factormin, max_steps, return_full, de_guard_eps=1e-9, device=None, warps_per_block=0,
                on_failure="raise", sort_modes=True, return_stats=False, tau_start=None, switch_tau=None,
                as_tensor=False, method="structured"):
    """Integrate the given modes of one cosmology to ``tau_out`` on the GPU.

    Returns numpy ``y`` (``[K, nout, 20]`` or ``[K, nout, nvar]``); with
    ``return_stats`` also ``(status, nsteps)``.  ``tau_start`` [K] and ``switch_tau`` [K, 3]
    override the start times and approximation switch times derived from ``param`` (to hold
    these numerical choices fixed while parameters move, as forward-mode AD does).
    ``as_tensor``: return ``y`` as a device tensor (the caller's mode order) instead of numpy.
    ``method``: "structured" (FP64 chain factors) or "structured-mixed" (FP32 chain factors, one
    FP64 residual refinement of every chain solve).
    """
    methods = {"structured": _abi.METHOD_RODAS5_STRUCTURED, "structured-mixed": _abi.METHOD_RODAS5_STRUCTURED_MIXED}
    if method not in methods:
        raise ValueError(f"method must be one of {sorted(methods)}, not {method!r}")
    import torch
    if device is None:
        if not torch.cuda.is_available():
            raise RuntimeError("discoeb_b200 needs a CUDA device (there is no CPU path)")
        device = torch.device("cuda", torch.cuda.current_device())
    L = _abi.lib()
    kmodes = np.ascontiguousarray(kmodes, dtype=np.float64)
    tau_out = np.ascontiguousarray(np.atleast_1d(tau_out), dtype=np.float64)
    if np.any(np.diff(tau_out) <= 0):
        raise ValueError("aexp_out must map to strictly increasing output times")
    K = kmodes.shape[0]
    n = nvar_of(lmaxg, lmaxgp, lmaxr, lmaxnu, nqmax)
    nout = tau_out.shape[0]
    if tau_start is None:
        tau_s = determine_starting_time(param=param, k=kmodes)
        tau_start = 0.99 * np.minimum(tau_out.min(), tau_s)
    tau_start = np.ascontiguousarray(tau_start, dtype=np.float64)
    y0 = adiabatic_ics(tau=tau_start, param=param, kmode=kmodes, lmaxg=lmaxg, lmaxgp=lmaxgp, lmaxr=lmaxr,
                       lmaxnu=lmaxnu, nqmax=nqmax)
    sw = approximation_switch_times(param, kmodes) if switch_tau is None else \
        np.ascontiguousarray(switch_tau, dtype=np.float64)
    # longest modes (largest k) first so that the tail of the launch is short
    order = np.argsort(-kmodes, kind="stable") if sort_modes else np.arange(K)
    dc = DeviceCosmo(param, lmaxg=lmaxg, lmaxgp=lmaxgp, lmaxr=lmaxr, lmaxnu=lmaxnu, nqmax=nqmax,
                     de_guard_eps=de_guard_eps, device=device)
    f64 = dict(dtype=torch.float64, device=device)
    pin = dict(pin_memory=True)
    host_in = torch.from_numpy(np.concatenate([kmodes[order], tau_start[order], y0[order].ravel(),
                                               sw[order].ravel(), tau_out]))
    d_in = host_in.pin_memory().to(device, non_blocking=True) if pin else host_in.to(device)
    off = 0
    d_k = d_in[off:off + K]; off += K
    d_ts = d_in[off:off + K]; off += K
    d_y0 = d_in[off:off + K * n]; off += K * n
    d_sw = d_in[off:off + 3 * K]; off += 3 * K
    d_tout = d_in[off:off + nout]
    d_full = torch.empty((K, nout, n), **f64) if return_full else None
    d_out20 = None if return_full else torch.empty((K, nout, 20), **f64)
    d_stat = torch.empty((2, K), dtype=torch.int32, device=device)
    ctrl = _abi.DiscoebControl(rtol, atol, pcoeff, icoeff, dcoeff, factormax, factormin, int(max_steps),
                               methods[method], int(warps_per_block), 0)
    stream = torch.cuda.current_stream(device).cuda_stream
    rc = L.discoeb_fwd(dc.struct.data_ptr(), ctypes.byref(dc.host), 1, ctypes.byref(ctrl), K, None,
                       d_k.data_ptr(), d_ts.data_ptr(), d_y0.data_ptr(), d_sw.data_ptr(), nout, d_tout.data_ptr(),
                       d_full.data_ptr() if d_full is not None else None,
                       d_out20.data_ptr() if d_out20 is not None else None,
                       d_stat[0].data_ptr(), d_stat[1].data_ptr(), stream)
    if rc != 0:
        raise RuntimeError(f"discoeb_fwd failed with code {rc}")
    out_dev = d_full if return_full else d_out20
    inv = np.empty_like(order)
    inv[order] = np.arange(K)
    if as_tensor:
        y = out_dev.index_select(0, torch.from_numpy(inv).to(device))
    else:
        y = out_dev.cpu().numpy()[inv]
    stat = d_stat.cpu().numpy()
    status, nsteps = stat[0][inv], stat[1][inv]
    _check_status(status, nsteps, kmodes, on_failure)
    if return_stats:
        return y, status, nsteps
    return y


def _finish(param, y, kmodes, lmaxg, lmaxgp, lmaxr, lmaxnu, nqmax, nout, tau_out):
    param["lmaxg"] = lmaxg
    param["lmaxgp"] = lmaxgp
    param["lmaxr"] = lmaxr
    param["lmaxnu"] = lmaxnu
    param["nqmax"] = nqmax
    param["nout"] = nout
    param["tau_out"] = tau_out
    return y, kmodes, param


def evolve_perturbations(*, param, aexp_out, kmin: float, kmax: float, num_k: int, lmaxg: int = 11, lmaxgp: int = 11,
                         lmaxr: int = 11, lmaxnu: int = 8, nqmax: int = 3, rtol: float = 1e-4, atol: float = 1e-4,
                         pcoeff: float = 0.25, icoeff: float = 0.80, dcoeff: float = 0.0, factormax: float = 20.0,
                         factormin: float = 0.3, max_steps: int = 2048, return_full: bool = False,
                         k_sampling_method: str = "camb", **solver_options):
    """Evolve cosmological perturbations in the synchronous gauge (perturbations.py:1124-1226).

    Returns ``(y, kmodes, param)``; ``param`` gains lmaxg, lmaxgp, lmaxr, lmaxnu, nqmax,
    nout and tau_out as in the reference.
    """
    kmodes = k_sampling(param, kmin, kmax, num_k, k_sampling_method)
    aexp_out = np.atleast_1d(np.asarray(aexp_out, dtype=np.float64))
    tau_out = param["tau_of_a_spline"].evaluate(aexp_out)
    y = solve_modes(param=param, kmodes=kmodes, tau_out=tau_out, lmaxg=lmaxg, lmaxgp=lmaxgp, lmaxr=lmaxr,
                    lmaxnu=lmaxnu, nqmax=nqmax, rtol=rtol, atol=atol, pcoeff=pcoeff, icoeff=icoeff, dcoeff=dcoeff,
                    factormax=factormax, factormin=factormin, max_steps=max_steps, return_full=return_full,
                    **solver_options)
    return _finish(param, y, kmodes, lmaxg, lmaxgp, lmaxr, lmaxnu, nqmax, aexp_out.shape[0], tau_out)


def evolve_perturbations_batched(*, param, aexp_out, kmin: float, kmax: float, num_k: int, lmaxg: int = 11,
                                 lmaxgp: int = 11, lmaxr: int = 11, lmaxnu: int = 8, nqmax: int = 3,
                                 rtol: float = 1e-4, atol: float = 1e-4, pcoeff: float = 0.25, icoeff: float = 0.80,
                                 dcoeff: float = 0.0, factormax: float = 20.0, factormin: float = 0.3,
                                 max_steps: int = 2048, batch_size: int = 16, return_full: bool = False,
                                 k_sampling_method: str = "camb", **solver_options):
    """Batched variant (perturbations.py:1229-1337).  The reference shares one step size
    across each group of ``batch_size`` modes; here every mode of every group runs in the
    same launch with its own step size, which is never less accurate.  ``num_k`` must be
    divisible by ``batch_size`` as in the reference."""
    if num_k % batch_size != 0:
        raise ValueError(f"num_k={num_k} must be divisible by batch_size={batch_size}")
    return evolve_perturbations(param=param, aexp_out=aexp_out, kmin=kmin, kmax=kmax, num_k=num_k, lmaxg=lmaxg,
                                lmaxgp=lmaxgp, lmaxr=lmaxr, lmaxnu=lmaxnu, nqmax=nqmax, rtol=rtol, atol=atol,
                                pcoeff=pcoeff, icoeff=icoeff, dcoeff=dcoeff, factormax=factormax,
                                factormin=factormin, max_steps=max_steps, return_full=return_full,
                                k_sampling_method=k_sampling_method, **solver_options)


def get_power(*, k, y, idx: int, param):
    """P(k) = 2 pi^2 A_s (k/k_p)^(n_s-1) k^-3 y[..., idx]^2 (perturbations.py:1446-1468)."""
    return 2 * np.pi**2 * param["A_s"] * (k / param["k_p"]) ** (param["n_s"] - 1) * k ** (-3) * y[..., idx] ** 2


def compute_time_derivatives(yout, tau, kmodes, param, lmaxg, lmaxgp, lmaxr, lmaxnu, nqmax, *, de_guard_eps=1e-9,
                             device=None):
    """dy/dtau of states ``yout[K, T, nvar]`` at times ``tau[T]`` (perturbations.py:1339-1406),
    evaluated on the GPU with the approximation switches taken from (tau, a) as the
    reference does."""
    import torch
    if device is None:
        device = torch.device("cuda", torch.cuda.current_device())
    L = _abi.lib()
    yout = np.ascontiguousarray(yout, dtype=np.float64)
    K, T, n = yout.shape
    dc = DeviceCosmo(param, lmaxg=lmaxg, lmaxgp=lmaxgp, lmaxr=lmaxr, lmaxnu=lmaxnu, nqmax=nqmax,
                     de_guard_eps=de_guard_eps, device=device)
    taus = np.broadcast_to(np.asarray(tau, dtype=np.float64)[None, :], (K, T)).ravel().copy()
    ks = np.broadcast_to(np.asarray(kmodes, dtype=np.float64)[:, None], (K, T)).ravel().copy()
    d_y = torch.from_numpy(yout.reshape(K * T, n)).to(device)
    d_tau = torch.from_numpy(taus).to(device)
    d_k = torch.from_numpy(ks).to(device)
    d_f = torch.empty_like(d_y)
    stream = torch.cuda.current_stream(device).cuda_stream
    rc = L.discoeb_rhs(dc.struct.data_ptr(), ctypes.byref(dc.host), K * T, d_tau.data_ptr(), d_k.data_ptr(),
                       d_y.data_ptr(), -1, d_f.data_ptr(), stream)
    if rc != 0:
        raise RuntimeError(f"discoeb_rhs failed with code {rc}")
    return d_f.cpu().numpy().reshape(K, T, n)


class CosmologyBatch:
    """Device-resident inputs of one discoeb_fwd launch over several cosmologies (the prologue of
    solve_cosmologies); ``launch`` enqueues the kernel, ``result`` reads it back."""

    def __init__(self, *, params, kmodes, aexp_out, lmaxg, lmaxgp, lmaxr, lmaxnu, nqmax, rtol, atol, pcoeff=0.25,
                 icoeff=0.80, dcoeff=0.0, factormax=20.0, factormin=0.3, max_steps=100000, return_full=False,
                 de_guard_eps=1e-9, device=None, warps_per_block=0):
        import torch
        if device is None:
            if not torch.cuda.is_available():
                raise RuntimeError("discoeb_b200 needs a CUDA device (there is no CPU path)")
            device = torch.device("cuda", torch.cuda.current_device())
        self.torch, self.device, self.lib = torch, device, _abi.lib()
        C = len(params)
        if C < 1:
            raise ValueError("params must hold at least one cosmology")
        aexp_out = np.atleast_1d(np.asarray(aexp_out, dtype=np.float64))
        km = np.asarray(kmodes, dtype=np.float64)
        km = np.broadcast_to(km, (C, km.shape[-1])) if km.ndim == 1 else km
        K, nout, n = km.shape[1], aexp_out.shape[0], nvar_of(lmaxg, lmaxgp, lmaxr, lmaxnu, nqmax)
        L = dict(lmaxg=lmaxg, lmaxgp=lmaxgp, lmaxr=lmaxr, lmaxnu=lmaxnu, nqmax=nqmax)
        touts, ts, y0s, sws, self.dcs = [], [], [], [], []
        for c, p in enumerate(params):
            tout = p["tau_of_a_spline"].evaluate(aexp_out)
            if np.any(np.diff(tout) <= 0):
                raise ValueError("aexp_out must map to strictly increasing output times")
            t0 = 0.99 * np.minimum(tout.min(), determine_starting_time(param=p, k=km[c]))
            touts.append(tout)
            ts.append(t0)
            y0s.append(adiabatic_ics(tau=t0, param=p, kmode=km[c], **L))
            sws.append(approximation_switch_times(p, km[c]))
            self.dcs.append(DeviceCosmo(p, de_guard_eps=de_guard_eps, device=device, **L))
        self.C, self.K, self.nout, self.n, self.return_full = C, K, nout, n, return_full
        self.flat_k = km.reshape(-1)
        cidx = np.repeat(np.arange(C, dtype=np.int32), K)
        order = np.argsort(-self.flat_k, kind="stable")  # longest modes first across all cosmologies
        self.inv = np.empty_like(order)
        self.inv[order] = np.arange(C * K)
        raw = b"".join(bytes(ctypes.string_at(ctypes.addressof(d.host), ctypes.sizeof(d.host))) for d in self.dcs)
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(device)  # noqa: E731
        self.d_cosmos = torch.frombuffer(bytearray(raw), dtype=torch.uint8).to(device)
        self.d_k, self.d_mc = t(self.flat_k[order]), t(cidx[order])
        self.d_ts, self.d_y0 = t(np.concatenate(ts)[order]), t(np.concatenate(y0s)[order])
        self.d_sw, self.d_tout = t(np.concatenate(sws)[order]), t(np.stack(touts))
        f64 = dict(dtype=torch.float64, device=device)
        M = C * K
        self.d_full = torch.empty((M, nout, n), **f64) if return_full else None
        self.d_out20 = None if return_full else torch.empty((M, nout, 20), **f64)
        self.d_stat = torch.empty((2, M), dtype=torch.int32, device=device)
        self.ctrl = _abi.DiscoebControl(rtol, atol, pcoeff, icoeff, dcoeff, factormax, factormin, int(max_steps),
                                        _abi.METHOD_RODAS5_STRUCTURED, int(warps_per_block), 0)
        self.h2d_bytes = sum(x.numel() * x.element_size() for x in (self.d_cosmos, self.d_k, self.d_mc, self.d_ts,
                                                                   self.d_y0, self.d_sw, self.d_tout))
        self.h2d_bytes += sum(sum(x.numel() * 8 for x in d.tensors) for d in self.dcs)

    def launch(self):
        f = self.d_full, self.d_out20
        rc = self.lib.discoeb_fwd(self.d_cosmos.data_ptr(), ctypes.byref(self.dcs[0].host), self.C,
                                  ctypes.byref(self.ctrl), self.C * self.K, self.d_mc.data_ptr(), self.d_k.data_ptr(),
                                  self.d_ts.data_ptr(), self.d_y0.data_ptr(), self.d_sw.data_ptr(), self.nout,
                                  self.d_tout.data_ptr(), f[0].data_ptr() if f[0] is not None else None,
                                  f[1].data_ptr() if f[1] is not None else None, self.d_stat[0].data_ptr(),
                                  self.d_stat[1].data_ptr(), self.torch.cuda.current_stream(self.device).cuda_stream)
        if rc != 0:
            raise RuntimeError(f"discoeb_fwd failed with code {rc}")

    def result(self, on_failure="raise"):
        out = (self.d_full if self.return_full else self.d_out20).cpu().numpy()[self.inv]
        stat = self.d_stat.cpu().numpy()[:, self.inv]
        _check_status(stat[0], stat[1], self.flat_k, on_failure)
        return out.reshape(self.C, self.K, self.nout, -1), stat[0].reshape(self.C, self.K), \
            stat[1].reshape(self.C, self.K)


def solve_cosmologies(*, params, kmodes, aexp_out, lmaxg, lmaxgp, lmaxr, lmaxnu, nqmax, rtol, atol, pcoeff=0.25,
                      icoeff=0.80, dcoeff=0.0, factormax=20.0, factormin=0.3, max_steps=100000, return_full=False,
                      de_guard_eps=1e-9, device=None, warps_per_block=0, on_failure="raise", return_stats=False):
    """Forward solve of the k-modes of several cosmologies in ONE launch (what ``jax.vmap`` over
    cosmologies of the reference's ``evolve_perturbations`` computes).

    ``params``: list of C background dicts (``evolve_background`` outputs) with the same l_max /
    nqmax; ``kmodes``: ``[K]`` shared or ``[C, K]``; ``aexp_out``: ``[nout]`` scale factors (each
    cosmology's own output times).  Returns ``y [C, K, nout, 20]`` (or ``[C, K, nout, nvar]``).
    """
    b = CosmologyBatch(params=params, kmodes=kmodes, aexp_out=aexp_out, lmaxg=lmaxg, lmaxgp=lmaxgp, lmaxr=lmaxr,
                       lmaxnu=lmaxnu, nqmax=nqmax, rtol=rtol, atol=atol, pcoeff=pcoeff, icoeff=icoeff, dcoeff=dcoeff,
                       factormax=factormax, factormin=factormin, max_steps=max_steps, return_full=return_full,
                       de_guard_eps=de_guard_eps, device=device, warps_per_block=warps_per_block)
    b.launch()
    y, status, nsteps = b.result(on_failure)
    if return_stats:
        return y, status, nsteps
    return y


def _background_worker(p):
    import warnings
    from .background import evolve_background
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        return evolve_background(param=p)


def backgrounds(param_dicts, processes=1, device=None, num_thermo=256):
    """evolve_background of many cosmologies.  The native background takes a few milliseconds per
    cosmology, so they run in this process by default; ``processes`` > 1 (or 0: the host's cores)
    spreads them over a pool of spawned processes (safe after CUDA is initialised); ``device``
    (a CUDA device) computes them all in one GPU launch (discoeb_background_batch)."""
    param_dicts = list(param_dicts)
    if device is not None:
        from .background import background_from_buffer, native_backgrounds_device
        out, _ = native_backgrounds_device(param_dicts, num_thermo, device=device)
        out = out.cpu().numpy()
        return [background_from_buffer(p, out[c], num_thermo) for c, p in enumerate(param_dicts)]
    if len(param_dicts) <= 1 or processes == 1:
        return [_background_worker(p) for p in param_dicts]
    import multiprocessing as mp
    import os
    nproc = processes or min(len(param_dicts), os.cpu_count() or 1)
    with mp.get_context("spawn").Pool(nproc) as pool:
        return pool.map(_background_worker, param_dicts)


# the reference's perturbations module also holds the power-spectrum observables
from .observables import get_power_smoothed, get_xi_from_P, power_Kaiser, power_multipoles  # noqa: E402,F401
