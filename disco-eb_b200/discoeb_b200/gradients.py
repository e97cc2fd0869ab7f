"""Derivatives of P(k) with respect to cosmological parameters.

The reference obtains them with ``jax.jacfwd`` through ``evolve_background`` and the diffrax
solve (``DirectAdjoint``, perturbations.py:919; the gradient notebooks
``notebooks/nb_minimal_example.ipynb``, ``paper_scripts/nb_discoeb_fisher_forecast.ipynb``).
Here the same forward-mode derivative is assembled from two exact pieces:

* the background tables, scalar parameters, initial states and output times are
  differentiated on the host by complex-step differentiation of the background restatement
  with its Recfast step sequence replayed (so the derivative is that of the discrete
  background, branch choices held, as forward-mode AD gives);
* the perturbation solve is differentiated on the GPU by ``discoeb_jvp``: the tangent of the
  discrete Rodas5 solution with the accepted step sequence held fixed (the step-size
  controller is not differentiated, exactly as diffrax's stop-gradient on the step factor).

The start times of the modes (a numerical choice) and the approximation switch times are held
fixed.  n_s and A_s enter P(k) only through the primordial spectrum and are differentiated
analytically.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np

from . import _abi
from .background import evolve_background
from .perturbations import (DeviceCosmo, adiabatic_ics, approximation_switch_times, determine_starting_time, k_sampling,
                            nvar_of, _check_status)
from .workloads import cosmo_params

THETA_NAMES = ("omega_c", "omega_b", "h", "n_s", "ln10As", "w0", "wa", "m_nu")
ODE_DIRECTIONS = ("omega_c", "omega_b", "h", "w0", "wa", "m_nu")
_TABLES = (("xe_of_loga_spline", "xe"), ("cs2a_of_loga_spline", "cs2a"), ("logrhonu_of_loga_spline", "logrhonu"),
           ("logpnu_of_loga_spline", "logpnu"))
_CSTEP = 1e-30


def theta_to_params(theta, **extra):
    """Reference param dict of theta = (omega_c, omega_b, h, n_s, ln10As, w0, wa, m_nu)."""
    t = dict(theta)
    return cosmo_params(h=t["h"], omega_b=t["omega_b"], omega_c=t["omega_c"], A_s=np.exp(t["ln10As"]) / 1e10,
                        n_s=t["n_s"], m_nu=t["m_nu"], w0=t["w0"], wa=t["wa"], **extra)


def background_tangents(theta, bg, trace, directions, *, aexp_out, tau_start, kmodes, L):
    """Host-side tangents along each direction: scalars, tables, output times, initial states."""
    out = []
    for name in directions:
        tc = dict(theta)
        tc[name] = tc[name] + 1j * _CSTEP
        bgc = evolve_background(param=theta_to_params(tc), replay=trace)
        d = {"scalars": {}, "tables": {}}
        for key, field in (("grhom", "grhom"), ("Omegam", "Omegam"), ("Omegab", "Omegab"), ("OmegaDE", "OmegaDE"),
                           ("amnu", "amnu"), ("w_DE_0", "w0"), ("w_DE_a", "wa"), ("H0", "H0")):
            d["scalars"][field] = float(np.imag(bgc[key]) / _CSTEP)
        for key, short in _TABLES:
            s = bgc[key]
            d["tables"][short] = (np.ascontiguousarray(np.imag(s.y) / _CSTEP),
                                  np.ascontiguousarray(np.imag(s.S) / _CSTEP))
        d["tau_out"] = np.imag(bgc["tau_of_a_spline"].evaluate(aexp_out)) / _CSTEP
        y0c = adiabatic_ics(tau=tau_start, param=bgc, kmode=kmodes, **L)
        d["y0"] = np.ascontiguousarray(np.imag(y0c) / _CSTEP)
        out.append(d)
    return out


def power_spectrum_jacobian(theta, *, aexp_out=(1.0,), kmin=1e-4, kmax=1.0, num_k=64, lmaxg=12, lmaxgp=12, lmaxr=17,
                            lmaxnu=17, nqmax=5, rtol=1e-5, atol=1e-8, pcoeff=0.25, icoeff=0.80, dcoeff=0.0,
                            factormax=20.0, factormin=0.3, max_steps=100000, k_sampling_method="log", idx=4,
                            num_thermo=256, de_guard_eps=1e-9, device=None, warps_per_block=0, on_failure="raise",
                            return_stats=False):
    """P(k, a_out) of field ``idx`` (4: total matter) and its Jacobian with respect to theta.

    theta: dict with keys THETA_NAMES.  Returns (k, P[K, nout], J[8, K, nout]) with the rows
    of J in THETA_NAMES order.
    """
    import torch
    if device is None:
        device = torch.device("cuda", torch.cuda.current_device())
    L = dict(lmaxg=lmaxg, lmaxgp=lmaxgp, lmaxr=lmaxr, lmaxnu=lmaxnu, nqmax=nqmax)
    lib = _abi.lib()
    trace = {}
    bg = evolve_background(param=theta_to_params(theta), trace=trace, num_thermo=num_thermo)
    kmodes = k_sampling(bg, kmin, kmax, num_k, k_sampling_method)
    aexp_out = np.atleast_1d(np.asarray(aexp_out, dtype=np.float64))
    tau_out = bg["tau_of_a_spline"].evaluate(aexp_out)
    K, nout, n = kmodes.shape[0], tau_out.shape[0], nvar_of(**L)
    tau_s = determine_starting_time(param=bg, k=kmodes)
    tau_start = 0.99 * np.minimum(tau_out.min(), tau_s)
    y0 = adiabatic_ics(tau=tau_start, param=bg, kmode=kmodes, **L)
    sw = approximation_switch_times(bg, kmodes)
    dirs = ODE_DIRECTIONS
    tans = background_tangents(theta, bg, trace, dirs, aexp_out=aexp_out, tau_start=tau_start, kmodes=kmodes, L=L)
    order = np.argsort(-kmodes, kind="stable")
    dc = DeviceCosmo(bg, de_guard_eps=de_guard_eps, device=device, **L)
    f64 = dict(dtype=torch.float64, device=device)
    keep = []
    tstructs = []
    for d in tans:
        t = _abi.DiscoebTangent()
        for f, v in d["scalars"].items():
            setattr(t, f, v)
        for short, (yy, SS) in d["tables"].items():
            ty = torch.from_numpy(yy).to(device)
            tS = torch.from_numpy(SS).to(device)
            keep += [ty, tS]
            setattr(t, short + "_y", ty.data_ptr())
            setattr(t, short + "_S", tS.data_ptr())
        tstructs.append(t)
    tan_arr = (_abi.DiscoebTangent * len(tstructs))(*tstructs)
    d_tan = torch.frombuffer(bytearray(bytes(tan_arr)), dtype=torch.uint8).to(device)
    d_k = torch.tensor(kmodes[order], **f64)
    d_ts = torch.tensor(tau_start[order], **f64)
    d_y0 = torch.tensor(y0[order], **f64).contiguous()
    d_y0d = torch.tensor(np.stack([d["y0"][order] for d in tans]), **f64).contiguous()
    d_sw = torch.tensor(sw[order], **f64).contiguous()
    d_tout = torch.tensor(tau_out, **f64)
    d_toutd = torch.tensor(np.stack([d["tau_out"] for d in tans]), **f64).contiguous()
    d_out = torch.empty((K, nout, 20), **f64)
    d_outd = torch.empty((len(dirs), K, nout, 20), **f64)
    d_stat = torch.empty((2, K), dtype=torch.int32, device=device)
    ctrl = _abi.DiscoebControl(rtol, atol, pcoeff, icoeff, dcoeff, factormax, factormin, int(max_steps),
                               _abi.METHOD_RODAS5_STRUCTURED, int(warps_per_block), 0)
    stream = torch.cuda.current_stream(device).cuda_stream
    rc = lib.discoeb_jvp(dc.struct.data_ptr(), ctypes.byref(dc.host), d_tan.data_ptr(), len(dirs), ctypes.byref(ctrl),
                         K, d_k.data_ptr(), d_ts.data_ptr(), d_y0.data_ptr(), d_y0d.data_ptr(), d_sw.data_ptr(), nout,
                         d_tout.data_ptr(), d_toutd.data_ptr(), d_out.data_ptr(), d_outd.data_ptr(),
                         d_stat[0].data_ptr(), d_stat[1].data_ptr(), stream)
    if rc != 0:
        raise RuntimeError(f"discoeb_jvp failed with code {rc}")
    inv = np.empty_like(order)
    inv[order] = np.arange(K)
    y = d_out.cpu().numpy()[inv]
    yd = d_outd.cpu().numpy()[:, inv]
    stat = d_stat.cpu().numpy()
    status, nsteps = stat[0][inv], stat[1][inv]
    _check_status(status, nsteps, kmodes, on_failure)
    delta = y[..., idx]
    P = 2 * np.pi**2 * bg["A_s"] * (kmodes[:, None] / bg["k_p"]) ** (bg["n_s"] - 1) * kmodes[:, None] ** -3 * delta**2
    J = np.zeros((len(THETA_NAMES), K, nout))
    for di, name in enumerate(dirs):
        J[THETA_NAMES.index(name)] = 2.0 * P * yd[di, ..., idx] / delta
    J[THETA_NAMES.index("n_s")] = P * np.log(kmodes[:, None] / bg["k_p"])
    J[THETA_NAMES.index("ln10As")] = P
    if return_stats:
        return kmodes, P, J, status, nsteps
    return kmodes, P, J
