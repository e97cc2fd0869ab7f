"""Background cosmology and thermal history (host side, float64 numpy).

Mirrors ``src/discoeb/background.py`` of the reference: ``evolve_background`` takes the
same cosmological ``param`` dict (``Omegam, Omegab, H0, Tcmb, YHe, Neff, Nmnu, mnu,
w_DE_0, w_DE_a, cs2_DE, Omegak, A_s, n_s, k_p``) and returns it completed with the
derived densities and the spline tables the perturbation solve reads.  It is the
producer of the device kernels' inputs and runs on the host.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np

from .romberg import romb
from .spline import spline_interpolation
from . import thermodynamics_recfast as _recfast

FERMI_DIRAC_CONST = 5.682196976983475  # 7 pi^4 / 120


def generalized_gauss_laguerre_weights(n: int, alpha: float):
    """Golub-Welsch nodes/weights for int_0^inf x^alpha f(x) e^-x dx (util.py:83-124)."""
    i = np.arange(1, n + 1)
    diag = 2 * i - 1 + alpha
    io = np.arange(1, n)
    off = np.sqrt(io * (io + alpha))
    J = np.diag(diag) + np.diag(off, 1) + np.diag(off, -1)
    nodes, V = np.linalg.eigh(J)
    weights = V[0, :] ** 2 * math.gamma(alpha + 1)
    return nodes, weights


def get_neutrino_momentum_bins(nqmax: int):
    """Momentum bins q and quadrature weights for massive neutrinos (background.py:14-45).

    nqmax = 3, 4, 5 use CAMB's tabulated nodes; other values a generalized
    Gauss-Laguerre rule with alpha = 1.
    """
    if nqmax == 3:
        q = np.array([0.913201, 3.37517, 7.79184])
        w0 = np.array([0.0687359, 3.31435, 2.29911])
    elif nqmax == 4:
        q = np.array([0.7, 2.62814, 5.90428, 12.0])
        w0 = np.array([0.0200251, 1.84539, 3.52736, 0.289427])
    elif nqmax == 5:
        q = np.array([0.583165, 2.0, 4.0, 7.26582, 13.0])
        w0 = np.array([0.0081201, 0.689407, 2.8063, 2.05156, 0.12681])
    else:
        alpha = 1
        q, w = generalized_gauss_laguerre_weights(nqmax, alpha)
        w = w * q**3 / (1 + np.exp(-q)) * q ** (-alpha)
        return q, w / FERMI_DIRAC_CONST
    dlfdlq = -q / (1 + np.exp(-q))
    w = w0 / (-0.25 * dlfdlq)
    return q, w / FERMI_DIRAC_CONST


def nu_background(a, amnu, nq: int = 8):
    """rho_nu/rho_nu0, p_nu/p_nu0, pseudo-pressure of one massive flavour (background.py:48-69)."""
    a = np.asarray(a, dtype=np.float64)
    q, w = get_neutrino_momentum_bins(nq)
    v = 1.0 / np.sqrt(1.0 + (a[..., None] * amnu / q) ** 2)
    return (w / v).sum(-1), (w * v / 3).sum(-1), (w * v**3 / 3).sum(-1)


def _rho_Q(a, p):
    return a ** (-3 * (1 + p["w_DE_0"] + p["w_DE_a"])) * np.exp(3 * (a - 1) * p["w_DE_a"])


def get_aprimeoa(*, param, aexp):
    """Conformal Hubble rate a'/a in 1/Mpc (background.py:101-123)."""
    aexp = np.asarray(aexp, dtype=np.float64)
    rhonu = np.exp(param["logrhonu_of_loga_spline"].evaluate(np.log(aexp)))
    grho = (param["grhom"] * param["Omegam"] / aexp
            + (param["grhog"] + param["grhor"] * (param["Neff"] + param["Nmnu"] * rhonu)) / aexp**2
            + param["grhom"] * param["OmegaDE"] * _rho_Q(aexp, param) * aexp**2
            + param["grhom"] * param["Omegak"])
    return np.sqrt(grho / 3.0)


def dadtau(a, param):
    """da/dtau (background.py:84-93)."""
    a = np.asarray(a, dtype=np.float64)
    rhonu = np.exp(param["logrhonu_of_loga_spline"].evaluate(np.log(a)))
    grho2 = (param["grhom"] * param["Omegam"] * a
             + (param["grhog"] + param["grhor"] * (param["Neff"] + param["Nmnu"] * rhonu))
             + param["grhom"] * param["OmegaDE"] * _rho_Q(a, param) * a**4
             + param["grhom"] * param["Omegak"] * a**2)
    return np.sqrt(grho2 / 3.0)


def dtauda(a, param):
    return 1.0 / dadtau(a, param)


def setup_background_evolution(*, amin, amax, param):
    """Densities, massive-neutrino tables and the tau range (background.py:141-189)."""
    c2ok = 1.62581581e4
    num_neutrino = 512
    param["amin"] = amin
    param["amax"] = amax
    param["grhom"] = 3.33795017e-11 * param["H0"] ** 2
    param["grhog"] = 1.49594245e-13 * param["Tcmb"] ** 4
    param["grhor"] = 3.39739477e-14 * param["Tcmb"] ** 4
    param["adotrad"] = math.sqrt((param["grhog"] + param["grhor"] * (param["Neff"] + param["Nmnu"])) / 3.0)
    param["amnu"] = param["mnu"] * c2ok / param["Tcmb"]
    a = np.geomspace(amin * 0.9, amax * 1.1, num_neutrino)
    loga = np.log(a)
    param["a"] = a
    rhonu_, pnu_, ppnu_ = nu_background(a, param["amnu"])
    param["logrhonu_of_loga_spline"] = spline_interpolation(loga, np.log(rhonu_), uniform=True)
    param["logpnu_of_loga_spline"] = spline_interpolation(loga, np.log(pnu_), uniform=True)
    param["logppseudonu_of_loga_spline"] = spline_interpolation(loga, np.log(ppnu_), uniform=True)
    rhonu0 = np.exp(param["logrhonu_of_loga_spline"].evaluate(0.0))
    param["Omegamnu"] = param["grhor"] * rhonu0 / param["grhom"]
    Omegar = (param["Neff"] + param["Nmnu"] * rhonu0) * param["grhor"] / param["grhom"]
    Omegag = param["grhog"] / param["grhom"]
    param["OmegaDE"] = 1.0 - param["Omegak"] - Omegar - Omegag - param["Omegam"]
    param["taumin"] = amin / param["adotrad"]
    param["taumax"] = param["taumin"] + romb(lambda x: dtauda(x, param), amin, amax)
    return param


_PARAM_FIELDS = ("H0", "Omegab", "Omegam", "mnu", "w_DE_0", "w_DE_a", "Tcmb", "YHe", "Neff", "Nmnu", "cs2_DE", "Omegak")
_DIFF_FIELDS = _PARAM_FIELDS[:6]


def _is_complex(param):
    return any(np.iscomplexobj(param.get(k, 0.0)) for k in _PARAM_FIELDS)


def _params_struct(param, fields=_PARAM_FIELDS):
    from . import _abi
    c = _abi.DiscoebCosmoParams()
    for f in fields:
        setattr(c, f, float(np.real(param.get(f, 0.0))))
    return c


def native_background(param, num_thermo=256, param_dots=(), n_threads=0):
    """``discoeb_background``: the values (one flat buffer, layout ``_abi.background_layout``) and,
    for each entry of ``param_dots`` (dicts of d(H0, Omegab, Omegam, mnu, w_DE_0, w_DE_a)), the
    exact tangent buffer (Recfast branches and steps held fixed)."""
    from . import _abi
    lib = _abi.lib()
    _, size = _abi.background_layout(num_thermo)
    out = np.empty(size)
    nd = len(param_dots)
    dots = (_abi.DiscoebCosmoParams * max(nd, 1))(*[_params_struct(d, _DIFF_FIELDS) for d in param_dots])
    out_dot = np.empty((nd, size)) if nd else None
    rc = lib.discoeb_background(ctypes.byref(_params_struct(param)), ctypes.cast(dots, ctypes.c_void_p) if nd else None,
                                nd, int(num_thermo), out.ctypes.data, out_dot.ctypes.data if nd else None,
                                int(n_threads))
    if rc != 0:
        raise ValueError(f"discoeb_background rejected its arguments (code {rc}; num_thermo >= 32 required)")
    return out, out_dot


def native_backgrounds_device(params, num_thermo=256, param_dots=None, device=None):
    """``discoeb_background_batch``: the backgrounds of many cosmologies (and, with ``param_dots``,
    a list per cosmology of dicts of d(H0, Omegab, Omegam, mnu, w_DE_0, w_DE_a), the same number for
    every cosmology) in one GPU launch.  Returns device tensors (values [C, size], tangents
    [C, n_dir, size] or None)."""
    import torch

    from . import _abi
    lib = _abi.lib()
    if device is None:
        device = torch.device("cuda", torch.cuda.current_device())
    C = len(params)
    nd = len(param_dots[0]) if param_dots else 0
    if param_dots and any(len(d) != nd for d in param_dots):
        raise ValueError("every cosmology needs the same number of tangent directions")
    _, size = _abi.background_layout(num_thermo)
    host = (_abi.DiscoebCosmoParams * C)(*[_params_struct(p) for p in params])
    par = torch.frombuffer(bytearray(bytes(host)), dtype=torch.uint8).to(device)
    dots = None
    if nd:
        hd = (_abi.DiscoebCosmoParams * (C * nd))(*[_params_struct(d, _DIFF_FIELDS) for ds in param_dots for d in ds])
        dots = torch.frombuffer(bytearray(bytes(hd)), dtype=torch.uint8).to(device)
    wsb = lib.discoeb_background_batch_workspace_bytes(C, nd, int(num_thermo))
    if wsb < 0:
        raise ValueError("discoeb_background_batch_workspace_bytes rejected its arguments (num_thermo >= 32)")
    ws = torch.empty(int(wsb) + 256, dtype=torch.uint8, device=device)
    base = (ws.data_ptr() + 255) & ~255
    out = torch.empty((C, size), dtype=torch.float64, device=device)
    out_dot = torch.empty((C, nd, size), dtype=torch.float64, device=device) if nd else None
    rc = lib.discoeb_background_batch(par.data_ptr(), dots.data_ptr() if nd else None, C, nd, int(num_thermo), base,
                                      int(wsb), out.data_ptr(), out_dot.data_ptr() if nd else None,
                                      torch.cuda.current_stream(device).cuda_stream)
    if rc != 0:
        raise RuntimeError(f"discoeb_background_batch failed with code {rc}")
    return out, out_dot


def background_from_buffer(param, buf, num_thermo):
    """The evolve_background dict of ``param`` from a discoeb_background value buffer."""
    from . import _abi
    lay, _ = _abi.background_layout(num_thermo)
    S = lambda nm: buf[lay["s:" + nm]]  # noqa: E731
    N = lambda nm: buf[lay["n:" + nm]]  # noqa: E731
    T = lambda nm: buf[lay["t:" + nm]]  # noqa: E731
    param = dict(param)
    param.setdefault("Omegak", 0.0)
    for nm in ("amin", "amax", "grhom", "grhog", "grhor", "adotrad", "amnu", "Omegamnu", "OmegaDE", "taumin", "taumax",
               "fHe", "tau0", "tau_maxvis"):
        param[nm] = float(S(nm))
    param["a"] = N("a")
    spl = spline_interpolation.from_table
    param["logrhonu_of_loga_spline"] = spl(N("loga"), N("logrhonu_y"), N("logrhonu_S"), uniform=True)
    param["logpnu_of_loga_spline"] = spl(N("loga"), N("logpnu_y"), N("logpnu_S"), uniform=True)
    param["logppseudonu_of_loga_spline"] = spl(N("loga"), N("logppnu_y"), N("logppnu_S"), uniform=True)
    aexp, tau = T("aexp"), T("tau")
    for nm in ("aexp", "tau", "xe", "xeHI", "xeHeI", "xeHeII", "cs2", "Tm", "optical_depth", "opac", "gvis",
               "gvisprime", "gvispprime", "xeprime_recf", "xeprime"):
        param[nm] = T(nm)
    param["tau_of_a_spline"] = spl(aexp, tau, T("tau_of_a_S"))
    param["a_of_tau_spline"] = spl(tau, aexp, T("a_of_tau_S"))
    param["xe_of_tau_spline"] = spl(tau, T("xe"), T("xe_of_tau_S"))
    param["cs2a_of_tau_spline"] = spl(tau, T("cs2a"), T("cs2a_of_tau_S"))
    param["tempba_of_tau_spline"] = spl(tau, T("tempba"), T("tempba_of_tau_S"))
    param["xe_of_loga_spline"] = spl(T("loga"), T("xe"), T("xe_of_loga_S"))
    param["cs2a_of_loga_spline"] = spl(T("loga"), T("cs2a"), T("cs2a_of_loga_S"))
    return param


def evolve_background(*, param, thermo_module="RECFAST", num_thermo: int = 256, rtol: float = 1e-5,
                      atol: float = 1e-7, order: int = 5, class_thermo=None, trace=None, replay=None,
                      backend="native"):
    """Background + Recfast thermal history + visibility (background.py:191-345).

    Returns a new dict (the caller's dict is not modified, as under the
    reference's ``jax.jit``).  Only ``thermo_module='RECFAST'`` is provided.
    ``backend``: "native" (``discoeb_background``, C++ host code) or "numpy" (this module's
    restatement, which also takes complex parameters for complex-step derivatives).  Complex
    parameters, ``trace`` or ``replay`` select the numpy restatement.
    ``trace``/``replay``: record / repeat the Recfast step sequence (see
    thermodynamics_recfast.solve_pid_grk4a), for derivatives with respect to parameters.
    """
    if thermo_module != "RECFAST":
        raise ValueError(f"thermo_module {thermo_module!r} is not provided; use 'RECFAST'")
    if backend not in ("native", "numpy"):
        raise ValueError(f"unknown backend {backend!r}")
    if backend == "native" and trace is None and replay is None and not _is_complex(param):
        buf, _ = native_background(param, num_thermo)
        return background_from_buffer(param, buf, num_thermo)
    param = dict(param)
    param.setdefault("Omegak", 0.0)
    amin, amax = 1e-9, 1.01
    param = setup_background_evolution(amin=amin, amax=amax, param=param)
    param, tau, aexp, cs2, Tm, mu, xe, xeHI, xeHeI, xeHeII, xeprime_recfast = _recfast.evaluate_thermo(
        param=param, num_thermo=num_thermo,
        aprimeoa_fn=lambda a: get_aprimeoa(param=param, aexp=a)[()],
        dadtau_fn=lambda a: dadtau(a, param),
        dtauda_fn=lambda a: dtauda(a, param), trace=trace, replay=replay)
    param["aexp"] = aexp
    param["tau"] = tau
    param["xe"] = xe
    param["xeHI"] = xeHI
    param["xeHeI"] = xeHeI
    param["xeHeII"] = xeHeII
    param["cs2"] = cs2
    param["Tm"] = Tm
    param["tau_of_a_spline"] = spline_interpolation(aexp, tau)
    param["a_of_tau_spline"] = spline_interpolation(tau, aexp)
    param["xe_of_tau_spline"] = spline_interpolation(tau, xe)
    param["cs2a_of_tau_spline"] = spline_interpolation(tau, aexp * cs2)
    param["tempba_of_tau_spline"] = spline_interpolation(tau, aexp * Tm)
    param["xe_of_loga_spline"] = spline_interpolation(np.log(aexp), xe)
    param["cs2a_of_loga_spline"] = spline_interpolation(np.log(aexp), aexp * cs2)

    akthom = 2.3038921003709498e-9 * (1.0 - param["YHe"]) * param["Omegab"] * param["H0"] ** 2
    tau_pre_recomb = param["tau_of_a_spline"].evaluate(1e-4)
    xe_full = 1 + param["YHe"] / (1 - param["YHe"])
    xe_v = np.where(tau <= tau_pre_recomb, xe_full, param["xe_of_tau_spline"].evaluate(tau))
    xeprime = np.where(tau <= tau_pre_recomb, 0.0, param["xe_of_tau_spline"].derivative(tau))
    opac = xe_v * akthom / aexp**2
    opacspline = spline_interpolation(tau, opac, integrate_from_start=True)
    opacprime, opacpprime = opacspline.derivative12(tau)
    optical_depth_today = opacspline.integral(param["tau_of_a_spline"].evaluate(1.0))
    optical_depth = optical_depth_today - opacspline.integral(tau)
    expmmu = np.exp(-optical_depth)
    vis = opac * expmmu
    param["optical_depth"] = optical_depth
    param["opac"] = opac
    param["gvis"] = vis
    param["gvisprime"] = (opacprime + opac**2) * expmmu
    param["gvispprime"] = (opacpprime + 3 * opac * opacprime + opac**3) * expmmu
    param["tau0"] = param["tau_of_a_spline"].evaluate(1.0)[()]
    param["tau_maxvis"] = np.real(param["tau"][int(np.argmax(np.real(param["gvis"])))])[()]
    param["xeprime_recf"] = xeprime_recfast
    param["xeprime"] = xeprime
    return param


def compute_background_quantities(aexp, param):
    """rho_nu, rho_Q and w_Q at the given scale factors (background.py:348-406)."""
    a = np.atleast_1d(np.asarray(aexp, dtype=np.float64))
    return {
        "rhonu": np.exp(param["logrhonu_of_loga_spline"].evaluate(np.log(a))),
        "rho_Q": _rho_Q(a, param),
        "w_Q": param["w_DE_0"] + param["w_DE_a"] * (1.0 - a),
    }
