"""CMB temperature source functions, line-of-sight multipoles and C_l on the GPU.

Mirrors the call surface of the reference's ``src/discoeb/cmb.py``:
``compute_visibility_functions`` (host, 1-D tables), ``compute_source_function`` ->
``discoeb_sources``, ``compute_theta_ell`` -> ``discoeb_los`` (FFTLog: cuFFT + one FP64 GEMM),
``compute_Cell`` -> ``discoeb_cell``, ``compute_Dell`` (unit conversion) and
``compute_Cell_spectrum_from_cosmo_params`` (the whole chain with every large array resident on
the device).  The per-stage intermediates of the reference (metric, polarisation and neutrino
terms) are fields of the same source kernel, returned by ``compute_sources``.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np

from . import _abi
from .background import compute_background_quantities, evolve_background, get_aprimeoa, get_neutrino_momentum_bins
from .perturbations import (DeviceCosmo, _check_status, adiabatic_ics, approximation_switch_times,
                            determine_starting_time, k_sampling, solve_modes)
from .spline import spline_interpolation

BG_FIELDS = ("a", "aprimeoa", "rhonu", "rho_Q", "w_Q", "opac", "opacprime", "gvis", "gvisprime", "gvispprime",
             "optical_depth")
SRC_FIELDS = ("S", "S1", "S2", "S3", "S4", "potential", "alpha", "alphaprime", "alphapprime", "hprime", "etaprime",
              "aprimeoaprime", "polarization_term", "polarization_termprime", "polarization_termpprime", "drhonu",
              "dpnu", "fnu", "shearnu", "rho_nu_prime", "shear_nu_prime", "thetabprime", "E")


def _device(device):
    import torch
    if device is None:
        if not torch.cuda.is_available():
            raise RuntimeError("discoeb_b200 needs a CUDA device (there is no CPU path)")
        device = torch.device("cuda", torch.cuda.current_device())
    return torch, device


def compute_visibility_functions(tau, param):
    """Opacity, visibility g and its derivatives, optical depth at ``tau`` (cmb.py:95-163):
    natural cubic splines in ln(tau) of the thermal-history arrays of ``evolve_background``."""
    tau = np.asarray(tau, dtype=np.float64)
    lt, ltn = np.log(param["tau"]), np.log(tau)
    op = spline_interpolation(lt, param["opac"])
    od = spline_interpolation(lt, np.log(np.maximum(param["optical_depth"], 1e-10)))
    return {
        "opac": op.evaluate(ltn),
        "opacprime": op.derivative(ltn) / tau,
        "gvis": spline_interpolation(lt, param["gvis"]).evaluate(ltn),
        "gvisprime": spline_interpolation(lt, param["gvisprime"]).evaluate(ltn),
        "gvispprime": spline_interpolation(lt, param["gvispprime"]).evaluate(ltn),
        "optical_depth": np.exp(od.evaluate(ltn)),
    }


def background_table(aexp_out, tau, param):
    """``float64[DISCOEB_BG_NFIELDS, n_tau]``: the per-output-time inputs of discoeb_sources."""
    aexp_out = np.asarray(aexp_out, dtype=np.float64)
    bq = compute_background_quantities(aexp_out, param)
    vis = compute_visibility_functions(tau, param)
    rows = {"a": aexp_out, "aprimeoa": get_aprimeoa(param=param, aexp=aexp_out), **bq, **vis}
    return np.ascontiguousarray(np.stack([np.broadcast_to(rows[f], aexp_out.shape) for f in BG_FIELDS]))


# points (modes x output times) that discoeb_sources_noalloc's own scratch array holds
NOALLOC_MAX_POINTS = 1 << 20


def noalloc_check(n_modes, n_tau):
    """Raise ValueError if discoeb_sources_noalloc would refuse these sizes (its scratch array
    holds NOALLOC_MAX_POINTS points)."""
    if n_modes * n_tau > NOALLOC_MAX_POINTS:
        raise ValueError(f"no_alloc: {n_modes} modes x {n_tau} times exceeds the {NOALLOC_MAX_POINTS} points of "
                         "the library's scratch")


def compute_sources(*, param, yout, kmodes, aexp_out, lmaxg, lmaxgp, lmaxr, lmaxnu, nqmax, de_guard_eps=1e-9,
                    device=None, no_alloc=False):
    """All source fields of compute_source_function and its intermediates (cmb.py:17-633).

    ``yout``: the RSA-projected full states ``[K, n_tau, nvar]`` at ``tau(aexp_out)`` (numpy or
    a device tensor).  Returns a dict of device tensors ``[K, n_tau]`` keyed by SRC_FIELDS.
    ``no_alloc``: use discoeb_sources_noalloc, which needs no scratch buffer from the caller (for
    callers that cannot allocate device memory; the library's own 8 MiB array limits
    K * n_tau to 2^20, and calls must not overlap on one device).
    """
    torch, device = _device(device)
    lib = _abi.lib()
    aexp_out = np.asarray(aexp_out, dtype=np.float64)
    tau = param["tau_of_a_spline"].evaluate(aexp_out)
    kmodes = np.ascontiguousarray(kmodes, dtype=np.float64)
    K, T = kmodes.shape[0], tau.shape[0]
    dc = DeviceCosmo(param, lmaxg=lmaxg, lmaxgp=lmaxgp, lmaxr=lmaxr, lmaxnu=lmaxnu, nqmax=nqmax,
                     de_guard_eps=de_guard_eps, device=device)
    f64 = dict(dtype=torch.float64, device=device)
    y = yout if isinstance(yout, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(yout))
    y = y.to(**f64).contiguous()
    if y.shape[:2] != (K, T):
        raise ValueError(f"yout must have shape [{K}, {T}, nvar], got {tuple(y.shape)}")
    if no_alloc:
        noalloc_check(K, T)
    d_k = torch.from_numpy(kmodes).to(device)
    d_tau = torch.from_numpy(np.ascontiguousarray(tau)).to(device)
    d_bt = torch.from_numpy(background_table(aexp_out, tau, param)).to(device)
    fields = torch.empty((len(SRC_FIELDS), K, T), **f64)
    stream = torch.cuda.current_stream(device).cuda_stream
    if no_alloc:
        rc = lib.discoeb_sources_noalloc(dc.struct.data_ptr(), ctypes.byref(dc.host), K, d_k.data_ptr(), T,
                                         d_tau.data_ptr(), d_bt.data_ptr(), y.data_ptr(), fields.data_ptr(), stream)
    else:
        scratch = torch.empty((K, T), **f64)
        rc = lib.discoeb_sources(dc.struct.data_ptr(), ctypes.byref(dc.host), K, d_k.data_ptr(), T, d_tau.data_ptr(),
                                 d_bt.data_ptr(), y.data_ptr(), fields.data_ptr(), scratch.data_ptr(), stream)
    if rc != 0:
        raise RuntimeError(f"discoeb_sources failed with code {rc}")
    return {name: fields[i] for i, name in enumerate(SRC_FIELDS)}


def solve_sources(*, param, kmodes, aexp_out, lmaxg, lmaxgp, lmaxr, lmaxnu, nqmax, rtol, atol, max_steps,
                  de_guard_eps=1e-9, device=None, return_states=False, on_failure="raise"):
    """The full perturbation solve and the source assembly in one pass (discoeb_fwd_sources):
    the same fields as solve_modes(return_full=True) followed by compute_sources, without the full
    states going through device memory.  The step controller is the reference pipeline's (PID
    coefficients 0.25 / 0.80 / 0, factors 20 / 0.3).  Returns the dict of source fields (device
    tensors [K, n_tau], caller's mode order), and with ``return_states`` also the projected states
    [K, n_tau, nvar]."""
    torch, device = _device(device)
    lib = _abi.lib()
    aexp_out = np.asarray(aexp_out, dtype=np.float64)
    tau = param["tau_of_a_spline"].evaluate(aexp_out)
    if np.any(np.diff(tau) <= 0):
        raise ValueError("aexp_out must map to strictly increasing output times")
    kmodes = np.ascontiguousarray(kmodes, dtype=np.float64)
    K, T = kmodes.shape[0], tau.shape[0]
    L = dict(lmaxg=lmaxg, lmaxgp=lmaxgp, lmaxr=lmaxr, lmaxnu=lmaxnu, nqmax=nqmax)
    tau_start = 0.99 * np.minimum(tau.min(), determine_starting_time(param=param, k=kmodes))
    y0 = adiabatic_ics(tau=tau_start, param=param, kmode=kmodes, **L)
    sw = approximation_switch_times(param, kmodes)
    order = np.argsort(-kmodes, kind="stable")  # longest modes first
    inv_np = np.argsort(order)
    dc = DeviceCosmo(param, de_guard_eps=de_guard_eps, device=device, **L)
    f64 = dict(dtype=torch.float64, device=device)
    as_dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(device)  # noqa: E731
    d_k, d_ts, d_y0, d_sw = as_dev(kmodes[order]), as_dev(tau_start[order]), as_dev(y0[order]), as_dev(sw[order])
    d_tau = as_dev(tau)
    d_bt = as_dev(background_table(aexp_out, tau, param))
    n = y0.shape[1]
    d_full = torch.empty((K, T, n), **f64) if return_states else None
    fields = torch.empty((len(SRC_FIELDS), K, T), **f64)
    scratch = torch.empty((K, T), **f64)
    d_stat = torch.empty((2, K), dtype=torch.int32, device=device)
    ctrl = _abi.DiscoebControl(rtol, atol, 0.25, 0.80, 0.0, 20.0, 0.3, int(max_steps), _abi.METHOD_RODAS5_STRUCTURED,
                               0, 0)
    rc = lib.discoeb_fwd_sources(dc.struct.data_ptr(), ctypes.byref(dc.host), ctypes.byref(ctrl), K, d_k.data_ptr(),
                                 d_ts.data_ptr(), d_y0.data_ptr(), d_sw.data_ptr(), T, d_tau.data_ptr(),
                                 d_bt.data_ptr(), d_full.data_ptr() if d_full is not None else None,
                                 fields.data_ptr(), scratch.data_ptr(), d_stat[0].data_ptr(), d_stat[1].data_ptr(),
                                 torch.cuda.current_stream(device).cuda_stream)
    if rc != 0:
        raise RuntimeError(f"discoeb_fwd_sources failed with code {rc}")
    stat = d_stat.cpu().numpy()
    _check_status(stat[0][inv_np], stat[1][inv_np], kmodes, on_failure)
    inv = torch.from_numpy(inv_np).to(device)
    out = {name: fields[i].index_select(0, inv) for i, name in enumerate(SRC_FIELDS)}
    if return_states:
        return out, d_full.index_select(0, inv)
    return out


def compute_theta_ell(ellmax, kmodes, tau, S, tau0, n_fftlog=16384, n_k_dense=0, device=None, kind="T"):
    """Theta_l(k) by FFTLog line-of-sight integration (cmb.py:680-835).

    ``kind="T"``: the temperature multipoles of the source S (the reference's path); ``kind="E"``:
    the E-mode multipoles sqrt((l+2)!/(l-2)!) int S_E j_l(x) / x^2 dtau of the E source
    (``compute_sources(...)["E"]``; discoeb_los_e, no counterpart in the reference).
    Returns ``(theta [K', ellmax+1], kmodes [K'])`` as device tensors (K' = n_k_dense if > 0).
    """
    if kind not in ("T", "E"):
        raise ValueError(f"kind must be 'T' or 'E', not {kind!r}")
    torch, device = _device(device)
    lib = _abi.lib()
    f64 = dict(dtype=torch.float64, device=device)
    d_k = torch.as_tensor(np.asarray(kmodes, dtype=np.float64) if not isinstance(kmodes, torch.Tensor) else kmodes)
    d_k = d_k.to(**f64).contiguous()
    d_tau = torch.as_tensor(np.asarray(tau, dtype=np.float64) if not isinstance(tau, torch.Tensor) else tau)
    d_tau = d_tau.to(**f64).contiguous()
    d_S = S if isinstance(S, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(S, dtype=np.float64))
    d_S = d_S.to(**f64).contiguous()
    K, T = d_S.shape
    if d_k.shape[0] != K or d_tau.shape[0] != T:
        raise ValueError("S must have shape [len(kmodes), len(tau)]")
    size_fn, entry = ((lib.discoeb_los_workspace_bytes, lib.discoeb_los) if kind == "T" else
                      (lib.discoeb_los_e_workspace_bytes, lib.discoeb_los_e))
    nb = size_fn(K, T, int(ellmax), int(n_fftlog), int(n_k_dense))
    if nb < 0:
        raise ValueError(f"invalid sizes for the line-of-sight integral (code {nb})")
    ws = torch.empty(int(nb) // 8 + 32, dtype=torch.float64, device=device)
    rows = int(n_k_dense) if n_k_dense > 0 else K
    theta = torch.empty((rows, int(ellmax) + 1), **f64)
    k_out = torch.empty(rows, **f64)
    stream = torch.cuda.current_stream(device).cuda_stream
    base = ws.data_ptr()
    aligned = (base + 255) // 256 * 256
    rc = entry(K, d_k.data_ptr(), T, d_tau.data_ptr(), d_S.data_ptr(), float(tau0), int(ellmax), int(n_fftlog),
               int(n_k_dense), aligned, int(nb), theta.data_ptr(), k_out.data_ptr(), stream)
    if rc != 0:
        raise RuntimeError(f"line-of-sight integral ({kind}) failed with code {rc}")
    return theta, k_out


LOS_CONTRACTIONS = {"fp64": 0, "int8": 1}


def set_los_contraction(kind="int8", slices=7):
    """Choose how the line of sight contracts its frequency sum (library-wide): ``"int8"`` (the
    default) on the int8 tensor cores with `slices` digit planes per operand (``dgemm_i8``; 7 give
    ~1e-13 of each row's largest |theta_l(k)|, 8 ~1e-14), or ``"fp64"``, a cuBLAS DGEMM."""
    if kind not in LOS_CONTRACTIONS:
        raise ValueError(f"kind must be one of {sorted(LOS_CONTRACTIONS)}, not {kind!r}")
    rc = _abi.lib().discoeb_set_los_contraction(LOS_CONTRACTIONS[kind], int(slices))
    if rc != 0:
        raise ValueError(f"invalid line-of-sight contraction ({kind!r}, slices={slices})")


def get_los_contraction():
    """(kind, slices) of the current line-of-sight contraction."""
    k, s = ctypes.c_int32(), ctypes.c_int32()
    _abi.lib().discoeb_get_los_contraction(ctypes.byref(k), ctypes.byref(s))
    return {v: n for n, v in LOS_CONTRACTIONS.items()}[k.value], s.value


def dgemm_i8(A, B, slices=7, split=0, device=None, trans_a=False, trans_b=False):
    """C = op(A) op(B)^T in FP64 on the int8 tensor cores (``discoeb_dgemm_i8``: `slices` digit
    planes per row of each operand, the digit products summed exactly in int32).  op(A) = A [m, k],
    or A^T when ``trans_a`` (A [k, m]); op(B) = B [n, k], or B^T when ``trans_b``.  numpy arrays or
    torch tensors; returns a torch float64 tensor [m, n] on the device."""
    torch, device = _device(device)
    lib = _abi.lib()
    f64 = dict(dtype=torch.float64, device=device)
    dA = (A if isinstance(A, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(A, dtype=np.float64)))
    dB = (B if isinstance(B, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(B, dtype=np.float64)))
    dA, dB = dA.to(**f64).contiguous(), dB.to(**f64).contiguous()
    if dA.dim() != 2 or dB.dim() != 2:
        raise ValueError("A and B must be matrices")
    (k, m) = dA.shape if trans_a else dA.shape[::-1]
    (kb, n) = dB.shape if trans_b else dB.shape[::-1]
    if k != kb:
        raise ValueError("op(A) [m, k] and op(B) [n, k] must share k")
    nb = lib.discoeb_dgemm_i8_workspace_bytes(m, n, k, int(slices), int(split))
    if nb < 0:
        raise ValueError(f"invalid sizes or slice count for dgemm_i8 (code {nb})")
    ws = torch.empty(int(nb) // 8 + 32, **f64)
    aligned = (ws.data_ptr() + 255) // 256 * 256
    C = torch.empty((m, n), **f64)
    rc = lib.discoeb_dgemm_i8(m, n, k, dA.data_ptr(), dA.shape[1], int(trans_a), dB.data_ptr(), dB.shape[1],
                              int(trans_b), C.data_ptr(), n, int(slices), int(split), aligned, int(nb),
                              torch.cuda.current_stream(device).cuda_stream)
    if rc != 0:
        raise RuntimeError(f"dgemm_i8 failed with code {rc}")
    return C


def compute_Cell(theta_ell, kmodes, n_s, k_p, device=None, theta_ell_b=None):
    """C_l = int d ln k (k/k_p)^(n_s-1) Theta_l^2, trapezoid (cmb.py:838-873); device tensor.
    ``theta_ell_b``: the cross spectrum int d ln k (k/k_p)^(n_s-1) Theta_l Theta^b_l (C_l^TE from
    the T and E multipoles; discoeb_cell_cross)."""
    torch, device = _device(device)
    lib = _abi.lib()
    f64 = dict(dtype=torch.float64, device=device)
    as_dev = lambda a: (a if isinstance(a, torch.Tensor) else torch.from_numpy(  # noqa: E731
        np.ascontiguousarray(a))).to(**f64).contiguous()
    th, kk = as_dev(theta_ell), as_dev(kmodes)
    K, L = th.shape
    cell = torch.empty(L, **f64)
    stream = torch.cuda.current_stream(device).cuda_stream
    if theta_ell_b is None:
        rc = lib.discoeb_cell(K, kk.data_ptr(), L, th.data_ptr(), float(n_s), float(k_p), cell.data_ptr(), stream)
    else:
        tb = as_dev(theta_ell_b)
        if tuple(tb.shape) != (K, L):
            raise ValueError("theta_ell_b must have the shape of theta_ell")
        rc = lib.discoeb_cell_cross(K, kk.data_ptr(), L, th.data_ptr(), tb.data_ptr(), float(n_s), float(k_p),
                                    cell.data_ptr(), stream)
    if rc != 0:
        raise RuntimeError(f"discoeb_cell failed with code {rc}")
    return cell


def compute_Cell_tangent(ellmax, kmodes, tau, S, tau0, n_s, k_p, tau_dot, S_dot, tau0_dot, n_fftlog=16384,
                         n_k_dense=0, device=None):
    """C_l of the line of sight (compute_theta_ell then compute_Cell) and its derivatives along
    the input directions (``tau_dot [D, n_tau]``, ``S_dot [D, K, n_tau]``, ``tau0_dot [D]``) in
    forward mode (discoeb_los_cell_jvp).  Returns ``(cell [ellmax+1], cell_dot [D, ellmax+1],
    cell_dns [ellmax+1])`` as device tensors, the last d C_l / d n_s."""
    torch, device = _device(device)
    lib = _abi.lib()
    f64 = dict(dtype=torch.float64, device=device)
    as_dev = lambda a: (a if isinstance(a, torch.Tensor) else torch.from_numpy(  # noqa: E731
        np.ascontiguousarray(a, dtype=np.float64))).to(**f64).contiguous()
    d_k, d_tau, d_S = as_dev(kmodes), as_dev(tau), as_dev(S)
    d_td, d_Sd = as_dev(tau_dot), as_dev(S_dot)
    t0d = np.ascontiguousarray(tau0_dot, dtype=np.float64)
    K, T = d_S.shape
    nd = int(t0d.shape[0])
    if d_k.shape[0] != K or d_tau.shape[0] != T or tuple(d_td.shape) != (nd, T) or tuple(d_Sd.shape) != (nd, K, T):
        raise ValueError("inconsistent shapes for the line-of-sight tangent")
    nb = lib.discoeb_los_cell_jvp_workspace_bytes(K, T, int(ellmax), int(n_fftlog), int(n_k_dense))
    if nb < 0:
        raise ValueError(f"invalid sizes for the line-of-sight tangent (code {nb})")
    ws = torch.empty(int(nb) // 8 + 32, **f64)
    aligned = (ws.data_ptr() + 255) // 256 * 256
    cell = torch.empty(int(ellmax) + 1, **f64)
    cell_dot = torch.empty((max(nd, 1), int(ellmax) + 1), **f64)
    cell_dns = torch.empty(int(ellmax) + 1, **f64)
    rc = lib.discoeb_los_cell_jvp(K, d_k.data_ptr(), T, d_tau.data_ptr(), d_S.data_ptr(), float(tau0), nd,
                                  d_td.data_ptr(), d_Sd.data_ptr(), t0d.ctypes.data, int(ellmax), int(n_fftlog),
                                  int(n_k_dense), float(n_s), float(k_p), aligned, int(nb), cell.data_ptr(),
                                  cell_dot.data_ptr(), cell_dns.data_ptr(), torch.cuda.current_stream(device).cuda_stream)
    if rc != 0:
        raise RuntimeError(f"discoeb_los_cell_jvp failed with code {rc}")
    return cell, cell_dot[:nd], cell_dns


def compute_Dell(Cell, A_s, Tcmb, ellmax=None):
    """D_l = l(l+1) C_l A_s 2 T_cmb^2 1e12 for l >= 2 (the reference's convention, cmb.py:876-927)."""
    C = Cell.detach().cpu().numpy() if hasattr(Cell, "detach") else np.asarray(Cell)
    if ellmax is None:
        ellmax = C.shape[0] - 1
    ell = np.arange(ellmax + 1)
    return ell[2:], ell[2:] * (ell[2:] + 1) * C[2:ellmax + 1] * A_s * 2 * Tcmb**2 * 1e12


def cmb_aexp_out(n_early=32, n_pre_recomb=64, n_recomb=128, n_post=96):
    """Output scale factors of compute_Cell_spectrum_from_cosmo_params (cmb.py:1006-1022)."""
    a_b1, a_b2, a_b3 = 1.0 / 3001.0, 1.0 / 1401.0, 1.0 / 601.0
    return np.concatenate([np.geomspace(1e-4, a_b1, n_early, endpoint=False),
                           np.geomspace(a_b1, a_b2, n_pre_recomb, endpoint=False),
                           np.geomspace(a_b2, a_b3, n_recomb, endpoint=False), np.geomspace(a_b3, 1.0, n_post)])


def compute_Cell_spectrum_from_cosmo_params(param_dict, ellmax=2500, nmodes=128, kmin=1e-4, kmax=1.0, n_k_dense=8192,
                                            n_fftlog=16384, lmaxg=11, lmaxgp=11, lmaxr=11, lmaxnu=8, nqmax=3,
                                            num_thermo=1024, rtol=1e-4, atol=1e-4, max_steps=2048,
                                            k_sampling_method="camb", aexp_out=None, device=None,
                                            return_intermediates=False, spectra=("TT",), fused_sources=False):
    """C_l^TT of a cosmology (cmb.py:931-1090): background (host), full perturbation solve,
    sources, FFTLog line of sight and C_l on the GPU, large arrays never leaving the device.

    Returns ``(Cell [ellmax+1] numpy, param)`` like the reference.  ``spectra`` naming more than TT
    (any of "TT", "TE", "EE"; the reference has temperature only) returns ``({name: Cell}, param)``
    with the E-mode multipoles from the same solve (compute_theta_ell(kind="E")).
    ``fused_sources``: the solve and the source assembly in one pass (solve_sources), the full
    states never written to device memory (the same sources; intermediates then hold no states).
    """
    spectra = tuple(spectra)
    if not spectra or any(x not in ("TT", "TE", "EE") for x in spectra):
        raise ValueError(f"spectra must name TT, TE and/or EE, not {spectra!r}")
    torch, device = _device(device)
    param = evolve_background(param=dict(param_dict), thermo_module="RECFAST", num_thermo=num_thermo)
    aexp_out = cmb_aexp_out() if aexp_out is None else np.asarray(aexp_out, dtype=np.float64)
    kmodes = k_sampling(param, kmin, kmax, nmodes, k_sampling_method)
    tau = param["tau_of_a_spline"].evaluate(aexp_out)
    L = dict(lmaxg=lmaxg, lmaxgp=lmaxgp, lmaxr=lmaxr, lmaxnu=lmaxnu, nqmax=nqmax)
    if fused_sources:
        y = None
        src = solve_sources(param=param, kmodes=kmodes, aexp_out=aexp_out, rtol=rtol, atol=atol, max_steps=max_steps,
                            device=device, **L)
    else:
        y = solve_modes(param=param, kmodes=kmodes, tau_out=tau, rtol=rtol, atol=atol, pcoeff=0.25, icoeff=0.80,
                        dcoeff=0.0, factormax=20.0, factormin=0.3, max_steps=max_steps, return_full=True,
                        device=device, as_tensor=True, **L)
        src = compute_sources(param=param, yout=y, kmodes=kmodes, aexp_out=aexp_out, device=device, **L)
    tau0 = float(param["tau_of_a_spline"].evaluate(1.0))
    theta = theta_e = None
    if "TT" in spectra or "TE" in spectra:
        theta, kk = compute_theta_ell(ellmax, kmodes, tau, src["S"], tau0, n_fftlog=n_fftlog, n_k_dense=n_k_dense,
                                      device=device)
    if "TE" in spectra or "EE" in spectra:
        theta_e, kk = compute_theta_ell(ellmax, kmodes, tau, src["E"], tau0, n_fftlog=n_fftlog,
                                        n_k_dense=n_k_dense, device=device, kind="E")
    cells = {}
    for name in spectra:
        a = theta if name[0] == "T" else theta_e
        b = None if name in ("TT", "EE") else theta_e
        cells[name] = compute_Cell(a, kk, param["n_s"], param["k_p"], device=device, theta_ell_b=b).cpu().numpy()
    for key, v in (("lmaxg", lmaxg), ("lmaxgp", lmaxgp), ("lmaxr", lmaxr), ("lmaxnu", lmaxnu), ("nqmax", nqmax),
                   ("nout", aexp_out.shape[0]), ("tau_out", tau)):
        param[key] = v
    out = cells["TT"] if spectra == ("TT",) else cells
    if return_intermediates:
        return out, param, {"kmodes": kmodes, "aexp_out": aexp_out, "tau": tau, "y": y, "sources": src,
                            "theta": theta, "theta_E": theta_e, "kmodes_los": kk}
    return out, param


def compute_Cell_sharded(param_dict, *, dist=None, device=None, ellmax=2500, nmodes=128, kmin=1e-4, kmax=1.0,
                         n_fftlog=16384, lmaxg=11, lmaxgp=11, lmaxr=11, lmaxnu=8, nqmax=3, num_thermo=1024, rtol=1e-4,
                         atol=1e-4, max_steps=2048, k_sampling_method="camb", aexp_out=None, spectra=("TT",)):
    """compute_Cell_spectrum_from_cosmo_params on the modes' own k grid (n_k_dense = 0) with the
    modes spread over the ranks of ``dist`` (a torch.distributed process group, one process per
    GPU): every rank solves its share of the modes (``replicas.shard``), takes their sources and
    line of sight (rows of the line of sight are independent on the modes' own grid) and its
    partial trapezoid sum over ln k of C_l, and the partial sums are added over the ranks
    (``replicas.sum_over_ranks``; ``device``: where the collective's tensor lives, the rank's GPU
    with NCCL, None with gloo).  Every rank returns the whole result, ``(Cell, param)`` as
    compute_Cell_spectrum_from_cosmo_params with ``n_k_dense=0`` (a dict of spectra when
    ``spectra`` names more than TT).  One process (dist None): the same computation on one GPU."""
    from . import replicas
    spectra = tuple(spectra)
    if not spectra or any(x not in ("TT", "TE", "EE") for x in spectra):
        raise ValueError(f"spectra must name TT, TE and/or EE, not {spectra!r}")
    torch, dev = _device(None)
    rank, world = (dist.get_rank(), dist.get_world_size()) if dist is not None else (0, 1)
    param = evolve_background(param=dict(param_dict), thermo_module="RECFAST", num_thermo=num_thermo)
    aexp_out = cmb_aexp_out() if aexp_out is None else np.asarray(aexp_out, dtype=np.float64)
    kmodes = k_sampling(param, kmin, kmax, nmodes, k_sampling_method)
    idx = replicas.shard(kmodes, rank, world)
    mine = kmodes[idx]
    tau = param["tau_of_a_spline"].evaluate(aexp_out)
    L = dict(lmaxg=lmaxg, lmaxgp=lmaxgp, lmaxr=lmaxr, lmaxnu=lmaxnu, nqmax=nqmax)
    # the trapezoid weights in ln k of the whole grid, for this rank's rows
    dlk = np.diff(np.log(kmodes))
    wt = np.zeros(kmodes.shape[0])
    wt[:-1] += 0.5 * dlk
    wt[1:] += 0.5 * dlk
    partial = {name: np.zeros(ellmax + 1) for name in spectra}
    if mine.shape[0] > 0:
        y = solve_modes(param=param, kmodes=mine, tau_out=tau, rtol=rtol, atol=atol, pcoeff=0.25, icoeff=0.80,
                        dcoeff=0.0, factormax=20.0, factormin=0.3, max_steps=max_steps, return_full=True,
                        device=dev, as_tensor=True, **L)
        src = compute_sources(param=param, yout=y, kmodes=mine, aexp_out=aexp_out, device=dev, **L)
        tau0 = float(param["tau_of_a_spline"].evaluate(1.0))
        th = {}
        if "TT" in spectra or "TE" in spectra:
            th["T"], _ = compute_theta_ell(ellmax, mine, tau, src["S"], tau0, n_fftlog=n_fftlog, n_k_dense=0,
                                           device=dev)
        if "TE" in spectra or "EE" in spectra:
            th["E"], _ = compute_theta_ell(ellmax, mine, tau, src["E"], tau0, n_fftlog=n_fftlog, n_k_dense=0,
                                           device=dev, kind="E")
        f64 = dict(dtype=torch.float64, device=dev)
        w = torch.as_tensor(wt[idx] * (mine / param["k_p"]) ** (param["n_s"] - 1.0), **f64)
        for name in spectra:
            partial[name] = (w[:, None] * th[name[0]] * th[name[1]]).sum(dim=0).cpu().numpy()
    cells = {name: replicas.sum_over_ranks(partial[name], dist, device) for name in spectra}
    for key, v in (("lmaxg", lmaxg), ("lmaxgp", lmaxgp), ("lmaxr", lmaxr), ("lmaxnu", lmaxnu), ("nqmax", nqmax),
                   ("nout", aexp_out.shape[0]), ("tau_out", tau)):
        param[key] = v
    return (cells["TT"] if spectra == ("TT",) else cells), param


def compute_Cell_jacobian(theta, *, ellmax=2500, nmodes=128, kmin=1e-4, kmax=1.0, n_k_dense=8192, n_fftlog=16384,
                          lmaxg=11, lmaxgp=11, lmaxr=11, lmaxnu=8, nqmax=3, num_thermo=1024, rtol=1e-4, atol=1e-4,
                          max_steps=2048, k_sampling_method="camb", aexp_out=None, de_guard_eps=1e-9, device=None,
                          rel_step=1e-4, los="tangent", sources="tangent", spectra=("TT",)):
    """C_l^TT and dC_l/dtheta for theta = (omega_c, omega_b, h, n_s, ln10As, w0, wa, m_nu)
    (``gradients.THETA_NAMES``), what ``jax.jacfwd`` of the reference's
    compute_Cell_spectrum_from_cosmo_params (cmb.py:931-1090) gives.

    The background and its six parameter tangents come from discoeb_background (forward mode,
    Recfast steps held), the perturbation states at every output time and their tangents from one
    discoeb_jvp_full launch (forward mode, accepted steps held).  The stages after the solve
    (sources, line of sight, C_l) involve no adaptive choice.  The sources' tangent along each
    direction: ``sources="tangent"`` in forward mode (discoeb_sources_jvp: y' and the source
    assembly in dual numbers from the state, output-time and table tangents; only the 1-D
    background rows, host tables, are differenced, centrally with the background moved by +-h
    along its exact tangent, h = ``rel_step`` max(|theta_d|, 0.01)), ``sources="differences"`` by a
    central difference of the whole source stage along the same tangents (O(h^2)).  The line of sight and C_l then take that tangent with the output
    times' and tau0's: ``los="tangent"`` in forward mode (discoeb_los_cell_jvp: the resampling, the
    FFT coefficients and the table M_l(p) differentiated as the FFTLog grid moves with tau0, one
    GEMM per direction), ``los="differences"`` by a fourth-order central difference along the
    first-order path (four lines of sight per direction; fourth order because the discrete C_l
    ripples as the grid moves: O(h^4) plus rounding, a few 1e-12 of C_l at low l, over h).
    n_s enters through the primordial weight of C_l alone (in closed form with ``los="tangent"``,
    by a fourth-order difference of compute_Cell with ``los="differences"``); C_l does not depend
    on A_s (D_l carries it).  The k sampling, start times and approximation switch times are held
    at the base point (the camb sampling's dependence on tau_maxvis is not differentiated).

    Returns ``(Cell [ellmax+1], J [8, ellmax+1], param)`` (numpy; param as
    compute_Cell_spectrum_from_cosmo_params returns it).

    ``spectra`` naming TE or EE (E-mode polarisation, which the reference does not compute) returns
    ``({name: Cell}, {name: J}, param)``: the E source and its tangent come from the same forward-mode
    solve and sources (discoeb_sources_jvp's SE_dot), and the E-mode line of sight and the cross and
    auto C_l along each direction's first-order path by fourth-order differences (as ``los=
    "differences"`` does for TT).
    """
    spectra = tuple(spectra)
    if not spectra or any(x not in ("TT", "TE", "EE") for x in spectra):
        raise ValueError(f"spectra must name TT, TE and/or EE, not {spectra!r}")
    pol = "TE" in spectra or "EE" in spectra
    from .background import _DIFF_FIELDS, background_from_buffer, native_background
    from .gradients import ODE_DIRECTIONS, THETA_NAMES, JacobianProblem, param_dots, theta_to_params
    if los not in ("tangent", "differences"):
        raise ValueError(f"los must be 'tangent' or 'differences', not {los!r}")
    if sources not in ("tangent", "differences"):
        raise ValueError(f"sources must be 'tangent' or 'differences', not {sources!r}")
    torch, device = _device(device)
    L = dict(lmaxg=lmaxg, lmaxgp=lmaxgp, lmaxr=lmaxr, lmaxnu=lmaxnu, nqmax=nqmax)
    aexp_out = cmb_aexp_out() if aexp_out is None else np.asarray(aexp_out, dtype=np.float64)
    p = theta_to_params(theta)
    pdots = param_dots(theta, ODE_DIRECTIONS)
    buf, bdots = native_background(p, num_thermo, pdots)
    bg = background_from_buffer(p, buf, num_thermo)
    kmodes = k_sampling(bg, kmin, kmax, nmodes, k_sampling_method)
    prob = JacobianProblem(theta, aexp_out=aexp_out, kmodes=kmodes, rtol=rtol, atol=atol, max_steps=max_steps,
                           num_thermo=num_thermo, de_guard_eps=de_guard_eps, device=device, full_state=True,
                           buffers=(buf, bdots), **L)
    prob.launch()
    if sources == "tangent":
        # the source stages run on the launch's row order (modes by descending k): the full states
        # and their tangents are read where the launch wrote them (no reordering copy of the
        # [K, nout, n] arrays, 7 GB per direction at l_max 50 and 2000 x 2000), and only the
        # [K, n_tau] source rows are put back into the caller's order
        y, k_rows, inv_rows = prob.launch_states()
    else:
        y, k_rows, inv_rows = prob.state(), kmodes, None

    def source_S(param, states):
        f = compute_sources(param=param, yout=states, kmodes=kmodes, aexp_out=aexp_out, de_guard_eps=de_guard_eps,
                            device=device, **L)
        return (f["S"], f["E"]) if pol else f["S"]

    def times(param):
        return param["tau_of_a_spline"].evaluate(aexp_out), float(param["tau_of_a_spline"].evaluate(1.0))

    def los_cell(S, tau, tau0):
        th, kk = compute_theta_ell(ellmax, kmodes, tau, S, tau0, n_fftlog=n_fftlog, n_k_dense=n_k_dense,
                                   device=device)
        return th, kk, compute_Cell(th, kk, bg["n_s"], bg["k_p"], device=device).cpu().numpy()

    fields0 = compute_sources(param=bg, yout=y, kmodes=k_rows, aexp_out=aexp_out, de_guard_eps=de_guard_eps,
                              device=device, **L)
    S0_rows = fields0["S"]  # the row order of y: the launch's (sources="tangent") or the caller's
    S0 = fields0["S"] if inv_rows is None else fields0["S"][inv_rows]
    SE0 = fields0["E"] if inv_rows is None else fields0["E"][inv_rows]

    def pol_cells(S, SE, tau, tau0):
        """C_l^TE and C_l^EE (numpy) of the line of sight of (S, S_E)."""
        out = {}
        the, kk = compute_theta_ell(ellmax, kmodes, tau, SE, tau0, n_fftlog=n_fftlog, n_k_dense=n_k_dense,
                                    device=device, kind="E")
        if "TE" in spectra:
            tht, _ = compute_theta_ell(ellmax, kmodes, tau, S, tau0, n_fftlog=n_fftlog, n_k_dense=n_k_dense,
                                       device=device)
            out["TE"] = compute_Cell(tht, kk, bg["n_s"], bg["k_p"], device=device, theta_ell_b=the)
        if "EE" in spectra:
            out["EE"] = compute_Cell(the, kk, bg["n_s"], bg["k_p"], device=device)
        return out
    tau_b, tau0_b = times(bg)
    if sources == "tangent":
        lib = _abi.lib()
        f64 = dict(dtype=torch.float64, device=device)
        K, T = S0.shape
        d_k = torch.from_numpy(np.ascontiguousarray(k_rows)).to(device)
        d_tau = torch.from_numpy(np.ascontiguousarray(tau_b)).to(device)
        d_bt = torch.from_numpy(background_table(aexp_out, tau_b, bg)).to(device)
    if los == "differences":
        th, kk, cell = los_cell(S0, tau_b, tau0_b)
    J = np.zeros((len(THETA_NAMES), ellmax + 1))
    Jp = {name: np.zeros((len(THETA_NAMES), ellmax + 1)) for name in ("TE", "EE") if name in spectra}
    stencil = ((2.0, -1.0 / 12.0), (1.0, 8.0 / 12.0), (-1.0, -8.0 / 12.0), (-2.0, 1.0 / 12.0))
    tangents = []

    def side_tables(di, name):
        """the direction's step h and the backgrounds moved by +-h along its exact tangent: their
        output times, tau0 and (sources="tangent") background rows, or (differences) sources"""
        h = rel_step * max(abs(float(theta[name])), 1e-2)
        side = []
        for sgn in (1.0, -1.0):
            ps = dict(p)
            for f in _DIFF_FIELDS:
                ps[f] = p[f] + sgn * h * pdots[di][f]
            bgs = background_from_buffer(ps, buf + sgn * h * bdots[di], num_thermo)
            tau_s, tau0_s = times(bgs)
            if sources == "tangent":  # the background rows of the sources, differenced on the host
                side.append((background_table(aexp_out, tau_s, bgs), tau_s, tau0_s))
            else:
                ydot = prob.state_tangent(di)
                side.append((source_S(bgs, torch.add(y, ydot, alpha=sgn * h)), tau_s, tau0_s))
                del ydot
        return h, side

    if sources == "tangent":
        # every direction's source tangents in one discoeb_sources_jvp call: one warp per (mode,
        # time) evaluates the base point's y' once and each direction's derivative after it
        ND = len(ODE_DIRECTIONS)
        sides = [side_tables(di, name) for di, name in enumerate(ODE_DIRECTIONS)]
        tau_dots = np.stack([(sd[0][1] - sd[1][1]) / (2 * h) for h, sd in sides])
        bt_dots = np.stack([(sd[0][0] - sd[1][0]) / (2 * h) for h, sd in sides])
        d_tau_dot = torch.from_numpy(np.ascontiguousarray(tau_dots)).to(device)
        d_bt_dot = torch.from_numpy(np.ascontiguousarray(bt_dots)).to(device)
        S_dot_all = torch.empty((ND, K, T), **f64)
        SE_dot_all = torch.empty((ND, K, T), **f64) if pol else None
        scratch = torch.empty(8 * ND * K * T, **f64)
        rc = lib.discoeb_sources_jvp(prob.dc.struct.data_ptr(), ctypes.byref(prob.dc.host), prob.d_tan.data_ptr(), ND,
                                     K, d_k.data_ptr(), T, d_tau.data_ptr(), d_tau_dot.data_ptr(), d_bt.data_ptr(),
                                     d_bt_dot.data_ptr(), y.data_ptr(), prob.d_outd.data_ptr(), S0_rows.data_ptr(),
                                     S_dot_all.data_ptr(), scratch.data_ptr(),
                                     SE_dot_all.data_ptr() if pol else None,
                                     torch.cuda.current_stream(device).cuda_stream)
        if rc != 0:
            raise RuntimeError(f"discoeb_sources_jvp failed with code {rc}")
        del scratch
    for di, name in enumerate(ODE_DIRECTIONS):
        if sources == "tangent":
            h, side = sides[di]
        else:
            h, side = side_tables(di, name)
        tau_dot = (side[0][1] - side[1][1]) / (2 * h)
        tau0_dot = (side[0][2] - side[1][2]) / (2 * h)
        SE_dot = None
        if sources == "tangent":
            S_dot = S_dot_all[di][inv_rows]
            SE_dot = SE_dot_all[di][inv_rows] if pol else None
        elif pol:
            S_dot = (side[0][0][0] - side[1][0][0]) / (2 * h)
            SE_dot = (side[0][0][1] - side[1][0][1]) / (2 * h)
        else:
            S_dot = (side[0][0] - side[1][0]) / (2 * h)
        del side
        if pol:  # E-mode line of sight and C_l^TE / C_l^EE along the path, fourth order
            acc = {sp: 0.0 for sp in Jp}
            for m, wgt in stencil:
                pc = pol_cells(torch.add(S0, S_dot, alpha=m * h), torch.add(SE0, SE_dot, alpha=m * h),
                               tau_b + m * h * tau_dot, tau0_b + m * h * tau0_dot)
                for sp in Jp:
                    acc[sp] = acc[sp] + wgt * pc[sp].cpu().numpy()
            for sp in Jp:
                Jp[sp][THETA_NAMES.index(name)] = acc[sp] / h
            del SE_dot
        if los == "tangent":
            tangents.append((S_dot, tau_dot, tau0_dot))
            continue
        # the line of sight and C_l along that first-order path (the derivative at the base point
        # depends on the path's slope only): fourth order, the discrete C_l ripples in tau0
        acc = np.zeros(ellmax + 1)
        for m, wgt in stencil:
            acc += wgt * los_cell(torch.add(S0, S_dot, alpha=m * h), tau_b + m * h * tau_dot,
                                  tau0_b + m * h * tau0_dot)[2]
        J[THETA_NAMES.index(name)] = acc / h
    if los == "tangent":
        cell, cdot, cdns = compute_Cell_tangent(ellmax, kmodes, tau_b, S0, tau0_b, bg["n_s"], bg["k_p"],
                                                np.stack([t[1] for t in tangents]),
                                                torch.stack([t[0] for t in tangents]),
                                                np.array([t[2] for t in tangents]), n_fftlog=n_fftlog,
                                                n_k_dense=n_k_dense, device=device)
        cell, cdot = cell.cpu().numpy(), cdot.cpu().numpy()
        for di, name in enumerate(ODE_DIRECTIONS):
            J[THETA_NAMES.index(name)] = cdot[di]
        J[THETA_NAMES.index("n_s")] = cdns.cpu().numpy()
    else:
        h = rel_step * max(abs(float(bg["n_s"])), 1e-2)
        acc = np.zeros(ellmax + 1)
        for m, wgt in stencil:
            acc += wgt * compute_Cell(th, kk, bg["n_s"] + m * h, bg["k_p"], device=device).cpu().numpy()
        J[THETA_NAMES.index("n_s")] = acc / h
    param = dict(bg)
    for key, v in (("lmaxg", lmaxg), ("lmaxgp", lmaxgp), ("lmaxr", lmaxr), ("lmaxnu", lmaxnu), ("nqmax", nqmax),
                   ("nout", aexp_out.shape[0]), ("tau_out", bg["tau_of_a_spline"].evaluate(aexp_out))):
        param[key] = v
    if not pol:
        return cell, J, param
    cells, jacs = {}, {}
    if "TT" in spectra:
        cells["TT"], jacs["TT"] = cell, J
    # the base point's polarisation spectra, and their n_s row (the primordial weight alone)
    the, kk = compute_theta_ell(ellmax, kmodes, tau_b, SE0, tau0_b, n_fftlog=n_fftlog, n_k_dense=n_k_dense,
                                device=device, kind="E")
    tht = None
    if "TE" in spectra:
        tht, _ = compute_theta_ell(ellmax, kmodes, tau_b, S0, tau0_b, n_fftlog=n_fftlog, n_k_dense=n_k_dense,
                                   device=device)
    h = rel_step * max(abs(float(bg["n_s"])), 1e-2)
    for sp in Jp:
        a, b = (tht, the) if sp == "TE" else (the, None)
        cells[sp] = compute_Cell(a, kk, bg["n_s"], bg["k_p"], device=device, theta_ell_b=b).cpu().numpy()
        acc = np.zeros(ellmax + 1)
        for m, wgt in stencil:
            acc += wgt * compute_Cell(a, kk, bg["n_s"] + m * h, bg["k_p"], device=device,
                                      theta_ell_b=b).cpu().numpy()
        Jp[sp][THETA_NAMES.index("n_s")] = acc / h
        jacs[sp] = Jp[sp]
    return {sp: cells[sp] for sp in spectra}, {sp: jacs[sp] for sp in spectra}, param


def cell_spectrum_function(**options):
    """A ``torch.autograd.Function`` mapping theta (float64[8], ``gradients.THETA_NAMES`` order)
    to C_l^TT (float64[ellmax+1]).

    The forward pass runs compute_Cell_jacobian and keeps the Jacobian; the backward pass
    contracts it with the incoming gradient, so ``torch.autograd`` sees the derivative of the
    discrete chain (for a likelihood of C_l, or of D_l = l(l+1) C_l A_s 2 T_cmb^2 1e12 built from
    it with A_s = exp(theta[4]) / 1e10).  ``options`` are those of compute_Cell_jacobian.
    """
    import torch

    from .gradients import THETA_NAMES

    class CellSpectrum(torch.autograd.Function):
        @staticmethod
        def forward(ctx, theta):
            if theta.shape != (len(THETA_NAMES),):
                raise ValueError(f"theta must have shape ({len(THETA_NAMES)},) in the order {THETA_NAMES}")
            th = dict(zip(THETA_NAMES, theta.detach().to("cpu", torch.float64).tolist()))
            C, J, _ = compute_Cell_jacobian(th, **options)
            ctx.save_for_backward(torch.from_numpy(J).to(theta.device))
            return torch.from_numpy(C).to(theta.device)

        @staticmethod
        def backward(ctx, grad_C):
            (J,) = ctx.saved_tensors
            return J @ grad_C.to(J.dtype)

    return CellSpectrum
