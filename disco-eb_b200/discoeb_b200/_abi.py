"""ctypes mirror of ``include/discoeb.h`` and the loader of the CUDA library.

The shared library ``libdiscoeb_b200.so`` is built in-tree by ``build.py``.  There is
no CPU fallback: if the library (or a GPU) is missing, the entry points raise.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

MAX_NQ = 16
ABI_VERSION = 1
HERE = os.path.dirname(os.path.abspath(__file__))
LIB_NAME = "libdiscoeb_b200.so"
LIB_PATH = os.path.join(HERE, LIB_NAME)

METHOD_RODAS5_STRUCTURED = 0
METHOD_RODAS5_DENSE = 1
METHOD_RODAS5_DENSE_MIXED = 2
METHOD_RODAS5_STRUCTURED_MIXED = 3

STATUS_NAMES = {0: "ok", 1: "max_steps exceeded", 2: "non-finite state", 3: "step size underflow", 4: "singular",
                5: "cosmology index out of range",
                6: "aborted (a cooperating warp gave up waiting)",
                7: "step record full (raise step_capacity)"}

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int32)


class DiscoebSpline(ctypes.Structure):
    _fields_ = [("n_knots", ctypes.c_int32), ("uniform", ctypes.c_int32),
                ("x", ctypes.c_void_p), ("y", ctypes.c_void_p), ("S", ctypes.c_void_p)]


class DiscoebCosmo(ctypes.Structure):
    _fields_ = ([(f, ctypes.c_int32) for f in ("lmaxg", "lmaxgp", "lmaxr", "lmaxnu", "nqmax",
                                                "use_tca", "use_rsa", "use_ufa")]
                + [(f, ctypes.c_double) for f in ("tca_tau_c_over_tau_h", "tca_tau_c_over_tau_k",
                                                   "rsa_tau_c_over_tau", "rsa_tau_over_tau_k", "ufa_tau_over_tau_k",
                                                   "grhom", "grhog", "grhor", "Omegam", "Omegab", "OmegaDE", "Omegak",
                                                   "Neff", "Nmnu", "amnu", "w0", "wa", "cs2_DE", "YHe", "H0",
                                                   "de_guard_eps")]
                + [("q", ctypes.c_double * MAX_NQ), ("wq", ctypes.c_double * MAX_NQ)]
                + [(f, DiscoebSpline) for f in ("xe_loga", "cs2a_loga", "logrhonu_loga", "logpnu_loga")])


class DiscoebTangent(ctypes.Structure):
    _fields_ = ([(f, ctypes.c_double) for f in ("grhom", "Omegam", "Omegab", "OmegaDE", "amnu", "w0", "wa", "H0")]
                + [(f, ctypes.c_void_p) for f in ("xe_y", "xe_S", "cs2a_y", "cs2a_S", "logrhonu_y", "logrhonu_S",
                                                   "logpnu_y", "logpnu_S")])


class DiscoebControl(ctypes.Structure):
    _fields_ = ([(f, ctypes.c_double) for f in ("rtol", "atol", "pcoeff", "icoeff", "dcoeff", "factormax", "factormin")]
                + [(f, ctypes.c_int32) for f in ("max_steps", "method", "warps_per_block", "max_polls")])


class DiscoebCosmoParams(ctypes.Structure):
    _fields_ = [(f, ctypes.c_double) for f in ("H0", "Omegab", "Omegam", "mnu", "w_DE_0", "w_DE_a", "Tcmb", "YHe",
                                                "Neff", "Nmnu", "cs2_DE", "Omegak")]


# discoeb_background output layout (the DISCOEB_BGS_* / DISCOEB_BGN_* / DISCOEB_BGT_* enums)
NU_KNOTS = 512
BGS = ("amin", "amax", "grhom", "grhog", "grhor", "adotrad", "amnu", "Omegamnu", "OmegaDE", "taumin", "taumax", "fHe",
       "tau0", "tau_maxvis", "H0", "Omegab", "Omegam", "mnu", "w_DE_0", "w_DE_a")
BGN = ("a", "loga", "logrhonu_y", "logrhonu_S", "logpnu_y", "logpnu_S", "logppnu_y", "logppnu_S")
BGT = ("aexp", "loga", "tau", "xe", "xeHI", "xeHeI", "xeHeII", "cs2", "Tm", "mu", "xeprime_recf", "cs2a", "tempba",
       "tau_of_a_S", "a_of_tau_S", "xe_of_tau_S", "cs2a_of_tau_S", "tempba_of_tau_S", "xe_of_loga_S", "cs2a_of_loga_S",
       "opac", "opac_S", "optical_depth", "gvis", "gvisprime", "gvispprime", "xeprime", "rec_case", "rec_steps")


def background_layout(num_thermo):
    """Split of one discoeb_background output buffer: {name: slice} for the scalars (``s:``),
    the neutrino tables (``n:``) and the Recfast-grid tables (``t:``), and the total size."""
    out, o = {}, 0
    for nm in BGS:
        out["s:" + nm] = o
        o += 1
    for nm in BGN:
        out["n:" + nm] = slice(o, o + NU_KNOTS)
        o += NU_KNOTS
    for nm in BGT:
        out["t:" + nm] = slice(o, o + num_thermo)
        o += num_thermo
    return out, o


def nvar(lmaxg, lmaxgp, lmaxr, lmaxnu, nqmax):
    return 7 + (lmaxg + 1) + (lmaxgp + 1) + (lmaxr + 1) + nqmax * (lmaxnu + 1) + 2


def approximation_settings(param):
    """Defaults of get_approximation_settings (src/discoeb/approximations.py:9-20)."""
    return {
        "use_tca": bool(param.get("use_tca", False)),
        "tca_tau_c_over_tau_h_trigger": float(param.get("tca_tau_c_over_tau_h_trigger", 0.015)),
        "tca_tau_c_over_tau_k_trigger": float(param.get("tca_tau_c_over_tau_k_trigger", 0.010)),
        "use_rsa": bool(param.get("use_rsa", True)),
        "tau_c_over_tau_trigger": float(param.get("rsa_tau_c_over_tau_trigger", 10.0)),
        "tau_over_tau_k_trigger": float(param.get("rsa_tau_over_tau_k_trigger", 80.0)),
        "use_ur_fluid": bool(param.get("use_ur_fluid", True)),
        "ur_fluid_tau_over_tau_k_trigger": float(param.get("ur_fluid_tau_over_tau_k_trigger", 120.0)),
    }


def make_cosmo(param, *, lmaxg, lmaxgp, lmaxr, lmaxnu, nqmax, de_guard_eps, table_ptrs):
    """Fill a DiscoebCosmo from a background ``param`` dict.

    ``table_ptrs`` maps spline keys to (n, uniform, x_ptr, y_ptr, S_ptr) with pointers
    valid where the struct is consumed (device pointers for the CUDA library).
    """
    from .background import get_neutrino_momentum_bins
    if nqmax > MAX_NQ:
        raise ValueError(f"nqmax={nqmax} exceeds the supported maximum {MAX_NQ}")
    if min(lmaxg, lmaxgp, lmaxr, lmaxnu) < 3:
        raise ValueError("lmaxg, lmaxgp, lmaxr and lmaxnu must be >= 3")
    s = approximation_settings(param)
    c = DiscoebCosmo()
    c.lmaxg, c.lmaxgp, c.lmaxr, c.lmaxnu, c.nqmax = lmaxg, lmaxgp, lmaxr, lmaxnu, nqmax
    c.use_tca = int(s["use_tca"])
    c.use_rsa = int(s["use_rsa"])
    c.use_ufa = int(s["use_ur_fluid"])
    c.tca_tau_c_over_tau_h = s["tca_tau_c_over_tau_h_trigger"]
    c.tca_tau_c_over_tau_k = s["tca_tau_c_over_tau_k_trigger"]
    c.rsa_tau_c_over_tau = s["tau_c_over_tau_trigger"]
    c.rsa_tau_over_tau_k = s["tau_over_tau_k_trigger"]
    c.ufa_tau_over_tau_k = s["ur_fluid_tau_over_tau_k_trigger"]
    for f in ("grhom", "grhog", "grhor", "Omegam", "Omegab", "OmegaDE", "Omegak", "Neff", "Nmnu", "amnu",
              "cs2_DE", "YHe", "H0"):
        setattr(c, f, float(param[f]))
    c.w0 = float(param["w_DE_0"])
    c.wa = float(param["w_DE_a"])
    c.de_guard_eps = float(de_guard_eps)
    q, w = get_neutrino_momentum_bins(nqmax)
    for i in range(nqmax):
        c.q[i] = float(q[i])
        c.wq[i] = float(w[i])
    for name, key in (("xe_loga", "xe_of_loga_spline"), ("cs2a_loga", "cs2a_of_loga_spline"),
                      ("logrhonu_loga", "logrhonu_of_loga_spline"), ("logpnu_loga", "logpnu_of_loga_spline")):
        n, uni, xp, yp, sp = table_ptrs[key]
        setattr(c, name, DiscoebSpline(n, uni, xp, yp, sp))
    return c


_lib = None


def lib():
    """Load the CUDA library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_NAME} not found at {LIB_PATH}: build it with disco-eb_b200/build.py "
                               "(there is no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        L.discoeb_abi_version.restype = ctypes.c_int32
        L.discoeb_nvar.argtypes = [ctypes.POINTER(DiscoebCosmo)]
        L.discoeb_nvar.restype = ctypes.c_int32
        vp = ctypes.c_void_p
        L.discoeb_fwd.argtypes = [vp, ctypes.POINTER(DiscoebCosmo), ctypes.c_int32, ctypes.POINTER(DiscoebControl),
                                  ctypes.c_int32, vp, vp, vp, vp, vp, ctypes.c_int32, vp, vp, vp, vp, vp, vp]
        L.discoeb_fwd.restype = ctypes.c_int32
        L.discoeb_rhs.argtypes = [vp, ctypes.POINTER(DiscoebCosmo), ctypes.c_int32, vp, vp, vp, ctypes.c_int32, vp, vp]
        L.discoeb_jvp.argtypes = [vp, ctypes.POINTER(DiscoebCosmo), ctypes.c_int32, vp, vp, ctypes.c_int32,
                                  ctypes.POINTER(DiscoebControl), ctypes.c_int32, vp, vp, vp, vp, vp, ctypes.c_int32,
                                  vp, vp, vp, vp, vp, vp, vp]
        L.discoeb_jvp.restype = ctypes.c_int32
        i32, i64 = ctypes.c_int32, ctypes.c_int64
        CPp, CTp = ctypes.POINTER(DiscoebCosmo), ctypes.POINTER(DiscoebControl)
        L.discoeb_step_record_doubles.argtypes = [i32, i32, i32]
        L.discoeb_step_record_doubles.restype = i64
        L.discoeb_fwd_record.argtypes = [vp, CPp, i32, CTp, i32, vp, vp, vp, vp, vp, i32, vp, vp, vp, vp, i32, i32, vp, vp,
                                         vp]
        L.discoeb_fwd_record.restype = i32
        L.discoeb_bwd_workspace_bytes.argtypes = [CPp, i32, i32]
        L.discoeb_bwd_workspace_bytes.restype = i64
        L.discoeb_bwd.argtypes = [vp, CPp, i32, vp, i32, vp, vp, vp, i32, vp, i32, i32, vp, vp, vp, vp, vp, vp, vp, vp,
                                  i32, i32, vp, i64, vp, vp]
        L.discoeb_bwd.restype = i32
        L.discoeb_bwd_contract.argtypes = [vp, i32, vp, i32, i32, i32, vp, i32, vp, vp, vp, vp, vp, vp, i32, i32, vp,
                                           vp]
        L.discoeb_bwd_contract.restype = i32
        L.discoeb_los_e_workspace_bytes.argtypes = [i32, i32, i32, i32, i32]
        L.discoeb_los_e_workspace_bytes.restype = i64
        L.discoeb_los_e.argtypes = [i32, vp, i32, vp, vp, ctypes.c_double, i32, i32, i32, vp, i64, vp, vp, vp]
        L.discoeb_los_e.restype = i32
        L.discoeb_cell_cross.argtypes = [i32, vp, i32, vp, vp, ctypes.c_double, ctypes.c_double, vp, vp]
        L.discoeb_cell_cross.restype = i32
        L.discoeb_jvp_full.argtypes = L.discoeb_jvp.argtypes
        L.discoeb_jvp_full.restype = ctypes.c_int32
        L.discoeb_jvp_records_bytes.argtypes = [ctypes.POINTER(DiscoebCosmo), ctypes.c_int32, ctypes.c_int32]
        L.discoeb_jvp_records_bytes.restype = ctypes.c_int64
        L.discoeb_jvp_split_records_bytes.argtypes = [ctypes.POINTER(DiscoebCosmo), ctypes.c_int32, ctypes.c_int32]
        L.discoeb_jvp_split_records_bytes.restype = ctypes.c_int64
        L.discoeb_jvp_records.argtypes = L.discoeb_jvp.argtypes[:-1] + [ctypes.c_int32, vp, ctypes.c_int64, vp]
        L.discoeb_jvp_records.restype = ctypes.c_int32
        L.discoeb_rhs.restype = ctypes.c_int32
        L.discoeb_sources.argtypes = [vp, ctypes.POINTER(DiscoebCosmo), ctypes.c_int32, vp, ctypes.c_int32, vp, vp, vp,
                                      vp, vp, vp]
        L.discoeb_sources.restype = ctypes.c_int32
        L.discoeb_sources_noalloc.argtypes = [vp, ctypes.POINTER(DiscoebCosmo), ctypes.c_int32, vp, ctypes.c_int32, vp,
                                              vp, vp, vp, vp]
        L.discoeb_sources_noalloc.restype = ctypes.c_int32
        L.discoeb_fwd_sources.argtypes = [vp, ctypes.POINTER(DiscoebCosmo), ctypes.POINTER(DiscoebControl),
                                          ctypes.c_int32, vp, vp, vp, vp, ctypes.c_int32, vp, vp, vp, vp, vp, vp, vp, vp]
        L.discoeb_fwd_sources.restype = ctypes.c_int32
        L.discoeb_los_workspace_bytes.argtypes = [ctypes.c_int32] * 5
        L.discoeb_los_workspace_bytes.restype = ctypes.c_int64
        L.discoeb_los.argtypes = [ctypes.c_int32, vp, ctypes.c_int32, vp, vp, ctypes.c_double, ctypes.c_int32,
                                  ctypes.c_int32, ctypes.c_int32, vp, ctypes.c_int64, vp, vp, vp]
        L.discoeb_los.restype = ctypes.c_int32
        L.discoeb_set_los_contraction.argtypes = [ctypes.c_int32, ctypes.c_int32]
        L.discoeb_set_los_contraction.restype = ctypes.c_int32
        L.discoeb_get_los_contraction.argtypes = [ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32)]
        L.discoeb_get_los_contraction.restype = ctypes.c_int32
        L.discoeb_dgemm_i8_workspace_bytes.argtypes = [ctypes.c_int32] * 5
        L.discoeb_dgemm_i8_workspace_bytes.restype = ctypes.c_int64
        L.discoeb_dgemm_i8.argtypes = [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, vp, ctypes.c_int64,
                                       ctypes.c_int32, vp, ctypes.c_int64, ctypes.c_int32, vp, ctypes.c_int64,
                                       ctypes.c_int32, ctypes.c_int32, vp, ctypes.c_int64, vp]
        L.discoeb_dgemm_i8.restype = ctypes.c_int32
        L.discoeb_cell.argtypes = [ctypes.c_int32, vp, ctypes.c_int32, vp, ctypes.c_double, ctypes.c_double, vp, vp]
        L.discoeb_sources_jvp.argtypes = [vp, ctypes.POINTER(DiscoebCosmo), vp, ctypes.c_int32, ctypes.c_int32, vp,
                                          ctypes.c_int32, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp]
        L.discoeb_sources_jvp.restype = ctypes.c_int32
        L.discoeb_los_cell_jvp_workspace_bytes.argtypes = [ctypes.c_int32] * 5
        L.discoeb_los_cell_jvp_workspace_bytes.restype = ctypes.c_int64
        L.discoeb_los_cell_jvp.argtypes = [ctypes.c_int32, vp, ctypes.c_int32, vp, vp, ctypes.c_double, ctypes.c_int32,
                                           vp, vp, vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_double,
                                           ctypes.c_double, vp, ctypes.c_int64, vp, vp, vp, vp]
        L.discoeb_los_cell_jvp.restype = ctypes.c_int32
        L.discoeb_cell.restype = ctypes.c_int32
        c32, c64, cd = ctypes.c_int32, ctypes.c_int64, ctypes.c_double
        L.discoeb_power_amplitudes.argtypes = [c32, vp, vp, c32, c32, cd, cd, cd, c32, vp, vp]
        L.discoeb_savgol_log_power.argtypes = [c32, vp, c32, vp, vp, vp]
        L.discoeb_power_kaiser.argtypes = [c32, vp, vp, cd, c32, vp, vp, vp]
        L.discoeb_power_multipoles.argtypes = [c32, vp, vp, cd, vp, vp, vp, vp]
        L.discoeb_xi_workspace_bytes.argtypes = [c32]
        L.discoeb_xi_workspace_bytes.restype = c64
        L.discoeb_xi_from_power.argtypes = [c32, vp, vp, c32, vp, c64, vp, vp, vp]
        for nm in ("discoeb_power_amplitudes", "discoeb_savgol_log_power", "discoeb_power_kaiser",
                   "discoeb_power_multipoles", "discoeb_xi_from_power"):
            getattr(L, nm).restype = c32
        L.discoeb_background_size.argtypes = [ctypes.c_int32]
        L.discoeb_background_size.restype = ctypes.c_int64
        L.discoeb_background.argtypes = [ctypes.POINTER(DiscoebCosmoParams), vp, ctypes.c_int32, ctypes.c_int32, vp, vp,
                                         ctypes.c_int32]
        L.discoeb_background.restype = ctypes.c_int32
        L.discoeb_background_batch_workspace_bytes.argtypes = [c32, c32, c32]
        L.discoeb_background_batch_workspace_bytes.restype = c64
        L.discoeb_background_batch.argtypes = [vp, vp, c32, c32, c32, vp, c64, vp, vp, vp]
        L.discoeb_background_batch.restype = c32
        L.discoeb_natural_spline_second.argtypes = [c32, vp, vp, vp]
        L.discoeb_natural_spline_second.restype = c32
        L.discoeb_fma_rate_threads.argtypes = []
        L.discoeb_fma_rate_threads.restype = c64
        L.discoeb_fma_rate.argtypes = [c64, vp, c64, ctypes.POINTER(ctypes.c_double), vp]
        L.discoeb_fma_rate.restype = c32
        if L.discoeb_abi_version() != ABI_VERSION:
            raise RuntimeError("libdiscoeb_b200.so ABI version mismatch; rebuild it")
        _lib = L
    return _lib


def host_table_ptrs(param, keep):
    """Table pointers into host numpy arrays (for the CPU model test harness)."""
    out = {}
    for key in ("xe_of_loga_spline", "cs2a_of_loga_spline", "logrhonu_of_loga_spline", "logpnu_of_loga_spline"):
        s = param[key]
        arrs = [np.ascontiguousarray(s.x, dtype=np.float64), np.ascontiguousarray(s.y, dtype=np.float64),
                np.ascontiguousarray(s.S, dtype=np.float64)]
        keep.extend(arrs)
        out[key] = (s.n, int(s.uniform), arrs[0].ctypes.data, arrs[1].ctypes.data, arrs[2].ctypes.data)
    # xe and cs2*a are tabulated on the same knots: share the x pointer so the kernel does one search
    xe, cs = param["xe_of_loga_spline"], param["cs2a_of_loga_spline"]
    if xe.n == cs.n and np.array_equal(xe.x, cs.x):
        n, u, _, yp, sp = out["cs2a_of_loga_spline"]
        out["cs2a_of_loga_spline"] = (n, u, out["xe_of_loga_spline"][2], yp, sp)
    rn, rp = param["logrhonu_of_loga_spline"], param["logpnu_of_loga_spline"]
    if rn.n == rp.n and np.array_equal(rn.x, rp.x):
        n, u, _, yp, sp = out["logpnu_of_loga_spline"]
        out["logpnu_of_loga_spline"] = (n, u, out["logrhonu_of_loga_spline"][2], yp, sp)
    return out
