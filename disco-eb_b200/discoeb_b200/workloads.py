"""Named workloads: cosmologies and solver settings of the measured problems.

Cosmological parameters are given as (h, omega_b, omega_c, A_s, n_s, ...) and mapped to
the reference's parameter dict: H0 = 100 h, Omegab = omega_b/h^2,
Omegam = (omega_b + omega_c)/h^2 (massive neutrinos are not part of Omegam,
background.py:170-178), YHe = 0.248 and cs2_DE = 1 as in the reference's tests.  The
reference has no reionisation, so tau_reio has no counterpart and is not used.
"""
from __future__ import annotations

import numpy as np


def cosmo_params(*, h=0.674, omega_b=0.0224, omega_c=0.120, A_s=2.1e-9, n_s=0.965, Tcmb=2.7255, Neff=3.046,
                 m_nu=0.0, w0=-1.0, wa=0.0, YHe=0.248, cs2_DE=1.0, k_p=0.05):
    """Reference param dict; ``m_nu > 0`` adds one massive species and moves one unit of
    N_eff from the massless to the massive sector (the reference tests' convention)."""
    massive = bool(np.real(m_nu) > 0.0)
    return {
        "Omegam": (omega_b + omega_c) / h**2,
        "Omegab": omega_b / h**2,
        "H0": 100.0 * h,
        "n_s": n_s,
        "A_s": A_s,
        "mnu": m_nu,
        "Tcmb": Tcmb,
        "YHe": YHe,
        "Neff": Neff - 1.0 if massive else Neff,
        "Nmnu": 1 if massive else 0,
        "w_DE_0": w0,
        "w_DE_a": wa,
        "cs2_DE": cs2_DE,
        "Omegak": 0.0,
        "k_p": k_p,
    }


# z in {2, 1, 0.5, 0} as increasing scale factors
A_OUT_4Z = np.array([1.0 / 3.0, 0.5, 2.0 / 3.0, 1.0])

# w0 of the cosmological-constant workloads.  The reference's dark-energy fluid equations divide by
# 1 + w (perturbations.py:521-523: NaN at w = -1 exactly), so its LCDM point is taken at
# w0 = -1 + 1e-6, where they are regular: P(k) equals the w = -1 limit to < 1e-6 (the same step
# counts), and dP/dw0, dP/dwa include the fluid's clustering response, as the limit does (the
# solver's guard at w = -1 exactly would hold the fluid's perturbations at zero and drop it).
W0_LCDM = -1.0 + 1e-6

WORKLOADS = {
    # flat LCDM, massless neutrinos only, P(k, z=0) on 128 log-spaced modes
    "pk_lcdm_massless_k128": dict(
        cosmo=dict(w0=W0_LCDM), theta=dict(m_nu=0.0, w0=W0_LCDM, wa=0.0), kmin=1e-4, kmax=1.0, num_k=128, aexp_out=np.array([1.0]),
        lmaxg=12, lmaxgp=12, lmaxr=17, lmaxnu=3, nqmax=3, rtol=1e-5, atol=1e-8),
    # + one 0.06 eV neutrino (5 momentum bins, l_max 17): 512 modes to k = 10/Mpc, P(k) at z = 0, 0.5, 1, 2
    "pk_lcdm_mnu_k512_z4": dict(
        cosmo=dict(m_nu=0.06, w0=W0_LCDM), theta=dict(m_nu=0.06, w0=W0_LCDM, wa=0.0), kmin=1e-4, kmax=10.0, num_k=512, aexp_out=A_OUT_4Z,
        lmaxg=12, lmaxgp=12, lmaxr=17, lmaxnu=17, nqmax=5, rtol=1e-5, atol=1e-8),
}


# the LCDM point of both workloads as theta = (omega_c, omega_b, h, n_s, ln(10^10 A_s), w0, wa, m_nu)
_THETA_LCDM = dict(omega_c=0.120, omega_b=0.0224, h=0.674, n_s=0.965, ln10As=float(np.log(2.1e-9 * 1e10)))


def workload(name):
    w = dict(WORKLOADS[name])
    w["param"] = cosmo_params(**w.pop("cosmo"))
    w["theta"] = dict(_THETA_LCDM, **w["theta"])
    return w


# the uneven-batch box: theta ranges of the many-cosmology workload
THETA_BOX = {"omega_c": (0.10, 0.14), "omega_b": (0.020, 0.025), "h": (0.60, 0.76), "n_s": (0.92, 1.00),
             "ln10As": (2.9, 3.2), "w0": (-1.3, -0.7), "wa": (-0.5, 0.5), "m_nu": (0.02, 0.3)}


def sample_thetas(n, seed=0):
    """n cosmologies drawn uniformly from THETA_BOX with numpy's default_rng(seed)."""
    rng = np.random.default_rng(seed)
    names = list(THETA_BOX)
    u = rng.uniform(size=(n, len(names)))
    return [{nm: THETA_BOX[nm][0] + (THETA_BOX[nm][1] - THETA_BOX[nm][0]) * u[i, j] for j, nm in enumerate(names)}
            for i in range(n)]


def crosses_phantom_divide(theta):
    """Whether w(a) = w0 + wa (1 - a) equals -1 for some a in (0, 1]."""
    w_early, w_today = theta["w0"] + theta["wa"], theta["w0"]
    return (w_early + 1.0) * (w_today + 1.0) <= 0.0
