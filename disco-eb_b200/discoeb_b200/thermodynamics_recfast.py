"""Recfast recombination history (host side, float64 numpy).

Restates ``src/discoeb/thermodynamics_recfast.py`` of the reference: the three-variable
Recfast ODE (x_H, x_He, T_mat) of Seager, Sasselov & Scott (1999, 2000) with the
Wong, Moss & Scott (2008) fudges, integrated interval by interval on the adaptive
a-grid with the Kaps-Rentrop GRK4A Rosenbrock method and a PI step controller,
plus the Saha HeII correction.  This is the producer of the ``xe`` and ``c_s^2``
tables that the perturbation kernels read; it is not on the device path.

The Jacobian of the GRK4A step is taken by complex-step differentiation, which gives
the exact derivative to rounding, as the reference's forward-mode ``jacfwd`` does.
"""
from __future__ import annotations

import math

import numpy as np

from .romberg import romb

# physical constants (thermodynamics_recfast.py:38-53)
const_G = 6.67430e-11
const_mH = 1.67353284e-27
const_me = 9.1093837015e-31
const_mHe_mH = 3.97146570884
const_c = 2.99792458e08
const_h = 6.62607015e-34
const_kB = 1.380649e-23
const_sigma = 6.6524587321e-29
const_arad = 4 * 5.670374419e-8 / const_c
bigH = 3.2407792902755102e-18
const_dens_fac = 11.223810928601939
const_c2ok = 1.62581581e4
const_c_Mpc_s = 9.71561189e-15
const_EionHe12s = 6.314878282674e5

# atomic data (thermodynamics_recfast.py:57-122)
Lambda = 8.2245809
Lambda_He = 51.3
L_H_ion = 1.096787737e7
L_H_alpha = 8.225916453e6
L_He1_ion = 1.98310772e7
L_He2_ion = 4.389088863e7
L_He_2s = 1.66277434e7
L_He_2p = 1.71134891e7
A2P_s = 1.798287e9
A2P_t = 177.58
L_He_2Pt = 1.690871466e7
L_He_2St = 1.5985597526e7
L_He2St_ion = 3.8454693845e6
sigma_He_2Ps = 1.436289e-22
sigma_He_2Pt = 1.484872e-22
AGauss1 = -0.14
AGauss2 = 0.05
zGauss1 = 7.28
zGauss2 = 6.75
wGauss1 = 0.18
wGauss2 = 0.33
H_frac = 1.0e-3

Lalpha = 1.0 / L_H_alpha
Lalpha_He = 1.0 / L_He_2p
DeltaB = const_h * const_c * (L_H_ion - L_H_alpha)
CDB = DeltaB / const_kB
DeltaB_He = const_h * const_c * (L_He1_ion - L_He_2s)
CDB_He = DeltaB_He / const_kB
CB1 = const_h * const_c * L_H_ion / const_kB
CB1_He1 = const_h * const_c * L_He1_ion / const_kB
CB1_He2 = const_h * const_c * L_He2_ion / const_kB
CR = 2.0 * math.pi * (const_me / const_h) * (const_kB / const_h)
CK = Lalpha**3 / (8.0 * math.pi)
CK_He = Lalpha_He**3 / (8.0 * math.pi)
CL = const_c * const_h / (const_kB * Lalpha)
CL_He = const_c * const_h / (const_kB / L_He_2s)
CT = (8.0 / 3.0) * (const_sigma / (const_me * const_c)) * const_arad
Bfact = const_h * const_c * (L_He_2p - L_He_2s) / const_kB
CL_PSt = const_h * const_c * (L_He_2Pt - L_He_2St) / const_kB
const_h_c_L_He_2St_kB = const_h * const_c * L_He_2St / const_kB

a_PPB = 4.309
b_PPB = -0.6166
c_PPB = 0.6703
d_PPB = 0.5300
a_VF = 10.0 ** (-16.744)
b_VF = 0.711
T_0 = 10 ** 0.477121
T_1 = 10 ** 5.114
a_trip = 10.0 ** (-16.306)
b_trip = 0.761


def _re(x):
    return np.real(x)


class _Plasma:
    """What the three rate equations share at scale factor ``a``: 1 + z, the hydrogen and helium
    number densities [m^-3], the radiation and matter temperatures [K], the Hubble rate [1/s] and
    the ionised fractions (x_e = x_H + f_He x_He electrons per hydrogen nucleus).  ``y`` may be
    complex (complex-step derivatives); branches use its real part."""

    __slots__ = ("zp1", "nH", "nHe", "Tr", "Tm", "Hs", "xH", "xHe", "xe", "fHe", "h")

    def __init__(self, a, y, param, aprimeoa):
        yhe = param["YHe"]
        self.h = param["H0"] / 100.0
        self.zp1 = 1.0 / a
        self.fHe = yhe / (const_mHe_mH * (1.0 - yhe))
        # hydrogen nuclei per m^3: rho_b (1 - Y) / m_H, with rho_crit / m_H = const_dens_fac h^2
        self.nH = const_dens_fac * self.h * self.h * param["Omegab"] * (1.0 - yhe) * self.zp1**3
        self.nHe = self.fHe * self.nH
        self.Tr = param["Tcmb"] * self.zp1
        self.Tm = np.where(_re(y[2]) >= 0, y[2], -y[2])
        # conformal a'/a [1/Mpc] -> H(z) [1/s]
        self.Hs = 1e-5 * aprimeoa * self.zp1 * const_c * bigH
        self.xH = y[0]
        self.xHe = y[1]
        self.xe = self.xH + self.fHe * self.xHe


def _escape(tau):
    """Sobolev escape probability (1 - e^-tau) / tau of a line of optical depth tau."""
    return (1.0 - np.exp(-tau)) / tau


def _he_line_broadening(s, wavenumber, einstein_a, sigma_abs):
    """Ratio gamma of the rate at which H continuum absorption removes photons from a HeI line to
    the line's decay rate (Kholupenko, Ivanchik & Varshalovich 2007; Switzer & Hirata 2008), with
    the line's thermal Doppler width at T_m."""
    vth = np.sqrt(2.0 * const_kB * s.Tm / (const_mH * const_mHe_mH * const_c**2))
    doppler = const_c * wavenumber * vth
    lam_inv_c = const_c * wavenumber
    return (3.0 * einstein_a * s.fHe * (1.0 - s.xHe) * const_c**2) / (
        math.sqrt(math.pi) * sigma_abs * 8.0 * math.pi * doppler * (1.0 - s.xH) * lam_inv_c**2)


def _hydrogen_dxdz(s):
    """dx_H/dz: Peebles' effective three-level atom (Seager, Sasselov & Scott 1999) with the Recfast
    fudge F = 1.105 and the two-Gaussian correction of the Lyman-alpha escape rate (Wong, Moss &
    Scott 2008).  Zero while x_H > 0.99, the Saha-limited rate without the Peebles factor for
    0.985 < x_H <= 0.99."""
    t4 = s.Tm / 1e4
    # case-B recombination coefficient, fit of Pequignot, Petitjean & Boisson (1991) [m^3/s]
    alpha_B = 1e-19 * a_PPB * t4**b_PPB / (1.0 + c_PPB * t4**d_PPB)
    # photo-ionisation rate from n = 2, by detailed balance [1/s]
    beta_B = alpha_B * (CR * s.Tm) ** 1.5 * np.exp(-CDB / s.Tm)
    lnzp1 = math.log(s.zp1)
    k_fix = 1.0 + AGauss1 * math.exp(-(((lnzp1 - zGauss1) / wGauss1) ** 2)) \
        + AGauss2 * math.exp(-(((lnzp1 - zGauss2) / wGauss2) ** 2))
    K_alpha = CK / s.Hs * k_fix          # Lyman-alpha redshifting factor lambda^3 / (8 pi H)
    n_1s = s.nH * (1.0 - s.xH)           # atoms in the ground state
    # recombinations minus ionisations out of the ground state, per unit redshift
    net = (s.xe * s.xH * s.nH * alpha_B - beta_B * (1.0 - s.xH) * np.exp(-CL / s.Tm)) / (s.Hs * s.zp1)
    # Peebles factor: chance that an atom in n = 2 decays (2s two-photon, or Lyman-alpha escape)
    # before it is photo-ionised, with the case-B coefficient divided by the fudge F
    decay = 1.0 + K_alpha * Lambda * n_1s
    peebles = decay / (decay / 1.105 + K_alpha * beta_B * n_1s)
    full = net * peebles
    return np.where(_re(s.xH) > 0.99, 0.0 * s.xH, np.where(_re(s.xH) > 0.985, net, full))


def _helium_singlet_dxdz(s):
    """dx_He/dz through the HeI singlet 2^1P -> 1^1S channel (Seager et al. 2000; Wong et al. 2008):
    Verner & Ferland (1996) recombination fit, Sobolev escape of the 584 A line plus its removal by
    H continuum absorption (fit parameters p = 0.36, q = 0.86) once hydrogen starts recombining."""
    r0 = np.sqrt(s.Tm / T_0)
    r1 = np.sqrt(s.Tm / T_1)
    alpha_He = a_VF / (r0 * (1.0 + r0) ** (1.0 - b_VF) * (1.0 + r1) ** (1.0 + b_VF))
    beta_He = 4.0 * alpha_He * (CR * s.Tm) ** 1.5 * np.exp(-CDB_He / s.Tm)
    n_HeI = s.nHe * (1.0 - s.xHe)        # neutral helium
    K_line = CK_He / s.Hs
    p_esc = _escape(A2P_s * K_line * 3.0 * n_HeI)
    gamma = _he_line_broadening(s, L_He_2p, A2P_s, sigma_He_2Ps)
    a_cont = A2P_s / (1.0 + 0.36 * gamma**0.86)
    # effective K of the line: plain redshifting at the ends of He recombination, else the inverse
    # escape rate (Sobolev, with the H continuum term while x_H < 0.9999999)
    ends = (_re(s.xHe) < 5e-9) | (_re(s.xHe) > 0.98)
    esc_rate = np.where(_re(s.xH) < 0.9999999, A2P_s * p_esc + a_cont, A2P_s * p_esc)
    K_He = np.where(ends, K_line, 1.0 / (esc_rate * 3.0 * n_HeI))
    boltz = np.exp(np.where(_re(Bfact / s.Tm) < 680.0, Bfact / s.Tm, 680.0))  # 2s-2p energy gap factor
    net = (s.xe * s.xHe * s.nH * alpha_He - beta_He * (1.0 - s.xHe) * np.exp(-CL_He / s.Tm)) / (s.Hs * s.zp1)
    k_n = K_He * n_HeI * boltz
    return net * (1.0 + k_n * Lambda_He) / (1.0 + k_n * (Lambda_He + beta_He))


def _helium_triplet_dxdz(s):
    """dx_He/dz through the HeI triplet 2^3P -> 1^1S intercombination line (Wong et al. 2008):
    recombination fit, detailed-balance ionisation from 2^3S, Sobolev escape and H continuum
    absorption (p = 0.66, q = 0.9).  Omitted at the ends of He recombination."""
    r0 = np.sqrt(s.Tm / T_0)
    r1 = np.sqrt(s.Tm / T_1)
    alpha_t = a_trip / (r0 * (1.0 + r0) ** (1.0 - b_trip) * (1.0 + r1) ** (1.0 + b_trip))
    beta_t = (4.0 / 3.0) * alpha_t * np.exp(-const_h * const_c * L_He2St_ion / (const_kB * s.Tm)) * (CR * s.Tm) ** 1.5
    n_HeI = s.nHe * (1.0 - s.xHe)
    p_esc = _escape(A2P_t * n_HeI * 3.0 / (8.0 * math.pi * s.Hs * L_He_2Pt**3))
    gamma = _he_line_broadening(s, L_He_2Pt, A2P_t, sigma_He_2Pt)
    a_cont = A2P_t / (1.0 + 0.66 * gamma**0.9) / 3.0
    decay = np.where(_re(s.xH) > 0.99999, A2P_t * p_esc, A2P_t * p_esc + a_cont) * np.exp(-CL_PSt / s.Tm)
    c_trip = decay / (beta_t + decay)    # probability that an atom in 2^3P reaches the ground state
    net = s.xe * s.xHe * s.nH * alpha_t - 3.0 * beta_t * (1.0 - s.xHe) * np.exp(-const_h_c_L_He_2St_kB / s.Tm)
    ends = (_re(s.xHe) < 5e-9) | (_re(s.xHe) > 0.98)
    return np.where(ends, 0.0 * s.xHe, net * c_trip / (s.Hs * s.zp1))


def _matter_temperature_dTdz(s):
    """dT_m/dz: Compton coupling to the radiation against adiabatic cooling; T_m follows T_rad while
    the Compton time is below 1e-3 of the Hubble time (Seager et al. 1999, eq. 3)."""
    heat = CT * s.Tr**4 * s.xe / (1.0 + s.xe + s.fHe)   # inverse Compton time [1/s]
    t_compton = 1.0 / heat
    t_hubble = 2.0 / (3.0 * s.h * bigH * s.zp1**1.5)
    coupled = s.Tm / s.zp1
    free = heat * (s.Tm - s.Tr) / (s.Hs * s.zp1) + 2.0 * s.Tm / s.zp1
    return np.where(_re(t_compton) < H_frac * t_hubble, coupled, free)


def ionization(a, y, param, aprimeoa):
    """d(x_H, x_He, T_m)/da of the Recfast model (replaces thermodynamics_recfast.py:124-281).

    ``a`` is a real scalar; ``y`` may be complex (complex-step Jacobian) and may carry trailing
    batch axes; branches use the real part.  ``aprimeoa`` is the conformal Hubble rate at ``a``
    (``get_aprimeoa``), passed in because it only depends on ``a``.
    """
    with np.errstate(all="ignore"):
        s = _Plasma(a, y, param, aprimeoa)
        dxH = _hydrogen_dxdz(s)
        dxHe = np.where(_re(s.xHe) < 1e-8, 0.0 * s.xHe, _helium_singlet_dxdz(s) + _helium_triplet_dxdz(s))
        dTm = _matter_temperature_dTdz(s)
        dzda = -1.0 / a**2
        return np.stack([dxH * dzda, dxHe * dzda, dTm * dzda])


# Kaps & Rentrop (1979) GRK4A coefficients (thermodynamics via ode_integrators_stiff.py:176-196)
_G = dict(gamma=0.395, gamma21=-0.767672395484, gamma31=-0.851675323742, gamma32=0.522967289188,
          gamma41=0.288463109545, gamma42=0.880214273381e-1, gamma43=-0.337389840627,
          alpha21=0.438, alpha31=0.796920457938, alpha32=0.730795420615e-1,
          chat1=0.346325833758, chat2=0.285693175712, chat3=0.367980990530,
          c1=0.199293275701, c2=0.482645235674, c3=0.680614886256e-1, c4=0.25)


def _lu3(A):
    """No-pivot 3x3 LU (ode_integrators_stiff.py:77-96)."""
    u00, u01, u02 = A[0, 0], A[0, 1], A[0, 2]
    l10 = A[1, 0] / u00
    u11 = A[1, 1] - l10 * u01
    u12 = A[1, 2] - l10 * u02
    l20 = A[2, 0] / u00
    r21 = A[2, 1] - l20 * u01
    r22 = A[2, 2] - l20 * u02
    l21 = r21 / u11
    u22 = r22 - l21 * u12
    return (u00, u01, u02, l10, u11, u12, l20, l21, u22)


def _lu3_solve(f, b):
    u00, u01, u02, l10, u11, u12, l20, l21, u22 = f
    y0 = b[0]
    y1 = b[1] - l10 * y0
    y2 = b[2] - l20 * y0 - l21 * y1
    x2 = y2 / u22
    x1 = (y1 - u12 * x2) / u11
    x0 = (y0 - u01 * x1 - u02 * x2) / u00
    return np.array([x0, x1, x2])


def _grk4a_step(fun, t0, t1, y0):
    """One GRK4A step (ode_integrators_stiff.py:157-254); all stages at t0 as the reference."""
    g = _G
    dt = t1 - t0
    if np.iscomplexobj(y0) or np.iscomplexobj(fun(t0, y0)):
        # parameters carry a complex-step perturbation: the Jacobian by central differences
        # of the (complex) RHS, relative step 1e-7
        hv = 1e-7 * np.maximum(np.abs(np.real(y0)), 1e-10)
        J = np.stack([(fun(t0, y0 + hv[j] * np.eye(3)[j]) - fun(t0, y0 - hv[j] * np.eye(3)[j])) / (2 * hv[j])
                      for j in range(3)], axis=1) * dt
    else:
        # J = d(dt*f)/dy by complex step (three columns at once)
        h = 1e-40
        Y = y0[:, None] + 1j * h * np.eye(3)
        J = np.imag(fun(t0, Y)) / h * dt
    A = np.eye(3) - g["gamma"] * J
    lu = _lu3(A)
    b1 = dt * fun(t0, y0)
    k1 = _lu3_solve(lu, b1)
    y1 = y0 + g["alpha21"] * k1
    f1 = dt * fun(t0, y1)
    Jk1 = J @ k1
    k2 = _lu3_solve(lu, f1 + g["gamma21"] * Jk1)
    y2 = y0 + g["alpha31"] * k1 + g["alpha32"] * k2
    f2 = dt * fun(t0, y2)
    Jk2 = J @ k2
    k3 = _lu3_solve(lu, f2 + g["gamma31"] * Jk1 + g["gamma32"] * Jk2)
    Jk3 = J @ k3
    k4 = _lu3_solve(lu, f2 + g["gamma41"] * Jk1 + g["gamma42"] * Jk2 + g["gamma43"] * Jk3)
    y_new = y0 + g["c1"] * k1 + g["c2"] * k2 + g["c3"] * k3 + g["c4"] * k4
    y_err = (g["c1"] - g["chat1"]) * k1 + (g["c2"] - g["chat2"]) * k2 + (g["c3"] - g["chat3"]) * k3 + g["c4"] * k4
    return y_new, y_err


def _clip_to_end(tprev, tnext, t1, keep):
    tol = 1e-10 * abs(tnext)
    if tnext > t1 - tol:
        return t1 if keep else tprev + 0.5 * (t1 - tprev)
    return tnext


def solve_pid_grk4a(fun, t0, t1, y0, dt0, rtol, atol, max_steps, steps=None, replay=None):
    """Adaptive GRK4A solve with an integral controller (diffrax ``PIDController``
    defaults: icoeff=1, pcoeff=dcoeff=0, safety 0.9, factor in [0.2, 10],
    RMS norm, error order 3).  Returns y(t1) (``throw=False``: the last accepted
    state is returned when ``max_steps`` is exhausted).

    ``steps`` (a list) receives the accepted step end times; ``replay`` (such a list)
    repeats them without error control, which makes the result a smooth function of the
    parameters (used for derivatives with the step sequence held fixed, as forward-mode
    AD through the reference's diffrax loop does)."""
    y = np.array(y0, dtype=np.result_type(np.asarray(y0).dtype, np.float64))
    if replay is not None:
        t = t0
        for tn in replay:
            y, _ = _grk4a_step(fun, t, tn, y)
            t = tn
        return y
    t = t0
    tn = _clip_to_end(t0, t0 + dt0, t1, True)
    for _ in range(max_steps):
        if not (t < t1):
            break
        y1, yerr = _grk4a_step(fun, t, tn, y)
        sc = yerr / (atol + rtol * np.maximum(np.abs(y), np.abs(y1)))
        err = math.sqrt(float(np.mean(sc * sc)))
        keep = err < 1.0
        inv = 1.0 / err if err > 0 else math.inf
        factor = 0.9 * inv ** (1.0 / 3.0) if math.isfinite(inv) else 10.0
        fmin = 1.0 if keep else 0.2
        factor = min(max(factor, fmin), 10.0)
        dt = (tn - t) * factor
        if keep:
            t, y = tn, y1
            if steps is not None:
                steps.append(tn)
        tn = _clip_to_end(t, t + dt, t1, keep)
    return y


def Saha_HeII(a, param):
    """Saha HeII electron fraction (thermodynamics_recfast.py:303-322); ``a`` may be complex."""
    const_Hfac = 1 / (1.0e06 * 3.0856775807e13)
    mu_H = 1 / (1 - param["YHe"])
    rho_c = 3 * (param["H0"] * const_Hfac) ** 2 / (8 * math.pi * const_G)
    NH = rho_c * param["Omegab"] / (const_mH * mu_H) / a**3
    T = param["Tcmb"] / a
    betaE = const_EionHe12s / T
    fHe = param["fHe"]
    A = 1 + fHe
    B = 1 + 2 * fHe
    R = (2 * math.pi * const_me * const_kB / const_h**2 * T) ** 1.5 / NH * np.exp(-betaE)
    with np.errstate(all="ignore"):
        big = fHe * (1 - B / R + (1 + 5 * fHe + 6 * fHe**2) / R**2)
        small = -(R - A) / 2 + np.sqrt((R - A) ** 2 / 4 + R * B) - A
    return np.where(np.real(R) > 1e5, big, small)


def _get_adaptive_sampling(a0, a1, N):
    """Four geometric segments concentrated on recombination (thermodynamics_recfast.py:325-361)."""
    n_very_early = max(8, int(N * 0.05))
    n_pre = max(8, int(N * 0.10))
    n_rec = int(N * 0.50)
    n_post = N - n_very_early - n_pre - n_rec
    ab1 = max(1.0 / (1.0 + 10000), a0)
    ab2 = 1.0 / (1.0 + 1400)
    ab3 = 1.0 / (1.0 + 600)
    return np.concatenate([
        np.geomspace(a0, ab1, n_very_early, endpoint=False),
        np.geomspace(ab1, ab2, n_pre, endpoint=False),
        np.geomspace(ab2, ab3, n_rec, endpoint=False),
        np.geomspace(ab3, a1, n_post),
    ])


def compute_thermal_history(*, a0, a1, N, param, aprimeoa_fn, rtol=1e-3, atol=1e-6, trace=None, replay=None):
    """Interval-by-interval ionisation history (thermodynamics_recfast.py:363-453).

    Returns ``y[6, N]`` = (x_H, x_He, T_m, dx_H/da, dx_He/da, dT_m/da) at ``a[1:]``.
    ``trace`` (a dict) records the branch taken and the accepted steps of every interval;
    ``replay`` (such a dict) repeats them.
    """
    if trace is not None:
        trace["case"], trace["steps"] = [], []
    a = _get_adaptive_sampling(a0, a1, N + 1)
    cplx = any(np.iscomplexobj(param[k]) for k in ("H0", "Omegab", "Omegam", "OmegaDE", "amnu", "w_DE_0", "w_DE_a"))
    y = np.zeros((6, N), dtype=complex if cplx else np.float64)
    H = param["H0"] / 100.0
    HO = H * bigH
    mu_H = 1.0 / (1.0 - param["YHe"])
    Nnow = 3.0 * HO * HO * param["Omegab"] / (8.0 * math.pi * const_G * mu_H * const_mH)
    fHe = param["YHe"] / (const_mHe_mH * (1.0 - param["YHe"]))
    Tcmb = param["Tcmb"]
    Tcmb3 = Tcmb**3

    def fun(t, yy):
        return ionization(t, yy, param, aprimeoa_fn(t))

    for i in range(N):
        astart = a[i]
        zstart = 1.0 / astart - 1.0
        aend = a[i + 1]
        zend = 1.0 / aend - 1.0
        dzda = -1.0 / aend**2
        if i > 0:
            y_prev = y[:, i - 1].copy()
        else:
            y_prev = np.array([1.0, 1.0, Tcmb * (1.0 + zstart), 0.0, 0.0, -Tcmb * (1.0 + zstart)], dtype=y.dtype)
        if replay is not None:
            case = replay["case"][i]
        else:
            case = 1 if zend > 3500.0 else (2 if (i > 0 and np.real(y_prev[1]) > 0.99) else
                                            (3 if (i > 0 and np.real(y_prev[0]) > 0.99) else 4))
        steps = [] if trace is not None else None
        rsteps = replay["steps"][i] if replay is not None else None
        if trace is not None:
            trace["case"].append(case)
            trace["steps"].append(steps)
        if case == 1:
            new = np.array([1.0, 1.0, Tcmb * (1.0 + zend), 0.0, 0.0, -Tcmb * (1.0 + zend)])
        elif case == 2:
            rhs = (np.exp(1.5 * np.log(CR * Tcmb / (1.0 + zend)) - CB1_He1 / (Tcmb * (1.0 + zend))) / Nnow) * 4.0
            x_He0 = 0.5 * (np.sqrt((rhs - 1.0) ** 2 + 4.0 * (1.0 + fHe) * rhs) - (rhs - 1.0))
            q = -((CB1_He1 - CR * Tcmb**2) / (Tcmb * (1 + zend)))
            dxHeIdz = ((-3 * (-(CB1_He1 / Tcmb) + CR * Tcmb) ** 1.5 * (Nnow + 2 * fHe * Nnow + 4 * q**1.5
                        - np.sqrt(Nnow**2 + (16 * (-CB1_He1 + CR * Tcmb**2) ** 3) / (Tcmb3 * (1 + zend) ** 3)
                                    + 8 * (1 + 2 * fHe) * Nnow * q**1.5)))
                       / (Nnow * (1 + zend) ** 2.5 * np.sqrt(Nnow**2 + (16 * (-CB1_He1 + CR * Tcmb**2) ** 3)
                                                                / (Tcmb**3 * (1 + zend) ** 3)
                                                                + 8 * (1 + 2 * fHe) * Nnow
                                                                * (-((CB1_He1 - CR * Tcmb**2) / (Tcmb + Tcmb * zend))) ** 1.5)))
            new = np.array([1.0, (x_He0 - 1.0) / fHe, Tcmb * (1.0 + zend), 0.0, dxHeIdz * dzda, -Tcmb * (1.0 + zend)])
        elif case == 3:
            rhs = np.exp(1.5 * np.log(CR * Tcmb / (1.0 + zend)) - CB1 / (Tcmb * (1.0 + zend))) / Nnow
            x_H0 = 0.5 * (np.sqrt(rhs**2 + 4.0 * rhs) - rhs)
            q = -((CB1 - CR * Tcmb**2) / (Tcmb * (1 + zend)))
            dxHdz = ((3 * ((2 * q**1.5) / (1 + zend)
                           + ((CB1 - CR * Tcmb**2) * (2 * CB1**2 - 4 * CB1 * CR * Tcmb**2 + Tcmb**2
                                                      * (2 * CR**2 * Tcmb**2 + Nnow * (1 + zend) ** 2 * np.sqrt(q))))
                           / (Tcmb**1.5 * (1 + zend) ** 2.5 * np.sqrt((-CB1 + CR * Tcmb**2)
                              * (CB1**2 - 2 * CB1 * CR * Tcmb**2 + Tcmb**2 * (CR**2 * Tcmb**2 + Nnow * (1 + zend) ** 2
                                                                          * np.sqrt(q)))))))
                     / (2.0 * Nnow))
            new = _solve_ionization(fun, astart, aend, y_prev, rtol, atol, steps=steps, replay=rsteps)
            new[0] = x_H0
            new[3] = dxHdz * dzda
        else:
            new = _solve_ionization(fun, astart, aend, y_prev, rtol, atol, steps=steps, replay=rsteps)
        y[:, i] = new
    return y, a[1:]


def _solve_ionization(fun, astart, aend, ystart, rtol, atol, max_steps=128, steps=None, replay=None):
    """thermodynamics_recfast.py:283-301: state at ``aend`` and its derivative."""
    y_end = solve_pid_grk4a(fun, astart, aend, ystart[:3], abs(astart * 1e-3), rtol, atol, max_steps, steps=steps,
                            replay=replay)
    dyda = fun(aend, y_end)
    return np.array([y_end[0], y_end[1], y_end[2], dyda[0], dyda[1], dyda[2]])


def evaluate_thermo(*, param, num_thermo, aprimeoa_fn, dadtau_fn, dtauda_fn, trace=None, replay=None):
    """Thermal history tables on the Recfast a-grid (thermodynamics_recfast.py:456-492)."""
    param["fHe"] = param["YHe"] / (const_mHe_mH * (1.0 - param["YHe"]))
    y, a = compute_thermal_history(a0=param["amin"], a1=param["amax"], N=num_thermo, param=param,
                                   aprimeoa_fn=aprimeoa_fn, trace=trace, replay=replay)
    xeHI = y[0]
    xeHeI = y[1]
    xeHeII = Saha_HeII(a, param)
    xe = xeHI + param["fHe"] * xeHeI + xeHeII
    mu = 1 / (1 + (1 / const_mHe_mH - 1) * param["YHe"] + (1 - param["YHe"]) * xe)
    Tm = y[2]
    dxeHIda = y[3]
    dxeHeIda = y[4]
    if np.iscomplexobj(param["H0"]) or np.iscomplexobj(param["Omegab"]):
        hc = 1e-6 * a
        dxHeIIda = (Saha_HeII(a + hc, param) - Saha_HeII(a - hc, param)) / (2 * hc)
    else:
        hc = 1e-30 * a
        dxHeIIda = np.imag(Saha_HeII(a + 1j * hc, param)) / hc
    dTmda = y[5]
    daTmda = Tm + a * dTmda
    cs2 = const_kB / const_mH / const_c**2 / mu * Tm * (4 - daTmda / Tm) / 3
    dxedtau = (dxeHIda + param["fHe"] * dxeHeIda + dxHeIIda) * dadtau_fn(a)
    inc = np.array([romb(dtauda_fn, lo, hi) for lo, hi in zip(a[:-1], a[1:])])
    tau = param["taumin"] + np.concatenate([[0.0], np.cumsum(inc)])
    return param, tau, a, cs2, Tm, mu, xe, xeHI, xeHeI, xeHeII, dxedtau
