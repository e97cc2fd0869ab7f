"""CPU restatement of the reference's CMB source and line-of-sight chain: TEST INFRASTRUCTURE ONLY.

Only tests/ and the CPU-baseline legs of bench.py use this module, as the checker.  numpy
float64 / complex128, one function per stage of src/discoeb/cmb.py (reference line numbers in
each docstring):

  visibility_functions    cmb.py:95-163     splines in ln(tau) of the thermal-history arrays
  background_quantities   background.py:348-406
  neutrino_perturbations  cmb.py:165-238, perturbations.py:29-85 (nu_perturb, nu_perturb_prime)
  metric_perturbations    cmb.py:241-338
  polarization_terms      cmb.py:341-389
  source terms S1..S4, S  cmb.py:392-633
  theta_ell (FFTLog)      cmb.py:680-835 (+ the lngamma of util.py:13-45)
  Cell, Dell              cmb.py:838-927
  e_source, theta_ell_E   E-mode polarisation (no counterpart in the reference): the source of
                          Zaldarriaga & Seljak (1997) and its line of sight with j_l(x) / x^2

Index layout of the state (extract_perturbations, cmb.py:17-92): 2 eta, 3/4 delta_c/theta_c,
5/6 delta_b/theta_b, 7.. photon temperature (lmaxg+1), then polarisation (lmaxgp+1), massless
neutrinos (lmaxr+1) from idxr = 9 + lmaxg + lmaxgp, massive neutrinos from
iq0 = 10 + lmaxg + lmaxgp + lmaxr in l-major blocks of nq, dark energy last two.
"""
from __future__ import annotations

import math

import numpy as np

# multipole from which the E-mode line of sight uses the Bessel recurrence (theta_ell_E)
E_L_SWITCH = 8


class NaturalSpline:
    """Natural cubic spline through (x, y) (spline_interpolation.py:6-116; index rule :132-145)."""

    def __init__(self, x, y):
        x = np.asarray(x, dtype=np.float64)
        y = np.asarray(y)
        n = x.shape[0]
        h = np.diff(x)
        S = np.zeros(n, dtype=y.dtype)
        m = n - 2
        if m > 0:
            a, b, c = h[:-1], 2.0 * (h[:-1] + h[1:]), h[1:]
            d = 6.0 * ((y[2:] - y[1:-1]) / h[1:] - (y[1:-1] - y[:-2]) / h[:-1])
            cp = np.zeros(m)
            dp = np.zeros(m, dtype=y.dtype)
            cp[0], dp[0] = c[0] / b[0], d[0] / b[0]
            for i in range(1, m):
                den = b[i] - a[i] * cp[i - 1]
                cp[i] = c[i] / den if i < m - 1 else 0.0
                dp[i] = (d[i] - a[i] * dp[i - 1]) / den
            Si = np.zeros(m, dtype=y.dtype)
            Si[-1] = dp[-1]
            for i in range(m - 2, -1, -1):
                Si[i] = dp[i] - cp[i] * Si[i + 1]
            S[1:-1] = Si
        self.x, self.y, self.S, self.n = x, y, S, n

    def _idx(self, xn):
        return np.clip(np.searchsorted(self.x, xn, side="left") - 1, 0, self.n - 2)

    def evaluate(self, xn):
        i = self._idx(xn)
        h = self.x[i + 1] - self.x[i]
        t = (xn - self.x[i]) / h
        A, B = 1.0 - t, t
        return (A * self.y[i] + B * self.y[i + 1]
                + ((A**3 - A) * self.S[i] + (B**3 - B) * self.S[i + 1]) * h**2 / 6.0)

    def derivative(self, xn):
        i = self._idx(xn)
        h = self.x[i + 1] - self.x[i]
        d = xn - self.x[i]
        y, S = self.y, self.S
        b = (y[i + 1] - y[i]) / h - h * (S[i + 1] + 2.0 * S[i]) / 6.0
        c = S[i] / 2.0
        dd = (S[i + 1] - S[i]) / (6.0 * h)
        return b + 2.0 * c * d + 3.0 * dd * d**2


def _spl(s, xn):
    """Evaluate a host spline table (x, y, S) with the reference's index rule."""
    ns = NaturalSpline.__new__(NaturalSpline)
    ns.x, ns.y, ns.S, ns.n = s.x, s.y, s.S, s.n
    return ns.evaluate(xn)


def visibility_functions(tau, param):
    """compute_visibility_functions (cmb.py:95-163)."""
    lt = np.log(param["tau"])
    ltn = np.log(tau)
    op = NaturalSpline(lt, param["opac"])
    od = NaturalSpline(lt, np.log(np.maximum(param["optical_depth"], 1e-10)))
    return {
        "opac": op.evaluate(ltn),
        "opacprime": op.derivative(ltn) / tau,
        "gvis": NaturalSpline(lt, param["gvis"]).evaluate(ltn),
        "gvisprime": NaturalSpline(lt, param["gvisprime"]).evaluate(ltn),
        "gvispprime": NaturalSpline(lt, param["gvispprime"]).evaluate(ltn),
        "optical_depth": np.exp(od.evaluate(ltn)),
    }


def background_quantities(aexp, param):
    """compute_background_quantities (background.py:348-406)."""
    a = np.asarray(aexp, dtype=np.float64)
    return {
        "rhonu": np.exp(_spl(param["logrhonu_of_loga_spline"], np.log(a))),
        "rho_Q": a ** (-3 * (1 + param["w_DE_0"] + param["w_DE_a"])) * np.exp(3 * (a - 1) * param["w_DE_a"]),
        "w_Q": param["w_DE_0"] + param["w_DE_a"] * (1.0 - a),
    }


def aprimeoa(a, param):
    """get_aprimeoa (background.py:101-123)."""
    rhonu = np.exp(_spl(param["logrhonu_of_loga_spline"], np.log(a)))
    rho_Q = a ** (-3 * (1 + param["w_DE_0"] + param["w_DE_a"])) * np.exp(3 * (a - 1) * param["w_DE_a"])
    grho = (param["grhom"] * param["Omegam"] / a
            + (param["grhog"] + param["grhor"] * (param["Neff"] + param["Nmnu"] * rhonu)) / a**2
            + param["grhom"] * param["OmegaDE"] * rho_Q * a**2 + param["grhom"] * param["Omegak"])
    return np.sqrt(grho / 3.0)


def neutrino_perturbations(yout, yprime, aexp, param, q, w, iq0):
    """compute_neutrino_perturbations (cmb.py:165-238) with nu_perturb / nu_perturb_prime
    (perturbations.py:29-85).  yout, yprime: [K, T, n]; q, w: momentum bins [nq]."""
    nq = len(q)
    aH = aprimeoa(aexp, param)                            # [T]
    aq = aexp[:, None] * param["amnu"] / q[None, :]       # [T, nq]
    v = 1.0 / np.sqrt(1.0 + aq**2)
    vprime = -0.5 * aq * aH[:, None] * v**3              # as the reference writes it
    p0 = yout[..., iq0:iq0 + nq]
    p1 = yout[..., iq0 + nq:iq0 + 2 * nq]
    p2 = yout[..., iq0 + 2 * nq:iq0 + 3 * nq]
    p0p = yprime[..., iq0:iq0 + nq]
    p2p = yprime[..., iq0 + 2 * nq:iq0 + 3 * nq]
    return {
        "drhonu": np.sum(w * p0 / v, axis=-1),
        "dpnu": np.sum(w * p0 * v, axis=-1) / 3,
        "fnu": np.sum(w * p1, axis=-1),
        "shearnu": np.sum(w * p2 * v, axis=-1) * 2 / 3,
        "rho_nu_prime": np.sum(w * (p0p / v - p0 / v**2 * vprime), axis=-1),
        "shear_nu_prime": np.sum(w * (p2p * v + p2 * vprime), axis=-1) * 2 / 3,
        "aprimeoa": aH,
    }


def extract(yout, yprime, lmaxg, lmaxgp, lmaxr):
    """extract_perturbations (cmb.py:17-92)."""
    idxg, idxgp, idxr = 7, 7 + lmaxg + 1, 9 + lmaxg + lmaxgp
    return {
        "idxg": idxg, "idxgp": idxgp, "idxr": idxr, "iq0": 10 + lmaxg + lmaxgp + lmaxr,
        "eta": yout[..., 2], "deltac": yout[..., 3], "thetac": yout[..., 4],
        "deltab": yout[..., 5], "thetab": yout[..., 6], "thetabprime": yprime[..., 6],
        "deltag": yout[..., idxg], "thetag": yout[..., idxg + 1], "shearg": yout[..., idxg + 2] / 2.0,
        "thetagprime": yprime[..., idxg + 1], "sheargprime": yprime[..., idxg + 2] / 2.0,
        "deltar": yout[..., idxr], "thetar": yout[..., idxr + 1], "shearr": yout[..., idxr + 2] / 2.0,
        "shearrprime": yprime[..., idxr + 2] / 2.0,
        "deltaq": yout[..., -2], "thetaq": yout[..., -1],
    }


def metric_perturbations(pt, nu, bq, param, kmodes, aexp):
    """compute_metric_perturbations (cmb.py:241-338)."""
    k = kmodes[:, None]
    a = aexp
    Omegac = param["Omegam"] - param["Omegab"]
    rhonu, rho_Q, w_Q = bq["rhonu"], bq["rho_Q"], bq["w_Q"]
    aH = nu["aprimeoa"]
    rpt = (1 + w_Q) * rho_Q * param["grhom"] * param["OmegaDE"] * pt["thetaq"] * a**2
    grhoprime = (
        -param["grhom"] * param["Omegam"] / a
        - 2 * (param["grhog"] + param["grhor"] * (param["Neff"] + param["Nmnu"] * rhonu)) / a**2
        + param["grhom"] * param["OmegaDE"] * (-3 * (1 + param["w_DE_0"] + (1 - a) * param["w_DE_a"]) * rho_Q * a**2
                                              + 2 * rho_Q * a**2)
    ) * aH + param["grhor"] * param["Nmnu"] * nu["rho_nu_prime"] / a**2
    aHprime = grhoprime / (6 * aH)
    dgrho = (param["grhom"] * (Omegac * pt["deltac"] + param["Omegab"] * pt["deltab"]) / a
             + (param["grhog"] * pt["deltag"] + param["grhor"] * (param["Neff"] * pt["deltar"]
                                                                  + param["Nmnu"] * nu["drhonu"])) / a**2
             + param["grhom"] * param["OmegaDE"] * pt["deltaq"] * rho_Q * a**2)
    dgtheta = (param["grhom"] * (Omegac * pt["thetac"] + param["Omegab"] * pt["thetab"]) / a
               + 4.0 / 3.0 * (param["grhog"] * pt["thetag"] + param["Neff"] * param["grhor"] * pt["thetar"]) / a**2
               + param["Nmnu"] * param["grhor"] * k * nu["fnu"] / a**2 + rpt)
    dgshear = (4.0 / 3.0 * (param["grhog"] * pt["shearg"] + param["Neff"] * param["grhor"] * pt["shearr"]) / a**2
               + param["Nmnu"] * param["grhor"] * nu["shearnu"] / a**2)
    dgshearprime = (4.0 / 3.0 * (param["grhog"] * pt["sheargprime"] + param["Neff"] * param["grhor"]
                                 * pt["shearrprime"]) / a**2
                    + param["Nmnu"] * param["grhor"] * nu["shear_nu_prime"] / a**2 - 2 * aH * dgshear)
    hprime = (2.0 * k**2 * pt["eta"] + dgrho) / aH
    etaprime = 0.5 * dgtheta / k**2
    alpha = (hprime + 6.0 * etaprime) / 2.0 / k**2
    alphaprime = -3 * dgshear / (2 * k**2) + pt["eta"] - 2 * aH * alpha
    alphapprime = -3 * dgshearprime / (2 * k**2) + etaprime - 2 * (aHprime * alpha + aH * alphaprime)
    return {"hprime": hprime, "etaprime": etaprime, "alpha": alpha, "alphaprime": alphaprime,
            "alphapprime": alphapprime, "aprimeoa": aH, "aprimeoaprime": aHprime}


def polarization_terms(pt, metric, vis, yout, yprime, kmodes):
    """compute_polarization_terms (cmb.py:341-389)."""
    k = kmodes[:, None]
    ig, igp = pt["idxg"], pt["idxgp"]
    couplprime = (8 * (pt["thetagprime"] + k**2 * metric["alphaprime"]) / 15
                  - k * 0.6 * (yprime[..., ig + 3] + yprime[..., igp + 1] + yprime[..., igp + 3]))
    P = yout[..., ig + 2] + yout[..., igp] + yout[..., igp + 2]
    Pp = yprime[..., ig + 2] + yprime[..., igp] + yprime[..., igp + 2]
    Ppp = couplprime - 0.3 * (vis["opacprime"] * P + vis["opac"] * Pp)
    return {"polarization_term": P, "polarization_termprime": Pp, "polarization_termpprime": Ppp}


def source_terms(pt, metric, vis, pol, kmodes, tau):
    """compute_source_term_isw / _sachs_wolfe / _doppler / _polarization and their sum
    (cmb.py:392-633).  S1 differentiates eta + alpha' along tau with a natural cubic spline
    per mode."""
    k = kmodes[:, None]
    pot = pt["eta"] + metric["alphaprime"]
    s1 = np.stack([NaturalSpline(tau, pot[i]).derivative(tau) for i in range(pot.shape[0])])
    S1 = np.exp(-vis["optical_depth"]) * s1
    S2 = vis["gvis"] * (0.25 * pt["deltag"] + 2 * metric["alphaprime"] + pol["polarization_term"] / 16
                        + (pt["thetabprime"] + 3 / 16 * pol["polarization_termpprime"]) / k**2)
    S3 = vis["gvisprime"] * (metric["alpha"] + (pt["thetab"] + 3 / 8 * pol["polarization_termprime"]) / k**2)
    S4 = vis["gvispprime"] * 3 / 16 * pol["polarization_term"] / k**2
    return {"S1": S1, "S2": S2, "S3": S3, "S4": S4, "S": S1 + S2 + S3 + S4}


def sources(yout, yprime, kmodes, aexp, tau, param, q, w, lmaxg, lmaxgp, lmaxr):
    """The chain of compute_Cell_spectrum_from_cosmo_params steps 6-10 (cmb.py:1052-1076)."""
    pt = extract(yout, yprime, lmaxg, lmaxgp, lmaxr)
    bq = background_quantities(aexp, param)
    vis = visibility_functions(tau, param)
    nu = neutrino_perturbations(yout, yprime, aexp, param, q, w, pt["iq0"])
    metric = metric_perturbations(pt, nu, bq, param, kmodes, aexp)
    pol = polarization_terms(pt, metric, vis, yout, yprime, kmodes)
    src = source_terms(pt, metric, vis, pol, kmodes, tau)
    src["E"] = e_source(vis["gvis"], pol["polarization_term"])
    return {**src, "metric": metric, "pol": pol, "nu": nu, "vis": vis, "bq": bq, "pt": pt}


_LANCZOS7 = np.array([0.99999999999980993227684700473478, 676.520368121885098567009190444019,
                      -1259.13921672240287047156078755283, 771.3234287776530788486528258894,
                      -176.61502916214059906584551354, 12.507343278686904814458936853,
                      -0.13857109526572011689554707, 9.984369578019570859563e-6, 1.50563273514931155834e-7])


def lngamma_complex(z):
    """log Gamma(z), complex, Lanczos g = 7 / 9 terms with reflection for Re z <= 0.5
    (util.py:13-45; Lanczos, SIAM J. Numer. Anal. B 1 (1964) 86)."""
    z = np.asarray(z, dtype=np.complex128)

    def lanczos(zz):
        zz = zz - 1.0
        Ag = np.full(zz.shape, _LANCZOS7[0], dtype=np.complex128)
        for j in range(1, 9):
            zj = zz + j
            Ag += _LANCZOS7[j] / np.abs(zj) ** 2 * np.conj(zj)
        return (zz + 0.5) * np.log(zz + 7.5) - (zz + 7.5) + 0.9189385332046727418 + np.log(Ag)

    refl = np.real(z) <= 0.5
    out = np.empty_like(z)
    if np.any(~refl):
        out[~refl] = lanczos(z[~refl])
    if np.any(refl):
        zr = z[refl]
        out[refl] = 1.14472988584940017414342735135 - np.log(np.sin(np.pi * zr)) - lanczos(1.0 - zr)
    return out


def fftlog_coefficients(ells, p):
    """M_l(p) = 2^(p-1) sqrt(pi) Gamma((1+l+p)/2) / Gamma((2+l-p)/2) (cmb.py:636-677)."""
    l = np.asarray(ells, dtype=np.float64)[:, None]
    p = np.asarray(p)[None, :]
    lc = (p - 1.0) * math.log(2.0) + 0.5 * math.log(math.pi) + lngamma_complex((1.0 + l + p) / 2.0) \
        - lngamma_complex((2.0 + l - p) / 2.0)
    return np.exp(lc)


def theta_ell(ellmax, kmodes, tau, S, tau0, n_fftlog=16384, n_k_dense=0, abs_sums=False):
    """compute_theta_ell (cmb.py:680-835): optional dense-k spline resampling, spline
    resampling onto a log-chi grid padded by 2 in ln chi, bias -1.1, rfft, analytic
    power-law Bessel integrals.  Returns (theta [K', ellmax+1], kmodes').

    ``abs_sums``: also return the sums of magnitudes that bound the rounding of each multipole
    (the FFT's, sum |S_f chi^1.1| / n per coefficient, and the sum over coefficients of
    |c_p M_l(p)|), so that eps times them is the scale of a correctly rounded evaluation's error."""
    if n_k_dense > 0:
        lk = np.log(kmodes)
        lkd = np.linspace(lk[0], lk[-1], n_k_dense)
        S = np.stack([NaturalSpline(lk, S[:, j]).evaluate(lkd) for j in range(S.shape[1])], axis=1)
        kmodes = np.exp(lkd)
    chi = (tau0 - tau)[::-1]
    S_chi = S[:, ::-1]
    lmin, lmax = math.log(max(chi[0], 1.0)), math.log(chi[-1])
    lo, hi = lmin - 2.0, lmax + 2.0
    dl = (hi - lo) / n_fftlog
    chi_f = np.exp(lo + np.arange(n_fftlog) * dl)
    lchi = np.log(np.maximum(chi, 1e-10))
    S_f = np.stack([NaturalSpline(lchi, S_chi[i]).evaluate(np.log(chi_f)) for i in range(S.shape[0])])
    bias = -1.1
    nf = n_fftlog // 2 + 1
    eta = 2.0 * math.pi * np.arange(nf) / (n_fftlog * dl)
    p = bias + 1j * eta
    c = np.fft.rfft(S_f * chi_f[None, :] ** (-bias), axis=-1) * np.exp(-1j * eta * lo) / n_fftlog
    M = fftlog_coefficients(np.arange(ellmax + 1), p)
    ck = c * np.exp(-(p[None, :] + 1.0) * np.log(kmodes)[:, None])
    th = np.real(ck[:, :1]) @ np.real(M[:, :1]).T
    if n_fftlog % 2 == 0:
        th = th + 2.0 * (np.real(ck[:, 1:-1]) @ np.real(M[:, 1:-1]).T - np.imag(ck[:, 1:-1]) @ np.imag(M[:, 1:-1]).T)
        th = th + np.real(ck[:, -1:]) @ np.real(M[:, -1:]).T - np.imag(ck[:, -1:]) @ np.imag(M[:, -1:]).T
    else:
        th = th + 2.0 * (np.real(ck[:, 1:]) @ np.real(M[:, 1:]).T - np.imag(ck[:, 1:]) @ np.imag(M[:, 1:]).T)
    if not abs_sums:
        return th, kmodes
    w = np.exp(-(bias + 1.0) * np.log(kmodes))[:, None]  # |k^-(p+1)|
    fft_abs = np.abs(S_f * chi_f[None, :] ** (-bias)).sum(axis=-1, keepdims=True) / n_fftlog * w
    return th, kmodes, 2.0 * (np.abs(ck) @ np.abs(M).T) + 2.0 * fft_abs * np.abs(M).sum(axis=1)[None, :]


def e_source(gvis, pol):
    """E-mode polarisation source (3/4) g Pi of Zaldarriaga & Seljak (1997, ApJ 482, 6), whose
    Pi is a quarter of the reference's polarisation term pol (F_g2 + G_g0 + G_g2).  No counterpart
    in the reference, which computes temperature only."""
    return gvis * 3.0 / 16.0 * pol


def e_factor(ell):
    """sqrt((l+2)!/(l-2)!) for l >= 2, else 0."""
    ell = np.asarray(ell, dtype=np.float64)
    return np.where(ell >= 2, np.sqrt(np.maximum((ell + 2) * (ell + 1) * ell * (ell - 1), 0.0)), 0.0)


def theta_ell_E(ellmax, kmodes, tau, S_E, tau0, n_fftlog=16384, n_k_dense=0, l_switch=E_L_SWITCH, abs_sums=False):
    """E-mode multipoles Theta_E,l(k) = sqrt((l+2)!/(l-2)!) int S_E j_l(x) / x^2 dtau, x = k (tau0 - tau).

    For l < l_switch: theta_ell of S_E / chi^2 (chi held >= 1 Mpc) divided by k^2.  For l >= l_switch,
    where the FFTLog's absolute error of that integral, multiplied by l^2 / k^2, would swamp the
    signal: the identity j_l / x^2 = [j_{l-2} / (2l-1) + j_l (1/(2l-1) + 1/(2l+3)) + j_{l+2} / (2l+3)]
    / (2l+1) (from j_{l-1} + j_{l+1} = (2l+1) j_l / x) turns it into theta_ell of S_E itself at
    l - 2, l, l + 2.  ``abs_sums``: also return theta_ell's sums of magnitudes carried through the
    same combination (eps times them is the rounding scale of each multipole)."""
    ell = np.arange(ellmax + 1, dtype=np.float64)
    F = e_factor(ell)
    nlo = min(l_switch, ellmax + 1)
    r = theta_ell(nlo - 1, kmodes, tau, S_E / np.maximum(tau0 - tau, 1.0)[None, :] ** 2, tau0,
                  n_fftlog=n_fftlog, n_k_dense=n_k_dense, abs_sums=abs_sums)
    th_lo, kk = r[0], r[1]
    out = np.zeros((th_lo.shape[0], ellmax + 1))
    parts = [(out, th_lo)] + ([(np.zeros_like(out), r[2])] if abs_sums else [])
    for o, t in parts:
        o[:, :nlo] = t * F[None, :nlo] / kk[:, None] ** 2
    if ellmax >= l_switch:
        r = theta_ell(ellmax + 2, kmodes, tau, S_E, tau0, n_fftlog=n_fftlog, n_k_dense=n_k_dense, abs_sums=abs_sums)
        l = ell[l_switch:]
        cm = 1.0 / ((2 * l + 1) * (2 * l - 1))
        c0 = (1.0 / (2 * l - 1) + 1.0 / (2 * l + 3)) / (2 * l + 1)
        cp = 1.0 / ((2 * l + 1) * (2 * l + 3))
        li = l.astype(int)
        for (o, _), t in zip(parts, r[::2]):
            o[:, l_switch:] = F[None, l_switch:] * (cm * t[:, li - 2] + c0 * t[:, li] + cp * t[:, li + 2])
    return (out, kk, parts[1][0]) if abs_sums else (out, kk)


def Cell(theta, kmodes, n_s, k_p, theta_b=None):
    """compute_Cell (cmb.py:838-873): trapezoid in ln k of (k/k_p)^(n_s-1) theta^2; with theta_b
    the cross spectrum of theta and theta_b."""
    f = (kmodes[:, None] / k_p) ** (n_s - 1) * theta * (theta if theta_b is None else theta_b)
    lk = np.log(kmodes)
    return np.sum(0.5 * (f[1:] + f[:-1]) * np.diff(lk)[:, None], axis=0)


def Dell(C, A_s, Tcmb):
    """compute_Dell (cmb.py:876-927): l(l+1) C_l A_s 2 T_cmb^2 1e12 for l >= 2."""
    ell = np.arange(C.shape[0])
    return ell[2:], ell[2:] * (ell[2:] + 1) * C[2:] * A_s * 2 * Tcmb**2 * 1e12


def aexp_out_cmb(n_early=32, n_pre_recomb=64, n_recomb=128, n_post=96):
    """The output scale factors of compute_Cell_spectrum_from_cosmo_params (cmb.py:1006-1022)."""
    a1 = np.geomspace(1e-4, 1.0 / 3001.0, n_early, endpoint=False)
    a2 = np.geomspace(1.0 / 3001.0, 1.0 / 1401.0, n_pre_recomb, endpoint=False)
    a3 = np.geomspace(1.0 / 1401.0, 1.0 / 601.0, n_recomb, endpoint=False)
    a4 = np.geomspace(1.0 / 601.0, 1.0, n_post)
    return np.concatenate([a1, a2, a3, a4])
