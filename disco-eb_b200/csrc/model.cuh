// Synchronous-gauge Boltzmann model of one k-mode, written as coefficient functions.
//
// The right-hand side of model_synchronous (src/discoeb/perturbations.py:88-525) is linear
// in the perturbation variables y[1:] once the scale factor a = y[0] and tau are fixed:
//
//     f_0 = (a'/a) a
//     f_i = sum_m S_{i,i+m*s_i} y_{i+m*s_i} + S_{i,eta} y_2 + sum_r U_{i,r} g_r      (i >= 2)
//     f_1 = sum_j F1_j y_j + sum_r F1U_r g_r
//     g   = G y,   g_0 = h' (metric trace), g_1 = eta' , g_2 = polter (photon polarisation sum)
//
// S is a set of independent banded chains (CDM, photon temperature + baryons, photon
// polarisation, massless neutrinos, one chain per massive-neutrino momentum bin, dark
// energy), U/G are three rank-one couplings through the metric and the Thomson
// polarisation term.  The same coefficient functions give the RHS (f = J y) and the
// Jacobian J = S + U G used by the implicit stepper, so the two can never disagree.
// Instantiated with T = double, or T = Dual (seeded in a) for the column d f / d a.
#pragma once

#include "dual.cuh"
#include "discoeb.h"

#if defined(__CUDACC__) && defined(__CUDA_ARCH__)
#define DLDG(p) __ldg(p)
#else
#define DLDG(p) (*(p))
#endif

namespace dscb {

struct Dims {
    int n, lmaxg, lmaxgp, lmaxr, lmaxnu, nq, idxgp, idxr, iq0;
};

DHD Dims make_dims(const DiscoebCosmo& c)
{
    Dims d;
    d.lmaxg = c.lmaxg;
    d.lmaxgp = c.lmaxgp;
    d.lmaxr = c.lmaxr;
    d.lmaxnu = c.lmaxnu;
    d.nq = c.nqmax;
    d.n = 7 + (c.lmaxg + 1) + (c.lmaxgp + 1) + (c.lmaxr + 1) + c.nqmax * (c.lmaxnu + 1) + 2;
    d.idxgp = 8 + c.lmaxg;
    d.idxr = 9 + c.lmaxg + c.lmaxgp;
    d.iq0 = 10 + c.lmaxg + c.lmaxgp + c.lmaxr;
    return d;
}

DHD int row_stride(const Dims& D, int i) { return (i >= D.iq0 && i < D.n - 2) ? D.nq : 1; }

// ---- natural cubic spline lookup (spline_interpolation.py:132-228) ----
DHD int spline_index(const DiscoebSpline& s, double xn)
{
    const int n = s.n_knots;
    if (s.uniform) {
        double x0 = DLDG(s.x), x1 = DLDG(s.x + 1);
        double fi = floor((xn - x0) * (1.0 / (x1 - x0)));
        if (!(fi >= 0.0)) return 0;
        return fi > (double)(n - 2) ? n - 2 : (int)fi;
    }
    int lo = 0, hi = n;  // first knot >= xn
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (DLDG(s.x + mid) < xn) lo = mid + 1; else hi = mid;
    }
    int i = lo - 1;
    if (i < 0) i = 0;
    if (i > n - 2) i = n - 2;
    return i;
}

template <class T> DHD T spline_eval_at(const DiscoebSpline& s, int i, T xn)
{
    double xi = DLDG(s.x + i), xj = DLDG(s.x + i + 1);
    double h = xj - xi;
    T t = (xn - xi) / h;
    T A = 1.0 - t, B = t;
    return A * DLDG(s.y + i) + B * DLDG(s.y + i + 1) +
           ((A * A * A - A) * DLDG(s.S + i) + (B * B * B - B) * DLDG(s.S + i + 1)) * (h * h / 6.0);
}

template <class T> DHD T spline_deriv_at(const DiscoebSpline& s, int i, T xn)
{
    double xi = DLDG(s.x + i), xj = DLDG(s.x + i + 1);
    double h = xj - xi;
    double yi = DLDG(s.y + i), yj = DLDG(s.y + i + 1), Si = DLDG(s.S + i), Sj = DLDG(s.S + i + 1);
    T d = xn - xi;
    double b = (yj - yi) / h - h * (Sj + 2.0 * Si) / 6.0;
    double c = Si / 2.0;
    double dd = (Sj - Si) / (6.0 * h);
    return b + 2.0 * c * d + 3.0 * dd * d * d;
}

template <class T> DHD T spline_eval(const DiscoebSpline& s, T xn) { return spline_eval_at(s, spline_index(s, val(xn)), xn); }

// ---- background quantities at (a, tau) ----
template <class T> struct Bg {
    T a, a2, aH, opac, tauc, taucprime, cs2, pb43, rho_Q, w_Q, ca2_Q, pnu, aprimeprimeoa;
    T v[DISCOEB_MAX_NQ];
    bool rsa, ufa, tca, de_frozen;
};

template <class T> DHD T aprimeoa_of(const DiscoebCosmo& P, T a, T loga)
{
    T rhonu = xexp(spline_eval(P.logrhonu_loga, loga));
    T rho_Q = xpow(a, -3.0 * (1.0 + P.w0 + P.wa)) * xexp(3.0 * (a - 1.0) * P.wa);
    T grho = P.grhom * P.Omegam / a + (P.grhog + P.grhor * (P.Neff + P.Nmnu * rhonu)) / (a * a) +
             P.grhom * P.OmegaDE * rho_Q * a * a + P.grhom * P.Omegak;
    return xsqrt(grho / 3.0);
}

// regime < 0: switches from (tau, a) exactly as model_synchronous evaluates them;
// otherwise bitmask 1 = RSA, 2 = UFA, 4 = TCA.
template <class T> DHD void bg_eval(const DiscoebCosmo& P, T a, double tau, double k, int regime, Bg<T>& b)
{
    b.a = a;
    b.a2 = a * a;
    T loga = xlog(a);
    // xe and cs2*a share the knot grid (both tabulated on log of the Recfast a-grid)
    int ix = spline_index(P.xe_loga, val(loga));
    T xe = spline_eval_at(P.xe_loga, ix, loga);
    T xep = spline_deriv_at(P.xe_loga, ix, loga);
    int ic = (P.cs2a_loga.x == P.xe_loga.x) ? ix : spline_index(P.cs2a_loga, val(loga));
    b.cs2 = spline_eval_at(P.cs2a_loga, ic, loga) / a;
    int inu = spline_index(P.logrhonu_loga, val(loga));
    T rhonu = xexp(spline_eval_at(P.logrhonu_loga, inu, loga));
    int ip = (P.logpnu_loga.x == P.logrhonu_loga.x) ? inu : spline_index(P.logpnu_loga, val(loga));
    b.pnu = xexp(spline_eval_at(P.logpnu_loga, ip, loga));
    T photbar = P.grhog / (P.grhom * P.Omegab * a);
    b.pb43 = 4.0 / 3.0 * photbar;
    b.w_Q = P.w0 + P.wa * (1.0 - a);
    b.rho_Q = xpow(a, -3.0 * (1.0 + P.w0 + P.wa)) * xexp(3.0 * (a - 1.0) * P.wa);
    T grho = P.grhom * P.Omegam / a + (P.grhog + P.grhor * (P.Neff + P.Nmnu * rhonu)) / b.a2 +
             P.grhom * P.OmegaDE * b.rho_Q * b.a2 + P.grhom * P.Omegak;
    b.aH = xsqrt(grho / 3.0);
    T xeprime = xep * b.aH;
    T gpres = ((P.grhog + P.grhor * P.Neff) / 3.0 + P.grhor * P.Nmnu * b.pnu) / b.a2 +
              b.w_Q * P.grhom * P.OmegaDE * b.rho_Q * b.a2;
    b.aprimeprimeoa = 0.5 * (b.aH * b.aH - gpres);
    T w_Q_prime = -P.wa * b.aH * a;
    b.ca2_Q = b.w_Q - w_Q_prime / 3.0 / ((1.0 + b.w_Q) + 1e-6) / b.aH;
    const double akthom = 2.3038921003709498e-9 * (1.0 - P.YHe) * P.Omegab * P.H0 * P.H0;
    b.opac = xe * akthom / b.a2;
    b.tauc = 1.0 / xmaxc(b.opac, 1e-30);
    b.taucprime = b.tauc * (2.0 * b.aH - xeprime / xmaxc(xe, 1e-30));
    for (int q = 0; q < P.nqmax; ++q) {
        T aq = a * (P.amnu / P.q[q]);
        b.v[q] = 1.0 / xsqrt(1.0 + aq * aq);
    }
    if (regime < 0) {
        double tcr = val(b.tauc), thr = 1.0 / (val(b.aH) > 1e-30 ? val(b.aH) : 1e-30);
        double tk = 1.0 / (k > 1e-30 ? k : 1e-30);
        b.rsa = P.use_rsa && (tcr / (tau > 1e-30 ? tau : 1e-30) > P.rsa_tau_c_over_tau) && (tau * k > P.rsa_tau_over_tau_k);
        b.ufa = !b.rsa && P.use_ufa && (tau * k > P.ufa_tau_over_tau_k);
        bool unc = (tcr / tk > P.tca_tau_c_over_tau_k) ||
                   ((tcr / thr > P.tca_tau_c_over_tau_h) && (tcr / tk > 0.1 * P.tca_tau_c_over_tau_k));
        b.tca = !b.rsa && P.use_tca && !unc;
    } else {
        b.rsa = (regime & 1) != 0;
        b.ufa = !b.rsa && (regime & 2) != 0;
        b.tca = !b.rsa && (regime & 4) != 0;
    }
    b.de_frozen = P.de_guard_eps > 0.0 && fabs(val(1.0 + b.w_Q)) < P.de_guard_eps;
}

DHD double dlfdlq_of(double q) { return -q / (1.0 + exp(-q)); }

// ---- G: column j of the three functionals (h', eta', polter) ----
template <class T>
DHD void gcol(const DiscoebCosmo& P, const Dims& D, const Bg<T>& b, double k, int j, T g[3])
{
    g[0] = 0.0; g[1] = 0.0; g[2] = 0.0;
    const double k2 = k * k;
    const double Omegac = P.Omegam - P.Omegab;
    const T a = b.a, a2 = b.a2;
    const T invaH = 1.0 / (b.rsa ? xmaxc(b.aH, 1e-30) : b.aH);
    const double hE = 0.5 / k2;
    const int nq = D.nq;
    // h' = (2 k^2 eta + dgrho) / (a'/a)   (perturbations.py:294-306, :346)
    if (j == 2) g[0] = 2.0 * k2 * invaH;
    else if (j == 3) g[0] = P.grhom * Omegac / a * invaH;
    else if (j == 5) g[0] = P.grhom * P.Omegab / a * invaH;
    else if (j == 7) { if (!b.rsa) g[0] = P.grhog / a2 * invaH; }
    else if (j == D.idxr) { if (!b.rsa) g[0] = P.grhor * P.Neff / a2 * invaH; }
    else if (j >= D.iq0 && j < D.iq0 + nq) { int q = j - D.iq0; g[0] = P.grhor * P.Nmnu * P.wq[q] / b.v[q] / a2 * invaH; }
    else if (j == D.n - 2) g[0] = P.grhom * P.OmegaDE * b.rho_Q * a2 * invaH;
    // eta' = dgtheta / (2 k^2)   (perturbations.py:330-335, :349)
    if (j == 4) g[1] = hE * P.grhom * Omegac / a;
    else if (j == 6) g[1] = hE * P.grhom * P.Omegab / a;
    else if (j == 8) { if (!b.rsa) g[1] = hE * (4.0 / 3.0) * P.grhog / a2; }
    else if (j == D.idxr + 1) { if (!b.rsa) g[1] = hE * (4.0 / 3.0) * P.Neff * P.grhor / a2; }
    else if (j >= D.iq0 + nq && j < D.iq0 + 2 * nq) { int q = j - D.iq0 - nq; g[1] = hE * P.Nmnu * P.grhor * k * P.wq[q] / a2; }
    else if (j == D.n - 1) g[1] = hE * (1.0 + b.w_Q) * b.rho_Q * P.grhom * P.OmegaDE * a2;
    if (b.rsa) {
        // theta_gamma and theta_r replaced by the RSA fields (approximations.py:28-47)
        const double sk2 = k2 > 1e-30 ? k2 : 1e-30;
        const T stc = xmaxc(b.tauc, 1e-30);
        const T cg = hE * (4.0 / 3.0) * P.grhog / a2;
        const T fac = 3.0 / (sk2 * stc);
        if (j == 6) g[1] = g[1] + cg * fac * (-b.taucprime / stc - b.aH);
        else if (j == 5) g[1] = g[1] + cg * fac * (b.cs2 * sk2);
        else if (j == 2) g[1] = g[1] + cg * fac * sk2;
        const T eH = cg * (-0.5 - 0.5 * fac * b.taucprime / stc) + hE * (4.0 / 3.0) * P.Neff * P.grhor / a2 * (-0.5);
        g[1] = g[1] + eH * g[0];
    } else if (!b.tca) {
        if (j == 9 || j == D.idxgp || j == D.idxgp + 2) g[2] = 1.0;
    }
}

// ---- row i >= 2: band entries band[m+3] for column i + m*stride, eta coupling, U ----
template <class T>
DHD void rowc(const DiscoebCosmo& P, const Dims& D, const Bg<T>& b, double k, double tau, int i, T band[7], T& etac, T u[3])
{
    for (int m = 0; m < 7; ++m) band[m] = 0.0;
    etac = 0.0;
    u[0] = 0.0; u[1] = 0.0; u[2] = 0.0;
    const double k2 = k * k;
    if (i == 2) { u[1] = 1.0; return; }
    if (i == 3) { band[4] = -1.0; u[0] = -0.5; return; }
    if (i == 4) { band[3] = -b.aH; return; }
    if (i == 5) { band[4] = -1.0; u[0] = -0.5; return; }
    if (i == 6) {
        const T po = b.pb43 * b.opac;
        if (!b.rsa) {
            band[2] = k2 * b.cs2;
            band[3] = -b.aH - po;
            band[5] = po;
        } else {
            const double sk2 = k2 > 1e-30 ? k2 : 1e-30;
            const T stc = xmaxc(b.tauc, 1e-30);
            const T fac = 3.0 / (sk2 * stc);
            band[2] = k2 * b.cs2 + po * fac * (b.cs2 * sk2);
            band[3] = -b.aH - po + po * fac * (-b.taucprime / stc - b.aH);
            etac = po * fac * sk2;
            u[0] = po * (-0.5 - 0.5 * fac * b.taucprime / stc);
        }
        return;
    }
    if (i <= 7 + D.lmaxg) {  // photon temperature, l = i - 7
        if (b.rsa) return;
        const int l = i - 7, L = D.lmaxg;
        if (l == 0) { band[4] = -4.0 / 3.0; u[0] = -2.0 / 3.0; }
        else if (l == 1) { band[1] = b.opac; band[2] = 0.25 * k2; band[3] = -b.opac; band[4] = -0.5 * k2; }
        else if (l == 2) {
            band[2] = 8.0 / 15.0; band[3] = -b.opac; band[4] = -0.6 * k;
            u[0] = 4.0 / 15.0; u[1] = 8.0 / 5.0; u[2] = 0.1 * b.opac;
        } else if (l < L) {
            band[2] = k * l / (2.0 * l + 1.0); band[3] = -b.opac; band[4] = -k * (l + 1.0) / (2.0 * l + 1.0);
        } else {
            band[2] = k; band[3] = -(L + 1.0) / tau - b.opac;
        }
        return;
    }
    if (i <= D.idxgp + D.lmaxgp) {  // photon polarisation
        if (b.rsa || b.tca) return;
        const int l = i - D.idxgp, L = D.lmaxgp;
        if (l < L) {
            if (l > 0) band[2] = k * l / (2.0 * l + 1.0);
            band[3] = -b.opac;
            band[4] = -k * (l + 1.0) / (2.0 * l + 1.0);
            if (l == 0) u[2] = 0.5 * b.opac;
            if (l == 2) u[2] = 0.1 * b.opac;
        } else {
            band[2] = k; band[3] = -(L + 1.0) / tau - b.opac;
        }
        return;
    }
    if (i <= D.idxr + D.lmaxr) {  // massless neutrinos
        if (b.rsa) return;
        const int l = i - D.idxr, L = D.lmaxr;
        if (l == 0) { band[4] = -4.0 / 3.0; u[0] = -2.0 / 3.0; }
        else if (l == 1) { band[2] = 0.25 * k2; band[4] = -0.5 * k2; }
        else if (l == 2) {
            if (b.ufa) {
                band[2] = 4.0 / 15.0;
                band[3] = -1.5 / (tau > 1e-30 ? tau : 1e-30);
                u[0] = 2.0 / 15.0;
            } else {
                band[2] = 8.0 / 15.0; band[4] = -0.6 * k; u[0] = 4.0 / 15.0; u[1] = 8.0 / 5.0;
            }
        } else if (!b.ufa) {
            if (l < L) { band[2] = k * l / (2.0 * l + 1.0); band[4] = -k * (l + 1.0) / (2.0 * l + 1.0); }
            else { band[2] = k; band[3] = -(L + 1.0) / tau; }
        }
        return;
    }
    if (i < D.n - 2) {  // massive neutrinos, l-major blocks of nq bins
        const int r = i - D.iq0, l = r / D.nq, q = r - l * D.nq, L = D.lmaxnu;
        const T kv = k * b.v[q];
        const double dl = dlfdlq_of(P.q[q]);
        if (l == 0) { band[4] = -kv; u[0] = dl / 6.0; }
        else if (l == 1) { band[2] = kv / 3.0; band[4] = -2.0 * kv / 3.0; }
        else if (l == 2 && L > 2) { band[2] = 2.0 * kv / 5.0; band[4] = -3.0 * kv / 5.0; u[0] = -dl / 15.0; u[1] = -0.4 * dl; }
        else if (l < L) { band[2] = kv * (double)l / (2.0 * l + 1.0); band[4] = -kv * (l + 1.0) / (2.0 * l + 1.0); }
        else { band[2] = kv; band[3] = -(L + 1.0) / tau; }
        return;
    }
    if (b.de_frozen) return;
    const double cs2Q = P.cs2_DE;
    const T opw = 1.0 + b.w_Q;
    if (i == D.n - 2) {
        band[3] = -3.0 * (cs2Q - b.w_Q) * b.aH;
        band[4] = -opw - 9.0 * opw * (cs2Q - b.ca2_Q) * b.aH * b.aH / k2;
        u[0] = -0.5 * opw;
    } else {
        band[2] = cs2Q / opw * k2;
        band[3] = -(1.0 - 3.0 * cs2Q) * b.aH;
    }
}

// ---- row 1 (a h'), read by no other equation: f_1 = sum_j F1_j y_j + F1U . g ----
template <class T>
DHD T f1col(const DiscoebCosmo& P, const Dims& D, const Bg<T>& b, double k, int j)
{
    const double k2 = k * k;
    const double Omegac = P.Omegam - P.Omegab;
    const T a = b.a, a2 = b.a2;
    const int nq = D.nq;
    T rho = 0.0, pres = 0.0;  // coefficients of y_j in dgrho and dgpres
    if (j == 3) rho = P.grhom * Omegac / a;
    else if (j == 5) rho = P.grhom * P.Omegab / a;
    else if (j == 7) { rho = P.grhog / a2; if (!b.rsa) pres = P.grhog / a2 / 3.0; }
    else if (j == D.idxr) { rho = P.grhor * P.Neff / a2; if (!b.rsa) pres = P.grhor * P.Neff / a2 / 3.0; }
    else if (j >= D.iq0 && j < D.iq0 + nq) {
        int q = j - D.iq0;
        rho = P.grhor * P.Nmnu * P.wq[q] / b.v[q] / a2;
        pres = P.grhor * P.Nmnu / a2 * P.wq[q] * b.v[q] / 3.0;
    } else if (j == D.n - 2) {
        rho = P.grhom * P.OmegaDE * b.rho_Q * a2;
        pres = P.cs2_DE * P.grhom * P.OmegaDE * b.rho_Q * a2;
    } else if (j == D.n - 1) {
        pres = (P.cs2_DE - b.ca2_Q) * (3.0 * b.aH * (1.0 + b.w_Q) * b.rho_Q * P.grhom * P.OmegaDE * a2 / k2);
    }
    if (b.rsa) {
        const double sk2 = k2 > 1e-30 ? k2 : 1e-30;
        const T stc = xmaxc(b.tauc, 1e-30);
        if (j == 2) pres = pres + (P.grhog + P.grhor * P.Neff) / a2 / 3.0 * (-4.0);
        else if (j == 6) pres = pres + P.grhog / a2 / 3.0 * (4.0 / (sk2 * stc));
    }
    return -a * (rho + 3.0 * pres);
}

template <class T>
DHD void f1u(const DiscoebCosmo& P, const Bg<T>& b, double k, T u[3])
{
    u[0] = 0.0; u[1] = 0.0; u[2] = 0.0;
    if (b.rsa) {
        const double k2 = k * k, sk2 = k2 > 1e-30 ? k2 : 1e-30;
        const T stc = xmaxc(b.tauc, 1e-30);
        const T a2 = b.a2;
        T presH = P.grhog / a2 / 3.0 * (4.0 * b.aH / sk2 + 2.0 / (sk2 * stc)) + P.grhor * P.Neff / a2 / 3.0 * (4.0 * b.aH / sk2);
        u[0] = -b.a * 3.0 * presH;
    }
}

// explicit tau dependence d f / d tau at fixed y (truncation terms and the UFA closure)
template <class T>
DHD double dtau_row(const Dims& D, const Bg<T>& b, double tau, int i, const double* y)
{
    if (i < 7) return 0.0;
    const double it2 = 1.0 / (tau * tau);
    if (i == 7 + D.lmaxg) return b.rsa ? 0.0 : (D.lmaxg + 1.0) * it2 * y[i];
    if (i == D.idxgp + D.lmaxgp) return (b.rsa || b.tca) ? 0.0 : (D.lmaxgp + 1.0) * it2 * y[i];
    if (i == D.idxr + 2) return (!b.rsa && b.ufa && tau > 1e-30) ? 1.5 * it2 * y[i] : 0.0;
    if (i == D.idxr + D.lmaxr) return (b.rsa || b.ufa) ? 0.0 : (D.lmaxr + 1.0) * it2 * y[i];
    if (i >= D.iq0 + D.lmaxnu * D.nq && i < D.n - 2) return (D.lmaxnu + 1.0) * it2 * y[i];
    return 0.0;
}

}  // namespace dscb

namespace dscb {

// ---- RSA output projection (approximations.py:84-176): the fields that replace the
// photon and massless-neutrino moments at an output time.  Returns true when the RSA
// condition holds there (evaluated from (tau, a) as the reference does).
DHD bool rsa_projection(const DiscoebCosmo& P, const Dims& D, double tau, double k, const double* y, double out[4])
{
    const double a = y[0], loga = log(a), eta = y[2], deltab = y[5], thetab = y[6];
    const double aH = aprimeoa_of(P, a, loga);
    const int ix = spline_index(P.xe_loga, loga);
    const double xe = spline_eval_at(P.xe_loga, ix, loga);
    const double xeprime = spline_deriv_at(P.xe_loga, ix, loga) * aH;
    const double cs2 = spline_eval(P.cs2a_loga, loga) / a;
    const double akthom = 2.3038921003709498e-9 * (1.0 - P.YHe) * P.Omegab * P.H0 * P.H0;
    const double opac = xe * akthom / (a * a);
    const double tau_c = 1.0 / (opac > 1e-30 ? opac : 1e-30);
    const double tau_c_prime = tau_c * (2.0 * aH - xeprime / (xe > 1e-30 ? xe : 1e-30));
    const double Omegac = P.Omegam - P.Omegab;
    double drhonu = 0.0;
    for (int q = 0; q < D.nq; ++q) {
        const double aq = a * P.amnu / P.q[q];
        drhonu += P.wq[q] * y[D.iq0 + q] * sqrt(1.0 + aq * aq);
    }
    const double rho_Q = pow(a, -3.0 * (1.0 + P.w0 + P.wa)) * exp(3.0 * (a - 1.0) * P.wa);
    const double dgrho_wo_rel = P.grhom * (Omegac * y[3] + P.Omegab * deltab) / a + P.grhor * P.Nmnu * drhonu / (a * a) +
                                P.grhom * P.OmegaDE * y[D.n - 2] * rho_Q * a * a;
    const double k2 = k * k;
    const double hprime = (2.0 * k2 * eta + dgrho_wo_rel) / (aH > 1e-30 ? aH : 1e-30);
    const double sk2 = k2 > 1e-30 ? k2 : 1e-30, stc = tau_c > 1e-30 ? tau_c : 1e-30;
    out[0] = 4.0 / sk2 * (aH * hprime - sk2 * eta) + 4.0 / (sk2 * stc) * (thetab + 0.5 * hprime);
    out[1] = -0.5 * hprime + 3.0 / (sk2 * stc) *
             (-tau_c_prime / stc * (thetab + 0.5 * hprime) + (-aH * thetab + cs2 * sk2 * deltab + sk2 * eta));
    out[2] = 4.0 / sk2 * (aH * hprime - sk2 * eta);
    out[3] = -0.5 * hprime;
    return P.use_rsa && (tau_c / (tau > 1e-30 ? tau : 1e-30) > P.rsa_tau_c_over_tau) && (tau * k > P.rsa_tau_over_tau_k);
}

// is index i one of the moments the RSA projection overwrites?  (value slot or -1 for zero)
DHD int rsa_slot(const Dims& D, int i)
{
    if (i == 7) return 0;
    if (i == 8) return 1;
    if (i > 8 && i <= D.idxgp + D.lmaxgp) return -1;  // shear, l >= 3 and all polarisation
    if (i == D.idxr) return 2;
    if (i == D.idxr + 1) return 3;
    if (i > D.idxr + 1 && i <= D.idxr + D.lmaxr) return -1;
    return -2;  // untouched
}

// ---- convert_to_output_variables (perturbations.py:528-677) ----
DHD void output_vars(const DiscoebCosmo& P, const Dims& D, double k, const double* y, double* o)
{
    const double Omegac = P.Omegam - P.Omegab;
    const int n = D.n, nq = D.nq, iq0 = D.iq0, iq1 = iq0 + nq;
    const double a = y[0], eta = y[2], deltac = y[3], thetac = y[4], deltab = y[5], thetab = y[6];
    const double deltag = y[7], thetag = y[8], deltar = y[D.idxr], thetar = y[D.idxr + 1];
    const double loga = log(a);
    const int inu = spline_index(P.logrhonu_loga, loga);
    const double rhonu = exp(spline_eval_at(P.logrhonu_loga, inu, loga));
    const int ip = (P.logpnu_loga.x == P.logrhonu_loga.x) ? inu : spline_index(P.logpnu_loga, loga);
    const double pnu = exp(spline_eval_at(P.logpnu_loga, ip, loga));
    double drhonu = 0.0, fnu = 0.0;
    for (int q = 0; q < nq; ++q) {
        const double aq = a * P.amnu / P.q[q];
        drhonu += P.wq[q] * y[iq0 + q] * sqrt(1.0 + aq * aq);
        fnu += P.wq[q] * y[iq1 + q];
    }
    const double deltanu = drhonu / rhonu, thetanu = k * fnu / (rhonu + pnu);
    const double deltaq = y[n - 2], thetaq = y[n - 1];
    const double w_Q = P.w0 + P.wa * (1.0 - a);
    const double rho_Q = pow(a, -3.0 * (1.0 + P.w0 + P.wa)) * exp(3.0 * (a - 1.0) * P.wa);
    const double rpt = (1.0 + w_Q) * rho_Q * P.grhom * P.OmegaDE * thetaq * a * a;
    const double a2 = a * a;
    const double grho = P.grhom * P.Omegam / a + (P.grhog + P.grhor * (P.Neff + P.Nmnu * rhonu)) / a2 +
                        P.grhom * P.OmegaDE * rho_Q * a2 + P.grhom * P.Omegak;
    const double aH = sqrt(grho / 3.0);
    const double dgrho = P.grhom * (Omegac * deltac + P.Omegab * deltab) / a +
                         (P.grhog * deltag + P.grhor * (P.Neff * deltar + P.Nmnu * drhonu)) / a2 +
                         P.grhom * P.OmegaDE * deltaq * rho_Q * a2;
    const double dgtheta = P.grhom * (Omegac * thetac + P.Omegab * thetab) / a +
                           4.0 / 3.0 * (P.grhog * thetag + P.Neff * P.grhor * thetar) / a2 +
                           P.Nmnu * P.grhor * k * fnu / a2 + rpt;
    const double k2 = k * k;
    const double hprime = (2.0 * k2 * eta + dgrho) / aH;
    const double etaprime = 0.5 * dgtheta / k2;
    const double alpha = (hprime + 6.0 * etaprime) / 2.0 / k2;
    const double mden = P.grhom * P.Omegam / a + P.grhor * P.Nmnu * rhonu / a2;
    const double deltam = (P.grhom * (Omegac * deltac + P.Omegab * deltab) / a + P.grhor * P.Nmnu * drhonu / a2) / mden;
    double thetam = (P.grhom * (Omegac * thetac + P.Omegab * thetab) / a + P.Nmnu * P.grhor * k * fnu / a2) / (3.0 * mden);
    const double deltabc = (P.grhom * (Omegac * deltac + P.Omegab * deltab) / a) / (P.grhom * P.Omegam / a);
    double thetabc = (P.grhom * (Omegac * thetac + P.Omegab * thetab) / a) / (3.0 * (P.grhom * P.Omegam / a) / a2);
    thetam += alpha * k2;
    thetabc += alpha * k2;
    o[0] = eta; o[1] = etaprime; o[2] = hprime; o[3] = alpha;
    o[4] = deltam; o[5] = thetam / aH; o[6] = deltabc; o[7] = thetabc / aH;
    o[8] = deltac; o[9] = thetac / aH; o[10] = deltab; o[11] = thetab / aH;
    o[12] = deltag; o[13] = thetag / aH; o[14] = deltar; o[15] = thetar / aH;
    o[16] = deltanu; o[17] = thetanu / aH; o[18] = deltaq; o[19] = thetaq / aH;
}

}  // namespace dscb
