/*
 * CPU oracle for the per-k-mode linear perturbation solve: TEST INFRASTRUCTURE ONLY.
 * See oracle.h for the list of restated reference functions.
 */
#include "oracle.h"

#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

static int spline_index(const OracleSpline* s, double xn)
{
    int i;
    if (s->uniform) {
        double dx_inv = 1.0 / (s->x[1] - s->x[0]);
        double fi = floor((xn - s->x[0]) * dx_inv);
        if (!(fi >= 0.0)) fi = 0.0; /* also catches NaN */
        i = fi > (double)(s->n - 2) ? s->n - 2 : (int)fi;
    } else {
        /* count of knots strictly below xn, minus one */
        int lo = 0, hi = s->n; /* first index with x >= xn */
        while (lo < hi) {
            int mid = (lo + hi) >> 1;
            if (s->x[mid] < xn) lo = mid + 1; else hi = mid;
        }
        i = lo - 1;
        if (i < 0) i = 0;
        if (i > s->n - 2) i = s->n - 2;
    }
    return i;
}

/* ---- real instantiation ---- */
#define NUM double
#define FN(x) x##_r
#define RE(x) (x)
#define EXP exp
#define LOG log
#define SQRT sqrt
#define POW pow
#include "rhs_body.h"
#undef NUM
#undef FN
#undef RE
#undef EXP
#undef LOG
#undef SQRT
#undef POW

/* ---- complex instantiation (complex-step derivatives) ---- */
#define NUM double complex
#define FN(x) x##_c
#define RE(x) creal(x)
#define EXP cexp
#define LOG clog
#define SQRT csqrt
#define POW cpow
#include "rhs_body.h"
#undef NUM
#undef FN
#undef RE
#undef EXP
#undef LOG
#undef SQRT
#undef POW

int oracle_nvar(const OracleProblem* P)
{
    return 7 + (P->lmaxg + 1) + (P->lmaxgp + 1) + (P->lmaxr + 1) + P->nqmax * (P->lmaxnu + 1) + 2;
}

void oracle_rhs(const OracleProblem* P, double tau, const double* y, double k, double* f, int regime)
{
    rhs_r(P, tau, y, k, f, regime);
}

static const double CSTEP = 1e-100;

void oracle_jacobian(const OracleProblem* P, double tau, const double* y, double k, double* J, double* dT, int regime)
{
    const int n = P->n;
    double complex* yc = (double complex*)malloc(sizeof(double complex) * n);
    double complex* fc = (double complex*)malloc(sizeof(double complex) * n);
    double* e = (double*)calloc(n, sizeof(double));
    double* col = (double*)malloc(sizeof(double) * n);
    /* column 0: complex step in a */
    for (int i = 0; i < n; ++i) yc[i] = y[i];
    yc[0] = y[0] + I * (CSTEP * y[0]);
    rhs_c(P, tau, yc, k, fc, regime);
    for (int i = 0; i < n; ++i) J[i * n + 0] = cimag(fc[i]) / (CSTEP * y[0]);
    /* columns 1..n-1: f is linear homogeneous in y[1:], so column j = f(tau, [a, e_j]) */
    e[0] = y[0];
    for (int j = 1; j < n; ++j) {
        e[j] = 1.0;
        rhs_r(P, tau, e, k, col, regime);
        for (int i = 0; i < n; ++i) J[i * n + j] = (i == 0) ? 0.0 : col[i];
        e[j] = 0.0;
    }
    if (dT) {
        for (int i = 0; i < n; ++i) yc[i] = y[i];
        rhs_c(P, tau + I * (CSTEP * tau), yc, k, fc, regime);
        for (int i = 0; i < n; ++i) dT[i] = cimag(fc[i]) / (CSTEP * tau);
    }
    free(yc); free(fc); free(e); free(col);
}

/* ---- start time (perturbations.py:784-835) ---- */
static double cond_large_k(const OracleProblem* P, double logtau, double k)
{
    double tau = exp(logtau);
    double a = spl_eval_r(&P->a_of_tau, tau);
    double tau_H = 1.0 / aprimeoa_r(P, a);
    double tau_k = 1.0 / k;
    return tau_H / tau_k / 0.07 - 1.0;
}

static double cond_small_k(const OracleProblem* P, double logtau)
{
    double tau = exp(logtau);
    double akthom = 2.3048e-9 * (1.0 - P->YHe) * P->Omegab * P->H0 * P->H0;
    double xe = spl_eval_r(&P->xe_of_tau, tau);
    double a = spl_eval_r(&P->a_of_tau, tau);
    double opac = xe * akthom / (a * a);
    double tau_c = 1.0 / opac, tau_H = 1.0 / aprimeoa_r(P, a);
    return tau_c / tau_H / 0.0004 - 1.0;
}

double oracle_start_time(const OracleProblem* P, double k)
{
    double x0 = log(P->taumin), x1 = log(spl_eval_r(&P->tau_of_a, 0.1));
    double l = x0, r = x1;
    for (int it = 0; it < 7; ++it) { /* util.root_find_bisect */
        double m = 0.5 * (l + r);
        if (cond_large_k(P, m, k) * cond_large_k(P, l, k) > 0) l = m; else r = m;
    }
    double lt_large = 0.5 * (l + r);
    l = x0; r = x1;
    for (int it = 0; it < 7; ++it) {
        double m = 0.5 * (l + r);
        if (cond_small_k(P, m) * cond_small_k(P, l) > 0) l = m; else r = m;
    }
    double lt_small = 0.5 * (l + r);
    return exp(lt_small < lt_large ? lt_small : lt_large);
}

/* ---- adiabatic ICs (perturbations.py:680-781) ---- */
void oracle_ics(const OracleProblem* P, double tau, double kmode, double* y)
{
    const int n = P->n, lmaxg = P->lmaxg, lmaxgp = P->lmaxgp, lmaxr = P->lmaxr, nq = P->nqmax;
    const int iq0 = 10 + lmaxg + lmaxgp + lmaxr, iq1 = iq0 + nq, iq2 = iq1 + nq;
    for (int i = 0; i < n; ++i) y[i] = 0.0;
    double a = spl_eval_r(&P->a_of_tau, tau);
    double rhonu_bg = exp(spl_eval_r(&P->logrhonu_loga, log(a)));
    double rhom = P->grhom * P->Omegam / (a * a * a);
    double rhor = (P->grhog + P->grhor * (P->Neff + P->Nmnu * rhonu_bg)) / (a * a * a * a);
    double rhonu = P->grhor * (P->Neff + P->Nmnu * rhonu_bg) / (a * a * a * a);
    double fracb = P->Omegab / P->Omegam;
    double fracnu = rhonu / rhor;
    double om = a * rhom / sqrt(rhor);
    double ci = -1.0, s2 = 1.0;
    double kt = kmode * tau;
    double deltag = -(kt * kt) / 3.0 * (1.0 - om * tau / 5.0) * ci * s2;
    double thetag = -(kt * kt * kt) / tau / 36.0 *
                    (1.0 - 3.0 * (1.0 + 5.0 * fracb - fracnu) / 20.0 / (1.0 - fracnu) * om * tau) * ci * s2;
    double deltab = 0.75 * deltag, thetab = thetag, deltac = 0.75 * deltag, thetac = 0.0;
    double deltar = deltag;
    double thetar = -(kt * kt * kt * kt) / tau / 36.0 / (4.0 * fracnu + 15.0) *
                    (4.0 * fracnu + 11.0 + 12.0 -
                     3.0 * (8.0 * fracnu * fracnu + 50.0 * fracnu + 275.0) / 20.0 / (2.0 * fracnu + 15.0) * tau * om) * ci;
    double shearr = (kt * kt) / (45.0 + 12.0 * fracnu) * (3.0 * s2 - 1.0) *
                    (1.0 + (4.0 * fracnu - 5.0) / 4.0 / (2.0 * fracnu + 15.0) * tau * om) * ci;
    double cs2_Q = P->cs2_DE, w_Q = P->w0 + P->wa * (1.0 - a);
    double deltaq = (kt * kt) / 4.0 * (1.0 + w_Q) * (4.0 - 3.0 * cs2_Q) / (4.0 - 6.0 * w_Q + 3.0 * cs2_Q) * ci * s2;
    double thetaq = (kt * kt * kt * kt) / tau / 4.0 * cs2_Q / (4.0 - 6.0 * w_Q + 3.0 * cs2_Q) * ci * s2;
    double eta = ci * (1.0 - (kt * kt) / 12.0 / (15.0 + 4.0 * fracnu) *
                                 (5.0 + 4.0 * s2 * fracnu -
                                  (16.0 * fracnu * fracnu + 280.0 * fracnu + 325.0) / 10.0 / (2.0 * fracnu + 15.0) * tau * om));
    y[0] = a; y[1] = 0.0; y[2] = eta;
    y[3] = deltac; y[4] = thetac; y[5] = deltab; y[6] = thetab; y[7] = deltag; y[8] = thetag;
    y[9 + lmaxg + lmaxgp] = deltar;
    y[10 + lmaxg + lmaxgp] = thetar;
    y[11 + lmaxg + lmaxgp] = shearr * 2.0;
    for (int i = 0; i < nq; ++i) {
        double q = P->q[i];
        double aq = a * P->amnu / q;
        double v = 1.0 / sqrt(1.0 + aq * aq);
        double dlfdlq = -q / (1.0 + exp(-q));
        y[iq0 + i] = -0.25 * dlfdlq * deltar;
        y[iq1 + i] = -dlfdlq * thetar / v / kmode / 3.0;
        y[iq2 + i] = -0.5 * dlfdlq * shearr;
    }
    y[n - 2] = deltaq;
    y[n - 1] = thetaq;
}

/* ---- RSA output projection (approximations.py:84-176) ---- */
void oracle_rsa_project(const OracleProblem* P, double tau, double kmode, const double* y, double* out)
{
    const int n = P->n, lmaxg = P->lmaxg, lmaxgp = P->lmaxgp, lmaxr = P->lmaxr, nq = P->nqmax;
    memcpy(out, y, sizeof(double) * n);
    double a = y[0], loga = log(a), eta = y[2], deltab = y[5], thetab = y[6];
    double aprimeoa = aprimeoa_r(P, a);
    double cs2 = spl_eval_r(&P->cs2a_loga, loga) / a;
    double xe = spl_eval_r(&P->xe_loga, loga);
    double xeprime = spl_deriv_r(&P->xe_loga, loga) * aprimeoa;
    double akthom = 2.3038921003709498e-9 * (1.0 - P->YHe) * P->Omegab * P->H0 * P->H0;
    double opac = xe * akthom / (a * a);
    double tau_c = 1.0 / (opac > 1e-30 ? opac : 1e-30);
    double tau_c_prime = tau_c * (2.0 * aprimeoa - xeprime / (xe > 1e-30 ? xe : 1e-30));
    double Omegac = P->Omegam - P->Omegab;
    const int iq0 = 10 + lmaxg + lmaxgp + lmaxr;
    double drhonu = 0.0;
    for (int i = 0; i < nq; ++i) {
        double aq = a * P->amnu / P->q[i];
        double v = 1.0 / sqrt(1.0 + aq * aq);
        drhonu += P->w[i] * y[iq0 + i] / v;
    }
    double rho_Q = pow(a, -3.0 * (1.0 + P->w0 + P->wa)) * exp(3.0 * (a - 1.0) * P->wa);
    double dgrho_wo_rel = P->grhom * (Omegac * y[3] + P->Omegab * deltab) / a + P->grhor * P->Nmnu * drhonu / (a * a) +
                          P->grhom * P->OmegaDE * y[n - 2] * rho_Q * a * a;
    double k2 = kmode * kmode;
    double hprime = (2.0 * k2 * eta + dgrho_wo_rel) / (aprimeoa > 1e-30 ? aprimeoa : 1e-30);
    double sk2 = k2 > 1e-30 ? k2 : 1e-30, stc = tau_c > 1e-30 ? tau_c : 1e-30;
    double deltag = 4.0 / sk2 * (aprimeoa * hprime - sk2 * eta) + 4.0 / (sk2 * stc) * (thetab + 0.5 * hprime);
    double thetag = -0.5 * hprime + 3.0 / (sk2 * stc) *
                    (-tau_c_prime / stc * (thetab + 0.5 * hprime) + (-aprimeoa * thetab + cs2 * sk2 * deltab + sk2 * eta));
    double deltar = 4.0 / sk2 * (aprimeoa * hprime - sk2 * eta);
    double thetar = -0.5 * hprime;
    int do_rsa = P->use_rsa && (tau_c / (tau > 1e-30 ? tau : 1e-30) > P->rsa_tau_c_over_tau) &&
                 (tau * kmode > P->rsa_tau_over_tau_k);
    if (!do_rsa) return;
    const int idxg = 7, idxgp = 7 + lmaxg + 1, idxr = 9 + lmaxg + lmaxgp;
    out[idxg] = deltag; out[idxg + 1] = thetag; out[idxg + 2] = 0.0;
    for (int l = 3; l <= lmaxg; ++l) out[idxg + l] = 0.0;
    for (int l = 0; l <= lmaxgp; ++l) out[idxgp + l] = 0.0;
    out[idxr] = deltar; out[idxr + 1] = thetar; out[idxr + 2] = 0.0;
    for (int l = 3; l <= lmaxr; ++l) out[idxr + l] = 0.0;
}

/* ---- output fields (perturbations.py:528-677) ---- */
void oracle_output_vars(const OracleProblem* P, double kmode, const double* y, double* o)
{
    const int n = P->n, lmaxg = P->lmaxg, lmaxgp = P->lmaxgp, lmaxr = P->lmaxr, nq = P->nqmax;
    const double Omegac = P->Omegam - P->Omegab;
    const int iq0 = 10 + lmaxg + lmaxgp + lmaxr, iq1 = iq0 + nq;
    double a = y[0], eta = y[2], deltac = y[3], thetac = y[4], deltab = y[5], thetab = y[6];
    double deltag = y[7], thetag = y[8], deltar = y[9 + lmaxg + lmaxgp], thetar = y[10 + lmaxg + lmaxgp];
    double rhonu = exp(spl_eval_r(&P->logrhonu_loga, log(a)));
    double pnu = exp(spl_eval_r(&P->logpnu_loga, log(a)));
    double rho_plus_p = rhonu + pnu;
    double drhonu = 0.0, fnu = 0.0;
    for (int i = 0; i < nq; ++i) {
        double aq = a * P->amnu / P->q[i];
        double v = 1.0 / sqrt(1.0 + aq * aq);
        drhonu += P->w[i] * y[iq0 + i] / v;
        fnu += P->w[i] * y[iq1 + i];
    }
    double deltanu = drhonu / rhonu, thetanu = kmode * fnu / rho_plus_p;
    double deltaq = y[n - 2], thetaq = y[n - 1];
    double w_Q = P->w0 + P->wa * (1.0 - a);
    double rho_Q = pow(a, -3.0 * (1.0 + P->w0 + P->wa)) * exp(3.0 * (a - 1.0) * P->wa);
    double rpt = (1.0 + w_Q) * rho_Q * P->grhom * P->OmegaDE * thetaq * a * a;
    double a2 = a * a;
    double grho = P->grhom * P->Omegam / a + (P->grhog + P->grhor * (P->Neff + P->Nmnu * rhonu)) / a2 +
                  P->grhom * P->OmegaDE * rho_Q * a2 + P->grhom * P->Omegak;
    double aprimeoa = sqrt(grho / 3.0);
    double dgrho = P->grhom * (Omegac * deltac + P->Omegab * deltab) / a +
                   (P->grhog * deltag + P->grhor * (P->Neff * deltar + P->Nmnu * drhonu)) / a2 +
                   P->grhom * P->OmegaDE * deltaq * rho_Q * a2;
    double dgtheta = P->grhom * (Omegac * thetac + P->Omegab * thetab) / a +
                     4.0 / 3.0 * (P->grhog * thetag + P->Neff * P->grhor * thetar) / a2 +
                     P->Nmnu * P->grhor * kmode * fnu / a2 + rpt;
    double k2 = kmode * kmode;
    double hprime = (2.0 * k2 * eta + dgrho) / aprimeoa;
    double etaprime = 0.5 * dgtheta / k2;
    double alpha = (hprime + 6.0 * etaprime) / 2.0 / k2;
    double deltam = (P->grhom * (Omegac * deltac + P->Omegab * deltab) / a + (P->grhor * P->Nmnu * drhonu) / a2) /
                    (P->grhom * P->Omegam / a + (P->grhor * P->Nmnu * rhonu) / a2);
    double thetam = (P->grhom * (Omegac * thetac + P->Omegab * thetab) / a + P->Nmnu * P->grhor * kmode * fnu / a2) /
                    (3.0 * (P->grhom * P->Omegam / a + P->grhor * P->Nmnu * rhonu / a2));
    double deltabc = (P->grhom * (Omegac * deltac + P->Omegab * deltab) / a) / (P->grhom * P->Omegam / a);
    double thetabc = (P->grhom * (Omegac * thetac + P->Omegab * thetab) / a) / (3.0 * (P->grhom * P->Omegam / a) / a2);
    thetam += alpha * k2;
    thetabc += alpha * k2;
    double v[20] = {eta, etaprime, hprime, alpha, deltam, thetam / aprimeoa, deltabc, thetabc / aprimeoa,
                    deltac, thetac / aprimeoa, deltab, thetab / aprimeoa, deltag, thetag / aprimeoa,
                    deltar, thetar / aprimeoa, deltanu, thetanu / aprimeoa, deltaq, thetaq / aprimeoa};
    memcpy(o, v, sizeof(v));
}

/* ---- approximation switch times (used by the clipped, per-step-regime mode) ---- */
static double tauc_of_tau(const OracleProblem* P, double tau)
{
    double a = spl_eval_r(&P->a_of_tau, tau);
    double xe = spl_eval_r(&P->xe_loga, log(a));
    double akthom = 2.3038921003709498e-9 * (1.0 - P->YHe) * P->Omegab * P->H0 * P->H0;
    double opac = xe * akthom / (a * a);
    return 1.0 / (opac > 1e-30 ? opac : 1e-30);
}

static double bisect_increasing(const OracleProblem* P, double (*g)(const OracleProblem*, double, double), double par,
                                double lo, double hi)
{
    /* root of increasing g on [lo, hi] in log tau */
    double l = log(lo), r = log(hi);
    if (g(P, exp(l), par) > 0) return lo;
    if (g(P, exp(r), par) <= 0) return INFINITY;
    for (int it = 0; it < 200; ++it) {
        double m = 0.5 * (l + r);
        if (g(P, exp(m), par) > 0) r = m; else l = m;
        if (r - l < 1e-15) break;
    }
    return exp(r);
}

static double g_rsa(const OracleProblem* P, double tau, double par)
{
    (void)par;
    return tauc_of_tau(P, tau) / tau - P->rsa_tau_c_over_tau;
}

static double g_tca(const OracleProblem* P, double tau, double k)
{
    double tc = tauc_of_tau(P, tau);
    double a = spl_eval_r(&P->a_of_tau, tau);
    double th = 1.0 / aprimeoa_r(P, a);
    double tk = 1.0 / k;
    int unc = (tc / tk > P->tca_tau_c_over_tau_k) ||
              ((tc / th > P->tca_tau_c_over_tau_h) && (tc / tk > 0.1 * P->tca_tau_c_over_tau_k));
    return unc ? 1.0 : -1.0;
}

void oracle_switch_times(const OracleProblem* P, double k, double* sw)
{
    double lo = P->a_of_tau.x[0], hi = P->a_of_tau.x[P->a_of_tau.n - 1];
    double t_rsa = INFINITY, t_ufa = INFINITY, t_tca = INFINITY;
    if (P->use_rsa) {
        double tc = bisect_increasing(P, g_rsa, 0.0, lo, hi);
        double tk = P->rsa_tau_over_tau_k / k;
        t_rsa = tc > tk ? tc : tk;
    }
    if (P->use_ufa) t_ufa = P->ufa_tau_over_tau_k / k;
    if (P->use_tca) t_tca = bisect_increasing(P, g_tca, k, lo, hi);
    sw[0] = t_rsa; sw[1] = t_ufa; sw[2] = t_tca;
}

int oracle_regime(const OracleProblem* P, double tau, const double* sw)
{
    int rsa = P->use_rsa && tau >= sw[0];
    int ufa = !rsa && P->use_ufa && tau >= sw[1];
    int tca = !rsa && P->use_tca && tau < sw[2];
    return (rsa ? 1 : 0) | (ufa ? 2 : 0) | (tca ? 4 : 0);
}

/* ---- dense LU with partial pivoting (jax.scipy.linalg.lu_factor / lu_solve) ---- */
static int lu_factor(int n, double* A, int* piv)
{
    for (int k = 0; k < n; ++k) {
        int p = k;
        double m = fabs(A[k * n + k]);
        for (int i = k + 1; i < n; ++i) {
            double v = fabs(A[i * n + k]);
            if (v > m) { m = v; p = i; }
        }
        piv[k] = p;
        if (p != k)
            for (int j = 0; j < n; ++j) { double t = A[k * n + j]; A[k * n + j] = A[p * n + j]; A[p * n + j] = t; }
        double d = A[k * n + k];
        if (d == 0.0) return 1;
        for (int i = k + 1; i < n; ++i) {
            double l = A[i * n + k] / d;
            A[i * n + k] = l;
            if (l != 0.0)
                for (int j = k + 1; j < n; ++j) A[i * n + j] -= l * A[k * n + j];
        }
    }
    return 0;
}

static void lu_solve(int n, const double* LU, const int* piv, double* b)
{
    for (int k = 0; k < n; ++k) {
        int p = piv[k];
        if (p != k) { double t = b[k]; b[k] = b[p]; b[p] = t; }
    }
    for (int i = 0; i < n; ++i) {
        double s = b[i];
        for (int j = 0; j < i; ++j) s -= LU[i * n + j] * b[j];
        b[i] = s;
    }
    for (int i = n - 1; i >= 0; --i) {
        double s = b[i];
        for (int j = i + 1; j < n; ++j) s -= LU[i * n + j] * b[j];
        b[i] = s / LU[i * n + i];
    }
}

/* ---- Rodas5 tableau (Di Marzo 1993), as used at ode_integrators_stiff.py:680-746 ---- */
static const double R5_gamma = 0.19;
static const double R5_a[8][8] = {
    {0},
    {2.0},
    {3.040894194418781, 1.041747909077569},
    {2.576417536461461, 1.622083060776640, -0.9089668560264532},
    {2.760842080225597, 1.446624659844071, -0.3036980084553738, 0.2877498600325443},
    {-14.09640773051259, 6.925207756232704, -41.47510893210728, 2.343771018586405, 24.13215229196062},
    {0}, {0}};
static const double R5_C[8][8] = {
    {0},
    {-10.31323885133993},
    {-21.04823117650003, -7.234992135176716},
    {32.22751541853323, -4.943732386540191, 19.44922031041879},
    {-20.69865579590063, -8.816374604402768, 1.260436877740897, -0.7495647613787146},
    {-46.22004352711257, -17.49534862857472, -289.6389582892057, 93.60855400400906, 318.3822534212147},
    {34.20013733472935, -14.15535402717690, 57.82335640988400, 25.83362985412365, 1.408950972071624, -6.551835421242162},
    {42.57076742291101, -13.80770672017997, 93.98938432427124, 18.77919633714503, -31.58359187223370, -6.685968952921985,
     -5.810979938412932}};
static const double R5_c[6] = {0.0, 0.38, 0.3878509998321533, 0.4839718937873840, 0.4570477008819580, 1.0};
static const double R5_d[5] = {0.19, -0.1823079225333714636, -0.319231832186874912, 0.3449828624725343,
                               -0.377417564392089818};

typedef struct {
    double *J, *dT, *K, *u, *f, *rhs;
    int* piv;
} Work;

/* one Rodas5 step for one mode; returns y1 and err (= k8); regime fixed or literal */
static int rodas5_step(const OracleProblem* P, double k, double t0, double dt, const double* y0, double* y1,
                       double* err, Work* W, int regime)
{
    const int n = P->n;
    double* J = W->J;
    oracle_jacobian(P, t0, y0, k, J, W->dT, regime);
    double ig = 1.0 / (dt * R5_gamma);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) J[i * n + j] = (i == j ? ig : 0.0) - J[i * n + j];
    if (lu_factor(n, J, W->piv)) return 2;
    double* K = W->K; /* 8 x n */
    for (int s = 0; s < 8; ++s) {
        double ts;
        if (s == 0) {
            memcpy(W->u, y0, sizeof(double) * n);
            ts = t0;
        } else if (s <= 5) {
            for (int i = 0; i < n; ++i) {
                double v = y0[i];
                for (int j = 0; j < s; ++j) v += R5_a[s][j] * K[j * n + i];
                W->u[i] = v;
            }
            ts = t0 + R5_c[s] * dt;
        } else {
            for (int i = 0; i < n; ++i) W->u[i] += K[(s - 1) * n + i];
            ts = t0 + dt;
        }
        rhs_r(P, ts, W->u, k, W->f, regime);
        for (int i = 0; i < n; ++i) {
            double r = W->f[i];
            if (s < 5) r += dt * R5_d[s] * W->dT[i];
            for (int j = 0; j < s; ++j) r += R5_C[s][j] / dt * K[j * n + i];
            W->rhs[i] = r;
        }
        lu_solve(n, J, W->piv, W->rhs);
        memcpy(&K[s * n], W->rhs, sizeof(double) * n);
    }
    for (int i = 0; i < n; ++i) {
        y1[i] = W->u[i] + K[7 * n + i];
        err[i] = K[7 * n + i];
    }
    for (int i = 0; i < n; ++i)
        if (!isfinite(y1[i])) return 2;
    return 0;
}

static int next_event(int nout, const double* tout, int iout, const double* sw, int use_sw, double t, double t1,
                      double* tev)
{
    double te = t1;
    if (iout < nout && tout[iout] < te) te = tout[iout];
    if (use_sw)
        for (int i = 0; i < 3; ++i)
            if (sw[i] > t && sw[i] < te) te = sw[i];
    *tev = te;
    return 0;
}

int oracle_solve(const OracleProblem* P, const OracleControl* C, int nb, const double* kv, double t0,
                 const double* y0, int nout, const double* tout, const double* sw, double* yout, OracleStats* st)
{
    const int n = P->n;
    Work W;
    W.J = (double*)malloc(sizeof(double) * n * n);
    W.dT = (double*)malloc(sizeof(double) * n);
    W.K = (double*)malloc(sizeof(double) * 8 * n);
    W.u = (double*)malloc(sizeof(double) * n);
    W.f = (double*)malloc(sizeof(double) * n);
    W.rhs = (double*)malloc(sizeof(double) * n);
    W.piv = (int*)malloc(sizeof(int) * n);
    double* y = (double*)malloc(sizeof(double) * nb * n);
    double* y1 = (double*)malloc(sizeof(double) * nb * n);
    double* er = (double*)malloc(sizeof(double) * nb * n);
    memcpy(y, y0, sizeof(double) * nb * n);
    memset(st, 0, sizeof(*st));

    double t1 = tout[0];
    for (int i = 1; i < nout; ++i) if (tout[i] > t1) t1 = tout[i];
    const double error_order = 6.0; /* Rodas5 order 5, diffrax error order = order + 1 */
    const double c1 = (C->icoeff + C->pcoeff + C->dcoeff) / error_order;
    const double c2 = -(C->pcoeff + 2.0 * C->dcoeff) / error_order;
    const double c3 = C->dcoeff / error_order;
    double prev_inv = 1.0, prev_prev_inv = 1.0;
    double t = t0;
    double dt = fmin(t0 / 4.0, 0.5 * (t1 - t0));
    int iout = 0;
    const int idx[6] = {0, 2, 3, 5, 6, 7};
    int status = 0;
    const int use_sw = !C->literal_regime;
    while (t < t1) {
        if (st->steps >= C->max_steps) { status = 1; break; }
        double tn, tev;
        int clipped = 0;
        const double dt_try = dt;
        if (C->linear_interp) {
            tn = t + dt;
            double tol = 1e-10 * fabs(tn);
            if (tn > t1 - tol) tn = t1;
        } else {
            next_event(nout, tout, iout, sw, use_sw && nb == 1, t, t1, &tev);
            tn = t + dt;
            if (tn >= tev - 1e-12 * fabs(tev)) { clipped = (tn > tev); tn = tev; }
        }
        double h = tn - t;
        double sumsq = 0.0;
        int bad = 0;
        for (int b = 0; b < nb && !bad; ++b) {
            int regime = C->literal_regime ? -1 : oracle_regime(P, t, sw + 3 * b);
            int rc = rodas5_step(P, kv[b], t, h, y + b * n, y1 + b * n, er + b * n, &W, regime);
            if (rc) { bad = 1; break; }
            double wts[6] = {1.0, kv[b] * kv[b], 1.0, 1.0, 1.0 / (kv[b] * kv[b]), 1.0};
            for (int m = 0; m < 6; ++m) {
                int i = idx[m];
                double sc = fabs(y[b * n + i]) > fabs(y1[b * n + i]) ? fabs(y[b * n + i]) : fabs(y1[b * n + i]);
                double e = er[b * n + i] / (C->atol + C->rtol * sc) * wts[m];
                sumsq += e * e;
            }
        }
        st->steps++;
        double err = bad ? INFINITY : sqrt(sumsq / (6.0 * nb));
        int keep = err < 1.0;
        double inv = 1.0 / err;
        double f1 = pow(inv, c1);
        double f2 = (c2 == 0.0) ? 1.0 : pow(prev_inv, c2);
        double f3 = (c3 == 0.0) ? 1.0 : pow(prev_prev_inv, c3);
        double fmn = keep ? 1.0 : C->factormin;
        double factor = 0.9 * f1 * f2 * f3;
        if (!(factor == factor)) factor = fmn;
        if (factor < fmn) factor = fmn;
        if (factor > C->factormax) factor = C->factormax;
        if (inv == 0.0 || isinf(inv)) inv = 1.0;
        double dtn = h * factor;
        if (keep) {
            st->accepted++;
            if (C->linear_interp) {
                while (iout < nout && tout[iout] <= tn) {
                    double c = (tout[iout] - t) / h;
                    for (int b = 0; b < nb; ++b)
                        for (int i = 0; i < n; ++i)
                            yout[((size_t)b * nout + iout) * n + i] =
                                y[b * n + i] + c * (y1[b * n + i] - y[b * n + i]);
                    iout++;
                }
            } else {
                while (iout < nout && tout[iout] <= tn) {
                    for (int b = 0; b < nb; ++b)
                        memcpy(&yout[((size_t)b * nout + iout) * n], y1 + b * n, sizeof(double) * n);
                    iout++;
                }
                if (clipped && dt_try > dtn) dtn = dt_try;
            }
            memcpy(y, y1, sizeof(double) * nb * n);
            t = tn;
            prev_prev_inv = prev_inv;
            prev_inv = inv;
        } else {
            st->rejected++;
            if (bad && h < 1e-300) { status = 2; break; }
        }
        dt = dtn;
    }
    st->status = status;
    free(W.J); free(W.dT); free(W.K); free(W.u); free(W.f); free(W.rhs); free(W.piv);
    free(y); free(y1); free(er);
    return status;
}
