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
#include "team.cuh"

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

// knot values, with tangent arrays (may be null) seeded into the first-derivative slot
template <class T> DHD T knot(const double* a, const double* ad, int i)
{
    return seed_t<T>(DLDG(a + i), ad ? DLDG(ad + i) : 0.0);
}

template <class T>
DHD T spline_eval_at(const DiscoebSpline& s, int i, T xn, const double* yd = nullptr, const double* Sd = nullptr)
{
    double xi = DLDG(s.x + i), xj = DLDG(s.x + i + 1);
    double h = xj - xi;
    T t = (xn - xi) * (1.0 / h);
    T A = 1.0 - t, B = t;
    return A * knot<T>(s.y, yd, i) + B * knot<T>(s.y, yd, i + 1) +
           ((A * A * A - A) * knot<T>(s.S, Sd, i) + (B * B * B - B) * knot<T>(s.S, Sd, i + 1)) * (h * h / 6.0);
}

template <class T>
DHD T spline_deriv_at(const DiscoebSpline& s, int i, T xn, const double* yd = nullptr, const double* Sd = nullptr)
{
    double xi = DLDG(s.x + i), xj = DLDG(s.x + i + 1);
    double h = xj - xi;
    const T yi = knot<T>(s.y, yd, i), yj = knot<T>(s.y, yd, i + 1), Si = knot<T>(s.S, Sd, i), Sj = knot<T>(s.S, Sd, i + 1);
    T d = xn - xi;
    T b = (yj - yi) * (1.0 / h) - h * (Sj + 2.0 * Si) * (1.0 / 6.0);
    T c = Si * 0.5;
    T dd = (Sj - Si) * (1.0 / (6.0 * h));
    return b + 2.0 * c * d + 3.0 * dd * d * d;
}

template <class T> DHD T spline_eval(const DiscoebSpline& s, T xn) { return spline_eval_at(s, spline_index(s, val(xn)), xn); }

// ---- parameters that depend on the cosmological parameters (typed, so that tangents flow) ----
template <class T> struct Par {
    T grhom, Omegam, Omegab, OmegaDE, amnu, w0, wa, akthom;
};

// parameter values, with their derivatives along a tangent direction seeded into the
// first-derivative slot of T (tn == nullptr: no tangent)
template <class T> DHD Par<T> make_par(const DiscoebCosmo& P, const DiscoebTangent* tn)
{
    Par<T> r;
    const double z = 0.0;
    r.grhom = seed_t<T>(P.grhom, tn ? tn->grhom : z);
    r.Omegam = seed_t<T>(P.Omegam, tn ? tn->Omegam : z);
    r.Omegab = seed_t<T>(P.Omegab, tn ? tn->Omegab : z);
    r.OmegaDE = seed_t<T>(P.OmegaDE, tn ? tn->OmegaDE : z);
    r.amnu = seed_t<T>(P.amnu, tn ? tn->amnu : z);
    r.w0 = seed_t<T>(P.w0, tn ? tn->w0 : z);
    r.wa = seed_t<T>(P.wa, tn ? tn->wa : z);
    const double c = 2.3038921003709498e-9 * (1.0 - P.YHe);
    const T H0 = seed_t<T>(P.H0, tn ? tn->H0 : z);
    r.akthom = c * r.Omegab * H0 * H0;
    return r;
}

// ---- background quantities at (a, tau) ----
template <class T> struct Bg {
    Par<T> par;
    T a, ia, a2, ia2, aH, iaHG, opac, po, tauc, taucprime, cs2, pb43, rho_Q, w_Q, opw, iopw, ca2_Q, pnu;
    T rsa_fac, rsa_tcs;  // 3/(k^2 tau_c), tau_c'/tau_c (RSA fields)
    T aprimeprimeoa;
    double itau;
    bool rsa, ufa, tca, de_frozen;
};

// value part of a background evaluated in dual numbers (the same operations on the values): a
// Bg<Dual> gives the double background, a Bg<HDual> the Bg<Dual> of its first direction
template <class B> DHD Bg<B> bg_value(const Bg<DualT<B>>& d)
{
    Bg<B> b;
    b.par = Par<B>{d.par.grhom.v, d.par.Omegam.v, d.par.Omegab.v, d.par.OmegaDE.v, d.par.amnu.v, d.par.w0.v,
                   d.par.wa.v, d.par.akthom.v};
    b.a = d.a.v; b.ia = d.ia.v; b.a2 = d.a2.v; b.ia2 = d.ia2.v; b.aH = d.aH.v; b.iaHG = d.iaHG.v;
    b.opac = d.opac.v; b.po = d.po.v; b.tauc = d.tauc.v; b.taucprime = d.taucprime.v; b.cs2 = d.cs2.v;
    b.pb43 = d.pb43.v; b.rho_Q = d.rho_Q.v; b.w_Q = d.w_Q.v; b.opw = d.opw.v; b.iopw = d.iopw.v;
    b.ca2_Q = d.ca2_Q.v; b.pnu = d.pnu.v; b.rsa_fac = d.rsa_fac.v; b.rsa_tcs = d.rsa_tcs.v;
    b.aprimeprimeoa = d.aprimeprimeoa.v;
    b.itau = d.itau;
    b.rsa = d.rsa; b.ufa = d.ufa; b.tca = d.tca; b.de_frozen = d.de_frozen;
    return b;
}

// velocity of momentum bin q: v = 1/sqrt(1 + (a m/q)^2), and its inverse
template <class T> DHD T inv_vq(const DiscoebCosmo& P, const Bg<T>& b, int q)
{
    const T aq = b.a * b.par.amnu * (1.0 / P.q[q]);
    return xsqrt(1.0 + aq * aq);
}

// a'/a (get_aprimeoa, background.py:101-123) from the massive-neutrino density rho_nu at a
template <class T> DHD T aprimeoa_from(const DiscoebCosmo& P, const Par<T>& par, T a, T loga, T rhonu)
{
    T rho_Q = xexp(-3.0 * (1.0 + par.w0 + par.wa) * loga + 3.0 * (a - 1.0) * par.wa);
    T grho = par.grhom * par.Omegam / a + (P.grhog + P.grhor * (P.Neff + P.Nmnu * rhonu)) / (a * a) +
             par.grhom * par.OmegaDE * rho_Q * a * a + par.grhom * P.Omegak;
    return xsqrt(grho * (1.0 / 3.0));
}

template <class T> DHD T aprimeoa_of(const DiscoebCosmo& P, const Par<T>& par, const DiscoebTangent* tn, T a, T loga)
{
    const int i = spline_index(P.logrhonu_loga, val(loga));
    T rhonu = xexp(spline_eval_at(P.logrhonu_loga, i, loga, tn ? tn->logrhonu_y : nullptr, tn ? tn->logrhonu_S : nullptr));
    return aprimeoa_from(P, par, a, loga, rhonu);
}

// index of a non-uniform spline searched from a hint (the previous index): same result
// as spline_index (count of knots below xn, minus one, clipped) in O(|step|) loads
DHD int spline_index_from(const DiscoebSpline& s, double xn, int& hint)
{
    if (s.uniform) return spline_index(s, xn);
    const int n = s.n_knots;
    int i = hint < 0 ? 0 : (hint > n - 2 ? n - 2 : hint);
    while (i > 0 && !(DLDG(s.x + i) < xn)) --i;
    while (i < n - 2 && DLDG(s.x + i + 1) < xn) ++i;
    hint = i;
    return i;
}

// The six table-derived quantities at log a: xe, dxe/dloga, cs2*a, rho_nu, p_nu, rho_Q.
// Table slot t (0..4) is computed by one lane of a team (t % nl), with the same
// instruction stream on every lane, and broadcast.
template <class T> struct BgTables {
    T xe, xep, cs2a, rhonu, pnu, rho_Q;
};

DHD const DiscoebSpline& table_slot_spline(const DiscoebCosmo& P, int t)
{
    return t == 0 ? P.xe_loga : (t == 1 ? P.cs2a_loga : (t == 2 ? P.logrhonu_loga : P.logpnu_loga));
}

// interval index of table slot t (0..3) at log a; slot 0 (xe) moves the hint
DHD int table_slot_index(const DiscoebCosmo& P, int t, double loga, int& hint)
{
    int h = hint;
    const int i = spline_index_from(table_slot_spline(P, t), loga, h);
    if (t == 0) hint = h;
    return i;
}

// value of table slot t at log a in interval i (t: 0 xe with its derivative, 1 cs2*a,
// 2 log rho_nu, 3 log p_nu, 4 log rho_Q, which needs no table)
template <class T>
DHD T table_slot_eval(const DiscoebCosmo& P, const Par<T>& par, const DiscoebTangent* tn, int t, int i, T a, T loga,
                      T& deriv)
{
    if (t == 4) {
        deriv = 0.0;
        return -3.0 * (1.0 + par.w0 + par.wa) * loga + 3.0 * (a - 1.0) * par.wa;
    }
    const DiscoebSpline& s = table_slot_spline(P, t);
    const double* yd = nullptr;
    const double* Sd = nullptr;
    if (tn) {
        yd = t == 0 ? tn->xe_y : (t == 1 ? tn->cs2a_y : (t == 2 ? tn->logrhonu_y : tn->logpnu_y));
        Sd = t == 0 ? tn->xe_S : (t == 1 ? tn->cs2a_S : (t == 2 ? tn->logrhonu_S : tn->logpnu_S));
    }
    deriv = spline_deriv_at(s, i, loga, yd, Sd);
    return spline_eval_at(s, i, loga, yd, Sd);
}

template <class T>
DHD T table_slot_value(const DiscoebCosmo& P, const Par<T>& par, const DiscoebTangent* tn, int t, T a, T loga,
                       int& hint, T& deriv)
{
    if (t == 4) return table_slot_eval(P, par, tn, 4, 0, a, loga, deriv);
    const DiscoebSpline& s = table_slot_spline(P, t);
    const double* yd = nullptr;
    const double* Sd = nullptr;
    if (tn) {
        yd = t == 0 ? tn->xe_y : (t == 1 ? tn->cs2a_y : (t == 2 ? tn->logrhonu_y : tn->logpnu_y));
        Sd = t == 0 ? tn->xe_S : (t == 1 ? tn->cs2a_S : (t == 2 ? tn->logrhonu_S : tn->logpnu_S));
    }
    int h = hint;
    const int i = spline_index_from(s, val(loga), h);
    if (t == 0) hint = h;
    deriv = spline_deriv_at(s, i, loga, yd, Sd);
    return spline_eval_at(s, i, loga, yd, Sd);
}

template <class TM, class T>
DHD BgTables<T> bg_tables(const TM& tm, const DiscoebCosmo& P, const Par<T>& par, const DiscoebTangent* tn, T a,
                          int& hint)
{
    const T loga = xlog(a);
    BgTables<T> r;
    if (tm.nl == 1) {
        T d;
        int h = hint;
        r.xe = table_slot_value(P, par, tn, 0, a, loga, h, r.xep);
        r.cs2a = table_slot_value(P, par, tn, 1, a, loga, hint, d);
        r.rhonu = xexp(table_slot_value(P, par, tn, 2, a, loga, hint, d));
        r.pnu = xexp(table_slot_value(P, par, tn, 3, a, loga, hint, d));
        r.rho_Q = xexp(table_slot_value(P, par, tn, 4, a, loga, hint, d));
        hint = h;
        return r;
    }
    // lanes 0..4 each evaluate one table slot, then broadcast.  The lanes reach their interval
    // index by different paths (uniform knots, a search from the hint, none for rho_Q).  With
    // TM::reconverge the team reconverges after the index and again before the exponential, so
    // that the evaluation and the exponential run once for all five lanes rather than once per
    // path; otherwise each lane runs its slot in one piece.
    int h = hint;
    T v = 0.0, d = 0.0;
    if constexpr (TM::reconverge) {
        int idx = 0;
        if (tm.lane < 4) idx = table_slot_index(P, tm.lane, val(loga), h);
        tm.sync();
        if (tm.lane < 5) v = table_slot_eval(P, par, tn, tm.lane, idx, a, loga, d);
        tm.sync();
        if (tm.lane >= 2 && tm.lane < 5) v = xexp(v);
    } else {
        if (tm.lane < 5) {
            v = table_slot_value(P, par, tn, tm.lane, a, loga, h, d);
            if (tm.lane >= 2) v = xexp(v);
        }
    }
    r.xe = tm.bcast(v, 0);
    r.xep = tm.bcast(d, 0);
    r.cs2a = tm.bcast(v, 1);
    r.rhonu = tm.bcast(v, 2);
    r.pnu = tm.bcast(v, 3);
    r.rho_Q = tm.bcast(v, 4);
    hint = (int)tm.bcast((double)h, 0);
    return r;
}

// regime < 0: switches from (tau, a) exactly as model_synchronous evaluates them;
// otherwise bitmask 1 = RSA, 2 = UFA, 4 = TCA.
template <class T>
DHD void bg_finish(const DiscoebCosmo& P, const Par<T>& par, T a, const BgTables<T>& tb, double tau, double k,
                   int regime, Bg<T>& b)
{
    b.par = par;
    b.a = a;
    b.ia = rcp(a);
    b.a2 = a * a;
    b.ia2 = b.ia * b.ia;
    b.itau = rcp(tau);
    const T& xe = tb.xe;
    b.cs2 = tb.cs2a * b.ia;
    b.pnu = tb.pnu;
    b.pb43 = (4.0 / 3.0) * P.grhog * rcp(par.grhom * par.Omegab) * b.ia;
    b.w_Q = par.w0 + par.wa * (1.0 - a);
    b.opw = 1.0 + b.w_Q;
    b.iopw = rcp(b.opw);
    b.rho_Q = tb.rho_Q;
    T grho = par.grhom * par.Omegam * b.ia + (P.grhog + P.grhor * (P.Neff + P.Nmnu * tb.rhonu)) * b.ia2 +
             par.grhom * par.OmegaDE * b.rho_Q * b.a2 + par.grhom * P.Omegak;
    b.aH = xsqrt(grho * (1.0 / 3.0));
    const T iaH = rcp(b.aH);
    T xeprime = tb.xep * b.aH;
    T gpres = ((P.grhog + P.grhor * P.Neff) * (1.0 / 3.0) + P.grhor * P.Nmnu * b.pnu) * b.ia2 +
              b.w_Q * par.grhom * par.OmegaDE * b.rho_Q * b.a2;
    b.aprimeprimeoa = 0.5 * (b.aH * b.aH - gpres);
    T w_Q_prime = -par.wa * b.aH * a;
    b.ca2_Q = b.w_Q - w_Q_prime * (1.0 / 3.0) / ((1.0 + b.w_Q) + 1e-6) * iaH;
    b.opac = xe * par.akthom * b.ia2;
    b.po = b.pb43 * b.opac;
    b.tauc = rcp(xmaxc(b.opac, 1e-30));
    b.taucprime = b.tauc * (2.0 * b.aH - xeprime / xmaxc(xe, 1e-30));
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
    b.iaHG = b.rsa ? rcp(xmaxc(b.aH, 1e-30)) : iaH;
    if (b.rsa) {
        const double k2 = k * k, sk2 = k2 > 1e-30 ? k2 : 1e-30;
        const T stc = xmaxc(b.tauc, 1e-30);
        const T istc = rcp(stc);
        b.rsa_fac = (3.0 / sk2) * istc;
        b.rsa_tcs = b.taucprime * istc;
    } else {
        b.rsa_fac = 0.0;
        b.rsa_tcs = 0.0;
    }
    b.de_frozen = P.de_guard_eps > 0.0 && fabs(val(1.0 + b.w_Q)) < P.de_guard_eps;
}

template <class TM, class T>
DHD void bg_eval_team(const TM& tm, const DiscoebCosmo& P, T a, double tau, double k, int regime, Bg<T>& b, int& hint,
                      const DiscoebTangent* tn = nullptr)
{
    const Par<T> par = make_par<T>(P, tn);
    const BgTables<T> tb = bg_tables(tm, P, par, tn, a, hint);
    bg_finish(P, par, a, tb, tau, k, regime, b);
}

template <class T>
DHD void bg_eval(const DiscoebCosmo& P, T a, double tau, double k, int regime, Bg<T>& b, int& hint,
                 const DiscoebTangent* tn = nullptr)
{
    bg_eval_team(HostTeam(), P, a, tau, k, regime, b, hint, tn);
}

template <class T> DHD void bg_eval(const DiscoebCosmo& P, T a, double tau, double k, int regime, Bg<T>& b)
{
    int hint = P.xe_loga.n_knots / 2;
    bg_eval(P, a, tau, k, regime, b, hint);
}

DHD double dlfdlq_of(double q) { return -q / (1.0 + exp(-q)); }

// 1/(2l+1)
DHD double inv_odd(int l) { return rcp(2.0 * l + 1.0); }

// ---- slots: the state indices read by the functionals G and the leaf row F1 ----
DHD int n_slots(const Dims& D) { return 14 + 2 * D.nq; }
DHD int slot_index(const Dims& D, int s)
{
    if (s < 8) return 2 + s;
    if (s == 8) return D.idxgp;
    if (s == 9) return D.idxgp + 2;
    if (s == 10) return D.idxr;
    if (s == 11) return D.idxr + 1;
    if (s < 12 + D.nq) return D.iq0 + (s - 12);
    if (s < 12 + 2 * D.nq) return D.iq0 + D.nq + (s - 12 - D.nq);
    return s == 12 + 2 * D.nq ? D.n - 2 : D.n - 1;
}

// ---- G: column j of the three functionals (h', eta', polter) ----
template <class T>
DHD void gcol(const DiscoebCosmo& P, const Dims& D, const Bg<T>& b, double k, int j, T g[3])
{
    g[0] = 0.0; g[1] = 0.0; g[2] = 0.0;
    const double k2 = k * k;
    const T Omegac = b.par.Omegam - b.par.Omegab;
    const T& ia = b.ia;
    const T& ia2 = b.ia2;
    const T& invaH = b.iaHG;
    const double hE = 0.5 / k2;
    const int nq = D.nq;
    // h' = (2 k^2 eta + dgrho) / (a'/a)   (perturbations.py:294-306, :346)
    if (j == 2) g[0] = 2.0 * k2 * invaH;
    else if (j == 3) g[0] = b.par.grhom * Omegac * ia * invaH;
    else if (j == 5) g[0] = b.par.grhom * b.par.Omegab * ia * invaH;
    else if (j == 7) { if (!b.rsa) g[0] = P.grhog * ia2 * invaH; }
    else if (j == D.idxr) { if (!b.rsa) g[0] = P.grhor * P.Neff * ia2 * invaH; }
    else if (j >= D.iq0 && j < D.iq0 + nq) { int q = j - D.iq0; g[0] = P.grhor * P.Nmnu * P.wq[q] * inv_vq(P, b, q) * ia2 * invaH; }
    else if (j == D.n - 2) g[0] = b.par.grhom * b.par.OmegaDE * b.rho_Q * b.a2 * invaH;
    // eta' = dgtheta / (2 k^2)   (perturbations.py:330-335, :349)
    if (j == 4) g[1] = hE * b.par.grhom * Omegac * ia;
    else if (j == 6) g[1] = hE * b.par.grhom * b.par.Omegab * ia;
    else if (j == 8) { if (!b.rsa) g[1] = hE * (4.0 / 3.0) * P.grhog * ia2; }
    else if (j == D.idxr + 1) { if (!b.rsa) g[1] = hE * (4.0 / 3.0) * P.Neff * P.grhor * ia2; }
    else if (j >= D.iq0 + nq && j < D.iq0 + 2 * nq) { int q = j - D.iq0 - nq; g[1] = hE * P.Nmnu * P.grhor * k * P.wq[q] * ia2; }
    else if (j == D.n - 1) g[1] = hE * b.opw * b.rho_Q * b.par.grhom * b.par.OmegaDE * b.a2;
    if (b.rsa) {
        // theta_gamma and theta_r replaced by the RSA fields (approximations.py:28-47)
        const double sk2 = k2 > 1e-30 ? k2 : 1e-30;
        const T cg = hE * (4.0 / 3.0) * P.grhog * ia2;
        const T& fac = b.rsa_fac;
        if (j == 6) g[1] = g[1] + cg * fac * (-b.rsa_tcs - b.aH);
        else if (j == 5) g[1] = g[1] + cg * fac * (b.cs2 * sk2);
        else if (j == 2) g[1] = g[1] + cg * fac * sk2;
        const T eH = cg * (-0.5 - 0.5 * fac * b.rsa_tcs) + hE * (4.0 / 3.0) * P.Neff * P.grhor * ia2 * (-0.5);
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
    if (i < 7) {
        if (i == 2) { u[1] = 1.0; }
        else if (i == 3 || i == 5) { band[4] = -1.0; u[0] = -0.5; }
        else if (i == 4) { band[3] = -b.aH; }
        else if (!b.rsa) {  // i == 6: baryon velocity
            band[2] = k2 * b.cs2;
            band[3] = -b.aH - b.po;
            band[5] = b.po;
        } else {
            const double sk2 = k2 > 1e-30 ? k2 : 1e-30;
            const T pf = b.po * b.rsa_fac;
            band[2] = k2 * b.cs2 + pf * (b.cs2 * sk2);
            band[3] = -b.aH - b.po + pf * (-b.rsa_tcs - b.aH);
            etac = pf * sk2;
            u[0] = b.po * (-0.5 - 0.5 * b.rsa_fac * b.rsa_tcs);
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
            const double ki = k * inv_odd(l);
            band[2] = ki * l; band[3] = -b.opac; band[4] = -ki * (l + 1.0);
        } else {
            band[2] = k; band[3] = -(L + 1.0) * b.itau - b.opac;
        }
        return;
    }
    if (i <= D.idxgp + D.lmaxgp) {  // photon polarisation
        if (b.rsa || b.tca) return;
        const int l = i - D.idxgp, L = D.lmaxgp;
        if (l < L) {
            const double ki = k * inv_odd(l);
            band[2] = ki * l;
            band[3] = -b.opac;
            band[4] = -ki * (l + 1.0);
            if (l == 0) u[2] = 0.5 * b.opac;
            if (l == 2) u[2] = 0.1 * b.opac;
        } else {
            band[2] = k; band[3] = -(L + 1.0) * b.itau - b.opac;
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
                band[3] = -1.5 * (tau > 1e-30 ? b.itau : 1e30);
                u[0] = 2.0 / 15.0;
            } else {
                band[2] = 8.0 / 15.0; band[4] = -0.6 * k; u[0] = 4.0 / 15.0; u[1] = 8.0 / 5.0;
            }
        } else if (!b.ufa) {
            if (l < L) { const double ki = k * inv_odd(l); band[2] = ki * l; band[4] = -ki * (l + 1.0); }
            else { band[2] = k; band[3] = -(L + 1.0) * b.itau; }
        }
        return;
    }
    if (i < D.n - 2) {  // massive neutrinos, l-major blocks of nq bins
        const int r = i - D.iq0, l = r / D.nq, q = r - l * D.nq, L = D.lmaxnu;
        const T kv = k * rcp(inv_vq(P, b, q));
        const double dl = dlfdlq_of(P.q[q]);
        if (l == 0) { band[4] = -kv; u[0] = dl * (1.0 / 6.0); }
        else if (l == 1) { band[2] = kv * (1.0 / 3.0); band[4] = -2.0 * kv * (1.0 / 3.0); }
        else if (l == 2 && L > 2) { band[2] = 2.0 * kv * 0.2; band[4] = -3.0 * kv * 0.2; u[0] = -dl * (1.0 / 15.0); u[1] = -0.4 * dl; }
        else if (l < L) { const double io = inv_odd(l); band[2] = kv * ((double)l * io); band[4] = -kv * ((l + 1.0) * io); }
        else { band[2] = kv; band[3] = -(L + 1.0) * b.itau; }
        return;
    }
    if (b.de_frozen) return;
    const double cs2Q = P.cs2_DE;
    if (i == D.n - 2) {
        band[3] = -3.0 * (cs2Q - b.w_Q) * b.aH;
        band[4] = -b.opw - 9.0 * b.opw * (cs2Q - b.ca2_Q) * b.aH * b.aH * (1.0 / k2);
        u[0] = -0.5 * b.opw;
    } else {
        band[2] = cs2Q * b.iopw * k2;
        band[3] = -(1.0 - 3.0 * cs2Q) * b.aH;
    }
}

// ---- row classes ----
// Hierarchy rows (photon temperature l >= 3, photon polarisation, massless neutrinos l >= 3,
// massive neutrinos) are tridiagonal with coefficients that depend on (species, l) through a
// few selects; evaluating them as one class keeps all lanes of a warp on the same path.
// The remaining "special" rows (a, a h', eta, CDM, baryons, photon l <= 2, massless l <= 2,
// dark energy) go through rowc.
DHD int n_hier_rows(const Dims& D) { return (D.lmaxg - 2) + (D.lmaxgp + 1) + (D.lmaxr - 2) + D.nq * (D.lmaxnu + 1); }
DHD int hier_row(const Dims& D, int h)
{
    const int nT = D.lmaxg - 2;
    if (h < nT) return 10 + h;
    h -= nT;
    const int nP = D.lmaxgp + 1;
    if (h < nP) return D.idxgp + h;
    h -= nP;
    const int nR = D.lmaxr - 2;
    if (h < nR) return D.idxr + 3 + h;
    return D.iq0 + (h - nR);
}
DHD int n_special_rows() { return 15; }
DHD int special_row(const Dims& D, int s)
{
    if (s < 10) return s;
    if (s < 13) return D.idxr + (s - 10);
    return s == 13 ? D.n - 2 : D.n - 1;
}
// momentum bin of a massive-neutrino row (0 for other rows)
// m / nq for 0 <= m < 2^16 and 1 <= nq <= 16.  On the device through a float reciprocal: with
// m = l nq + r, (m + 1/2)/nq lies at least 1/(2 nq) >= 1/32 away from an integer and the two float
// roundings move it by less than 2^-22 (m + 1/2) < 0.016, so the truncation is exact (an integer
// division by a run-time value would cost some twenty instructions per row).
DHD int div_nq(int m, int nq)
{
#if defined(__CUDA_ARCH__)
    return __float2int_rz(((float)m + 0.5f) * __frcp_rn((float)nq));
#else
    return m / nq;
#endif
}
DHD int hier_bin(const Dims& D, int i)
{
    if (i < D.iq0) return 0;
    const int m = i - D.iq0;
    return m - div_nq(m, D.nq) * D.nq;
}

// tridiagonal coefficients of hierarchy row i: f_i = lo*y[i-s] + di*y[i] + up*y[i+s] + u.g;
// vq = velocity of the row's momentum bin and dl = d ln f0 / d ln q of that bin (both ignored for
// massless species)
template <class T>
DHD void hier_coef(const DiscoebCosmo& P, const Dims& D, const Bg<T>& b, double k, int i, const T& vq, double dl, T& lo,
                   T& di, T& up, T u[3], int& stride, bool& trunc)
{
    int l, L, species;
    if (i <= 7 + D.lmaxg) { l = i - 7; L = D.lmaxg; species = 0; }
    else if (i <= D.idxgp + D.lmaxgp) { l = i - D.idxgp; L = D.lmaxgp; species = 1; }
    else if (i <= D.idxr + D.lmaxr) { l = i - D.idxr; L = D.lmaxr; species = 2; }
    else { l = div_nq(i - D.iq0, D.nq); L = D.lmaxnu; species = 3; }
    const bool massive = species == 3;
    const T scale = massive ? T(k) * vq : T(k);
    trunc = (l == L);
    const double io = inv_odd(l);
    lo = trunc ? scale : scale * ((double)l * io);
    up = trunc ? T(0.0) : -scale * ((l + 1.0) * io);
    di = (species <= 1 ? -b.opac : T(0.0)) - (trunc ? T((L + 1.0) * b.itau) : T(0.0));
    u[0] = 0.0; u[1] = 0.0; u[2] = 0.0;
    if (species == 1) u[2] = l == 0 ? 0.5 * b.opac : (l == 2 ? 0.1 * b.opac : T(0.0));
    if (massive) {
        u[0] = l == 0 ? T(dl * (1.0 / 6.0)) : (l == 2 ? T(-dl * (1.0 / 15.0)) : T(0.0));
        u[1] = l == 2 ? T(-0.4 * dl) : T(0.0);
    }
    const bool frozen = (species <= 2 && b.rsa) || (species == 2 && b.ufa) || (species == 1 && b.tca);
    if (frozen) { lo = 0.0; di = 0.0; up = 0.0; u[2] = 0.0; }
    stride = massive ? D.nq : 1;
}

// ---- row 1 (a h'), read by no other equation: f_1 = sum_j F1_j y_j + F1U . g ----
template <class T>
DHD T f1col(const DiscoebCosmo& P, const Dims& D, const Bg<T>& b, double k, int j)
{
    const double k2 = k * k;
    const T Omegac = b.par.Omegam - b.par.Omegab;
    const T& ia = b.ia;
    const T& ia2 = b.ia2;
    const int nq = D.nq;
    T rho = 0.0, pres = 0.0;  // coefficients of y_j in dgrho and dgpres
    if (j == 3) rho = b.par.grhom * Omegac * ia;
    else if (j == 5) rho = b.par.grhom * b.par.Omegab * ia;
    else if (j == 7) { rho = P.grhog * ia2; if (!b.rsa) pres = P.grhog * ia2 * (1.0 / 3.0); }
    else if (j == D.idxr) { rho = P.grhor * P.Neff * ia2; if (!b.rsa) pres = P.grhor * P.Neff * ia2 * (1.0 / 3.0); }
    else if (j >= D.iq0 && j < D.iq0 + nq) {
        const int q = j - D.iq0;
        const T iv = inv_vq(P, b, q);
        rho = P.grhor * P.Nmnu * P.wq[q] * iv * ia2;
        pres = P.grhor * P.Nmnu * ia2 * P.wq[q] * rcp(iv) * (1.0 / 3.0);
    } else if (j == D.n - 2) {
        rho = b.par.grhom * b.par.OmegaDE * b.rho_Q * b.a2;
        pres = P.cs2_DE * b.par.grhom * b.par.OmegaDE * b.rho_Q * b.a2;
    } else if (j == D.n - 1) {
        pres = (P.cs2_DE - b.ca2_Q) * (3.0 * b.aH * b.opw * b.rho_Q * b.par.grhom * b.par.OmegaDE * b.a2 * (1.0 / k2));
    }
    if (b.rsa) {
        const double sk2 = k2 > 1e-30 ? k2 : 1e-30;
        if (j == 2) pres = pres + (P.grhog + P.grhor * P.Neff) * ia2 * (1.0 / 3.0) * (-4.0);
        else if (j == 6) pres = pres + P.grhog * ia2 * (1.0 / 3.0) * (4.0 / sk2) * (b.rsa_fac * (sk2 / 3.0));
    }
    return -b.a * (rho + 3.0 * pres);
}

template <class T>
DHD void f1u(const DiscoebCosmo& P, const Bg<T>& b, double k, T u[3])
{
    u[0] = 0.0; u[1] = 0.0; u[2] = 0.0;
    if (b.rsa) {
        const double k2 = k * k, sk2 = k2 > 1e-30 ? k2 : 1e-30;
        const T itc = b.rsa_fac * (sk2 / 3.0);  // 1 / max(tau_c, 1e-30)
        T presH = P.grhog * b.ia2 * (1.0 / 3.0) * (4.0 * b.aH / sk2 + 2.0 / sk2 * itc) +
                  P.grhor * P.Neff * b.ia2 * (1.0 / 3.0) * (4.0 * b.aH / sk2);
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
// condition holds there (evaluated from (tau, a) as the reference does).  rsa_fields takes the
// state through Y(i) and the table values at a (rho_nu, x_e, dx_e/dln a, c_s^2 a); rsa_projection
// reads them from the tables, with the state's tangent yd (may be null) and the parameter tangent
// tn (may be null).
template <class T, class YF>
DHD bool rsa_fields(const DiscoebCosmo& P, const Par<T>& par, const Dims& D, double tau, double k, const YF& Y,
                    const T& a, const T& loga, const T& rhonu, const T& xe, const T& dxe_dloga, const T& cs2a,
                    T out[4])
{
    const T eta = Y(2), deltab = Y(5), thetab = Y(6);
    const T aH = aprimeoa_from(P, par, a, loga, rhonu);
    const T xeprime = dxe_dloga * aH;
    const T cs2 = cs2a / a;
    const T opac = xe * par.akthom / (a * a);
    const T tau_c = rcp(xmaxc(opac, 1e-30));
    const T tau_c_prime = tau_c * (2.0 * aH - xeprime / xmaxc(xe, 1e-30));
    const T Omegac = par.Omegam - par.Omegab;
    T drhonu = 0.0;
    for (int q = 0; q < D.nq; ++q) {
        const T aq = a * par.amnu * (1.0 / P.q[q]);
        drhonu = drhonu + P.wq[q] * Y(D.iq0 + q) * xsqrt(1.0 + aq * aq);
    }
    const T rho_Q = xexp(-3.0 * (1.0 + par.w0 + par.wa) * loga + 3.0 * (a - 1.0) * par.wa);
    const T dgrho_wo_rel = par.grhom * (Omegac * Y(3) + par.Omegab * deltab) / a + P.grhor * P.Nmnu * drhonu / (a * a) +
                           par.grhom * par.OmegaDE * Y(D.n - 2) * rho_Q * a * a;
    const double k2 = k * k;
    const T hprime = (2.0 * k2 * eta + dgrho_wo_rel) / xmaxc(aH, 1e-30);
    const double sk2 = k2 > 1e-30 ? k2 : 1e-30;
    const T stc = xmaxc(tau_c, 1e-30);
    out[0] = (4.0 / sk2) * (aH * hprime - sk2 * eta) + 4.0 / (sk2 * stc) * (thetab + 0.5 * hprime);
    out[1] = -0.5 * hprime + 3.0 / (sk2 * stc) *
             (-tau_c_prime / stc * (thetab + 0.5 * hprime) + (-aH * thetab + cs2 * sk2 * deltab + sk2 * eta));
    out[2] = (4.0 / sk2) * (aH * hprime - sk2 * eta);
    out[3] = -0.5 * hprime;
    const double tcr = val(tau_c);
    return P.use_rsa && (tcr / (tau > 1e-30 ? tau : 1e-30) > P.rsa_tau_c_over_tau) && (tau * k > P.rsa_tau_over_tau_k);
}

template <class T>
DHD bool rsa_projection(const DiscoebCosmo& P, const DiscoebTangent* tn, const Dims& D, double tau, double k,
                        const double* y, const double* yd, T out[4])
{
    const Par<T> par = make_par<T>(P, tn);
    auto Y = [&](int i) { return seed_t<T>(y[i], yd ? yd[i] : 0.0); };
    const T a = Y(0), loga = xlog(a);
    const int ir = spline_index(P.logrhonu_loga, val(loga));
    const T rhonu = xexp(spline_eval_at(P.logrhonu_loga, ir, loga, tn ? tn->logrhonu_y : nullptr,
                                        tn ? tn->logrhonu_S : nullptr));
    const int ix = spline_index(P.xe_loga, val(loga));
    const T xe = spline_eval_at(P.xe_loga, ix, loga, tn ? tn->xe_y : nullptr, tn ? tn->xe_S : nullptr);
    const T dxe = spline_deriv_at(P.xe_loga, ix, loga, tn ? tn->xe_y : nullptr, tn ? tn->xe_S : nullptr);
    const int ic = spline_index(P.cs2a_loga, val(loga));
    const T cs2a = spline_eval_at(P.cs2a_loga, ic, loga, tn ? tn->cs2a_y : nullptr, tn ? tn->cs2a_S : nullptr);
    return rsa_fields(P, par, D, tau, k, Y, a, loga, rhonu, xe, dxe, cs2a, out);
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
// output_fields takes the state through Y(i) and the table values rho_nu, p_nu at a;
// output_vars reads them from the tables, with the state's tangent yd and parameter tangent tn
// (either may be null).
template <class T, class YF>
DHD void output_fields(const DiscoebCosmo& P, const Par<T>& par, const Dims& D, double k, const YF& Y, const T& a,
                       const T& loga, const T& rhonu, const T& pnu, T* o)
{
    const T Omegac = par.Omegam - par.Omegab;
    const int n = D.n, nq = D.nq, iq0 = D.iq0, iq1 = iq0 + nq;
    const T eta = Y(2), deltac = Y(3), thetac = Y(4), deltab = Y(5), thetab = Y(6);
    const T deltag = Y(7), thetag = Y(8), deltar = Y(D.idxr), thetar = Y(D.idxr + 1);
    T drhonu = 0.0, fnu = 0.0;
    for (int q = 0; q < nq; ++q) {
        const T aq = a * par.amnu * (1.0 / P.q[q]);
        drhonu = drhonu + P.wq[q] * Y(iq0 + q) * xsqrt(1.0 + aq * aq);
        fnu = fnu + P.wq[q] * Y(iq1 + q);
    }
    const T deltanu = drhonu / rhonu, thetanu = k * fnu / (rhonu + pnu);
    const T deltaq = Y(n - 2), thetaq = Y(n - 1);
    const T w_Q = par.w0 + par.wa * (1.0 - a);
    const T rho_Q = xexp(-3.0 * (1.0 + par.w0 + par.wa) * loga + 3.0 * (a - 1.0) * par.wa);
    const T rpt = (1.0 + w_Q) * rho_Q * par.grhom * par.OmegaDE * thetaq * a * a;
    const T a2 = a * a;
    const T grho = par.grhom * par.Omegam / a + (P.grhog + P.grhor * (P.Neff + P.Nmnu * rhonu)) / a2 +
                   par.grhom * par.OmegaDE * rho_Q * a2 + par.grhom * P.Omegak;
    const T aH = xsqrt(grho * (1.0 / 3.0));
    const T dgrho = par.grhom * (Omegac * deltac + par.Omegab * deltab) / a +
                    (P.grhog * deltag + P.grhor * (P.Neff * deltar + P.Nmnu * drhonu)) / a2 +
                    par.grhom * par.OmegaDE * deltaq * rho_Q * a2;
    const T dgtheta = par.grhom * (Omegac * thetac + par.Omegab * thetab) / a +
                      (4.0 / 3.0) * (P.grhog * thetag + P.Neff * P.grhor * thetar) / a2 +
                      P.Nmnu * P.grhor * k * fnu / a2 + rpt;
    const double k2 = k * k;
    const T hprime = (2.0 * k2 * eta + dgrho) / aH;
    const T etaprime = 0.5 * dgtheta / k2;
    const T alpha = (hprime + 6.0 * etaprime) / 2.0 / k2;
    const T mden = par.grhom * par.Omegam / a + P.grhor * P.Nmnu * rhonu / a2;
    const T deltam = (par.grhom * (Omegac * deltac + par.Omegab * deltab) / a + P.grhor * P.Nmnu * drhonu / a2) / mden;
    T thetam = (par.grhom * (Omegac * thetac + par.Omegab * thetab) / a + P.Nmnu * P.grhor * k * fnu / a2) / (3.0 * mden);
    const T deltabc = (par.grhom * (Omegac * deltac + par.Omegab * deltab) / a) / (par.grhom * par.Omegam / a);
    T thetabc = (par.grhom * (Omegac * thetac + par.Omegab * thetab) / a) / (3.0 * (par.grhom * par.Omegam / a) / a2);
    thetam = thetam + alpha * k2;
    thetabc = thetabc + alpha * k2;
    const T iaH = rcp(aH);
    o[0] = eta; o[1] = etaprime; o[2] = hprime; o[3] = alpha;
    o[4] = deltam; o[5] = thetam * iaH; o[6] = deltabc; o[7] = thetabc * iaH;
    o[8] = deltac; o[9] = thetac * iaH; o[10] = deltab; o[11] = thetab * iaH;
    o[12] = deltag; o[13] = thetag * iaH; o[14] = deltar; o[15] = thetar * iaH;
    o[16] = deltanu; o[17] = thetanu * iaH; o[18] = deltaq; o[19] = thetaq * iaH;
}


template <class T>
DHD void output_vars(const DiscoebCosmo& P, const DiscoebTangent* tn, const Dims& D, double k, const double* y,
                     const double* yd, T* o)
{
    const Par<T> par = make_par<T>(P, tn);
    auto Y = [&](int i) { return seed_t<T>(y[i], yd ? yd[i] : 0.0); };
    const T a = Y(0), loga = xlog(a);
    const int inu = spline_index(P.logrhonu_loga, val(loga));
    const T rhonu = xexp(spline_eval_at(P.logrhonu_loga, inu, loga, tn ? tn->logrhonu_y : nullptr,
                                        tn ? tn->logrhonu_S : nullptr));
    const int ip = spline_index(P.logpnu_loga, val(loga));
    const T pnu = xexp(spline_eval_at(P.logpnu_loga, ip, loga, tn ? tn->logpnu_y : nullptr, tn ? tn->logpnu_S : nullptr));
    output_fields(P, par, D, k, Y, a, loga, rhonu, pnu, o);
}

}  // namespace dscb
