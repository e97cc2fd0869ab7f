// Discrete adjoint of the structured Rodas5 solve (the reverse of stepper.cuh).
//
// For one accepted step from y_n (stages K_s, stage states u_s, W = I/(gamma h) - J(y_n)):
//   r_s = f(t_s, u_s) + [s < 5] h d_s f_tau(y_n) + sum_{j<s} (C_sj / h) K_j,   K_s = W^{-1} r_s,
//   y_{n+1} = u_7 + K_7,
// the reverse sweep takes ybar_{n+1} to ybar_n and accumulates the cotangents of the background
// inputs, stage by stage from s = 7 down to 0:
//   rbar_s = W^{-T} Kbar_s                     (transposed chain LU + Woodbury on the transpose)
//   ubar_s += J(u_s)^T rbar_s                  (stage RHS)
//   Jbar   += rbar_s K_s^T                     (W depends on y_n through J(y_n))
//   ybar_n += h d_s f_tau^T rbar_s, Kbar_j += (C_sj / h) rbar_s, then ubar_s flows to y_n and K_j.
// The step sizes are the forward's (the derivative of the discrete solution with the accepted
// step sequence held fixed, the derivative discoeb_jvp computes in forward mode).
//
// Products with transposed Jacobians and the cotangents of the parameters and table values come
// from "functionals" lambda . f(y; b) evaluated in dual numbers, one seed per lane: the background
// b depends on a = y[0], on eight parameters and on five table values at a (the 14 "x" inputs);
// the 15 special rows and the metric functionals h', eta', polter are the straight-line code the
// RHS itself uses (special_part), and the hierarchy rows enter through a few lane-reduced sums
// (their coefficients depend on the background only through the opacity and the neutrino bin
// velocities).  The hierarchy rows' own transposed band product is a gather over neighbouring
// rows.  Table-value cotangents are spread onto the spline knots (y and S arrays) with the
// spline's basis weights.
#pragma once

#include "stepper.cuh"

namespace dscb {

// ---- seeds ----
// The background inputs of a functional: a, the eight parameters the RHS reads, and the four
// knot values of each table's interval at a (y_i, y_i+1, S_i, S_i+1 of the x_e, c_s^2 a, ln rho_nu
// and ln p_nu splines): a knot seed carries the knot's effect on the spline's value and slope
// alike, which second derivatives (d/da of the Jacobian column) need.
constexpr int kNTabSeeds = 16;
constexpr int kNX = 9 + kNTabSeeds;
enum {
    X_A = 0,
    X_GRHOM, X_OMEGAM, X_OMEGAB, X_OMEGADE, X_AMNU, X_W0, X_WA, X_H0,  // DiscoebTangent's scalar order
    X_KNOT0                                                           // 4 table x 4 knot values
};
// table (0 x_e, 1 c_s^2 a, 2 ln rho_nu, 3 ln p_nu) and knot value (0 y_i, 1 y_i+1, 2 S_i, 3 S_i+1)
// of knot seed xs; its row of the cotangent array (DiscoebTangent's table order) and knot offset
DHD int kseed_table(int xs) { return (xs - X_KNOT0) >> 2; }
DHD int kseed_knot(int xs) { return (xs - X_KNOT0) & 3; }
DHD int kseed_row(int xs) { return 2 * kseed_table(xs) + (kseed_knot(xs) >> 1); }
DHD int kseed_offset(int xs) { return kseed_knot(xs) & 1; }

// value with derivative e in the "outer" direction (the one a gradient is taken along): Dual
// carries it directly; HDual carries d/da in its inner level and the outer direction outside
DHD Dual outer_as(const Dual*, double v, double e) { return Dual(v, e); }
DHD HDual outer_as(const HDual*, double v, double e) { return HDual(Dual(v, 0.0), Dual(e, 0.0)); }
template <class T> DHD T oseed(double v, double e) { return outer_as((const T*)nullptr, v, e); }
// the scale factor: (HDual) inner direction d/da, plus the outer seed e
DHD Dual a_as(const Dual*, double a, double e) { return Dual(a, e); }
DHD HDual a_as(const HDual*, double a, double e) { return HDual(Dual(a, 1.0), Dual(e, 0.0)); }
template <class T> DHD T aseed(double a, double e) { return a_as((const T*)nullptr, a, e); }
// the gradient part: Dual d/d(outer); HDual d/d(outer) d/da
DHD double gpart(const Dual& q) { return q.d; }
DHD double gpart(const HDual& q) { return q.d.d; }

DDV void add_global(double* p, double v)
{
#if defined(__CUDA_ARCH__)
    atomicAdd(p, v);
#else
    *p += v;
#endif
}

// interval index of each of the four tables at ln a (the index the forward's evaluation uses)
struct TabIdx {
    int i[4];
};
DHD TabIdx tab_idx(const DiscoebCosmo& P, double loga)
{
    TabIdx t;
    for (int q = 0; q < 4; ++q) t.i[q] = spline_index(table_slot_spline(P, q), loga);
    return t;
}

// the knot value of table t seeded by xs (-1: none)
DHD int kseed_in(int xs, int t) { return (xs >= X_KNOT0 && kseed_table(xs) == t) ? kseed_knot(xs) : -1; }

// Value (or, deriv, derivative in x) of a natural spline in interval i with knot value js
// (0 y_i, 1 y_i+1, 2 S_i, 3 S_i+1; -1: none) seeded: spline_eval_at / spline_deriv_at.
template <class T> DHD T spline_kseed(const DiscoebSpline& s, int i, const T& xn, int js, bool deriv)
{
    const double xi = DLDG(s.x + i), xj = DLDG(s.x + i + 1);
    const double h = xj - xi;
    const T yi = oseed<T>(DLDG(s.y + i), js == 0 ? 1.0 : 0.0), yj = oseed<T>(DLDG(s.y + i + 1), js == 1 ? 1.0 : 0.0);
    const T Si = oseed<T>(DLDG(s.S + i), js == 2 ? 1.0 : 0.0), Sj = oseed<T>(DLDG(s.S + i + 1), js == 3 ? 1.0 : 0.0);
    if (!deriv) {
        const T t = (xn - xi) * (1.0 / h);
        const T A = 1.0 - t, B = t;
        return A * yi + B * yj + ((A * A * A - A) * Si + (B * B * B - B) * Sj) * (h * h / 6.0);
    }
    const T d = xn - xi;
    const T b = (yj - yi) * (1.0 / h) - h * (Sj + 2.0 * Si) * (1.0 / 6.0);
    const T c = Si * 0.5;
    const T dd = (Sj - Si) * (1.0 / (6.0 * h));
    return b + 2.0 * c * d + 3.0 * dd * d * d;
}

// Background at (a, tau) with input xs seeded (xs < 0: none; the HDual form always carries d/da
// in its inner level).  Same arithmetic as bg_eval (make_par, bg_tables, bg_finish).
template <class T>
DHD void bg_seeded(const DiscoebCosmo& P, double a, double tau, double k, int regime, const TabIdx& ti, int xs, Bg<T>& b)
{
    auto sd = [&](double v, int id) { return oseed<T>(v, xs == id ? 1.0 : 0.0); };
    Par<T> par;
    par.grhom = sd(P.grhom, X_GRHOM);
    par.Omegam = sd(P.Omegam, X_OMEGAM);
    par.Omegab = sd(P.Omegab, X_OMEGAB);
    par.OmegaDE = sd(P.OmegaDE, X_OMEGADE);
    par.amnu = sd(P.amnu, X_AMNU);
    par.w0 = sd(P.w0, X_W0);
    par.wa = sd(P.wa, X_WA);
    const double c = 2.3038921003709498e-9 * (1.0 - P.YHe);
    const T H0 = sd(P.H0, X_H0);
    par.akthom = c * par.Omegab * H0 * H0;
    const T A = aseed<T>(a, xs == X_A ? 1.0 : 0.0);
    const T loga = xlog(A);
    BgTables<T> tb;
    tb.xe = spline_kseed(P.xe_loga, ti.i[0], loga, kseed_in(xs, 0), false);
    tb.xep = spline_kseed(P.xe_loga, ti.i[0], loga, kseed_in(xs, 0), true);
    tb.cs2a = spline_kseed(P.cs2a_loga, ti.i[1], loga, kseed_in(xs, 1), false);
    tb.rhonu = xexp(spline_kseed(P.logrhonu_loga, ti.i[2], loga, kseed_in(xs, 2), false));
    tb.pnu = xexp(spline_kseed(P.logpnu_loga, ti.i[3], loga, kseed_in(xs, 3), false));
    tb.rho_Q = xexp(-3.0 * (1.0 + par.w0 + par.wa) * loga + 3.0 * (A - 1.0) * par.wa);
    bg_finish(P, par, A, tb, tau, k, regime, b);
}

// ---- the state entries the special rows and the metric functionals read ----
DHD int n_read(const Dims& D) { return 17 + 2 * D.nq; }
DHD int read_index(const Dims& D, int r)
{
    if (r < 9) return 2 + r;  // eta .. photon l = 3
    switch (r) {
        case 9: return D.idxgp;
        case 10: return D.idxgp + 2;
        case 11: return D.idxr;
        case 12: return D.idxr + 1;
        case 13: return D.idxr + 2;
        case 14: return D.idxr + 3;
        case 15: return D.n - 2;
        case 16: return D.n - 1;
        default: return D.iq0 + (r - 17);  // massive bins, l = 0 then l = 1
    }
}

// ---- hierarchy rows in a functional lambda . f ----
// A hierarchy row's coefficients depend on the background only through the opacity (photon
// rows: the diagonal and the polarisation source u_2) and, for massive neutrinos, the bin velocity
// (off-diagonals).  Sum over the hierarchy rows of lambda_i f_i(y):
//   opac * aop + sum_q v_q * bq[q] + sum_r g_r (gc[r] + opac * gop[r]) + terms without b.
struct HierStat {
    double aop, gc[3], gop[3], bq[DISCOEB_MAX_NQ];
};

DHD void hier_stat_zero(HierStat& h)
{
    h.aop = 0.0;
    for (int r = 0; r < 3; ++r) h.gc[r] = h.gop[r] = 0.0;
    for (int q = 0; q < DISCOEB_MAX_NQ; ++q) h.bq[q] = 0.0;
}

// Coefficients of hierarchy row i and their derivatives with respect to the opacity (.v.d) and
// the bin velocity (.d.v), from hier_coef in hyper-dual numbers.
DHD void hier_coef_parts(const DiscoebCosmo& P, const Dims& D, const Bg<double>& b, double k, int i, double vq,
                         double dlq, HDual& lo, HDual& di, HDual& up, HDual u[3], int& st, bool& trunc)
{
    Bg<HDual> bh;
    bh.opac = HDual(Dual(b.opac, 1.0), Dual(0.0, 0.0));
    bh.itau = b.itau;
    bh.rsa = b.rsa;
    bh.ufa = b.ufa;
    bh.tca = b.tca;
    hier_coef(P, D, bh, k, i, HDual(Dual(vq, 0.0), Dual(1.0, 0.0)), dlq, lo, di, up, u, st, trunc);
}

// This lane's share of the hierarchy statistics of lambda . f(y) at background b (a sum over the
// lanes gives the whole).
template <class TM>
DDV void hier_stat_lane(const TM& tm, const DiscoebCosmo& P, const Dims& D, const Bg<double>& b, double k,
                        const double* lam, const double* y, HierStat& h)
{
    const int nh = n_hier_rows(D);
    for (int hh = tm.lane; hh < nh; hh += tm.nl) {
        const int i = hier_row(D, hh);
        const double li = lam[i];
        if (li == 0.0) continue;
        const int q = hier_bin(D, i);
        const double vq = rcp(inv_vq(P, b, q));
        HDual lo, di, up, u[3];
        int st;
        bool trunc;
        hier_coef_parts(P, D, b, k, i, vq, dlfdlq_of(P.q[q]), lo, di, up, u, st, trunc);
        const double ylo = y[i - st], yi = y[i], yup = trunc ? 0.0 : y[i + st];
        h.aop += li * (lo.v.d * ylo + di.v.d * yi + up.v.d * yup);
        h.bq[q] += li * (lo.d.v * ylo + di.d.v * yi + up.d.v * yup);
        for (int r = 0; r < 3; ++r) {
            h.gop[r] += li * u[r].v.d;
            h.gc[r] += li * (u[r].v.v - b.opac * u[r].v.d);
        }
    }
}

template <class TM> DDV void hier_stat_reduce(const TM& tm, const Dims& D, HierStat& h)
{
    h.aop = tm.sum(h.aop);
    for (int r = 0; r < 3; ++r) {
        h.gc[r] = tm.sum(h.gc[r]);
        h.gop[r] = tm.sum(h.gop[r]);
    }
    for (int q = 0; q < D.nq; ++q) h.bq[q] = tm.sum(h.bq[q]);
}

// The hierarchy rows' coefficients at one background, computed once and reused by the statistics
// and the transposed band product of every cotangent taken at that background: per row i (state
// index) the values c[3i + m] of (lo, di, up), their opacity derivatives ca and bin-velocity
// derivatives cq, the coupling coefficients u[r] (uv) with their opacity derivatives (ua), and
// tr[i] = 1 for a truncation row (its band has no upper neighbour; its upper entries are zero).
struct HierCoef {
    double *c, *ca, *cq, *uv, *ua, *tr;
};
DHD int hier_coef_doubles(const Dims& D) { return 16 * D.n; }
DHD HierCoef carve_hier_coef(double* base, const Dims& D)
{
    const int n = D.n;
    return HierCoef{base, base + 3 * n, base + 6 * n, base + 9 * n, base + 12 * n, base + 15 * n};
}

template <class TM>
DDV void hier_coef_fill(const TM& tm, const DiscoebCosmo& P, const Dims& D, const Bg<double>& b, double k,
                        const HierCoef& HC)
{
    const int nh = n_hier_rows(D);
    // the bin velocities and d ln f0 / d ln q on lanes, broadcast (every lane runs the same number
    // of iterations: the shuffles need all lanes)
    double vlane = 1.0, dll = 0.0;
    if (tm.full() && tm.lane < D.nq) {
        vlane = rcp(inv_vq(P, b, tm.lane));
        dll = dlfdlq_of(P.q[tm.lane]);
    }
    for (int h0 = 0; h0 < nh; h0 += tm.nl) {
        const int hh = h0 + tm.lane;
        const bool act = hh < nh;
        const int i = hier_row(D, act ? hh : 0);
        const int q = hier_bin(D, i);
        const double vq = tm.full() ? tm.bcast(vlane, q) : rcp(inv_vq(P, b, q));
        const double dlq = tm.full() ? tm.bcast(dll, q) : dlfdlq_of(P.q[q]);
        if (!act) continue;
        HDual lo, di, up, u[3];
        int st;
        bool trunc;
        hier_coef_parts(P, D, b, k, i, vq, dlq, lo, di, up, u, st, trunc);
        HC.c[3 * i] = lo.v.v; HC.c[3 * i + 1] = di.v.v; HC.c[3 * i + 2] = trunc ? 0.0 : up.v.v;
        HC.ca[3 * i] = lo.v.d; HC.ca[3 * i + 1] = di.v.d; HC.ca[3 * i + 2] = trunc ? 0.0 : up.v.d;
        HC.cq[3 * i] = lo.d.v; HC.cq[3 * i + 1] = di.d.v; HC.cq[3 * i + 2] = trunc ? 0.0 : up.d.v;
        for (int r = 0; r < 3; ++r) {
            HC.uv[3 * i + r] = u[r].v.v;
            HC.ua[3 * i + r] = u[r].v.d;
        }
        HC.tr[i] = trunc ? 1.0 : 0.0;
    }
    tm.sync();
}

// hier_stat_lane + hier_stat_reduce from cached coefficients (opac: the background's opacity).
// The massive-neutrino rows run with a fixed bin per lane, so that each lane keeps its bin's
// velocity statistic in a register; part: tm.nl doubles of scratch for the per-bin sums.
template <class TM>
DDV void hier_stat_cached(const TM& tm, const Dims& D, const HierCoef& HC, double opac, const double* lam,
                          const double* y, HierStat& h, double* part)
{
    hier_stat_zero(h);
    double aop = 0.0, gc[3] = {0.0, 0.0, 0.0}, gop[3] = {0.0, 0.0, 0.0};
    auto row = [&](int i, double& bacc) {
        const double li = lam[i];
        if (li == 0.0) return;
        const int st = row_stride(D, i);
        const double ylo = y[i - st], yi = y[i];
        const double yup = HC.tr[i] != 0.0 ? 0.0 : y[i + st];
        aop += li * (HC.ca[3 * i] * ylo + HC.ca[3 * i + 1] * yi + HC.ca[3 * i + 2] * yup);
        bacc += li * (HC.cq[3 * i] * ylo + HC.cq[3 * i + 1] * yi + HC.cq[3 * i + 2] * yup);
        for (int r = 0; r < 3; ++r) {
            gop[r] += li * HC.ua[3 * i + r];
            gc[r] += li * (HC.uv[3 * i + r] - opac * HC.ua[3 * i + r]);
        }
    };
    const int nq = D.nq;
    const int nmass = nq * (D.lmaxnu + 1);
    const int nlight = n_hier_rows(D) - nmass;  // photon and massless-neutrino rows come first
    double unused = 0.0;
    for (int hh = tm.lane; hh < nlight; hh += tm.nl) row(hier_row(D, hh), unused);
    if (nq > 0 && TM::nl >= nq) {
        const int per = TM::nl / nq;  // lanes per bin
        const int q = tm.lane % nq;
        double bacc = 0.0;
        if (tm.lane < per * nq)
            for (int l = tm.lane / nq; l <= D.lmaxnu; l += per) row(D.iq0 + l * nq + q, bacc);
        part[tm.lane] = bacc;
        tm.sync();
        for (int qq = 0; qq < nq; ++qq) {
            double v = 0.0;
            for (int p = 0; p < per; ++p) v += part[p * nq + qq];
            h.bq[qq] = v;
        }
        tm.sync();
    } else {
        for (int m = tm.lane; m < nmass; m += tm.nl) {
            double bacc = 0.0;
            row(D.iq0 + m, bacc);
            h.bq[m % nq] += bacc;
        }
        for (int qq = 0; qq < nq; ++qq) h.bq[qq] = tm.sum(h.bq[qq]);
    }
    h.aop = tm.sum(aop);
    for (int r = 0; r < 3; ++r) {
        h.gc[r] = tm.sum(gc[r]);
        h.gop[r] = tm.sum(gop[r]);
    }
}

// lambda . f(y) at background b, up to terms that do not depend on b or y, with the hierarchy rows
// through h (hier_stat of the same lambda and y); lam0 = false leaves out row 0 (a' = a'/a a).
// Y(j) gives state entry j as a T.
// LF(ss) gives lambda at special row ss.
template <class T, class YF, class LF>
DHD T functional_l(const DiscoebCosmo& P, const Dims& D, const Bg<T>& b, double k, double tau, const LF& L,
                   bool lam0, const YF& Y, const HierStat& h)
{
    const HostTeam ht;
    T sp[15], g0, g1, g2;
    special_part<HostTeam, T, T>(ht, P, D, b, k, tau, Y, T(1.0), T(1.0), sp, g0, g1, g2);
    T Q = 0.0;
    for (int ss = lam0 ? 0 : 1; ss < 15; ++ss) Q = Q + L(ss) * sp[ss];
    Q = Q + b.opac * h.aop;
    for (int q = 0; q < D.nq; ++q) Q = Q + rcp(inv_vq(P, b, q)) * h.bq[q];
    Q = Q + g0 * (h.gc[0] + b.opac * h.gop[0]) + g1 * (h.gc[1] + b.opac * h.gop[1]) +
        g2 * (h.gc[2] + b.opac * h.gop[2]);
    return Q;
}
template <class T, class YF>
DHD T functional(const DiscoebCosmo& P, const Dims& D, const Bg<T>& b, double k, double tau, const double* lam,
                 bool lam0, const YF& Y, const HierStat& h)
{
    return functional_l<T>(P, D, b, k, tau, [&](int ss) { return lam[special_row(D, ss)]; }, lam0, Y, h);
}

// ---- table knot cotangents ----
// One accumulator per knot seed: the interval it collects for and the cotangent so far; flushed
// to the caller's tbar (atomically: all modes of a cosmology share it) when the interval changes
// and at the end of the mode.
struct TabAcc {
    int cur;
    double w;
};

DDV void tab_flush(TabAcc& acc, int xs, double* tbar, int stride)
{
    if (acc.cur >= 0 && tbar && acc.w != 0.0)
        add_global(tbar + (size_t)kseed_row(xs) * stride + acc.cur + kseed_offset(xs), acc.w);
    acc.cur = -1;
    acc.w = 0.0;
}

// cotangent g of knot seed xs in interval i of its table
DDV void tab_add(TabAcc& acc, int xs, int i, double g, double* tbar, int stride)
{
    if (acc.cur != i) {
        tab_flush(acc, xs, tbar, stride);
        acc.cur = i;
    }
    acc.w += g;
}

// ---- deferred functionals ----
// The parameter and table-knot cotangents of a reverse step do not feed back into the state
// cotangents, so their functionals can be evaluated after the step (or by another warp): a
// record holds what a functional lambda . f(Y; b) needs besides the seed, compactly:
//   [0] a, [1] tau, [2] regime, [3] unused, [4, 19) lambda on the 15 special rows,
//   [19, 19 + n_read) Y on the entries the special rows read, then the hierarchy statistics.
// A step leaves 17 records: its 8 stage functionals (Dual, at the stage states), the 8 terms
// of W's dependence on y_n through J(y_n) (Dual, at y_n, row 0 left out) and the column-0 term
// (hyper-dual, at y_n).
constexpr int kRecPerStep = 17;
constexpr int kDeferredSeeds = kNX - 1;  // every x input but a
// scalars a step leaves for achain_step (c_s, K_s[0] per stage, W_00, h, the output layer's a term)
enum { AS_C = 0, AS_K0 = 8, AS_W00 = 16, AS_H = 17, AS_LAM0 = 18, kAScalars = 20 };
constexpr int kAScratch = 32;  // achain_step's scratch (26 used)
DHD int hs_doubles() { return (int)(sizeof(HierStat) / sizeof(double)); }
DHD int drec_doubles(const Dims& D) { return 19 + n_read(D) + hs_doubles(); }
// inverse of read_index (-1: not read)
DHD int read_slot(const Dims& D, int j)
{
    if (j >= 2 && j <= 10) return j - 2;
    if (j == D.idxgp) return 9;
    if (j == D.idxgp + 2) return 10;
    if (j >= D.idxr && j <= D.idxr + 3) return 11 + (j - D.idxr);
    if (j == D.n - 2) return 15;
    if (j == D.n - 1) return 16;
    if (j >= D.iq0 && j < D.iq0 + 2 * D.nq) return 17 + (j - D.iq0);
    return -1;
}

// write record rec (team-parallel): lambda from lam (full length), Y from y (full length), hs
template <class TM>
DDV void drec_write(const TM& tm, const Dims& D, double* rec, double a, double tau, int regime, const double* lam,
                    const double* y, const HierStat& hs)
{
    const int nr = n_read(D);
    if (tm.leader()) {
        rec[0] = a;
        rec[1] = tau;
        rec[2] = (double)regime;
        rec[3] = 0.0;
        const double* h = reinterpret_cast<const double*>(&hs);
        for (int q = 0; q < hs_doubles(); ++q) rec[19 + nr + q] = h[q];
    }
    for (int ss = tm.lane; ss < 15; ss += tm.nl) rec[4 + ss] = lam[special_row(D, ss)];
    for (int r = tm.lane; r < nr; r += tm.nl) rec[19 + r] = y[read_index(D, r)];
}

// gpart of the functional of record rec (kind 0: stage, 1: W term, 2: column-0 term) seeded in xs
template <class T>
DHD double drec_eval(const DiscoebCosmo& P, const Dims& D, double k, const double* rec, int kind, int xs)
{
    const double a = rec[0], tau = rec[1];
    const int regime = (int)rec[2];
    const TabIdx ti = tab_idx(P, log(a));
    Bg<T> b;
    bg_seeded(P, a, tau, k, regime, ti, xs, b);
    HierStat hs;
    double* h = reinterpret_cast<double*>(&hs);
    const int nr = n_read(D);
    for (int q = 0; q < hs_doubles(); ++q) h[q] = rec[19 + nr + q];
    auto Y = [&](int j) {
        const int r = read_slot(D, j);
        return T(r >= 0 ? rec[19 + r] : nan(""));  // an entry outside the read list would poison the result
    };
    auto L = [&](int ss) { return rec[4 + ss]; };
    return gpart(functional_l<T>(P, D, b, k, tau, L, kind != 1, Y, hs));
}

// Accumulators of the deferred seeds: parameter cotangents pb[16] (index = seed) and one table
// accumulator per knot seed.  The lane that evaluates seed xs is the only one touching its entry.
struct DefAcc {
    double* pb;
    TabAcc* tab;
};

// ---- per-warp adjoint workspace ----
// With own_step_buffers the workspace also holds the step's U columns, Zt and deferred records
// (the single-team sweep); the warp-split kernel keeps those in its shared step slots.
struct AdjMem {
    double *Uk, *Zt, *Kb, *us, *ub, *yb, *rho, *lam, *pb, *sc, *rec, *as, *scr, *g, *hc;
    TabAcc* tab;
};
DHD int adj_mem_doubles(const Dims& D, bool own_step_buffers = true)
{
    return 13 * D.n + 16 + 32 + 2 * kNTabSeeds + hier_coef_doubles(D) +
           (own_step_buffers
                ? 6 * D.n + kRecPerStep * drec_doubles(D) + kAScalars + kAScratch + kRecPerStep * kDeferredSeeds
                : 0);
}
DHD AdjMem carve_adj(double* base, const Dims& D, bool own_step_buffers = true)
{
    const int n = D.n;
    AdjMem A;
    A.Kb = base;          // 8n  stage cotangents Kbar_s, replaced by rbar_s = W^{-T} Kbar_s in turn
    A.us = A.Kb + 8 * n;  // n   current stage state
    A.ub = A.us + n;      // n   ubar of the current stage
    A.yb = A.ub + n;      // n   ybar_n being accumulated
    A.rho = A.yb + n;     // n   sum_s K_s[0] rbar_s
    A.lam = A.rho + n;    // n   the running cotangent ybar (input and output of a step)
    A.pb = A.lam + n;     // 16  parameter cotangents (index = seed)
    A.sc = A.pb + 16;     // 32  scalars
    A.tab = reinterpret_cast<TabAcc*>(A.sc + 32);  // kNTabSeeds accumulators (2 doubles each)
    A.hc = A.sc + 32 + 2 * kNTabSeeds;  // cached hierarchy coefficients (HierCoef)
    double* rest = A.hc + hier_coef_doubles(D);
    if (own_step_buffers) {
        A.Uk = rest;          // 3n  U columns at the step start (the factorisation overwrites M.Z)
        A.Zt = A.Uk + 3 * n;  // 3n  A^{-T} G^T
        A.rec = A.Zt + 3 * n; // the step's deferred records
        A.as = A.rec + kRecPerStep * drec_doubles(D);  // the step's scalars for achain_step
        A.scr = A.as + kAScalars;                       // achain_step's scratch
        A.g = A.scr + kAScratch;                        // deferred_records' staging
    } else {
        A.Uk = A.Zt = A.rec = A.as = A.scr = A.g = nullptr;
    }
    return A;
}
static_assert(sizeof(TabAcc) <= 2 * sizeof(double), "TabAcc must fit two doubles");

// ---- transposed solves ----
// A^T z = r for one chain of the factorisation (unit-lower L, upper U with reciprocal pivots).
// The last two solved values ride in registers (the sweeps never reload what they just stored).
DDV void solve_chain_T(const double* A, const Chain& ch, double* z)
{
    const int st = ch.stride, len = ch.len;
    // U^T w = r: forward
    double p1 = 0.0, p2 = 0.0;
#pragma unroll 4
    for (int p = 0; p < len; ++p) {
        const int i = ch.start + p * st;
        double v = z[i];
        if (p >= 1) v -= A[7 * (i - st) + 4] * p1;
        if (ch.ku >= 2 && p >= 2) v -= A[7 * (i - 2 * st) + 5] * p2;
        v *= A[7 * i + 3];
        z[i] = v;
        p2 = p1;
        p1 = v;
    }
    // L^T z = w: backward
    double n1 = 0.0, n2 = 0.0;
#pragma unroll 4
    for (int p = len - 1; p >= 0; --p) {
        const int i = ch.start + p * st;
        double v = z[i];
        if (p + 1 < len) v -= A[7 * (i + st) + 2] * n1;
        if (ch.kl >= 2 && p + 2 < len) v -= A[7 * (i + 2 * st) + 1] * n2;
        z[i] = v;
        n2 = n1;
        n1 = v;
    }
}

// A^T z = r for rows >= 2 (in place): the chains, then row 2 (A's row 6 holds -etac in column 2)
template <class TM> DDV void solve_AT(const TM& tm, const Dims& D, const ModeMem& M, double gh, double* z)
{
    tm.sync();
    const int nc = n_chains(D);
    for (int c = tm.lane; c < nc; c += tm.nl) solve_chain_T(M.A, chain_of(D, c), z);
    tm.sync();
    if (tm.leader()) z[2] = gh * (z[2] + M.sc[SC_ETAC] * z[6]);
    tm.sync();
}

// Zt = A^{-T} G^T (three columns), after factor_W
template <class TM> DDV void make_Zt(const TM& tm, const Dims& D, const ModeMem& M, double h, double* Zt)
{
    const int n = D.n, ns = n_slots(D);
    const double gh = kR5.gamma * h;
    for (int r = 0; r < 3; ++r) {
        double* z = Zt + r * n;
        for (int i = tm.lane; i < n; i += tm.nl) z[i] = 0.0;
        tm.sync();
        for (int sl = tm.lane; sl < ns; sl += tm.nl) z[slot_index(D, sl)] = M.Gs[r * kMaxSlots + sl];
        solve_AT(tm, D, M, gh, z);
    }
}

// v = W^{-T} g in place (W = I/(gamma h) - J(y_n) as factored by factor_W; Uk its U columns)
// c_out (may be null): receives c = sum_{i >= 1} J_i0 v_i (with v_1's row-1 form), so that
// v_0 = (g_0 + c) / W_00: the only place the a-component enters.
template <class TM>
DDV void solve_WT(const TM& tm, const Dims& D, const ModeMem& M, const double* Uk, const double* Zt, double h, double* v,
                  double* c_out = nullptr)
{
    const int n = D.n, ns = n_slots(D);
    const double gh = kR5.gamma * h;
    const double g0 = v[0];
    const double v1 = gh * v[1];
    const double* F1U = M.sc + SC_F1U;
    tm.sync();
    // g_r + v_1 (F1 + G^T F1U) on the slots (row 1 of W reads the slots)
    for (int sl = tm.lane; sl < ns; sl += tm.nl) {
        const int j = slot_index(D, sl);
        v[j] += v1 * (M.F1s[sl] + M.Gs[sl] * F1U[0] + M.Gs[kMaxSlots + sl] * F1U[1] +
                      M.Gs[2 * kMaxSlots + sl] * F1U[2]);
    }
    if (tm.leader()) v[1] = 0.0;  // rows 0 and 1 are not part of the chains
    solve_AT(tm, D, M, gh, v);
    // Woodbury on the transpose: v_r = z + Zt C^{-T} (U^T z)
    double a0 = 0.0, a1 = 0.0, a2 = 0.0;
    for (int i = tm.lane; i < n; i += tm.nl) {
        if (i < 2) continue;
        a0 += Uk[i] * v[i];
        a1 += Uk[n + i] * v[i];
        a2 += Uk[2 * n + i] * v[i];
    }
    const double u0 = tm.sum(a0), u1 = tm.sum(a1), u2 = tm.sum(a2);
    const double* Ci = M.sc + SC_CINV;
    const double c0 = Ci[0] * u0 + Ci[3] * u1 + Ci[6] * u2;
    const double c1 = Ci[1] * u0 + Ci[4] * u1 + Ci[7] * u2;
    const double c2 = Ci[2] * u0 + Ci[5] * u1 + Ci[8] * u2;
    tm.sync();
    double acc = 0.0;
    for (int i = tm.lane; i < n; i += tm.nl) {
        if (i < 2) continue;
        const double vi = v[i] + Zt[i] * c0 + Zt[n + i] * c1 + Zt[2 * n + i] * c2;
        v[i] = vi;
        acc += M.col0[i] * vi;
    }
    const double c0v = tm.sum(acc);
    tm.sync();
    if (tm.leader()) {
        v[1] = v1;
        v[0] = (g0 + c0v + M.col0[1] * v1) / M.sc[SC_W00];
        if (c_out) *c_out = c0v + M.col0[1] * v1;
    }
    tm.sync();
}

// ---- transposed products ----
// a coefficient's value (double), or its derivative in a (Dual seeded in a)
DHD double apart(double x) { return x; }
DHD double apart(const Dual& x) { return x.d; }

// out[j] += sum over the hierarchy rows i of C_ij lam_i (the rows' band entries), for every
// column j >= 2, at background b (T = double) or, T = Dual in a, the a-derivative of those
// entries (C'_ij).
template <class TM, class T>
DDV void hier_gather(const TM& tm, const DiscoebCosmo& P, const Dims& D, const Bg<T>& b, double k, const double* lam,
                     double* out)
{
    const int n = D.n;
    auto is_hier = [&](int i) {
        return (i >= 10 && i <= 7 + D.lmaxg) || (i >= D.idxgp && i <= D.idxgp + D.lmaxgp) ||
               (i >= D.idxr + 3 && i <= D.idxr + D.lmaxr) || (i >= D.iq0 && i < n - 2);
    };
    for (int j = tm.lane; j < n; j += tm.nl) {
        if (j < 2) continue;
        const int stj = row_stride(D, j);
        double acc = 0.0;
        for (int m = -1; m <= 1; ++m) {
            const int i = j - m * stj;
            if (i < 2 || i >= n || !is_hier(i) || row_stride(D, i) != stj) continue;
            const double li = lam[i];
            if (li == 0.0) continue;
            const int q = hier_bin(D, i);
            const T vq = rcp(inv_vq(P, b, q));
            T lo, di, up, u[3];
            int st;
            bool trunc;
            hier_coef(P, D, b, k, i, vq, dlfdlq_of(P.q[q]), lo, di, up, u, st, trunc);
            if (m == 1 && trunc) continue;                   // a truncation row has no upper entry
            const T c = m == -1 ? lo : (m == 0 ? di : up);  // row i's entry in column j = i + m st
            acc += apart(c) * li;
        }
        out[j] += acc;
    }
}

// hier_gather at a background whose coefficients are cached (hier_coef_fill)
template <class TM>
DDV void hier_gather_cached(const TM& tm, const Dims& D, const HierCoef& HC, const double* lam, double* out)
{
    const int n = D.n;
    auto is_hier = [&](int i) {
        return (i >= 10 && i <= 7 + D.lmaxg) || (i >= D.idxgp && i <= D.idxgp + D.lmaxgp) ||
               (i >= D.idxr + 3 && i <= D.idxr + D.lmaxr) || (i >= D.iq0 && i < n - 2);
    };
    for (int j = tm.lane; j < n; j += tm.nl) {
        if (j < 2) continue;
        const int stj = row_stride(D, j);
        double acc = 0.0;
        for (int m = -1; m <= 1; ++m) {
            const int i = j - m * stj;
            if (i < 2 || i >= n || !is_hier(i) || row_stride(D, i) != stj) continue;
            const double li = lam[i];
            if (li == 0.0) continue;
            if (m == 1 && HC.tr[i] != 0.0) continue;  // a truncation row has no upper entry
            acc += HC.c[3 * i + 1 + m] * li;        // row i's entry in column j = i + m st
        }
        out[j] += acc;
    }
}

// ---- output layer ----
// The cotangent of the pre-projection state at an output time, and of the background inputs,
// from the cotangent ob[20] of the output fields (RSA projection then convert_to_output_variables):
// one lane per seed over the x inputs and the state entries the output layer reads.
DHD int n_out_read(const Dims& D) { return 11 + 2 * D.nq; }
DHD int out_read_index(const Dims& D, int r)
{
    if (r < 7) return 2 + r;  // eta, delta_c, theta_c, delta_b, theta_b, delta_g, theta_g
    if (r == 7) return D.idxr;
    if (r == 8) return D.idxr + 1;
    if (r == 9) return D.n - 2;
    if (r == 10) return D.n - 1;
    return D.iq0 + (r - 11);
}

// output fields o[20] at state y with input xs seeded, or state entry yj seeded (xs < 0)
template <class T>
DHD void output_seeded(const DiscoebCosmo& P, const Dims& D, double tau, double k, const double* y, int xs, int yj,
                       T o[20])
{
    auto sd = [&](double v, int id) { return oseed<T>(v, xs == id ? 1.0 : 0.0); };
    Par<T> par;
    par.grhom = sd(P.grhom, X_GRHOM);
    par.Omegam = sd(P.Omegam, X_OMEGAM);
    par.Omegab = sd(P.Omegab, X_OMEGAB);
    par.OmegaDE = sd(P.OmegaDE, X_OMEGADE);
    par.amnu = sd(P.amnu, X_AMNU);
    par.w0 = sd(P.w0, X_W0);
    par.wa = sd(P.wa, X_WA);
    const double c = 2.3038921003709498e-9 * (1.0 - P.YHe);
    const T H0 = sd(P.H0, X_H0);
    par.akthom = c * par.Omegab * H0 * H0;
    auto Y = [&](int i) { return i == 0 ? sd(y[0], X_A) : oseed<T>(y[i], i == yj ? 1.0 : 0.0); };
    const T a = Y(0), loga = xlog(a);
    const TabIdx ti = tab_idx(P, val(loga));
    const T rhonu = xexp(spline_kseed(P.logrhonu_loga, ti.i[2], loga, kseed_in(xs, 2), false));
    const T pnu = xexp(spline_kseed(P.logpnu_loga, ti.i[3], loga, kseed_in(xs, 3), false));
    const T xe = spline_kseed(P.xe_loga, ti.i[0], loga, kseed_in(xs, 0), false);
    const T dxe = spline_kseed(P.xe_loga, ti.i[0], loga, kseed_in(xs, 0), true);
    const T cs2a = spline_kseed(P.cs2a_loga, ti.i[1], loga, kseed_in(xs, 1), false);
    T fld[4];
    const bool rsa = rsa_fields(P, par, D, tau, k, Y, a, loga, rhonu, xe, dxe, cs2a, fld);
    auto Yp = [&](int i) {
        if (rsa) {
            const int s = rsa_slot(D, i);
            if (s >= 0) return fld[s];
            if (s == -1) return T(0.0);
        }
        return Y(i);
    };
    output_fields(P, par, D, k, Yp, a, loga, rhonu, pnu, o);
}

// Adds the output layer's cotangents: lam[.] += dL/dy (pre-projection state), A.pb / tables for the
// x inputs.  ob[20] is the cotangent of the output fields at (tau, y).
template <class TM>
DDV void output_adjoint(const TM& tm, const DiscoebCosmo& P, const Dims& D, double tau, double k, const double* y,
                        const double* ob, const AdjMem& A, double* lam, double* tbar, int tstride)
{
    const int nseed = kNX + n_out_read(D);
    const double loga = log(y[0]);
    const TabIdx ti = tab_idx(P, loga);
    for (int base = 0; base < nseed; base += tm.nl) {
        const int sid = base + tm.lane;
        if (sid < nseed) {
            const int xs = sid < kNX ? sid : -1;
            const int yj = sid < kNX ? -1 : out_read_index(D, sid - kNX);
            Dual o[20];
            output_seeded<Dual>(P, D, tau, k, y, xs, yj, o);
            double g = 0.0;
            for (int q = 0; q < 20; ++q) g += ob[q] * o[q].d;
            if (xs < 0) lam[yj] += g;
            else if (xs == X_A) lam[0] += g;
            else if (xs < X_KNOT0) A.pb[xs] += g;
            else tab_add(A.tab[xs - X_KNOT0], xs, ti.i[kseed_table(xs)], g, tbar, tstride);
        }
        tm.sync();
    }
}

// ---- the reverse of one step ----
// The a-component of the cotangents forms a chain of its own: rows >= 1 of f are linear in
// y[1:] with coefficients that depend on a, and a' depends on a only, so no cotangent of
// y[1:] depends on one of a (W^{-T}'s row 0 is solved last, v_0 = (g_0 + c)/W_00, and every
// y-derivative of lambda_0 f_0 vanishes).  The reverse step therefore runs in two parts:
// adjoint_step carries the cotangents of y[1:] (the critical chain) and leaves per step the 17
// functional records and a few scalars; achain_step then carries the a-component through the
// same stages as a scalar recurrence, with the a-derivatives of the recorded functionals, and
// completes the records' lambda_0 for the parameter and table seeds (deferred_records).

// scalars a step leaves for achain_step

template <class T, class S, class F> DHD Bg<T> bg_convert(const Bg<S>& s, const F& cv)
{
    Bg<T> b;
    b.par = Par<T>{cv(s.par.grhom), cv(s.par.Omegam), cv(s.par.Omegab), cv(s.par.OmegaDE), cv(s.par.amnu),
                   cv(s.par.w0), cv(s.par.wa), cv(s.par.akthom)};
    b.a = cv(s.a); b.ia = cv(s.ia); b.a2 = cv(s.a2); b.ia2 = cv(s.ia2); b.aH = cv(s.aH); b.iaHG = cv(s.iaHG);
    b.opac = cv(s.opac); b.po = cv(s.po); b.tauc = cv(s.tauc); b.taucprime = cv(s.taucprime); b.cs2 = cv(s.cs2);
    b.pb43 = cv(s.pb43); b.rho_Q = cv(s.rho_Q); b.w_Q = cv(s.w_Q); b.opw = cv(s.opw); b.iopw = cv(s.iopw);
    b.ca2_Q = cv(s.ca2_Q); b.pnu = cv(s.pnu); b.rsa_fac = cv(s.rsa_fac); b.rsa_tcs = cv(s.rsa_tcs);
    b.aprimeprimeoa = cv(s.aprimeprimeoa);
    b.itau = s.itau;
    b.rsa = s.rsa; b.ufa = s.ufa; b.tca = s.tca; b.de_frozen = s.de_frozen;
    return b;
}

// The backgrounds at the eight stage states of a recomputed step (M), in the order of the reverse
// stage loop's use, stored as Bg<double> images at out [8 x bg_image_doubles()]; the stage scale
// factors are formed exactly as adjoint_step forms u_s[0].
DHD int bg_image_doubles() { return (int)((sizeof(Bg<double>) + sizeof(double) - 1) / sizeof(double)); }
template <class TM>
DDV void stage_backgrounds(const TM& tm, const DiscoebCosmo& P, const Dims& D, double k, double t, double h,
                           int regime, const ModeMem& M, double* out, int& hint)
{
    const int n = D.n;
    for (int s = 7; s >= 0; --s) {
        double v = M.y[0];
        const int sl = s <= 5 ? s : 5;
        for (int j = 0; j < sl; ++j) v += kR5.a[sl][j] * M.K[j * n];
        if (s >= 6) v += M.K[5 * n];
        if (s == 7) v += M.K[6 * n];
        const double ts = (s <= 5) ? t + kR5.c[s] * h : t + h;
        Bg<double> bs;
        bg_eval_team(tm, P, v, ts, k, regime, bs, hint);
        if (tm.leader()) *reinterpret_cast<Bg<double>*>(out + (size_t)s * bg_image_doubles()) = bs;
    }
    tm.sync();
}

// On entry: M holds the step's forward recomputation (rodas5_step from y_n = M.y, with factor_W's
// U columns in Uk) and Zt = A^{-T} G^T; A.lam[1:] = ybar_{n+1}[1:].  On return A.lam[1:] =
// ybar_n[1:] (A.lam[0] = 0: the a-component is achain_step's).  lam0_out: the a-cotangent added at
// this step's end by the output layer (the caller's), passed on in the step scalars sc.
template <class TM>
DDV void adjoint_step(const TM& tm, const DiscoebCosmo& P, const Dims& D, double k, double t, double h, int regime,
                      const ModeMem& M, const AdjMem& A, const double* Uk, const double* Zt, double* recs, double* sc,
                      double lam0_out, int& hint, const double* stage_bg = nullptr)
{
    const int n = D.n;
    const double ih = 1.0 / h;
    const int rd = drec_doubles(D);
    // stage cotangents: Kbar_7 = ybar_{n+1}, the others start at zero; ubar_7 = ybar_{n+1}
    for (int i = tm.lane; i < n; i += tm.nl) {
        const double l = i == 0 ? 0.0 : A.lam[i];
        for (int s = 0; s < 7; ++s) A.Kb[s * n + i] = 0.0;
        A.Kb[7 * n + i] = l;
        A.ub[i] = l;
        A.yb[i] = 0.0;
        A.rho[i] = 0.0;
    }
    if (tm.leader()) {
        sc[AS_W00] = M.sc[SC_W00];
        sc[AS_H] = h;
        sc[AS_LAM0] = lam0_out;
        for (int s = 0; s < 8; ++s) sc[AS_K0 + s] = M.K[s * n];
    }
    tm.sync();
    Bg<double> bflags;
    bflags.rsa = (regime & 1) != 0;
    bflags.ufa = !bflags.rsa && (regime & 2) != 0;
    bflags.tca = !bflags.rsa && (regime & 4) != 0;
    const int nseed = n_read(D);  // the state entries the special rows and the metric functionals read
    for (int s = 7; s >= 0; --s) {
        const double* Ks = M.K + s * n;
        // rbar_s[1:] = (W^{-T} Kbar_s)[1:], in place (Kbar_s is complete: only later stages add to it)
        double* rb = A.Kb + s * n;
        solve_WT(tm, D, M, Uk, Zt, h, rb, sc + AS_C + s);
        if (tm.leader()) rb[0] = 0.0;  // the a-component: achain_step
        tm.sync();
        // stage state u_s
        for (int i = tm.lane; i < n; i += tm.nl) {
            double v = M.y[i];
            const int sl = s <= 5 ? s : 5;
            for (int j = 0; j < sl; ++j) v += kR5.a[sl][j] * M.K[j * n + i];
            if (s >= 6) v += M.K[5 * n + i];
            if (s == 7) v += M.K[6 * n + i];
            A.us[i] = v;
            A.rho[i] += Ks[0] * rb[i];
        }
        tm.sync();
        // ubar_s[1:] += (J(u_s)^T rbar_s)[1:]: hierarchy rows by the gather, the special rows and
        // the metric functionals by the functional seeded in the state entries it reads, at the
        // stage's background (no input of the background is seeded: a plain background in dual
        // form); its a- and x-seeds are the record's
        const double ts = (s <= 5) ? t + kR5.c[s] * h : t + h;
        Bg<double> bs;
        if (stage_bg) bs = *reinterpret_cast<const Bg<double>*>(stage_bg + (size_t)s * bg_image_doubles());
        else bg_eval_team(tm, P, A.us[0], ts, k, regime, bs, hint);
        const HierCoef HC = carve_hier_coef(A.hc, D);
        hier_coef_fill(tm, P, D, bs, k, HC);
        HierStat hs;
        hier_stat_cached(tm, D, HC, bs.opac, rb, A.us, hs, A.sc);
        hier_gather_cached(tm, D, HC, rb, A.ub);
        drec_write(tm, D, recs + (size_t)s * rd, A.us[0], ts, regime, rb, A.us, hs);
        tm.sync();
        {
            const Bg<Dual> bd = bg_convert<Dual>(bs, [](double v) { return Dual(v, 0.0); });
            for (int base = 0; base < nseed; base += tm.nl) {
                const int sid = base + tm.lane;
                if (sid < nseed) {
                    const int yj = read_index(D, sid);
                    auto Y = [&](int j) { return Dual(A.us[j], j == yj ? 1.0 : 0.0); };
                    A.ub[yj] += gpart(functional<Dual>(P, D, bd, k, ts, rb, true, Y, hs));
                }
                tm.sync();
            }
        }
        // the explicit tau dependence (s < 5) and the stage couplings C_sj / h
        for (int i = tm.lane; i < n; i += tm.nl) {
            const double r = rb[i];
            if (s < 5) A.yb[i] += h * kR5.d[s] * dtau_row(D, bflags, t, i, rb);
            for (int j = 0; j < s; ++j) A.Kb[j * n + i] += kR5.C[s][j] * ih * r;
            // ubar_s flows to its sources
            const double u = A.ub[i];
            if (s <= 5) {
                A.yb[i] += u;
                for (int j = 0; j < s; ++j) A.Kb[j * n + i] += kR5.a[s][j] * u;
                A.ub[i] = 0.0;
            } else {
                A.Kb[(s - 1) * n + i] += u;  // u_s = u_{s-1} + K_{s-1}
                // A.ub keeps u: it is ubar_{s-1}'s start
            }
        }
        tm.sync();
    }
    // W depends on y_n through J(y_n), i.e. through a = y_n[0] alone: the term sum_s rbar_s^T J(y_n)
    // K_s contributes to a's cotangent and the inputs' only (records 8..15)
    {
        Bg<double> b0;
        bg_eval_team(tm, P, M.y[0], t, k, regime, b0, hint);
        const HierCoef HC = carve_hier_coef(A.hc, D);
        hier_coef_fill(tm, P, D, b0, k, HC);
        for (int s = 0; s < 8; ++s) {
            HierStat hs;
            hier_stat_cached(tm, D, HC, b0.opac, A.Kb + s * n, M.K + s * n, hs, A.sc);
            drec_write(tm, D, recs + (size_t)(8 + s) * rd, M.y[0], t, regime, A.Kb + s * n, M.K + s * n, hs);
        }
        tm.sync();
        // column 0: rho . (d f / d a)(y_n) with rho = sum_s K_s[0] rbar_s; its gradient in y_n[1:] is
        // C'(a)^T rho (hierarchy rows by the gather in Dual a, the rest by the functional in
        // hyper-dual numbers seeded in the state entries); a- and x-gradients: record 16
        HierStat hs;
        hier_stat_cached(tm, D, HC, b0.opac, A.rho, M.y, hs, A.sc);
        Bg<Dual> bda;
        {
            int hh = hint;
            bg_eval_team(tm, P, Dual(M.y[0], 1.0), t, k, regime, bda, hh);
            hier_gather(tm, P, D, bda, k, A.rho, A.yb);
        }
        drec_write(tm, D, recs + (size_t)16 * rd, M.y[0], t, regime, A.rho, M.y, hs);
        tm.sync();
        const Bg<HDual> bh = bg_convert<HDual>(bda, [](const Dual& v) { return HDual(v, Dual(0.0, 0.0)); });
        for (int base = 0; base < nseed; base += tm.nl) {
            const int sid = base + tm.lane;
            if (sid < nseed) {
                const int yj = read_index(D, sid);
                auto Y = [&](int j) { return HDual(Dual(M.y[j], 0.0), Dual(j == yj ? 1.0 : 0.0, 0.0)); };
                A.yb[yj] += gpart(functional<HDual>(P, D, bh, k, t, A.rho, true, Y, hs));
            }
            tm.sync();
        }
    }
    for (int i = tm.lane; i < n; i += tm.nl) A.lam[i] = i == 0 ? 0.0 : A.yb[i];
    tm.sync();
}

// d f_0 / d a (T = Dual) or d^2 f_0 / d a^2 (T = HDual) at (a, tau): f_0 = a' = a (a'/a)
template <class T> DHD double f0_a_derivative(const DiscoebCosmo& P, double a, double tau, double k, int regime)
{
    const TabIdx ti = tab_idx(P, log(a));
    Bg<T> b;
    bg_seeded(P, a, tau, k, regime, ti, X_A, b);
    return gpart(b.aH * b.a);
}

// The a-component of one reverse step (after adjoint_step left recs and sc): lam0 = ybar_{n+1}[0]
// on entry (before this step's output-layer term, which sc carries), ybar_n[0] on return; the
// records' lambda_0 (stage records: rbar_s[0]; record 16: rho_0) are filled in.  The recurrence
// is adjoint_step's on the a-component: rbar_s[0] = (Kbar_s[0] + c_s) / W_00, ubar_s[0] gains
// rbar_s[0] d f_0/d a + (the a-derivative of the rest of the stage functional), W's a-dependence
// and the column-0 term add their a-derivatives.
template <class TM>
DDV void achain_step(const TM& tm, const DiscoebCosmo& P, const Dims& D, double k, double* recs, const double* sc,
                     double& lam0, double* scratch)
{
    const int rd = drec_doubles(D);
    // scratch: [0, 8) d f_0/d a at the stages, [8, 16) the stage functionals' a-derivatives without
    // row 0, [16, 24) the W terms' a-derivatives, 24: the column-0 term's without row 0, 25: d^2 f_0 / da^2
    for (int q = tm.lane; q < 26; q += tm.nl) {
        double v;
        if (q < 8) {
            const double* rec = recs + (size_t)q * rd;
            v = f0_a_derivative<Dual>(P, rec[0], rec[1], k, (int)rec[2]);
        } else if (q < 16) {
            v = drec_eval<Dual>(P, D, k, recs + (size_t)(q - 8) * rd, 1, X_A);  // kind 1: row 0 left out
        } else if (q < 24) {
            v = drec_eval<Dual>(P, D, k, recs + (size_t)(q - 8) * rd, 1, X_A);
        } else if (q == 24) {
            v = drec_eval<HDual>(P, D, k, recs + (size_t)16 * rd, 1, X_A);
        } else {
            const double* rec = recs + (size_t)16 * rd;
            v = f0_a_derivative<HDual>(P, rec[0], rec[1], k, (int)rec[2]);
        }
        scratch[q] = v;
    }
    tm.sync();
    double rb0[8], rho0 = 0.0;
    double l = lam0 + sc[AS_LAM0];
    {
        const double ih = 1.0 / sc[AS_H];
        double Kb0[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        Kb0[7] = l;
        double ub0 = l, yb0 = 0.0;
        for (int s = 7; s >= 0; --s) {
            const double r = (Kb0[s] + sc[AS_C + s]) / sc[AS_W00];
            rb0[s] = r;
            rho0 += sc[AS_K0 + s] * r;
            ub0 += r * scratch[s] + scratch[8 + s];
            for (int j = 0; j < s; ++j) Kb0[j] += kR5.C[s][j] * ih * r;
            if (s <= 5) {
                yb0 += ub0;
                for (int j = 0; j < s; ++j) Kb0[j] += kR5.a[s][j] * ub0;
                ub0 = 0.0;
            } else {
                Kb0[s - 1] += ub0;
            }
        }
        for (int s = 0; s < 8; ++s) yb0 += scratch[16 + s];
        yb0 += rho0 * scratch[25] + scratch[24];
        l = yb0;
    }
    tm.sync();
    if (tm.leader()) {
        for (int s = 0; s < 8; ++s) recs[(size_t)s * rd + 4] = rb0[s];  // lambda on special row 0 (= row 0)
        recs[(size_t)16 * rd + 4] = rho0;
    }
    lam0 = l;
    tm.sync();
}

// The parameter and table-knot seeds of records [r0, r1) of one step (their lambda_0 filled in):
// the (record, seed) pairs spread over the lanes, the results staged in g [(r1 - r0) x
// kDeferredSeeds], then each seed's lane adds its column into acc in record order.
template <class TM>
DDV void deferred_records(const TM& tm, const DiscoebCosmo& P, const Dims& D, double k, const double* recs, int r0,
                          int r1, double* g, const DefAcc& acc, double* tbar, int tstride)
{
    const int rd = drec_doubles(D);
    const int npairs = (r1 - r0) * kDeferredSeeds;
    for (int pq = tm.lane; pq < npairs; pq += tm.nl) {
        const int r = r0 + pq / kDeferredSeeds, xs = 1 + pq % kDeferredSeeds;
        const double* rec = recs + (size_t)r * rd;
        const int kind = r < 8 ? 0 : (r < 16 ? 1 : 2);
        g[pq] = kind == 2 ? drec_eval<HDual>(P, D, k, rec, kind, xs) : drec_eval<Dual>(P, D, k, rec, kind, xs);
    }
    tm.sync();
    for (int sd = tm.lane; sd < kDeferredSeeds; sd += tm.nl) {
        const int xs = 1 + sd;
        for (int r = r0; r < r1; ++r) {
            const double v = g[(r - r0) * kDeferredSeeds + sd];
            if (xs < X_KNOT0) {
                acc.pb[xs] += v;
            } else {
                const TabIdx ti = tab_idx(P, log(recs[(size_t)r * rd]));
                tab_add(acc.tab[xs - X_KNOT0], xs, ti.i[kseed_table(xs)], v, tbar, tstride);
            }
        }
    }
    tm.sync();
}

// ---- forward step records and the reverse sweep of one mode ----
// A mode's record: the end time of every accepted step (tlog[cap]) and the start state of every
// every-th accepted step (ckpt[(cap + every - 1) / every][n]).  The start time of step m is
// tlog[m - 1] (t0 for m = 0), its size tlog[m] minus that, its regime regime_at(its start), so the
// record replays the accepted step sequence exactly.
DHD long long record_doubles(int n, int cap, int every) { return cap + (long long)((cap + every - 1) / every) * n; }

template <class TM> struct Recorder {
    const TM* tm;
    const ModeMem* M;
    double* tlog;
    double* ckpt;
    int cap, every, n, count;
    DDV bool operator()(double, double, double tnext, int)
    {
        if (count >= cap) return false;
        if (count % every == 0) {
            double* c = ckpt + (size_t)(count / every) * n;
            for (int i = tm->lane; i < n; i += tm->nl) c[i] = M->y[i];
        }
        if (tm->leader()) tlog[count] = tnext;
        ++count;
        return true;
    }
};

// Reverse sweep of one mode from its record (nacc accepted steps): the cotangents ob[nout][20] of
// the output fields become y0bar [n] (the initial state's), toutbar [nout] (the output times',
// through y' = f, the convention of discoeb_jvp), the parameters' (A.pb[X_GRHOM..X_H0]) and the
// tables' (added to tbar [8][tstride] in DiscoebTangent's array order).  Each segment of `every`
// steps is recomputed from its checkpoint into seg [every][n], then reversed step by step, each
// step's stages recomputed from its start state.
template <class TM>
DDV void bwd_mode(const TM& tm, const DiscoebCosmo& P, const Dims& D, double k, double t0, const double* sw, int nout,
                  const double* tout, const double* tlog, const double* ckpt, int every, int nacc, double* seg,
                  const double* ob, const ModeMem& M, const AdjMem& A, double* y0bar, double* toutbar, double* tbar,
                  int tstride)
{
    const int n = D.n;
    int hint = P.xe_loga.n_knots / 2;
    double lam0 = 0.0;  // the a-component of the running cotangent (achain_step's)
    for (int i = tm.lane; i < n; i += tm.nl) A.lam[i] = 0.0;
    for (int q = tm.lane; q < 16; q += tm.nl) A.pb[q] = 0.0;
    for (int q = tm.lane; q < kNTabSeeds; q += tm.nl) {
        A.tab[q].cur = -1;
        A.tab[q].w = 0.0;
    }
    tm.sync();
    int jout = nout - 1;
    for (int sg = (nacc - 1) / every; sg >= 0 && nacc > 0; --sg) {
        const int n0 = sg * every, n1 = nacc < n0 + every ? nacc : n0 + every;
        const double* ck = ckpt + (size_t)sg * n;
        // the segment's states n0 + 1 .. n1 - 1
        for (int i = tm.lane; i < n; i += tm.nl) M.y[i] = ck[i];
        tm.sync();
        double t = n0 == 0 ? t0 : tlog[n0 - 1];
        for (int m = n0; m < n1 - 1; ++m) {
            const double tn = tlog[m];
            rodas5_step(tm, P, D, k, t, tn - t, regime_at(P, t, sw), M, hint);
            for (int i = tm.lane; i < n; i += tm.nl) {
                const double y1 = M.u[i] + M.K[7 * n + i];
                M.y[i] = y1;
                seg[(size_t)(m + 1 - n0) * n + i] = y1;
            }
            tm.sync();
            t = tn;
        }
        for (int m = n1 - 1; m >= n0; --m) {
            const double* ym = (m == n0) ? ck : seg + (size_t)(m - n0) * n;
            for (int i = tm.lane; i < n; i += tm.nl) M.y[i] = ym[i];
            tm.sync();
            const double tm0 = m == 0 ? t0 : tlog[m - 1], h = tlog[m] - tm0;
            const int regime = regime_at(P, tm0, sw);
            rodas5_step(tm, P, D, k, tm0, h, regime, M, hint, (const DiscoebTangent*)nullptr, (const TanMem*)nullptr,
                        A.Uk);
            make_Zt(tm, D, M, h, A.Zt);
            // outputs emitted at the end of this step
            double lam0_out = 0.0;
            while (jout >= 0 && tout[jout] > tm0) {
                for (int i = tm.lane; i < n; i += tm.nl) {
                    A.us[i] = M.u[i] + M.K[7 * n + i];
                    A.ub[i] = 0.0;
                }
                tm.sync();
                output_adjoint(tm, P, D, tout[jout], k, A.us, ob + (size_t)jout * 20, A, A.ub, tbar, tstride);
                Bg<double> bo;
                bg_eval_team(tm, P, A.us[0], tout[jout], k, regime, bo, hint);
                rhs_team(tm, P, D, bo, k, tout[jout], A.us, A.yb, (double*)nullptr);
                tm.sync();
                double acc = 0.0;
                for (int i = tm.lane; i < n; i += tm.nl) {
                    acc += A.ub[i] * A.yb[i];
                    if (i > 0) A.lam[i] += A.ub[i];
                }
                const double tb = tm.sum(acc);
                if (tm.leader() && toutbar) toutbar[jout] = tb;
                lam0_out += A.ub[0];
                tm.sync();
                --jout;
            }
            adjoint_step(tm, P, D, k, tm0, h, regime, M, A, A.Uk, A.Zt, A.rec, A.as, lam0_out, hint);
            achain_step(tm, P, D, k, A.rec, A.as, lam0, A.scr);
            deferred_records(tm, P, D, k, A.rec, 0, kRecPerStep, A.g, DefAcc{A.pb, A.tab}, tbar, tstride);
        }
    }
    if (toutbar && tm.leader())
        for (; jout >= 0; --jout) toutbar[jout] = 0.0;
    for (int i = tm.lane; i < n; i += tm.nl) y0bar[i] = i == 0 ? lam0 : A.lam[i];
    for (int xs = X_KNOT0 + tm.lane; xs < X_KNOT0 + kNTabSeeds; xs += tm.nl) tab_flush(A.tab[xs - X_KNOT0], xs, tbar, tstride);
    tm.sync();
}


}  // namespace dscb
