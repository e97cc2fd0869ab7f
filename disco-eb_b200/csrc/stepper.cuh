// Rodas5 step with structured linear algebra, and the adaptive solve of one k-mode.
//
// The method is the 8-stage Rosenbrock scheme of Di Marzo (1993), as used by the
// reference's Rodas5Transformed (src/discoeb/ode_integrators_stiff.py:680-892); step
// control is diffrax's PIDController rule (perturbations.py:913-914) restated from its
// documentation.  Differences from the reference, all of them documented: steps end
// exactly on every output time and approximation switch time (no linear interpolation
// between accepted steps), and the approximation regime is held fixed within a step.
//
// W = I/(gamma h) - J is never formed densely.  With the model in coefficient form
// (model.cuh), J = [[j00, 0], [c0, S + U G]] plus the leaf row 1:
//   * x_0 from the 1x1 row of the scale factor,
//   * A = I/(gamma h) - S is a set of independent banded chains, factored without pivoting
//     (all chain pivots are >= 1/(gamma h) > 0 for these free-streaming / Thomson blocks),
//     one chain per lane,
//   * the rank-3 coupling U G (metric h', eta', polarisation sum) by the Woodbury identity,
//   * x_1 (a h', read by no equation) last.
// Work per step: O(n) instead of the (2/3) n^3 of a dense LU.
#pragma once

#include "model.cuh"
#include "team.cuh"

namespace dscb {

struct Rodas5Tab {
    double gamma;
    double a[6][5];
    double C[8][7];
    double c[6];
    double d[5];
};

#if defined(__CUDACC__)
__constant__ __device__
#endif
static const Rodas5Tab kR5 = {
    0.19,
    {{0, 0, 0, 0, 0},
     {2.0, 0, 0, 0, 0},
     {3.040894194418781, 1.041747909077569, 0, 0, 0},
     {2.576417536461461, 1.622083060776640, -0.9089668560264532, 0, 0},
     {2.760842080225597, 1.446624659844071, -0.3036980084553738, 0.2877498600325443, 0},
     {-14.09640773051259, 6.925207756232704, -41.47510893210728, 2.343771018586405, 24.13215229196062}},
    {{0, 0, 0, 0, 0, 0, 0},
     {-10.31323885133993, 0, 0, 0, 0, 0, 0},
     {-21.04823117650003, -7.234992135176716, 0, 0, 0, 0, 0},
     {32.22751541853323, -4.943732386540191, 19.44922031041879, 0, 0, 0, 0},
     {-20.69865579590063, -8.816374604402768, 1.260436877740897, -0.7495647613787146, 0, 0, 0},
     {-46.22004352711257, -17.49534862857472, -289.6389582892057, 93.60855400400906, 318.3822534212147, 0, 0},
     {34.20013733472935, -14.15535402717690, 57.82335640988400, 25.83362985412365, 1.408950972071624,
      -6.551835421242162, 0},
     {42.57076742291101, -13.80770672017997, 93.98938432427124, 18.77919633714503, -31.58359187223370,
      -6.685968952921985, -5.810979938412932}},
    {0.0, 0.38, 0.3878509998321533, 0.4839718937873840, 0.4570477008819580, 1.0},
    {0.19, -0.1823079225333714636, -0.319231832186874912, 0.3449828624725343, -0.377417564392089818}};

// ---- chain table ----
struct Chain {
    int start, len, stride, kl, ku;
};

DHD int n_chains(const Dims& D) { return 5 + D.nq; }

DHD Chain chain_of(const Dims& D, int c)
{
    Chain ch;
    ch.stride = 1;
    ch.kl = 1;
    ch.ku = 1;
    if (c == 0) { ch.start = 5; ch.len = D.lmaxg + 3; ch.kl = 2; ch.ku = 2; }
    else if (c == 1) { ch.start = D.idxgp; ch.len = D.lmaxgp + 1; }
    else if (c == 2) { ch.start = D.idxr; ch.len = D.lmaxr + 1; }
    else if (c < 3 + D.nq) { ch.start = D.iq0 + (c - 3); ch.len = D.lmaxnu + 1; ch.stride = D.nq; }
    else if (c == 3 + D.nq) { ch.start = 3; ch.len = 2; }
    else { ch.start = D.n - 2; ch.len = 2; }
    return ch;
}

// number of doubles of per-mode workspace
constexpr int kMaxSlots = 48;  // >= 14 + 2 * DISCOEB_MAX_NQ
DHD int mode_mem_doubles(const Dims& D) { return 23 * D.n + 4 * kMaxSlots + 32; }

struct ModeMem {
    double *y, *u, *f, *dT, *col0, *K, *A, *Z, *Gs, *F1s, *sc;
    // mixed-precision form only (teams with TM::mixed): the chain factors in FP32 (7 n floats;
    // A then keeps W's band unfactored, in FP64, for the residuals) and n doubles of scratch
    float* Af = nullptr;
    double* rs = nullptr;
};
// extra doubles per mode of the mixed-precision form, after mode_mem_doubles
DHD int mixed_mem_doubles(const Dims& D) { return (7 * D.n + 1) / 2 + D.n; }
DHD void carve_mixed(double* base, const Dims& D, ModeMem& M)
{
    M.Af = reinterpret_cast<float*>(base);
    M.rs = base + (7 * D.n + 1) / 2;
}

DHD ModeMem carve(double* base, const Dims& D)
{
    const int n = D.n;
    ModeMem m;
    m.y = base;
    m.u = m.y + n;
    m.f = m.u + n;
    m.dT = m.f + n;
    m.col0 = m.dT + n;
    m.K = m.col0 + n;          // 8n stage vectors
    m.A = m.K + 8 * n;         // 7n banded chain factors
    m.Z = m.A + 7 * n;         // 3n  A^{-1} U
    m.Gs = m.Z + 3 * n;        // 3 x kMaxSlots functional rows on the slot list
    m.F1s = m.Gs + 3 * kMaxSlots;
    m.sc = m.F1s + kMaxSlots;  // 32 scalars
    return m;
}
// the same fields with the first 13 n (y .. K) at g and the rest (A .. sc) at f
DHD ModeMem carve_split(double* g, double* f, const Dims& D)
{
    const int n = D.n;
    ModeMem m = carve(g, D);
    m.A = f;
    m.Z = m.A + 7 * n;
    m.Gs = m.Z + 3 * n;
    m.F1s = m.Gs + 3 * kMaxSlots;
    m.sc = m.F1s + kMaxSlots;
    return m;
}
// scalar slots
enum { SC_W00 = 0, SC_ETAC = 1, SC_CINV = 2, SC_F1Z = 11, SC_F1U = 14 };

// tangent workspace: y', the stage state tangent u', two n-vector scratches, d/de of the
// Jacobian column d f/d a, and the 8 stage tangents K'
struct TanMem {
    double *yd, *ud, *fd, *jk, *c0d, *Kd;
};
DHD int tan_mem_doubles(const Dims& D) { return 13 * D.n; }
DHD TanMem carve_tan(double* base, const Dims& D)
{
    const int n = D.n;
    TanMem t;
    t.yd = base;
    t.ud = t.yd + n;
    t.fd = t.ud + n;
    t.jk = t.fd + n;
    t.c0d = t.jk + n;
    t.Kd = t.c0d + n;
    return t;
}

DHD double dual_with(double x, double) { return x; }
DHD Dual dual_with(const Dual& x, double d) { return Dual(x.v, d); }

// state entry with its first-direction part yd and second-direction part yk (null = 0)
DHD double mk_state(const double*, double y, double, double) { return y; }
DHD Dual mk_state(const Dual*, double y, double yd, double) { return Dual(y, yd); }
DHD HDual mk_state(const HDual*, double y, double yd, double yk) { return HDual(Dual(y, yd), Dual(yk, 0.0)); }
template <class T> DHD T state_at(const double* y, const double* yd, const double* yk, int j)
{
    return mk_state((const T*)nullptr, y[j], yd ? yd[j] : 0.0, yk ? yk[j] : 0.0);
}
// component c of a value: 0 value, 1 first direction, 2 second direction, 3 mixed
DHD double comp(double x, int c) { return c == 0 ? x : 0.0; }
DHD double comp(const Dual& x, int c) { return c == 0 ? x.v : (c == 1 ? x.d : 0.0); }
DHD double comp(const HDual& x, int c) { return c == 0 ? x.v.v : (c == 1 ? x.v.d : (c == 2 ? x.d.v : x.d.d)); }

// ---- the 15 special rows and the metric functionals ----
// Rows a, a h', eta, CDM, baryons, photon l <= 2, massless l <= 2 and dark energy (sp, in the
// order of special_row) and the three functionals g = (h', eta', polter) through which the
// hierarchy rows couple, in straight-line code (every lane of a team computes them; no
// divergence, no reductions).  Y(j) gives state entry j (type S); ivl / vl are 1/v and v of
// momentum bin tm.lane, read through tm.bcast when tm.full().  Same equations as
// model_synchronous (perturbations.py:88-525).
template <class TM, class T, class S, class YF>
DHD void special_part(const TM& tm, const DiscoebCosmo& P, const Dims& D, const Bg<T>& b, double k, double tau,
                      YF Y, const T ivl, const T vl, T sp[15], T& g0, T& g1, T& g2)
{
    const int n = D.n, nq = D.nq, iq0 = D.iq0, idxr = D.idxr;
    const double k2 = k * k;
    const T Omegac = b.par.Omegam - b.par.Omegab;
    T drho = 0.0, dp = 0.0, fnu = 0.0;
#pragma unroll
    for (int q = 0; q < DISCOEB_MAX_NQ; ++q) {
        if (q < nq) {
            const T iv = tm.full() ? tm.bcast(ivl, q) : inv_vq(P, b, q);
            const T v = tm.full() ? tm.bcast(vl, q) : rcp(iv);
            const double w = P.wq[q];
            drho = drho + (w * Y(iq0 + q)) * iv;
            dp = dp + (w * Y(iq0 + q)) * v;
            fnu = fnu + w * Y(iq0 + nq + q);
        }
    }
    dp = dp * (1.0 / 3.0);
    const S eta = Y(2), deltac = Y(3), thetac = Y(4), deltab = Y(5), thetab = Y(6);
    const S deltag = Y(7), thetag = Y(8), y9 = Y(9);
    const S deltar = Y(idxr), thetar = Y(idxr + 1), yr2 = Y(idxr + 2);
    const S deltaq = Y(n - 2), thetaq = Y(n - 1);
    const T rQa2 = b.rho_Q * b.a2;
    const T dgm = b.par.grhom * (Omegac * deltac + b.par.Omegab * deltab) * b.ia;
    const T dgnu = P.grhor * P.Nmnu * drho * b.ia2;
    const T dgq = b.par.grhom * b.par.OmegaDE * deltaq * rQa2;
    const T dgrho = dgm + (P.grhog * deltag + P.grhor * P.Neff * deltar) * b.ia2 + dgnu + dgq;
    const T dgrho_wo_rel = dgm + dgnu + dgq;
    T H, thg, thr, dge, dre;
    if (b.rsa) {
        const double sk2 = k2 > 1e-30 ? k2 : 1e-30;
        H = (2.0 * k2 * eta + dgrho_wo_rel) * b.iaHG;
        dre = (4.0 / sk2) * (b.aH * H - sk2 * eta);
        dge = dre + (4.0 / 3.0) * b.rsa_fac * (thetab + 0.5 * H);
        thg = -0.5 * H + b.rsa_fac * (-b.rsa_tcs * (thetab + 0.5 * H) + (-b.aH * thetab + b.cs2 * sk2 * deltab + sk2 * eta));
        thr = -0.5 * H;
    } else {
        H = (2.0 * k2 * eta + dgrho) * b.iaHG;
        dge = deltag;
        dre = deltar;
        thg = thetag;
        thr = thetar;
    }
    const T rptq = b.opw * b.par.grhom * b.par.OmegaDE * thetaq * rQa2;
    const T dgtheta = b.par.grhom * (Omegac * thetac + b.par.Omegab * thetab) * b.ia +
                      (4.0 / 3.0) * (P.grhog * thg + P.Neff * P.grhor * thr) * b.ia2 + P.Nmnu * P.grhor * k * fnu * b.ia2 +
                      rptq;
    const T E = (0.5 / k2) * dgtheta;
    const double cs2Q = P.cs2_DE;
    const T dgpres = (P.grhog * dge + P.grhor * P.Neff * dre) * b.ia2 * (1.0 / 3.0) + P.grhor * P.Nmnu * dp * b.ia2 +
                     (cs2Q * b.par.grhom * b.par.OmegaDE * deltaq * rQa2 + (cs2Q - b.ca2_Q) * (3.0 * b.aH * rptq * (1.0 / k2)));
    const bool hier_photons = !b.rsa && !b.tca;
    const T polter = hier_photons ? T(y9 + Y(D.idxgp) + Y(D.idxgp + 2)) : T(0.0);
    const T alpha = (H + 6.0 * E) * (0.5 / k2);
    // special rows
    sp[0] = b.aH * b.a;
    sp[1] = -(dgrho + 3.0 * dgpres) * b.a;
    sp[2] = E;
    sp[3] = -thetac - 0.5 * H;
    sp[4] = -b.aH * thetac;
    sp[5] = -thetab - 0.5 * H;
    sp[6] = -b.aH * thetab + k2 * b.cs2 * deltab + b.po * (thg - thetab);
    if (!b.rsa) {
        sp[7] = (4.0 / 3.0) * (-thg - 0.5 * H);
        sp[8] = k2 * (0.25 * dge - 0.5 * y9) - b.opac * (thg - thetab);
        sp[9] = (8.0 / 15.0) * (thg + k2 * alpha) - 0.6 * k * Y(10) - b.opac * (y9 - 0.1 * polter);
        sp[10] = (4.0 / 3.0) * (-thr - 0.5 * H);
        sp[11] = k2 * (0.25 * dre - 0.5 * yr2);
        sp[12] = b.ufa ? -1.5 * (tau > 1e-30 ? b.itau : 1e30) * yr2 + (4.0 / 15.0) * (thr + 0.5 * H)
                       : (8.0 / 15.0) * (thr + k2 * alpha) - 0.6 * k * Y(idxr + 3);
    } else {
        for (int q = 7; q < 13; ++q) sp[q] = 0.0;
    }
    if (b.de_frozen) {
        sp[13] = 0.0;
        sp[14] = 0.0;
    } else {
        sp[13] = -b.opw * (thetaq + 0.5 * H) - 3.0 * (cs2Q - b.w_Q) * b.aH * deltaq -
                 9.0 * b.opw * (cs2Q - b.ca2_Q) * b.aH * b.aH * (1.0 / k2) * thetaq;
        sp[14] = -(1.0 - 3.0 * cs2Q) * b.aH * thetaq + cs2Q * b.iopw * k2 * deltaq;
    }
    g0 = H;
    g1 = E;
    g2 = polter;
}

// ---- RHS f(tau, y) (all entries), T = double or Dual in a ----
// The metric functionals and the 15 "special" rows are computed in straight-line code by every
// lane (no divergence, no reductions); the hierarchy rows are spread over the lanes as one
// uniform class.  Same equations as model_synchronous (perturbations.py:88-525).
// S is the type of the state entries: T when the state carries derivative parts (yd, yk), or
// double for a plain state under a dual background, where the products of coefficients and state
// entries then cost the dual-times-double form.
template <class TM, class T, class S = T>
DDV void rhs_team(const TM& tm, const DiscoebCosmo& P, const Dims& D, const Bg<T>& b, double k, double tau,
                  const double* y, double* f, double* dfda, const double* yd = nullptr, const double* yk = nullptr,
                  int fcomp = 0, int dcomp = 1)
{
    auto Y = [&](int j) { return state_at<S>(y, yd, yk, j); };
    const int nq = D.nq;
    // 1/v of momentum bin q on lane q
    T ivl = 1.0;
    if (tm.full() && tm.lane < nq) ivl = inv_vq(P, b, tm.lane);
    const T vl = rcp(ivl);
    // d ln f0 / d ln q of bin q on lane q
    const double dll = (tm.full() && tm.lane < nq) ? dlfdlq_of(P.q[tm.lane]) : 0.0;
    T sp[15], g0, g1, g2;
    special_part<TM, T, S>(tm, P, D, b, k, tau, Y, ivl, vl, sp, g0, g1, g2);
    if (tm.leader()) {
#pragma unroll
        for (int ss = 0; ss < 15; ++ss) {
            const int i = special_row(D, ss);
            f[i] = comp(sp[ss], fcomp);
            if (dfda) dfda[i] = comp(sp[ss], dcomp);
        }
    }
    const int nh = n_hier_rows(D);
    // every lane runs the same number of iterations: the shuffle in the loop needs all lanes
    for (int h0 = 0; h0 < nh; h0 += tm.nl) {
        const int hh = h0 + tm.lane;
        const bool act = hh < nh;
        const int i = hier_row(D, act ? hh : 0);
        const int q = hier_bin(D, i);
        const T vq = tm.full() ? tm.bcast(vl, q) : rcp(inv_vq(P, b, q));
        const double dlq = tm.full() ? tm.bcast(dll, q) : dlfdlq_of(P.q[q]);
        if (!act) continue;
        T lo, di, up, u[3];
        int st;
        bool trunc;
        hier_coef(P, D, b, k, i, vq, dlq, lo, di, up, u, st, trunc);
        const T fi = lo * Y(i - st) + di * Y(i) + up * Y(trunc ? i : i + st) + u[0] * g0 + u[1] * g1 + u[2] * g2;
        f[i] = comp(fi, fcomp);
        if (dfda) dfda[i] = comp(fi, dcomp);
    }
}

// ---- chain LU (no pivoting) and solves ----
// E: the element type of the factors (double; float in the mixed-precision form)
template <class E> DHD E& bandA(E* A, int i, int m) { return A[7 * i + m + 3]; }
DHD float rcp(float x) { return 1.0f / x; }

template <class E> DDV bool factor_chain(E* A, const Chain& ch)
{
    bool ok = true;
    for (int p = 0; p < ch.len; ++p) {
        const int i = ch.start + p * ch.stride;
        const E piv = bandA(A, i, 0);
        if (!(fabs(piv) > E(0)) || !xfinite((double)piv)) ok = false;
        const E rp = rcp(piv);  // correctly rounded, as 1 / piv
        bandA(A, i, 0) = rp;
        for (int d = 1; d <= ch.kl && p + d < ch.len; ++d) {
            const int r = i + d * ch.stride;
            const E l = bandA(A, r, -d) * rp;
            bandA(A, r, -d) = l;
            if (l != E(0))
                for (int m = 1; m <= ch.ku && p + m < ch.len; ++m) bandA(A, r, m - d) -= l * bandA(A, i, m);
        }
    }
    return ok;
}

// Forward and back substitution along one chain.  With CH = 4 the sweeps run in chunks of four
// elements whose loads are issued together before the dependent arithmetic (the loads do not
// depend on the recurrence), so a chunk costs one shared-memory latency instead of four; CH = 1 is
// the plain element-by-element sweep.  The arithmetic and its order are the same for both.  E: the
// element type of the factors and of the arithmetic (float in the mixed-precision form, where z
// stays double in memory).
template <int CH, class E = double> DDV void solve_chain(const E* A, const Chain& ch, double* z)
{
    const int st = ch.stride, len = ch.len;
    if (ch.kl == 1 && ch.ku == 1) {
        // tridiagonal: carry the neighbour in a register
        int i = ch.start;
        E prev = E(z[i]);
        int p = 1;
        for (; CH > 1 && p + 4 <= len; p += 4) {
            E zz[4], a2[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int j = i + (q + 1) * st;
                zz[q] = E(z[j]);
                a2[q] = A[7 * j + 2];
            }
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                prev = zz[q] - a2[q] * prev;
                z[i + (q + 1) * st] = prev;
            }
            i += 4 * st;
        }
        for (; p < len; ++p) {
            i += st;
            prev = E(z[i]) - A[7 * i + 2] * prev;
            z[i] = prev;
        }
        E next = prev * A[7 * i + 3];
        z[i] = next;
        p = len - 2;
        for (; CH > 1 && p >= 3; p -= 4) {
            E zz[4], a4[4], a3[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int j = i - (q + 1) * st;
                zz[q] = E(z[j]);
                a4[q] = A[7 * j + 4];
                a3[q] = A[7 * j + 3];
            }
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                next = (zz[q] - a4[q] * next) * a3[q];
                z[i - (q + 1) * st] = next;
            }
            i -= 4 * st;
        }
        for (; p >= 0; --p) {
            i -= st;
            next = (E(z[i]) - A[7 * i + 4] * next) * A[7 * i + 3];
            z[i] = next;
        }
        return;
    }
    // pentadiagonal (kl = ku = 2)
    int i = ch.start;
    E p1 = E(z[i]), p2 = E(0);
    int p = 1;
    if (len > 1) {  // the second element has one sub-diagonal neighbour
        i += st;
        const E v = E(z[i]) - A[7 * i + 2] * p1;
        z[i] = v;
        p2 = p1;
        p1 = v;
        p = 2;
    }
    for (; CH > 1 && p + 4 <= len; p += 4) {
        E zz[4], a2[4], a1[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int j = i + (q + 1) * st;
            zz[q] = E(z[j]);
            a2[q] = A[7 * j + 2];
            a1[q] = A[7 * j + 1];
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            E v = zz[q] - a2[q] * p1;
            v -= a1[q] * p2;
            z[i + (q + 1) * st] = v;
            p2 = p1;
            p1 = v;
        }
        i += 4 * st;
    }
    for (; p < len; ++p) {
        i += st;
        E v = E(z[i]) - A[7 * i + 2] * p1;
        v -= A[7 * i + 1] * p2;
        z[i] = v;
        p2 = p1;
        p1 = v;
    }
    E n1 = p1 * A[7 * i + 3], n2 = E(0);
    z[i] = n1;
    p = len - 2;
    if (p >= 0) {  // the last-but-one element has one super-diagonal neighbour
        i -= st;
        E v = E(z[i]) - A[7 * i + 4] * n1;
        v *= A[7 * i + 3];
        z[i] = v;
        n2 = n1;
        n1 = v;
        --p;
    }
    for (; CH > 1 && p >= 3; p -= 4) {
        E zz[4], a4[4], a5[4], a3[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int j = i - (q + 1) * st;
            zz[q] = E(z[j]);
            a4[q] = A[7 * j + 4];
            a5[q] = A[7 * j + 5];
            a3[q] = A[7 * j + 3];
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            E v = zz[q] - a4[q] * n1;
            v -= a5[q] * n2;
            v *= a3[q];
            z[i - (q + 1) * st] = v;
            n2 = n1;
            n1 = v;
        }
        i -= 4 * st;
    }
    for (; p >= 0; --p) {
        i -= st;
        E v = E(z[i]) - A[7 * i + 4] * n1;
        v -= A[7 * i + 5] * n2;
        v *= A[7 * i + 3];
        z[i] = v;
        n2 = n1;
        n1 = v;
    }
}

// Mixed precision: A z = r along one chain with the FP32 factors Af and one step of iterative
// refinement, the residual r - A z0 taken in FP64 with the unfactored band A:
//   z0 = A32^{-1} r,  z = z0 + A32^{-1} (r - A z0).
// rs (n doubles, each chain its own entries) holds r, then the residual and its correction.
DDV void solve_chain_mixed(const double* A, const float* Af, const Chain& ch, double* z, double* rs)
{
    const int st = ch.stride, len = ch.len;
    for (int p = 0; p < len; ++p) rs[ch.start + p * st] = z[ch.start + p * st];
    solve_chain<1, float>(Af, ch, z);
    for (int p = 0; p < len; ++p) {
        const int i = ch.start + p * st;
        double r = rs[i] - A[7 * i + 3] * z[i];
        for (int d = 1; d <= ch.kl && p - d >= 0; ++d) r -= A[7 * i + 3 - d] * z[i - d * st];
        for (int d = 1; d <= ch.ku && p + d < len; ++d) r -= A[7 * i + 3 + d] * z[i + d * st];
        rs[i] = r;
    }
    solve_chain<1, float>(Af, ch, rs);
    for (int p = 0; p < len; ++p) z[ch.start + p * st] += rs[ch.start + p * st];
}

// A z = r for rows >= 2 (in place); gh = gamma*h
template <class TM> DDV void solve_A(const TM& tm, const Dims& D, const ModeMem& M, double gh, double* z)
{
    if (tm.leader()) z[2] *= gh;
    tm.sync();
    const int nc = n_chains(D);
    const double etac = M.sc[SC_ETAC];
    for (int c = tm.lane; c < nc; c += tm.nl) {
        const Chain ch = chain_of(D, c);
        if (c == 0) z[6] += etac * z[2];
        if constexpr (TM::mixed) solve_chain_mixed(M.A, M.Af, ch, z, M.rs);
        else solve_chain<TM::chunk>(M.A, ch, z);
    }
    tm.sync();
}

// Assemble and factor W at (t, y) for step size h.  Needs M.col0 (d f/d a) already set.
// ukeep (may be null): receives the coupling columns U (3 n doubles) before the factorisation
// replaces them by A^{-1} U (the transposed solves of the adjoint need U itself).
template <class TM>
DDV bool factor_W(const TM& tm, const DiscoebCosmo& P, const Dims& D, const Bg<double>& b, double k, double tau,
                  double h, const ModeMem& M, double* ukeep = nullptr)
{
    const int n = D.n;
    const double gh = kR5.gamma * h;
    const double igh = 1.0 / gh;
    double vlane = 1.0;
    if (tm.full() && tm.lane < D.nq) vlane = rcp(inv_vq(P, b, tm.lane));
    const double dll = (tm.full() && tm.lane < D.nq) ? dlfdlq_of(P.q[tm.lane]) : 0.0;
    const int nh = n_hier_rows(D);
    // every lane runs the same number of iterations: the shuffle in the loop needs all lanes
    for (int h0 = 0; h0 < nh; h0 += tm.nl) {
        const int hh = h0 + tm.lane;
        const bool act = hh < nh;
        const int i = hier_row(D, act ? hh : 0);
        const int q = hier_bin(D, i);
        const double vq = tm.full() ? tm.bcast(vlane, q) : rcp(inv_vq(P, b, q));
        const double dlq = tm.full() ? tm.bcast(dll, q) : dlfdlq_of(P.q[q]);
        if (!act) continue;
        double lo, di, up, u[3];
        int st;
        bool trunc;
        hier_coef(P, D, b, k, i, vq, dlq, lo, di, up, u, st, trunc);
        double* Ai = M.A + 7 * i;
        Ai[0] = 0.0; Ai[1] = 0.0; Ai[2] = -lo; Ai[3] = igh - di; Ai[4] = -up; Ai[5] = 0.0; Ai[6] = 0.0;
        M.Z[i] = u[0];
        M.Z[n + i] = u[1];
        M.Z[2 * n + i] = u[2];
    }
    for (int ss = tm.lane; ss < n_special_rows(); ss += tm.nl) {
        const int i = special_row(D, ss);
        double band[7], etac, u[3];
        if (i >= 2) {
            rowc(P, D, b, k, tau, i, band, etac, u);
        } else {
            for (int m = 0; m < 7; ++m) band[m] = 0.0;
            etac = 0.0; u[0] = u[1] = u[2] = 0.0;
        }
        for (int m = 0; m < 7; ++m) M.A[7 * i + m] = -band[m];
        M.A[7 * i + 3] += igh;
        if (i == 6) M.sc[SC_ETAC] = etac;
        M.Z[i] = u[0];
        M.Z[n + i] = u[1];
        M.Z[2 * n + i] = u[2];
    }
    const int ns = n_slots(D);
    for (int sl = tm.lane; sl < ns; sl += tm.nl) {
        const int j = slot_index(D, sl);
        double gc[3];
        gcol(P, D, b, k, j, gc);
        M.Gs[sl] = gc[0];
        M.Gs[kMaxSlots + sl] = gc[1];
        M.Gs[2 * kMaxSlots + sl] = gc[2];
        M.F1s[sl] = f1col(P, D, b, k, j);
    }
    if (tm.leader()) {
        M.sc[SC_W00] = igh - M.col0[0];
        double u[3];
        f1u(P, b, k, u);
        M.sc[SC_F1U] = u[0];
        M.sc[SC_F1U + 1] = u[1];
        M.sc[SC_F1U + 2] = u[2];
    }
    tm.sync();
    if (ukeep)
        for (int i = tm.lane; i < 3 * n; i += tm.nl) ukeep[i] = M.Z[i];
    bool ok = true;
    const int nc = n_chains(D);
    for (int c = tm.lane; c < nc; c += tm.nl) {
        const Chain ch = chain_of(D, c);
        if constexpr (TM::mixed) {  // FP32 factors; A keeps the FP64 band for the residuals
            for (int p = 0; p < ch.len; ++p)
                for (int m = 0; m < 7; ++m) {
                    const int i = ch.start + p * ch.stride;
                    M.Af[7 * i + m] = (float)M.A[7 * i + m];
                }
            ok = factor_chain(M.Af, ch) && ok;
        } else {
            ok = factor_chain(M.A, ch) && ok;
        }
    }
    tm.sync();
    // Z = A^{-1} U
    for (int r = 0; r < 3; ++r) solve_A(tm, D, M, gh, M.Z + r * n);
    // C = I - G Z, F1Z = F1 . Z
    double acc[12];
    for (int q = 0; q < 12; ++q) acc[q] = 0.0;
    for (int sl = tm.lane; sl < ns; sl += tm.nl) {
        const int j = slot_index(D, sl);
        for (int r = 0; r < 3; ++r)
            for (int s = 0; s < 3; ++s) acc[3 * r + s] += M.Gs[r * kMaxSlots + sl] * M.Z[s * n + j];
        for (int s = 0; s < 3; ++s) acc[9 + s] += M.F1s[sl] * M.Z[s * n + j];
    }
    double C[9];
    for (int q = 0; q < 9; ++q) C[q] = ((q % 4) == 0 ? 1.0 : 0.0) - tm.sum(acc[q]);
    double F1Z[3];
    for (int s = 0; s < 3; ++s) F1Z[s] = tm.sum(acc[9 + s]);
    // 3x3 inverse by cofactors
    const double c00 = C[4] * C[8] - C[5] * C[7];
    const double c01 = C[5] * C[6] - C[3] * C[8];
    const double c02 = C[3] * C[7] - C[4] * C[6];
    const double det = C[0] * c00 + C[1] * c01 + C[2] * c02;
    const double id = 1.0 / det;
    double Ci[9];
    Ci[0] = c00 * id;
    Ci[1] = (C[2] * C[7] - C[1] * C[8]) * id;
    Ci[2] = (C[1] * C[5] - C[2] * C[4]) * id;
    Ci[3] = c01 * id;
    Ci[4] = (C[0] * C[8] - C[2] * C[6]) * id;
    Ci[5] = (C[2] * C[3] - C[0] * C[5]) * id;
    Ci[6] = c02 * id;
    Ci[7] = (C[1] * C[6] - C[0] * C[7]) * id;
    Ci[8] = (C[0] * C[4] - C[1] * C[3]) * id;
    if (tm.leader()) {
        for (int q = 0; q < 9; ++q) M.sc[SC_CINV + q] = Ci[q];
        for (int s = 0; s < 3; ++s) M.sc[SC_F1Z + s] = F1Z[s];
    }
    tm.sync();
    return ok && xfinite(det) && det != 0.0;
}

// x = W^{-1} r, in place in v
template <class TM> DDV void solve_W(const TM& tm, const Dims& D, const ModeMem& M, double h, double* v)
{
    const int n = D.n;
    const double gh = kR5.gamma * h;
    const double x0 = v[0] / M.sc[SC_W00];
    tm.sync();
    for (int i = tm.lane; i < n; i += tm.nl)
        if (i >= 1) v[i] += M.col0[i] * x0;
    tm.sync();
    solve_A(tm, D, M, gh, v);
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
    const int ns = n_slots(D);
    for (int sl = tm.lane; sl < ns; sl += tm.nl) {
        const double zj = v[slot_index(D, sl)];
        a0 += M.Gs[sl] * zj;
        a1 += M.Gs[kMaxSlots + sl] * zj;
        a2 += M.Gs[2 * kMaxSlots + sl] * zj;
        a3 += M.F1s[sl] * zj;
    }
    const double gz0 = tm.sum(a0), gz1 = tm.sum(a1), gz2 = tm.sum(a2), f1z = tm.sum(a3);
    const double* Ci = M.sc + SC_CINV;
    const double c0 = Ci[0] * gz0 + Ci[1] * gz1 + Ci[2] * gz2;
    const double c1 = Ci[3] * gz0 + Ci[4] * gz1 + Ci[5] * gz2;
    const double c2 = Ci[6] * gz0 + Ci[7] * gz1 + Ci[8] * gz2;
    const double r1 = v[1];
    tm.sync();
    for (int i = tm.lane; i < n; i += tm.nl)
        if (i >= 2) v[i] += M.Z[i] * c0 + M.Z[n + i] * c1 + M.Z[2 * n + i] * c2;
    if (tm.leader()) {
        const double* F1Z = M.sc + SC_F1Z;
        const double* F1U = M.sc + SC_F1U;
        v[1] = gh * (r1 + f1z + (F1Z[0] + F1U[0]) * c0 + (F1Z[1] + F1U[1]) * c1 + (F1Z[2] + F1U[2]) * c2);
        v[0] = x0;
    }
    tm.sync();
}

DHD int regime_at(const DiscoebCosmo& P, double t, const double* sw)
{
    const bool rsa = P.use_rsa && t >= sw[0];
    const bool ufa = !rsa && P.use_ufa && t >= sw[1];
    const bool tca = !rsa && P.use_tca && t < sw[2];
    return (rsa ? 1 : 0) | (ufa ? 2 : 0) | (tca ? 4 : 0);
}

struct SolveResult {
    int status, steps, accepted, outputs;
};

// Tangent of stage s of the Rosenbrock step along one parameter direction: with
// k_s = W^{-1} r_s, the derivative is k_s' = W^{-1} (r_s' + J' k_s), where r_s' holds the
// directional derivative of f at the stage state (state tangent u_s' and the parameter /
// table tangents tn) and J' k_s = d/de [J(y_n + e y_n', p + e p') k_s].  Rows >= 1 of f are
// linear and homogeneous in y[1:] with coefficients that depend on a (through the background)
// and the parameters, so the columns >= 1 of J' applied to k_s are the e-part of f evaluated at
// the state k_s with the dual background bj of the step start; column 0 contributes
// k_s[0] d/de(d f/d a), computed once per step into c0d.  The step sizes are the forward solve's
// (the derivative of the discrete scheme with the accepted step sequence held fixed).
// Stage 0's f' (the e-part of f at the step start) comes from the same once-per-step
// hyper-dual pass as c0d and is in TT.fd on entry for s = 0.
template <class TM>
DDV void tangent_stage(const TM& tm, const DiscoebCosmo& P, const Dims& D, double k, double t, double h, int regime,
                       const ModeMem& M, const TanMem& TT, const DiscoebTangent* tn, const Bg<Dual>& bj, int s,
                       int& hint)
{
    const int n = D.n;
    const double* us = (s == 0) ? M.y : M.u;
    for (int i = tm.lane; i < n; i += tm.nl) {
        double v;
        if (s == 0) v = TT.yd[i];
        else if (s <= 5) {
            v = TT.yd[i];
            for (int j = 0; j < s; ++j) v += kR5.a[s][j] * TT.Kd[j * n + i];
        } else {
            v = TT.ud[i] + TT.Kd[(s - 1) * n + i];
        }
        TT.ud[i] = v;
    }
    tm.sync();
    if (s > 0) {
        const double ts = (s <= 5) ? t + kR5.c[s] * h : t + h;
        Bg<Dual> bt;
        bg_eval_team(tm, P, Dual(us[0], TT.ud[0]), ts, k, regime, bt, hint, tn);
        rhs_team(tm, P, D, bt, k, ts, us, TT.fd, (double*)nullptr, TT.ud, (const double*)nullptr, 1, 1);
    }
    const double* Ks = M.K + s * n;
    rhs_team<TM, Dual, double>(tm, P, D, bj, k, t, Ks, TT.jk, (double*)nullptr, (const double*)nullptr,
                               (const double*)nullptr, 1, 1);
    tm.sync();
    {
        const double k0 = Ks[0];
        for (int i = tm.lane; i < n; i += tm.nl) TT.jk[i] = (i == 0 ? 0.0 : TT.jk[i]) + k0 * TT.c0d[i];
    }
    tm.sync();
    Bg<double> b0;
    b0.rsa = (regime & 1) != 0;
    b0.ufa = !b0.rsa && (regime & 2) != 0;
    b0.tca = !b0.rsa && (regime & 4) != 0;
    double* Kds = TT.Kd + s * n;
    const double ih = 1.0 / h;
    for (int i = tm.lane; i < n; i += tm.nl) {
        double r = TT.fd[i] + TT.jk[i];
        if (s < 5) r += h * kR5.d[s] * dtau_row(D, b0, t, i, TT.yd);
        for (int j = 0; j < s; ++j) r += kR5.C[s][j] * ih * TT.Kd[j * n + i];
        Kds[i] = r;
    }
    tm.sync();
    solve_W(tm, D, M, h, Kds);
}

// Tangent of one accepted Rodas5 step from a record of the forward step: M.y (start state),
// M.K (the 8 stages) and the factorisation of W (M.A, M.Z, M.Gs, M.F1s, M.sc, M.col0), with
// M.u a buffer of this team's own where the stage states are rebuilt.  Same arithmetic as the
// tangent part of rodas5_step; on return TT.yd holds the tangent at t + h.
template <class TM>
DDV void tangent_step(const TM& tm, const DiscoebCosmo& P, const Dims& D, double k, double t, double h, int regime,
                      const ModeMem& M, const TanMem& TT, const DiscoebTangent* tn, int& hint)
{
    const int n = D.n;
    // once per step: the background at the step start in hyper-dual numbers (direction e, and a);
    // its e-part is the dual background bj, and one RHS pass gives d/de(d f/d a) (c0d) and
    // stage 0's f' (fd)
    Bg<Dual> bj;
    {
        Bg<HDual> bh;
        bg_eval_team(tm, P, HDual(Dual(M.y[0], TT.yd[0]), Dual(1.0, 0.0)), t, k, regime, bh, hint, tn);
        bj = bg_value(bh);
        rhs_team(tm, P, D, bh, k, t, M.y, TT.c0d, TT.fd, TT.yd, (const double*)nullptr, 3, 1);
        tm.sync();
    }
    for (int s = 0; s < 8; ++s) {
        if (s > 0) {
            for (int i = tm.lane; i < n; i += tm.nl) {
                double v;
                if (s <= 5) {
                    v = M.y[i];
                    for (int j = 0; j < s; ++j) v += kR5.a[s][j] * M.K[j * n + i];
                } else {
                    v = M.u[i] + M.K[(s - 1) * n + i];
                }
                M.u[i] = v;
            }
            tm.sync();
        }
        tangent_stage(tm, P, D, k, t, h, regime, M, TT, tn, bj, s, hint);
    }
    for (int i = tm.lane; i < n; i += tm.nl) TT.yd[i] = TT.ud[i] + TT.Kd[7 * n + i];
    tm.sync();
}

// One Rodas5 step from (t, y) with size h: on return M.u + M.K[7] is the candidate and
// M.K[7] the error estimate.  Returns false on a non-finite factorisation.
template <class TM>
DDV bool rodas5_step(const TM& tm, const DiscoebCosmo& P, const Dims& D, double k, double t, double h, int regime,
                     const ModeMem& M, int& hint, const DiscoebTangent* tn = nullptr, const TanMem* TT = nullptr,
                     double* ukeep = nullptr)
{
    const int n = D.n;
    // Jacobian column d f/d a and f(y) in one dual pass
    Bg<Dual> bd;
    bg_eval_team(tm, P, Dual(M.y[0], 1.0), t, k, regime, bd, hint);
    rhs_team<TM, Dual, double>(tm, P, D, bd, k, t, M.y, M.f, M.col0);
    const Bg<double> b = bg_value(bd);
    for (int i = tm.lane; i < n; i += tm.nl) M.dT[i] = dtau_row(D, b, t, i, M.y);
    tm.sync();
    const bool ok = factor_W(tm, P, D, b, k, t, h, M, ukeep);
    // tangent, once per step: the background at the step start with its derivative along the
    // direction, and d/de of the Jacobian column d f / d a (see tangent_stage)
    Bg<Dual> bj;
    if (TT) {
        Bg<HDual> bh;
        bg_eval_team(tm, P, HDual(Dual(M.y[0], TT->yd[0]), Dual(1.0, 0.0)), t, k, regime, bh, hint, tn);
        bj = bg_value(bh);
        rhs_team(tm, P, D, bh, k, t, M.y, TT->c0d, TT->fd, TT->yd, (const double*)nullptr, 3, 1);
        tm.sync();
    }
    const double ih = 1.0 / h;
    for (int s = 0; s < 8; ++s) {
        double* Ks = M.K + s * n;
        if (s > 0) {
            for (int i = tm.lane; i < n; i += tm.nl) {
                double v;
                if (s <= 5) {
                    v = M.y[i];
                    for (int j = 0; j < s; ++j) v += kR5.a[s][j] * M.K[j * n + i];
                } else {
                    v = M.u[i] + M.K[(s - 1) * n + i];
                }
                M.u[i] = v;
            }
            tm.sync();
            const double ts = (s <= 5) ? t + kR5.c[s] * h : t + h;
            Bg<double> bs;
            bg_eval_team(tm, P, M.u[0], ts, k, regime, bs, hint);
            rhs_team(tm, P, D, bs, k, ts, M.u, M.f, (double*)nullptr);
            tm.sync();
        }
        for (int i = tm.lane; i < n; i += tm.nl) {
            double r = M.f[i];
            if (s < 5) r += h * kR5.d[s] * M.dT[i];
            for (int j = 0; j < s; ++j) r += kR5.C[s][j] * ih * M.K[j * n + i];
            Ks[i] = r;
        }
        tm.sync();
        solve_W(tm, D, M, h, Ks);
        if (TT) tangent_stage(tm, P, D, k, t, h, regime, M, *TT, tn, bj, s, hint);
    }
    return ok;
}

// Adaptive solve of one mode from y(t0) in M.y.  At every output time the team calls
// emit(j, y) with the state exactly at tout[j].  sw[3]: RSA start, UFA start, TCA end.
// called for every accepted step before the state advances, with (t, h, t + h as the solver
// rounds it, regime) of the step and M still holding its start state, stages and
// factorisation; returning false stops the solve (DISCOEB_ABORTED)
struct NoAccept {
    DHD bool operator()(double, double, double, int) const { return true; }
};

template <class TM, class Emit, class Accept = NoAccept>
DDV SolveResult solve_mode(const TM& tm, const DiscoebCosmo& P, const Dims& D, const DiscoebControl& C, double k,
                           double t0, const double* sw, int nout, const double* tout, const ModeMem& M, Emit& emit,
                           const DiscoebTangent* tn = nullptr, const TanMem* TT = nullptr, double* tlog = nullptr,
                           int tlog_cap = 0, Accept* accept = nullptr)
{
    const int n = D.n;
    SolveResult R = {DISCOEB_OK, 0, 0, 0};
    double t1 = tout[0];
    for (int j = 1; j < nout; ++j) t1 = tout[j] > t1 ? tout[j] : t1;
    const double eo = 6.0;  // diffrax error order of a 5th-order method: order + 1
    const double c1 = (C.icoeff + C.pcoeff + C.dcoeff) / eo;
    const double c2 = -(C.pcoeff + 2.0 * C.dcoeff) / eo;
    const double c3 = C.dcoeff / eo;
    double prev_inv = 1.0, prev_prev_inv = 1.0;
    double t = t0;
    double dt = fmin(t0 / 4.0, 0.5 * (t1 - t0));  // dt0 of perturbations.py:910
    int iout = 0;
    const int idx[6] = {0, 2, 3, 5, 6, 7};
    const double w6[6] = {1.0, k * k, 1.0, 1.0, 1.0 / (k * k), 1.0};
    int hint = P.xe_loga.n_knots / 2;
    while (t < t1) {
        if (R.steps >= C.max_steps) { R.status = DISCOEB_MAX_STEPS; break; }
        double tev = t1;
        if (iout < nout && tout[iout] < tev) tev = tout[iout];
        for (int q = 0; q < 3; ++q)
            if (sw[q] > t && sw[q] < tev) tev = sw[q];
        const double dt_try = dt;
        double tnext = t + dt;
        bool clipped = false;
        if (tnext >= tev - 1e-12 * fabs(tev)) { clipped = tnext > tev; tnext = tev; }
        const double h = tnext - t;
        if (!(h > 1e-14 * fabs(t))) { R.status = DISCOEB_DT_UNDERFLOW; break; }
        const int regime = regime_at(P, t, sw);
        const bool ok = rodas5_step(tm, P, D, k, t, h, regime, M, hint, tn, TT);
        R.steps++;
        // weighted RMS error over (a, eta, delta_c, delta_b, theta_b, delta_gamma)
        // (perturbations.py:855-878 with the weights of :913)
        double sumsq = 0.0;
        for (int q = 0; q < 6; ++q) {
            const int i = idx[q];
            const double y1 = M.u[i] + M.K[7 * n + i];
            const double sc = fmax(fabs(M.y[i]), fabs(y1));
            const double e = M.K[7 * n + i] / (C.atol + C.rtol * sc) * w6[q];
            sumsq += e * e;
        }
        // non-finite candidate entries count 1, non-finite entries of the step start (state or
        // Jacobian column d f/d a: a NaN or an infinity in an input table) count 1024
        double lf = 0.0;
        for (int i = tm.lane; i < n; i += tm.nl) {
            lf += xfinite(M.u[i] + M.K[7 * n + i]) ? 0.0 : 1.0;
            lf += (xfinite(M.y[i]) && xfinite(M.col0[i])) ? 0.0 : 1024.0;
        }
        const double nbad = tm.sum(lf);
        if (nbad >= 1024.0) { R.status = DISCOEB_NONFINITE; break; }  // no step size can help
        const bool finite = ok && nbad == 0.0;
        const double err = finite ? sqrt(sumsq / 6.0) : INFINITY;
        const bool keep = err < 1.0;
        double inv = 1.0 / err;
        const double f1 = pow(inv, c1);
        const double f2 = (c2 == 0.0) ? 1.0 : pow(prev_inv, c2);
        const double f3 = (c3 == 0.0) ? 1.0 : pow(prev_prev_inv, c3);
        const double fmn = keep ? 1.0 : C.factormin;
        double factor = 0.9 * f1 * f2 * f3;
        if (!(factor == factor)) factor = fmn;
        factor = fmin(fmax(factor, fmn), C.factormax);
        if (inv == 0.0 || !xfinite(inv)) inv = 1.0;
        double dtn = h * factor;
        tm.sync();
        if (keep) {
            if (accept && !(*accept)(t, h, tnext, regime)) { R.status = DISCOEB_ABORTED; break; }
            R.accepted++;
            for (int i = tm.lane; i < n; i += tm.nl) M.y[i] = M.u[i] + M.K[7 * n + i];
            if (TT)
                for (int i = tm.lane; i < n; i += tm.nl) TT->yd[i] = TT->ud[i] + TT->Kd[7 * n + i];
            tm.sync();
            if (tlog && R.accepted <= tlog_cap) tlog[R.accepted - 1] = tnext;
            t = tnext;
            while (iout < nout && tout[iout] <= t) {
                emit(iout, M.y, regime);
                iout++;
            }
            if (clipped && dt_try > dtn) dtn = dt_try;
            prev_prev_inv = prev_inv;
            prev_inv = inv;
        }
        dt = dtn;
        tm.sync();
    }
    if (R.status == DISCOEB_OK && iout < nout) R.status = DISCOEB_MAX_STEPS;
    R.outputs = iout;
    return R;
}

}  // namespace dscb
