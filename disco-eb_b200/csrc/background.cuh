// Background cosmology and Recfast thermal history, templated on the number type.
//
// The producer of the perturbation solve's input tables: densities and the massive-neutrino
// tables (background.py:141-189 of the reference), the conformal-time integral, the Recfast
// ionisation history with its GRK4A Rosenbrock solve (thermodynamics_recfast.py:124-492,
// ode_integrators_stiff.py:157-254) and the visibility tables (background.py:191-345).
//
// T = double gives the values.  T = Fw<double> carries one directional derivative with respect
// to the cosmological parameters through the very same operations: every branch, table index and
// step-size decision is taken on the value part, so the value part is the double computation and
// the derivative part is the exact derivative of the discrete result with the Recfast step
// sequence held fixed (what forward-mode AD through the reference's solver loop gives).  The
// Recfast Jacobian d f / d y is itself taken in forward mode (Fw<T>), so its parameter
// derivative is exact as well.
//
// All arrays are the caller's: nothing here allocates.
#pragma once

#include <cmath>
#include <cstdint>

#include "discoeb.h"

#if defined(__CUDACC__)
#define BGF __host__ __device__ inline
#else
#define BGF inline
#endif

namespace dscb {
namespace bgn {

// ---------------------------------------------------------------------------------------------
// Forward-mode number with correctly rounded division (the value part of a quotient is the
// double quotient, so T = Fw<double> reproduces the double path's values exactly).
template <class B> struct Fw {
    B v, d;
    BGF Fw() : v(0.0), d(0.0) {}
    BGF Fw(double x) : v(x), d(0.0) {}
    BGF Fw(const B& x, const B& dx) : v(x), d(dx) {}
};

BGF double re(double x) { return x; }
template <class B> BGF double re(const Fw<B>& x) { return re(x.v); }

template <class B> BGF Fw<B> operator+(const Fw<B>& a, const Fw<B>& b) { return Fw<B>(a.v + b.v, a.d + b.d); }
template <class B> BGF Fw<B> operator-(const Fw<B>& a, const Fw<B>& b) { return Fw<B>(a.v - b.v, a.d - b.d); }
template <class B> BGF Fw<B> operator-(const Fw<B>& a) { return Fw<B>(-a.v, -a.d); }
template <class B> BGF Fw<B> operator*(const Fw<B>& a, const Fw<B>& b) { return Fw<B>(a.v * b.v, a.d * b.v + a.v * b.d); }
template <class B> BGF Fw<B> operator/(const Fw<B>& a, const Fw<B>& b)
{
    const B q = a.v / b.v;
    return Fw<B>(q, (a.d - q * b.d) / b.v);
}
template <class B> BGF Fw<B> operator+(const Fw<B>& a, double b) { return Fw<B>(a.v + b, a.d); }
template <class B> BGF Fw<B> operator+(double a, const Fw<B>& b) { return Fw<B>(a + b.v, b.d); }
template <class B> BGF Fw<B> operator-(const Fw<B>& a, double b) { return Fw<B>(a.v - b, a.d); }
template <class B> BGF Fw<B> operator-(double a, const Fw<B>& b) { return Fw<B>(a - b.v, -b.d); }
template <class B> BGF Fw<B> operator*(const Fw<B>& a, double b) { return Fw<B>(a.v * b, a.d * b); }
template <class B> BGF Fw<B> operator*(double a, const Fw<B>& b) { return Fw<B>(a * b.v, a * b.d); }
template <class B> BGF Fw<B> operator/(const Fw<B>& a, double b) { return Fw<B>(a.v / b, a.d / b); }
template <class B> BGF Fw<B> operator/(double a, const Fw<B>& b)
{
    const B q = a / b.v;
    return Fw<B>(q, -(q * b.d) / b.v);
}
template <class B> BGF Fw<B>& operator+=(Fw<B>& a, const Fw<B>& b) { a.v += b.v; a.d += b.d; return a; }
template <class B> BGF Fw<B>& operator-=(Fw<B>& a, const Fw<B>& b) { a.v -= b.v; a.d -= b.d; return a; }

BGF double bexp(double x) { return exp(x); }
BGF double blog(double x) { return log(x); }
BGF double bsqrt(double x) { return sqrt(x); }
BGF double bpow(double x, double p) { return pow(x, p); }
template <class B> BGF Fw<B> bexp(const Fw<B>& x)
{
    const B e = bexp(x.v);
    return Fw<B>(e, e * x.d);
}
template <class B> BGF Fw<B> blog(const Fw<B>& x) { return Fw<B>(blog(x.v), x.d / x.v); }
template <class B> BGF Fw<B> bsqrt(const Fw<B>& x)
{
    const B s = bsqrt(x.v);
    return Fw<B>(s, x.d / (2.0 * s));
}
template <class B> BGF Fw<B> bpow(const Fw<B>& x, double p) { return Fw<B>(bpow(x.v, p), p * bpow(x.v, p - 1.0) * x.d); }
// x ** y with both arguments carrying derivatives
BGF double bpow2(double x, double y) { return pow(x, y); }
template <class B> BGF Fw<B> bpow2(const Fw<B>& x, const Fw<B>& y)
{
    const B v = bpow2(x.v, y.v);
    return Fw<B>(v, v * (y.d * blog(x.v) + y.v * x.d / x.v));
}
template <class B> BGF Fw<B> bpow2(double x, const Fw<B>& y)
{
    const B v = bpow2(x, y.v);
    return Fw<B>(v, v * y.d * log(x));
}
// select on a condition taken on value parts
template <class T> BGF T bsel(bool c, const T& a, const T& b) { return c ? a : b; }

// Conversion of a number to a type that carries one more derivative level (zero derivative).
BGF double up(double x, const double*) { return x; }
template <class B> BGF Fw<B> up(const B& x, const Fw<B>*) { return Fw<B>(x, B(0.0)); }
template <class B> BGF Fw<B> up(const Fw<B>& x, const Fw<B>*) { return x; }
template <class Y, class T> BGF Y lift(const T& x) { return up(x, (const Y*)nullptr); }

// value and first derivative parts as doubles
BGF double vpart(double x) { return x; }
BGF double dpart(double) { return 0.0; }
BGF double vpart(const Fw<double>& x) { return x.v; }
BGF double dpart(const Fw<double>& x) { return x.d; }

// ---------------------------------------------------------------------------------------------
// Physical constants (thermodynamics_recfast.py:38-122; background.py:146-150).
constexpr double kPi = 3.141592653589793;
constexpr double const_G = 6.67430e-11;
constexpr double const_mH = 1.67353284e-27;
constexpr double const_me = 9.1093837015e-31;
constexpr double const_mHe_mH = 3.97146570884;
constexpr double const_c = 2.99792458e08;
constexpr double const_h = 6.62607015e-34;
constexpr double const_kB = 1.380649e-23;
constexpr double const_sigma = 6.6524587321e-29;
constexpr double const_arad = 4 * 5.670374419e-8 / const_c;
constexpr double bigH = 3.2407792902755102e-18;
constexpr double const_dens_fac = 11.223810928601939;
constexpr double const_EionHe12s = 6.314878282674e5;
constexpr double Lambda_ = 8.2245809;
constexpr double Lambda_He = 51.3;
constexpr double L_H_ion = 1.096787737e7;
constexpr double L_H_alpha = 8.225916453e6;
constexpr double L_He1_ion = 1.98310772e7;
constexpr double L_He2_ion = 4.389088863e7;
constexpr double L_He_2s = 1.66277434e7;
constexpr double L_He_2p = 1.71134891e7;
constexpr double A2P_s = 1.798287e9;
constexpr double A2P_t = 177.58;
constexpr double L_He_2Pt = 1.690871466e7;
constexpr double L_He_2St = 1.5985597526e7;
constexpr double L_He2St_ion = 3.8454693845e6;
constexpr double sigma_He_2Ps = 1.436289e-22;
constexpr double sigma_He_2Pt = 1.484872e-22;
constexpr double AGauss1 = -0.14;
constexpr double AGauss2 = 0.05;
constexpr double zGauss1 = 7.28;
constexpr double zGauss2 = 6.75;
constexpr double wGauss1 = 0.18;
constexpr double wGauss2 = 0.33;
constexpr double H_frac = 1.0e-3;
constexpr double kC2ok = 1.62581581e4;
constexpr double kAkthom = 2.3038921003709498e-9;

// Derived atomic constants, evaluated once (the expressions of thermodynamics_recfast.py:61-78).
struct RecConst {
    double Lalpha, Lalpha_He, CDB, CDB_He, CB1, CB1_He1, CR, CK, CK_He, CL, CL_He, CT, Bfact, CL_PSt, hcL2St_kB;
    double a_PPB, b_PPB, c_PPB, d_PPB, a_VF, b_VF, T_0, T_1, a_trip, b_trip, sqrt_pi;
};
BGF RecConst rec_const()
{
    RecConst k;
    k.Lalpha = 1.0 / L_H_alpha;
    k.Lalpha_He = 1.0 / L_He_2p;
    const double DeltaB = const_h * const_c * (L_H_ion - L_H_alpha);
    k.CDB = DeltaB / const_kB;
    const double DeltaB_He = const_h * const_c * (L_He1_ion - L_He_2s);
    k.CDB_He = DeltaB_He / const_kB;
    k.CB1 = const_h * const_c * L_H_ion / const_kB;
    k.CB1_He1 = const_h * const_c * L_He1_ion / const_kB;
    k.CR = 2.0 * kPi * (const_me / const_h) * (const_kB / const_h);
    k.CK = pow(k.Lalpha, 3.0) / (8.0 * kPi);
    k.CK_He = pow(k.Lalpha_He, 3.0) / (8.0 * kPi);
    k.CL = const_c * const_h / (const_kB * k.Lalpha);
    k.CL_He = const_c * const_h / (const_kB / L_He_2s);
    k.CT = (8.0 / 3.0) * (const_sigma / (const_me * const_c)) * const_arad;
    k.Bfact = const_h * const_c * (L_He_2p - L_He_2s) / const_kB;
    k.CL_PSt = const_h * const_c * (L_He_2Pt - L_He_2St) / const_kB;
    k.hcL2St_kB = const_h * const_c * L_He_2St / const_kB;
    k.a_PPB = 4.309;
    k.b_PPB = -0.6166;
    k.c_PPB = 0.6703;
    k.d_PPB = 0.5300;
    k.a_VF = pow(10.0, -16.744);
    k.b_VF = 0.711;
    k.T_0 = pow(10.0, 0.477121);
    k.T_1 = pow(10.0, 5.114);
    k.a_trip = pow(10.0, -16.306);
    k.b_trip = 0.761;
    k.sqrt_pi = sqrt(kPi);
    return k;
}

// ---------------------------------------------------------------------------------------------
// Natural cubic spline (spline_interpolation.py:6-228): second derivatives S from the Thomas
// solve with natural ends; the interval index is floor((x - x0)/dx) on uniform knots, else the
// number of knots strictly below x minus one, clipped to [0, n-2].
template <class T> struct Spline {
    int n;
    bool uniform;
    const T* x;
    const T* y;
    const T* S;
    const T* Icum;  // cumulative interval integrals (may be null when not integrated)
};

// S[n] of the natural spline through (x, y); cp, dp: scratch of n doubles' worth of T each.
template <class T> BGF void spline_build(int n, const T* x, const T* y, T* S, T* cp, T* dp)
{
    for (int i = 0; i < n; ++i) S[i] = T(0.0);
    const int m = n - 2;
    if (m <= 0) return;
    // row i of the interior system couples S[i], S[i+1], S[i+2] (knots i .. i+2)
    for (int i = 0; i < m; ++i) {
        const T h0 = x[i + 1] - x[i], h1 = x[i + 2] - x[i + 1];
        const T a = h0, b = 2.0 * (h0 + h1), c = h1;
        const T d = 6.0 * ((y[i + 2] - y[i + 1]) / h1 - (y[i + 1] - y[i]) / h0);
        if (i == 0) {
            cp[0] = c / b;
            dp[0] = d / b;
        } else {
            const T denom = b - a * cp[i - 1];
            cp[i] = (i < m - 1) ? c / denom : T(0.0);
            dp[i] = (d - a * dp[i - 1]) / denom;
        }
    }
    S[m] = dp[m - 1];
    for (int i = m - 2; i >= 0; --i) S[i + 1] = dp[i] - cp[i] * S[i + 2];
}

// Icum[n]: Icum[0] = 0, Icum[i+1] = Icum[i] + integral over interval i.
template <class T> BGF void spline_integrals(int n, const T* x, const T* y, const T* S, T* Icum)
{
    Icum[0] = T(0.0);
    for (int i = 0; i + 1 < n; ++i) {
        const T h = x[i + 1] - x[i];
        const T a = y[i];
        const T b = (y[i + 1] - y[i]) / h - h * (S[i + 1] + 2.0 * S[i]) / 6.0;
        const T c = S[i] / 2.0;
        const T dd = (S[i + 1] - S[i]) / (6.0 * h);
        const T h2 = h * h, h3 = h2 * h, h4 = h3 * h;
        Icum[i + 1] = Icum[i] + (a * h + b * h2 / 2.0 + c * h3 / 3.0 + dd * h4 / 4.0);
    }
}

template <class T> BGF int spline_index(const Spline<T>& s, double xn)
{
    long idx;
    if (s.uniform) {
        const double x0 = re(s.x[0]);
        const double dxinv = 1.0 / (re(s.x[1]) - x0);
        idx = (long)floor((xn - x0) * dxinv);
    } else {
        // count of knots strictly below xn, minus one (binary search: knots increase)
        int lo = 0, hi = s.n;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (re(s.x[mid]) < xn) lo = mid + 1; else hi = mid;
        }
        idx = lo - 1;
    }
    if (idx < 0) idx = 0;
    if (idx > s.n - 2) idx = s.n - 2;
    return (int)idx;
}

template <class T, class Q> BGF T spline_eval(const Spline<T>& s, const Q& xq)
{
    const int i = spline_index(s, re(xq));
    const T h = s.x[i + 1] - s.x[i];
    const T d = xq - s.x[i];
    const T t = d / h;
    const T A = 1.0 - t, B = t;
    return A * s.y[i] + B * s.y[i + 1] + ((A * A * A - A) * s.S[i] + (B * B * B - B) * s.S[i + 1]) * (h * h) / 6.0;
}

template <class T, class Q> BGF void spline_d12(const Spline<T>& s, const Q& xq, T& d1, T& d2)
{
    const int i = spline_index(s, re(xq));
    const T h = s.x[i + 1] - s.x[i];
    const T d = xq - s.x[i];
    const T b = (s.y[i + 1] - s.y[i]) / h - h * (s.S[i + 1] + 2.0 * s.S[i]) / 6.0;
    const T c = s.S[i] / 2.0;
    const T dd = (s.S[i + 1] - s.S[i]) / (6.0 * h);
    d1 = b + 2.0 * c * d + 3.0 * dd * (d * d);
    d2 = 2.0 * c + 6.0 * dd * d;
}

template <class T, class Q> BGF T spline_integral(const Spline<T>& s, const Q& xq)
{
    const int i = spline_index(s, re(xq));
    const T h = s.x[i + 1] - s.x[i];
    const T d = xq - s.x[i];
    const T b = (s.y[i + 1] - s.y[i]) / h - h * (s.S[i + 1] + 2.0 * s.S[i]) / 6.0;
    const T c = s.S[i] / 2.0;
    const T dd = (s.S[i + 1] - s.S[i]) / (6.0 * h);
    const T d2 = d * d, d3 = d2 * d, d4 = d3 * d;
    return s.Icum[i] + (s.y[i] * d + b * d2 / 2.0 + c * d3 / 3.0 + dd * d4 / 4.0);
}

// ---------------------------------------------------------------------------------------------
// numpy's pairwise summation order for up to 128 terms (what np.sum does on a short array), so
// that Romberg sums match the numpy restatement to the last bit where the terms do.
template <class T> BGF T pairwise_sum(const T* a, int n)
{
    if (n < 8) {
        T r = T(0.0);
        for (int i = 0; i < n; ++i) r += a[i];
        return r;
    }
    T r[8];
    for (int j = 0; j < 8; ++j) r[j] = a[j];
    int i = 8;
    for (; i < n - (n % 8); i += 8)
        for (int j = 0; j < 8; ++j) r[j] += a[i + j];
    T res = ((r[0] + r[1]) + (r[2] + r[3])) + ((r[4] + r[5]) + (r[6] + r[7]));
    for (; i < n; ++i) res += a[i];
    return res;
}

// Romberg quadrature on 2^6 panels (jax_cosmo romb as used at background.py:183-186 and
// thermodynamics_recfast.py:488): trapezoid sums refined by Richardson extrapolation.
template <class T, class F> BGF T romb6(const F& f, double a, double b)
{
    constexpr int divmax = 6;
    const double rng = b - a;
    T ordsum = 0.5 * (f(a) + f(b));
    T prev[divmax + 1], row[divmax + 1];
    prev[0] = rng * ordsum;
    int n = 1;
    T buf[32];
    for (int i = 1; i <= divmax; ++i) {
        n *= 2;
        const int ntosum = n / 2;
        const double h = rng / ntosum;
        for (int j = 0; j < ntosum; ++j) buf[j] = f(a + 0.5 * h + h * (double)j);
        ordsum = ordsum + pairwise_sum(buf, ntosum);
        row[0] = rng * ordsum / (double)n;
        double p = 1.0;
        for (int k = 1; k <= i; ++k) {
            p *= 4.0;
            row[k] = (p * row[k - 1] - prev[k - 1]) / (p - 1.0);
        }
        for (int k = 0; k <= i; ++k) prev[k] = row[k];
    }
    return prev[divmax];
}

// numpy.geomspace(start, stop, num, endpoint): 10 ** linspace(log10 start, log10 stop), with the
// first (and with endpoint the last) point set to the arguments exactly.
BGF void geomspace(double start, double stop, int num, bool endpoint, double* out)
{
    const double ls = log10(start), le = log10(stop);
    const int div = endpoint ? num - 1 : num;
    const double step = (le - ls) / (double)div;
    for (int i = 0; i < num; ++i) out[i] = pow(10.0, (double)i * step + ls);
    if (endpoint && num > 1) out[num - 1] = stop;
    out[0] = start;
}

// ---------------------------------------------------------------------------------------------
// Cosmology.  Parameters that carry a derivative are of type T.
template <class T> struct Params {
    T H0, Omegab, Omegam, mnu, w0, wa;
    double Tcmb, YHe, Neff, Nmnu, cs2_DE, Omegak;
};

constexpr int kNuKnots = 512;   // massive-neutrino table knots (background.py:156)
constexpr int kNuQuad = 8;      // momentum quadrature points of the background integrals
constexpr double kAmin = 1e-9, kAmax = 1.01;  // background.py:206

template <class T> struct Bg {
    Params<T> p;
    T grhom;
    double grhog, grhor, adotrad;
    T amnu, Omegamnu, OmegaDE;
    double taumin;
    T taumax;
    double fHe;
    Spline<T> lrho;  // log rho_nu(log a), uniform knots
};

// rho_Q(a) / rho_Q(1) of the w0-wa fluid (background.py:71-72)
template <class T, class A> BGF T rho_Q(const A& a, const Params<T>& p)
{
    const T e = -3.0 * (1.0 + p.w0 + p.wa);
    return bpow2(a, e) * bexp(3.0 * (a - 1.0) * p.wa);
}

template <class T> BGF T rhonu_of(const Bg<T>& g, double a) { return bexp(spline_eval(g.lrho, blog(a))); }


// conformal Hubble rate a'/a in 1/Mpc (background.py:101-123)
template <class T> BGF T aprimeoa(const Bg<T>& g, double a)
{
    const Params<T>& p = g.p;
    const T rhonu = rhonu_of(g, a);
    const T grho = g.grhom * p.Omegam / a + (g.grhog + g.grhor * (p.Neff + p.Nmnu * rhonu)) / (a * a)
                   + g.grhom * g.OmegaDE * rho_Q(a, p) * (a * a) + g.grhom * p.Omegak;
    return bsqrt(grho / 3.0);
}

// da/dtau (background.py:84-93)
template <class T> BGF T dadtau(const Bg<T>& g, double a)
{
    const Params<T>& p = g.p;
    const T rhonu = rhonu_of(g, a);
    const T grho2 = g.grhom * p.Omegam * a + (g.grhog + g.grhor * (p.Neff + p.Nmnu * rhonu))
                    + g.grhom * g.OmegaDE * rho_Q(a, p) * pow(a, 4.0) + g.grhom * p.Omegak * (a * a);
    return bsqrt(grho2 / 3.0);
}
template <class T> BGF T dtauda(const Bg<T>& g, double a) { return 1.0 / dadtau(g, a); }

// Momentum quadrature of the background neutrino integrals: the 8-point generalised
// Gauss-Laguerre rule (alpha = 1) with the weights of background.py:34-45
// (w q^3 / (1 + e^-q) q^-1, over 7 pi^4 / 120), as numpy's Golub-Welsch solve gives them.
BGF double nu_quad_q(int i)
{
    constexpr double q[kNuQuad] = {0.4093835732031853, 1.3849631848031398, 2.956254556168862,
                                   5.181943101040074, 8.161709688145818, 12.070055126837152,
                                   17.249735526149, 24.585955243652784};
    return q[i];
}
BGF double nu_quad_w(int i)
{
    constexpr double w[kNuQuad] = {0.003325706033494454, 0.11851805400577503, 0.42397302528642805,
                                   0.35311449652949917, 0.09296943503649908, 0.007913251189502262,
                                   0.00017537121510859883, 5.022593429551112e-07};
    return w[i];
}

// rho_nu / rho_nu0, p_nu / p_nu0 and the pseudo-pressure of one massive flavour (background.py:48-69)
template <class T> BGF void nu_background(double a, const T& amnu, T& rho, T& p, T& pp)
{
    T tr[kNuQuad], tp[kNuQuad], tq[kNuQuad];
    for (int i = 0; i < kNuQuad; ++i) {
        const double q = nu_quad_q(i), w = nu_quad_w(i);
        const T r = a * amnu / q;
        const T v = 1.0 / bsqrt(1.0 + r * r);
        tr[i] = w / v;
        tp[i] = w * v / 3.0;
        tq[i] = w * bpow(v, 3.0) / 3.0;
    }
    rho = pairwise_sum(tr, kNuQuad);
    p = pairwise_sum(tp, kNuQuad);
    pp = pairwise_sum(tq, kNuQuad);
}

// ---------------------------------------------------------------------------------------------
// Recfast model (replaces thermodynamics_recfast.py:124-281): d(x_H, x_He, T_mat)/da, one
// function per process, from Seager, Sasselov & Scott (1999, 2000) and Wong, Moss & Scott (2008).
// Y is the state's number type (T, or Fw<T> for the Jacobian); parameters of type T are lifted
// to Y.  Branches are taken on value parts.
template <class T> struct RecCtx {
    const Bg<T>* g;
    RecConst k;
};

// What the rate equations share at scale factor a: 1 + z, hydrogen and helium number densities
// [m^-3], radiation and matter temperatures [K], the Hubble rate [1/s] and the ionised fractions
// (x_e = x_H + f_He x_He electrons per hydrogen nucleus).
template <class Y> struct Plasma {
    double zp1, Tr, fHe;
    Y h, nH, nHe, Tm, Hs, xH, xHe, xe;
};

template <class Y, class T>
BGF Plasma<Y> plasma_at(double a, const Y* y, const Params<T>& P, const T& aprime_t)
{
    Plasma<Y> s;
    const double yhe = P.YHe;
    s.h = lift<Y>(P.H0) / 100.0;
    s.zp1 = 1.0 / a;
    s.fHe = yhe / (const_mHe_mH * (1.0 - yhe));
    // hydrogen nuclei per m^3: rho_b (1 - Y) / m_H, with rho_crit / m_H = const_dens_fac h^2
    s.nH = const_dens_fac * s.h * s.h * lift<Y>(P.Omegab) * (1.0 - yhe) * pow(s.zp1, 3.0);
    s.nHe = s.fHe * s.nH;
    s.Tr = P.Tcmb * s.zp1;
    s.Tm = re(y[2]) >= 0.0 ? y[2] : -y[2];
    // conformal a'/a [1/Mpc] -> H(z) [1/s]
    s.Hs = 1e-5 * lift<Y>(aprime_t) * s.zp1 * const_c * bigH;
    s.xH = y[0];
    s.xHe = y[1];
    s.xe = s.xH + s.fHe * s.xHe;
    return s;
}

// Sobolev escape probability (1 - e^-tau) / tau
template <class Y> BGF Y rec_escape(const Y& tau) { return (1.0 - bexp(-tau)) / tau; }

// Ratio of the rate at which H continuum absorption removes photons from a HeI line to the line's
// decay rate (Kholupenko, Ivanchik & Varshalovich 2007), with the line's Doppler width at T_m.
template <class Y>
BGF Y he_line_broadening(const Plasma<Y>& s, const RecConst& K, double wavenumber, double einstein_a, double sigma_abs)
{
    const double c2 = const_c * const_c;
    const Y vth = bsqrt(2.0 * const_kB * s.Tm / (const_mH * const_mHe_mH * c2));
    const Y doppler = const_c * wavenumber * vth;
    const double lc = const_c * wavenumber;
    return (3.0 * einstein_a * s.fHe * (1.0 - s.xHe) * c2) /
           (K.sqrt_pi * sigma_abs * 8.0 * kPi * doppler * (1.0 - s.xH) * (lc * lc));
}

// dx_H/dz: Peebles' effective three-level atom with the Recfast fudge F = 1.105 and the
// two-Gaussian correction of the Lyman-alpha escape rate.  Zero while x_H > 0.99, the rate
// without the Peebles factor for 0.985 < x_H <= 0.99.
template <class Y> BGF Y rec_hydrogen(const Plasma<Y>& s, const RecConst& K)
{
    const Y t4 = s.Tm / 1e4;
    // case-B recombination coefficient (Pequignot, Petitjean & Boisson 1991 fit) [m^3/s]
    const Y alpha_B = 1e-19 * K.a_PPB * bpow(t4, K.b_PPB) / (1.0 + K.c_PPB * bpow(t4, K.d_PPB));
    // photo-ionisation rate from n = 2, by detailed balance [1/s]
    const Y beta_B = alpha_B * bpow(K.CR * s.Tm, 1.5) * bexp(-K.CDB / s.Tm);
    const double lz = log(s.zp1);
    const double g1 = (lz - zGauss1) / wGauss1, g2 = (lz - zGauss2) / wGauss2;
    const double k_fix = 1.0 + AGauss1 * exp(-(g1 * g1)) + AGauss2 * exp(-(g2 * g2));
    const Y K_alpha = K.CK / s.Hs * k_fix;  // Lyman-alpha redshifting factor lambda^3 / (8 pi H)
    const Y n_1s = s.nH * (1.0 - s.xH);
    const Y net = (s.xe * s.xH * s.nH * alpha_B - beta_B * (1.0 - s.xH) * bexp(-K.CL / s.Tm)) / (s.Hs * s.zp1);
    if (re(s.xH) > 0.99) return 0.0 * s.xH;
    if (re(s.xH) > 0.985) return net;
    // Peebles factor, with the case-B coefficient divided by the fudge F
    const Y decay = 1.0 + K_alpha * Lambda_ * n_1s;
    return net * (decay / (decay / 1.105 + K_alpha * beta_B * n_1s));
}

// dx_He/dz through the HeI singlet 2^1P -> 1^1S channel: Verner & Ferland (1996) recombination fit,
// Sobolev escape plus H continuum absorption (p = 0.36, q = 0.86).
template <class Y> BGF Y rec_helium_singlet(const Plasma<Y>& s, const RecConst& K)
{
    const Y r0 = bsqrt(s.Tm / K.T_0), r1 = bsqrt(s.Tm / K.T_1);
    const Y alpha_He = K.a_VF / (r0 * bpow(1.0 + r0, 1.0 - K.b_VF) * bpow(1.0 + r1, 1.0 + K.b_VF));
    const Y beta_He = 4.0 * alpha_He * bpow(K.CR * s.Tm, 1.5) * bexp(-K.CDB_He / s.Tm);
    const Y n_HeI = s.nHe * (1.0 - s.xHe);
    const Y K_line = K.CK_He / s.Hs;
    const Y p_esc = rec_escape(A2P_s * K_line * 3.0 * n_HeI);
    const Y a_cont = A2P_s / (1.0 + 0.36 * bpow(he_line_broadening(s, K, L_He_2p, A2P_s, sigma_He_2Ps), 0.86));
    const bool ends = re(s.xHe) < 5e-9 || re(s.xHe) > 0.98;
    const Y esc_rate = re(s.xH) < 0.9999999 ? A2P_s * p_esc + a_cont : A2P_s * p_esc;
    const Y K_He = ends ? K_line : 1.0 / (esc_rate * 3.0 * n_HeI);
    const Y bt = K.Bfact / s.Tm;
    const Y boltz = bexp(re(bt) < 680.0 ? bt : Y(680.0));  // 2s-2p energy gap factor
    const Y net = (s.xe * s.xHe * s.nH * alpha_He - beta_He * (1.0 - s.xHe) * bexp(-K.CL_He / s.Tm)) / (s.Hs * s.zp1);
    const Y k_n = K_He * n_HeI * boltz;
    return net * (1.0 + k_n * Lambda_He) / (1.0 + k_n * (Lambda_He + beta_He));
}

// dx_He/dz through the HeI triplet 2^3P -> 1^1S intercombination line (p = 0.66, q = 0.9); omitted
// at the ends of helium recombination.
template <class Y> BGF Y rec_helium_triplet(const Plasma<Y>& s, const RecConst& K)
{
    if (re(s.xHe) < 5e-9 || re(s.xHe) > 0.98) return 0.0 * s.xHe;
    const Y r0 = bsqrt(s.Tm / K.T_0), r1 = bsqrt(s.Tm / K.T_1);
    const Y alpha_t = K.a_trip / (r0 * bpow(1.0 + r0, 1.0 - K.b_trip) * bpow(1.0 + r1, 1.0 + K.b_trip));
    const Y beta_t = (4.0 / 3.0) * alpha_t * bexp((-const_h * const_c * L_He2St_ion) / (const_kB * s.Tm)) *
                     bpow(K.CR * s.Tm, 1.5);
    const Y n_HeI = s.nHe * (1.0 - s.xHe);
    const Y p_esc = rec_escape(A2P_t * n_HeI * 3.0 / (8.0 * kPi * s.Hs * pow(L_He_2Pt, 3.0)));
    const Y a_cont = A2P_t / (1.0 + 0.66 * bpow(he_line_broadening(s, K, L_He_2Pt, A2P_t, sigma_He_2Pt), 0.9)) / 3.0;
    const Y decay = (re(s.xH) > 0.99999 ? A2P_t * p_esc : A2P_t * p_esc + a_cont) * bexp(-K.CL_PSt / s.Tm);
    const Y c_trip = decay / (beta_t + decay);  // chance that an atom in 2^3P reaches the ground state
    const Y net = s.xe * s.xHe * s.nH * alpha_t - 3.0 * beta_t * (1.0 - s.xHe) * bexp(-K.hcL2St_kB / s.Tm);
    return net * c_trip / (s.Hs * s.zp1);
}

// dT_m/dz: Compton coupling against adiabatic cooling; T_m follows T_rad while the Compton time
// is below 1e-3 of the Hubble time.
template <class Y> BGF Y rec_temperature(const Plasma<Y>& s, const RecConst& K)
{
    const Y heat = K.CT * pow(s.Tr, 4.0) * s.xe / (1.0 + s.xe + s.fHe);  // inverse Compton time [1/s]
    const Y t_hubble = 2.0 / (3.0 * s.h * bigH * pow(s.zp1, 1.5));
    if (re(1.0 / heat) < H_frac * re(t_hubble)) return s.Tm / s.zp1;
    return heat * (s.Tm - s.Tr) / (s.Hs * s.zp1) + 2.0 * s.Tm / s.zp1;
}

template <class Y, class T>
BGF void ionization(double a, const Y* y, const RecCtx<T>& c, const T& aprime_t, Y* f)
{
    const Plasma<Y> s = plasma_at(a, y, c.g->p, aprime_t);
    const Y dxH = rec_hydrogen(s, c.k);
    const Y dxHe = re(s.xHe) < 1e-8 ? 0.0 * s.xHe : rec_helium_singlet(s, c.k) + rec_helium_triplet(s, c.k);
    const Y dTm = rec_temperature(s, c.k);
    const double dzda = -1.0 / (a * a);
    f[0] = dxH * dzda;
    f[1] = dxHe * dzda;
    f[2] = dTm * dzda;
}

// Kaps & Rentrop (1979) GRK4A (ode_integrators_stiff.py:157-254): all stages at t0, as the
// reference.  The Jacobian d(dt f)/dy is taken in forward mode, one column per pass.
struct Grk4a {
    static constexpr double gamma = 0.395, gamma21 = -0.767672395484, gamma31 = -0.851675323742,
                            gamma32 = 0.522967289188, gamma41 = 0.288463109545, gamma42 = 0.880214273381e-1,
                            gamma43 = -0.337389840627, alpha21 = 0.438, alpha31 = 0.796920457938,
                            alpha32 = 0.730795420615e-1, chat1 = 0.346325833758, chat2 = 0.285693175712,
                            chat3 = 0.367980990530, c1 = 0.199293275701, c2 = 0.482645235674,
                            c3 = 0.680614886256e-1, c4 = 0.25;
};

template <class T> BGF void rec_rhs(const RecCtx<T>& c, double t, const T* y, T* f)
{
    const T ap = aprimeoa(*c.g, t);
    ionization<T, T>(t, y, c, ap, f);
}

template <class T> BGF void lu3_solve(const T* L, const T* b, T* x)
{
    // L = (u00, u01, u02, l10, u11, u12, l20, l21, u22), no pivoting (ode_integrators_stiff.py:77-96)
    const T y0 = b[0];
    const T y1 = b[1] - L[3] * y0;
    const T y2 = b[2] - L[6] * y0 - L[7] * y1;
    x[2] = y2 / L[8];
    x[1] = (y1 - L[5] * x[2]) / L[4];
    x[0] = (y0 - L[1] * x[1] - L[2] * x[2]) / L[0];
}

template <class T> BGF void mat3_vec(const T* J, const T* k, T* r)
{
    for (int i = 0; i < 3; ++i) r[i] = J[3 * i] * k[0] + J[3 * i + 1] * k[1] + J[3 * i + 2] * k[2];
}

template <class T> BGF void grk4a_step(const RecCtx<T>& c, double t0, double t1, const T* y0, T* ynew, T* yerr)
{
    using G = Grk4a;
    using FT = Fw<T>;
    const double dt = t1 - t0;
    const T ap = aprimeoa(*c.g, t0);
    T J[9];
    for (int j = 0; j < 3; ++j) {
        FT yy[3], ff[3];
        for (int i = 0; i < 3; ++i) yy[i] = FT(y0[i], T(i == j ? 1.0 : 0.0));
        ionization<FT, T>(t0, yy, c, ap, ff);
        for (int i = 0; i < 3; ++i) J[3 * i + j] = ff[i].d * dt;
    }
    T A[9];
    for (int i = 0; i < 9; ++i) A[i] = ((i % 4) == 0 ? T(1.0) : T(0.0)) - G::gamma * J[i];
    T L[9];
    L[0] = A[0]; L[1] = A[1]; L[2] = A[2];
    L[3] = A[3] / L[0];
    L[4] = A[4] - L[3] * L[1];
    L[5] = A[5] - L[3] * L[2];
    L[6] = A[6] / L[0];
    const T r21 = A[7] - L[6] * L[1];
    const T r22 = A[8] - L[6] * L[2];
    L[7] = r21 / L[4];
    L[8] = r22 - L[7] * L[5];

    T f[3], b[3], k1[3], k2[3], k3[3], k4[3], yv[3], Jk1[3], Jk2[3], Jk3[3];
    ionization<T, T>(t0, y0, c, ap, f);
    for (int i = 0; i < 3; ++i) b[i] = dt * f[i];
    lu3_solve(L, b, k1);
    for (int i = 0; i < 3; ++i) yv[i] = y0[i] + G::alpha21 * k1[i];
    ionization<T, T>(t0, yv, c, ap, f);
    mat3_vec(J, k1, Jk1);
    for (int i = 0; i < 3; ++i) b[i] = dt * f[i] + G::gamma21 * Jk1[i];
    lu3_solve(L, b, k2);
    for (int i = 0; i < 3; ++i) yv[i] = y0[i] + G::alpha31 * k1[i] + G::alpha32 * k2[i];
    ionization<T, T>(t0, yv, c, ap, f);
    T f2[3];
    for (int i = 0; i < 3; ++i) f2[i] = dt * f[i];
    mat3_vec(J, k2, Jk2);
    for (int i = 0; i < 3; ++i) b[i] = f2[i] + G::gamma31 * Jk1[i] + G::gamma32 * Jk2[i];
    lu3_solve(L, b, k3);
    mat3_vec(J, k3, Jk3);
    for (int i = 0; i < 3; ++i) b[i] = f2[i] + G::gamma41 * Jk1[i] + G::gamma42 * Jk2[i] + G::gamma43 * Jk3[i];
    lu3_solve(L, b, k4);
    const double e1 = G::c1 - G::chat1, e2 = G::c2 - G::chat2, e3 = G::c3 - G::chat3;
    for (int i = 0; i < 3; ++i) {
        ynew[i] = y0[i] + G::c1 * k1[i] + G::c2 * k2[i] + G::c3 * k3[i] + G::c4 * k4[i];
        yerr[i] = e1 * k1[i] + e2 * k2[i] + e3 * k3[i] + G::c4 * k4[i];
    }
}

BGF double clip_to_end(double tprev, double tnext, double t1, bool keep)
{
    const double tol = 1e-10 * fabs(tnext);
    if (tnext > t1 - tol) return keep ? t1 : tprev + 0.5 * (t1 - tprev);
    return tnext;
}

// Adaptive GRK4A solve with diffrax's integral controller defaults (thermodynamics_recfast.py:
// 283-301 via diffrax PIDController: safety 0.9, factor in [0.2, 10], RMS norm, order 3),
// max_steps attempts, the last accepted state returned when they run out (throw=False).
// Returns the number of accepted steps.
template <class T>
BGF int solve_grk4a(const RecCtx<T>& c, double t0, double t1, T* y, double dt0, double rtol, double atol, int max_steps)
{
    double t = t0;
    double tn = clip_to_end(t0, t0 + dt0, t1, true);
    int accepted = 0;
    for (int it = 0; it < max_steps; ++it) {
        if (!(t < t1)) break;
        T y1[3], ye[3];
        grk4a_step(c, t, tn, y, y1, ye);
        double ss = 0.0;
        for (int i = 0; i < 3; ++i) {
            const double sc = re(ye[i]) / (atol + rtol * fmax(fabs(re(y[i])), fabs(re(y1[i]))));
            ss += sc * sc;
        }
        const double err = sqrt(ss / 3.0);
        const bool keep = err < 1.0;
        const double inv = err > 0.0 ? 1.0 / err : INFINITY;
        double factor = inv < INFINITY ? 0.9 * pow(inv, 1.0 / 3.0) : 10.0;
        const double fmin = keep ? 1.0 : 0.2;
        factor = fmin > factor ? fmin : factor;
        factor = factor < 10.0 ? factor : 10.0;
        const double dt = (tn - t) * factor;
        if (keep) {
            t = tn;
            for (int i = 0; i < 3; ++i) y[i] = y1[i];
            ++accepted;
        }
        tn = clip_to_end(t, t + dt, t1, keep);
    }
    return accepted;
}

// Saha HeII electron fraction (thermodynamics_recfast.py:303-322) at scale factor a of type A
template <class A, class T> BGF A saha_HeII(const A& a, const Params<T>& P, double fHe)
{
    const double const_Hfac = 1.0 / (1.0e06 * 3.0856775807e13);
    const double mu_H = 1.0 / (1.0 - P.YHe);
    const A H0 = lift<A>(P.H0);
    const A hh = H0 * const_Hfac;
    const A rho_c = 3.0 * (hh * hh) / (8.0 * kPi * const_G);
    const A NH = rho_c * lift<A>(P.Omegab) / (const_mH * mu_H) / bpow(a, 3.0);
    const A Tt = P.Tcmb / a;
    const A betaE = const_EionHe12s / Tt;
    const double Aa = 1.0 + fHe, Bb = 1.0 + 2.0 * fHe;
    const A R = bpow(2.0 * kPi * const_me * const_kB / (const_h * const_h) * Tt, 1.5) / NH * bexp(-betaE);
    if (re(R) > 1e5) return fHe * (1.0 - Bb / R + (1.0 + 5.0 * fHe + 6.0 * (fHe * fHe)) / (R * R));
    const A Rm = R - Aa;
    return -Rm / 2.0 + bsqrt(Rm * Rm / 4.0 + R * Bb) - Aa;
}

// The four geometric segments of the Recfast a-grid (thermodynamics_recfast.py:325-361).
BGF void adaptive_sampling(double a0, double a1, int N, double* out)
{
    const int n_very_early = (int)(N * 0.05) > 8 ? (int)(N * 0.05) : 8;
    const int n_pre = (int)(N * 0.10) > 8 ? (int)(N * 0.10) : 8;
    const int n_rec = (int)(N * 0.50);
    const int n_post = N - n_very_early - n_pre - n_rec;
    const double ab1 = fmax(1.0 / (1.0 + 10000), a0);
    const double ab2 = 1.0 / (1.0 + 1400);
    const double ab3 = 1.0 / (1.0 + 600);
    geomspace(a0, ab1, n_very_early, false, out);
    geomspace(ab1, ab2, n_pre, false, out + n_very_early);
    geomspace(ab2, ab3, n_rec, false, out + n_very_early + n_pre);
    geomspace(ab3, a1, n_post, true, out + n_very_early + n_pre + n_rec);
}

// ---------------------------------------------------------------------------------------------
// evolve_background (background.py:191-345) of one cosmology.
//   scal [DISCOEB_BGS_COUNT], nu [DISCOEB_BGN_COUNT * DISCOEB_NU_KNOTS], th [DISCOEB_BGT_COUNT * N]
//   work: bg_work_count(N) numbers of type T; agrid: N + 1 doubles
BGF int bg_work_count(int N) { return 2 * (N > DISCOEB_NU_KNOTS ? N : DISCOEB_NU_KNOTS) + 6 * N; }

template <class T>
BGF void evolve_background_core(const Params<T>& P, int N, T* scal, T* nu, T* th, T* work, double* agrid)
{
    constexpr int NK = DISCOEB_NU_KNOTS;
    const int NS = N > NK ? N : NK;
    T* cp = work;
    T* dp = work + NS;
    T* dxHda = work + 2 * NS;
    T* dxHeda = dxHda + N;
    T* dTmda = dxHeda + N;
    T* opd1 = dTmda + N;
    T* opd2 = opd1 + N;
    T* icum = opd2 + N;
    auto NU = [&](int slot) { return nu + (size_t)slot * NK; };
    auto TH = [&](int slot) { return th + (size_t)slot * N; };

    // ---- densities and massive-neutrino tables (background.py:141-189)
    Bg<T> g;
    g.p = P;
    const double amin = kAmin, amax = kAmax;
    g.grhom = 3.33795017e-11 * (P.H0 * P.H0);
    g.grhog = 1.49594245e-13 * pow(P.Tcmb, 4.0);
    g.grhor = 3.39739477e-14 * pow(P.Tcmb, 4.0);
    g.adotrad = sqrt((g.grhog + g.grhor * (P.Neff + P.Nmnu)) / 3.0);
    g.amnu = P.mnu * kC2ok / P.Tcmb;
    // log-a knots: numpy.geomspace(amin * 0.9, amax * 1.1, 512)
    const double nls = log10(amin * 0.9), nle = log10(amax * 1.1);
    const double nstep = (nle - nls) / (double)(NK - 1);
    for (int i = 0; i < NK; ++i) {
        double a = pow(10.0, (double)i * nstep + nls);
        if (i == 0) a = amin * 0.9;
        if (i == NK - 1) a = amax * 1.1;
        NU(DISCOEB_BGN_A)[i] = T(a);
        NU(DISCOEB_BGN_LOGA)[i] = T(log(a));
        T rho, pr, pp;
        nu_background(a, g.amnu, rho, pr, pp);
        NU(DISCOEB_BGN_LOGRHONU_Y)[i] = blog(rho);
        NU(DISCOEB_BGN_LOGPNU_Y)[i] = blog(pr);
        NU(DISCOEB_BGN_LOGPPNU_Y)[i] = blog(pp);
    }
    spline_build(NK, NU(DISCOEB_BGN_LOGA), NU(DISCOEB_BGN_LOGRHONU_Y), NU(DISCOEB_BGN_LOGRHONU_S), cp, dp);
    spline_build(NK, NU(DISCOEB_BGN_LOGA), NU(DISCOEB_BGN_LOGPNU_Y), NU(DISCOEB_BGN_LOGPNU_S), cp, dp);
    spline_build(NK, NU(DISCOEB_BGN_LOGA), NU(DISCOEB_BGN_LOGPPNU_Y), NU(DISCOEB_BGN_LOGPPNU_S), cp, dp);
    g.lrho = Spline<T>{NK, true, NU(DISCOEB_BGN_LOGA), NU(DISCOEB_BGN_LOGRHONU_Y), NU(DISCOEB_BGN_LOGRHONU_S), nullptr};
    const T rhonu0 = bexp(spline_eval(g.lrho, 0.0));
    g.Omegamnu = g.grhor * rhonu0 / g.grhom;
    const T Omegar = (P.Neff + P.Nmnu * rhonu0) * g.grhor / g.grhom;
    const T Omegag = g.grhog / g.grhom;
    g.OmegaDE = 1.0 - P.Omegak - Omegar - Omegag - P.Omegam;
    g.taumin = amin / g.adotrad;
    g.taumax = g.taumin + romb6<T>([&](double a) { return dtauda(g, a); }, amin, amax);

    // ---- Recfast history on the adaptive a-grid (thermodynamics_recfast.py:363-453)
    const double YHe = P.YHe, Tcmb = P.Tcmb;
    g.fHe = YHe / (const_mHe_mH * (1.0 - YHe));
    const double fHe = g.fHe;
    adaptive_sampling(amin, amax, N + 1, agrid);
    RecCtx<T> rc;
    rc.g = &g;
    rc.k = rec_const();
    const RecConst& K = rc.k;
    const T H = P.H0 / 100.0;
    const T HO = H * bigH;
    const double mu_H = 1.0 / (1.0 - YHe);
    const T Nnow = 3.0 * HO * HO * P.Omegab / (8.0 * kPi * const_G * mu_H * const_mH);
    const double Tcmb3 = pow(Tcmb, 3.0);
    T* xH = TH(DISCOEB_BGT_XEHI);
    T* xHe = TH(DISCOEB_BGT_XEHEI);
    T* Tm = TH(DISCOEB_BGT_TM);
    T* rcase = TH(DISCOEB_BGT_REC_CASE);
    T* rsteps = TH(DISCOEB_BGT_REC_STEPS);
    for (int i = 0; i < N; ++i) {
        const double astart = agrid[i], aend = agrid[i + 1];
        const double zstart = 1.0 / astart - 1.0, zend = 1.0 / aend - 1.0;
        const double dzda = -1.0 / (aend * aend);
        T yp[6];
        if (i > 0) {
            yp[0] = xH[i - 1]; yp[1] = xHe[i - 1]; yp[2] = Tm[i - 1];
            yp[3] = dxHda[i - 1]; yp[4] = dxHeda[i - 1]; yp[5] = dTmda[i - 1];
        } else {
            yp[0] = T(1.0); yp[1] = T(1.0); yp[2] = T(Tcmb * (1.0 + zstart));
            yp[3] = T(0.0); yp[4] = T(0.0); yp[5] = T(-Tcmb * (1.0 + zstart));
        }
        int cs = zend > 3500.0 ? 1 : ((i > 0 && re(yp[1]) > 0.99) ? 2 : ((i > 0 && re(yp[0]) > 0.99) ? 3 : 4));
        T nw[6];
        int steps = 0;
        const double zt = 1.0 + zend;
        if (cs == 1) {
            nw[0] = T(1.0); nw[1] = T(1.0); nw[2] = T(Tcmb * zt); nw[3] = T(0.0); nw[4] = T(0.0); nw[5] = T(-Tcmb * zt);
        } else if (cs == 2) {
            const T rhs = (bexp(1.5 * log(K.CR * Tcmb / zt) - K.CB1_He1 / (Tcmb * zt)) / Nnow) * 4.0;
            const T rm1 = rhs - 1.0;
            const T x_He0 = 0.5 * (bsqrt(rm1 * rm1 + 4.0 * (1.0 + fHe) * rhs) - rm1);
            const double q = -((K.CB1_He1 - K.CR * (Tcmb * Tcmb)) / (Tcmb * zt));
            const double q15 = pow(q, 1.5);
            const double cc = -K.CB1_He1 + K.CR * (Tcmb * Tcmb);
            const double cc3 = pow(cc, 3.0);
            const double zt3 = pow(zt, 3.0);
            const double qb = -((K.CB1_He1 - K.CR * (Tcmb * Tcmb)) / (Tcmb + Tcmb * zend));
            const T num = -3.0 * pow(-(K.CB1_He1 / Tcmb) + K.CR * Tcmb, 1.5) *
                          (Nnow + 2.0 * fHe * Nnow + 4.0 * q15 -
                           bsqrt(Nnow * Nnow + (16.0 * cc3) / (Tcmb3 * zt3) + 8.0 * (1.0 + 2.0 * fHe) * Nnow * q15));
            const T den = Nnow * pow(zt, 2.5) *
                          bsqrt(Nnow * Nnow + (16.0 * cc3) / (pow(Tcmb, 3.0) * zt3) +
                                8.0 * (1.0 + 2.0 * fHe) * Nnow * pow(qb, 1.5));
            const T dxHeIdz = num / den;
            nw[0] = T(1.0); nw[1] = (x_He0 - 1.0) / fHe; nw[2] = T(Tcmb * zt); nw[3] = T(0.0);
            nw[4] = dxHeIdz * dzda; nw[5] = T(-Tcmb * zt);
        } else {
            T y3[3] = {yp[0], yp[1], yp[2]};
            steps = solve_grk4a(rc, astart, aend, y3, fabs(astart * 1e-3), 1e-3, 1e-6, 128);
            T dy[3];
            rec_rhs(rc, aend, y3, dy);
            nw[0] = y3[0]; nw[1] = y3[1]; nw[2] = y3[2]; nw[3] = dy[0]; nw[4] = dy[1]; nw[5] = dy[2];
            if (cs == 3) {
                const T rhs = bexp(1.5 * log(K.CR * Tcmb / zt) - K.CB1 / (Tcmb * zt)) / Nnow;
                const T x_H0 = 0.5 * (bsqrt(rhs * rhs + 4.0 * rhs) - rhs);
                const double q = -((K.CB1 - K.CR * (Tcmb * Tcmb)) / (Tcmb * zt));
                const double Tc2 = Tcmb * Tcmb;
                const double CB1 = K.CB1, CR = K.CR;
                const T sq = Nnow * (zt * zt) * sqrt(q);
                const T inner1 = 2.0 * (CB1 * CB1) - 4.0 * CB1 * CR * Tc2 + Tc2 * (2.0 * (CR * CR) * Tc2 + sq);
                const T inner2 = (CB1 * CB1) - 2.0 * CB1 * CR * Tc2 + Tc2 * ((CR * CR) * Tc2 + sq);
                const T dxHdz = (3.0 * ((2.0 * pow(q, 1.5)) / zt +
                                        ((CB1 - CR * Tc2) * inner1) /
                                            (pow(Tcmb, 1.5) * pow(zt, 2.5) * bsqrt((-CB1 + CR * Tc2) * inner2)))) /
                                (2.0 * Nnow);
                nw[0] = x_H0;
                nw[3] = dxHdz * dzda;
            }
        }
        xH[i] = nw[0]; xHe[i] = nw[1]; Tm[i] = nw[2];
        dxHda[i] = nw[3]; dxHeda[i] = nw[4]; dTmda[i] = nw[5];
        rcase[i] = T((double)cs);
        rsteps[i] = T((double)steps);
    }

    // ---- thermal tables (thermodynamics_recfast.py:456-492)
    T* aexp = TH(DISCOEB_BGT_AEXP);
    T* tau = TH(DISCOEB_BGT_TAU);
    T* xe = TH(DISCOEB_BGT_XE);
    T* xeHeII = TH(DISCOEB_BGT_XEHEII);
    T* mu = TH(DISCOEB_BGT_MU);
    T* cs2 = TH(DISCOEB_BGT_CS2);
    T* dxedtau = TH(DISCOEB_BGT_XEPRIME_RECF);
    for (int i = 0; i < N; ++i) {
        const double a = agrid[i + 1];
        aexp[i] = T(a);
        TH(DISCOEB_BGT_LOGA)[i] = T(log(a));
        xeHeII[i] = saha_HeII(T(a), P, fHe);
        using FT = Fw<T>;
        const T dHeII = saha_HeII(FT(T(a), T(1.0)), P, fHe).d;
        xe[i] = xH[i] + fHe * xHe[i] + xeHeII[i];
        mu[i] = 1.0 / (1.0 + (1.0 / const_mHe_mH - 1.0) * YHe + (1.0 - YHe) * xe[i]);
        const T daTmda = Tm[i] + a * dTmda[i];
        cs2[i] = const_kB / const_mH / (const_c * const_c) / mu[i] * Tm[i] * (4.0 - daTmda / Tm[i]) / 3.0;
        dxedtau[i] = (dxHda[i] + fHe * dxHeda[i] + dHeII) * dadtau(g, a);
        TH(DISCOEB_BGT_CS2A)[i] = a * cs2[i];
        TH(DISCOEB_BGT_TEMPBA)[i] = a * Tm[i];
    }
    {
        T acc = T(0.0);
        tau[0] = g.taumin + 0.0;
        for (int i = 1; i < N; ++i) {
            acc += romb6<T>([&](double a) { return dtauda(g, a); }, agrid[i], agrid[i + 1]);
            tau[i] = g.taumin + acc;
        }
    }

    // ---- splines and visibility (background.py:316-345)
    spline_build(N, aexp, tau, TH(DISCOEB_BGT_TAU_OF_A_S), cp, dp);
    spline_build(N, tau, aexp, TH(DISCOEB_BGT_A_OF_TAU_S), cp, dp);
    spline_build(N, tau, xe, TH(DISCOEB_BGT_XE_OF_TAU_S), cp, dp);
    spline_build(N, tau, TH(DISCOEB_BGT_CS2A), TH(DISCOEB_BGT_CS2A_OF_TAU_S), cp, dp);
    spline_build(N, tau, TH(DISCOEB_BGT_TEMPBA), TH(DISCOEB_BGT_TEMPBA_OF_TAU_S), cp, dp);
    spline_build(N, TH(DISCOEB_BGT_LOGA), xe, TH(DISCOEB_BGT_XE_OF_LOGA_S), cp, dp);
    spline_build(N, TH(DISCOEB_BGT_LOGA), TH(DISCOEB_BGT_CS2A), TH(DISCOEB_BGT_CS2A_OF_LOGA_S), cp, dp);
    const Spline<T> tau_of_a{N, false, aexp, tau, TH(DISCOEB_BGT_TAU_OF_A_S), nullptr};
    const Spline<T> xe_of_tau{N, false, tau, xe, TH(DISCOEB_BGT_XE_OF_TAU_S), nullptr};
    const T akthom = kAkthom * (1.0 - YHe) * P.Omegab * (P.H0 * P.H0);
    const T tau_pre = spline_eval(tau_of_a, 1e-4);
    const double xe_full = 1.0 + YHe / (1.0 - YHe);
    T* opac = TH(DISCOEB_BGT_OPAC);
    T* xeprime = TH(DISCOEB_BGT_XEPRIME);
    for (int i = 0; i < N; ++i) {
        const bool early = re(tau[i]) <= re(tau_pre);
        T d1, d2;
        spline_d12(xe_of_tau, tau[i], d1, d2);
        const T xv = early ? T(xe_full) : spline_eval(xe_of_tau, tau[i]);
        xeprime[i] = early ? T(0.0) : d1;
        opac[i] = xv * akthom / (aexp[i] * aexp[i]);
    }
    spline_build(N, tau, opac, TH(DISCOEB_BGT_OPAC_S), cp, dp);
    spline_integrals(N, tau, opac, TH(DISCOEB_BGT_OPAC_S), icum);
    const Spline<T> ops{N, false, tau, opac, TH(DISCOEB_BGT_OPAC_S), icum};
    const T tau0 = spline_eval(tau_of_a, 1.0);
    const T od_today = spline_integral(ops, tau0);
    int imax = 0;
    for (int i = 0; i < N; ++i) {
        spline_d12(ops, tau[i], opd1[i], opd2[i]);
        const T od = od_today - spline_integral(ops, tau[i]);
        TH(DISCOEB_BGT_OPTICAL_DEPTH)[i] = od;
        const T expmmu = bexp(-od);
        TH(DISCOEB_BGT_GVIS)[i] = opac[i] * expmmu;
        TH(DISCOEB_BGT_GVISPRIME)[i] = (opd1[i] + opac[i] * opac[i]) * expmmu;
        TH(DISCOEB_BGT_GVISPPRIME)[i] = (opd2[i] + 3.0 * opac[i] * opd1[i] + bpow(opac[i], 3.0)) * expmmu;
        if (re(TH(DISCOEB_BGT_GVIS)[i]) > re(TH(DISCOEB_BGT_GVIS)[imax])) imax = i;
    }

    scal[DISCOEB_BGS_AMIN] = T(amin);
    scal[DISCOEB_BGS_AMAX] = T(amax);
    scal[DISCOEB_BGS_GRHOM] = g.grhom;
    scal[DISCOEB_BGS_GRHOG] = T(g.grhog);
    scal[DISCOEB_BGS_GRHOR] = T(g.grhor);
    scal[DISCOEB_BGS_ADOTRAD] = T(g.adotrad);
    scal[DISCOEB_BGS_AMNU] = g.amnu;
    scal[DISCOEB_BGS_OMEGAMNU] = g.Omegamnu;
    scal[DISCOEB_BGS_OMEGADE] = g.OmegaDE;
    scal[DISCOEB_BGS_TAUMIN] = T(g.taumin);
    scal[DISCOEB_BGS_TAUMAX] = g.taumax;
    scal[DISCOEB_BGS_FHE] = T(g.fHe);
    scal[DISCOEB_BGS_TAU0] = tau0;
    scal[DISCOEB_BGS_TAU_MAXVIS] = tau[imax];
    scal[DISCOEB_BGS_H0] = P.H0;
    scal[DISCOEB_BGS_OMEGAB] = P.Omegab;
    scal[DISCOEB_BGS_OMEGAM] = P.Omegam;
    scal[DISCOEB_BGS_MNU] = P.mnu;
    scal[DISCOEB_BGS_W0] = P.w0;
    scal[DISCOEB_BGS_WA] = P.wa;
}

}  // namespace bgn
}  // namespace dscb
