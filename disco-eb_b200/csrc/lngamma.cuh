// Complex log Gamma on the device, shared by the FFTLog kernels (line of sight and correlation
// functions): the Lanczos approximation the reference uses (util.py:13-45), with a reflection for
// Re z <= 0.5 whose log sin(pi z) stays finite for large |Im z|.
#pragma once

#include <cmath>

// host and device (the host build is the CPU test harness of these formulas)
#if defined(__CUDACC__)
#define LGF __host__ __device__ inline
#else
#define LGF inline
#endif

namespace dscb {
namespace cplx {

struct Cx {
    double re, im;
};
LGF Cx cx(double r, double i) { return Cx{r, i}; }
LGF Cx operator+(Cx a, Cx b) { return cx(a.re + b.re, a.im + b.im); }
LGF Cx operator-(Cx a, Cx b) { return cx(a.re - b.re, a.im - b.im); }
LGF Cx operator*(Cx a, Cx b) { return cx(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re); }
LGF Cx cx_log(Cx z) { return cx(log(hypot(z.re, z.im)), atan2(z.im, z.re)); }

// log Gamma(z) for Re z > 0.5: Lanczos g = 7 with 9 terms (Lanczos, SIAM J. Numer. Anal. B 1
// (1964) 86; the coefficient set of util.py:26-36)
LGF Cx lngamma_lanczos(Cx z)
{
    const double c[9] = {0.99999999999980993227684700473478, 676.520368121885098567009190444019,
                         -1259.13921672240287047156078755283, 771.3234287776530788486528258894,
                         -176.61502916214059906584551354, 12.507343278686904814458936853,
                         -0.13857109526572011689554707, 9.984369578019570859563e-6, 1.50563273514931155834e-7};
    z = cx(z.re - 1.0, z.im);
    Cx A = cx(c[0], 0.0);
    for (int j = 1; j < 9; ++j) {
        const double re = z.re + j, im = z.im;
        const double s = c[j] / (re * re + im * im);
        A = A + cx(s * re, -s * im);
    }
    const Cx zh = cx(z.re + 0.5, z.im), zg = cx(z.re + 7.5, z.im);
    return zh * cx_log(zg) - zg + cx(0.9189385332046727418, 0.0) + cx_log(A);
}

// log sin(pi z), stable for large |Im z| (sin(pi z) = (e^{i pi z} - e^{-i pi z}) / 2i)
LGF Cx log_sin_pi(Cx z)
{
    const double x = M_PI * z.re, y = M_PI * z.im;
    if (fabs(y) < 20.0) {
        double sx, cxv;
        sincos(x, &sx, &cxv);
        return cx_log(cx(sx * cosh(y), cxv * sinh(y)));
    }
    // Where sin(x) cosh(y) or cos(x) sinh(y) exceeds DBL_MAX the reference's complex sin
    // overflows to infinity, its log is +inf, and the coefficient it feeds comes out as exactly
    // zero: keep that behaviour (709.782712893384 = ln DBL_MAX).
    {
        double sx, cxv;
        sincos(x, &sx, &cxv);
        if (fabs(y) - M_LN2 + log(fmax(fabs(sx), fabs(cxv))) > 709.782712893384) return cx(INFINITY, 0.0);
    }
    // |y| large: sin(pi z) = (i s / 2) e^{|y|} e^{-i s x} (1 - e^{-2|y|} e^{2 i s x}), s = sign(y)
    const double s = y > 0 ? 1.0 : -1.0, ay = fabs(y);
    double sn, cs;
    sincos(2.0 * s * x, &sn, &cs);
    const double e = exp(-2.0 * ay);
    const Cx corr = cx_log(cx(1.0 - e * cs, -e * sn));
    // log of the prefactor: log(i s / 2) = -log 2 + i s pi/2
    return cx(ay - M_LN2, -s * x + s * M_PI_2) + corr;
}

LGF Cx lngamma_c(Cx z)
{
    if (z.re <= 0.5) {  // reflection
        const Cx l = lngamma_lanczos(cx(1.0 - z.re, -z.im));
        const Cx ls = log_sin_pi(z);
        return cx(1.14472988584940017414342735135, 0.0) - ls - l;
    }
    return lngamma_lanczos(z);
}

LGF Cx operator/(Cx a, Cx b)
{
    const double d = b.re * b.re + b.im * b.im;
    return cx((a.re * b.re + a.im * b.im) / d, (a.im * b.re - a.re * b.im) / d);
}

// d/dz of lngamma_lanczos: the exact derivative of the same formula,
// ln(z' + 7.5) + (z' + 0.5) / (z' + 7.5) - 1 + A'(z') / A(z'), z' = z - 1
LGF Cx digamma_lanczos(Cx z)
{
    const double c[9] = {0.99999999999980993227684700473478, 676.520368121885098567009190444019,
                         -1259.13921672240287047156078755283, 771.3234287776530788486528258894,
                         -176.61502916214059906584551354, 12.507343278686904814458936853,
                         -0.13857109526572011689554707, 9.984369578019570859563e-6, 1.50563273514931155834e-7};
    z = cx(z.re - 1.0, z.im);
    Cx A = cx(c[0], 0.0), dA = cx(0.0, 0.0);
    for (int j = 1; j < 9; ++j) {
        const Cx inv = cx(1.0, 0.0) / cx(z.re + j, z.im);
        A = A + cx(c[j] * inv.re, c[j] * inv.im);
        const Cx inv2 = inv * inv;
        dA = dA - cx(c[j] * inv2.re, c[j] * inv2.im);
    }
    const Cx zh = cx(z.re + 0.5, z.im), zg = cx(z.re + 7.5, z.im);
    return cx_log(zg) + zh / zg - cx(1.0, 0.0) + dA / A;
}

// pi cot(pi z), stable for large |Im z|: i pi (E + 1) / (E - 1) with E = exp(2 i pi z) when
// Im z > 0, i pi (1 + E') / (1 - E') with E' = exp(-2 i pi z) otherwise (|E|, |E'| <= 1)
LGF Cx pi_cot_pi(Cx z)
{
    const double s = z.im > 0 ? 1.0 : -1.0;
    const double mag = exp(-2.0 * M_PI * fabs(z.im));
    double sn, cs;
    sincos(2.0 * M_PI * s * z.re, &sn, &cs);
    const Cx E = cx(mag * cs, mag * sn);
    const Cx q = (z.im > 0) ? (E + cx(1.0, 0.0)) / (E - cx(1.0, 0.0)) : (cx(1.0, 0.0) + E) / (cx(1.0, 0.0) - E);
    return cx(-M_PI * q.im, M_PI * q.re);
}

// digamma: the derivative of lngamma_c, branch for branch (reflection for Re z <= 0.5:
// d/dz [ln pi - ln sin(pi z) - lnGamma(1 - z)] = -pi cot(pi z) + psi(1 - z))
LGF Cx digamma_c(Cx z)
{
    if (z.re <= 0.5) return digamma_lanczos(cx(1.0 - z.re, -z.im)) - pi_cot_pi(z);
    return digamma_lanczos(z);
}

// One FFTLog kernel coefficient M_l(p), p = bias + i eta, eta = 2 pi q / (n_fft dl), as the pair
// (Re M, -Im M) that the frequency sum reads, and its derivative along a change dl_dot of the
// grid spacing (p moves by i eta_dot, eta_dot = -eta dl_dot / dl):
// ln M = (p - 1) ln 2 + ln(pi)/2 + lnGamma((1 + l + p)/2) - lnGamma((2 + l - p)/2)
// (cmb.py:636-677); d ln M / dp = ln 2 + psi((1 + l + p)/2)/2 + psi((2 + l - p)/2)/2.  Where the
// reference's log-Gamma overflows the coefficient is exactly zero, and so is its derivative.
LGF void fftlog_mcoef(int l, int q, int n_fft, double bias, double dl, double dl_dot, double* b, double* b_dot,
                      Cx* dlc_out = nullptr)
{
    const double eta = 2.0 * M_PI * q / (n_fft * dl);
    const Cx p = cx(bias, eta);
    const Cx a1 = cx((1.0 + l + p.re) / 2.0, p.im / 2.0), a2 = cx((2.0 + l - p.re) / 2.0, -p.im / 2.0);
    const Cx lc = cx((p.re - 1.0) * M_LN2 + 0.5 * log(M_PI), p.im * M_LN2) + lngamma_c(a1) - lngamma_c(a2);
    if (lc.re == -INFINITY) {
        b[0] = b[1] = 0.0;
        if (b_dot) b_dot[0] = b_dot[1] = 0.0;
        if (dlc_out) *dlc_out = cx(0.0, 0.0);
        return;
    }
    const double mag = exp(lc.re);
    double sn, cs;
    sincos(lc.im, &sn, &cs);
    b[0] = mag * cs;
    b[1] = -mag * sn;
    if (!b_dot) return;
    const Cx half = cx(0.5, 0.0);
    const Cx dlc = cx(M_LN2, 0.0) + half * digamma_c(a1) + half * digamma_c(a2);
    if (dlc_out) *dlc_out = dlc;
    const double eta_dot = -eta * dl_dot / dl;
    const Cx Mdot = cx(mag * cs, mag * sn) * dlc * cx(0.0, eta_dot);
    b_dot[0] = Mdot.re;
    b_dot[1] = -Mdot.im;
}

// fftlog_mcoef for l = l0, l0 + 2, ..., l0 + 2 (count - 1) at one frequency: log-Gamma at l0 only,
// then M_{l+2}(p) = M_l(p) (1 + l + p) / (2 + l - p) (Gamma(z + 1) = z Gamma(z) in both factors) and,
// for the tangent, d ln M / dp advanced by psi(z + 1) = psi(z) + 1/z in both digammas.  Output i at
// b + i * step and b_dot + i * step (either may be null); each step adds a few roundings, so a run
// of 16 stays within ~1e-14 of the direct evaluation.  For l0 >= 2 (l = 0, 1 take the reflection
// branch of the log-Gamma, whose overflow at large eta gives M = 0 there and only there).
LGF void fftlog_mcoef_run(int l0, int count, int q, int n_fft, double bias, double dl, double dl_dot, long long step,
                          double* b, double* b_dot)
{
    double b0[2], bd0[2];
    Cx dlc = cx(0.0, 0.0);
    fftlog_mcoef(l0, q, n_fft, bias, dl, dl_dot, b0, b_dot ? bd0 : nullptr, b_dot ? &dlc : nullptr);
    if (b) {
        b[0] = b0[0];
        b[1] = b0[1];
    }
    if (b_dot) {
        b_dot[0] = bd0[0];
        b_dot[1] = bd0[1];
    }
    const double eta = 2.0 * M_PI * q / (n_fft * dl);
    const double eta_dot = -eta * dl_dot / dl;
    Cx M = cx(b0[0], -b0[1]);
    for (int i = 1; i < count; ++i) {
        const int l = l0 + 2 * (i - 1);
        const double a = 1.0 + l + bias, c = 2.0 + l - bias;  // 2 a1 = a + i eta, 2 a2 = c - i eta
        const double da = a * a + eta * eta, dc = c * c + eta * eta;
        M = M * cx((a * c - eta * eta) / dc, eta * (a + c) / dc);
        if (b) {
            b[i * step] = M.re;
            b[i * step + 1] = -M.im;
        }
        if (b_dot) {
            dlc = dlc + cx(a / da + c / dc, eta / dc - eta / da);
            const Cx Md = M * dlc * cx(0.0, eta_dot);
            b_dot[i * step] = Md.re;
            b_dot[i * step + 1] = -Md.im;
        }
    }
}

}  // namespace cplx
}  // namespace dscb
