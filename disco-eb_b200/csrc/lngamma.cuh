// Complex log Gamma on the device, shared by the FFTLog kernels (line of sight and correlation
// functions): the Lanczos approximation the reference uses (util.py:13-45), with a reflection for
// Re z <= 0.5 whose log sin(pi z) stays finite for large |Im z|.
#pragma once

#include <cmath>

namespace dscb {
namespace cplx {

struct Cx {
    double re, im;
};
__device__ inline Cx cx(double r, double i) { return Cx{r, i}; }
__device__ inline Cx operator+(Cx a, Cx b) { return cx(a.re + b.re, a.im + b.im); }
__device__ inline Cx operator-(Cx a, Cx b) { return cx(a.re - b.re, a.im - b.im); }
__device__ inline Cx operator*(Cx a, Cx b) { return cx(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re); }
__device__ inline Cx cx_log(Cx z) { return cx(log(hypot(z.re, z.im)), atan2(z.im, z.re)); }

// log Gamma(z) for Re z > 0.5: Lanczos g = 7 with 9 terms (Lanczos, SIAM J. Numer. Anal. B 1
// (1964) 86; the coefficient set of util.py:26-36)
__device__ inline Cx lngamma_lanczos(Cx z)
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
__device__ inline Cx log_sin_pi(Cx z)
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

__device__ inline Cx lngamma_c(Cx z)
{
    if (z.re <= 0.5) {  // reflection
        const Cx l = lngamma_lanczos(cx(1.0 - z.re, -z.im));
        const Cx ls = log_sin_pi(z);
        return cx(1.14472988584940017414342735135, 0.0) - ls - l;
    }
    return lngamma_lanczos(z);
}

}  // namespace cplx
}  // namespace dscb
