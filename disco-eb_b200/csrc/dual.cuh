// Forward-mode dual numbers (value + derivative in one direction) and math wrappers
// shared by double and Dual code paths.  The derivative direction used by the solver
// is the scale factor a = y[0]: the Jacobian column d f / d a comes out of one RHS
// evaluation with a seeded as Dual{a, 1}.
#pragma once

#include <cmath>

#if defined(__CUDACC__)
#define DHD __host__ __device__ __forceinline__
#define DDV __device__
#else
#define DHD inline
#define DDV inline
#endif

namespace dscb {

struct Dual {
    double v, d;
    DHD Dual() : v(0.0), d(0.0) {}
    DHD Dual(double x) : v(x), d(0.0) {}
    DHD Dual(double x, double dx) : v(x), d(dx) {}
};

DHD Dual operator+(Dual a, Dual b) { return Dual(a.v + b.v, a.d + b.d); }
DHD Dual operator-(Dual a, Dual b) { return Dual(a.v - b.v, a.d - b.d); }
DHD Dual operator-(Dual a) { return Dual(-a.v, -a.d); }
DHD Dual operator*(Dual a, Dual b) { return Dual(a.v * b.v, a.d * b.v + a.v * b.d); }
DHD Dual operator/(Dual a, Dual b)
{
    double r = 1.0 / b.v;
    double q = a.v * r;
    return Dual(q, (a.d - q * b.d) * r);
}
DHD Dual operator+(Dual a, double b) { return Dual(a.v + b, a.d); }
DHD Dual operator+(double a, Dual b) { return Dual(a + b.v, b.d); }
DHD Dual operator-(Dual a, double b) { return Dual(a.v - b, a.d); }
DHD Dual operator-(double a, Dual b) { return Dual(a - b.v, -b.d); }
DHD Dual operator*(Dual a, double b) { return Dual(a.v * b, a.d * b); }
DHD Dual operator*(double a, Dual b) { return Dual(a * b.v, a * b.d); }
DHD Dual operator/(Dual a, double b) { return Dual(a.v / b, a.d / b); }
DHD Dual operator/(double a, Dual b)
{
    double q = a / b.v;
    return Dual(q, -q * b.d / b.v);
}
DHD Dual& operator+=(Dual& a, Dual b) { a.v += b.v; a.d += b.d; return a; }
DHD Dual& operator-=(Dual& a, Dual b) { a.v -= b.v; a.d -= b.d; return a; }

DHD double val(double x) { return x; }
DHD double val(const Dual& x) { return x.v; }
DHD double der(double) { return 0.0; }
DHD double der(const Dual& x) { return x.d; }

DHD double xexp(double x) { return exp(x); }
DHD double xlog(double x) { return log(x); }
DHD double xsqrt(double x) { return sqrt(x); }
DHD double xpow(double x, double p) { return pow(x, p); }

DHD Dual xexp(Dual x)
{
    double e = exp(x.v);
    return Dual(e, e * x.d);
}
DHD Dual xlog(Dual x) { return Dual(log(x.v), x.d / x.v); }
DHD Dual xsqrt(Dual x)
{
    double s = sqrt(x.v);
    return Dual(s, 0.5 * x.d / s);
}
DHD Dual xpow(Dual x, double p)
{
    double r = pow(x.v, p);
    return Dual(r, p * r / x.v * x.d);
}

DHD bool xfinite(double x)
{
#if defined(__CUDA_ARCH__)
    return isfinite(x);
#else
    return std::isfinite(x);
#endif
}

// max(x, lo) selecting on the value, as jnp.maximum does for the primal
template <class T> DHD T xmaxc(T x, double lo) { return val(x) > lo ? x : T(lo); }

}  // namespace dscb
