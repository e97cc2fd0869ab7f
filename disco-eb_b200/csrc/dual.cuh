// Forward-mode dual numbers and the math wrappers shared by the double and dual code paths.
//
// DualT<B> carries a value and one directional derivative, both of type B.  Dual =
// DualT<double> is used for the Jacobian column d f / d a (direction: the scale factor) and
// for tangents of the whole solve (direction: a parameter); HDual = DualT<Dual> carries two
// directions and their mixed second derivative, which the tangent of the Rosenbrock step
// needs (the derivative of J k along a parameter direction).
#pragma once

#include <cmath>

#if defined(__CUDACC__)
#define DHD __host__ __device__ __forceinline__
#define DDV __device__ inline
#else
#define DHD inline
#define DDV inline
#endif

namespace dscb {

template <class B> struct DualT {
    B v, d;
    DHD DualT() : v(0.0), d(0.0) {}
    DHD DualT(double x) : v(x), d(0.0) {}
    DHD DualT(const B& x, const B& dx) : v(x), d(dx) {}
};
using Dual = DualT<double>;
using HDual = DualT<Dual>;

template <class B> DHD DualT<B> operator+(const DualT<B>& a, const DualT<B>& b) { return DualT<B>(a.v + b.v, a.d + b.d); }
template <class B> DHD DualT<B> operator-(const DualT<B>& a, const DualT<B>& b) { return DualT<B>(a.v - b.v, a.d - b.d); }
template <class B> DHD DualT<B> operator-(const DualT<B>& a) { return DualT<B>(-a.v, -a.d); }
template <class B> DHD DualT<B> operator*(const DualT<B>& a, const DualT<B>& b)
{
    return DualT<B>(a.v * b.v, a.d * b.v + a.v * b.d);
}
template <class B> DHD DualT<B> rcp(const DualT<B>& x);
template <class B> DHD DualT<B> operator/(const DualT<B>& a, const DualT<B>& b) { return a * rcp(b); }
template <class B> DHD DualT<B> operator+(const DualT<B>& a, double b) { return DualT<B>(a.v + b, a.d); }
template <class B> DHD DualT<B> operator+(double a, const DualT<B>& b) { return DualT<B>(a + b.v, b.d); }
template <class B> DHD DualT<B> operator-(const DualT<B>& a, double b) { return DualT<B>(a.v - b, a.d); }
template <class B> DHD DualT<B> operator-(double a, const DualT<B>& b) { return DualT<B>(a - b.v, -b.d); }
template <class B> DHD DualT<B> operator*(const DualT<B>& a, double b) { return DualT<B>(a.v * b, a.d * b); }
template <class B> DHD DualT<B> operator*(double a, const DualT<B>& b) { return DualT<B>(a * b.v, a * b.d); }
template <class B> DHD DualT<B> operator/(const DualT<B>& a, double b) { return DualT<B>(a.v / b, a.d / b); }
template <class B> DHD DualT<B> operator/(double a, const DualT<B>& b) { return a * rcp(b); }
template <class B> DHD DualT<B>& operator+=(DualT<B>& a, const DualT<B>& b) { a.v += b.v; a.d += b.d; return a; }
template <class B> DHD DualT<B>& operator-=(DualT<B>& a, const DualT<B>& b) { a.v -= b.v; a.d -= b.d; return a; }

// innermost value (all comparisons and table indices use it)
DHD double val(double x) { return x; }
template <class B> DHD double val(const DualT<B>& x) { return val(x.v); }
// first-level derivative part
DHD double der(double) { return 0.0; }
DHD double der(const Dual& x) { return x.d; }

DHD double rcp(double x)
{
#if defined(__CUDA_ARCH__)
    return __drcp_rn(x);
#else
    return 1.0 / x;
#endif
}
template <class B> DHD DualT<B> rcp(const DualT<B>& x)
{
    const B r = rcp(x.v);
    return DualT<B>(r, -(r * r) * x.d);
}

DHD double xexp(double x) { return exp(x); }
DHD double xlog(double x) { return log(x); }
DHD double xsqrt(double x) { return sqrt(x); }
DHD double xpow(double x, double p) { return pow(x, p); }

template <class B> DHD DualT<B> xexp(const DualT<B>& x)
{
    const B e = xexp(x.v);
    return DualT<B>(e, e * x.d);
}
template <class B> DHD DualT<B> xlog(const DualT<B>& x) { return DualT<B>(xlog(x.v), x.d * rcp(x.v)); }
template <class B> DHD DualT<B> xsqrt(const DualT<B>& x)
{
    const B s = xsqrt(x.v);
    return DualT<B>(s, (0.5 * x.d) * rcp(s));
}
template <class B> DHD DualT<B> xpow(const DualT<B>& x, double p)
{
    const B r = xpow(x.v, p);
    return DualT<B>(r, (p * r) * rcp(x.v) * x.d);
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
template <class T> DHD T xmaxc(const T& x, double lo) { return val(x) > lo ? x : T(lo); }

// a value with first-direction part e (the "tangent" slot): double drops it, Dual stores it,
// HDual stores it in the inner dual of the value part
DHD double seed(double v, double) { return v; }
DHD Dual seed_as(const Dual*, double v, double e) { return Dual(v, e); }
DHD HDual seed_as(const HDual*, double v, double e) { return HDual(Dual(v, e), Dual(0.0)); }
DHD double seed_as(const double*, double v, double) { return v; }
template <class T> DHD T seed_t(double v, double e) { return seed_as((const T*)nullptr, v, e); }

}  // namespace dscb
