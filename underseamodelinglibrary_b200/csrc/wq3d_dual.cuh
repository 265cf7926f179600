/*
 * wq3d_dual.cuh -- forward-mode dual numbers for the adjoint's local
 * Jacobians.
 *
 * A Dual<N> carries a value and its derivatives along N input directions.
 * The reverse sweep of the adjoint (wq3d_adjoint.cuh) uses them to form
 * the Jacobian of one ray's step, or of one reflection chain, with respect
 * to that step's inputs; the sweep itself then applies the transposes.
 * The value part of every operation is the plain double operation, in the
 * same order as the engine's double code, so a Dual evaluation retraces
 * the engine's arithmetic and takes the same branches.  Branches on Dual
 * values compare the value part: the derivative is that of the branch the
 * value took (a frozen topology).
 */
#pragma once

#include <math.h>

namespace wq3d {

template <int N>
struct Dual {
    double v;
    double d[N];

    __device__ __forceinline__ Dual() {}
    __device__ __forceinline__ Dual(double x) : v(x) {
#pragma unroll
        for (int k = 0; k < N; ++k) d[k] = 0.0;
    }
    /* an input: value x, unit derivative along direction k (k < 0: none) */
    __device__ __forceinline__ static Dual var(double x, int k) {
        Dual r(x);
        if (k >= 0 && k < N) r.d[k] = 1.0;
        return r;
    }
};

/* plain double forms, so that templated code calls the same names for
 * double and Dual arguments inside this namespace */
__device__ __forceinline__ double sqrt(double x) { return ::sqrt(x); }
__device__ __forceinline__ double sin(double x) { return ::sin(x); }
__device__ __forceinline__ double cos(double x) { return ::cos(x); }
__device__ __forceinline__ double exp(double x) { return ::exp(x); }
__device__ __forceinline__ double log10(double x) { return ::log10(x); }
__device__ __forceinline__ double asin(double x) { return ::asin(x); }
__device__ __forceinline__ double fabs(double x) { return ::fabs(x); }
__device__ __forceinline__ double atan2(double y, double x) { return ::atan2(y, x); }
__device__ __forceinline__ double fmax(double a, double b) { return ::fmax(a, b); }

template <int N>
__device__ __forceinline__ double val(const Dual<N>& a) { return a.v; }
__device__ __forceinline__ double val(double a) { return a; }

/* a value with derivative g * a' (the chain rule for a unary function) */
template <int N>
__device__ __forceinline__ Dual<N> chain(double v, double g, const Dual<N>& a) {
    Dual<N> r;
    r.v = v;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = g * a.d[k];
    return r;
}

template <int N>
__device__ __forceinline__ Dual<N> operator+(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r;
    r.v = a.v + b.v;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = a.d[k] + b.d[k];
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator-(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r;
    r.v = a.v - b.v;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = a.d[k] - b.d[k];
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator-(const Dual<N>& a) {
    Dual<N> r;
    r.v = -a.v;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = -a.d[k];
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator*(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r;
    r.v = a.v * b.v;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator/(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r;
    r.v = a.v / b.v;
    const double ib = 1.0 / b.v;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = (a.d[k] - r.v * b.d[k]) * ib;
    return r;
}
/* mixed forms: the double operand has no derivative */
template <int N>
__device__ __forceinline__ Dual<N> operator+(const Dual<N>& a, double b) {
    Dual<N> r = a;
    r.v = a.v + b;
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator+(double a, const Dual<N>& b) {
    Dual<N> r = b;
    r.v = a + b.v;
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator-(const Dual<N>& a, double b) {
    Dual<N> r = a;
    r.v = a.v - b;
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator-(double a, const Dual<N>& b) {
    Dual<N> r;
    r.v = a - b.v;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = -b.d[k];
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator*(const Dual<N>& a, double b) {
    Dual<N> r;
    r.v = a.v * b;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = a.d[k] * b;
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator*(double a, const Dual<N>& b) {
    Dual<N> r;
    r.v = a * b.v;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = a * b.d[k];
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator/(const Dual<N>& a, double b) {
    Dual<N> r;
    r.v = a.v / b;
    const double ib = 1.0 / b;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = a.d[k] * ib;
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator/(double a, const Dual<N>& b) {
    const double v = a / b.v;
    return chain(v, -v / b.v, b);
}

template <int N>
__device__ __forceinline__ Dual<N> sqrt(const Dual<N>& a) {
    const double s = ::sqrt(a.v);
    return chain(s, s > 0.0 ? 0.5 / s : 0.0, a);
}
template <int N>
__device__ __forceinline__ Dual<N> sin(const Dual<N>& a) { return chain(::sin(a.v), ::cos(a.v), a); }
template <int N>
__device__ __forceinline__ Dual<N> cos(const Dual<N>& a) { return chain(::cos(a.v), -::sin(a.v), a); }
template <int N>
__device__ __forceinline__ Dual<N> exp(const Dual<N>& a) {
    const double e = ::exp(a.v);
    return chain(e, e, a);
}
template <int N>
__device__ __forceinline__ Dual<N> log10(const Dual<N>& a) {
    return chain(::log10(a.v), 1.0 / (a.v * 2.302585092994045684), a);
}
template <int N>
__device__ __forceinline__ Dual<N> asin(const Dual<N>& a) {
    return chain(::asin(a.v), 1.0 / ::sqrt(1.0 - a.v * a.v), a);
}
template <int N>
__device__ __forceinline__ Dual<N> fabs(const Dual<N>& a) { return a.v < 0.0 ? -a : a; }
/* atan2(y, x): d = (x dy - y dx) / (x^2 + y^2) */
template <int N>
__device__ __forceinline__ Dual<N> atan2(const Dual<N>& y, const Dual<N>& x) {
    Dual<N> r;
    r.v = ::atan2(y.v, x.v);
    const double q = x.v * x.v + y.v * y.v;
    const double a = q > 0.0 ? x.v / q : 0.0, b = q > 0.0 ? -y.v / q : 0.0;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = a * y.d[k] + b * x.d[k];
    return r;
}
/* fmax(a, b) with a double bound: the bound carries no derivative */
template <int N>
__device__ __forceinline__ Dual<N> fmax(const Dual<N>& a, double b) { return (a.v >= b) ? a : Dual<N>(b); }
template <int N>
__device__ __forceinline__ Dual<N> fmax(double b, const Dual<N>& a) { return (a.v >= b) ? a : Dual<N>(b); }
template <int N>
__device__ __forceinline__ Dual<N> fmax(const Dual<N>& a, const Dual<N>& b) { return (a.v >= b.v) ? a : b; }

}  // namespace wq3d
