// dual.cuh - forward-mode dual numbers for the local Jacobians of the adjoint (adjoint.cuh).
//
// Dual<N> carries a value and N directional derivatives, all in double. The device building
// blocks of the large step (model.cuh) are templates over their scalar type, so instantiating
// them with Dual<N> gives the partial derivatives of a cell's outputs with respect to N seeded
// inputs in one evaluation. Branches and min/max select on the value, so a derivative is the
// derivative of the branch the forward step took (the one-sided derivative at a kink).
//
// The mm:: overloads must be declared before model.cuh is parsed: its templates call mm::mpow
// and friends by qualified name, which binds to the overloads visible at the template's
// definition.
#pragma once

#include "moist_math.h"

namespace mm {

template <int N>
struct Dual {
    double v;
    double d[N];
    MM_HD Dual() : v(0.0) {
#pragma unroll
        for (int j = 0; j < N; j++) d[j] = 0.0;
    }
    MM_HD Dual(double x) : v(x) {
#pragma unroll
        for (int j = 0; j < N; j++) d[j] = 0.0;
    }
    // a value seeded in direction j
    MM_HD static Dual seed(double x, int j) {
        Dual r(x);
#pragma unroll
        for (int q = 0; q < N; q++) r.d[q] = (q == j) ? 1.0 : 0.0;
        return r;
    }
};

template <int N>
MM_HD Dual<N> operator+(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r;
    r.v = a.v + b.v;
#pragma unroll
    for (int j = 0; j < N; j++) r.d[j] = a.d[j] + b.d[j];
    return r;
}
template <int N>
MM_HD Dual<N> operator-(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r;
    r.v = a.v - b.v;
#pragma unroll
    for (int j = 0; j < N; j++) r.d[j] = a.d[j] - b.d[j];
    return r;
}
template <int N>
MM_HD Dual<N> operator-(const Dual<N>& a) {
    Dual<N> r;
    r.v = -a.v;
#pragma unroll
    for (int j = 0; j < N; j++) r.d[j] = -a.d[j];
    return r;
}
template <int N>
MM_HD Dual<N> operator*(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r;
    r.v = a.v * b.v;
#pragma unroll
    for (int j = 0; j < N; j++) r.d[j] = a.d[j] * b.v + a.v * b.d[j];
    return r;
}
// 1/b for the derivative part of a quotient. On the device: the hardware approximation refined
// by two Newton-Raphson steps y <- y + y (1 - b y) (each squares the relative error, from about
// 2^-22 to below the double rounding), for |b| in [2^-1000, 2^1000]; elsewhere, and on the
// host, the IEEE quotient. The value part of every quotient stays the IEEE quotient.
MM_HD double drcp(double b) {
#ifdef __CUDA_ARCH__
    const double ab = fabs(b);
    if (ab >= 0x1p-1000 && ab <= 0x1p1000) {
        double y;
        asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(b));
        double e = fma(-b, y, 1.0);
        y = fma(y, e, y);
        e = fma(-b, y, 1.0);
        return fma(y, e, y);
    }
#endif
    return 1.0 / b;
}

template <int N>
MM_HD Dual<N> operator/(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r;
    const double q = a.v / b.v;
    const double rb = drcp(b.v);
    r.v = q;
#pragma unroll
    for (int j = 0; j < N; j++) r.d[j] = (a.d[j] - q * b.d[j]) * rb;
    return r;
}
template <int N>
MM_HD Dual<N>& operator+=(Dual<N>& a, const Dual<N>& b) {
    a = a + b;
    return a;
}
template <int N>
MM_HD Dual<N>& operator-=(Dual<N>& a, const Dual<N>& b) {
    a = a - b;
    return a;
}
template <int N>
MM_HD Dual<N>& operator*=(Dual<N>& a, const Dual<N>& b) {
    a = a * b;
    return a;
}

// mixed forms (template deduction does not apply the converting constructor)
#define MM_DUAL_MIXED(op)                                                                  \
    template <int N>                                                                       \
    MM_HD Dual<N> operator op(const Dual<N>& a, double b) { return a op Dual<N>(b); }      \
    template <int N>                                                                       \
    MM_HD Dual<N> operator op(double a, const Dual<N>& b) { return Dual<N>(a) op b; }
MM_DUAL_MIXED(+)
MM_DUAL_MIXED(-)
MM_DUAL_MIXED(*)
MM_DUAL_MIXED(/)
#undef MM_DUAL_MIXED

#define MM_DUAL_CMP(op)                                                                    \
    template <int N>                                                                       \
    MM_HD bool operator op(const Dual<N>& a, const Dual<N>& b) { return a.v op b.v; }     \
    template <int N>                                                                       \
    MM_HD bool operator op(const Dual<N>& a, double b) { return a.v op b; }               \
    template <int N>                                                                       \
    MM_HD bool operator op(double a, const Dual<N>& b) { return a op b.v; }
MM_DUAL_CMP(<)
MM_DUAL_CMP(>)
MM_DUAL_CMP(<=)
MM_DUAL_CMP(>=)
MM_DUAL_CMP(==)
MM_DUAL_CMP(!=)
#undef MM_DUAL_CMP

template <int N>
MM_HD bool signbit_(const Dual<N>& x) {
    return signbit_(x.v);
}

template <int N>
MM_HD Dual<N> mexp(const Dual<N>& x) {
    Dual<N> r;
    const double e = exp_d(x.v);
    r.v = e;
#pragma unroll
    for (int j = 0; j < N; j++) r.d[j] = e * x.d[j];
    return r;
}

// x^y for x > 0: d(x^y) = x^y (y dx / x + log(x) dy)
template <int N>
MM_HD Dual<N> mpow(const Dual<N>& x, const Dual<N>& y) {
    Dual<N> r;
    const double p = pow_d(x.v, y.v);
    r.v = p;
    bool dy = false;
#pragma unroll
    for (int j = 0; j < N; j++) dy = dy || (y.d[j] != 0.0);
    const double lx = (dy && x.v > 0.0) ? log_d(x.v) : 0.0;
    const double gx = x.v != 0.0 ? p * y.v / x.v : 0.0;
#pragma unroll
    for (int j = 0; j < N; j++) r.d[j] = gx * x.d[j] + p * lx * y.d[j];
    return r;
}
template <int N>
MM_HD Dual<N> mpow(const Dual<N>& x, double y) {
    return mpow(x, Dual<N>(y));
}

// x^4 (gray radiation): d(x^4) = 4 x^3 dx
template <int N>
MM_HD Dual<N> mpow4(const Dual<N>& x) {
    Dual<N> r;
    r.v = mpow4(x.v);
    const double g = 4.0 * x.v * x.v * x.v;
#pragma unroll
    for (int j = 0; j < N; j++) r.d[j] = g * x.d[j];
    return r;
}

template <int N>
MM_HD Dual<N> msqrt(const Dual<N>& x) {
    Dual<N> r;
    const double s = sqrt(x.v);
    r.v = s;
    const double g = s > 0.0 ? 0.5 / s : 0.0;
#pragma unroll
    for (int j = 0; j < N; j++) r.d[j] = g * x.d[j];
    return r;
}

// |x| with the value of fabs (+0 for -0, which the sign-bit selects of jmin/jmax can see)
template <int N>
MM_HD Dual<N> mabs(const Dual<N>& x) {
    Dual<N> r = x.v < 0.0 ? -x : x;
    r.v = fabs(x.v);
    return r;
}

}  // namespace mm
