// moist_math.h - scalar math shared bit-for-bit by the CUDA kernels and the CPU oracle.
//
// The large step needs exp (Tetens saturation pressure, moist.jl:257) and real powers
// (Exner function and pressure, moist.jl:583-587, 1058; terminal velocity, moist.jl:685).
// Library exp/pow differ between glibc and the CUDA math library in the last bit, and a
// convective flow amplifies last-bit differences, so both sides use the functions below,
// written from published methods:
//   exp : Cody-Waite argument reduction x = n*ln2 + r (W. J. Cody and W. Waite, "Software
//         Manual for the Elementary Functions", 1980) with ln2 split into a 32-bit head and a
//         tail, followed by the Taylor series of e^r to degree 13 (|r| <= ln2/2, truncation
//         < 5e-18 relative) evaluated by Horner's rule with fused multiply-adds.
//   log : x = 2^k * m, m in [sqrt(1/2), sqrt(2)), log m = 2 atanh(s), s = (m-1)/(m+1), with
//         the atanh series to s^21; the leading term 2s is carried as a double-double so the
//         result has ~2^-60 relative error.
//   pow : x^y = exp(y log x) with y*log x formed in double-double arithmetic and the tail
//         applied as exp(t_hi) * (1 + t_lo).
// Accuracy against glibc: exp <= 1 ulp, pow <= 2 ulp on the model's argument ranges (checked
// by tests/test_math.py). Float versions evaluate in double and round once, which is how Julia
// evaluates Float32 ^ (moist.jl runs ^ on Float32 through its Float64 kernel).
//
// Min/max follow Julia's IEEE semantics (NaN-propagating; min(0.0,-0.0) = -0.0), which C's
// fmin/fmax and std::min/max do not.
//
// Everything here uses only IEEE-exact primitives (+ - * / sqrt fma rint and bit moves), so
// the same source compiled by nvcc (with --fmad=false) and by g++ (with -ffp-contract=off)
// gives identical bits.
#pragma once

#include <math.h>
#include <stdint.h>
#include <string.h>

#if defined(__CUDACC__)
#define MM_HD __host__ __device__ __forceinline__
#else
#define MM_HD inline
#endif

namespace mm {

MM_HD uint64_t dbits(double x) {
#if defined(__CUDA_ARCH__)
    return (uint64_t)__double_as_longlong(x);
#else
    uint64_t u;
    memcpy(&u, &x, sizeof u);
    return u;
#endif
}

MM_HD double dfrom(uint64_t u) {
#if defined(__CUDA_ARCH__)
    return __longlong_as_double((long long)u);
#else
    double x;
    memcpy(&x, &u, sizeof x);
    return x;
#endif
}

MM_HD double dfma(double a, double b, double c) {
#if defined(__CUDA_ARCH__)
    return __fma_rn(a, b, c);
#else
    return fma(a, b, c);
#endif
}

// 2^n for -1022 <= n <= 1023
MM_HD double pow2i(int n) { return dfrom((uint64_t)(n + 1023) << 52); }

// ln 2 = LN2_HI + LN2_LO; LN2_HI has 32 significant bits so n*LN2_HI is exact for |n| < 2^21
constexpr double LN2_HI = 0x1.62e42fee00000p-1;
constexpr double LN2_LO = 0x1.a39ef35793c76p-33;
constexpr double INV_LN2 = 0x1.71547652b82fep+0;
constexpr double SQRT2 = 1.4142135623730951;

MM_HD double exp_d(double x) {
    if (x != x) return x;
    if (x > 709.8) return (double)INFINITY;
    if (x < -745.2) return 0.0;
    const double nd = rint(x * INV_LN2);
    const int n = (int)nd;
    const double r = (x - nd * LN2_HI) - nd * LN2_LO;
    // Taylor coefficients 1/k!, k = 13 .. 0 (each a single correctly rounded division)
    double p = 1.0 / 6227020800.0;
    p = dfma(p, r, 1.0 / 479001600.0);
    p = dfma(p, r, 1.0 / 39916800.0);
    p = dfma(p, r, 1.0 / 3628800.0);
    p = dfma(p, r, 1.0 / 362880.0);
    p = dfma(p, r, 1.0 / 40320.0);
    p = dfma(p, r, 1.0 / 5040.0);
    p = dfma(p, r, 1.0 / 720.0);
    p = dfma(p, r, 1.0 / 120.0);
    p = dfma(p, r, 1.0 / 24.0);
    p = dfma(p, r, 1.0 / 6.0);
    p = dfma(p, r, 0.5);
    p = dfma(p, r, 1.0);
    p = dfma(p, r, 1.0);
    if (n > 1023) return (p * pow2i(1023)) * pow2i(n - 1023);
    if (n < -1022) return (p * pow2i(n + 600)) * pow2i(-600);
    return p * pow2i(n);
}

// natural log of a positive finite x as a double-double hi + lo
MM_HD void log_dd(double x, double* hi, double* lo) {
    int k = 0;
    if (x < 0x1p-1022) {  // subnormal: scale into the normal range
        x *= 0x1p54;
        k = -54;
    }
    const uint64_t u = dbits(x);
    k += (int)((u >> 52) & 0x7ff) - 1023;
    double m = dfrom((u & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL);  // [1, 2)
    if (m > SQRT2) {
        m *= 0.5;
        k += 1;
    }
    const double f = m - 1.0;                // exact
    const double uh = 2.0 + f;               // 2 + f as a double-double uh + ul
    const double ul = (2.0 - uh) + f;
    const double s = f / uh;
    const double sl = (dfma(-s, uh, f) - s * ul) / uh;  // s + sl = f / (2 + f) to ~2^-106
    const double z = s * s;
    double P = 1.0 / 21.0;  // atanh series: sum z^(j-1) / (2j+1), j = 1 .. 10
    P = dfma(P, z, 1.0 / 19.0);
    P = dfma(P, z, 1.0 / 17.0);
    P = dfma(P, z, 1.0 / 15.0);
    P = dfma(P, z, 1.0 / 13.0);
    P = dfma(P, z, 1.0 / 11.0);
    P = dfma(P, z, 1.0 / 9.0);
    P = dfma(P, z, 1.0 / 7.0);
    P = dfma(P, z, 1.0 / 5.0);
    P = dfma(P, z, 1.0 / 3.0);
    const double tail = (2.0 * s) * (z * P);
    const double lh = 2.0 * s;
    const double ll = 2.0 * sl + tail;
    const double kd = (double)k;
    const double kh = kd * LN2_HI;           // exact
    const double kl = kd * LN2_LO;
    // two-sum kh + lh, then fold in the small terms
    const double sh = kh + lh;
    const double bb = sh - kh;
    double se = (kh - (sh - bb)) + (lh - bb);
    se += ll + kl;
    const double rh = sh + se;
    *hi = rh;
    *lo = se - (rh - sh);
}

MM_HD double log_d(double x) {
    if (x != x || x < 0.0) return (double)NAN;
    if (x == 0.0) return -(double)INFINITY;
    if (x == (double)INFINITY) return x;
    double h, l;
    log_dd(x, &h, &l);
    return h + l;
}

// x^y for the model's real exponents. A negative base gives NaN (Julia raises DomainError
// for a negative base with a non-integer exponent; the model's NaN check then reports it).
MM_HD double pow_d(double x, double y) {
    if (y == 0.0) return 1.0;
    if (x != x || y != y) return (double)NAN;
    if (x < 0.0) return (double)NAN;
    if (x == 0.0) return y > 0.0 ? 0.0 : (double)INFINITY;
    if (x == (double)INFINITY) return y > 0.0 ? x : 0.0;
    if (x == 1.0) return 1.0;
    double lh, ll;
    log_dd(x, &lh, &ll);
    const double th = y * lh;
    const double tl = dfma(y, lh, -th) + y * ll;
    const double e = exp_d(th);
    if (e == (double)INFINITY || e == 0.0) return e;
    return dfma(e, tl, e);
}

// precision-generic entry points used by the model code
MM_HD double mexp(double x) { return exp_d(x); }
MM_HD float mexp(float x) { return (float)exp_d((double)x); }
MM_HD double mpow(double x, double y) { return pow_d(x, y); }
MM_HD float mpow(float x, float y) { return (float)pow_d((double)x, (double)y); }
// x^4 as Julia evaluates a literal integer power (power by squaring, compensated in Float64;
// Float32 goes through Float64): x^2 is exact in the wider format, one rounding for x^4.
MM_HD float mpow4(float x) {
    const double d = (double)x * (double)x;
    return (float)(d * d);
}
MM_HD double mpow4(double x) {
    const double h = x * x;
    const double l = dfma(x, x, -h);
    const double hh = h * h;
    const double e = dfma(h, h, -hh) + (2.0 * h) * l;
    return hh + e;
}
MM_HD double msqrt(double x) { return sqrt(x); }
MM_HD float msqrt(float x) { return sqrtf(x); }
MM_HD double mabs(double x) { return fabs(x); }
MM_HD float mabs(float x) { return fabsf(x); }

MM_HD bool signbit_(double x) { return (dbits(x) >> 63) != 0; }
MM_HD bool signbit_(float x) {
#if defined(__CUDA_ARCH__)
    return (__float_as_uint(x) >> 31) != 0;
#else
    uint32_t u;
    memcpy(&u, &x, sizeof u);
    return (u >> 31) != 0;
#endif
}

// Julia Base.min / Base.max for IEEE floats
template <class T>
MM_HD T jmin(T x, T y) {
    const T diff = x - y;
    const T argmin = signbit_(diff) ? x : y;
    const bool anynan = (x != x) || (y != y);
    return anynan ? diff : argmin;
}
template <class T>
MM_HD T jmax(T x, T y) {
    const T diff = x - y;
    const T argmax = signbit_(diff) ? y : x;
    const bool anynan = (x != x) || (y != y);
    return anynan ? diff : argmax;
}

}  // namespace mm
