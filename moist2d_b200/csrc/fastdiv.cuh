// fastdiv.cuh - branch-free, correctly rounded Float32 division for the tracer sweep.
//
// CUDA's IEEE division (div.rn.f32) ends every quotient with a range check and a branch to a
// slow path (very slow for subnormal results), so consecutive divisions cannot overlap and the
// code between them cannot be scheduled together: a tracer cell update with ~25 divisions costs
// ~1800 cycles of dependent latency, and the Gauss-Seidel tracer sweep walks long chains of
// such updates. Here float division is RN32(RN64(a * y)) with y = 1/b in double precision
// (proof at div64), which returns the IEEE quotient for every input except ties in the
// subnormal range; those are reported through a guard word (Div64) or rounded explicitly
// (Div64X). tests/fastdiv_check.cu checks both against IEEE division on the GPU, exhaustively
// over all numerators for the model's denominators and on random bit patterns of every class.
#pragma once

#include <cuda_runtime.h>

namespace moist {

// The sign of a zero result: for a nonzero quotient q and q0 (two roundings of the same value)
// share their sign, so OR-ing the sign bit of q0 into q only changes a zero.
__device__ __forceinline__ float with_sign_of(float q, float q0) {
    return __int_as_float(__float_as_int(q) | (__float_as_int(q0) & (int)0x80000000));
}

// Selects the compiler cannot turn into branches: both operands are always computed, so the
// independent parts of a cell update stay in one basic block and overlap.
__device__ __forceinline__ float sel_gt(float a, float b, float x, float y) {  // a > b ? x : y
    float r;
    asm("{\n\t.reg .pred p;\n\tsetp.gt.f32 p, %1, %2;\n\tselp.f32 %0, %3, %4, p;\n\t}"
        : "=f"(r) : "f"(a), "f"(b), "f"(x), "f"(y));
    return r;
}
__device__ __forceinline__ float sel_lt(float a, float b, float x, float y) {  // a < b ? x : y
    float r;
    asm("{\n\t.reg .pred p;\n\tsetp.lt.f32 p, %1, %2;\n\tselp.f32 %0, %3, %4, p;\n\t}"
        : "=f"(r) : "f"(a), "f"(b), "f"(x), "f"(y));
    return r;
}
__device__ __forceinline__ float sel_u(unsigned c, float x, float y) {  // c != 0 ? x : y
    float r;
    asm("{\n\t.reg .pred p;\n\tsetp.ne.u32 p, %1, 0;\n\tselp.f32 %0, %2, %3, p;\n\t}"
        : "=f"(r) : "r"(c), "f"(x), "f"(y));
    return r;
}

// Julia's min / max (NaN-propagating, -0 < +0) as single PTX instructions
__device__ __forceinline__ float jmin_f(float a, float b) {
    float r;
    asm("min.NaN.f32 %0, %1, %2;" : "=f"(r) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ float jmax_f(float a, float b) {
    float r;
    asm("max.NaN.f32 %0, %1, %2;" : "=f"(r) : "f"(a), "f"(b));
    return r;
}

// ---- FP64-reciprocal division: RN32(a/b) = RN32(RN64(a * y)) for y = 1/b to within 2^-51
//
// For floats a, b whose quotient is not a float itself, a/b lies at a relative distance of at
// least 2^-48 from every float rounding boundary (a midpoint between neighbouring floats, or
// the overflow threshold): with A, B the integer significands, a boundary M near A/B gives
// |A/B - M| >= 1/(B 2^25), and in the subnormal range the distance is larger still. A normal
// quotient is never exactly a boundary (that needs 25 significant bits from a product of
// B <= 24 bits and A); a subnormal one can be, e.g. (3 * 2^-149) / 6 = 2^-150. The product a*y
// rounded to double is within 2^-52 + 2^-51 of a/b (the double product neither underflows nor
// overflows), so it lies on the same side of every boundary and rounding it to float gives the
// IEEE quotient, except for those exact subnormal ties. Every quotient q in 0 < |q| <= 2^-126
// is therefore reported through a guard word (subnormal_guard), and the caller recomputes such
// a cell with IEEE division; zeros, infinities and NaN come out as IEEE division gives them.
__device__ __forceinline__ float div64(float a, double y) { return __double2float_rn((double)a * y); }

// div64 exact for every input: a quotient below 2^-125 in magnitude (float spacing 2^-149) is
// rounded explicitly on that grid. w = p 2^149 is the quotient in grid units, within 2^-28 of
// the exact value; an exact quotient that is not a tie lies at least 2^-25 from every
// half-integer (the nonzero integer |A 2^e - B (2k+1)| over 2B, with B >= 2^23 since b is
// normal whenever a/b < 2^-125), so |w - fl - 1/2| < 2^-26 detects the ties, which go to the
// even neighbour; every other w rounds to its nearest integer. The sign of a zero is p's.
__device__ __forceinline__ float div64x(float a, double y) {
    const double p = (double)a * y;
    const float qn = __double2float_rn(p);
    const double w = p * 0x1p149;
    const double fl = floor(w);
    const bool tie = fabs((w - fl) - 0.5) < 0x1p-26;
    const double even = (fl - 2.0 * floor(fl * 0.5)) == 0.0 ? fl : fl + 1.0;
    const float qs = with_sign_of((float)((tie ? even : rint(w)) * 0x1p-149), qn);
    return fabs(p) < 0x1p-125 ? qs : qn;
}

// fold q into the guard word g (start from ~0u): afterwards g < 2^24 iff some q had
// 0 < |q| <= 2^-126 (the doubled bit pattern of 2^-126 is 2^24; zero maps to ~0u)
__device__ __forceinline__ void subnormal_guard(unsigned& g, float q) { g = min(g, (__float_as_uint(q) << 1) - 1u); }
__device__ __forceinline__ bool guard_hit(unsigned g) { return g < (1u << 24); }

// 1/b to within 2^-51 relative (b finite and nonzero): the hardware approximation and two
// Newton steps e = 1 - b y, y += y e in double precision
__device__ __forceinline__ double rcp64(float b) {
    const double bd = (double)b;
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(bd));
    double e = __fma_rn(-bd, y, 1.0);
    y = __fma_rn(y, e, y);
    e = __fma_rn(-bd, y, 1.0);
    return __fma_rn(y, e, y);
}

// division policies of the fast tracer cell: cdiv(a, b, y, g) with y = 1/b prepared once,
// vdiv(a, b, g) for a variable denominator, div3(a) = a / 3; g is the subnormal guard word
struct Div64 {  // FP64 reciprocal: exact for every input but subnormal ties, which g reports
    using R = double;
    __device__ __forceinline__ static R rcp(float b) { return 1.0 / (double)b; }
    __device__ __forceinline__ static float cdiv(float a, float, R y, unsigned& g) {
        const float q = div64(a, y);
        subnormal_guard(g, q);
        return q;
    }
    __device__ __forceinline__ static float vdiv(float a, float b, unsigned& g) {
        const float q = div64(a, rcp64(b));
        subnormal_guard(g, q);
        return q;
    }
    // (1 + 2r) / 3: the numerator is 0 or at least 2^-24 in magnitude, so no subnormal quotient
    __device__ __forceinline__ static float div3(float a) { return div64(a, 1.0 / 3.0); }
};
struct Div64X {  // FP64 reciprocal with explicit rounding of subnormal quotients: exact for every input
    using R = double;
    __device__ __forceinline__ static R rcp(float b) { return 1.0 / (double)b; }
    __device__ __forceinline__ static float cdiv(float a, float, R y, unsigned&) { return div64x(a, y); }
    __device__ __forceinline__ static float vdiv(float a, float b, unsigned&) { return div64x(a, rcp64(b)); }
    __device__ __forceinline__ static float div3(float a) { return div64(a, 1.0 / 3.0); }
};

// ---- the correctly rounded double quotient a/b without a division on the dependent path
//
// Given y = RN(1/b) (formed ahead, off the path): q0 = RN(a y) lies within 1.5 ulp of a/b; one
// correction with its remainder, q1 = RN(q0 + (a - b q0) y), brings it to the correctly rounded
// quotient in all but rare cases. q1 is then checked exactly: when q1 lies within one ulp of
// a/b, the remainder r1 = a - b q1 is a double and the FMA forms it exactly (no underflow for
// the operand ranges admitted below), and |r1| < |b| u/2, with u the smaller of the two ulps
// around q1 (the ulp below a power of two is half the one above), says that a/b is nearer to
// q1 than to the midpoint towards either neighbour, i.e. q1 = RN(a/b). |b| u/2 is a power-of-two
// multiple of b, hence exact. When q1 is farther than one ulp the computed |r1| is at least
// RN(|b| u) = 2 (|b| u/2), so the test fails. ok is cleared where the test fails or the operands
// leave 2^-960 <= |a| <= 2^1000, 2^-1000 <= |b| <= 2^1000 (non-finite values included): the
// caller then divides again with IEEE division. a = 0 gives q0 = a y, the IEEE result with its
// sign. The method is the remainder correction of Markstein's division (IBM J. Res. Dev. 34,
// 1990) with an exact acceptance test in place of a proof for every operand. On B200 the
// dependent path is 69 cycles against 112 for IEEE division (with the multiply-subtract of a
// Thomas level in both).
__device__ __forceinline__ double qdiv_checked(double a, double b, double y, bool& ok) {
    const double q0 = a * y;
    const double r0 = fma(-b, q0, a);
    const double q1 = fma(r0, y, q0);
    const double r1 = fma(-b, q1, a);
    const unsigned long long bits = (unsigned long long)__double_as_longlong(q1) & 0x7fffffffffffffffULL;
    const long long e = (long long)(bits >> 52);                                   // biased exponent of q1
    const long long he = e - 53 - ((bits & 0xfffffffffffffULL) == 0 ? 1 : 0);  // half of the smaller ulp
    const double half_u = __longlong_as_double((he < 1 ? 1LL : he) << 52);
    const double aa = fabs(a), ab = fabs(b);
    const bool zero = aa == 0.0;
    const bool in_range = aa >= 0x1p-960 && aa <= 0x1p1000 && ab >= 0x1p-1000 && ab <= 0x1p1000 && he >= 1;
    ok = ok && (zero || (in_range && fabs(r1) < ab * half_u));
    return zero ? q0 : q1;
}

// division policies for the templated tracer arithmetic: div(a, b) with a variable
// denominator, divr(a, b, y) with y = RN(1/b) prepared in advance
template <class T>
struct DivIEEE {
    __device__ __forceinline__ static T div(T a, T b, bool&) { return a / b; }
    __device__ __forceinline__ static T divr(T a, T b, T, bool&) { return a / b; }
};


}  // namespace moist
