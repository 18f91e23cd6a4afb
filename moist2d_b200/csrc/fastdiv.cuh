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

// division policies for the templated tracer arithmetic: div(a, b) with a variable
// denominator, divr(a, b, y) with y = RN(1/b) prepared in advance
template <class T>
struct DivIEEE {
    __device__ __forceinline__ static T div(T a, T b, bool&) { return a / b; }
    __device__ __forceinline__ static T divr(T a, T b, T, bool&) { return a / b; }
};


}  // namespace moist
