// fastdiv.cuh - branch-free, correctly rounded Float32 division by a known denominator.
//
// CUDA's IEEE division (div.rn.f32) ends every quotient with a range check and a branch to a
// slow path, so consecutive divisions cannot overlap: a tracer cell update with ~20 of them
// costs ~1000 cycles of dependent latency, and the Gauss-Seidel tracer sweep walks long
// chains of such updates. Most of those divisions have a denominator that is fixed for the
// whole sweep (dx, dz, z differences, dz sums, 3, the cell density), so its correctly rounded
// reciprocal y = RN(1/b) can be formed once (with an IEEE division) and each quotient
// obtained by Markstein's correction (P. Markstein, "Computation of elementary functions on
// the IBM RISC System/6000 processor", IBM J. Res. Dev. 34(1), 1990; see also the Handbook
// of Floating-Point Arithmetic, 2nd ed., section 4.7):
//
//     q0 = RN(a*y);  r0 = RN(a - b*q0);  q1 = RN(q0 + r0*y)     (q1 is faithful)
//     r1 = RN(a - b*q1);  q = RN(q1 + r1*y)                    (r1 exact, q = RN(a/b))
//
// with the r's and q's formed by fused multiply-adds. The theorem holds when no intermediate
// underflows or overflows; callers pass a flag that is raised when |a| is outside
// [2^-100, 2^100] or |b| outside [2^-20, 2^20] (so every quotient and remainder stays normal),
// and such a cell is recomputed with IEEE division. A zero numerator returns a*y, which has the sign IEEE division gives.
// tests/test_fastdiv.py checks the routine against IEEE division exhaustively over all finite
// numerators for the denominators the model uses.
#pragma once

#include <cuda_runtime.h>

namespace moist {

__device__ __forceinline__ float mdiv_r(float a, float b, float y, bool& bad) {
    const float q0 = a * y;
    const float r0 = __fmaf_rn(-b, q0, a);
    const float q1 = __fmaf_rn(r0, y, q0);
    const float r1 = __fmaf_rn(-b, q1, a);
    const float q = __fmaf_rn(r1, y, q1);
    const float aa = fabsf(a), bb = fabsf(b);
    bad |= ((a != 0.0f) && !(aa >= 0x1p-100f && aa <= 0x1p100f)) || !(bb >= 0x1p-20f && bb <= 0x1p20f);
    return a == 0.0f ? q0 : q;
}

// ---- branch-free primitives of the fast tracer cell (no flags; callers guarantee the ranges)
//
// rcp_rn(b) = RN(1/b): the hardware approximation rcp.approx (relative error below 1 ulp)
// refined by one Markstein step y = y0 + y0 (1 - b y0) (Markstein 1990, reciprocal theorem).
// Checked against IEEE 1/b for every b with 2^-100 <= |b| < 2^101 (tests/fastdiv_check.cu).
__device__ __forceinline__ float rcp_rn(float b) {
    float y0;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y0) : "f"(b));
    const float e = __fmaf_rn(-b, y0, 1.0f);
    return __fmaf_rn(e, y0, y0);
}

// The corrections of a zero numerator can turn -0 into +0; the sign of q0 = a*y is the sign
// IEEE division gives, and for a nonzero quotient q0 and q have the same sign, so OR-ing the
// sign bit of q0 into q restores the zero's sign without a compare.
__device__ __forceinline__ float with_sign_of(float q, float q0) {
    return __int_as_float(__float_as_int(q) | (__float_as_int(q0) & (int)0x80000000));
}

// two-correction quotient with y = RN(1/b) (the sequence of mdiv_r, without its flag)
__device__ __forceinline__ float mq2(float a, float b, float y) {
    const float q0 = a * y;
    const float r0 = __fmaf_rn(-b, q0, a);
    const float q1 = __fmaf_rn(r0, y, q0);
    const float r1 = __fmaf_rn(-b, q1, a);
    return with_sign_of(__fmaf_rn(r1, y, q1), q0);
}

// one-correction quotient; equal to IEEE division for b = 3 and every a == 0 or
// 2^-100 <= |a| <= 2^100 (checked exhaustively)
__device__ __forceinline__ float mq1(float a, float b, float y) {
    const float q0 = a * y;
    const float r0 = __fmaf_rn(-b, q0, a);
    return with_sign_of(__fmaf_rn(r0, y, q0), q0);
}

// a / b for a variable denominator: equal to IEEE division when 2^-100 <= |b| < 2^101 and
// either a == 0 or |a| >= 2^-100 and 2^-125 <= |a/b| <= 2^126. Every pair of significands is
// checked exhaustively (tests/fastdiv_check.cu); inside these bounds every rounded intermediate
// is a normal number or a remainder that is exact in both ranges (the remainders are multiples
// of 2^(e_a - 48) >= 2^-148), so each operation scales exactly with the exponents of a and b.
__device__ __forceinline__ float vq(float a, float b) { return mq2(a, b, rcp_rn(b)); }

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

// v != 0 and |v| < 2^-100 (below the range of the Markstein quotients)
__device__ __forceinline__ bool tiny_nz(float v) { return ((__float_as_uint(v) << 1) - 1u) < ((27u << 24) - 1u); }
// v == 0 or 2^-48 <= |v| < 2^49: the range of mixing ratios for which the fast cell's variable
// quotients stay inside the bounds of vq (differences of such values are 0 or in [2^-71, 2^50),
// so their quotients lie in [2^-121, 2^121])
__device__ __forceinline__ bool s_range(float v) {
    const unsigned u2 = __float_as_uint(v) << 1;
    return (u2 == 0u) | ((u2 - (79u << 24)) < (97u << 24));
}
// 2^-20 <= v < 2^21 (positive): the range of the fixed denominators (dx, dz, densities, ...)
__device__ __forceinline__ bool d_range(float v) { return (__float_as_uint(v) - (107u << 23)) < (41u << 23); }

// ---- FP64-reciprocal division: RN32(a/b) = RN32(RN64(a * y)) for y = 1/b to within 2^-51
//
// For floats a, b the quotient a/b is never a float rounding boundary (a midpoint between
// neighbouring floats, subnormal ones included) and, when it is not a float itself, lies at a
// relative distance of at least 2^-49 from every boundary: with A, B the 24-bit integer
// significands, a boundary M near A/B gives |A/B - M| >= 1/(B 2^25) >= 2^-49 |A/B|. The product
// a*y rounded to double is within 2^-52 + 2^-51 < 2^-49 of a/b, so it lies on the same side of
// every boundary and rounding it to float gives the IEEE quotient, for every float a and every
// b with y accurate (zeros, subnormals, infinities and overflow included, since the double
// product neither underflows nor overflows). No range checks are needed.
__device__ __forceinline__ float div64(float a, double y) { return __double2float_rn((double)a * y); }

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

// division policies of the fast tracer cell: cdiv(a, b, y) with y = 1/b prepared once (type R),
// vdiv(a, b) for a variable denominator, div3(a) = a / 3
struct Div32 {  // Markstein on FP32 FMAs: exact inside ranges the caller guards
    using R = float;
    static constexpr bool kGuarded = true;
    __device__ __forceinline__ static R rcp(float b) { return 1.0f / b; }
    __device__ __forceinline__ static float cdiv(float a, float b, R y) { return mq2(a, b, y); }
    __device__ __forceinline__ static float vdiv(float a, float b) { return vq(a, b); }
    __device__ __forceinline__ static float div3(float a) { return mq1(a, 3.0f, 1.0f / 3.0f); }
};
struct Div64 {  // FP64 reciprocal: exact for every input
    using R = double;
    static constexpr bool kGuarded = false;
    __device__ __forceinline__ static R rcp(float b) { return 1.0 / (double)b; }
    __device__ __forceinline__ static float cdiv(float a, float, R y) { return div64(a, y); }
    __device__ __forceinline__ static float vdiv(float a, float b) { return div64(a, rcp64(b)); }
    __device__ __forceinline__ static float div3(float a) { return div64(a, 1.0 / 3.0); }
};

// division policies for the templated tracer arithmetic: div(a, b) with a variable
// denominator, divr(a, b, y) with y = RN(1/b) prepared in advance
template <class T>
struct DivIEEE {
    __device__ __forceinline__ static T div(T a, T b, bool&) { return a / b; }
    __device__ __forceinline__ static T divr(T a, T b, T, bool&) { return a / b; }
};

struct DivMarkstein {
    __device__ __forceinline__ static float div(float a, float b, bool&) { return a / b; }
    __device__ __forceinline__ static float divr(float a, float b, float y, bool& bad) { return mdiv_r(a, b, y, bad); }
};

}  // namespace moist
