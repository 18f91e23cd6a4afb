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
