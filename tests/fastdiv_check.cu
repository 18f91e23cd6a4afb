// GPU checks of the branch-free divisions of moist2d_b200/csrc/fastdiv.cuh against CUDA's IEEE
// division (div.rn), bit for bit (any NaN matches any NaN). Every mode prints one line per case:
//
//   div64 b...        every float numerator a (all 2^32 patterns) divided by each b through the
//                     variable (rcp64) and prepared (1 / (double)b) forms of Div64, counting only
//                     quotients its subnormal guard lets through, and of Div64X, counting all:
//                     "<b> <mism64_v> <mism64_c> <guarded> <mism64x_v> <mism64x_c>"
//   random n seed     n random (a, b) bit patterns of every class (zeros, subnormals, infinities,
//                     NaN), same columns: "random <mism64_v> <mism64_c> <guarded> <mism64x_v>
//                     <mism64x_c> <vdiv_skipped>" (the variable form needs b finite and nonzero)
//   rcp64             max |1 - b * rcp64(b)| over every finite nonzero float b: "rcp64 <max * 2^53>"
//   minmax            jmin_f / jmax_f vs Julia's min / max on special values and random pairs: "minmax <mismatches>"
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "../moist2d_b200/csrc/fastdiv.cuh"
#include "../moist2d_b200/csrc/moist_math.h"

using namespace moist;

__device__ __forceinline__ bool same(float x, float y) {
    return (x != x && y != y) || __float_as_uint(x) == __float_as_uint(y);
}

__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {  // splitmix64 finaliser
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

// out[0..4]: Div64 variable / prepared mismatches (unguarded only), guarded, Div64X variable / prepared
__device__ __forceinline__ void check_pair(float a, float b, double yb, bool with_v, unsigned long long* c) {
    const float r = a / b;
    unsigned gv = ~0u, gc = ~0u, g = ~0u;
    const float qc = Div64::cdiv(a, b, yb, gc);
    c[1] += !guard_hit(gc) && !same(qc, r);
    c[2] += guard_hit(gc);
    c[4] += !same(Div64X::cdiv(a, b, yb, g), r);
    if (with_v) {
        const float qv = Div64::vdiv(a, b, gv);
        c[0] += !guard_hit(gv) && !same(qv, r);
        c[3] += !same(Div64X::vdiv(a, b, g), r);
    }
}

__global__ void k_div64(float b, unsigned long long* out) {
    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    const double yb = 1.0 / (double)b;
    unsigned long long c[5] = {0, 0, 0, 0, 0};
    for (unsigned long long u = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; u < (1ull << 32); u += stride)
        check_pair(__uint_as_float((unsigned)u), b, yb, true, c);
    for (int j = 0; j < 5; j++) atomicAdd(out + j, c[j]);
}

__global__ void k_random(unsigned long long n, unsigned long long seed, unsigned long long* out) {
    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    unsigned long long c[5] = {0, 0, 0, 0, 0}, skip = 0;
    for (unsigned long long j = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; j < n; j += stride) {
        const unsigned long long h = mix64(seed * 0x9e3779b97f4a7c15ull + j);
        const float a = __uint_as_float((unsigned)h), b = __uint_as_float((unsigned)(h >> 32));
        const bool with_v = !(b == 0.0f || fabsf(b) > 3.4028235e38f || b != b);
        skip += !with_v;
        check_pair(a, b, 1.0 / (double)b, with_v, c);
    }
    for (int j = 0; j < 5; j++) atomicAdd(out + j, c[j]);
    atomicAdd(out + 5, skip);
}

__global__ void k_rcp64(unsigned long long* out) {  // max residual in units of 2^-53 (as an integer)
    unsigned long long worst = 0;
    for (unsigned long long u = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; u < (1ull << 32);
         u += (unsigned long long)gridDim.x * blockDim.x) {
        const float b = __uint_as_float((unsigned)u);
        if (b == 0.0f || !(fabsf(b) <= 3.4028235e38f)) continue;
        const double e = fabs(__fma_rn(-(double)b, rcp64(b), 1.0)) * 0x1p53;
        const unsigned long long q = (unsigned long long)(e * 1024.0);
        worst = q > worst ? q : worst;
    }
    atomicMax(out, worst);
}

__global__ void k_minmax(unsigned long long* out) {
    const float sp[] = {0.0f, -0.0f, 1.0f, -1.0f, __int_as_float(0x7f800000), __int_as_float(0xff800000),
                        __int_as_float(0x7fc00000), 1e-40f, -1e-40f, 2.0f, 3.4e38f};
    unsigned long long n = 0;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        for (float x : sp)
            for (float y : sp) n += !same(mm::jmin(x, y), jmin_f(x, y)) + !same(mm::jmax(x, y), jmax_f(x, y));
    }
    unsigned long long st = 12345ull + 7919ull * (blockIdx.x * blockDim.x + threadIdx.x);
    for (int it = 0; it < 4096; it++) {
        st = mix64(st);
        const float x = __uint_as_float((unsigned)st);
        const float y = (it & 1) ? __uint_as_float((unsigned)(st >> 32)) : x * 1.0000001f;
        n += !same(mm::jmin(x, y), jmin_f(x, y)) + !same(mm::jmax(x, y), jmax_f(x, y));
    }
    atomicAdd(out, n);
}

int main(int argc, char** argv) {
    if (argc < 2) return 2;
    unsigned long long* d;
    if (cudaMalloc(&d, 64) != cudaSuccess) return 2;
    unsigned long long h[8];
    auto run = [&](auto launch) {
        cudaMemset(d, 0, 64);
        launch();
        if (cudaMemcpy(h, d, 64, cudaMemcpyDeviceToHost) != cudaSuccess) {
            printf("cuda error\n");
            exit(2);
        }
    };
    const dim3 g(148 * 8), b(256);
    int fails = 0;
    const char* mode = argv[1];
    if (!strcmp(mode, "div64")) {
        for (int j = 2; j < argc; j++) {
            const float bv = strtof(argv[j], nullptr);
            run([&] { k_div64<<<g, b>>>(bv, d); });
            printf("%a %llu %llu %llu %llu %llu\n", bv, h[0], h[1], h[2], h[3], h[4]);
            fails += h[0] != 0 || h[1] != 0 || h[3] != 0 || h[4] != 0;
        }
    } else if (!strcmp(mode, "random")) {
        const unsigned long long n = strtoull(argv[2], nullptr, 10), seed = strtoull(argv[3], nullptr, 10);
        run([&] { k_random<<<g, b>>>(n, seed, d); });
        printf("random %llu %llu %llu %llu %llu %llu\n", h[0], h[1], h[2], h[3], h[4], h[5]);
        fails += h[0] != 0 || h[1] != 0 || h[3] != 0 || h[4] != 0;
    } else if (!strcmp(mode, "rcp64")) {
        run([&] { k_rcp64<<<g, b>>>(d); });
        printf("rcp64 %.4f\n", h[0] / 1024.0);
    } else if (!strcmp(mode, "minmax")) {
        run([&] { k_minmax<<<dim3(148), b>>>(d); });
        printf("minmax %llu\n", h[0]);
        fails += h[0] != 0;
    } else {
        return 2;
    }
    cudaFree(d);
    return fails ? 1 : 0;
}
