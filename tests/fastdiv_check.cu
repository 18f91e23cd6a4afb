// Exhaustive check of moist::mdiv_r (moist2d_b200/csrc/fastdiv.cuh) against IEEE division:
// every finite numerator a with a == 0 or 2^-100 <= |a| <= 2^100 (the routine's unflagged
// range), for each denominator given on the command line. Prints "<b> <mismatches> <flagged>".
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include "../moist2d_b200/csrc/fastdiv.cuh"

__global__ void check(float b, float y, unsigned long long* mism, unsigned long long* flagged) {
    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    unsigned long long mm = 0, ff = 0;
    for (unsigned long long u = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; u < (1ull << 32); u += stride) {
        const float a = __uint_as_float((unsigned)u);
        if (!isfinite(a)) continue;
        bool bad = false;
        const float q = moist::mdiv_r(a, b, y, bad);
        if (bad) { ff++; continue; }
        const float r = a / b;
        if (__float_as_uint(q) != __float_as_uint(r)) mm++;
    }
    atomicAdd(mism, mm);
    atomicAdd(flagged, ff);
}

int main(int argc, char** argv) {
    unsigned long long *d;
    cudaMalloc(&d, 16);
    int fails = 0;
    for (int j = 1; j < argc; j++) {
        const float b = strtof(argv[j], nullptr);
        const float y = 1.0f / b;  // RN(1/b) (host IEEE division)
        cudaMemset(d, 0, 16);
        check<<<148 * 16, 256>>>(b, y, d, d + 1);
        unsigned long long h[2];
        if (cudaMemcpy(h, d, 16, cudaMemcpyDeviceToHost) != cudaSuccess) { printf("cuda error\n"); return 2; }
        printf("%a %llu %llu\n", b, h[0], h[1]);
        fails += h[0] != 0;
    }
    return fails ? 1 : 0;
}
