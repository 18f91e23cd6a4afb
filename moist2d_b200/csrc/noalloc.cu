// noalloc.cu - an allocation-free entry point: the vertically implicit w-p column solve
// (implicit_correction!) for many columns at once, on device buffers the caller owns.
//
// Who needs it: callers that must not have a library allocate device memory behind them. A
// Julia host routes every device allocation through CUDA.jl's memory pool and counts on it to
// reclaim memory under pressure; a host with a fixed device-memory budget reserves all of it
// up front and cannot meet an out-of-memory failure in the middle of a run; and a host that
// keeps other streams busy cannot afford cudaFree, which waits for the whole device.
// moist_implicit_correction allocates its column buffers on every call; this variant
// allocates nothing. The grid vectors travel in the kernel's parameter block (so the call
// issues no host-to-device copy either), and the scratch of the elimination (the modified
// super-diagonal and right-hand side of every column) lives in one file-scope __device__ array
// of fixed size that every GPU loading the library holds until the process exits.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/moist2d.h"
#include "model.cuh"

namespace {

constexpr size_t kScratchDoubles = MOIST_NOALLOC_SCRATCH_BYTES / sizeof(double);
static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

// the grid vectors dz and z, passed by value in the kernel's parameter block (at most
// MOIST_NOALLOC_MAX_NZ levels: 16 KiB in Float64, within the 32 KiB parameter limit)
template <class T>
struct ColumnGrid {
    T dz[MOIST_NOALLOC_MAX_NZ];
    T z[MOIST_NOALLOC_MAX_NZ];
};

// device address of g_noalloc_scratch, looked up once per device with that device current
constexpr int kMaxDevices = 64;
void* g_scratch_addr[kMaxDevices] = {nullptr};
std::mutex g_scratch_mutex;

void put_msg(char* err, size_t errlen, const char* msg) {
    if (err && errlen) {
        std::strncpy(err, msg, errlen - 1);
        err[errlen - 1] = '\0';
    }
}

// one thread per column; column j of each (nz, ncols) array starts at j * nz (z fastest, the
// reference layout). Same arithmetic as implicit_correction! (moist.jl:974-1030) and
// solve_tridiagonal! (moist.jl:952-971), with the elimination in TT.
template <class T, class TT>
__global__ void k_implicit_columns_noalloc(int nz, int ncols, T grav, T beta, T* rho_w, const T* drho_w,
                                          const T* theta, const T* rt2pres, T dt,
                                          const __grid_constant__ ColumnGrid<T> grid, TT* work) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= ncols) return;
    const T* dz = grid.dz;  // every thread reads the same level at the same time: broadcast
    const T* z = grid.z;
    const int n = nz - 1, ke = nz - 1;
    T* w = rho_w + (size_t)j * nz;
    const T* dw = drho_w + (size_t)j * nz;
    const T* th = theta + (size_t)j * nz;
    const T* r2 = rt2pres + (size_t)j * nz;
    TT* cps = work + (size_t)j * 2 * n;
    TT* dps = cps + n;
    const T fact_tp = T(0.5) * (T(1.0) + beta);
    const T fact_tm = T(0.5) * (T(1.0) - beta);
    const T dt_tp2 = (dt * fact_tp) * (dt * fact_tp);
    const T fact = fact_tm / fact_tp;
    TT cp_prev = TT(0), d_prev = TT(0);
    for (int k = 0; k < n; k++) {
        const T th_cur = moist::f2h(th[k], th[k + 1], dz[k], dz[k + 1]);
        const T th_prev = k > 0 ? moist::f2h(th[k - 1], th[k], dz[k - 1], dz[k]) : T(0);
        const T th_next = (k + 1 <= ke - 1) ? moist::f2h(th[k + 1], th[k + 2], dz[k + 1], dz[k + 2]) : T(0);
        const T b = dt_tp2 * (r2[k] / dz[k] + r2[k + 1] / dz[k + 1]) * th_cur / (z[k + 1] - z[k]);
        const T a = (k > 0) ? -dt_tp2 * (r2[k] * th_prev / ((z[k + 1] - z[k]) * dz[k]) - grav / (dz[k] + dz[k + 1])) : T(0);
        const T c = (k < ke - 1) ? -dt_tp2 * (r2[k + 1] * th_next / ((z[k + 1] - z[k]) * dz[k + 1]) + grav / (dz[k] + dz[k + 1])) : T(0);
        T d = w[k] + dw[k];
        if (k > 0) d -= a * fact * w[k];
        d -= b * fact * w[k];
        const T bb = b + T(1.0);
        if (k < ke - 1) d -= c * fact * w[k + 1];
        TT piv, cpk, dpk;
        if (k == 0) {
            piv = (TT)bb;
            cpk = (TT)c / piv;
            dpk = (TT)d / piv;
        } else {
            piv = (TT)bb - (TT)a * cp_prev;
            cpk = (TT)c / piv;
            dpk = ((TT)d - (TT)a * d_prev) / piv;
        }
        cps[k] = cpk;
        dps[k] = dpk;
        cp_prev = cpk;
        d_prev = dpk;
    }
    TT x = dps[n - 1];
    w[n - 1] = (T)x;
    for (int k = n - 2; k >= 0; k--) {
        x = dps[k] - cps[k] * x;
        w[k] = (T)x;
    }
}

template <class T, class TT>
int run_noalloc(const moist_params* p, int ncols, void* rho_w, const void* drho_w, const void* theta,
                const void* rt2pres, double dt, cudaStream_t st, double* base, char* err, size_t errlen) {
    const int nz = p->nz;
    // scratch: the elimination work (TT, 2 (nz-1) per column)
    const size_t work_bytes = 2 * (size_t)(nz - 1) * ncols * sizeof(TT);
    if (work_bytes > MOIST_NOALLOC_SCRATCH_BYTES) {
        char msg[256];
        std::snprintf(msg, sizeof msg,
                      "moist_implicit_correction_noalloc: %d columns of %d levels need %zu scratch bytes, "
                      "more than the fixed %d-byte scratch array",
                      ncols, nz, work_bytes, (int)MOIST_NOALLOC_SCRATCH_BYTES);
        put_msg(err, errlen, msg);
        return MOIST_ERR_ARG;
    }
    ColumnGrid<T> grid;
    std::memset(&grid, 0, sizeof grid);
    std::memcpy(grid.dz, p->dz, nz * sizeof(T));
    std::memcpy(grid.z, p->z, nz * sizeof(T));
    TT* work = reinterpret_cast<TT*>(base);
    const int threads = 128;
    k_implicit_columns_noalloc<T, TT><<<(ncols + threads - 1) / threads, threads, 0, st>>>(
        nz, ncols, (T)p->grav, (T)p->beta_offcenter, (T*)rho_w, (const T*)drho_w, (const T*)theta,
        (const T*)rt2pres, (T)dt, grid, work);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        put_msg(err, errlen, cudaGetErrorString(e));
        return MOIST_ERR_CUDA;
    }
    return MOIST_OK;
}

}  // namespace

extern "C" {
#pragma GCC visibility push(default)

int moist_implicit_correction_noalloc(const moist_params* p, int precision, int flags, int ncols, void* rho_w,
                                      const void* drho_w, const void* theta, const void* rt2pres, double dt,
                                      void* stream, char* err, size_t errlen) {
    put_msg(err, errlen, "");
    if (!p || !p->dz || !p->z || p->nz < 2 || ncols < 0 || !rho_w || !drho_w || !theta || !rt2pres) {
        put_msg(err, errlen, "moist_implicit_correction_noalloc: invalid argument");
        return MOIST_ERR_ARG;
    }
    if (p->nz > MOIST_NOALLOC_MAX_NZ) {
        char msg[160];
        std::snprintf(msg, sizeof msg, "moist_implicit_correction_noalloc: nz = %d is above the limit of %d levels",
                      p->nz, (int)MOIST_NOALLOC_MAX_NZ);
        put_msg(err, errlen, msg);
        return MOIST_ERR_ARG;
    }
    if (precision != MOIST_F32 && precision != MOIST_F64) {
        put_msg(err, errlen, "moist_implicit_correction_noalloc: unknown precision");
        return MOIST_ERR_ARG;
    }
    if (ncols == 0) return MOIST_OK;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        put_msg(err, errlen, e != cudaSuccess ? cudaGetErrorString(e) : "device index out of range");
        return MOIST_ERR_CUDA;
    }
    void* base;
    {
        // first call on this device: look up the scratch array's device address with the device
        // current (the host-side symbol is only a stand-in and must never reach a kernel). The
        // address is kept for the life of the process; it is not looked up again after a
        // cudaDeviceReset, so no call may follow a reset of the device.
        std::lock_guard<std::mutex> lock(g_scratch_mutex);
        if (!g_scratch_addr[dev]) {
            void* ptr = nullptr;
            e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
            if (e != cudaSuccess || !ptr) {
                put_msg(err, errlen, e != cudaSuccess ? cudaGetErrorString(e) : "null symbol address");
                return MOIST_ERR_CUDA;
            }
            g_scratch_addr[dev] = ptr;
        }
        base = g_scratch_addr[dev];
    }
    cudaStream_t st = (cudaStream_t)stream;
    double* b = (double*)base;
    if (precision == MOIST_F64) return run_noalloc<double, double>(p, ncols, rho_w, drho_w, theta, rt2pres, dt, st, b, err, errlen);
    if (flags & MOIST_FLAG_TRI_NATIVE) return run_noalloc<float, float>(p, ncols, rho_w, drho_w, theta, rt2pres, dt, st, b, err, errlen);
    return run_noalloc<float, double>(p, ncols, rho_w, drho_w, theta, rt2pres, dt, st, b, err, errlen);
}

#pragma GCC visibility pop
}  // extern "C"
