// tracer_tiles.cuh - the reference's in-place Gauss-Seidel tracer sweep, computed in parallel
// tiles and repaired to a bitwise fixed point.
//
// The reference updates rho_q in place in lexicographic order (moist.jl:1469-1518), so cell
// (k, i) reads the updated values at (k, i-1), (k, i-2), (k-1, i), (k-2, i) and the
// stage-start values everywhere else. Write F for the map "recompute every cell from the
// current values of its predecessors": the reference result is the unique fixed point of F
// (unique by induction along the dependency order). Here the domain is cut into 32x32 tiles.
// Inside a tile the order is exact: one warp per tracer, lane r owns row z0+r and processes
// column c at wavefront step c + r, receiving the row below through warp shuffles. Across tile
// boundaries each tile starts from speculative values of its left and bottom neighbours'
// boundary strips (the stage-start values), publishes its own right and top strips after
// every pass, and is recomputed only when a neighbour's strip changed. A pass in which no
// strip changes leaves every tile computed from its neighbours' final values: a fixed point,
// hence the reference's result bit for bit. Influence between cells decays roughly like the
// Courant number per cell, so two or three passes suffice; the pass count is bounded by
// tiles_x + tiles_z + 1 (information crosses one tile per pass).
//
// The kernel is persistent (cooperative launch, all tiles resident); passes are separated by
// a grid barrier whose wait is bounded: on timeout it records MOIST_ERR_TIMEOUT and returns.
#pragma once

#include "fastdiv.cuh"
#include "kernels.cuh"

namespace moist {

constexpr int TT_W = 32;       // tile width (columns) = tile height (rows) = warp size
constexpr int TT_S = TT_W + 2; // staged extent with a two-cell halo

struct TileCtl {
    int tiles_x, tiles_z, ntiles, max_pass;
    int* ver;           // dataflow sweep: [3][ntiles] words (version << 1 | final) of each tile's strips
    unsigned* bar;      // [0] arrival counter, [1] generation
    int* changed;       // [2][3][ntiles][2] per pass parity: rows whose right-strip entries changed, columns whose top-strip entries changed (bit masks)
    int* any_changed;   // [max_pass + 1]
    int* passes;        // out: passes run
    int* timeout;       // out: barrier timeout flag
    long long spin_limit;
    unsigned long long* pass_ts;  // optional diagnostic [max_pass + 3]: globaltimer at the start of each
                                  // pass, and at [max_pass + 2] when block 0 leaves
    int* pass_work;               // optional diagnostic: [pass] warps that recomputed their tile
};

__device__ __forceinline__ unsigned long long globaltimer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// bounded grid barrier; every block must call it the same number of times
__device__ __forceinline__ bool grid_barrier(const TileCtl& c, unsigned nblocks) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned* vb = c.bar;
        const unsigned gen = vb[1];
        __threadfence();
        const unsigned arrived = atomicAdd(c.bar, 1u);
        int ok = 1;
        if (arrived == nblocks - 1) {
            c.bar[0] = 0;
            __threadfence();
            atomicAdd(c.bar + 1, 1u);
        } else {
            const long long t0 = clock64();
            while (vb[1] == gen) {
                if (clock64() - t0 > c.spin_limit) {
                    ok = 0;
                    atomicExch(c.timeout, 1);
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
        s_ok = ok && (*(volatile int*)c.timeout == 0);
    }
    __syncthreads();
    return s_ok != 0;
}

// Per-row reciprocals RN(1/b) of the sweep-constant denominators of the tracer update (ignored
// by DivIEEE, whose divr divides).
template <class T>
struct RowRcp {
    T dx, dz_k, sum_kp, sum_km, zd_kp, zd_km;
};

template <class D, class T>
__device__ __forceinline__ T koren_d(T r, bool& bad) {  // moist.jl:846
    return jmax(T(0.0), jmin(T(2.0) * r, jmin(D::divr(T(1.0) + T(2.0) * r, T(3.0), T(1.0) / T(3.0), bad), T(2.0))));
}

template <class D, class T>
__device__ __forceinline__ T f2h_d(T vf1, T vf2, T dz1, T dz2, T r_sum, bool& bad) {  // moist.jl:249
    return D::divr(vf1 * dz2 + vf2 * dz1, dz1 + dz2, r_sum, bad);
}

// limited_flux_x / limited_flux_z of model.cuh with the division policy D
template <class D, class T>
__device__ __forceinline__ T lflux_x(T vel, T s_m1, T s_0, T s_p1, T s_p2, T EPS, bool& bad) {
    const bool pos = vel > EPS, neg = vel < -EPS;
    const T r_num = pos ? (s_p1 - s_0) : (s_0 - s_p1);
    const T r_den = pos ? (s_0 - s_m1) : (s_p1 - s_p2);
    const T q = D::div(r_num, r_den, bad);
    const T r = mm::mabs(r_den) < EPS ? T(1.0) : q;
    const T lim = (pos ? s_0 : s_p1) + T(0.5) * koren_d<D>(r, bad) * r_den;
    const T cen = T(0.5) * (s_0 + s_p1);
    return ((pos || neg) ? lim : cen) * vel;
}

template <class D, class T>
__device__ __forceinline__ T lflux_z(T vel, T s_m1, T s_0, T s_p1, T s_p2, int k, int nz, T dz_k, T dz_kp1,
                                     T r_sum, T lin_k, T lin_kp1, T dt_big, T EPS, bool& bad) {
    const bool pos = vel > EPS, neg = vel < -EPS;
    const T f2 = f2h_d<D>(s_0, s_p1, dz_k, dz_kp1, r_sum, bad);
    const T clamp = jmin(f2, D::div(pos ? lin_k : lin_kp1, pos ? (vel * dt_big) : (-vel * dt_big), bad));
    const T r_num = pos ? (s_p1 - s_0) : (s_0 - s_p1);
    const T r_den = pos ? (s_0 - s_m1) : (s_p1 - s_p2);
    const T q = D::div(r_num, r_den, bad);
    const T r = mm::mabs(r_den) < EPS ? T(1.0) : q;
    const T half = T(0.5) * koren_d<D>(r, bad) * r_den;
    const T lim = pos ? (s_0 + half) : (s_p1 - half);
    const T face = pos ? ((k == 0) ? clamp : lim) : (neg ? ((k == nz - 2) ? clamp : lim) : f2);
    return face * vel;
}

// The tracer update of one cell (moist.jl:1479-1515) from values already gathered: the same
// operations, in the same order, as tracer_cell in kernels.cuh, with the division policy D
// (DivIEEE: plain IEEE division; used for Float64 and for the cells the fast cell leaves).
template <class D, class T>
__device__ __forceinline__ T tracer_cell_t(const DevParams<T>& p, int k, T dt_stage, T s_c, T s_ip1, T s_ip2,
                                           T s_kp1, T s_kp2, T s_im1, T s_im2, T s_km1, T s_km2, T lin_km1,
                                           T lin_k, T lin_kp1, T mfx_i, T mfx_im, T mfz_k, T mfz_km, T rho_c,
                                           T rho_ip, T rho_im, T rho_kp, T rho_km, T dz_k, T dz_kp1, T dz_km1,
                                           T z_k, T z_kp1, T z_km1, T q0, T dph, const RowRcp<T>& rr, bool& bad) {
    const int nz = p.nz, ke = nz - 1;
    const T EPS = p.EPS, dx = p.dx;
    const T fx_ip = lflux_x<D>(mfx_i, s_im1, s_c, s_ip1, s_ip2, EPS, bad);
    const T fx_im = lflux_x<D>(mfx_im, s_im2, s_im1, s_c, s_ip1, EPS, bad);
    const T adv_x = D::divr(fx_ip - fx_im, dx, rr.dx, bad);
    const T fz_kp = k == ke ? T(0.0)
                            : lflux_z<D>(mfz_k, s_km1, s_c, s_kp1, s_kp2, k, nz, dz_k, dz_kp1, rr.sum_kp, lin_k,
                                         lin_kp1, p.dt, EPS, bad);
    const T fz_km = k == 0 ? T(0.0)
                           : lflux_z<D>(mfz_km, s_km2, s_km1, s_c, s_kp1, k - 1, nz, dz_km1, dz_k, rr.sum_km,
                                        lin_km1, lin_k, p.dt, EPS, bad);
    const T adv_z = D::divr(fz_kp - fz_km, dz_k, rr.dz_k, bad);
    const T advection = -(adv_x + adv_z);
    const T scalar_kp = k == ke ? T(0.0) : s_kp1;
    const T scalar_km = k == 0 ? T(0.0) : s_km1;
    const T dsdx_ip = D::divr((rho_ip + rho_c) * T(0.5) * (s_ip1 - s_c), dx, rr.dx, bad);
    const T dsdx_im = D::divr((rho_c + rho_im) * T(0.5) * (s_c - s_im1), dx, rr.dx, bad);
    const T diff_x = D::divr(p.kappa * (dsdx_ip - dsdx_im), dx, rr.dx, bad);
    const T dsdz_kp = k == ke ? T(0.0)
                              : D::divr(f2h_d<D>(rho_kp, rho_c, dz_kp1, dz_k, rr.sum_kp, bad) * (scalar_kp - s_c),
                                        z_kp1 - z_k, rr.zd_kp, bad);
    const T dsdz_km = k == 0 ? T(0.0)
                             : D::divr(f2h_d<D>(rho_c, rho_km, dz_k, dz_km1, rr.sum_km, bad) * (s_c - scalar_km),
                                       z_k - z_km1, rr.zd_km, bad);
    const T diff_z = D::divr(p.kappa * (dsdz_kp - dsdz_km), dz_k, rr.dz_k, bad);
    const T diffusion = diff_x + diff_z;
    return q0 + dt_stage * (advection + diffusion + dph);
}

// ---- the Float32 cell without branches (the fast path of the tiled sweep)
//
// Same operations and order as tracer_cell_t, with every division done by the branch-free
// primitives of fastdiv.cuh and every select an explicit selp, so the four face fluxes and the
// diffusion terms overlap in one basic block instead of waiting on one another. Those
// primitives equal IEEE division inside stated ranges, which hold when (checked by the caller)
// the stencil's stage-start mixing ratios are 0 or 2^-48 <= |s| < 2^49 and the densities and
// grid constants lie in [2^-20, 2^21), and (checked here) the four updated neighbours are in
// the same range and the five numerators that can still come out tiny or huge do not: then
// every variable quotient lies in [2^-121, 2^121] and every fixed-denominator numerator in
// [2^-100, 2^100]. Otherwise `bad` is set and the caller recomputes the cell with IEEE
// division. The two clamp quotients of the vertical limiter (used on four rows only) come
// precomputed with IEEE division in cl_kp / cl_km.

template <class D>
__device__ __forceinline__ float koren_f(float r) {  // moist.jl:846
    const float t = 2.0f * r;
    return jmax_f(0.0f, jmin_f(t, jmin_f(D::div3(1.0f + t), 2.0f)));
}

// (pos || neg) is |vel| > EPS: both are false for a NaN velocity
template <class D>
__device__ __forceinline__ float lflux_x_f(float vel, float s_m1, float s_0, float s_p1, float s_p2, float EPS, unsigned& g) {
    const float r_num = sel_gt(vel, EPS, s_p1 - s_0, s_0 - s_p1);
    const float r_den = sel_gt(vel, EPS, s_0 - s_m1, s_p1 - s_p2);
    const float r = sel_lt(fabsf(r_den), EPS, 1.0f, D::vdiv(r_num, r_den, g));
    const float lim = sel_gt(vel, EPS, s_0, s_p1) + 0.5f * koren_f<D>(r) * r_den;
    const float cen = 0.5f * (s_0 + s_p1);
    return sel_gt(fabsf(vel), EPS, lim, cen) * vel;
}

// face k+1/2 of limited_flux_z with kk = the face's lower cell; at0 / atnm2 are kk == 0 / nz-2
template <class D>
__device__ __forceinline__ float lflux_z_f(float vel, float s_m1, float s_0, float s_p1, float s_p2, unsigned at0,
                                           unsigned atnm2, float dz_a, float dz_b, float sum_ab, typename D::R rsum_ab, float cl,
                                           float EPS, unsigned& g) {
    const float f2 = D::cdiv(s_0 * dz_b + s_p1 * dz_a, sum_ab, rsum_ab, g);
    const float clamp = jmin_f(f2, cl);
    const float r_num = sel_gt(vel, EPS, s_p1 - s_0, s_0 - s_p1);
    const float r_den = sel_gt(vel, EPS, s_0 - s_m1, s_p1 - s_p2);
    const float r = sel_lt(fabsf(r_den), EPS, 1.0f, D::vdiv(r_num, r_den, g));
    const float half = 0.5f * koren_f<D>(r) * r_den;
    const float lim = sel_gt(vel, EPS, s_0 + half, s_p1 - half);
    // pos: kk == 0 takes the clamp; neg: kk == nz-2 takes it; neither: the face average f2
    const float pos_face = sel_u(at0, clamp, lim), neg_face = sel_u(atnm2, clamp, lim);
    const float face = sel_gt(vel, EPS, pos_face, sel_lt(vel, -EPS, neg_face, f2));
    return face * vel;
}

// per-lane (row) constants of the fast cell (reciprocals in the policy's type R); flags are 0 / 1
template <class R>
struct FastRow {
    float dx, dz_k, dz_kp1, dz_km1, sum_kp, sum_km, zd_kp, zd_km;
    R rdx, rdz_k, rsum_kp, rsum_km, rzd_kp, rzd_km;
    float kappa, EPS, dt_stage;
    unsigned k0, ke, kp_at0, kp_atnm2, km_at0, km_atnm2;
};

template <class D>
__device__ __forceinline__ float tracer_cell_f(const FastRow<typename D::R>& w, float s_c, float s_ip1, float s_ip2, float s_kp1,
                                               float s_kp2, float s_im1, float s_im2, float s_km1, float s_km2,
                                               float cl_kp, float cl_km, float mfx_i, float mfx_im, float mfz_k,
                                               float mfz_km, float rho_c, float rho_ip, float rho_im, float rho_kp,
                                               float rho_km, float q0, float dph, unsigned& g, bool& bad) {
    const float fx_ip = lflux_x_f<D>(mfx_i, s_im1, s_c, s_ip1, s_ip2, w.EPS, g);
    const float fx_im = lflux_x_f<D>(mfx_im, s_im2, s_im1, s_c, s_ip1, w.EPS, g);
    const float ndx = fx_ip - fx_im;
    const float adv_x = D::cdiv(ndx, w.dx, w.rdx, g);
    const float fz_kp = sel_u(w.ke, 0.0f,
                              lflux_z_f<D>(mfz_k, s_km1, s_c, s_kp1, s_kp2, w.kp_at0, w.kp_atnm2, w.dz_k, w.dz_kp1,
                                        w.sum_kp, w.rsum_kp, cl_kp, w.EPS, g));
    const float fz_km = sel_u(w.k0, 0.0f,
                              lflux_z_f<D>(mfz_km, s_km2, s_km1, s_c, s_kp1, w.km_at0, w.km_atnm2, w.dz_km1, w.dz_k,
                                        w.sum_km, w.rsum_km, cl_km, w.EPS, g));
    const float ndz = fz_kp - fz_km;
    const float adv_z = D::cdiv(ndz, w.dz_k, w.rdz_k, g);
    const float advection = -(adv_x + adv_z);
    const float scalar_kp = sel_u(w.ke, 0.0f, s_kp1);
    const float scalar_km = sel_u(w.k0, 0.0f, s_km1);
    const float dsdx_ip = D::cdiv((rho_ip + rho_c) * 0.5f * (s_ip1 - s_c), w.dx, w.rdx, g);
    const float dsdx_im = D::cdiv((rho_c + rho_im) * 0.5f * (s_c - s_im1), w.dx, w.rdx, g);
    const float kx = w.kappa * (dsdx_ip - dsdx_im);
    const float diff_x = D::cdiv(kx, w.dx, w.rdx, g);
    const float dsdz_kp = sel_u(w.ke, 0.0f,
                                D::cdiv(D::cdiv(rho_kp * w.dz_k + rho_c * w.dz_kp1, w.sum_kp, w.rsum_kp, g) * (scalar_kp - s_c),
                                        w.zd_kp, w.rzd_kp, g));
    const float dsdz_km = sel_u(w.k0, 0.0f,
                                D::cdiv(D::cdiv(rho_c * w.dz_km1 + rho_km * w.dz_k, w.sum_km, w.rsum_km, g) * (s_c - scalar_km),
                                        w.zd_km, w.rzd_km, g));
    const float kz = w.kappa * (dsdz_kp - dsdz_km);
    const float diff_z = D::cdiv(kz, w.dz_k, w.rdz_k, g);
    const float diffusion = diff_x + diff_z;
    const float q = q0 + w.dt_stage * (advection + diffusion + dph);
    bad = !(fabsf(q) <= 0x1.fffffep127f);  // non-finite results are left to IEEE division
    return q;
}

// q0, the phys tendency and the results are staged in shared memory for Float32; Float64
// reads and writes them in global memory so that enough tiles stay resident
using FastDiv = Div64;  // division policy of the Float32 fast cell (fastdiv.cuh); Div64X for its fallback

template <class T>
struct TileQ {
    typename FastDiv::R rrho[TT_W][TT_W + 2];  // 1/rho of the tile cells in the fast cell's form
    T snp[3][TT_W][TT_W + 2];  // per tracer: s = q / rho of the last pass (the rows a repair pass replays)
    T q0[3][TT_W][TT_W + 2];   // row stride 34: lane r reads column step - r, conflict-free
    T dph[3][TT_W][TT_W + 2];
    T qn[3][TT_W][TT_W + 2];
};
template <>
struct TileQ<double> {};
template <class T>
constexpr bool kStageQ = sizeof(T) == 4;

template <class T>
struct TileSmem {
    TileQ<T> q;
    T bot[3][2][TT_W];       // per tracer: the lower tile's top strip for the current pass
    T rho[TT_S][TT_S];       // rows z0-1 .. z0+32, cols x0-1 .. x0+32 (row stride 34: conflict-free wavefront reads)
    T mx[TT_W][TT_S];        // mfx faces x0-1 .. x0+31 (index c+1), rows z0 .. z0+31
    T mz[TT_W + 1][TT_S];    // mfz faces z0-1 .. z0+31 (index r+1), cols x0 .. x0+31
    T s[3][TT_S][TT_S];      // per tracer: stage-start s = q/rho, rows z0 .. z0+33, cols x0 .. x0+33
    T lin[3][TT_S + 1];      // per tracer: column 1 of the reference array (interior nx-2), rows z0-1 .. z0+33
    T strip_out[3][4][TT_W]; // per tracer: right strip cols x0+30, x0+31 (0, 1), top strip rows z0+30, z0+31 (2, 3)
    T cl[3][2][2][TT_W];     // per tracer: clamp quotients of the vertical limiter [kp, km][low, high row][column]
};

// the staging loops of k_tracer_tiles: every thread loads TT_BATCH elements (load(j) returns
// an element's values), then stores them (store(j, v)); elements j = threadIdx.x + u blockDim.x
constexpr int TT_BATCH = 8;
template <class T>
struct Pair {
    T x, y;
};
template <class T>
struct Triple {
    T x, y, z;
};
template <class V, class L, class S>
__device__ __forceinline__ void stage_batched(int total, L load, S store) {
    for (int j0 = threadIdx.x; j0 < total; j0 += TT_BATCH * (int)blockDim.x) {
        V v[TT_BATCH];
#pragma unroll
        for (int u = 0; u < TT_BATCH; u++) {
            const int j = j0 + u * (int)blockDim.x;
            if (j < total) v[u] = load(j);
        }
#pragma unroll
        for (int u = 0; u < TT_BATCH; u++) {
            const int j = j0 + u * (int)blockDim.x;
            if (j < total) store(j, v[u]);
        }
    }
}

// strips in global memory: [parity][tracer][tile][4][32]
template <class T>
__device__ __forceinline__ T* strip_ptr(T* strips, int parity, int t, int tile, int ntiles) {
    return strips + ((((size_t)parity * 3 + t) * ntiles + tile) * 4) * TT_W;
}
// the dataflow sweep keeps the last TT_RING versions of each tile's strips:
// [tracer][tile][version % TT_RING][4][32]
constexpr int TT_RING = 4;
template <class T>
__device__ __forceinline__ T* strip_ver_ptr(T* strips, int t, int tile, int ver, int ntiles) {
    return strips + ((((size_t)t * ntiles + tile) * TT_RING + (ver % TT_RING)) * 4) * TT_W;
}
__device__ __forceinline__ int ld_acquire(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(int* p, int v) {
    asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// DF = false: passes separated by grid barriers (all tiles advance pass by pass). DF = true: no
// grid barrier; every tile publishes numbered versions of its strips and recomputes whenever its
// left or lower neighbour publishes a new version, so a chain of changes crosses the tiles at the
// pace of its own work. A tile is final once it has computed from its neighbours' final strips
// (the left column and the bottom row of tiles have fixed inputs), which every tile reaches
// because the dependencies run only left-to-right and bottom-to-top.
template <class T, bool DF>
__global__ void __launch_bounds__(96) k_tracer_tiles(DevParams<T> p, TracerArgs<T> a, TileCtl ctl, T* strips,
                                                     const int* err) {
    extern __shared__ unsigned char smem_raw[];
    TileSmem<T>& sm = *reinterpret_cast<TileSmem<T>*>(smem_raw);
    const int nx = p.nx, nz = p.nz, P = p.P;
    const int tile = blockIdx.x;
    const int tx = tile % ctl.tiles_x, tz = tile / ctl.tiles_x;
    const int x0 = tx * TT_W, z0 = tz * TT_W;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const unsigned nblocks = gridDim.x;
    const bool halt = halted(err);  // uniform across the grid: every block still meets every barrier

    // ---- stage the stage-start values this tile reads (coalesced rows). Each thread issues the
    // loads of TT_BATCH elements before it stores (or divides) any, so that it waits for one
    // memory round trip per batch rather than per element.
    stage_batched<T>(TT_S * TT_S, [&](int j) {
        const int rr = j / TT_S, cc = j % TT_S;
        const int k = z0 - 1 + rr, i = wrapx(x0 - 1 + cc, nx);
        // columns beyond nx+1 are never read; the bound also keeps wrapx within one period
        return (k >= 0 && k < nz && x0 - 1 + cc < nx + 2) ? a.rho[MOIST_IDX(k, i)] : T(1);
    }, [&](int j, T v) { sm.rho[j / TT_S][j % TT_S] = v; });
    stage_batched<T>(TT_W * (TT_W + 1), [&](int j) {
        const int rr = j / (TT_W + 1), cc = j % (TT_W + 1);
        const int k = z0 + rr, i = wrapx(x0 - 1 + cc, nx);
        // faces x0-1 .. nx-1 only: face i-1 and i of the cells i < nx
        return (k < nz && x0 - 1 + cc < nx) ? a.mfx[MOIST_IDX(k, i)] : T(0);
    }, [&](int j, T v) { sm.mx[j / (TT_W + 1)][j % (TT_W + 1)] = v; });
    stage_batched<T>((TT_W + 1) * TT_W, [&](int j) {
        const int rr = j / TT_W, cc = j % TT_W;
        const int k = z0 - 1 + rr, i = x0 + cc;
        return (k >= 0 && k < nz && i < nx) ? a.mfz[MOIST_IDX(k, i)] : T(0);
    }, [&](int j, T v) { sm.mz[j / TT_W][j % TT_W] = v; });
    for (int t = 0; t < 3; t++) {
        const T* qo = a.q_old[t];
        // s = rho_q / rho, the quotient formed after the batch's loads
        stage_batched<Pair<T>>(TT_S * TT_S, [&](int j) {
            const int rr = j / TT_S, cc = j % TT_S;
            const int k = z0 + rr, i = wrapx(x0 + cc, nx);
            Pair<T> v{T(0), T(1)};
            if (k < nz && x0 + cc < nx + 2) {
                const size_t c = MOIST_IDX(k, i);
                v.x = qo[c];
                v.y = a.rho[c];
            }
            return v;
        }, [&](int j, Pair<T> v) { sm.s[t][j / TT_S][j % TT_S] = v.x / v.y; });
        for (int j = threadIdx.x; j < TT_S + 1; j += blockDim.x) {
            const int k = z0 - 1 + j;
            sm.lin[t][j] = (k >= 0 && k < nz) ? qo[MOIST_IDX(k, nx - 2)] : T(0);
        }
        if constexpr (kStageQ<T>) {
            stage_batched<Triple<T>>(TT_W * TT_W, [&](int j) {
                const int rr = j / TT_W, cc = j % TT_W;
                const int k = z0 + rr, i = x0 + cc;
                const bool ok = k < nz && i < nx;
                Triple<T> v{T(0), T(0), T(1)};
                if (ok) {
                    const size_t c = MOIST_IDX(k, i);
                    v.x = a.q0[t][c];
                    v.y = a.dphys[t][c];
                    if (t == 0) v.z = a.rho[c];
                }
                return v;
            }, [&](int j, Triple<T> v) {
                const int rr = j / TT_W, cc = j % TT_W;
                sm.q.q0[t][rr][cc] = v.x;
                sm.q.dph[t][rr][cc] = v.y;
                if (t == 0) sm.q.rrho[rr][cc] = FastDiv::rcp(v.z);
            });
        }
    }
    __syncthreads();
    const int t = warp;  // this warp's tracer
    if constexpr (kStageQ<T>) {
        // the clamp quotients lin / (+-vel dt) of limited_flux_z on the four rows that can use them:
        // face k+1/2 from rows k = 0 and nz-2, face k-1/2 from rows k = 1 and nz-1 (IEEE division)
        const int c = lane;
        for (int slot = 0; slot < 2; slot++) {
            T vkp = T(0), vkm = T(0);
            const int kp = slot == 0 ? 0 : nz - 2;  // face kp+1/2 between cells kp, kp+1
            const int km = slot == 0 ? 1 : nz - 1;  // face km-1/2 between cells km-1, km
            if (kp >= 0 && kp < nz - 1 && kp >= z0 && kp < z0 + TT_W && x0 + c < nx) {
                const T vel = sm.mz[kp - z0 + 1][c];
                const T lin_a = sm.lin[t][kp - z0 + 1], lin_b = sm.lin[t][kp - z0 + 2];
                vkp = vel > p.EPS ? lin_a / (vel * p.dt) : lin_b / (-vel * p.dt);
            }
            if (km >= 1 && km < nz && km >= z0 && km < z0 + TT_W && x0 + c < nx) {
                const T vel = sm.mz[km - z0][c];
                const T lin_a = sm.lin[t][km - z0], lin_b = sm.lin[t][km - z0 + 1];
                vkm = vel > p.EPS ? lin_a / (vel * p.dt) : lin_b / (-vel * p.dt);
            }
            sm.cl[t][0][slot][c] = vkp;
            sm.cl[t][1][slot][c] = vkm;
        }
        __syncwarp();
    }

    // ---- pass-0 strips: the stage-start values (the speculation)
    if constexpr (!DF) {
        T* out = strip_ptr(strips, 0, t, tile, ctl.ntiles);
        const int r = lane;
        __stcg(out + 0 * TT_W + r, sm.s[t][r][TT_W - 2]);
        __stcg(out + 1 * TT_W + r, sm.s[t][r][TT_W - 1]);
        __stcg(out + 2 * TT_W + r, sm.s[t][TT_W - 2][r]);
        __stcg(out + 3 * TT_W + r, sm.s[t][TT_W - 1][r]);
        if (!grid_barrier(ctl, nblocks)) return;
    }

    // lane-constant row data
    const int r = lane;
    const int k = z0 + r;
    const bool row_ok = k < nz;
    const int ke = nz - 1;
    const T dz_k = row_ok ? p.dz[k] : T(1);
    const T dz_kp1 = (row_ok && k < ke) ? p.dz[k + 1] : T(1);
    const T dz_km1 = (row_ok && k > 0) ? p.dz[k - 1] : T(1);
    const T z_k = row_ok ? p.z[k] : T(0);
    const T z_kp1 = (row_ok && k < ke) ? p.z[k + 1] : T(1);
    const T z_km1 = (row_ok && k > 0) ? p.z[k - 1] : T(-1);
    RowRcp<T> rr;  // IEEE reciprocals, correctly rounded
    rr.dx = T(1) / p.dx;
    rr.dz_k = T(1) / dz_k;
    rr.sum_kp = T(1) / (dz_k + dz_kp1);
    rr.sum_km = T(1) / (dz_km1 + dz_k);
    rr.zd_kp = T(1) / (z_kp1 - z_k);
    rr.zd_km = T(1) / (z_k - z_km1);
    FastRow<FastDiv::R> fw{};
    if constexpr (kStageQ<T>) {
        fw.dx = p.dx;
        fw.dz_k = dz_k;
        fw.dz_kp1 = dz_kp1;
        fw.dz_km1 = dz_km1;
        fw.sum_kp = dz_k + dz_kp1;
        fw.sum_km = dz_km1 + dz_k;
        fw.zd_kp = z_kp1 - z_k;
        fw.zd_km = z_k - z_km1;
        fw.rdx = FastDiv::rcp(fw.dx);
        fw.rdz_k = FastDiv::rcp(fw.dz_k);
        fw.rsum_kp = FastDiv::rcp(fw.sum_kp);
        fw.rsum_km = FastDiv::rcp(fw.sum_km);
        fw.rzd_kp = FastDiv::rcp(fw.zd_kp);
        fw.rzd_km = FastDiv::rcp(fw.zd_km);
        fw.kappa = p.kappa;
        fw.EPS = p.EPS;
        fw.dt_stage = a.dt;
        fw.k0 = k == 0;
        fw.ke = k == ke;
        fw.kp_at0 = k == 0;
        fw.kp_atnm2 = k == nz - 2;
        fw.km_at0 = k - 1 == 0;
        fw.km_atnm2 = k - 1 == nz - 2;
    }
    const int width = min(TT_W, nx - x0);
    const T* q0 = a.q0[t];
    const T* dph = a.dphys[t];
    T* qn = a.q_new[t];

    const int left = tx > 0 ? tile - 1 : -1;
    const int below = tz > 0 ? tile - ctl.tiles_x : -1;
    // Dataflow state (DF): the left-strip values (this lane's row) and the bottom strip (sm.bot)
    // of the last computation, the neighbours' versions they came from and the words read with
    // them (version << 1 | final), this tile's published version and the values it published.
    T in_p1 = T(0), in_p2 = T(0);
    int used_lv = 0, used_bv = 0, lw_cur = 0, bw_cur = 0, my_ver = 0;
    T pub[4] = {T(0), T(0), T(0), T(0)};
    // a strip entry the tile does not own (partial tile) keeps its stage-start value
    auto pass0 = [&](int q) {
        return q == 0 ? sm.s[t][r][TT_W - 2]
                      : q == 1 ? sm.s[t][r][TT_W - 1] : q == 2 ? sm.s[t][TT_W - 2][r] : sm.s[t][TT_W - 1][r];
    };
    if constexpr (DF) {
        // the inputs of the first computation are the neighbours' stage-start strips, which every
        // tile forms from the stage-start values exactly as the neighbour stages them: no wait
        auto s0 = [&](int kk, int ii) {
            return (kk >= 0 && kk < nz) ? a.q_old[t][MOIST_IDX(kk, ii)] / a.rho[MOIST_IDX(kk, ii)] : T(0);
        };
        in_p1 = row_ok ? s0(k, wrapx(x0 - 1, nx)) : T(0);
        in_p2 = row_ok ? s0(k, wrapx(x0 - 2, nx)) : T(0);
        const bool cin = below >= 0 && x0 + r < nx + 2;
        sm.bot[t][0][r] = cin ? s0(z0 - 2, wrapx(x0 + r, nx)) : T(0);  // row z0-2
        sm.bot[t][1][r] = cin ? s0(z0 - 1, wrapx(x0 + r, nx)) : T(0);  // row z0-1
        for (int q = 0; q < 4; q++) pub[q] = pass0(q);
        __syncwarp();
    }
    int* const my_word = ctl.ver + (size_t)t * ctl.ntiles + tile;
    int pass = 1;
    for (;; pass++) {
        if constexpr (!DF) {
            if (pass > ctl.max_pass) break;
        }
        const int cur = pass & 1, prv = cur ^ 1;
        const int* chg_prev = ctl.changed + ((size_t)prv * 3 * ctl.ntiles + (size_t)t * ctl.ntiles) * 2;
        int* chg_cur = ctl.changed + ((size_t)cur * 3 * ctl.ntiles + (size_t)t * ctl.ntiles) * 2;
        unsigned lmask = 0u, bmask = 0u;
        bool df_timeout = false;
        if constexpr (DF) {
            if (pass > 1) {
                // wait until a neighbour has published a version this tile has not used (bounded)
                const int* lwp = ctl.ver + (size_t)t * ctl.ntiles + left;
                const int* bwp = ctl.ver + (size_t)t * ctl.ntiles + below;
                int lw = lw_cur, bw = bw_cur;
                const long long t0 = clock64();
                while (true) {
                    lw = left >= 0 ? ld_acquire(lwp) : 0;
                    bw = below >= 0 ? ld_acquire(bwp) : 0;
                    const bool news = (left >= 0 && (lw >> 1) > used_lv) || (below >= 0 && (bw >> 1) > used_bv);
                    if (__shfl_sync(0xffffffffu, (int)news, 0)) break;
                    if (__shfl_sync(0xffffffffu, (int)(clock64() - t0 > ctl.spin_limit), 0)) {
                        df_timeout = true;
                        break;
                    }
                    __nanosleep(32);
                }
                if (df_timeout) {
                    if (lane == 0) atomicExch(ctl.timeout, 1);
                    break;
                }
                lw = __shfl_sync(0xffffffffu, lw, 0);
                bw = __shfl_sync(0xffffffffu, bw, 0);
                // the newest strips, read from the ring slot of their version; a slot the neighbour
                // may have begun to overwrite meanwhile (it got TT_RING - 1 versions ahead) is read again
                T np1 = in_p1, np2 = in_p2, nb0 = sm.bot[t][0][r], nb1 = sm.bot[t][1][r];
                if (left >= 0 && (lw >> 1) > used_lv) {
                    for (int tries = 0;; tries++) {
                        const int v = lw >> 1;
                        const T* ls = strip_ver_ptr(strips, t, left, v, ctl.ntiles);
                        np2 = __ldcg(ls + 0 * TT_W + r);
                        np1 = __ldcg(ls + 1 * TT_W + r);
                        const int again = __shfl_sync(0xffffffffu, ld_acquire(lwp), 0);
                        if ((again >> 1) <= v + TT_RING - 2 || tries > 1000) break;
                        lw = again;
                    }
                    used_lv = lw >> 1;
                    lw_cur = lw;
                }
                if (below >= 0 && (bw >> 1) > used_bv) {
                    for (int tries = 0;; tries++) {
                        const int v = bw >> 1;
                        const T* bs = strip_ver_ptr(strips, t, below, v, ctl.ntiles);
                        nb0 = __ldcg(bs + 2 * TT_W + r);
                        nb1 = __ldcg(bs + 3 * TT_W + r);
                        const int again = __shfl_sync(0xffffffffu, ld_acquire(bwp), 0);
                        if ((again >> 1) <= v + TT_RING - 2 || tries > 1000) break;
                        bw = again;
                    }
                    used_bv = bw >> 1;
                    bw_cur = bw;
                }
                auto differs = [](T x, T y) { return !(x == y || (x != x && y != y)); };
                lmask = __ballot_sync(0xffffffffu, differs(np1, in_p1) || differs(np2, in_p2));
                bmask = __ballot_sync(0xffffffffu, differs(nb0, sm.bot[t][0][r]) || differs(nb1, sm.bot[t][1][r]));
                in_p1 = np1;
                in_p2 = np2;
                sm.bot[t][0][r] = nb0;
                sm.bot[t][1][r] = nb1;
                __syncwarp();
            }
        } else {
            // neighbours' strips and masks are written by other SMs: read them through L2 (__ldcg)
            lmask = left >= 0 ? (unsigned)__ldcg(chg_prev + 2 * left) : 0u;
            bmask = below >= 0 ? (unsigned)__ldcg(chg_prev + 2 * below + 1) : 0u;
        }
        const bool compute = !halt && (pass == 1 || lmask != 0u || bmask != 0u);
        // Rows below the lowest changed row of the left strip have unchanged inputs when the
        // lower strip did not change: a repair pass replays their last values (Float32)
        const int rmin = (pass == 1 || bmask != 0u || !kStageQ<T>) ? 0 : __ffs((int)lmask) - 1;
        if (ctl.pass_ts && pass <= ctl.max_pass) {
            if constexpr (DF) {
                if (lane == 0) atomicMax(ctl.pass_ts + pass, globaltimer_ns());
            } else if (blockIdx.x == 0 && threadIdx.x == 0) {
                ctl.pass_ts[pass] = globaltimer_ns();
            }
        }
        if (ctl.pass_work && compute && lane == 0 && pass <= ctl.max_pass) atomicAdd(ctl.pass_work + pass, 1);
        const T* sp_prev = strip_ptr(strips, prv, t, tile, ctl.ntiles);
        T* sp_cur = strip_ptr(strips, cur, t, tile, ctl.ntiles);
        bool right_changed = false, top_changed = false;
        if (compute) {
            // left inputs: the left tile's right strip, or at the periodic seam the halo columns'
            // stage-start values; bottom inputs: the lower tile's top strip (none at k = 0)
            T prev1, prev2;
            if constexpr (DF) {
                prev1 = in_p1;
                prev2 = in_p2;
            } else {
                if (left >= 0) {
                    const T* ls = strip_ptr(strips, prv, t, left, ctl.ntiles);
                    prev2 = __ldcg(ls + 0 * TT_W + r);
                    prev1 = __ldcg(ls + 1 * TT_W + r);
                } else {
                    prev1 = row_ok ? a.q_old[t][MOIST_IDX(k, nx - 1)] / a.rho[MOIST_IDX(k, nx - 1)] : T(0);
                    prev2 = row_ok ? a.q_old[t][MOIST_IDX(k, nx - 2)] / a.rho[MOIST_IDX(k, nx - 2)] : T(0);
                }
                const T* bs = below >= 0 ? strip_ptr(strips, prv, t, below, ctl.ntiles) : nullptr;
                sm.bot[t][0][r] = bs ? __ldcg(bs + 2 * TT_W + r) : T(0);  // row z0-2
                sm.bot[t][1][r] = bs ? __ldcg(bs + 3 * TT_W + r) : T(0);  // row z0-1
            }
            __syncwarp();
            T sn_last = T(0), km1_used = T(0);
            const int nsteps = width + TT_W - 1;
            // Float64: q0 and the phys tendency of this lane's next cell, loaded one step ahead
            T q0_next = T(0), dph_next = T(0);
            if constexpr (!kStageQ<T>) {
                if (row_ok) {  // every active lane starts at column x0 (c = 0); width >= 1
                    q0_next = q0[MOIST_IDX(k, x0)];
                    dph_next = dph[MOIST_IDX(k, x0)];
                }
            }
#define MOIST_TILE_CELL(D, flag)                                                                          \
    tracer_cell_t<D>(p, k, a.dt, sm.s[t][r][c], sm.s[t][r][c + 1], sm.s[t][r][c + 2], sm.s[t][r + 1][c],        \
                     sm.s[t][r + 2][c], prev1, prev2, s_km1, s_km2, sm.lin[t][r], sm.lin[t][r + 1],             \
                     sm.lin[t][r + 2], sm.mx[r][c + 1], sm.mx[r][c], sm.mz[r + 1][c], sm.mz[r][c],              \
                     sm.rho[r + 1][c + 1], sm.rho[r + 1][c + 2], sm.rho[r + 1][c], sm.rho[r + 2][c + 1],        \
                     sm.rho[r][c + 1], dz_k, dz_kp1, dz_km1, z_k, z_kp1, z_km1, q0_c, dph_c, rr, flag)
            if constexpr (kStageQ<T>) {
                // Float32: every lane evaluates the branch-free cell at a clamped column each step
                // (inactive lanes on throw-away values) and only the stores are predicated, so a
                // step is one basic block; a cell outside the fast cell's proven ranges is
                // recomputed with IEEE division (fastdiv.cuh). The strips are formed after the loop.
                const T* bot0 = sm.bot[t][0];
                const T* bot1 = sm.bot[t][1];
                const T* cl_kp = sm.cl[t][0][k == 0 ? 0 : 1];
                const T* cl_km = sm.cl[t][1][k == 1 ? 0 : 1];
                // Repair passes recompute only where an input changed. A cell reads four updated
                // values: (k, i-1), (k, i-2) of its own row and (k-1, i), (k-2, i) from the rows
                // below; each lane carries, with every value it passes on, whether that value
                // changed in this pass. The stage-start values never change, so a cell whose
                // four updated inputs are all unchanged returns its last value. A step in which
                // no lane has a changed input replays the stored values only.
                const bool all_dirty = pass == 1;
                const bool left_chg = ((lmask >> r) & 1u) != 0u;  // this row's left-strip inputs
                bool c1 = left_chg, c2 = left_chg;                // prev1, prev2 changed
                bool chg_last = false, km1_chg_used = false;
                // replayed rows start two steps early: the first recomputed row reads the two below
                for (int step = rmin >= 2 ? rmin - 2 : 0; step < nsteps; step++) {
                    const int c_raw = step - r;
                    const bool active = row_ok && c_raw >= 0 && c_raw < width;
                    const int c = min(max(c_raw, 0), TT_W - 1);
                    // row-below values: lane r-1's result of the previous step and the value it used
                    const T up_sn = __shfl_up_sync(0xffffffffu, sn_last, 1);
                    const T up_km1 = __shfl_up_sync(0xffffffffu, km1_used, 1);
                    const bool up_chg = __shfl_up_sync(0xffffffffu, chg_last, 1);
                    const bool up_km1_chg = __shfl_up_sync(0xffffffffu, km1_chg_used, 1);
                    const T b1 = bot1[c], b0 = bot0[c];
                    const bool bchg = ((bmask >> c) & 1u) != 0u;  // the lower tile's top strip at column c
                    const T s_km1 = r == 0 ? b1 : up_sn;
                    const T s_km2 = r == 0 ? b0 : (r == 1 ? b1 : up_km1);
                    const bool km1_chg = r == 0 ? bchg : up_chg;
                    const bool km2_chg = r == 0 ? bchg : (r == 1 ? bchg : up_km1_chg);
                    const bool dirty = active && (all_dirty || c1 || c2 || km1_chg || km2_chg);
                    T qn_v = T(0), sn = sm.q.snp[t][r][c];
                    bool changed = false;
                    if (__any_sync(0xffffffffu, dirty)) {
                        const T q0_c = sm.q.q0[t][r][c], dph_c = sm.q.dph[t][r][c];
                        const T rho_c = sm.rho[r + 1][c + 1];
                        bool bad;
                        unsigned g = ~0u;
                        qn_v = tracer_cell_f<FastDiv>(fw, sm.s[t][r][c], sm.s[t][r][c + 1], sm.s[t][r][c + 2],
                                                      sm.s[t][r + 1][c], sm.s[t][r + 2][c], prev1, prev2, s_km1,
                                                      s_km2, cl_kp[c], cl_km[c], sm.mx[r][c + 1], sm.mx[r][c],
                                                      sm.mz[r + 1][c], sm.mz[r][c], rho_c, sm.rho[r + 1][c + 2],
                                                      sm.rho[r + 1][c], sm.rho[r + 2][c + 1], sm.rho[r][c + 1], q0_c,
                                                      dph_c, g, bad);
                        T snc = FastDiv::cdiv(qn_v, rho_c, sm.q.rrho[r][c], g);
                        bad |= guard_hit(g);
                        if (dirty && bad) {
                            // a subnormal-range quotient or a non-finite result: the same cell with
                            // subnormal quotients rounded explicitly (exact for every input), and
                            // IEEE division if the result is still not finite
                            unsigned g2 = ~0u;
                            bool bad2;
                            qn_v = tracer_cell_f<Div64X>(fw, sm.s[t][r][c], sm.s[t][r][c + 1], sm.s[t][r][c + 2],
                                                         sm.s[t][r + 1][c], sm.s[t][r + 2][c], prev1, prev2, s_km1,
                                                         s_km2, cl_kp[c], cl_km[c], sm.mx[r][c + 1], sm.mx[r][c],
                                                         sm.mz[r + 1][c], sm.mz[r][c], rho_c, sm.rho[r + 1][c + 2],
                                                         sm.rho[r + 1][c], sm.rho[r + 2][c + 1], sm.rho[r][c + 1],
                                                         q0_c, dph_c, g2, bad2);
                            snc = Div64X::cdiv(qn_v, rho_c, sm.q.rrho[r][c], g2);
                            if (bad2) {
                                bool unused = false;
                                qn_v = MOIST_TILE_CELL(DivIEEE<T>, unused);
                                snc = qn_v / rho_c;
                            }
                        }
                        if (dirty) {
                            changed = !all_dirty && !(__float_as_uint(snc) == __float_as_uint(sn));
                            sn = snc;
                            sm.q.qn[t][r][c] = qn_v;
                            sm.q.snp[t][r][c] = snc;
                        }
                    }
                    if (active) {
                        prev2 = prev1;
                        prev1 = sn;
                        c2 = c1;
                        c1 = changed;
                    }
                    // lane r+1 reads these next step only for the column it shares with this step
                    sn_last = sn;
                    km1_used = s_km1;
                    chg_last = changed;
                    km1_chg_used = km1_chg;
                }
                __syncwarp();
                // the boundary strips s = q / rho of the values just computed (IEEE division, as
                // every s of the loop: the fast quotient equals it inside its guarded range)
                if (row_ok && width == TT_W) {
                    sm.strip_out[t][0][r] = sm.q.qn[t][r][TT_W - 2] / sm.rho[r + 1][TT_W - 1];
                    sm.strip_out[t][1][r] = sm.q.qn[t][r][TT_W - 1] / sm.rho[r + 1][TT_W];
                }
                if (r < width) {
                    if (z0 + TT_W - 2 < nz) sm.strip_out[t][2][r] = sm.q.qn[t][TT_W - 2][r] / sm.rho[TT_W - 1][r + 1];
                    if (z0 + TT_W - 1 < nz) sm.strip_out[t][3][r] = sm.q.qn[t][TT_W - 1][r] / sm.rho[TT_W][r + 1];
                }
            } else {
                for (int step = 0; step < nsteps; step++) {
                    const int c = step - r;
                    // row-below values: lane r-1's result of the previous step and the value it used
                    const T up_sn = __shfl_up_sync(0xffffffffu, sn_last, 1);
                    const T up_km1 = __shfl_up_sync(0xffffffffu, km1_used, 1);
                    if (row_ok && c >= 0 && c < width) {
                        T s_km1, s_km2;
                        if (r == 0) {
                            s_km1 = sm.bot[t][1][c];
                            s_km2 = sm.bot[t][0][c];
                        } else if (r == 1) {
                            s_km1 = up_sn;
                            s_km2 = sm.bot[t][1][c];
                        } else {
                            s_km1 = up_sn;
                            s_km2 = up_km1;
                        }
                        const int i = x0 + c;
                        const size_t cix = MOIST_IDX(k, i);
                        const T q0_c = q0_next, dph_c = dph_next;
                        if (c + 1 < width) {
                            q0_next = q0[cix + 1];
                            dph_next = dph[cix + 1];
                        }
                        const T rho_c = sm.rho[r + 1][c + 1];
                        bool unused = false;
                        const T qn_v = MOIST_TILE_CELL(DivIEEE<T>, unused);
                        const T sn = qn_v / rho_c;
                        qn[cix] = qn_v;
                        if (c == TT_W - 2) sm.strip_out[t][0][r] = sn;
                        if (c == TT_W - 1) sm.strip_out[t][1][r] = sn;
                        if (r == TT_W - 2) sm.strip_out[t][2][c] = sn;
                        if (r == TT_W - 1) sm.strip_out[t][3][c] = sn;
                        prev2 = prev1;
                        prev1 = sn;
                        sn_last = sn;
                        km1_used = s_km1;
                    }
                }
            }
#undef MOIST_TILE_CELL
            __syncwarp();
            if constexpr (kStageQ<T>) {  // coalesced write of the tile's results
                for (int rr = 0; rr < TT_W; rr++) {
                    const int kk = z0 + rr;
                    if (kk < nz && r < width) qn[MOIST_IDX(kk, x0 + r)] = sm.q.qn[t][rr][r];
                }
            }
            // publish this pass's strips; a strip entry the tile does not own (partial tile)
            // keeps the speculative value so it never registers a change
            if constexpr (!DF) {
                for (int q = 0; q < 4; q++) {
                    const bool owned =
                        (q < 2) ? (row_ok && width == TT_W) : ((z0 + 30 + (q - 2)) < nz && r < width);
                    const T old = __ldcg(sp_prev + q * TT_W + r);
                    const T v = owned ? sm.strip_out[t][q][r] : old;
                    __stcg(sp_cur + q * TT_W + r, v);
                    if (!(v == old || (v != v && old != old))) (q < 2 ? right_changed : top_changed) = true;
                }
            }
        } else if constexpr (!DF) {
            for (int q = 0; q < 4; q++) __stcg(sp_cur + q * TT_W + r, __ldcg(sp_prev + q * TT_W + r));
        }
        if constexpr (DF) {
            // a new version when the strips changed, or when the tile became final: it computed
            // from (or is unchanged by) its neighbours' final strips
            T v[4];
            bool chg = false;
            for (int q = 0; q < 4; q++) {
                const bool owned = (q < 2) ? (row_ok && width == TT_W) : ((z0 + 30 + (q - 2)) < nz && r < width);
                v[q] = (compute && owned) ? sm.strip_out[t][q][r] : pub[q];
                chg |= !(v[q] == pub[q] || (v[q] != v[q] && pub[q] != pub[q]));
            }
            const bool fin = (left < 0 || (lw_cur & 1)) && (below < 0 || (bw_cur & 1));
            if (__any_sync(0xffffffffu, chg) || fin) {
                T* out = strip_ver_ptr(strips, t, tile, my_ver + 1, ctl.ntiles);
                for (int q = 0; q < 4; q++) {
                    __stcg(out + q * TT_W + r, v[q]);
                    pub[q] = v[q];
                }
                __threadfence();
                __syncwarp();
                my_ver++;
                if (lane == 0) st_release(my_word, (my_ver << 1) | (fin ? 1 : 0));
            }
            if (fin || halt) break;
            continue;
        }
        // lane r: row r of the right strip, column r of the top strip
        const unsigned rmask = __ballot_sync(0xffffffffu, right_changed);
        const unsigned tmask = __ballot_sync(0xffffffffu, top_changed);
        if (lane == 0) {
            __stcg(chg_cur + 2 * tile, (int)rmask);
            __stcg(chg_cur + 2 * tile + 1, (int)tmask);
            if (rmask | tmask) atomicAdd(ctl.any_changed + pass, 1);
        }
        if (!grid_barrier(ctl, nblocks)) return;
        if (__ldcg(ctl.any_changed + pass) == 0) break;
    }
    if constexpr (DF) {  // the deepest tile's count of computations, and the moment the last tile leaves
        if (lane == 0) {
            atomicMax(ctl.passes, pass);
            if (ctl.pass_ts) atomicMax(ctl.pass_ts + ctl.max_pass + 2, globaltimer_ns());
        }
    } else if (blockIdx.x == 0 && threadIdx.x == 0) {
        *ctl.passes = pass;
        if (ctl.pass_ts) ctl.pass_ts[ctl.max_pass + 2] = globaltimer_ns();  // block 0 leaves the sweep
    }
}

// histogram of pass counts (diagnostic)
__global__ void k_pass_count(const int* passes, int* hist) {
    const int p = *passes;
    atomicAdd(hist + (p < 63 ? p : 63), 1);
}

}  // namespace moist
