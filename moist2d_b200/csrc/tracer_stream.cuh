// tracer_stream.cuh - the reference's in-place Gauss-Seidel tracer sweep as one exact wavefront
// per tracer, streaming every row through registers.
//
// Cell (k, i) of the in-place sweep (moist.jl:1469-1518) reads the updated values at (k, i-1),
// (k, i-2), (k-1, i), (k-2, i) and stage-start values elsewhere, so the anti-diagonals
// k + i = const can be updated together. One block sweeps one tracer of one domain: thread k
// owns row k (nz <= STREAM_MAX_ROWS) and updates column c = s - k at step s, for
// s = 0 .. nx + nz - 2. No speculation, no repair passes and no grid-wide barrier: blocks are
// independent, so any number of (domain, tracer) sweeps can share one launch.
//
// Each thread keeps a window of its own row (stage-start s = rho_q / rho at c .. c+2, density
// at c-1 .. c+1, mfx at c-1, c, mfz at c-1, c) and loads the next column one step ahead. The
// neighbouring rows come from the neighbouring threads, which stand one column behind (row
// k+1) or ahead (row k-1): warp shuffles inside a warp; across a warp boundary the stage-start
// values are loaded directly and the two updated values of the top rows of the warp below go
// through a small shared-memory ring, one block barrier per step.
//
// The cell update is the Float32 branch-free cell of tracer_tiles.cuh (FP64-reciprocal
// division, exact fallback) or the IEEE cell for Float64: the same operations as the tiled
// sweep, so the two kernels agree bit for bit.
#pragma once

#include "tracer_tiles.cuh"

namespace moist {

constexpr int STREAM_MAX_ROWS = 256;  // rows per block (threads); the register budget allows no more
constexpr int STREAM_RING = 8;        // columns kept of the two top rows of every warp

template <class T>
struct StreamArgs {
    TracerArgs<T> tr;
    const T* s_old[3];   // stage-start rho_q / rho, [nz][P]
    const double* rrho;  // 1 / rho in double precision, [nz][P] (Float32 fast cell)
};

__device__ __forceinline__ int pmod(int c, int n) {
    const int r = c % n;
    return r < 0 ? r + n : r;
}

// stage-start s = rho_q / rho and the reciprocal densities of the stream sweep
template <class T>
__device__ __forceinline__ void b_stream_prep(DevParams<T> p, TracerArgs<T> a, T* s0, T* s1, T* s2, double* rrho,
                                              const int* err, int bx, int by) {
    const int i = bx * blockDim.x + threadIdx.x;
    const int k = by * blockDim.y + threadIdx.y;
    const int nx = p.nx, nz = p.nz, P = p.P;
    if (i >= nx || k >= nz || halted(err)) return;
    const size_t c = MOIST_IDX(k, i);
    const T rho = a.rho[c];
    s0[c] = a.q_old[0][c] / rho;
    s1[c] = a.q_old[1][c] / rho;
    s2[c] = a.q_old[2][c] / rho;
    rrho[c] = 1.0 / (double)rho;
}
template <class T>
__global__ void k_stream_prep(DevParams<T> p, TracerArgs<T> a, T* s0, T* s1, T* s2, double* rrho, const int* err) {
    b_stream_prep(p, a, s0, s1, s2, rrho, err, blockIdx.x, blockIdx.y);
}

// one tracer t of one domain; blockDim.x = 32 * ceil(nz / 32); ring: [nwarps][2][STREAM_RING]
template <class T>
__device__ __forceinline__ void stream_sweep(const DevParams<T>& p, const StreamArgs<T>& a, int t, T* ring) {
    const int nx = p.nx, nz = p.nz, P = p.P, ke = nz - 1;
    const int k = threadIdx.x, lane = k & 31, w = k >> 5;
    const bool row_ok = k < nz;
    const T* so = a.s_old[t];
    const T* rho = a.tr.rho;
    const T* mfx = a.tr.mfx;
    const T* mfz = a.tr.mfz;
    const T* q0g = a.tr.q0[t];
    const T* dphg = a.tr.dphys[t];
    T* qn = a.tr.q_new[t];
    const T* qo = a.tr.q_old[t];
    // stage-start values of row kk at column c (periodic in x), with the padding of the tiled
    // sweep outside the domain: s = 0, rho = 1, mass fluxes 0
    auto S = [&](int kk, int c) { return (kk >= 0 && kk < nz) ? so[MOIST_IDX(kk, pmod(c, nx))] : T(0); };
    auto R = [&](int kk, int c) { return (kk >= 0 && kk < nz) ? rho[MOIST_IDX(kk, pmod(c, nx))] : T(1); };
    auto MX = [&](int kk, int c) { return (kk >= 0 && kk < nz) ? mfx[MOIST_IDX(kk, pmod(c, nx))] : T(0); };
    auto MZ = [&](int kk, int c) {
        return (kk >= 0 && kk < nz && c >= 0 && c < nx) ? mfz[MOIST_IDX(kk, c)] : T(0);
    };

    // row constants (as the tiled sweep forms them)
    const T dz_k = row_ok ? p.dz[k] : T(1);
    const T dz_kp1 = (row_ok && k < ke) ? p.dz[k + 1] : T(1);
    const T dz_km1 = (row_ok && k > 0) ? p.dz[k - 1] : T(1);
    const T z_k = row_ok ? p.z[k] : T(0);
    const T z_kp1 = (row_ok && k < ke) ? p.z[k + 1] : T(1);
    const T z_km1 = (row_ok && k > 0) ? p.z[k - 1] : T(-1);
    RowRcp<T> rr;
    rr.dx = T(1) / p.dx;
    rr.dz_k = T(1) / dz_k;
    rr.sum_kp = T(1) / (dz_k + dz_kp1);
    rr.sum_km = T(1) / (dz_km1 + dz_k);
    rr.zd_kp = T(1) / (z_kp1 - z_k);
    rr.zd_km = T(1) / (z_k - z_km1);
    const T lin_km1 = (k - 1 >= 0 && k - 1 < nz) ? qo[MOIST_IDX(k - 1, nx - 2)] : T(0);
    const T lin_k = row_ok ? qo[MOIST_IDX(k, nx - 2)] : T(0);
    const T lin_kp1 = (k + 1 < nz) ? qo[MOIST_IDX(k + 1, nx - 2)] : T(0);
    FastRow<double> fw{};
    if constexpr (sizeof(T) == 4) {
        fw.dx = p.dx;
        fw.dz_k = dz_k;
        fw.dz_kp1 = dz_kp1;
        fw.dz_km1 = dz_km1;
        fw.sum_kp = dz_k + dz_kp1;
        fw.sum_km = dz_km1 + dz_k;
        fw.zd_kp = z_kp1 - z_k;
        fw.zd_km = z_k - z_km1;
        fw.rdx = Div64::rcp(fw.dx);
        fw.rdz_k = Div64::rcp(fw.dz_k);
        fw.rsum_kp = Div64::rcp(fw.sum_kp);
        fw.rsum_km = Div64::rcp(fw.sum_km);
        fw.rzd_kp = Div64::rcp(fw.zd_kp);
        fw.rzd_km = Div64::rcp(fw.zd_km);
        fw.kappa = p.kappa;
        fw.EPS = p.EPS;
        fw.dt_stage = a.tr.dt;
        fw.k0 = k == 0;
        fw.ke = k == ke;
        fw.kp_at0 = k == 0;
        fw.kp_atnm2 = k == nz - 2;
        fw.km_at0 = k - 1 == 0;
        fw.km_atnm2 = k - 1 == nz - 2;
    }
    const bool clamp_kp_row = row_ok && (k == 0 || k == nz - 2) && k < ke;
    const bool clamp_km_row = row_ok && (k == 1 || k == nz - 1) && k >= 1;

    // the window at the virtual column c = s - k (every thread advances it every step, so that
    // its neighbours read the right columns before it starts and after it ends). Column indices
    // of the loads are kept wrapped into [0, nx) incrementally.
    int c = -k;
    auto wrap = [&](int x) { return x >= nx ? x - nx : x; };
    int cw1 = pmod(c + 1, nx), cw2 = pmod(c + 2, nx), cw3 = pmod(c + 3, nx);  // c+1, c+2, c+3 wrapped
    const bool rin = row_ok, rin_p1 = k + 1 < nz, rin_p2 = k + 2 < nz, rin_m1 = k >= 1 && k - 1 < nz;
    const T* so_k = so + (size_t)(rin ? k : 0) * P;
    const T* so_kp1 = so + (size_t)(rin_p1 ? k + 1 : 0) * P;
    const T* so_kp2 = so + (size_t)(rin_p2 ? k + 2 : 0) * P;
    const T* rho_k = rho + (size_t)(rin ? k : 0) * P;
    const T* rho_kp1 = rho + (size_t)(rin_p1 ? k + 1 : 0) * P;
    const T* rho_km1 = rho + (size_t)(rin_m1 ? k - 1 : 0) * P;
    const T* mfx_k = mfx + (size_t)(rin ? k : 0) * P;
    const T* mfz_k = mfz + (size_t)(rin ? k : 0) * P;
    const T* mfz_km1 = mfz + (size_t)(rin_m1 ? k - 1 : 0) * P;
    const T* q0_k = q0g + (size_t)(rin ? k : 0) * P;
    const T* dph_k = dphg + (size_t)(rin ? k : 0) * P;
    const double* rr_k = a.rrho + (size_t)(rin ? k : 0) * P;
    const int cw0 = pmod(c, nx), cwm = pmod(c - 1, nx);
    T s0 = rin ? so_k[cw0] : T(0), s1 = rin ? so_k[cw1] : T(0), s2 = rin ? so_k[cw2] : T(0);
    T rm = rin ? rho_k[cwm] : T(1), r0 = rin ? rho_k[cw0] : T(1), r1 = rin ? rho_k[cw1] : T(1);
    T xm = rin ? mfx_k[cwm] : T(0), x0 = rin ? mfx_k[cw0] : T(0);
    T zp = MZ(k, c - 1), z0 = MZ(k, c);
    T q0c = rin ? q0_k[cw0] : T(0), dphc = rin ? dph_k[cw0] : T(0);
    double rrc = rin ? rr_k[cw0] : 1.0;
    // warp-boundary values of column c: rows k+1, k+2 (top lanes), k-1 (lane 0)
    T b_s1 = S(k + 1, c), b_s2 = S(k + 2, c), b_r1 = R(k + 1, c), b_rm = R(k - 1, c), b_zm = MZ(k - 1, c);
    // the updated values of the two columns to the left; the seam reads the stage-start values
    T prev1 = S(k, nx - 1), prev2 = S(k, nx - 2);
    T sn_last = T(0), km1_used = T(0);
    T* top1 = ring;                                    // [w][STREAM_RING]: row 32w+31
    T* top2 = ring + (blockDim.x >> 5) * STREAM_RING;  // [w][STREAM_RING]: row 32w+30

    const int nsteps = nx + nz - 1;
    for (int step = 0; step < nsteps; step++, c++) {
        const bool active = row_ok && c >= 0 && c < nx;
        // loads for the next column c+1 (one step ahead); mfz only inside the domain
        const bool zin = c + 1 >= 0 && c + 1 < nx;
        const T n_s2 = rin ? so_k[cw3] : T(0);
        const T n_r1 = rin ? rho_k[cw2] : T(1);
        const T n_x0 = rin ? mfx_k[cw1] : T(0);
        const T n_z0 = (rin && zin) ? mfz_k[cw1] : T(0);
        const T n_q0 = rin ? q0_k[cw1] : T(0);
        const T n_dph = rin ? dph_k[cw1] : T(0);
        const double n_rr = rin ? rr_k[cw1] : 1.0;
        T n_bs1 = T(0), n_bs2 = T(0), n_br1 = T(1), n_brm = T(1), n_bzm = T(0);
        if (lane >= 30) {
            n_bs1 = rin_p1 ? so_kp1[cw1] : T(0);
            n_bs2 = rin_p2 ? so_kp2[cw1] : T(0);
            n_br1 = rin_p1 ? rho_kp1[cw1] : T(1);
        }
        if (lane == 0) {
            n_brm = rin_m1 ? rho_km1[cw1] : T(1);
            n_bzm = (rin_m1 && zin) ? mfz_km1[cw1] : T(0);
        }
        // neighbours: row k-1 stands one column ahead, rows k+1, k+2 one and two behind
        const T up_sn = __shfl_up_sync(0xffffffffu, sn_last, 1);
        const T up_km1 = __shfl_up_sync(0xffffffffu, km1_used, 1);
        const T up_rm = __shfl_up_sync(0xffffffffu, rm, 1);
        const T up_zp = __shfl_up_sync(0xffffffffu, zp, 1);
        const T dn_s1 = __shfl_down_sync(0xffffffffu, s1, 1);
        const T dn_s2 = __shfl_down_sync(0xffffffffu, s2, 2);
        const T dn_r1 = __shfl_down_sync(0xffffffffu, r1, 1);
        const int cc = c < 0 ? 0 : (c >= nx ? nx - 1 : c);
        const T t1 = (w > 0) ? top1[(w - 1) * STREAM_RING + (cc & (STREAM_RING - 1))] : T(0);
        const T t2 = (w > 0) ? top2[(w - 1) * STREAM_RING + (cc & (STREAM_RING - 1))] : T(0);
        const T s_km1 = lane == 0 ? t1 : up_sn;
        const T s_km2 = lane == 0 ? t2 : (lane == 1 ? t1 : up_km1);
        const T rho_km = lane == 0 ? b_rm : up_rm;
        const T mfz_km = lane == 0 ? b_zm : up_zp;
        const T s_kp1 = lane == 31 ? b_s1 : dn_s1;
        const T s_kp2 = lane >= 30 ? b_s2 : dn_s2;
        const T rho_kp = lane == 31 ? b_r1 : dn_r1;

        T qn_v = T(0), sn = T(0);
        if (active) {
            const size_t cix = MOIST_IDX(k, c);
            const T q0_c = q0c, dph_c = dphc;
            // the clamp quotients of limited_flux_z, on the four rows that can use them
            T cl_kp = T(0), cl_km = T(0);
            if (clamp_kp_row) cl_kp = z0 > p.EPS ? lin_k / (z0 * p.dt) : lin_kp1 / (-z0 * p.dt);
            if (clamp_km_row) cl_km = mfz_km > p.EPS ? lin_km1 / (mfz_km * p.dt) : lin_k / (-mfz_km * p.dt);
#define MOIST_STREAM_IEEE_CELL                                                                            \
    tracer_cell_t<DivIEEE<T>>(p, k, a.tr.dt, s0, s1, s2, s_kp1, s_kp2, prev1, prev2, s_km1, s_km2, lin_km1,     \
                              lin_k, lin_kp1, x0, xm, z0, mfz_km, r0, r1, rm, rho_kp, rho_km, dz_k, dz_kp1,       \
                              dz_km1, z_k, z_kp1, z_km1, q0_c, dph_c, rr, unused)
            if constexpr (sizeof(T) == 4) {
                bool bad;
                unsigned g = ~0u;
                qn_v = tracer_cell_f<Div64>(fw, s0, s1, s2, s_kp1, s_kp2, prev1, prev2, s_km1, s_km2, cl_kp, cl_km,
                                            x0, xm, z0, mfz_km, r0, r1, rm, rho_kp, rho_km, q0_c, dph_c, g, bad);
                sn = Div64::cdiv(qn_v, r0, rrc, g);
                if (bad || guard_hit(g)) {
                    unsigned g2 = ~0u;
                    bool bad2;
                    qn_v = tracer_cell_f<Div64X>(fw, s0, s1, s2, s_kp1, s_kp2, prev1, prev2, s_km1, s_km2, cl_kp,
                                                 cl_km, x0, xm, z0, mfz_km, r0, r1, rm, rho_kp, rho_km, q0_c, dph_c,
                                                 g2, bad2);
                    sn = Div64X::cdiv(qn_v, r0, rrc, g2);
                    if (bad2) {
                        bool unused = false;
                        qn_v = MOIST_STREAM_IEEE_CELL;
                        sn = qn_v / r0;
                    }
                }
            } else {
                bool unused = false;
                qn_v = MOIST_STREAM_IEEE_CELL;
                sn = qn_v / r0;
            }
#undef MOIST_STREAM_IEEE_CELL
            qn[cix] = qn_v;
            if (lane == 31) top1[w * STREAM_RING + (c & (STREAM_RING - 1))] = sn;
            if (lane == 30) top2[w * STREAM_RING + (c & (STREAM_RING - 1))] = sn;
            prev2 = prev1;
            prev1 = sn;
        }
        // lane k+1 reads these next step only for the column it shares with this step
        sn_last = sn;
        km1_used = s_km1;
        // advance the window to column c + 1
        s0 = s1;
        s1 = s2;
        s2 = n_s2;
        rm = r0;
        r0 = r1;
        r1 = n_r1;
        xm = x0;
        x0 = n_x0;
        zp = z0;
        z0 = n_z0;
        q0c = n_q0;
        dphc = n_dph;
        rrc = n_rr;
        b_s1 = n_bs1;
        b_s2 = n_bs2;
        b_r1 = n_br1;
        b_rm = n_brm;
        b_zm = n_bzm;
        cw1 = cw2;
        cw2 = cw3;
        cw3 = wrap(cw3 + 1);
        __syncthreads();
    }
}

// tracer t of one domain (the block's threads: 32 * ceil(nz / 32) or more)
template <class T>
__device__ __forceinline__ void b_tracer_stream(const DevParams<T>& p, const StreamArgs<T>& a, const int* err, int t) {
    __shared__ T ring[2 * (STREAM_MAX_ROWS / 32) * STREAM_RING];
    if (halted(err)) return;
    stream_sweep(p, a, t, ring);
}

// single domain: block t sweeps tracer t
template <class T>
__global__ void __launch_bounds__(STREAM_MAX_ROWS) k_tracer_stream(DevParams<T> p, StreamArgs<T> a, const int* err) {
    b_tracer_stream(p, a, err, blockIdx.x);
}

}  // namespace moist
