// kernels.cuh - CUDA kernels of the large step (sm_100a).
//
// One large step (rk3_step!, moist.jl:1589-1683) is
//   [sf] [rd] physics  ->  3 x ( diag, tend, thomas_factors, ns_s x substep, tracer, update )  ->  prec
// sf/rd run only when do_sf/do_rd are set. See model.cuh for the layout and arithmetic rules.
#pragma once

#include <climits>

#include "fastdiv.cuh"
#include "model.cuh"

namespace moist {

template <class T>
struct StateP {
    T *rho, *ru, *rw, *rt, *qv, *qc, *qr;
};

template <class T>
struct PhysP {  // the six phys tendencies of compute_step! (moist.jl:1039)
    T *d_rho, *d_u, *d_th, *d_qv, *d_qc, *d_qr;
};

// error word: err[0] = smallest MOIST_FIELD_* with a NaN (INT_MAX if none)
__device__ __forceinline__ bool halted(const int* err) { return *(volatile const int*)err != INT_MAX; }

#define MOIST_IDX(k, i) ((size_t)(k) * P + (i))

// Load of an input that no thread writes during the launch (it was produced by an earlier
// launch): the read-only data path, which also lets the compiler issue the load ahead of the
// launch's stores to other arrays, so a column walk keeps several levels' loads in flight.
template <class X>
__device__ __forceinline__ X ro(const X* q) {
    return __ldg(q);
}

// ----------------------------------------------------------------------------- physics

// surface_fluxes! (moist.jl:714-751), one thread per column. ru_left / rho_right are the
// reference's halo reads rho_u[ks, is-1] and rho[ks, ie+1], which hold the values of the
// last halo exchange (start of the last RK stage), not the current interior.
template <class T>
__device__ __forceinline__ void b_surface_fluxes(DevParams<T> p, StateP<T> s, const T* ru_left, const T* rho_right,
                                                 T* d_u_sf, T* d_th_sf, T* d_qv_sf, T* mflux, T* shflux, T* lhflux,
                                                 const int* err, int bx, int by) {
    const int i = bx * blockDim.x + threadIdx.x;
    const int nx = p.nx;
    if (i >= nx || halted(err)) return;
    const T rho = s.rho[i], qv = s.qv[i] / rho, qc = s.qc[i] / rho, qr = s.qr[i] / rho;
    const T qd = T(1.0) - qv - qc - qr;
    const T r = p.Rd * qd + p.Rv * qv;
    const T cp = p.Cpd * qd + p.Cpv * qv + p.Cpl * (qc + qr);
    const T cv = cp - r;
    const T ru_m = (i == 0) ? *ru_left : s.ru[i - 1];
    const T rho_p1 = (i == nx - 1) ? *rho_right : s.rho[i + 1];
    T uabs = mm::mabs(ru_m + s.ru[i]) * T(0.5) / rho;
    uabs = jmax(uabs, p.uabs_min);
    const T theta_ks = s.rt[i] / rho;
    const T pi_ks = mm::mpow(r * s.rt[i] / p.P0, r / cv);
    const T pi_surf = pi_ks + p.dz[0] * T(0.5) * p.GRAV / (cp * theta_ks);
    const T p_surf = p.P0 * mm::mpow(pi_surf, cp / r);
    const T rho_surf = p_surf / (r * p.temp_surf);
    const T theta_surf = p.temp_surf / pi_surf;
    const T u = s.ru[i] / (rho + rho_p1) * T(2.0);
    const T mf = -rho_surf * p.Cd * u * mm::mabs(u);
    mflux[i] = mf;
    d_u_sf[i] = mf / p.dz[0];
    const T sh = rho_surf * p.Ch * uabs * (theta_surf - theta_ks) * pi_surf;
    d_th_sf[i] = sh / (pi_ks * p.dz[0]);
    shflux[i] = sh * cp;
    T es, d1, qsat_s, d2;
    sat_vp(p.temp_surf, p, es, d1);
    sat_q(p_surf, es, p, qsat_s, d2);
    const T lh = rho_surf * p.Ce * uabs * (qsat_s - qv);
    d_qv_sf[i] = lh / p.dz[0];
    lhflux[i] = lh * p.Lv;
}
template <class T>
__global__ void k_surface_fluxes(DevParams<T> p, StateP<T> s, const T* ru_left, const T* rho_right,                                  T* d_u_sf, T* d_th_sf, T* d_qv_sf, T* mflux, T* shflux, T* lhflux,                                  const int* err) {
    b_surface_fluxes(p, s, ru_left, rho_right, d_u_sf, d_th_sf, d_qv_sf, mflux, shflux, lhflux, err, blockIdx.x, blockIdx.y);
}

template <class T>
__device__ __forceinline__ T tanh_m(T x) {  // tanh from the shared exp
    const T e = mm::mexp(T(2) * x);
    return (e - T(1)) / (e + T(1));
}

// gray_radiation! (moist.jl:776-840), one thread per column; LW_up / LW_dn scratch [nz+1][P]
template <class T>
__device__ __forceinline__ void b_gray_radiation(DevParams<T> p, StateP<T> s, const T* theta_ref, T* lw_up, T* lw_dn,
                                                 T* d_th_rd, const int* err, int bx, int by) {
    const int i = bx * blockDim.x + threadIdx.x;
    const int nx = p.nx, nz = p.nz, P = p.P;
    if (i >= nx || halted(err)) return;
    auto col = [&](int k, T& cpk, T& pik, T& tempk, T& epsk, T& tauk) {
        const size_t c = MOIST_IDX(k, i);
        const T rho = s.rho[c];
        const T qv = s.qv[c] / rho, qc = s.qc[c] / rho, qr = s.qr[c] / rho;
        const T qd = T(1.0) - qv - qc - qr;
        const T r = p.Rd * qd + p.Rv * qv;
        cpk = p.Cpd * qd + p.Cpv * qv + p.Cpl * (qc + qr);
        const T cv = cpk - r;
        pik = mm::mpow(r * s.rt[c] / p.P0, r / cv);
        tempk = s.rt[c] / rho * pik;
        const T dq = p.k_abs_qv * s.qv[c] * p.dz[k];
        const T dc = p.k_abs_qc * s.qc[c] * p.dz[k];
        const T dr = p.k_abs_qr * s.qr[c] * p.dz[k];
        epsk = T(1.0) - mm::mexp(-(dq + dc + dr));
        tauk = T(1.0) - epsk;
    };
    T cpk, pik, tempk, epsk, tauk;
    T up = p.surf_emissivity * p.SIGMA * mm::mpow4(p.temp_surf);
    lw_up[MOIST_IDX(0, i)] = up;
    for (int k = 0; k < nz; k++) {
        col(k, cpk, pik, tempk, epsk, tauk);
        up = up * tauk + epsk * p.SIGMA * mm::mpow4(tempk);
        lw_up[MOIST_IDX(k + 1, i)] = up;
    }
    T dn = T(0.0);
    lw_dn[MOIST_IDX(nz, i)] = dn;
    for (int k = nz - 1; k >= 0; k--) {
        col(k, cpk, pik, tempk, epsk, tauk);
        dn = dn * tauk + epsk * p.SIGMA * mm::mpow4(tempk);
        lw_dn[MOIST_IDX(k, i)] = dn;
    }
    const T dz_trans = T(2.0e3);
    for (int k = 0; k < nz; k++) {
        col(k, cpk, pik, tempk, epsk, tauk);
        const T divF = ((lw_up[MOIST_IDX(k + 1, i)] - lw_dn[MOIST_IDX(k + 1, i)]) -
                        (lw_up[MOIST_IDX(k, i)] - lw_dn[MOIST_IDX(k, i)])) / p.dz[k];
        const T hr = -divF / (cpk * pik);
        const T alpha = T(0.5) * (T(1.0) + tanh_m((p.z[k] - (p.z_trop + dz_trans * T(0.5))) / dz_trans)) /
                        p.tau_cooling;
        const size_t c = MOIST_IDX(k, i);
        const T cr = -(s.rt[c] - s.rho[c] * theta_ref[k]) * alpha;
        d_th_rd[c] = hr + cr;
    }
}
template <class T>
__global__ void k_gray_radiation(DevParams<T> p, StateP<T> s, const T* theta_ref, T* lw_up,                                  T* lw_dn, T* d_th_rd, const int* err) {
    b_gray_radiation(p, s, theta_ref, lw_up, lw_dn, d_th_rd, err, blockIdx.x, blockIdx.y);
}

// Kessler microphysics + rain sedimentation + assembly of the six phys tendencies
// (moist.jl:1593-1644), one thread per cell.
template <class T>
__device__ __forceinline__ void b_physics(DevParams<T> p, StateP<T> s, T* d_th_mp, T* d_qv_mp, T* d_qc_mp, T* d_qr_mp,
                                          T* d_qr_sed, T* d_prec, const T* d_th_rd, const T* d_u_sf, const T* d_th_sf,
                                          const T* d_qv_sf, PhysP<T> ph, const int* err, int bx, int by) {
    const int i = bx * blockDim.x + threadIdx.x;
    const int k = by * blockDim.y + threadIdx.y;
    const int nx = p.nx, nz = p.nz, P = p.P;
    if (i >= nx || k >= nz || halted(err)) return;
    const size_t c = MOIST_IDX(k, i);
    const T rho = s.rho[c], rt = s.rt[c], rqr = s.qr[c];
    T dqv = T(0), dqc = T(0), dqr = T(0), dth = T(0);
    if (p.do_mp) kessler_cell(rho, rt, s.qv[c], s.qc[c], rqr, p, dqv, dqc, dqr, dth);
    T sed = T(0);
    if (p.do_mp && p.do_sed) {
        const T vt = terminal_velocity(rqr, rho, p);
        const T flux_kp = (k == nz - 1) ? T(0.0) : s.qr[c + P] * terminal_velocity(s.qr[c + P], s.rho[c + P], p);
        const T flux_km = rqr * vt;
        sed = (flux_kp - flux_km) / p.dz[k];
        if (k == 0) d_prec[i] = rqr * vt;
    } else if (k == 0) {
        d_prec[i] = T(0);
    }
    d_th_mp[c] = dth;
    d_qv_mp[c] = dqv;
    d_qc_mp[c] = dqc;
    d_qr_mp[c] = dqr;
    d_qr_sed[c] = sed;
    // phys assembly, in the reference's order (moist.jl:1633-1643)
    const T th_rd = p.do_rd ? d_th_rd[c] : T(0.0);
    T d_rho = sed;
    if (k == 0) d_rho += d_qv_sf[i];
    T d_u = T(0.0);
    if (k == 0) d_u += d_u_sf[i];
    T d_th = dth + th_rd + d_rho * rt / rho;
    if (k == 0) d_th += d_th_sf[i];
    T d_qv = dqv;
    if (k == 0) d_qv += d_qv_sf[i];
    ph.d_rho[c] = d_rho;
    ph.d_u[c] = d_u;
    ph.d_th[c] = d_th;
    ph.d_qv[c] = d_qv;
    ph.d_qc[c] = dqc;
    ph.d_qr[c] = dqr + sed;
}
template <class T>
__global__ void k_physics(DevParams<T> p, StateP<T> s, T* d_th_mp, T* d_qv_mp, T* d_qc_mp, T* d_qr_mp,                           T* d_qr_sed, T* d_prec, const T* d_th_rd, const T* d_u_sf, const T* d_th_sf,                           const T* d_qv_sf, PhysP<T> ph, const int* err) {
    b_physics(p, s, d_th_mp, d_qv_mp, d_qc_mp, d_qr_mp, d_qr_sed, d_prec, d_th_rd, d_u_sf, d_th_sf, d_qv_sf, ph, err, blockIdx.x, blockIdx.y);
}

// ----------------------------------------------------------------------------- stage prologue

// diagnostics (moist.jl:1048-1062) and face velocities u_face, w_face (1091-1097, 1185-1189)
template <class T>
__device__ __forceinline__ void b_diag(DevParams<T> p, StateP<T> s, T* pres, T* theta, T* rt2pres, T* u_face,
                                       T* w_face, const int* err, int bx, int by) {
    const int i = bx * blockDim.x + threadIdx.x;
    const int k = by * blockDim.y + threadIdx.y;
    const int nx = p.nx, nz = p.nz, P = p.P;
    if (i >= nx || k >= nz || halted(err)) return;
    const size_t c = MOIST_IDX(k, i);
    const T rho = ro(s.rho + c), rt = ro(s.rt + c);
    const T qv = ro(s.qv + c) / rho, qc = ro(s.qc + c) / rho, qr = ro(s.qr + c) / rho;
    const T qd = T(1.0) - qv - qc - qr;
    const T r = p.Rd * qd + p.Rv * qv;
    const T cp = p.Cpd * qd + p.Cpv * qv + p.Cpl * (qc + qr);
    const T cv = cp - r;
    const T pr = p.P0 * mm::mpow(r * rt / p.P0, cp / cv);
    pres[c] = pr;
    theta[c] = rt / rho;
    rt2pres[c] = cp / cv * pr / rt;
    const int ip = wrapx(i + 1, nx);
    u_face[c] = ro(s.ru + c) * T(2.0) / (rho + ro(s.rho + (MOIST_IDX(k, ip))));
    if (k < nz - 1) w_face[c] = ro(s.rw + c) / f2h(rho, ro(s.rho + (c + P)), p.dz[k], p.dz[k + 1]);
}
template <class T>
__global__ void k_diag(DevParams<T> p, StateP<T> s, T* pres, T* theta, T* rt2pres, T* u_face,                        T* w_face, const int* err) {
    b_diag(p, s, pres, theta, rt2pres, u_face, w_face, err, blockIdx.x, blockIdx.y);
}

// columns of the per-row reciprocal table DevParams::trcp (filled by the host in double
// precision from the denominators as the type T forms them)
enum {
    TR_DX = 0,     // 1 / dx
    TR_SIX,        // 1 / 6 (third-order upwind faces)
    TR_DZ,         // 1 / dz[k]
    TR_DZ_KP1,     // 1 / dz[k+1]
    TR_SUM_KP,     // 1 / (dz[k] + dz[k+1])
    TR_SUM_KM,     // 1 / (dz[k-1] + dz[k])
    TR_ZD_KP,      // 1 / (z[k+1] - z[k])
    TR_ZD_KM,      // 1 / (z[k] - z[k-1])
    TR_ZSUM,       // 1 / (z[k] + z[k+1])
    TEND_NRCP
};

// the stencil fields of the slow tendencies (tend_cell reads them through an accessor)
enum { TS_RU = 0, TS_RW, TS_UF, TS_WF, TS_TH, TS_RHO, TS_PRES, TS_NF };
constexpr int TEND_TX = 32, TEND_TY = 8, TEND_H = 2;

template <class T>
struct TendArgs {
    StateP<T> s, s0;
    PhysP<T> ph;
    const T *pres, *theta, *u_face, *w_face;
    T *R_rho, *R_ru, *R_rw, *R_rt;
    T *rho_p, *ru_p, *rw_p, *rt_p, *mfx, *mfz;
    T *ru_left, *rho_right;  // halo values of the stage's exchange, for surface_fluxes!
};

// slow tendencies R_rho, R_rho_u, R_rho_w, R_rho_theta (moist.jl:1079-1332) of cell (k, i)
// into out[0..3] (out[2] only for k < ke), every division through the policy D and every read of
// the stencil fields through st(field, dk, di) = field at (k + dk, i + di), x periodic
template <class T, class D, class S>
__device__ __forceinline__ void tend_cell(const DevParams<T>& p, const TendArgs<T>& a, const S& st, int i, int k, D& dv,
                                          T out[4]) {
    const int nx = p.nx, nz = p.nz, P = p.P;
    const T EPS = p.EPS, dx = p.dx, GRAV = p.GRAV;
    const double* rc = p.trcp + (size_t)k * TEND_NRCP;
    // quotient x / d with the denominator's reciprocal rc[j]
    auto Q = [&](T x, T d, int j) { return dv.q(x, d, rc[j]); };
    auto up3q = [&](T flux, T a_, T b_, T c_) {  // up3 (model.cuh) with its division by 6
        return Q(flux * (-a_ + T(5.0) * b_ + T(2.0) * c_), T(6.0), TR_SIX);
    };
    // f2h (moist.jl:249) over the faces of this cell: (dz[k], dz[k+1]), (dz[k-1], dz[k]), (z[k], z[k+1])
    auto f2h_kp = [&](T v1, T v2, T d1, T d2) { return Q(v1 * d2 + v2 * d1, d1 + d2, TR_SUM_KP); };
    auto f2h_km = [&](T v1, T v2, T d1, T d2) { return Q(v1 * d2 + v2 * d1, d1 + d2, TR_SUM_KM); };
    auto f2h_z = [&](T v1, T v2, T d1, T d2) { return Q(v1 * d2 + v2 * d1, d1 + d2, TR_ZSUM); };
    const T* dz = p.dz;
    const T* z = p.z;
    const int ke = nz - 1;
    const size_t c = MOIST_IDX(k, i);

    // --- R_rho (1079-1086)
    {
        const T flux_kp = k == ke ? T(0.0) : st(TS_RW, 0, 0);
        const T flux_km = k == 0 ? T(0.0) : st(TS_RW, -1, 0);
        const T advection = -(Q(st(TS_RU, 0, 0) - st(TS_RU, 0, -1), dx, TR_DX) + Q(flux_kp - flux_km, dz[k], TR_DZ));
        out[0] = advection + ro(a.ph.d_rho + c);
    }
    // --- R_rho_u (1098-1178)
    {
        const T rho_u_ip = T(0.5) * (st(TS_RU, 0, 0) + st(TS_RU, 0, 1));
        T f_ip;
        if (rho_u_ip > EPS)
            f_ip = up3q(rho_u_ip, st(TS_UF, 0, -1), st(TS_UF, 0, 0), st(TS_UF, 0, 1));
        else if (rho_u_ip < -EPS)
            f_ip = up3q(rho_u_ip, st(TS_UF, 0, 2), st(TS_UF, 0, 1), st(TS_UF, 0, 0));
        else
            f_ip = rho_u_ip * (st(TS_UF, 0, 0) + st(TS_UF, 0, 1)) * T(0.5);
        const T rho_u_im = T(0.5) * (st(TS_RU, 0, -1) + st(TS_RU, 0, 0));
        T f_im;
        if (rho_u_im > EPS)
            f_im = up3q(rho_u_im, st(TS_UF, 0, -2), st(TS_UF, 0, -1), st(TS_UF, 0, 0));
        else if (rho_u_im < -EPS)
            f_im = up3q(rho_u_im, st(TS_UF, 0, 1), st(TS_UF, 0, 0), st(TS_UF, 0, -1));
        else
            f_im = rho_u_im * (st(TS_UF, 0, -1) + st(TS_UF, 0, 0)) * T(0.5);
        const T druudx = Q(f_ip - f_im, dx, TR_DX);
        T f_kp;
        if (k == ke) {
            f_kp = T(0.0);
        } else {
            const T rho_w_kp = T(0.5) * (st(TS_RW, 0, 0) + st(TS_RW, 0, 1));
            if (rho_w_kp > EPS && k > 0)
                f_kp = up3q(rho_w_kp, st(TS_UF, -1, 0), st(TS_UF, 0, 0), st(TS_UF, 1, 0));
            else if (rho_w_kp < -EPS && k < ke - 1)
                f_kp = up3q(rho_w_kp, st(TS_UF, 2, 0), st(TS_UF, 1, 0), st(TS_UF, 0, 0));
            else
                f_kp = rho_w_kp * f2h_kp(st(TS_UF, 0, 0), st(TS_UF, 1, 0), dz[k], dz[k + 1]);
        }
        T f_km;
        if (k == 0) {
            f_km = T(0.0);
        } else {
            const T rho_w_km = T(0.5) * (st(TS_RW, -1, 0) + st(TS_RW, -1, 1));
            if (rho_w_km > EPS && k > 1)
                f_km = up3q(rho_w_km, st(TS_UF, -2, 0), st(TS_UF, -1, 0), st(TS_UF, 0, 0));
            else if (rho_w_km < -EPS && k < ke)
                f_km = up3q(rho_w_km, st(TS_UF, 1, 0), st(TS_UF, 0, 0), st(TS_UF, -1, 0));
            else
                f_km = rho_w_km * f2h_km(st(TS_UF, -1, 0), st(TS_UF, 0, 0), dz[k - 1], dz[k]);
        }
        const T drwudz = Q(f_kp - f_km, dz[k], TR_DZ);
        const T advection = -druudx - drwudz;
        const T u_ip = Q(st(TS_UF, 0, 1) - st(TS_UF, 0, 0), dx, TR_DX);
        const T u_im = Q(st(TS_UF, 0, 0) - st(TS_UF, 0, -1), dx, TR_DX);
        const T u_xx = Q(u_ip * st(TS_RHO, 0, 1) - u_im * st(TS_RHO, 0, 0), dx, TR_DX);
        const T u_kp = k == ke ? T(0.0) : Q(st(TS_UF, 1, 0) - st(TS_UF, 0, 0), z[k + 1] - z[k], TR_ZD_KP);
        const T u_km = k == 0 ? T(0.0) : Q(st(TS_UF, 0, 0) - st(TS_UF, -1, 0), z[k] - z[k - 1], TR_ZD_KM);
        const T rho_kp = k == ke ? T(0.0) : T(0.25) * (st(TS_RHO, 0, 0) + st(TS_RHO, 1, 0) + st(TS_RHO, 0, 1) + st(TS_RHO, 1, 1));
        const T rho_km = k == 0 ? T(0.0) : T(0.25) * (st(TS_RHO, -1, 0) + st(TS_RHO, 0, 0) + st(TS_RHO, -1, 1) + st(TS_RHO, 0, 1));
        const T u_zz = Q(u_kp * rho_kp - u_km * rho_km, dz[k], TR_DZ);
        const T diffusion = p.nu * (u_xx + u_zz);
        const T dpdx = Q(st(TS_PRES, 0, 1) - st(TS_PRES, 0, 0), dx, TR_DX);
        out[1] = advection - dpdx + diffusion + ro(a.ph.d_u + c);
    }
    // --- R_rho_w (1190-1278)
    if (k < ke) {
        const T rho_u_ip = f2h_z(st(TS_RU, 0, 0), st(TS_RU, 1, 0), z[k], z[k + 1]);  // z weights, as written (1196)
        T f_ip;
        if (rho_u_ip > EPS)
            f_ip = up3q(rho_u_ip, st(TS_WF, 0, -1), st(TS_WF, 0, 0), st(TS_WF, 0, 1));
        else if (rho_u_ip < -EPS)
            f_ip = up3q(rho_u_ip, st(TS_WF, 0, 2), st(TS_WF, 0, 1), st(TS_WF, 0, 0));
        else
            f_ip = rho_u_ip * (st(TS_WF, 0, 0) + st(TS_WF, 0, 1)) * T(0.5);
        const T rho_u_im = f2h_kp(st(TS_RU, 0, -1), st(TS_RU, 1, -1), dz[k], dz[k + 1]);
        T f_im;
        if (rho_u_im > EPS)
            f_im = up3q(rho_u_im, st(TS_WF, 0, -2), st(TS_WF, 0, -1), st(TS_WF, 0, 0));
        else if (rho_u_im < -EPS)
            f_im = up3q(rho_u_im, st(TS_WF, 0, 1), st(TS_WF, 0, 0), st(TS_WF, 0, -1));
        else
            f_im = rho_u_im * (st(TS_WF, 0, -1) + st(TS_WF, 0, 0)) * T(0.5);
        const T drwudx = Q(f_ip - f_im, dx, TR_DX);
        T f_kp;
        if (k == ke - 1) {
            f_kp = T(0.0);
        } else {
            const T rho_w_kp = f2h_kp(st(TS_RW, 0, 0), st(TS_RW, 1, 0), dz[k], dz[k + 1]);
            if (rho_w_kp > EPS && k > 0)
                f_kp = up3q(rho_w_kp, st(TS_WF, -1, 0), st(TS_WF, 0, 0), st(TS_WF, 1, 0));
            else if (rho_w_kp < -EPS && k < ke - 2)
                f_kp = up3q(rho_w_kp, st(TS_WF, 2, 0), st(TS_WF, 1, 0), st(TS_WF, 0, 0));
            else
                f_kp = rho_w_kp * f2h_kp(st(TS_WF, 0, 0), st(TS_WF, 1, 0), dz[k], dz[k + 1]);
        }
        T f_km;
        if (k == 0) {
            f_km = T(0.0);
        } else {
            const T rho_w_km = f2h_km(st(TS_RW, -1, 0), st(TS_RW, 0, 0), dz[k - 1], dz[k]);
            if (rho_w_km > EPS && k > 1)
                f_km = up3q(rho_w_km, st(TS_WF, -2, 0), st(TS_WF, -1, 0), st(TS_WF, 0, 0));
            else if (rho_w_km < -EPS && k < ke - 1)
                f_km = up3q(rho_w_km, st(TS_WF, 1, 0), st(TS_WF, 0, 0), st(TS_WF, -1, 0));
            else
                f_km = rho_w_km * f2h_km(st(TS_WF, -1, 0), st(TS_WF, 0, 0), dz[k - 1], dz[k]);
        }
        const T drwwdz = Q(f_kp - f_km, z[k + 1] - z[k], TR_ZD_KP);
        const T advection = -drwudx - drwwdz;
        const T w_ip = Q(st(TS_WF, 0, 1) - st(TS_WF, 0, 0), dx, TR_DX);
        const T w_im = Q(st(TS_WF, 0, 0) - st(TS_WF, 0, -1), dx, TR_DX);
        const T rho_ip = T(0.25) * (st(TS_RHO, 0, 0) + st(TS_RHO, 1, 0) + st(TS_RHO, 0, 1) + st(TS_RHO, 1, 1));
        const T rho_im = T(0.25) * (st(TS_RHO, 0, -1) + st(TS_RHO, 1, -1) + st(TS_RHO, 0, 0) + st(TS_RHO, 1, 0));
        const T w_xx = Q(w_ip * rho_ip - w_im * rho_im, dx, TR_DX);
        const T w_kp = k == ke - 1 ? T(0.0) : Q(st(TS_WF, 1, 0) - st(TS_WF, 0, 0), dz[k + 1], TR_DZ_KP1);
        const T w_km = k == 0 ? T(0.0) : Q(st(TS_WF, 0, 0) - st(TS_WF, -1, 0), dz[k], TR_DZ);
        const T w_zz = Q(w_kp * st(TS_RHO, 1, 0) - w_km * st(TS_RHO, 0, 0), z[k + 1] - z[k], TR_ZD_KP);
        const T diffusion = p.nu * (w_xx + w_zz);
        T sigma = T(0.0);
        const T zfk = p.zf[k];
        if (zfk > (T(1.0) - p.zf_sponge) * p.H)
            sigma = (GRAV / T(30.0)) * ((zfk - (T(1.0) - p.zf_sponge) * p.H) / (p.zf_sponge * p.H));
        const T sponge = -sigma * st(TS_RW, 0, 0);
        const T dpdz = Q(st(TS_PRES, 1, 0) - st(TS_PRES, 0, 0), z[k + 1] - z[k], TR_ZD_KP);
        const T buoyancy = -GRAV * (st(TS_RHO, 0, 0) + st(TS_RHO, 1, 0)) * T(0.5);
        out[2] = advection - dpdz + buoyancy + diffusion + sponge;
    }
    // --- R_rho_theta (1284-1331)
    {
        const T ru_i = st(TS_RU, 0, 0), ru_m = st(TS_RU, 0, -1);
        T f_ip, f_im, f_kp, f_km;
        if (ru_i > EPS)
            f_ip = up3q(ru_i, st(TS_TH, 0, -1), st(TS_TH, 0, 0), st(TS_TH, 0, 1));
        else if (ru_i < -EPS)
            f_ip = up3q(ru_i, st(TS_TH, 0, 2), st(TS_TH, 0, 1), st(TS_TH, 0, 0));
        else
            f_ip = ru_i * (st(TS_TH, 0, 0) + st(TS_TH, 0, 1)) * T(0.5);
        if (ru_m > EPS)
            f_im = up3q(ru_m, st(TS_TH, 0, -2), st(TS_TH, 0, -1), st(TS_TH, 0, 0));
        else if (ru_m < -EPS)
            f_im = up3q(ru_m, st(TS_TH, 0, 1), st(TS_TH, 0, 0), st(TS_TH, 0, -1));
        else
            f_im = ru_m * (st(TS_TH, 0, -1) + st(TS_TH, 0, 0)) * T(0.5);
        if (k == ke) {
            f_kp = T(0.0);
        } else {
            const T w = st(TS_RW, 0, 0);
            if (w > EPS && k > 0)
                f_kp = up3q(w, st(TS_TH, -1, 0), st(TS_TH, 0, 0), st(TS_TH, 1, 0));
            else if (w < -EPS && k < ke - 1)
                f_kp = up3q(w, st(TS_TH, 2, 0), st(TS_TH, 1, 0), st(TS_TH, 0, 0));
            else
                f_kp = w * f2h_kp(st(TS_TH, 0, 0), st(TS_TH, 1, 0), dz[k], dz[k + 1]);
        }
        if (k == 0) {
            f_km = T(0.0);
        } else {
            const T w = st(TS_RW, -1, 0);
            if (w > EPS && k > 1)
                f_km = up3q(w, st(TS_TH, -2, 0), st(TS_TH, -1, 0), st(TS_TH, 0, 0));
            else if (w < -EPS && k < ke)
                f_km = up3q(w, st(TS_TH, 1, 0), st(TS_TH, 0, 0), st(TS_TH, -1, 0));
            else
                f_km = w * f2h_km(st(TS_TH, -1, 0), st(TS_TH, 0, 0), dz[k - 1], dz[k]);
        }
        const T advection = -(Q(f_ip - f_im, dx, TR_DX) + Q(f_kp - f_km, dz[k], TR_DZ));
        out[3] = advection + ro(a.ph.d_th + c);
    }
}

// Division policies of tend_cell: q(x, d, y) = x / d with y = 1/d in double precision. Every
// denominator of the slow tendencies is a grid constant (dx, 6, dz and z differences and sums
// of the cell's row), whose reciprocals are tabulated once per context (TEND_NRCP per row).
template <class T>
struct TendDivIEEE {
    __device__ __forceinline__ T q(T x, T d, double) const { return x / d; }
};
// Float32: RN32(RN64(x * y)), the IEEE quotient except at subnormal ties (fastdiv.cuh), with
// every quotient in 0 < |q| <= 2^-126 recorded in the guard word; such a cell is recomputed
// with IEEE division.
struct TendDiv64 {
    unsigned g = ~0u;
    __device__ __forceinline__ float q(float x, float, double y) {
        const float r = div64(x, y);
        subnormal_guard(g, r);
        return r;
    }
};

// The stencil fields of a (TEND_TY x TEND_TX) block of cells with a two-cell halo, staged in
// shared memory: every block issues all its loads at once (coalesced rows, x periodic) and the
// cells then read their 45 stencil values from the tile.
template <class T>
struct TendTile {
    T f[TS_NF][TEND_TY + 2 * TEND_H][TEND_TX + 2 * TEND_H];
};
template <class T>
struct TendStaged {
    const TendTile<T>& t;
    int tx, ty;
    __device__ __forceinline__ T operator()(int f, int dk, int di) const {
        return t.f[f][ty + TEND_H + dk][tx + TEND_H + di];
    }
};

// slow tendencies (moist.jl:1079-1332), perturbation initialisation and the saved momentum
// fluxes (1339-1348) of one block of TEND_TY x TEND_TX cells (blockDim = (TEND_TX, TEND_TY))
template <class T>
__device__ __forceinline__ void b_tend(DevParams<T> p, TendArgs<T> a, const int* err, int bx, int by) {
    __shared__ TendTile<T> tile;
    if (halted(err)) return;  // the same for every thread of the launch
    const int nx = p.nx, nz = p.nz, P = p.P;
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int i0 = bx * TEND_TX, k0 = by * TEND_TY;
    {
        const T* src[TS_NF] = {a.s.ru, a.s.rw, a.u_face, a.w_face, a.theta, a.s.rho, a.pres};
        constexpr int W = TEND_TX + 2 * TEND_H, H = TEND_TY + 2 * TEND_H;
        for (int j = ty * TEND_TX + tx; j < W * H; j += TEND_TX * TEND_TY) {
            const int rr = j / W, cc = j % W;
            const int kk = k0 - TEND_H + rr;
            int ii = (i0 - TEND_H + cc) % nx;
            if (ii < 0) ii += nx;
            const bool ok = kk >= 0 && kk < nz;  // rows outside the column are never read
            const size_t off = ok ? MOIST_IDX(kk, ii) : 0;
#pragma unroll
            for (int f = 0; f < TS_NF; f++) tile.f[f][rr][cc] = ok ? ro(src[f] + off) : T(0);
        }
    }
    __syncthreads();
    const int i = i0 + tx, k = k0 + ty;
    if (i >= nx || k >= nz) return;
    const TendStaged<T> st{tile, tx, ty};
    const size_t c = MOIST_IDX(k, i);
    if (k == 0 && i == 0) {
        *a.ru_left = ro(a.s.ru + MOIST_IDX(0, nx - 1));
        *a.rho_right = ro(a.s.rho + MOIST_IDX(0, 0));
    }
    T out[4];
    if constexpr (sizeof(T) == 4) {
        TendDiv64 dv;
        tend_cell(p, a, st, i, k, dv, out);
        if (guard_hit(dv.g)) {  // rare: recompute the cell with IEEE division
            TendDivIEEE<T> di;
            tend_cell(p, a, st, i, k, di, out);
        }
    } else {
        TendDivIEEE<T> di;
        tend_cell(p, a, st, i, k, di, out);
    }
    a.R_rho[c] = out[0];
    a.R_ru[c] = out[1];
    if (k < nz - 1) a.R_rw[c] = out[2];
    a.R_rt[c] = out[3];
    // --- perturbations and saved momentum fluxes (1339-1348)
    a.rho_p[c] = ro(a.s0.rho + c) - ro(a.s.rho + c);
    a.ru_p[c] = ro(a.s0.ru + c) - ro(a.s.ru + c);
    a.rw_p[c] = ro(a.s0.rw + c) - ro(a.s.rw + c);
    a.rt_p[c] = ro(a.s0.rt + c) - ro(a.s.rt + c);
    a.mfx[c] = ro(a.s.ru + c);
    a.mfz[c] = ro(a.s.rw + c);
}
template <class T>
__global__ void k_tend(DevParams<T> p, TendArgs<T> a, const int* err) {
    b_tend(p, a, err, blockIdx.x, blockIdx.y);
}

// Per-stage factorisation of the w-p tridiagonal system (implicit_correction!, moist.jl:
// 982-1021; solve_tridiagonal!, 956-966). The coefficients depend only on theta, rt2pres and
// dt_s, which are fixed during a stage, so the pivots and modified super-diagonal are formed
// once per stage; each substep then repeats only the right-hand-side recurrence.
template <class T, class TT>
__device__ __forceinline__ void b_thomas_col(DevParams<T> p, const T* theta, const T* rt2pres, T dt_s, T* ta, T* tb,
                                             T* tc, TT* tcp, TT* tpiv, const int* err, int bx) {
    const int i = bx * blockDim.x + threadIdx.x;
    const int nx = p.nx, nz = p.nz, P = p.P;
    if (i >= nx || halted(err)) return;
    const int ke = nz - 1, n = nz - 1;
    const T fact_tp = T(0.5) * (T(1.0) + p.beta);
    const T dt_tp2 = (dt_s * fact_tp) * (dt_s * fact_tp);
    // the walk keeps theta, rt2pres, dz and z of the levels it needs in registers and reads the
    // next level's new values one level ahead, so that no level waits for its loads
    auto TH = [&](int kk) { return kk <= ke ? ro(theta + MOIST_IDX(kk, i)) : T(0); };
    auto R2 = [&](int kk) { return kk <= ke ? ro(rt2pres + MOIST_IDX(kk, i)) : T(0); };
    auto DZ = [&](int kk) { return kk <= ke ? ro(p.dz + kk) : T(1); };
    auto ZZ = [&](int kk) { return kk <= ke ? ro(p.z + kk) : T(0); };
    T t1 = TH(1), t2 = TH(2);          // theta at k+1, k+2
    T rk = R2(0), rkp = R2(1);         // rt2pres at k, k+1
    T d0 = DZ(0), d1 = DZ(1), d2 = DZ(2);  // dz at k, k+1, k+2
    T z0 = ZZ(0), z1 = ZZ(1);          // z at k, k+1
    T th_prev = T(0), th_cur = f2h(TH(0), t1, d0, d1);
    TT cp_prev = TT(0);
    for (int j = 0; j < n; j++) {
        const int k = j;
        const T n_t = TH(k + 3), n_r = R2(k + 2), n_d = DZ(k + 3), n_z = ZZ(k + 2);
        const T th_next = (k + 1 <= ke - 1) ? f2h(t1, t2, d1, d2) : T(0);
        const T b = dt_tp2 * (rk / d0 + rkp / d1) * th_cur / (z1 - z0);
        const T a = (k > 0) ? -dt_tp2 * (rk * th_prev / ((z1 - z0) * d0) - p.GRAV / (d0 + d1)) : T(0);
        const T c = (k < ke - 1) ? -dt_tp2 * (rkp * th_next / ((z1 - z0) * d1) + p.GRAV / (d0 + d1)) : T(0);
        ta[MOIST_IDX(j, i)] = a;
        tb[MOIST_IDX(j, i)] = b;
        tc[MOIST_IDX(j, i)] = c;
        const T bb = b + T(1.0);
        TT piv, cpj;
        if (j == 0) {
            piv = (TT)bb;
            cpj = (TT)c / piv;
        } else {
            piv = (TT)bb - (TT)a * cp_prev;
            cpj = (TT)c / piv;
        }
        tcp[MOIST_IDX(j, i)] = cpj;
        tpiv[MOIST_IDX(j, i)] = piv;
        cp_prev = cpj;
        th_prev = th_cur;
        th_cur = th_next;
        t1 = t2;
        t2 = n_t;
        rk = rkp;
        rkp = n_r;
        d0 = d1;
        d1 = d2;
        d2 = n_d;
        z0 = z1;
        z1 = n_z;
    }
}


template <class T, class TT>
struct SubArgs {
    const T *R_rho, *R_ru, *R_rw, *R_rt, *theta, *rt2pres, *s_rw;
    const T *ru_in, *rt_in, *rt_old;  // rho_u_p, rho_theta_p and rho_theta_p_old at substep start
    T *ru_out, *rt_out;               // rho_u_p, rho_theta_p after the substep
    T *rho_p, *rw_p, *mfx, *mfz;      // updated in place (each column owns its entries)
    const T *ta, *tb, *tc;
    const TT *tcp, *tpiv;
    TT* dprime;                       // scratch [nz][P]
};

// One acoustic substep (moist.jl:1355-1459), one thread per column i (the ensembles' form):
// horizontal forward
// step of rho_u_p at faces i-1/2 (recomputed, bitwise equal to column i-1's) and i+1/2,
// explicit rho_p / rho_theta_p, off-centred right-hand side and elimination going up the
// column; back substitution for rho_w_p fused with the vertical rho_p / rho_theta_p updates
// and the time-averaged momentum fluxes going down. The inputs no thread of the launch writes
// (tendencies, theta, rt2pres, s.rho_w, the substep-start rho_u_p / rho_theta_p buffers, the
// stage factors) are read through ro().
template <class T, class TT>
__device__ __forceinline__ void b_substep_col(DevParams<T> p, SubArgs<T, TT> a, T dt_s, T ns_T, double fact_tp64,
                                              const int* err, int bx) {
    const int i = bx * blockDim.x + threadIdx.x;
    const int nx = p.nx, nz = p.nz, P = p.P;
    if (i >= nx || halted(err)) return;
    const T dx = p.dx, EPS = p.EPS;
    const T* dz = p.dz;
    const T* z = p.z;
    const int im = wrapx(i - 1, nx), ip = wrapx(i + 1, nx);
    const int ke = nz - 1, n = nz - 1;
    const T fact_tpT = T(0.5) * (T(1.0) + p.beta);
    const T fact_tmT = T(0.5) * (T(1.0) - p.beta);
    const T fact = fact_tmT / fact_tpT;
    auto u_update = [&](int k, int cc) {
        const int cn = wrapx(cc + 1, nx);
        const size_t a0 = MOIST_IDX(k, cc), a1 = MOIST_IDX(k, cn);
        T grad_x = (ro(a.rt_in + a1) - ro(a.rt_in + a0)) / dx;
        const T grad_x_old = (ro(a.rt_old + a1) - ro(a.rt_old + a0)) / dx;
        grad_x = grad_x + p.gamma_d * (grad_x - grad_x_old);
        const T rt2pres_h = (ro(a.rt2pres + a0) + ro(a.rt2pres + a1)) * T(0.5);
        return ro(a.ru_in + a0) + dt_s * (ro(a.R_ru + a0) - rt2pres_h * grad_x);
    };
    T rho_tp_prev = T(0), rt_tp_prev = T(0);
    TT dprev = TT(0);
    for (int k = 0; k < nz; k++) {
        const size_t c = MOIST_IDX(k, i);
        const T u_m = u_update(k, im);
        const T u_p = u_update(k, i);
        a.ru_out[c] = u_p;
        a.mfx[c] = a.mfx[c] + u_p / ns_T;
        T advection = -(u_p - u_m) / dx;
        T inc = dt_s * (ro(a.R_rho + c) + advection);
        const T rho_tp = (T)((double)a.rho_p[c] + fact_tp64 * (double)inc);
        a.rho_p[c] = a.rho_p[c] + inc;
        const T th_i = ro(a.theta + c), th_ip = ro(a.theta + MOIST_IDX(k, ip)), th_im = ro(a.theta + MOIST_IDX(k, im));
        const T flux_ip = (th_ip + th_i) * T(0.5) * u_p;
        const T flux_im = (th_i + th_im) * T(0.5) * u_m;
        advection = -(flux_ip - flux_im) / dx;
        inc = dt_s * (ro(a.R_rt + c) + advection);
        const T rtp = ro(a.rt_in + c);
        const T rt_tp = (T)((double)rtp + fact_tp64 * (double)inc);
        a.rt_out[c] = rtp + inc;
        if (k >= 1) {
            const int j = k - 1;
            const size_t cj = c - P;
            const T buoyancy = (rt_tp - rt_tp_prev) / (z[k] - z[j]);
            const T grav = -p.GRAV * T(0.5) * (rho_tp + rho_tp_prev);
            const T rt2pres_h = (ro(a.rt2pres + cj) + ro(a.rt2pres + c)) * T(0.5);
            const T drho_w = dt_s * (ro(a.R_rw + cj) - rt2pres_h * buoyancy + grav);
            const T w_j = a.rw_p[cj];
            const T aj = ro(a.ta + cj);
            T d = w_j + drho_w;
            if (j > 0) d -= aj * fact * w_j;
            d -= ro(a.tb + cj) * fact * w_j;
            if (j < n - 1) d -= ro(a.tc + cj) * fact * a.rw_p[c];
            TT dp;
            if (j == 0)
                dp = (TT)d / ro(a.tpiv + cj);
            else
                dp = ((TT)d - (TT)aj * dprev) / ro(a.tpiv + cj);
            a.dprime[cj] = dp;
            dprev = dp;
        }
        rho_tp_prev = rho_tp;
        rt_tp_prev = rt_tp;
    }
    // Back substitution (moist.jl:968-970) going down, fused with the vertical rho_p /
    // rho_theta_p updates (1412-1446) and the momentum flux average (1452-1458) of cell j + 1,
    // whose two face values rho_w_p[j + 1] (w_hi) and rho_w_p[j] are known once x_j is: every
    // cell's arithmetic is that of separate passes.
    const T* th = a.theta;
    auto vertical = [&](int k, T w_k, T w_km) {
        const size_t c = MOIST_IDX(k, i);
        {
            const T flux_kp = k == ke ? T(0.0) : w_k;
            const T flux_km = k == 0 ? T(0.0) : w_km;
            const T advection = -(flux_kp - flux_km) / dz[k];
            a.rho_p[c] = a.rho_p[c] + dt_s * advection;
        }
        T flux_kp, flux_km;
        if (k == ke) {
            flux_kp = T(0.0);
        } else {
            const T wp = w_k;
            if (wp > EPS && k > 0)
                flux_kp = up3(wp, ro(th + c - P), ro(th + c), ro(th + c + P));
            else if (ro(a.s_rw + c) < -EPS && k < ke - 1)  // selector on s.rho_w, as written (1426)
                flux_kp = up3(wp, ro(th + c + 2 * P), ro(th + c + P), ro(th + c));
            else
                flux_kp = wp * f2h(ro(th + c), ro(th + c + P), dz[k], dz[k + 1]);
        }
        if (k == 0) {
            flux_km = T(0.0);
        } else {
            const T wp = w_km;
            const T sw = ro(a.s_rw + c - P);
            if (sw > EPS && k > 1)
                flux_km = up3(wp, ro(th + c - 2 * P), ro(th + c - P), ro(th + c));
            else if (sw < -EPS && k < ke)
                flux_km = up3(wp, ro(th + c + P), ro(th + c), ro(th + c - P));
            else
                flux_km = wp * f2h(ro(th + c - P), ro(th + c), dz[k - 1], dz[k]);
        }
        const T advection = -(flux_kp - flux_km) / dz[k];
        a.rt_out[c] = a.rt_out[c] + dt_s * advection;
        if (k < ke) a.mfz[c] = a.mfz[c] + w_k / ns_T;
    };
    TT x = dprev;
    T w_hi = (T)x;
    a.rw_p[MOIST_IDX(n - 1, i)] = w_hi;
    vertical(ke, T(0.0), w_hi);
    for (int j = n - 2; j >= 0; j--) {
        x = a.dprime[MOIST_IDX(j, i)] - ro(a.tcp + MOIST_IDX(j, i)) * x;
        const T w_j = (T)x;
        a.rw_p[MOIST_IDX(j, i)] = w_j;
        vertical(j + 1, w_hi, w_j);
        w_hi = w_j;
    }
    vertical(0, w_hi, T(0.0));
}


// b_substep_col with its loads issued one level ahead. A column walk spends most of its time
// waiting for each level's loads: the loads of level k + 1 cannot move above the stores of level
// k to the arrays the walk updates in place (rho_p, mfx, rt_out, ...), so every level waits a
// full memory latency. Here every input of the next level is read into registers before the
// current level's arithmetic and stores (the addresses differ, so the values are those the
// walk would read later), and the values a level shares with its neighbour level (rho_w_p,
// rt2pres going up; theta, s.rho_w going down) stay in registers. The arithmetic is that of
// b_substep_col, operation for operation.
template <class T, class TT>
struct SubUpLevel {
    T rt_m, rt_c, rt_p, ro_m, ro_c, ro_p, r2_m, r2_c, r2_p, ru_m, ru_c, Ru_m, Ru_c;
    T mfx, Rrho, rhop, th_c, th_p, th_m, Rrt;
    T Rrw, rwp, ta, tb, tc;  // face k: R_rho_w, rho_w_p and the factors (used by level k + 1)
    TT piv;
};

template <class T, class TT>
__device__ __forceinline__ void b_substep_col_pf(DevParams<T> p, SubArgs<T, TT> a, T dt_s, T ns_T, double fact_tp64,
                                                 const int* err, int bx) {
    const int i = bx * blockDim.x + threadIdx.x;
    const int nx = p.nx, nz = p.nz, P = p.P;
    if (i >= nx || halted(err)) return;
    const T dx = p.dx, EPS = p.EPS;
    const T* dz = p.dz;
    const T* z = p.z;
    const int im = wrapx(i - 1, nx), ip = wrapx(i + 1, nx);
    const int ke = nz - 1, n = nz - 1;
    const T fact_tpT = T(0.5) * (T(1.0) + p.beta);
    const T fact_tmT = T(0.5) * (T(1.0) - p.beta);
    const T fact = fact_tmT / fact_tpT;
    using L = SubUpLevel<T, TT>;
    auto load_up = [&](int k, L& v) {
        const size_t c = MOIST_IDX(k, i), cm = MOIST_IDX(k, im), cp = MOIST_IDX(k, ip);
        v.rt_m = ro(a.rt_in + cm);
        v.rt_c = ro(a.rt_in + c);
        v.rt_p = ro(a.rt_in + cp);
        v.ro_m = ro(a.rt_old + cm);
        v.ro_c = ro(a.rt_old + c);
        v.ro_p = ro(a.rt_old + cp);
        v.r2_m = ro(a.rt2pres + cm);
        v.r2_c = ro(a.rt2pres + c);
        v.r2_p = ro(a.rt2pres + cp);
        v.ru_m = ro(a.ru_in + cm);
        v.ru_c = ro(a.ru_in + c);
        v.Ru_m = ro(a.R_ru + cm);
        v.Ru_c = ro(a.R_ru + c);
        v.mfx = a.mfx[c];
        v.Rrho = ro(a.R_rho + c);
        v.rhop = a.rho_p[c];
        v.th_c = ro(a.theta + c);
        v.th_p = ro(a.theta + cp);
        v.th_m = ro(a.theta + cm);
        v.Rrt = ro(a.R_rt + c);
        v.Rrw = ro(a.R_rw + c);
        v.rwp = a.rw_p[c];
        v.ta = ro(a.ta + c);
        v.tb = ro(a.tb + c);
        v.tc = ro(a.tc + c);
        v.piv = ro(a.tpiv + c);
    };
    L cur, nxt, prv;
    load_up(0, cur);
    T rho_tp_prev = T(0), rt_tp_prev = T(0);
    TT dprev = TT(0);
    for (int k = 0; k < nz; k++) {
        if (k + 1 < nz) load_up(k + 1, nxt);
        const size_t c = MOIST_IDX(k, i);
        // u_update at faces i-1/2 (column im) and i+1/2 (column i)
        T grad_m = (cur.rt_c - cur.rt_m) / dx;
        const T grad_m_old = (cur.ro_c - cur.ro_m) / dx;
        grad_m = grad_m + p.gamma_d * (grad_m - grad_m_old);
        const T rh_m = (cur.r2_m + cur.r2_c) * T(0.5);
        const T u_m = cur.ru_m + dt_s * (cur.Ru_m - rh_m * grad_m);
        T grad_p = (cur.rt_p - cur.rt_c) / dx;
        const T grad_p_old = (cur.ro_p - cur.ro_c) / dx;
        grad_p = grad_p + p.gamma_d * (grad_p - grad_p_old);
        const T rh_p = (cur.r2_c + cur.r2_p) * T(0.5);
        const T u_p = cur.ru_c + dt_s * (cur.Ru_c - rh_p * grad_p);
        a.ru_out[c] = u_p;
        a.mfx[c] = cur.mfx + u_p / ns_T;
        T advection = -(u_p - u_m) / dx;
        T inc = dt_s * (cur.Rrho + advection);
        const T rho_tp = (T)((double)cur.rhop + fact_tp64 * (double)inc);
        a.rho_p[c] = cur.rhop + inc;
        const T flux_ip = (cur.th_p + cur.th_c) * T(0.5) * u_p;
        const T flux_im = (cur.th_c + cur.th_m) * T(0.5) * u_m;
        advection = -(flux_ip - flux_im) / dx;
        inc = dt_s * (cur.Rrt + advection);
        const T rt_tp = (T)((double)cur.rt_c + fact_tp64 * (double)inc);
        a.rt_out[c] = cur.rt_c + inc;
        if (k >= 1) {
            const int j = k - 1;
            const size_t cj = c - P;
            const T buoyancy = (rt_tp - rt_tp_prev) / (ro(z + k) - ro(z + j));
            const T grav = -p.GRAV * T(0.5) * (rho_tp + rho_tp_prev);
            const T rt2pres_h = (prv.r2_c + cur.r2_c) * T(0.5);
            const T drho_w = dt_s * (prv.Rrw - rt2pres_h * buoyancy + grav);
            const T w_j = prv.rwp;
            const T aj = prv.ta;
            T d = w_j + drho_w;
            if (j > 0) d -= aj * fact * w_j;
            d -= prv.tb * fact * w_j;
            if (j < n - 1) d -= prv.tc * fact * cur.rwp;
            TT dp;
            if (j == 0)
                dp = (TT)d / prv.piv;
            else
                dp = ((TT)d - (TT)aj * dprev) / prv.piv;
            a.dprime[cj] = dp;
            dprev = dp;
        }
        rho_tp_prev = rho_tp;
        rt_tp_prev = rt_tp;
        prv = cur;
        cur = nxt;
    }
    // Back substitution going down fused with the vertical updates of cell k (moist.jl:
    // 968-970, 1412-1446, 1452-1458), as in b_substep_col: at level k the faces k (w_k, known
    // from level k + 1) and k - 1 (x_{k-1} = d'_{k-1} - c'_{k-1} x_k, computed here).
    const T* th = a.theta;
    // theta at k-2 .. k+2 and s.rho_w at k-1, k, kept in registers as k falls
    T t_m2 = ke >= 2 ? ro(th + MOIST_IDX(ke - 2, i)) : T(0);
    T t_m1 = ke >= 1 ? ro(th + MOIST_IDX(ke - 1, i)) : T(0);
    T t_0 = ro(th + MOIST_IDX(ke, i)), t_p1 = T(0), t_p2 = T(0);
    T sw_0 = ro(a.s_rw + MOIST_IDX(ke, i)), sw_m1 = ro(a.s_rw + MOIST_IDX(ke - 1, i));
    T v_rho = a.rho_p[MOIST_IDX(ke, i)], v_rt = a.rt_out[MOIST_IDX(ke, i)], v_mfz = a.mfz[MOIST_IDX(ke, i)];
    TT v_dp = dprev, v_cp = TT(0);  // d' and c' of face k - 1 (x_{ke-1} = d'_{ke-1} itself)
    TT x = TT(0);
    T w_k = T(0);
    for (int k = ke; k >= 0; k--) {
        // next level's inputs: cell k - 1 and face k - 2
        T n_rho = T(0), n_rt = T(0), n_mfz = T(0), n_t = T(0), n_sw = T(0);
        TT n_dp = TT(0), n_cp = TT(0);
        if (k >= 1) {
            const size_t cn = MOIST_IDX(k - 1, i);
            n_rho = a.rho_p[cn];
            n_rt = a.rt_out[cn];
            n_mfz = a.mfz[cn];
            if (k >= 3) n_t = ro(th + MOIST_IDX(k - 3, i));
            if (k >= 2) {
                n_sw = ro(a.s_rw + MOIST_IDX(k - 2, i));
                n_dp = a.dprime[MOIST_IDX(k - 2, i)];
                n_cp = ro(a.tcp + MOIST_IDX(k - 2, i));
            }
        }
        T w_km = T(0);
        if (k >= 1) {
            x = (k == ke) ? v_dp : v_dp - v_cp * x;
            w_km = (T)x;
            a.rw_p[MOIST_IDX(k - 1, i)] = w_km;
        }
        const size_t c = MOIST_IDX(k, i);
        {
            const T flux_kp = k == ke ? T(0.0) : w_k;
            const T flux_km = k == 0 ? T(0.0) : w_km;
            const T adv = -(flux_kp - flux_km) / ro(dz + k);
            a.rho_p[c] = v_rho + dt_s * adv;
        }
        T flux_kp, flux_km;
        if (k == ke) {
            flux_kp = T(0.0);
        } else {
            const T wp = w_k;
            if (wp > EPS && k > 0)
                flux_kp = up3(wp, t_m1, t_0, t_p1);
            else if (sw_0 < -EPS && k < ke - 1)  // selector on s.rho_w, as written (1426)
                flux_kp = up3(wp, t_p2, t_p1, t_0);
            else
                flux_kp = wp * f2h(t_0, t_p1, ro(dz + k), ro(dz + k + 1));
        }
        if (k == 0) {
            flux_km = T(0.0);
        } else {
            const T wp = w_km;
            const T sw = sw_m1;
            if (sw > EPS && k > 1)
                flux_km = up3(wp, t_m2, t_m1, t_0);
            else if (sw < -EPS && k < ke)
                flux_km = up3(wp, t_p1, t_0, t_m1);
            else
                flux_km = wp * f2h(t_m1, t_0, ro(dz + k - 1), ro(dz + k));
        }
        const T adv = -(flux_kp - flux_km) / ro(dz + k);
        a.rt_out[c] = v_rt + dt_s * adv;
        if (k < ke) a.mfz[c] = v_mfz + w_k / ns_T;
        // slide the windows down one level
        w_k = w_km;
        t_p2 = t_p1;
        t_p1 = t_0;
        t_0 = t_m1;
        t_m1 = t_m2;
        t_m2 = n_t;
        sw_0 = sw_m1;
        sw_m1 = n_sw;
        v_rho = n_rho;
        v_rt = n_rt;
        v_mfz = n_mfz;
        v_dp = n_dp;
        v_cp = n_cp;
    }
}


// Asynchronous copies global -> shared (cp.async, sm_80 and later): the copy proceeds while the
// thread computes; cp_async_wait<N>() waits until at most N of its committed groups are pending.
template <class X>
__device__ __forceinline__ void cp_async(X* s, const X* g) {
    static_assert(sizeof(X) == 4 || sizeof(X) == 8, "4- or 8-byte elements");
    const unsigned sa = (unsigned)__cvta_generic_to_shared(s);
    if constexpr (sizeof(X) == 4)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(g) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(g) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// the per-level inputs of the upward pass that b_substep_col_async stages in shared memory
enum {
    SU_RT_M = 0, SU_RT_C, SU_RT_P, SU_RO_M, SU_RO_C, SU_RO_P, SU_R2_M, SU_R2_C, SU_R2_P, SU_RU_M, SU_RU_C,
    SU_RRU_M, SU_RRU_C, SU_MFX, SU_RRHO, SU_RHOP, SU_TH_C, SU_TH_P, SU_TH_M, SU_RRT, SU_RRW, SU_RWP, SU_TA,
    SU_TB, SU_TC, SU_NV
};
// shared memory of b_substep_col_async per thread: nbuf levels of the SU_NV inputs and the pivot
template <class T, class TT>
__host__ __device__ constexpr size_t sub_async_bytes_per_thread(int nbuf) {
    return (size_t)nbuf * (SU_NV * sizeof(T) + sizeof(TT));
}

// b_substep_col_pf with the next levels' inputs brought in by asynchronous copies into this
// thread's slots of shared memory instead of registers: the copies of levels k + 1 .. k + NBUF - 1
// run during level k's arithmetic, and the registers they would hold are free, so more warps fit
// on an SM. Same arithmetic, operation for operation; the downward pass is b_substep_col_pf's.
template <class T, class TT, int NBUF>
__device__ __forceinline__ void b_substep_col_async(DevParams<T> p, SubArgs<T, TT> a, T dt_s, T ns_T,
                                                    double fact_tp64, const int* err, int bx) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int nt = blockDim.x, tid = threadIdx.x;
    const int i = bx * nt + tid;
    const int nx = p.nx, nz = p.nz, P = p.P;
    if (i >= nx || halted(err)) return;
    const T dx = p.dx, EPS = p.EPS;
    const T* dz = p.dz;
    const T* z = p.z;
    const int im = wrapx(i - 1, nx), ip = wrapx(i + 1, nx);
    const int ke = nz - 1, n = nz - 1;
    const T fact_tpT = T(0.5) * (T(1.0) + p.beta);
    const T fact_tmT = T(0.5) * (T(1.0) - p.beta);
    const T fact = fact_tmT / fact_tpT;
    T* fs = reinterpret_cast<T*>(smem_raw);                                             // [NBUF][SU_NV][nt]
    TT* ps = reinterpret_cast<TT*>(smem_raw + (size_t)NBUF * SU_NV * nt * sizeof(T));  // [NBUF][nt]
    auto slot = [&](int b, int f) { return fs + ((size_t)(b * SU_NV + f) * nt + tid); };
    auto issue = [&](int k, int b) {
        const size_t c = MOIST_IDX(k, i), cm = MOIST_IDX(k, im), cp = MOIST_IDX(k, ip);
        cp_async(slot(b, SU_RT_M), a.rt_in + cm);
        cp_async(slot(b, SU_RT_C), a.rt_in + c);
        cp_async(slot(b, SU_RT_P), a.rt_in + cp);
        cp_async(slot(b, SU_RO_M), a.rt_old + cm);
        cp_async(slot(b, SU_RO_C), a.rt_old + c);
        cp_async(slot(b, SU_RO_P), a.rt_old + cp);
        cp_async(slot(b, SU_R2_M), a.rt2pres + cm);
        cp_async(slot(b, SU_R2_C), a.rt2pres + c);
        cp_async(slot(b, SU_R2_P), a.rt2pres + cp);
        cp_async(slot(b, SU_RU_M), a.ru_in + cm);
        cp_async(slot(b, SU_RU_C), a.ru_in + c);
        cp_async(slot(b, SU_RRU_M), a.R_ru + cm);
        cp_async(slot(b, SU_RRU_C), a.R_ru + c);
        cp_async(slot(b, SU_MFX), (const T*)a.mfx + c);
        cp_async(slot(b, SU_RRHO), a.R_rho + c);
        cp_async(slot(b, SU_RHOP), (const T*)a.rho_p + c);
        cp_async(slot(b, SU_TH_C), a.theta + c);
        cp_async(slot(b, SU_TH_P), a.theta + cp);
        cp_async(slot(b, SU_TH_M), a.theta + cm);
        cp_async(slot(b, SU_RRT), a.R_rt + c);
        cp_async(slot(b, SU_RRW), a.R_rw + c);
        cp_async(slot(b, SU_RWP), (const T*)a.rw_p + c);
        cp_async(slot(b, SU_TA), a.ta + c);
        cp_async(slot(b, SU_TB), a.tb + c);
        cp_async(slot(b, SU_TC), a.tc + c);
        cp_async(ps + (size_t)b * nt + tid, a.tpiv + c);
        cp_async_commit();
    };
    for (int q = 0; q < NBUF - 1; q++) {  // levels 0 .. NBUF - 2 in flight before the walk starts
        if (q < nz)
            issue(q, q);
        else
            cp_async_commit();
    }
    // face k - 1 values the next level uses: R_rho_w, rho_w_p, the factors, the pivot, rt2pres
    T pv_r2c = T(0), pv_Rrw = T(0), pv_rwp = T(0), pv_ta = T(0), pv_tb = T(0), pv_tc = T(0);
    TT pv_piv = TT(1);
    T rho_tp_prev = T(0), rt_tp_prev = T(0);
    TT dprev = TT(0);
    for (int k = 0; k < nz; k++) {
        if (k + NBUF - 1 < nz)
            issue(k + NBUF - 1, (k + NBUF - 1) % NBUF);
        else
            cp_async_commit();     // an empty group keeps the count of pending groups uniform
        cp_async_wait<NBUF - 1>();  // level k's copies have landed
        const int bb = k % NBUF;
        auto V = [&](int f) { return *slot(bb, f); };
        const size_t c = MOIST_IDX(k, i);
        const T r2_c = V(SU_R2_C), rt_c = V(SU_RT_C), rwp = V(SU_RWP);
        T grad_m = (rt_c - V(SU_RT_M)) / dx;
        const T grad_m_old = (V(SU_RO_C) - V(SU_RO_M)) / dx;
        grad_m = grad_m + p.gamma_d * (grad_m - grad_m_old);
        const T rh_m = (V(SU_R2_M) + r2_c) * T(0.5);
        const T u_m = V(SU_RU_M) + dt_s * (V(SU_RRU_M) - rh_m * grad_m);
        T grad_p = (V(SU_RT_P) - rt_c) / dx;
        const T grad_p_old = (V(SU_RO_P) - V(SU_RO_C)) / dx;
        grad_p = grad_p + p.gamma_d * (grad_p - grad_p_old);
        const T rh_p = (r2_c + V(SU_R2_P)) * T(0.5);
        const T u_p = V(SU_RU_C) + dt_s * (V(SU_RRU_C) - rh_p * grad_p);
        a.ru_out[c] = u_p;
        a.mfx[c] = V(SU_MFX) + u_p / ns_T;
        T advection = -(u_p - u_m) / dx;
        T inc = dt_s * (V(SU_RRHO) + advection);
        const T rhop = V(SU_RHOP);
        const T rho_tp = (T)((double)rhop + fact_tp64 * (double)inc);
        a.rho_p[c] = rhop + inc;
        const T th_c = V(SU_TH_C);
        const T flux_ip = (V(SU_TH_P) + th_c) * T(0.5) * u_p;
        const T flux_im = (th_c + V(SU_TH_M)) * T(0.5) * u_m;
        advection = -(flux_ip - flux_im) / dx;
        inc = dt_s * (V(SU_RRT) + advection);
        const T rt_tp = (T)((double)rt_c + fact_tp64 * (double)inc);
        a.rt_out[c] = rt_c + inc;
        if (k >= 1) {
            const int j = k - 1;
            const size_t cj = c - P;
            const T buoyancy = (rt_tp - rt_tp_prev) / (ro(z + k) - ro(z + j));
            const T grav = -p.GRAV * T(0.5) * (rho_tp + rho_tp_prev);
            const T rt2pres_h = (pv_r2c + r2_c) * T(0.5);
            const T drho_w = dt_s * (pv_Rrw - rt2pres_h * buoyancy + grav);
            const T w_j = pv_rwp;
            const T aj = pv_ta;
            T d = w_j + drho_w;
            if (j > 0) d -= aj * fact * w_j;
            d -= pv_tb * fact * w_j;
            if (j < n - 1) d -= pv_tc * fact * rwp;
            TT dp;
            if (j == 0)
                dp = (TT)d / pv_piv;
            else
                dp = ((TT)d - (TT)aj * dprev) / pv_piv;
            a.dprime[cj] = dp;
            dprev = dp;
        }
        rho_tp_prev = rho_tp;
        rt_tp_prev = rt_tp;
        pv_r2c = r2_c;
        pv_Rrw = V(SU_RRW);
        pv_rwp = rwp;
        pv_ta = V(SU_TA);
        pv_tb = V(SU_TB);
        pv_tc = V(SU_TC);
        pv_piv = ps[(size_t)bb * nt + tid];
    }
    cp_async_wait<0>();
    // Back substitution going down fused with the vertical updates of cell k (moist.jl:
    // 968-970, 1412-1446, 1452-1458), as in b_substep_col: at level k the faces k (w_k, known
    // from level k + 1) and k - 1 (x_{k-1} = d'_{k-1} - c'_{k-1} x_k, computed here).
    const T* th = a.theta;
    // theta at k-2 .. k+2 and s.rho_w at k-1, k, kept in registers as k falls
    T t_m2 = ke >= 2 ? ro(th + MOIST_IDX(ke - 2, i)) : T(0);
    T t_m1 = ke >= 1 ? ro(th + MOIST_IDX(ke - 1, i)) : T(0);
    T t_0 = ro(th + MOIST_IDX(ke, i)), t_p1 = T(0), t_p2 = T(0);
    T sw_0 = ro(a.s_rw + MOIST_IDX(ke, i)), sw_m1 = ro(a.s_rw + MOIST_IDX(ke - 1, i));
    T v_rho = a.rho_p[MOIST_IDX(ke, i)], v_rt = a.rt_out[MOIST_IDX(ke, i)], v_mfz = a.mfz[MOIST_IDX(ke, i)];
    TT v_dp = dprev, v_cp = TT(0);  // d' and c' of face k - 1 (x_{ke-1} = d'_{ke-1} itself)
    TT x = TT(0);
    T w_k = T(0);
    for (int k = ke; k >= 0; k--) {
        // next level's inputs: cell k - 1 and face k - 2
        T n_rho = T(0), n_rt = T(0), n_mfz = T(0), n_t = T(0), n_sw = T(0);
        TT n_dp = TT(0), n_cp = TT(0);
        if (k >= 1) {
            const size_t cn = MOIST_IDX(k - 1, i);
            n_rho = a.rho_p[cn];
            n_rt = a.rt_out[cn];
            n_mfz = a.mfz[cn];
            if (k >= 3) n_t = ro(th + MOIST_IDX(k - 3, i));
            if (k >= 2) {
                n_sw = ro(a.s_rw + MOIST_IDX(k - 2, i));
                n_dp = a.dprime[MOIST_IDX(k - 2, i)];
                n_cp = ro(a.tcp + MOIST_IDX(k - 2, i));
            }
        }
        T w_km = T(0);
        if (k >= 1) {
            x = (k == ke) ? v_dp : v_dp - v_cp * x;
            w_km = (T)x;
            a.rw_p[MOIST_IDX(k - 1, i)] = w_km;
        }
        const size_t c = MOIST_IDX(k, i);
        {
            const T flux_kp = k == ke ? T(0.0) : w_k;
            const T flux_km = k == 0 ? T(0.0) : w_km;
            const T adv = -(flux_kp - flux_km) / ro(dz + k);
            a.rho_p[c] = v_rho + dt_s * adv;
        }
        T flux_kp, flux_km;
        if (k == ke) {
            flux_kp = T(0.0);
        } else {
            const T wp = w_k;
            if (wp > EPS && k > 0)
                flux_kp = up3(wp, t_m1, t_0, t_p1);
            else if (sw_0 < -EPS && k < ke - 1)  // selector on s.rho_w, as written (1426)
                flux_kp = up3(wp, t_p2, t_p1, t_0);
            else
                flux_kp = wp * f2h(t_0, t_p1, ro(dz + k), ro(dz + k + 1));
        }
        if (k == 0) {
            flux_km = T(0.0);
        } else {
            const T wp = w_km;
            const T sw = sw_m1;
            if (sw > EPS && k > 1)
                flux_km = up3(wp, t_m2, t_m1, t_0);
            else if (sw < -EPS && k < ke)
                flux_km = up3(wp, t_p1, t_0, t_m1);
            else
                flux_km = wp * f2h(t_m1, t_0, ro(dz + k - 1), ro(dz + k));
        }
        const T adv = -(flux_kp - flux_km) / ro(dz + k);
        a.rt_out[c] = v_rt + dt_s * adv;
        if (k < ke) a.mfz[c] = v_mfz + w_k / ns_T;
        // slide the windows down one level
        w_k = w_km;
        t_p2 = t_p1;
        t_p1 = t_0;
        t_0 = t_m1;
        t_m1 = t_m2;
        t_m2 = n_t;
        sw_0 = sw_m1;
        sw_m1 = n_sw;
        v_rho = n_rho;
        v_rt = n_rt;
        v_mfz = n_mfz;
        v_dp = n_dp;
        v_cp = n_cp;
    }
}


// ----------------------------------------------------------------------------- column strips
//
// Strip form of the per-stage factorisation and of the acoustic substep. A block of
// STRIP_THREADS threads owns wc adjacent columns (wc = 1, 2, 4 or 8) over all levels: the work
// that is independent per cell runs over all cells of the strip in parallel with coalesced
// loads, and only the Thomas recurrences run one thread per column, out of shared memory. The
// per-column bodies above put every load of a column on the recurrence's critical path, which
// a single domain's few columns cannot hide; here a substep costs about one recurrence of FP64
// latencies. Ensembles, whose many columns do hide it, use the per-column bodies (or these,
// as their autotuner finds). Each value goes through the same operations in both forms, so
// the results agree bit for bit.

constexpr int STRIP_THREADS = 256;

// shared memory of one strip block (bytes), laid out by StripSmem
template <class T, class TT>
__host__ __device__ inline size_t strip_smem_bytes(int nz, int wc) {
    const size_t n = (size_t)(nz - 1) * wc;
    return 5 * n * sizeof(TT) + (2 * n + 2 * (size_t)nz * wc + (size_t)nz * (wc + 1)) * sizeof(T);
}

// A loop whose iterations load from global memory and then compute, in batches: every thread
// loads the operands of SUB_BATCH iterations (load(e) returns them) before computing any
// (work(e, v)), so that it waits for one memory round trip per batch instead of one per
// iteration; a division in the computation ends the compiler's scheduling region, so it would
// not move the next iteration's loads above it.
constexpr int SUB_BATCH = 4;
template <class V, class L, class W>
__device__ __forceinline__ void batched_loop(int first, int end, int stride, L load, W work) {
    for (int b0 = first; b0 < end; b0 += SUB_BATCH * stride) {
        V v[SUB_BATCH];
#pragma unroll
        for (int u = 0; u < SUB_BATCH; u++) {
            const int e = b0 + u * stride;
            if (e < end) v[u] = load(e);
        }
#pragma unroll
        for (int u = 0; u < SUB_BATCH; u++) {
            const int e = b0 + u * stride;
            if (e < end) work(e, v[u]);
        }
    }
}
template <class T, int N>
struct Vals {
    T v[N];
};

template <class T, class TT>
struct StripSmem {
    TT *D, *Dp, *piv, *rp, *cp;  // [n][wc]: right-hand side, d', pivots, 1/pivots, modified super-diagonal
    T *a, *w;                    // [n][wc]: sub-diagonal, new rho_w_p
    T *rho_tp, *rt_tp;           // [nz][wc]: off-centred rho_p, rho_theta_p
    T* u;                        // [nz][wc+1]: rho_u_p at faces i0-1/2 .. i0+wc-1/2
    __device__ StripSmem(unsigned char* base, int nz, int wc) {
        const size_t n = (size_t)(nz - 1) * wc;
        D = (TT*)base;
        Dp = D + n;
        piv = Dp + n;
        rp = piv + n;
        cp = rp + n;
        a = (T*)(cp + n);
        w = a + n;
        rho_tp = w + n;
        rt_tp = rho_tp + (size_t)nz * wc;
        u = rt_tp + (size_t)nz * wc;
    }
};

// b_thomas_col over a strip: the coefficients of all rows in parallel, then the pivot
// recurrence per column
template <class T, class TT>
__device__ __forceinline__ void b_thomas_strip(DevParams<T> p, const T* theta, const T* rt2pres, T dt_s, int wc,
                                               T* ta, T* tb, T* tc, TT* tcp, TT* tpiv, const int* err, int bx,
                                               int by) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    if (halted(err)) return;
    const int nx = p.nx, nz = p.nz, P = p.P;
    const int i0 = bx * wc, ncol = min(wc, nx - i0);
    const int ke = nz - 1, n = nz - 1;
    const T* dz = p.dz;
    const T* z = p.z;
    StripSmem<T, TT> sm(smem_raw, nz, wc);
    T* th_h = sm.rho_tp;  // [n][wc] half-level theta, f2h of the two cells around face j+1/2
    const int col = threadIdx.x % wc, r0 = threadIdx.x / wc, rs = STRIP_THREADS / wc;
    const bool own = col < ncol;
    const int i = i0 + col;
    const T fact_tp = T(0.5) * (T(1.0) + p.beta);
    const T dt_tp2 = (dt_s * fact_tp) * (dt_s * fact_tp);
    batched_loop<Vals<T, 2>>(
        r0, own ? n : 0, rs, [&](int j) { return Vals<T, 2>{{theta[MOIST_IDX(j, i)], theta[MOIST_IDX(j + 1, i)]}}; },
        [&](int j, const Vals<T, 2>& v) { th_h[j * wc + col] = f2h(v.v[0], v.v[1], dz[j], dz[j + 1]); });
    __syncthreads();
    batched_loop<Vals<T, 2>>(
        r0, own ? n : 0, rs, [&](int j) { return Vals<T, 2>{{rt2pres[MOIST_IDX(j, i)], rt2pres[MOIST_IDX(j + 1, i)]}}; },
        [&](int j, const Vals<T, 2>& v) {
            const int k = j;
            const T th_cur = th_h[j * wc + col];
            const T th_prev = k > 0 ? th_h[(j - 1) * wc + col] : T(0);
            const T th_next = (k + 1 <= ke - 1) ? th_h[(j + 1) * wc + col] : T(0);
            const T r_k = v.v[0], r_kp = v.v[1];
            const T b = dt_tp2 * (r_k / dz[k] + r_kp / dz[k + 1]) * th_cur / (z[k + 1] - z[k]);
            const T a = (k > 0) ? -dt_tp2 * (r_k * th_prev / ((z[k + 1] - z[k]) * dz[k]) - p.GRAV / (dz[k] + dz[k + 1])) : T(0);
            const T c = (k < ke - 1) ? -dt_tp2 * (r_kp * th_next / ((z[k + 1] - z[k]) * dz[k + 1]) + p.GRAV / (dz[k] + dz[k + 1])) : T(0);
            ta[MOIST_IDX(j, i)] = a;
            tb[MOIST_IDX(j, i)] = b;
            tc[MOIST_IDX(j, i)] = c;
            sm.D[j * wc + col] = (TT)(b + T(1.0));
            sm.a[j * wc + col] = a;
            sm.cp[j * wc + col] = (TT)c;
        });
    __syncthreads();
    if (threadIdx.x < ncol) {
        // the pivot recurrence, the next level's operands read one level ahead (index clamped)
        const int cc = threadIdx.x;
        const TT* __restrict__ sD = sm.D;
        const T* __restrict__ sa = sm.a;
        TT* __restrict__ sc = sm.cp;
        TT* __restrict__ sp = sm.piv;
        TT cp_prev = TT(0);
        TT bn = sD[cc], an = (TT)sa[cc], cn = sc[cc];
#pragma unroll 4
        for (int j = 0; j < n; j++) {
            const TT bb = bn, aj = an, cj = cn;
            const int jn = j + 1 < n ? j + 1 : n - 1;
            bn = sD[jn * wc + cc];
            an = (TT)sa[jn * wc + cc];
            cn = sc[jn * wc + cc];
            const TT piv = j == 0 ? bb : bb - aj * cp_prev;
            const TT cpj = cj / piv;
            sp[j * wc + cc] = piv;
            sc[j * wc + cc] = cpj;
            cp_prev = cpj;
        }
    }
    __syncthreads();
    #pragma unroll 4
    for (int j = r0; j < n && own; j += rs) {
        tcp[MOIST_IDX(j, i)] = sm.cp[j * wc + col];
        tpiv[MOIST_IDX(j, i)] = sm.piv[j * wc + col];
    }
}
template <class T, class TT>
__global__ void __launch_bounds__(STRIP_THREADS) k_thomas_strip(DevParams<T> p, const T* theta, const T* rt2pres,                                                                  T dt_s, int wc, T* ta, T* tb, T* tc, TT* tcp,                                                                  TT* tpiv, const int* err) {
    b_thomas_strip(p, theta, rt2pres, dt_s, wc, ta, tb, tc, tcp, tpiv, err, blockIdx.x, blockIdx.y);
}

// b_substep_col over a strip (moist.jl:1355-1459)
template <class T, class TT>
__device__ __forceinline__ void b_substep_strip(DevParams<T> p, SubArgs<T, TT> a, T dt_s, T ns_T, double fact_tp64,
                                                int wc, const int* err, int bx, int by) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    if (halted(err)) return;
    const int nx = p.nx, nz = p.nz, P = p.P;
    const int i0 = bx * wc, ncol = min(wc, nx - i0);
    const int ke = nz - 1, n = nz - 1;
    const T dx = p.dx, EPS = p.EPS;
    const T* dz = p.dz;
    const T* z = p.z;
    StripSmem<T, TT> sm(smem_raw, nz, wc);
    const int tid = threadIdx.x;
    const T fact_tpT = T(0.5) * (T(1.0) + p.beta);
    const T fact_tmT = T(0.5) * (T(1.0) - p.beta);
    const T fact = fact_tmT / fact_tpT;
    // (1) horizontal forward step of rho_u_p at the ncol + 1 faces (1355-1366)
    {
        const int nf = ncol + 1, wf = wc + 1;
        batched_loop<Vals<T, 8>>(
            tid, nz * nf, STRIP_THREADS,
            [&](int e) {
                const int k = e / nf, f = e - k * nf;
                const int cc = wrapx(i0 + f - 1, nx), cn = wrapx(cc + 1, nx);
                const size_t a0 = MOIST_IDX(k, cc), a1 = MOIST_IDX(k, cn);
                return Vals<T, 8>{{ro(a.rt_in + a0), ro(a.rt_in + a1), ro(a.rt_old + a0), ro(a.rt_old + a1),
                                   ro(a.rt2pres + a0), ro(a.rt2pres + a1), ro(a.ru_in + a0), ro(a.R_ru + a0)}};
            },
            [&](int e, const Vals<T, 8>& v) {
                const int k = e / nf, f = e - k * nf;
                T grad_x = (v.v[1] - v.v[0]) / dx;
                const T grad_x_old = (v.v[3] - v.v[2]) / dx;
                grad_x = grad_x + p.gamma_d * (grad_x - grad_x_old);
                const T rt2pres_h = (v.v[4] + v.v[5]) * T(0.5);
                sm.u[k * wf + f] = v.v[6] + dt_s * (v.v[7] - rt2pres_h * grad_x);
            });
    }
    __syncthreads();
    const int col = tid % wc, r0 = tid / wc, rs = STRIP_THREADS / wc;
    const bool own = col < ncol;
    const int i = i0 + col;
    const int im = wrapx(i - 1, nx), ip = wrapx(i + 1, nx);
    // (2) explicit rho_p, rho_theta_p and their off-centred values (1367-1396)
    batched_loop<Vals<T, 8>>(
        r0, own ? nz : 0, rs,
        [&](int k) {
            const size_t c = MOIST_IDX(k, i);
            return Vals<T, 8>{{a.mfx[c], ro(a.R_rho + c), a.rho_p[c], ro(a.theta + c), ro(a.theta + MOIST_IDX(k, ip)),
                               ro(a.theta + MOIST_IDX(k, im)), ro(a.R_rt + c), ro(a.rt_in + c)}};
        },
        [&](int k, const Vals<T, 8>& v) {
            const size_t c = MOIST_IDX(k, i);
            const T u_m = sm.u[k * (wc + 1) + col], u_p = sm.u[k * (wc + 1) + col + 1];
            a.ru_out[c] = u_p;
            a.mfx[c] = v.v[0] + u_p / ns_T;
            T advection = -(u_p - u_m) / dx;
            T inc = dt_s * (v.v[1] + advection);
            const T rho_old = v.v[2];
            sm.rho_tp[k * wc + col] = (T)((double)rho_old + fact_tp64 * (double)inc);
            a.rho_p[c] = rho_old + inc;
            const T th_i = v.v[3], th_ip = v.v[4], th_im = v.v[5];
            const T flux_ip = (th_ip + th_i) * T(0.5) * u_p;
            const T flux_im = (th_i + th_im) * T(0.5) * u_m;
            advection = -(flux_ip - flux_im) / dx;
            inc = dt_s * (v.v[6] + advection);
            const T rtp = v.v[7];
            sm.rt_tp[k * wc + col] = (T)((double)rtp + fact_tp64 * (double)inc);
            a.rt_out[c] = rtp + inc;
        });
    __syncthreads();
    // (3) right-hand side of the w-p system (1397-1408) and the stage factors
    struct RhsIn {
        T r2j, r2k, rrw, wj, wk, ta, tb, tc;
        TT piv, cp;
    };
    batched_loop<RhsIn>(
        r0, own ? n : 0, rs,
        [&](int j) {
            const size_t c = MOIST_IDX(j + 1, i), cj = c - P;
            return RhsIn{ro(a.rt2pres + cj), ro(a.rt2pres + c), ro(a.R_rw + cj), a.rw_p[cj], a.rw_p[c],
                         ro(a.ta + cj),      ro(a.tb + cj),      ro(a.tc + cj),   ro(a.tpiv + cj), ro(a.tcp + cj)};
        },
        [&](int j, const RhsIn& v) {
            const int k = j + 1;
            const T buoyancy = (sm.rt_tp[k * wc + col] - sm.rt_tp[j * wc + col]) / (z[k] - z[j]);
            const T grav = -p.GRAV * T(0.5) * (sm.rho_tp[k * wc + col] + sm.rho_tp[j * wc + col]);
            const T rt2pres_h = (v.r2j + v.r2k) * T(0.5);
            const T drho_w = dt_s * (v.rrw - rt2pres_h * buoyancy + grav);
            const T w_j = v.wj;
            const T aj = v.ta;
            T d = w_j + drho_w;
            if (j > 0) d -= aj * fact * w_j;
            d -= v.tb * fact * w_j;
            if (j < n - 1) d -= v.tc * fact * v.wk;
            sm.D[j * wc + col] = (TT)d;
            sm.a[j * wc + col] = aj;
            sm.piv[j * wc + col] = v.piv;
            if constexpr (sizeof(TT) == 8) sm.rp[j * wc + col] = (TT)1 / v.piv;  // for the checked quotients of (4)
            sm.cp[j * wc + col] = v.cp;
        });
    __syncthreads();
    // (4) Thomas elimination per column (moist.jl:956-970). The loops read the next level's
    // operands one level ahead (clamped at the ends), unrolled so that the loads leave the
    // dependent path.
    if (tid < ncol) {
        const int cc = tid;
        const TT* __restrict__ sD = sm.D;
        const T* __restrict__ sa = sm.a;
        const TT* __restrict__ sp = sm.piv;
        TT* __restrict__ sDp = sm.Dp;
        TT dprev = (TT)0;
        bool ok = sizeof(TT) == 8;
        if constexpr (sizeof(TT) == 8) {
            // d'_j = (d_j - a_j d'_{j-1}) / piv_j with each quotient formed from 1/piv_j (divided in
            // (3) by all threads) and checked exact (qdiv_checked, fastdiv.cuh): 68 instead of 171
            // cycles per level. A column with any unproven quotient is eliminated again with IEEE
            // division below (the right-hand sides stay in D).
            const TT* __restrict__ sr = sm.rp;
            dprev = qdiv_checked(sD[cc], sp[cc], sr[cc], ok);
            sDp[cc] = dprev;
            const int j1 = n > 1 ? 1 : 0;
            TT dn = sD[j1 * wc + cc], an = (TT)sa[j1 * wc + cc], pn = sp[j1 * wc + cc], yn = sr[j1 * wc + cc];
#pragma unroll 4
            for (int j = 1; j < n; j++) {
                const TT dj = dn, aj = an, pj = pn, yj = yn;
                const int jn = j + 1 < n ? j + 1 : n - 1;
                dn = sD[jn * wc + cc];
                an = (TT)sa[jn * wc + cc];
                pn = sp[jn * wc + cc];
                yn = sr[jn * wc + cc];
                dprev = qdiv_checked(dj - aj * dprev, pj, yj, ok);
                sDp[j * wc + cc] = dprev;
            }
        }
        if (!ok) {
            dprev = sD[cc] / sp[cc];
            sDp[cc] = dprev;
            for (int j = 1; j < n; j++) {
                const TT dp = (sD[j * wc + cc] - (TT)sa[j * wc + cc] * dprev) / sp[j * wc + cc];
                sDp[j * wc + cc] = dp;
                dprev = dp;
            }
        }
        // back substitution x_j = d'_j - c'_j x_{j+1}: 43 instead of 64 cycles per level
        const TT* __restrict__ sc = sm.cp;
        T* __restrict__ sw = sm.w;
        TT x = dprev;
        sw[(n - 1) * wc + cc] = (T)x;
        const int jb = n >= 2 ? n - 2 : 0;
        TT dpn = sDp[jb * wc + cc], cpn = sc[jb * wc + cc];
#pragma unroll 4
        for (int j = n - 2; j >= 0; j--) {
            const TT dpj = dpn, cpj = cpn;
            const int jn = j >= 1 ? j - 1 : 0;
            dpn = sDp[jn * wc + cc];
            cpn = sc[jn * wc + cc];
            x = dpj - cpj * x;
            sw[j * wc + cc] = (T)x;
        }
    }
    __syncthreads();
    // (5) vertical rho_p, rho_theta_p updates (1412-1446), momentum flux averages (1452-1458)
    // every value a branch may read is loaded, in bounds, before the branches select
    const T* th = a.theta;
    batched_loop<Vals<T, 10>>(
        r0, own ? nz : 0, rs,
        [&](int k) {
            const size_t c = MOIST_IDX(k, i);
            return Vals<T, 10>{{a.rho_p[c], a.rt_out[c], k < ke ? a.mfz[c] : T(0), ro(a.s_rw + c),
                                k > 0 ? ro(a.s_rw + c - P) : T(0), k >= 2 ? ro(th + c - 2 * P) : T(0),
                                k >= 1 ? ro(th + c - P) : T(0), ro(th + c), k + 1 <= ke ? ro(th + c + P) : T(0),
                                k + 2 <= ke ? ro(th + c + 2 * P) : T(0)}};
        },
        [&](int k, const Vals<T, 10>& v) {
            const size_t c = MOIST_IDX(k, i);
            const T th_m2 = v.v[5], th_m1 = v.v[6], th_0 = v.v[7], th_p1 = v.v[8], th_p2 = v.v[9];
            const T w_k = k < ke ? sm.w[k * wc + col] : T(0.0);
            const T w_km = k > 0 ? sm.w[(k - 1) * wc + col] : T(0.0);
            if (k < ke) a.rw_p[c] = w_k;
            {
                const T flux_kp = k == ke ? T(0.0) : w_k;
                const T flux_km = k == 0 ? T(0.0) : w_km;
                const T advection = -(flux_kp - flux_km) / dz[k];
                a.rho_p[c] = v.v[0] + dt_s * advection;
            }
            T flux_kp, flux_km;
            if (k == ke) {
                flux_kp = T(0.0);
            } else {
                const T wp = w_k;
                if (wp > EPS && k > 0)
                    flux_kp = up3(wp, th_m1, th_0, th_p1);
                else if (v.v[3] < -EPS && k < ke - 1)  // selector on s.rho_w, as written (1426)
                    flux_kp = up3(wp, th_p2, th_p1, th_0);
                else
                    flux_kp = wp * f2h(th_0, th_p1, dz[k], dz[k + 1]);
            }
            if (k == 0) {
                flux_km = T(0.0);
            } else {
                const T wp = w_km;
                const T sw = v.v[4];
                if (sw > EPS && k > 1)
                    flux_km = up3(wp, th_m2, th_m1, th_0);
                else if (sw < -EPS && k < ke)
                    flux_km = up3(wp, th_p1, th_0, th_m1);
                else
                    flux_km = wp * f2h(th_m1, th_0, dz[k - 1], dz[k]);
            }
            const T advection = -(flux_kp - flux_km) / dz[k];
            a.rt_out[c] = v.v[1] + dt_s * advection;
            if (k < ke) a.mfz[c] = v.v[2] + w_k / ns_T;
        });
}
template <class T, class TT>
__global__ void __launch_bounds__(STRIP_THREADS) k_substep_strip(DevParams<T> p, SubArgs<T, TT> a, T dt_s, T ns_T,                                                                   double fact_tp64, int wc, const int* err) {
    b_substep_strip(p, a, dt_s, ns_T, fact_tp64, wc, err, blockIdx.x, blockIdx.y);
}

// ----------------------------------------------------------------------------- tracers

template <class T>
struct TracerArgs {
    const T* q_old[3];   // rho_qv, rho_qc, rho_qr at the start of the sweep
    T* q_new[3];         // results
    const T* q0[3];      // s0 tracers
    const T* dphys[3];   // d_rho_q*_phys
    const T *rho, *mfx, *mfz;
    T dt;                // stage dt
};

// The tracer update of one cell (moist.jl:1479-1515), given the scalar values s = rho_q/rho it
// reads: "new" values at (k, i-1), (k, i-2), (k-1, i), (k-2, i) and stage-start values elsewhere.
template <class T>
__device__ __forceinline__ T tracer_cell(const DevParams<T>& p, const TracerArgs<T>& a, int t, int k, int i,
                                         T s_c, T s_ip1, T s_ip2, T s_kp1, T s_kp2, T s_im1, T s_im2,
                                         T s_km1, T s_km2, T lin_km1, T lin_k, T lin_kp1) {
    const int nx = p.nx, nz = p.nz, P = p.P;
    const int ke = nz - 1;
    const T EPS = p.EPS, dx = p.dx;
    const T* dz = p.dz;
    const T* z = p.z;
    const size_t c = MOIST_IDX(k, i);
    const int im = wrapx(i - 1, nx), ip = wrapx(i + 1, nx);
    const T fx_ip = limited_flux_x(a.mfx[c], s_im1, s_c, s_ip1, s_ip2, EPS);
    const T fx_im = limited_flux_x(a.mfx[MOIST_IDX(k, im)], s_im2, s_im1, s_c, s_ip1, EPS);
    const T adv_x = (fx_ip - fx_im) / dx;
    const T fz_kp = k == ke ? T(0.0)
                            : limited_flux_z(a.mfz[c], s_km1, s_c, s_kp1, s_kp2, k, nz, dz[k], dz[k + 1], lin_k,
                                             lin_kp1, p.dt, EPS);
    const T fz_km = k == 0 ? T(0.0)
                           : limited_flux_z(a.mfz[c - P], s_km2, s_km1, s_c, s_kp1, k - 1, nz, dz[k - 1], dz[k],
                                            lin_km1, lin_k, p.dt, EPS);
    const T adv_z = (fz_kp - fz_km) / dz[k];
    const T advection = -(adv_x + adv_z);
    const T* rho = a.rho;
    const T r_c = rho[c];
    const T scalar_kp = k == ke ? T(0.0) : s_kp1;
    const T scalar_km = k == 0 ? T(0.0) : s_km1;
    const T dsdx_ip = (rho[MOIST_IDX(k, ip)] + r_c) * T(0.5) * (s_ip1 - s_c) / dx;
    const T dsdx_im = (r_c + rho[MOIST_IDX(k, im)]) * T(0.5) * (s_c - s_im1) / dx;
    const T diff_x = p.kappa * (dsdx_ip - dsdx_im) / dx;
    const T dsdz_kp = k == ke ? T(0.0) : f2h(rho[c + P], r_c, dz[k + 1], dz[k]) * (scalar_kp - s_c) / (z[k + 1] - z[k]);
    const T dsdz_km = k == 0 ? T(0.0) : f2h(r_c, rho[c - P], dz[k], dz[k - 1]) * (s_c - scalar_km) / (z[k] - z[k - 1]);
    const T diff_z = p.kappa * (dsdz_kp - dsdz_km) / dz[k];
    const T diffusion = diff_x + diff_z;
    return a.q0[t][c] + a.dt * (advection + diffusion + a.dphys[t][c]);
}

// Exact lexicographic Gauss-Seidel sweep (moist.jl:1469-1518: i outer, k inner, in place),
// one block per tracer, thread k owns row k and processes column i = t - k at wavefront step t.
// Cell (k, i) depends on updated (k, i-1), (k, i-2), (k-1, i), (k-2, i), which are final by step
// t - 1 / t - 2; a 3-slot ring in shared memory carries the row neighbours' new values.
template <class T>
__global__ void k_tracer_wavefront(DevParams<T> p, TracerArgs<T> a, const int* err) {
    extern __shared__ unsigned char smem_raw[];
    T* ring = reinterpret_cast<T*>(smem_raw);  // [3][nz]
    const int t = blockIdx.x;
    const int k = threadIdx.x;
    const int nx = p.nx, nz = p.nz, P = p.P;
    if (halted(err)) return;
    const T* qo = a.q_old[t];
    const T* rho = a.rho;
    auto s_old = [&](int kk, int ii) { const size_t cc = MOIST_IDX(kk, ii); return qo[cc] / rho[cc]; };
    // halo column read by the linear-index clamp: reference column 1 = interior column nx-2
    const int hcol = nx - 2;
    const bool active = k < nz;
    // values at (k, i-1), (k, i-2) for i = 0 are the halo columns' stage-start copies
    T prev1 = active ? s_old(k, nx - 1) : T(0);
    T prev2 = active ? s_old(k, nx - 2) : T(0);
    const int nsteps = nx + nz - 1;
    for (int step = 0; step < nsteps; step++) {
        const int i = step - k;
        if (active && i >= 0 && i < nx) {
            const int ip = wrapx(i + 1, nx), ip2 = wrapx(i + 2, nx);
            const T s_c = s_old(k, i);
            const T s_ip1 = s_old(k, ip);
            const T s_ip2 = s_old(k, ip2);
            const T s_kp1 = (k + 1 < nz) ? s_old(k + 1, i) : T(0);
            const T s_kp2 = (k + 2 < nz) ? s_old(k + 2, i) : T(0);
            const T s_km1 = (k >= 1) ? ring[((step - 1) % 3) * nz + (k - 1)] : T(0);
            const T s_km2 = (k >= 2) ? ring[((step - 2) % 3) * nz + (k - 2)] : T(0);
            const T lin_km1 = (k >= 1) ? qo[MOIST_IDX(k - 1, hcol)] : T(0);
            const T lin_k = qo[MOIST_IDX(k, hcol)];
            const T lin_kp1 = (k + 1 < nz) ? qo[MOIST_IDX(k + 1, hcol)] : T(0);
            const T qn = tracer_cell(p, a, t, k, i, s_c, s_ip1, s_ip2, s_kp1, s_kp2, prev1, prev2, s_km1, s_km2,
                                     lin_km1, lin_k, lin_kp1);
            const size_t c = MOIST_IDX(k, i);
            a.q_new[t][c] = qn;
            const T sn = qn / rho[c];
            ring[(step % 3) * nz + k] = sn;
            prev2 = prev1;
            prev1 = sn;
        }
        __syncthreads();
    }
}

// ----------------------------------------------------------------------------- state hash

// order-independent hash of the bit patterns of a field: out += sum_j bits(f[j]) * (2 j + 1)
// (mod 2^64), for checking that two runs produced the same State
template <class T>
__global__ void k_hash(const T* __restrict__ f, size_t n, unsigned long long* out) {
    unsigned long long h = 0;
    for (size_t j = (size_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (size_t)gridDim.x * blockDim.x) {
        const unsigned long long b = sizeof(T) == 4 ? (unsigned long long)__float_as_uint((float)f[j])
                                                    : (unsigned long long)__double_as_longlong((double)f[j]);
        h += b * (2ull * j + 1ull);
    }
    for (int o = 16; o > 0; o >>= 1) h += __shfl_xor_sync(0xffffffffu, h, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(out, h);
}

// ----------------------------------------------------------------------------- history output

constexpr int HIST_THREADS = 256;

// output_history's primitive variables (moist.jl:1795-1835), one thread per cell: out[f] holds
// field f (u, w, theta, qv, qc, qr, pres, temp, theta_e, RH) as an (nz, nx) array with z fastest
// (the history file's layout); part[block][6] = min w, max w, max qc, max qr, min RH, max RH of
// the block's cells.
template <class T>
__global__ void __launch_bounds__(HIST_THREADS) k_history_diag(DevParams<T> p, StateP<T> s, T* out, double* part) {
    const int nx = p.nx, nz = p.nz, P = p.P;
    const size_t ncell = (size_t)nx * nz;
    const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    double v6[6] = {1e300, -1e300, -1e300, -1e300, 1e300, -1e300};
    if (idx < ncell) {
        const int k = (int)(idx / nx), i = (int)(idx - (size_t)k * nx);
        const size_t c = MOIST_IDX(k, i);
        const T rho = s.rho[c], rt = s.rt[c];
        const T rho_inv = T(1.0) / rho;
        const T theta = rt * rho_inv;
        const T qv = s.qv[c] * rho_inv, qc = s.qc[c] * rho_inv, qr = s.qr[c] * rho_inv;
        const T u = (s.ru[c] + s.ru[MOIST_IDX(k, wrapx(i - 1, nx))]) * T(0.5) * rho_inv;
        const T w = k > 0 ? (s.rw[c] + s.rw[c - P]) * T(0.5) * rho_inv : s.rw[c] * T(0.5) * rho_inv;
        const T qt = qv + qc + qr;
        const T qd = T(1.0) - qt;
        const T r = p.Rd * qd + p.Rv * qv;
        T cp = p.Cpd * qd + p.Cpv * qv + p.Cpl * (qc + qr);
        const T cv = cp - r;
        const T pi = mm::mpow(r * rt / p.P0, r / cv);
        const T pres = p.P0 * mm::mpow(pi, cp / r);
        const T temp = theta * pi;
        T es, d1, qsat, d2;
        sat_vp(temp, p, es, d1);
        sat_q(pres, es, p, qsat, d2);
        const T RH = qsat > T(1e-10) ? qv / qsat * T(100.0) : T(0.0);
        const T presv = rho * qv * p.Rv * temp;  // partial pressure of vapour
        const T presd = pres - presv;
        cp = p.Cpd * qd + p.Cpl * qt;
        const T thetae = temp * mm::mpow(presd / p.P0, -p.Rd / cp) * mm::mexp(p.Lv * qv / (cp * temp));
        const T v[10] = {u, w, theta, qv, qc, qr, pres, temp, thetae, RH};
        const size_t o = (size_t)k + (size_t)nz * i;
        for (int f = 0; f < 10; f++) out[(size_t)f * ncell + o] = v[f];
        v6[0] = w;
        v6[1] = w;
        v6[2] = qc;
        v6[3] = qr;
        v6[4] = RH;
        v6[5] = RH;
    }
    __shared__ double red[6][HIST_THREADS / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int j = 0; j < 6; j++) {
        double x = v6[j];
        const bool mn = j == 0 || j == 4;
        for (int o = 16; o > 0; o >>= 1) {
            const double y = __shfl_xor_sync(0xffffffffu, x, o);
            x = mn ? fmin(x, y) : fmax(x, y);
        }
        if (lane == 0) red[j][wid] = x;
    }
    __syncthreads();
    if (threadIdx.x < 6) {
        const int j = threadIdx.x;
        const bool mn = j == 0 || j == 4;
        double x = red[j][0];
        for (int q = 1; q < HIST_THREADS / 32; q++) x = mn ? fmin(x, red[j][q]) : fmax(x, red[j][q]);
        part[(size_t)blockIdx.x * 6 + j] = x;
    }
}

// ----------------------------------------------------------------------------- stage epilogue

template <class T>
struct UpdArgs {
    StateP<T> s_in, s_out;  // s_out.X = s_in.X + X_p; s_out.q* are the sweep results
    const T *rho_p, *ru_p, *rw_p, *rt_p;
    PhysP<T> ph;
};

// state update (moist.jl:1522-1539) and NaN checks (1542-1578)
template <class T>
__device__ __forceinline__ void b_update(DevParams<T> p, UpdArgs<T> a, int* err, int bx, int by) {
    const int i = bx * blockDim.x + threadIdx.x;
    const int k = by * blockDim.y + threadIdx.y;
    const int nx = p.nx, nz = p.nz, P = p.P;
    if (i >= nx || k >= nz || halted(err)) return;
    const size_t c = MOIST_IDX(k, i);
    const T rho = a.s_in.rho[c] + a.rho_p[c];
    const T ru = a.s_in.ru[c] + a.ru_p[c];
    const T rt = a.s_in.rt[c] + a.rt_p[c];
    a.s_out.rho[c] = rho;
    a.s_out.ru[c] = ru;
    a.s_out.rt[c] = rt;
    T rw = a.s_in.rw[c];
    if (k < nz - 1) rw = rw + a.rw_p[c];
    a.s_out.rw[c] = rw;
    int bad = INT_MAX;
    const T v[12] = {rho, ru, rw, rt, a.s_out.qv[c], a.s_out.qc[c], a.s_out.qr[c], a.ph.d_u[c], a.ph.d_th[c],
                     a.ph.d_qv[c], a.ph.d_qc[c], a.ph.d_qr[c]};
#pragma unroll
    for (int f = 11; f >= 0; f--)
        if (v[f] != v[f]) bad = f;
    if (bad != INT_MAX) atomicMin(err + 1, bad);  // err[1]: pending, promoted at stage end
}
template <class T>
__global__ void k_update(DevParams<T> p, UpdArgs<T> a, int* err) {
    b_update(p, a, err, blockIdx.x, blockIdx.y);
}

// promote the stage's NaN report (err[1]) to the halt word (err[0])
__global__ void k_stage_end(int* err) {
    if (err[1] != INT_MAX && err[0] == INT_MAX) err[0] = err[1];
}

template <class T>
__device__ __forceinline__ void b_prec(DevParams<T> p, T* prec, const T* d_prec, const int* err, int bx, int by) {
    const int i = bx * blockDim.x + threadIdx.x;
    if (i >= p.nx || halted(err)) return;
    prec[i] = prec[i] + d_prec[i] * p.dt;
}
template <class T>
__global__ void k_prec(DevParams<T> p, T* prec, const T* d_prec, const int* err) {
    b_prec(p, prec, d_prec, err, blockIdx.x, blockIdx.y);
}

// ----------------------------------------------------------------------------- budgets
//
// Domain budgets as compensated FP64 sums (Neumaier's variant of Kahan summation; the library
// is built with --fmad=false, so the error terms are formed exactly). Per cell: mass rho dz dx,
// water (rho_qv + rho_qc + rho_qr) dz dx, and total energy (kinetic + potential + internal,
// each formed in the state precision exactly as output_history forms eng_k, eng_p, eng_i,
// moist.jl:1797-1841) times dz dx; per column: accumulated rain prec dx. A fixed grid of
// BUDGET_BLOCKS blocks, a fixed per-thread order, a fixed tree inside each block and a final
// sequential merge make the result reproducible bit for bit.

constexpr int BUDGET_BLOCKS = 256, BUDGET_THREADS = 256;

struct CSum {
    double s, c;  // running sum and the accumulated rounding errors
};
__device__ __forceinline__ void cs_add(CSum& a, double x) {
    const double t = a.s + x;
    a.c += fabs(a.s) >= fabs(x) ? (a.s - t) + x : (x - t) + a.s;
    a.s = t;
}
__device__ __forceinline__ void cs_merge(CSum& a, const CSum& b) {
    cs_add(a, b.s);
    a.c += b.c;
}

// energy density of one cell in the state precision (moist.jl:1799-1841)
template <class T>
__device__ __forceinline__ T cell_energy(const DevParams<T>& p, const StateP<T>& s, int k, int i) {
    const int nx = p.nx, P = p.P;
    const size_t c = MOIST_IDX(k, i);
    const T rho = s.rho[c];
    const T rho_inv = T(1.0) / rho;
    const T theta = s.rt[c] * rho_inv;
    const T qv = s.qv[c] * rho_inv, qc = s.qc[c] * rho_inv, qr = s.qr[c] * rho_inv;
    const T qt = qv + qc + qr;
    const T qd = T(1.0) - qt;
    const T r = p.Rd * qd + p.Rv * qv;
    const T cp = p.Cpd * qd + p.Cpv * qv + p.Cpl * (qc + qr);
    const T cv = cp - r;
    const T pi = mm::mpow(r * s.rt[c] / p.P0, r / cv);
    const T temp = theta * pi;
    const T u = (s.ru[c] + s.ru[MOIST_IDX(k, wrapx(i - 1, nx))]) * T(0.5) * rho_inv;
    const T w = k > 0 ? (s.rw[c] + s.rw[c - P]) * T(0.5) * rho_inv : s.rw[c] * T(0.5) * rho_inv;
    const T eng_k = T(0.5) * rho * (u * u + w * w);
    const T eng_p = rho * p.GRAV * p.z[k];
    const T eng_i = rho * (cv * temp + qv * p.Lv);
    return eng_k + eng_p + eng_i;
}

// the four sums of one block; out[blockIdx.x][4] pairs
template <class T>
__global__ void __launch_bounds__(BUDGET_THREADS) k_budget(DevParams<T> p, StateP<T> s, const T* prec, CSum* out) {
    const int nx = p.nx, nz = p.nz, P = p.P;
    CSum acc[4] = {{0, 0}, {0, 0}, {0, 0}, {0, 0}};
    const double dx = (double)p.dx;
    const long long n = (long long)nx * nz;
    for (long long e = blockIdx.x * (long long)BUDGET_THREADS + threadIdx.x; e < n;
         e += (long long)BUDGET_BLOCKS * BUDGET_THREADS) {
        const int k = (int)(e / nx), i = (int)(e - (long long)k * nx);
        const size_t c = MOIST_IDX(k, i);
        const double vol = (double)p.dz[k] * dx;
        cs_add(acc[0], (double)s.rho[c] * vol);
        cs_add(acc[1], ((double)s.qv[c] + (double)s.qc[c] + (double)s.qr[c]) * vol);
        const T e_kpi = cell_energy(p, s, k, i);
        cs_add(acc[2], (double)e_kpi * vol);
    }
    for (int i = blockIdx.x * BUDGET_THREADS + threadIdx.x; i < nx; i += BUDGET_BLOCKS * BUDGET_THREADS)
        cs_add(acc[3], (double)prec[i] * dx);
    __shared__ CSum part[4][BUDGET_THREADS];
    for (int q = 0; q < 4; q++) part[q][threadIdx.x] = acc[q];
    __syncthreads();
    for (int h = BUDGET_THREADS / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h)
            for (int q = 0; q < 4; q++) cs_merge(part[q][threadIdx.x], part[q][threadIdx.x + h]);
        __syncthreads();
    }
    if (threadIdx.x < 4) out[blockIdx.x * 4 + threadIdx.x] = part[threadIdx.x][0];
}

// sequential merge of the block sums: res = {mass, water + rain, energy, rain}
__global__ void k_budget_final(const CSum* part, double* res) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    CSum tot[4] = {{0, 0}, {0, 0}, {0, 0}, {0, 0}};
    for (int b = 0; b < BUDGET_BLOCKS; b++)
        for (int q = 0; q < 4; q++) cs_merge(tot[q], part[b * 4 + q]);
    cs_merge(tot[1], tot[3]);
    for (int q = 0; q < 4; q++) res[q] = tot[q].s + tot[q].c;
}

// ----------------------------------------------------------------------------- layout moves

// (ka, ia) column-major host layout <-> [nz][P] interior device layout, through a 32x32 tile
template <class T>
__device__ __forceinline__ void b_from_ref(int nx, int nz, int halo, int P, const T* __restrict__ src,
                                           T* __restrict__ dst, int bx, int by) {
    __shared__ T tile[32][33];
    const int k0 = bx * 32, i0 = by * 32;
    const int ka = nz;
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int i = i0 + r, k = k0 + threadIdx.x;
        if (i < nx && k < nz) tile[r][threadIdx.x] = src[(size_t)(i + halo) * ka + k];
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int k = k0 + r, i = i0 + threadIdx.x;
        if (i < nx && k < nz) dst[(size_t)k * P + i] = tile[threadIdx.x][r];
    }
}
template <class T>
__global__ void k_from_ref(int nx, int nz, int halo, int P, const T* __restrict__ src, T* __restrict__ dst) {
    b_from_ref(nx, nz, halo, P, src, dst, blockIdx.x, blockIdx.y);
}

template <class T>
__device__ __forceinline__ void b_to_ref(int nx, int nz, int halo, int P, const T* __restrict__ src,
                                         T* __restrict__ dst, int bx, int by) {
    __shared__ T tile[32][33];
    const int k0 = bx * 32;
    const int ia = nx + 2 * halo;
    const int j0 = by * 32;  // reference column index
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int k = k0 + r, j = j0 + threadIdx.x;
        if (j < ia && k < nz) {
            int i = j - halo;
            i = ((i % nx) + nx) % nx;  // halo columns as periodic copies
            tile[r][threadIdx.x] = src[(size_t)k * P + i];
        }
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int j = j0 + r, k = k0 + threadIdx.x;
        if (j < ia && k < nz) dst[(size_t)j * nz + k] = tile[threadIdx.x][r];
    }
}
template <class T>
__global__ void k_to_ref(int nx, int nz, int halo, int P, const T* __restrict__ src, T* __restrict__ dst) {
    b_to_ref(nx, nz, halo, P, src, dst, blockIdx.x, blockIdx.y);
}

// Up to 7 fields moved in one launch (blockIdx.z = field): the State's layout moves when the
// host arrays are page-locked and mapped, so that the kernel reads or writes them over the bus
// directly, every field's transfer in flight at once, without a staging copy.
template <class T>
struct FieldSet {
    const T* src[7];
    T* dst[7];
};
template <class T>
__global__ void k_from_ref_n(int nx, int nz, int halo, int P, FieldSet<T> f) {
    b_from_ref(nx, nz, halo, P, f.src[blockIdx.z], f.dst[blockIdx.z], blockIdx.x, blockIdx.y);
}
template <class T>
__global__ void k_to_ref_n(int nx, int nz, int halo, int P, FieldSet<T> f) {
    b_to_ref(nx, nz, halo, P, f.src[blockIdx.z], f.dst[blockIdx.z], blockIdx.x, blockIdx.y);
}

}  // namespace moist
