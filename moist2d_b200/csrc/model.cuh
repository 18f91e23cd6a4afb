// model.cuh - device-side building blocks of the large step (sm_100a).
//
// Device layout: every 2-D field is a row-major [nz][P] array (row k, column i, x contiguous),
// interior columns only (i = 0 .. nx-1 is reference column is + i), P = pitch >= nx. The
// reference's periodic halo columns are not stored; a read at i-1, i-2, i+1, i+2 wraps around,
// which is what the reference reads after its exchange_halo! calls (moist.jl:233-241).
//
// Every expression below keeps the reference's operation order (moist.jl line numbers in the
// comments), and the library is compiled with --fmad=false, so results match a CPU evaluation
// of the same expressions without contraction bit for bit.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "moist_math.h"
#include "dual.cuh"  // the templates below also instantiate over dual numbers (adjoint.cuh)

namespace moist {

using mm::jmax;
using mm::jmin;

template <class T>
struct DevParams {
    int nx, nz, P;
    T dx, dt, H, nu, kappa, gamma_d, beta, zf_sponge;
    T EPS, GRAV, Rd, Rv, Cpd, Cpv, Cpl, P0, Lv, SIGMA, EPSvap;
    T K_auto, Qc_threshold, K_accr, K_evap, A_term, B_term, T0, ES0, A_SAT, B_SAT;
    T Cd, Ch, Ce, uabs_min, temp_surf, k_abs_qv, k_abs_qc, k_abs_qr, surf_emissivity,
        tau_cooling, z_trop;
    int do_mp, do_auto, do_accr, do_revap, do_sed, do_rd, do_sf;
    const T* dz;
    const T* z;
    const T* zf;
    const double* trcp;  // [nz][TEND_NRCP] reciprocals of the slow tendencies' denominators (kernels.cuh)
};

__device__ __forceinline__ int wrapx(int i, int nx) { return i < 0 ? i + nx : (i >= nx ? i - nx : i); }

template <class T>
__device__ __forceinline__ T f2h(T vf1, T vf2, T dz1, T dz2) {
    return (vf1 * dz2 + vf2 * dz1) / (dz1 + dz2);  // moist.jl:249
}

template <class T>
__device__ __forceinline__ T koren(T r) {  // moist.jl:846
    return jmax(T(0.0), jmin(T(2.0) * r, jmin((T(1.0) + T(2.0) * r) / T(3.0), T(2.0))));
}

template <class T>
__device__ __forceinline__ void sat_vp(T T_k, const DevParams<T>& p, T& es, T& des_dT) {
    const T T_c = T_k - p.T0;  // moist.jl:255-258
    const T tmp = p.B_SAT + T_c;
    es = p.ES0 * mm::mexp(p.A_SAT * T_c / tmp);
    des_dT = es * p.A_SAT * (tmp - T_c) / (tmp * tmp);
}

template <class T>
__device__ __forceinline__ void sat_q(T pr, T es, const DevParams<T>& p, T& qsat, T& dqsat_des) {
    const T tmp = pr - (T(1.0) - p.EPSvap) * es;  // moist.jl:264-271
    if (tmp > p.EPS) {
        qsat = p.EPSvap * es / tmp;
        dqsat_des = p.EPSvap * pr / (tmp * tmp);
    } else {
        qsat = T(0.0);
        dqsat_des = T(1.0);
    }
}

// Kessler microphysics of one cell (moist.jl:561-668); returns the four tendencies
template <class T>
__device__ __forceinline__ void kessler_cell(T rho_k, T rt, T rqv, T rqc, T rqr, const DevParams<T>& p,
                                             T& dqv, T& dqc, T& dqr, T& dth) {
    const T Rd = p.Rd, Rv = p.Rv, Cpd = p.Cpd, Cpv = p.Cpv, Cpl = p.Cpl, P0 = p.P0, Lv = p.Lv;
    dqv = T(0.0);
    dqc = T(0.0);
    dqr = T(0.0);
    dth = T(0.0);
    const T rho_inv = T(1.0) / rho_k;
    T theta_k = rt * rho_inv;
    T qv_k = rqv * rho_inv;
    T qc_k = rqc * rho_inv;
    T qr_k = rqr * rho_inv;
    const T qd = T(1.0) - qv_k - qc_k - qr_k;
    T r = Rd * qd + Rv * qv_k;
    T cp = Cpd * qd + Cpv * qv_k + Cpl * (qc_k + qr_k);
    T cv = cp - r;
    T Pi_k = mm::mpow(r * rt / P0, r / cv);
    T T_k = theta_k * Pi_k;
    T p_k = P0 * mm::mpow(Pi_k, cp / r);
    T latent_heat_eff = Lv / (cp * Pi_k);
    const T qv_init = qv_k;
    T qsat_k = T(0);
    for (int iter = 0; iter < 3; iter++) {
        T es_k, des_dT, dqsat_des;
        sat_vp(T_k, p, es_k, des_dT);
        sat_q(p_k, es_k, p, qsat_k, dqsat_des);
        const T dqsat_dT = dqsat_des * des_dT;
        T cond_evap = (qv_k - qsat_k) / (T(1.0) + (Lv / cp) * dqsat_dT);
        cond_evap = jmin(cond_evap, qv_k);
        cond_evap = jmax(cond_evap, -qc_k);
        qv_k -= cond_evap;
        qc_k += cond_evap;
        theta_k += cond_evap * latent_heat_eff;
        r = Rd * qd + Rv * qv_k;
        cp = Cpd * qd + Cpv * qv_k + Cpl * (qc_k + qr_k);
        cv = cp - r;
        Pi_k = mm::mpow(r * rho_k * theta_k / P0, r / cv);
        T_k = theta_k * Pi_k;
        p_k = P0 * mm::mpow(Pi_k, cp / r);
        latent_heat_eff = Lv / (cp * Pi_k);
    }
    const T cond_evap = qv_init - qv_k;
    const T cond_evap_rate = cond_evap * rho_k / p.dt;
    dqv -= cond_evap_rate;
    dqc += cond_evap_rate;
    dth += cond_evap_rate * latent_heat_eff;
    if (p.do_auto) {
        T rate_auto = p.K_auto * jmax(T(0.0), qc_k - p.Qc_threshold);
        rate_auto = jmin(rate_auto, qc_k / p.dt);
        qc_k -= rate_auto * p.dt;
        qr_k += rate_auto * p.dt;
        rate_auto *= rho_k;
        dqc -= rate_auto;
        dqr += rate_auto;
    }
    if (p.do_accr) {
        T rate_accr = T(0.0);
        if (qr_k > T(1e-12) && qc_k > T(1e-12)) {
            rate_accr = p.K_accr * qc_k * qr_k;
            rate_accr = jmin(rate_accr, qc_k / p.dt);
        }
        qc_k -= rate_accr * p.dt;
        qr_k += rate_accr * p.dt;
        rate_accr *= rho_k;
        dqc -= rate_accr;
        dqr += rate_accr;
    }
    if (p.do_revap) {
        T rate_evap = T(0.0);
        if (qr_k > T(1e-12) && qv_k < qsat_k) {
            rate_evap = p.K_evap * (qsat_k - qv_k) * mm::msqrt(rho_k * qr_k);
            rate_evap = jmin(rate_evap, qr_k) / p.dt;
        }
        rate_evap *= rho_k;
        dqr -= rate_evap;
        dqv += rate_evap;
        r = Rd * qd + Rv * qv_k;
        cp = Cpd * qd + Cpv * qv_k + Cpl * (qc_k + qr_k);
        cv = cp - r;
        Pi_k = mm::mpow(r * rho_k * theta_k / P0, r / cv);
        latent_heat_eff = Lv / (cp * Pi_k);
        dth -= rate_evap * latent_heat_eff;
    }
}

// terminal velocity (moist.jl:681-686)
template <class T>
__device__ __forceinline__ T terminal_velocity(T rqr, T rho, const DevParams<T>& p) {
    const T eff = jmax(T(0.0), rqr);
    return eff > T(1e-12) ? p.A_term * mm::mpow(eff / rho, p.B_term) : T(0.0);
}

// compute_limited_flux_x (moist.jl:850-892) for the face between cells "0" and "p1", with
// the four scalar values s = scalar_rho / rho already formed. Written without branches: the
// upwind operands are selected first and one limiter evaluation follows, so the four face
// fluxes of a tracer cell overlap instead of running one after another. The selected operands
// go through the same operations as the reference's branches, so the result is identical.
template <class T>
__device__ __forceinline__ T limited_flux_x(T vel, T s_m1, T s_0, T s_p1, T s_p2, T EPS) {
    const bool pos = vel > EPS, neg = vel < -EPS;
    const T r_num = pos ? (s_p1 - s_0) : (s_0 - s_p1);
    const T r_den = pos ? (s_0 - s_m1) : (s_p1 - s_p2);
    const T q = r_num / r_den;
    const T r = mm::mabs(r_den) < EPS ? T(1.0) : q;
    const T lim = (pos ? s_0 : s_p1) + T(0.5) * koren(r) * r_den;
    const T cen = T(0.5) * (s_0 + s_p1);
    return ((pos || neg) ? lim : cen) * vel;
}

// compute_limited_flux_z (moist.jl:895-945) for face k+1/2 between cells k ("0") and k+1.
// lin_k / lin_kp1 are the reference's linear-index reads scalar_rho[k] / scalar_rho[k+1]
// (column 1 of the full array); dt_big is the large step p.dt. Branch-free like
// limited_flux_x; the downward limited value keeps the reference's minus sign.
template <class T>
__device__ __forceinline__ T limited_flux_z(T vel, T s_m1, T s_0, T s_p1, T s_p2, int k, int nz,
                                            T dz_k, T dz_kp1, T lin_k, T lin_kp1, T dt_big, T EPS) {
    const bool pos = vel > EPS, neg = vel < -EPS;
    const T f2 = f2h(s_0, s_p1, dz_k, dz_kp1);
    const T clamp = jmin(f2, (pos ? lin_k : lin_kp1) / (pos ? (vel * dt_big) : (-vel * dt_big)));
    const T r_num = pos ? (s_p1 - s_0) : (s_0 - s_p1);
    const T r_den = pos ? (s_0 - s_m1) : (s_p1 - s_p2);
    const T q = r_num / r_den;
    const T r = mm::mabs(r_den) < EPS ? T(1.0) : q;
    const T half = T(0.5) * koren(r) * r_den;
    const T lim = pos ? (s_0 + half) : (s_p1 - half);
    const T face = pos ? ((k == 0) ? clamp : lim) : (neg ? ((k == nz - 2) ? clamp : lim) : f2);
    return face * vel;
}

// third-order upwind face value times the face mass flux, the (-1, 5, 2)/6 form of
// moist.jl:1106, 1290: flux * (-a + 5 b + 2 c) / 6
template <class T>
__device__ __forceinline__ T up3(T flux, T a, T b, T c) {
    return flux * (-a + T(5.0) * b + T(2.0) * c) / T(6.0);
}

}  // namespace moist
