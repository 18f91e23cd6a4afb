// moist_oracle.hpp - CPU restatement of moist2d's large time step (TEST INFRASTRUCTURE).
//
// This is the oracle the CUDA library is checked against. It is not part of the product:
// only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it.
//
// It restates, in the reference's own array layout ((ka, ia) column-major, z fastest) and
// loop order (single thread, i outer ascending, k inner ascending), the Julia functions of
// moist.jl (seiya/moist2d):
//   exchange_halo!          moist.jl:233-241      f2h                  moist.jl:243-251
//   saturation_*            moist.jl:253-273      invert_T_for_thetae  moist.jl:275-289
//   cloud_microphysics!     moist.jl:554-671      rain_sedimentation!  moist.jl:674-707
//   surface_fluxes!         moist.jl:710-752      gray_radiation!      moist.jl:776-840
//   koren_limiter           moist.jl:844-847      compute_limited_flux_x/z moist.jl:850-945
//   solve_tridiagonal!      moist.jl:952-971      implicit_correction! moist.jl:974-1030
//   compute_step!           moist.jl:1039-1580    rk3_step!            moist.jl:1589-1683
// including the reference's quirks (linear-index boundary clamp and large dt in the z flux,
// the sign of the downward z-face value, z-position weights in one f2h, the mixed upwind
// selector of the substep theta flux, the in-place Gauss-Seidel tracer sweep, the Float64
// off-centring factor, mixed-unit rain evaporation cap, rigid lid).
//
// Template parameters: T = Float32/Float64 state type; TT = type of the Thomas elimination
// (T for the reference's literal arithmetic, double for the FP64-elimination mode).
// Scalar math (exp, ^) comes from moist_math.h so that the oracle and the kernels agree bit
// for bit; compile without floating-point contraction (-ffp-contract=off).
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <type_traits>
#include <vector>

#include "../include/moist2d.h"
#include "../moist2d_b200/csrc/moist_math.h"

// ORACLE_OMP builds the timed CPU baseline: the column loops run under OpenMP like the
// reference's Threads.@threads; without it every loop runs on one thread in reference order.
#ifdef ORACLE_OMP
#include <omp.h>
#define OMP_FOR _Pragma("omp parallel for schedule(static)")
#else
#define OMP_FOR
#endif

namespace oracle {

using mm::jmax;
using mm::jmin;

// Wide<T>: the Float64 in which the reference evaluates the off-centring factor even in Float32
// runs (moist.jl:1375). A derivative type (oracle_tangent.cpp instantiates the step with
// mm::Dual) is its own wide type, so that its derivative part is carried through.
template <class T>
using Wide = typename std::conditional<std::is_floating_point<T>::value, double, T>::type;

// Grid vectors arrive in the context precision; a derivative type reads them as Float64 values.
template <class T>
void grid_assign(std::vector<T>& v, const void* src, int n) {
    if (std::is_floating_point<T>::value) {
        v.assign((const T*)src, (const T*)src + n);
    } else {
        const double* d = (const double*)src;
        v.assign(d, d + n);
    }
}

template <class T>
struct Par {
    int Nx, Nz, halo, ia, ka, is, ie, ks, ke, ns;  // 0-based is/ie/ks/ke
    T Lx, H, dx, dt, nu, kappa, gamma_d, beta_offcenter, zf_sponge;
    bool do_mp, do_auto, do_accr, do_revap, do_sed, do_rd, do_sf;
    T Cd, Ch, Ce, uabs_min, temp_surf, k_abs_qv, k_abs_qc, k_abs_qr, surf_emissivity, tau_cooling,
        z_tropopose;
    T GRAV, Rd, Rv, Cpd, Cpv, Cpl, Cvd, P0, Lv, SIGMA, EPSvap;
    T K_auto, Qc_threshold, K_accr, K_evap, A_term, B_term;
    T T0, ES0, A_SAT, B_SAT, EPS;
    std::vector<T> zf, dz, z;

    static Par from_c(const moist_params& c) {
        Par p;
        p.Nx = c.nx;
        p.Nz = c.nz;
        p.halo = c.halo;
        p.ia = c.nx + 2 * c.halo;
        p.ka = c.nz;
        p.is = c.halo;
        p.ie = c.nx + c.halo - 1;
        p.ks = 0;
        p.ke = c.nz - 1;
        p.ns = c.ns;
        p.Lx = (T)c.lx;
        p.H = (T)c.h;
        p.dx = (T)c.dx;
        p.dt = (T)c.dt;
        p.nu = (T)c.nu;
        p.kappa = (T)c.kappa;
        p.gamma_d = (T)c.gamma_d;
        p.beta_offcenter = (T)c.beta_offcenter;
        p.zf_sponge = (T)c.zf_sponge;
        p.do_mp = c.do_mp != 0;
        p.do_auto = c.do_auto != 0;
        p.do_accr = c.do_accr != 0;
        p.do_revap = c.do_revap != 0;
        p.do_sed = c.do_sed != 0;
        p.do_rd = c.do_rd != 0;
        p.do_sf = c.do_sf != 0;
        p.Cd = (T)c.cd;
        p.Ch = (T)c.ch;
        p.Ce = (T)c.ce;
        p.uabs_min = (T)c.uabs_min;
        p.temp_surf = (T)c.temp_surf;
        p.k_abs_qv = (T)c.k_abs_qv;
        p.k_abs_qc = (T)c.k_abs_qc;
        p.k_abs_qr = (T)c.k_abs_qr;
        p.surf_emissivity = (T)c.surf_emissivity;
        p.tau_cooling = (T)c.tau_cooling;
        p.z_tropopose = (T)c.z_tropopause;
        p.GRAV = (T)c.grav;
        p.Rd = (T)c.rd;
        p.Rv = (T)c.rv;
        p.Cpd = (T)c.cpd;
        p.Cpv = (T)c.cpv;
        p.Cpl = (T)c.cpl;
        p.Cvd = (T)c.cvd;
        p.P0 = (T)c.p0;
        p.Lv = (T)c.lv;
        p.SIGMA = (T)c.sigma;
        p.EPSvap = (T)c.epsvap;
        p.K_auto = (T)c.k_auto;
        p.Qc_threshold = (T)c.qc_threshold;
        p.K_accr = (T)c.k_accr;
        p.K_evap = (T)c.k_evap;
        p.A_term = (T)c.a_term;
        p.B_term = (T)c.b_term;
        p.T0 = (T)c.t0;
        p.ES0 = (T)c.es0;
        p.A_SAT = (T)c.a_sat;
        p.B_SAT = (T)c.b_sat;
        p.EPS = (T)c.eps;
        grid_assign(p.zf, c.zf, c.nz);
        grid_assign(p.dz, c.dz, c.nz);
        grid_assign(p.z, c.z, c.nz);
        return p;
    }
};

// (ka, ia) column-major view
template <class T>
struct A2 {
    T* d;
    int ka;
    T& operator()(int k, int i) const { return d[k + (size_t)ka * i]; }
    T& lin(int j) const { return d[j]; }  // Julia linear indexing A[j] (0-based here)
};

template <class T>
struct Field {
    std::vector<T> v;
    int ka, ia;
    Field() : ka(0), ia(0) {}
    Field(int ka_, int ia_, T fill = T(0)) : v((size_t)ka_ * ia_, fill), ka(ka_), ia(ia_) {}
    A2<T> a() { return A2<T>{v.data(), ka}; }
    T* data() { return v.data(); }
};

template <class T>
struct State {
    Field<T> rho, rho_u, rho_w, rho_theta, rho_qv, rho_qc, rho_qr;
    std::vector<T> prec, mflux, shflux, lhflux, theta_ref;
    Field<T> d_rho_theta_mp, d_rho_qv_mp, d_rho_qc_mp, d_rho_qr_mp, d_rho_qr_sed;
    std::vector<T> d_rho_u_sf, d_rho_theta_sf, d_rho_qv_sf;
    Field<T> d_rho_theta_rd;

    explicit State(const Par<T>& p)
        : rho(p.ka, p.ia), rho_u(p.ka, p.ia), rho_w(p.ka, p.ia), rho_theta(p.ka, p.ia),
          rho_qv(p.ka, p.ia), rho_qc(p.ka, p.ia), rho_qr(p.ka, p.ia), prec(p.ia), mflux(p.ia),
          shflux(p.ia), lhflux(p.ia), theta_ref(p.ka), d_rho_theta_mp(p.ka, p.ia),
          d_rho_qv_mp(p.ka, p.ia), d_rho_qc_mp(p.ka, p.ia), d_rho_qr_mp(p.ka, p.ia),
          d_rho_qr_sed(p.ka, p.ia), d_rho_u_sf(p.ia), d_rho_theta_sf(p.ia), d_rho_qv_sf(p.ia),
          d_rho_theta_rd(p.ka, p.ia) {}
};

// ---------------------------------------------------------------- helpers (moist.jl:233-273)

template <class T>
void exchange_halo(A2<T> A, const Par<T>& p) {
    // moist.jl:233-241; sources are read before writing, as Julia's broadcast un-aliases
    std::vector<T> left((size_t)p.ka * p.halo), right((size_t)p.ka * p.halo);
    for (int h = 0; h < p.halo; h++)
        for (int k = 0; k < p.ka; k++) {
            left[k + (size_t)p.ka * h] = A(k, p.ie - p.halo + 1 + h);
            right[k + (size_t)p.ka * h] = A(k, p.is + h);
        }
    for (int h = 0; h < p.halo; h++)
        for (int k = 0; k < p.ka; k++) {
            A(k, h) = left[k + (size_t)p.ka * h];
            A(k, p.ie + 1 + h) = right[k + (size_t)p.ka * h];
        }
}

template <class T>
inline T f2h(T vf1, T vf2, T dz1, T dz2) {
    return (vf1 * dz2 + vf2 * dz1) / (dz1 + dz2);  // moist.jl:249
}

template <class T>
inline void saturation_vapor_pressure(T T_k, const Par<T>& p, T* es, T* des_dT) {
    const T T_c = T_k - p.T0;  // moist.jl:255-259
    const T tmp = p.B_SAT + T_c;
    *es = p.ES0 * mm::mexp(p.A_SAT * T_c / tmp);
    *des_dT = *es * p.A_SAT * (tmp - T_c) / (tmp * tmp);
}

template <class T>
inline void saturation_specific_humidity(T pr, T es, const Par<T>& p, T* qsat, T* dqsat_des) {
    const T tmp = pr - (T(1.0) - p.EPSvap) * es;  // moist.jl:264-272
    if (tmp > p.EPS) {
        *qsat = p.EPSvap * es / tmp;
        *dqsat_des = p.EPSvap * pr / (tmp * tmp);
    } else {
        *qsat = T(0.0);
        *dqsat_des = T(1.0);
    }
}

template <class T>
void invert_T_for_thetae(T qt, T theta_e, T p_k, const Par<T>& p, T* T_out, T* qsat_out) {
    T T_low = T(250.0), T_high = T(350.0);  // moist.jl:275-289
    T qsat = 0;
    for (int iter = 0; iter < 30; iter++) {
        const T t_mid = (T_low + T_high) / T(2);
        T es, d1, d2;
        saturation_vapor_pressure(t_mid, p, &es, &d1);
        saturation_specific_humidity(p_k, es, p, &qsat, &d2);
        const T p_d = p_k - es;
        const T qd = T(1.0) - qt;
        const T cp = p.Cpd * qd + p.Cpl * qt;
        const T theta_mid =
            t_mid * mm::mpow(p_d / p.P0, -p.Rd / cp) * mm::mexp(p.Lv * qsat / (cp * t_mid));
        if (theta_mid > theta_e)
            T_high = t_mid;
        else
            T_low = t_mid;
    }
    *T_out = (T_low + T_high) / T(2);
    *qsat_out = qsat;
}

// ---------------------------------------------------------------- physics (moist.jl:554-840)

template <class T>
void cloud_microphysics(A2<T> d_rho_qv_phys, A2<T> d_rho_qc_phys, A2<T> d_rho_qr_phys,
                        A2<T> d_rho_theta_phys, A2<T> rho, A2<T> rho_theta, A2<T> rho_qv,
                        A2<T> rho_qc, A2<T> rho_qr, const Par<T>& p) {
    const T Rd = p.Rd, Rv = p.Rv, Cpd = p.Cpd, Cpv = p.Cpv, Cpl = p.Cpl, P0 = p.P0, Lv = p.Lv;
    OMP_FOR
    for (int i = p.is; i <= p.ie; i++) {
        for (int k = p.ks; k <= p.ke; k++) {
            d_rho_qv_phys(k, i) = T(0.0);
            d_rho_qc_phys(k, i) = T(0.0);
            d_rho_qr_phys(k, i) = T(0.0);
            d_rho_theta_phys(k, i) = T(0.0);

            const T rho_k = rho(k, i);
            const T rho_inv = T(1.0) / rho_k;
            T theta_k = rho_theta(k, i) * rho_inv;
            T qv_k = rho_qv(k, i) * rho_inv;
            T qc_k = rho_qc(k, i) * rho_inv;
            T qr_k = rho_qr(k, i) * rho_inv;

            const T qd = T(1.0) - qv_k - qc_k - qr_k;
            T r = Rd * qd + Rv * qv_k;
            T cp = Cpd * qd + Cpv * qv_k + Cpl * (qc_k + qr_k);
            T cv = cp - r;
            T Pi_k = mm::mpow(r * rho_theta(k, i) / P0, r / cv);
            T T_k = theta_k * Pi_k;
            T p_k = P0 * mm::mpow(Pi_k, cp / r);
            T latent_heat_eff = Lv / (cp * Pi_k);

            const T qv_init = qv_k;
            T cond_evap = 0, qsat_k = 0;
            for (int iter = 0; iter < 3; iter++) {
                T es_k, des_dT, dqsat_des;
                saturation_vapor_pressure(T_k, p, &es_k, &des_dT);
                saturation_specific_humidity(p_k, es_k, p, &qsat_k, &dqsat_des);
                const T dqsat_dT = dqsat_des * des_dT;
                cond_evap = (qv_k - qsat_k) / (T(1.0) + (Lv / cp) * dqsat_dT);
                cond_evap = jmin(cond_evap, qv_k);
                cond_evap = jmax(cond_evap, -qc_k);
                qv_k -= cond_evap;
                qc_k += cond_evap;
                theta_k += cond_evap * latent_heat_eff;

                r = Rd * qd + Rv * qv_k;
                cp = Cpd * qd + Cpv * qv_k + Cpl * (qc_k + qr_k);
                cv = cp - r;
                Pi_k = mm::mpow(r * rho(k, i) * theta_k / P0, r / cv);
                T_k = theta_k * Pi_k;
                p_k = P0 * mm::mpow(Pi_k, cp / r);
                latent_heat_eff = Lv / (cp * Pi_k);
            }
            cond_evap = qv_init - qv_k;
            const T cond_evap_rate = cond_evap * rho_k / p.dt;
            d_rho_qv_phys(k, i) -= cond_evap_rate;
            d_rho_qc_phys(k, i) += cond_evap_rate;
            d_rho_theta_phys(k, i) += cond_evap_rate * latent_heat_eff;

            if (p.do_auto) {
                T rate_auto = p.K_auto * jmax(T(0.0), qc_k - p.Qc_threshold);
                rate_auto = jmin(rate_auto, qc_k / p.dt);
                qc_k -= rate_auto * p.dt;
                qr_k += rate_auto * p.dt;
                rate_auto *= rho_k;
                d_rho_qc_phys(k, i) -= rate_auto;
                d_rho_qr_phys(k, i) += rate_auto;
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
                d_rho_qc_phys(k, i) -= rate_accr;
                d_rho_qr_phys(k, i) += rate_accr;
            }
            if (p.do_revap) {
                T rate_evap = T(0.0);
                if (qr_k > T(1e-12) && qv_k < qsat_k) {
                    rate_evap = p.K_evap * (qsat_k - qv_k) * mm::msqrt(rho_k * qr_k);
                    rate_evap = jmin(rate_evap, qr_k) / p.dt;
                }
                rate_evap *= rho_k;
                d_rho_qr_phys(k, i) -= rate_evap;
                d_rho_qv_phys(k, i) += rate_evap;
                r = Rd * qd + Rv * qv_k;
                cp = Cpd * qd + Cpv * qv_k + Cpl * (qc_k + qr_k);
                cv = cp - r;
                Pi_k = mm::mpow(r * rho(k, i) * theta_k / P0, r / cv);
                latent_heat_eff = Lv / (cp * Pi_k);
                d_rho_theta_phys(k, i) -= rate_evap * latent_heat_eff;
            }
        }
    }
}

template <class T>
void rain_sedimentation(A2<T> d_rho_qr_sed, T* d_prec, A2<T> rho_qr, A2<T> rho, const Par<T>& p) {
    Field<T> Vt_f(p.ka, p.ia);
    A2<T> Vt = Vt_f.a();
    OMP_FOR
    for (int i = p.is; i <= p.ie; i++)
        for (int k = p.ks; k <= p.ke; k++) {
            const T rho_qr_eff = jmax(T(0.0), rho_qr(k, i));
            Vt(k, i) = rho_qr_eff > T(1e-12) ? p.A_term * mm::mpow(rho_qr_eff / rho(k, i), p.B_term)
                                             : T(0.0);
        }
    OMP_FOR
    for (int i = p.is; i <= p.ie; i++) {
        for (int k = p.ks; k <= p.ke; k++) {
            const T flux_kp = (k == p.ke) ? T(0.0) : rho_qr(k + 1, i) * Vt(k + 1, i);
            const T flux_km = rho_qr(k, i) * Vt(k, i);
            d_rho_qr_sed(k, i) = (flux_kp - flux_km) / p.dz[k];
        }
        d_prec[i] = rho_qr(p.ks, i) * Vt(p.ks, i);
    }
}

template <class T>
void surface_fluxes(T* d_rho_u_sf, T* d_rho_theta_sf, T* d_rho_qv_sf, T* mflux, T* shflux,
                    T* lhflux, A2<T> rho, A2<T> rho_u, A2<T> rho_theta, A2<T> rho_qv,
                    A2<T> rho_qc, A2<T> rho_qr, const Par<T>& p) {
    const int ks = p.ks;
    for (int i = p.is; i <= p.ie; i++) {  // moist.jl:714-751
        const T qv = rho_qv(ks, i) / rho(ks, i);
        const T qc = rho_qc(ks, i) / rho(ks, i);
        const T qr = rho_qr(ks, i) / rho(ks, i);
        const T qd = T(1.0) - qv - qc - qr;
        const T r = p.Rd * qd + p.Rv * qv;
        const T cp = p.Cpd * qd + p.Cpv * qv + p.Cpl * (qc + qr);
        const T cv = cp - r;
        T uabs = mm::mabs(rho_u(ks, i - 1) + rho_u(ks, i)) * T(0.5) / rho(ks, i);
        uabs = jmax(uabs, p.uabs_min);
        const T theta_ks = rho_theta(ks, i) / rho(ks, i);
        const T pi_ks = mm::mpow(r * rho_theta(ks, i) / p.P0, r / cv);
        const T pi_surf = pi_ks + p.dz[ks] * T(0.5) * p.GRAV / (cp * theta_ks);
        const T p_surf = p.P0 * mm::mpow(pi_surf, cp / r);
        const T rho_surf = p_surf / (r * p.temp_surf);
        const T theta_surf = p.temp_surf / pi_surf;
        const T u = rho_u(ks, i) / (rho(ks, i) + rho(ks, i + 1)) * T(2.0);
        mflux[i] = -rho_surf * p.Cd * u * mm::mabs(u);
        d_rho_u_sf[i] = mflux[i] / p.dz[ks];
        const T sh = rho_surf * p.Ch * uabs * (theta_surf - theta_ks) * pi_surf;
        d_rho_theta_sf[i] = sh / (pi_ks * p.dz[ks]);
        shflux[i] = sh * cp;
        T es, d1, qsat_s, d2;
        saturation_vapor_pressure(p.temp_surf, p, &es, &d1);
        saturation_specific_humidity(p_surf, es, p, &qsat_s, &d2);
        const T lh = rho_surf * p.Ce * uabs * (qsat_s - qv);
        d_rho_qv_sf[i] = lh / p.dz[ks];
        lhflux[i] = lh * p.Lv;
    }
}

// tanh from exp, for the radiation's Newtonian-cooling profile (moist.jl:834)
template <class T>
inline T mtanh(T x) {
    const T e = mm::mexp(T(2) * x);
    return (e - T(1)) / (e + T(1));
}

template <class T>
void gray_radiation(A2<T> d_rho_theta_rd, A2<T> rho, A2<T> rho_theta, A2<T> rho_qv, A2<T> rho_qc,
                    A2<T> rho_qr, const T* theta_ref, const Par<T>& p) {
    const int ks = p.ks, ke = p.ke;
    std::vector<T> LW_up(p.ka + 1), LW_dn(p.ka + 1), eps(p.ka), tau(p.ka), temp(p.ka), pi(p.ka),
        cpv(p.ka);
    for (size_t j = 0; j < d_rho_theta_rd.ka * (size_t)p.ia; j++) d_rho_theta_rd.d[j] = T(0.0);
    for (int i = p.is; i <= p.ie; i++) {  // moist.jl:791-839
        for (int k = ks; k <= ke; k++) {
            const T qv = rho_qv(k, i) / rho(k, i);
            const T qc = rho_qc(k, i) / rho(k, i);
            const T qr = rho_qr(k, i) / rho(k, i);
            const T qd = T(1.0) - qv - qc - qr;
            const T r = p.Rd * qd + p.Rv * qv;
            cpv[k] = p.Cpd * qd + p.Cpv * qv + p.Cpl * (qc + qr);
            const T cv = cpv[k] - r;
            pi[k] = mm::mpow(r * rho_theta(k, i) / p.P0, r / cv);
            temp[k] = rho_theta(k, i) / rho(k, i) * pi[k];
            const T dq = p.k_abs_qv * rho_qv(k, i) * p.dz[k];
            const T dc = p.k_abs_qc * rho_qc(k, i) * p.dz[k];
            const T dr = p.k_abs_qr * rho_qr(k, i) * p.dz[k];
            const T delta_opt = dq + dc + dr;
            eps[k] = T(1.0) - mm::mexp(-delta_opt);
            tau[k] = T(1.0) - eps[k];
        }
        const T ts = p.temp_surf;
        LW_up[ks] = p.surf_emissivity * p.SIGMA * mm::mpow4(ts);
        for (int k = ks; k <= ke; k++) {
            const T tk = temp[k];
            LW_up[k + 1] = LW_up[k] * tau[k] + eps[k] * p.SIGMA * mm::mpow4(tk);
        }
        LW_dn[ke + 1] = T(0.0);
        for (int k = ke; k >= ks; k--) {
            const T tk = temp[k];
            LW_dn[k] = LW_dn[k + 1] * tau[k] + eps[k] * p.SIGMA * mm::mpow4(tk);
        }
        const T dz_trans = T(2.0e3);
        for (int k = ks; k <= ke; k++) {
            const T divF = ((LW_up[k + 1] - LW_dn[k + 1]) - (LW_up[k] - LW_dn[k])) / p.dz[k];
            const T hr = -divF / (cpv[k] * pi[k]);
            const T alpha =
                T(0.5) * (T(1.0) + mtanh((p.z[k] - (p.z_tropopose + dz_trans * T(0.5))) / dz_trans)) /
                p.tau_cooling;
            const T cr = -(rho_theta(k, i) - rho(k, i) * theta_ref[k]) * alpha;
            d_rho_theta_rd(k, i) = hr + cr;
        }
    }
}

// ---------------------------------------------------------------- advection helpers (843-945)

template <class T>
inline T koren_limiter(T r) {
    return jmax(T(0.0), jmin(T(2.0) * r, jmin((T(1.0) + T(2.0) * r) / T(3.0), T(2.0))));
}

template <class T>
inline T compute_limited_flux_x(A2<T> scalar_rho, A2<T> rho, A2<T> rho_u, int k, int i,
                                const Par<T>& p) {
    const T EPS = p.EPS;
    const T rhou_face = rho_u(k, i);
    const T s_i = scalar_rho(k, i) / rho(k, i);
    const T s_ip1 = scalar_rho(k, i + 1) / rho(k, i + 1);
    T s_face;
    if (rhou_face > EPS) {
        const T s_im1 = scalar_rho(k, i - 1) / rho(k, i - 1);
        const T r_num = s_ip1 - s_i;
        const T r_den = s_i - s_im1;
        const T r = mm::mabs(r_den) < EPS ? T(1.0) : r_num / r_den;
        const T phi = koren_limiter(r);
        s_face = s_i + T(0.5) * phi * r_den;
    } else if (rhou_face < -EPS) {
        const T s_ip2 = scalar_rho(k, i + 2) / rho(k, i + 2);
        const T r_num = s_i - s_ip1;
        const T r_den = s_ip1 - s_ip2;
        const T r = mm::mabs(r_den) < EPS ? T(1.0) : r_num / r_den;
        const T phi = koren_limiter(r);
        s_face = s_ip1 + T(0.5) * phi * r_den;
    } else {
        s_face = T(0.5) * (s_i + s_ip1);
    }
    return s_face * rhou_face;
}

template <class T>
inline T compute_limited_flux_z(A2<T> scalar_rho, A2<T> rho, A2<T> rho_w, int k, int i,
                                const Par<T>& p, const T* lin = nullptr) {
    if (!lin) lin = scalar_rho.d;
    const T EPS = p.EPS;
    const T dt = p.dt;  // the large step (moist.jl:900)
    const T rhow_face = rho_w(k, i);
    const T s_k = scalar_rho(k, i) / rho(k, i);
    const T s_kp1 = scalar_rho(k + 1, i) / rho(k + 1, i);
    T s_face;
    if (rhow_face > EPS) {
        if (k == p.ks) {
            s_face = f2h(s_k, s_kp1, p.dz[k], p.dz[k + 1]);
            // linear index scalar_rho[k]: element (k, column 1) of the full array (moist.jl:917)
            s_face = jmin(s_face, lin[k] / (rhow_face * dt));
        } else {
            const T s_km1 = scalar_rho(k - 1, i) / rho(k - 1, i);
            const T r_num = s_kp1 - s_k;
            const T r_den = s_k - s_km1;
            const T r = mm::mabs(r_den) < EPS ? T(1.0) : r_num / r_den;
            const T phi = koren_limiter(r);
            s_face = s_k + T(0.5) * phi * r_den;
        }
    } else if (rhow_face < -EPS) {
        if (k == p.ke - 1) {
            s_face = f2h(s_k, s_kp1, p.dz[k], p.dz[k + 1]);
            s_face = jmin(s_face, lin[k + 1] / (-rhow_face * dt));  // moist.jl:930
        } else {
            const T s_kp2 = scalar_rho(k + 2, i) / rho(k + 2, i);
            const T r_num = s_k - s_kp1;
            const T r_den = s_kp1 - s_kp2;
            const T r = mm::mabs(r_den) < EPS ? T(1.0) : r_num / r_den;
            const T phi = koren_limiter(r);
            s_face = s_kp1 - T(0.5) * phi * r_den;  // minus sign as written (moist.jl:938)
        }
    } else {
        s_face = f2h(s_k, s_kp1, p.dz[k], p.dz[k + 1]);
    }
    return s_face * rhow_face;
}

// ---------------------------------------------------------------- tridiagonal (moist.jl:947-1030)

template <class TT>
void solve_tridiagonal(TT* a, TT* b, TT* c, TT* d, int n) {
    const TT c_1 = c[0] / b[0];
    const TT d_1 = d[0] / b[0];
    c[0] = c_1;
    d[0] = d_1;
    for (int i = 1; i < n; i++) {
        const TT temp = b[i] - a[i] * c[i - 1];
        const TT c_i = c[i] / temp;
        const TT d_i = (d[i] - a[i] * d[i - 1]) / temp;
        c[i] = c_i;
        d[i] = d_i;
    }
    for (int i = n - 2; i >= 0; i--) d[i] = d[i] - c[i] * d[i + 1];
}

// rho_w, drho_w, theta, rt2pres: one column, length ka
template <class T, class TT>
void implicit_correction(T* rho_w, const T* drho_w, const T* theta, const T* rt2pres, T dt,
                         const Par<T>& p) {
    const int ks = p.ks, ke = p.ke, n = p.Nz - 1;
    const std::vector<T>& z = p.z;
    const std::vector<T>& dz = p.dz;
    const T GRAV = p.GRAV;
    std::vector<T> theta_h(p.ka, T(0));
    for (int k = ks; k <= ke - 1; k++) theta_h[k] = f2h(theta[k], theta[k + 1], dz[k], dz[k + 1]);
    const T fact_tp = T(0.5) * (T(1.0) + p.beta_offcenter);
    const T fact_tm = T(0.5) * (T(1.0) - p.beta_offcenter);
    const T dt_tp2 = (dt * fact_tp) * (dt * fact_tp);
    std::vector<T> a(n, T(0)), b(n, T(0)), c(n, T(0)), d(n, T(0));
    for (int k = ks; k <= ke - 1; k++) {
        const int j = k - ks;
        b[j] = dt_tp2 * (rt2pres[k] / dz[k] + rt2pres[k + 1] / dz[k + 1]) * theta_h[k] /
               (z[k + 1] - z[k]);
        if (k > ks)
            a[j] = -dt_tp2 * (rt2pres[k] * theta_h[k - 1] / ((z[k + 1] - z[k]) * dz[k]) -
                              GRAV / (dz[k] + dz[k + 1]));
        if (k < ke - 1)
            c[j] = -dt_tp2 * (rt2pres[k + 1] * theta_h[k + 1] / ((z[k + 1] - z[k]) * dz[k + 1]) +
                              GRAV / (dz[k] + dz[k + 1]));
        d[j] = rho_w[k] + drho_w[k];
    }
    const T fact = fact_tm / fact_tp;
    for (int k = ks; k <= ke - 1; k++) {
        const int j = k - ks;
        if (k > ks) d[j] -= a[j] * fact * rho_w[k];  // rho_w[k], as written (moist.jl:1014)
        d[j] -= b[j] * fact * rho_w[k];
        b[j] += T(1.0);
        if (k < ke - 1) d[j] -= c[j] * fact * rho_w[k + 1];
    }
    std::vector<TT> A(a.begin(), a.end()), B(b.begin(), b.end()), C(c.begin(), c.end()),
        D(d.begin(), d.end());
    solve_tridiagonal<TT>(A.data(), B.data(), C.data(), D.data(), n);
    for (int k = ks; k <= ke - 1; k++) rho_w[k] = (T)D[k - ks];
}

// ---------------------------------------------------------------- one tracer cell (1479-1515)

// The update of rho_scalar at (k, i) (moist.jl:1479-1515), in place. lin is column 1 of the full
// array, which the linear-index boundary clamp of compute_limited_flux_z reads.
template <class T>
inline void tracer_cell(A2<T> rs, const T* lin, A2<T> rs0, A2<T> d_phys, A2<T> rho, A2<T> mom_flux_x,
                        A2<T> mom_flux_z, const Par<T>& p, T dt, int k, int i) {
    const int ks = p.ks, ke = p.ke;
    const T dx = p.dx, kappa = p.kappa;
    const std::vector<T>& dz = p.dz;
    const std::vector<T>& z = p.z;
    const T flux_x_ip = compute_limited_flux_x(rs, rho, mom_flux_x, k, i, p);
    const T flux_x_im = compute_limited_flux_x(rs, rho, mom_flux_x, k, i - 1, p);
    const T adv_x = (flux_x_ip - flux_x_im) / dx;
    const T flux_z_kp = k == ke ? T(0.0) : compute_limited_flux_z(rs, rho, mom_flux_z, k, i, p, lin);
    const T flux_z_km = k == ks ? T(0.0) : compute_limited_flux_z(rs, rho, mom_flux_z, k - 1, i, p, lin);
    const T adv_z = (flux_z_kp - flux_z_km) / dz[k];
    const T advection = -(adv_x + adv_z);
    const T scalar_c = rs(k, i) / rho(k, i);
    const T scalar_ip = rs(k, i + 1) / rho(k, i + 1);
    const T scalar_im = rs(k, i - 1) / rho(k, i - 1);
    const T scalar_kp = k == ke ? T(0.0) : rs(k + 1, i) / rho(k + 1, i);
    const T scalar_km = k == ks ? T(0.0) : rs(k - 1, i) / rho(k - 1, i);
    const T dsdx_ip = (rho(k, i + 1) + rho(k, i)) * T(0.5) * (scalar_ip - scalar_c) / dx;
    const T dsdx_im = (rho(k, i) + rho(k, i - 1)) * T(0.5) * (scalar_c - scalar_im) / dx;
    const T diff_x = kappa * (dsdx_ip - dsdx_im) / dx;
    const T dsdz_kp = k == ke ? T(0.0)
                              : f2h(rho(k + 1, i), rho(k, i), dz[k + 1], dz[k]) * (scalar_kp - scalar_c) /
                                    (z[k + 1] - z[k]);
    const T dsdz_km = k == ks ? T(0.0)
                              : f2h(rho(k, i), rho(k - 1, i), dz[k], dz[k - 1]) * (scalar_c - scalar_km) /
                                    (z[k] - z[k - 1]);
    const T diff_z = kappa * (dsdz_kp - dsdz_km) / dz[k];
    const T diffusion = diff_x + diff_z;
    rs(k, i) = rs0(k, i) + dt * (advection + diffusion + d_phys(k, i));
}

// ---------------------------------------------------------------- one RK stage (1039-1580)

// returns -1, or the index (MOIST_FIELD_*) of the first field found with a NaN
template <class T, class TT>
int compute_step(A2<T> d_rho_phys, A2<T> d_rho_u_phys, A2<T> d_rho_theta_phys, A2<T> d_rho_qv_phys,
                 A2<T> d_rho_qc_phys, A2<T> d_rho_qr_phys, State<T>& s, State<T>& s0,
                 const Par<T>& p, T dt, int ns) {
    const int ka = p.ka, ia = p.ia, ks = p.ks, ke = p.ke, is = p.is, ie = p.ie;
    const T dx = p.dx, nu = p.nu, kappa = p.kappa, gamma_d = p.gamma_d, zf_sponge = p.zf_sponge;
    const T EPS = p.EPS, GRAV = p.GRAV;
    const std::vector<T>& dz = p.dz;
    const std::vector<T>& z = p.z;
    const std::vector<T>& zf = p.zf;
    A2<T> rho = s.rho.a(), rho_u = s.rho_u.a(), rho_w = s.rho_w.a(), rho_theta = s.rho_theta.a();

    // --- diagnostics (moist.jl:1045-1065)
    Field<T> pres_f(ka, ia), theta_f(ka, ia), rt2pres_f(ka, ia);
    A2<T> pres = pres_f.a(), theta = theta_f.a(), rt2pres = rt2pres_f.a();
    OMP_FOR
    for (int i = is; i <= ie + 1; i++)
        for (int k = ks; k <= ke; k++) {
            const T qv = s.rho_qv.a()(k, i) / rho(k, i);
            const T qc = s.rho_qc.a()(k, i) / rho(k, i);
            const T qr = s.rho_qr.a()(k, i) / rho(k, i);
            const T qd = T(1.0) - qv - qc - qr;
            const T r = p.Rd * qd + p.Rv * qv;
            const T cp = p.Cpd * qd + p.Cpv * qv + p.Cpl * (qc + qr);
            const T cv = cp - r;
            pres(k, i) = p.P0 * mm::mpow(r * rho_theta(k, i) / p.P0, cp / cv);
            theta(k, i) = rho_theta(k, i) / rho(k, i);
            rt2pres(k, i) = cp / cv * pres(k, i) / rho_theta(k, i);
        }
    exchange_halo(pres, p);
    exchange_halo(theta, p);
    exchange_halo(rt2pres, p);
    exchange_halo(rho, p);
    exchange_halo(rho_u, p);
    exchange_halo(rho_w, p);

    Field<T> R_rho_f(ka, ia), R_rho_u_f(ka, ia), R_rho_w_f(ka, ia), R_rho_theta_f(ka, ia);
    A2<T> R_rho = R_rho_f.a(), R_rho_u = R_rho_u_f.a(), R_rho_w = R_rho_w_f.a(),
          R_rho_theta = R_rho_theta_f.a();

    // --- R_rho (moist.jl:1079-1086)
    OMP_FOR
    for (int i = is; i <= ie; i++)
        for (int k = ks; k <= ke; k++) {
            const T flux_kp = k == ke ? T(0.0) : rho_w(k, i);
            const T flux_km = k == ks ? T(0.0) : rho_w(k - 1, i);
            const T advection = -((rho_u(k, i) - rho_u(k, i - 1)) / dx + (flux_kp - flux_km) / dz[k]);
            R_rho(k, i) = advection + d_rho_phys(k, i);
        }

    // --- R_rho_u (moist.jl:1091-1179)
    Field<T> u_face_f(ka, ia);
    A2<T> u_face = u_face_f.a();
    OMP_FOR
    for (int i = is; i <= ie; i++)
        for (int k = ks; k <= ke; k++)
            u_face(k, i) = rho_u(k, i) * T(2.0) / (rho(k, i) + rho(k, i + 1));
    exchange_halo(u_face, p);
    OMP_FOR
    for (int i = is; i <= ie; i++)
        for (int k = ks; k <= ke; k++) {
            const T rho_u_ip = T(0.5) * (rho_u(k, i) + rho_u(k, i + 1));
            T flux_uu_x_ip;
            if (rho_u_ip > EPS)
                flux_uu_x_ip = rho_u_ip *
                               (-u_face(k, i - 1) + T(5.0) * u_face(k, i) + T(2.0) * u_face(k, i + 1)) /
                               T(6.0);
            else if (rho_u_ip < -EPS)
                flux_uu_x_ip = rho_u_ip *
                               (-u_face(k, i + 2) + T(5.0) * u_face(k, i + 1) + T(2.0) * u_face(k, i)) /
                               T(6.0);
            else
                flux_uu_x_ip = rho_u_ip * (u_face(k, i) + u_face(k, i + 1)) * T(0.5);
            const T rho_u_im = T(0.5) * (rho_u(k, i - 1) + rho_u(k, i));
            T flux_uu_x_im;
            if (rho_u_im > EPS)
                flux_uu_x_im = rho_u_im *
                               (-u_face(k, i - 2) + T(5.0) * u_face(k, i - 1) + T(2.0) * u_face(k, i)) /
                               T(6.0);
            else if (rho_u_im < -EPS)
                flux_uu_x_im = rho_u_im *
                               (-u_face(k, i + 1) + T(5.0) * u_face(k, i) + T(2.0) * u_face(k, i - 1)) /
                               T(6.0);
            else
                flux_uu_x_im = rho_u_im * (u_face(k, i - 1) + u_face(k, i)) * T(0.5);
            const T druudx = (flux_uu_x_ip - flux_uu_x_im) / dx;

            T flux_uw_z_kp;
            if (k == ke) {
                flux_uw_z_kp = T(0.0);
            } else {
                const T rho_w_kp = T(0.5) * (rho_w(k, i) + rho_w(k, i + 1));
                if (rho_w_kp > EPS && k > ks)
                    flux_uw_z_kp = rho_w_kp *
                                   (-u_face(k - 1, i) + T(5.0) * u_face(k, i) + T(2.0) * u_face(k + 1, i)) /
                                   T(6.0);
                else if (rho_w_kp < -EPS && k < ke - 1)
                    flux_uw_z_kp = rho_w_kp *
                                   (-u_face(k + 2, i) + T(5.0) * u_face(k + 1, i) + T(2.0) * u_face(k, i)) /
                                   T(6.0);
                else
                    flux_uw_z_kp = rho_w_kp * f2h(u_face(k, i), u_face(k + 1, i), dz[k], dz[k + 1]);
            }
            T flux_uw_z_km;
            if (k == ks) {
                flux_uw_z_km = T(0.0);
            } else {
                const T rho_w_km = T(0.5) * (rho_w(k - 1, i) + rho_w(k - 1, i + 1));
                if (rho_w_km > EPS && k > ks + 1)
                    flux_uw_z_km = rho_w_km *
                                   (-u_face(k - 2, i) + T(5.0) * u_face(k - 1, i) + T(2.0) * u_face(k, i)) /
                                   T(6.0);
                else if (rho_w_km < -EPS && k < ke)
                    flux_uw_z_km = rho_w_km *
                                   (-u_face(k + 1, i) + T(5.0) * u_face(k, i) + T(2.0) * u_face(k - 1, i)) /
                                   T(6.0);
                else
                    flux_uw_z_km = rho_w_km * f2h(u_face(k - 1, i), u_face(k, i), dz[k - 1], dz[k]);
            }
            const T drwudz = (flux_uw_z_kp - flux_uw_z_km) / dz[k];
            const T advection = -druudx - drwudz;

            const T u_ip = (u_face(k, i + 1) - u_face(k, i)) / dx;
            const T u_im = (u_face(k, i) - u_face(k, i - 1)) / dx;
            const T u_xx_term = (u_ip * rho(k, i + 1) - u_im * rho(k, i)) / dx;
            const T u_kp = k == ke ? T(0.0) : (u_face(k + 1, i) - u_face(k, i)) / (z[k + 1] - z[k]);
            const T u_km = k == ks ? T(0.0) : (u_face(k, i) - u_face(k - 1, i)) / (z[k] - z[k - 1]);
            const T rho_kp = k == ke ? T(0.0)
                                     : T(0.25) * (rho(k, i) + rho(k + 1, i) + rho(k, i + 1) + rho(k + 1, i + 1));
            const T rho_km = k == ks ? T(0.0)
                                     : T(0.25) * (rho(k - 1, i) + rho(k, i) + rho(k - 1, i + 1) + rho(k, i + 1));
            const T u_zz_term = (u_kp * rho_kp - u_km * rho_km) / dz[k];
            const T diffusion = nu * (u_xx_term + u_zz_term);
            const T dpdx = (pres(k, i + 1) - pres(k, i)) / dx;
            R_rho_u(k, i) = advection - dpdx + diffusion + d_rho_u_phys(k, i);
        }

    // --- R_rho_w (moist.jl:1184-1278)
    Field<T> w_face_f(ka, ia);
    A2<T> w_face = w_face_f.a();
    OMP_FOR
    for (int i = is - 2; i <= ie + 2; i++)
        for (int k = ks; k <= ke - 1; k++)
            w_face(k, i) = rho_w(k, i) / f2h(rho(k, i), rho(k + 1, i), dz[k], dz[k + 1]);
    OMP_FOR
    for (int i = is; i <= ie; i++)
        for (int k = ks; k <= ke - 1; k++) {
            const T rho_u_ip = f2h(rho_u(k, i), rho_u(k + 1, i), z[k], z[k + 1]);  // z weights (1196)
            T flux_uw_x_ip;
            if (rho_u_ip > EPS)
                flux_uw_x_ip = rho_u_ip *
                               (-w_face(k, i - 1) + T(5.0) * w_face(k, i) + T(2.0) * w_face(k, i + 1)) /
                               T(6.0);
            else if (rho_u_ip < -EPS)
                flux_uw_x_ip = rho_u_ip *
                               (-w_face(k, i + 2) + T(5.0) * w_face(k, i + 1) + T(2.0) * w_face(k, i)) /
                               T(6.0);
            else
                flux_uw_x_ip = rho_u_ip * (w_face(k, i) + w_face(k, i + 1)) * T(0.5);
            const T rho_u_im = f2h(rho_u(k, i - 1), rho_u(k + 1, i - 1), dz[k], dz[k + 1]);
            T flux_uw_x_im;
            if (rho_u_im > EPS)
                flux_uw_x_im = rho_u_im *
                               (-w_face(k, i - 2) + T(5.0) * w_face(k, i - 1) + T(2.0) * w_face(k, i)) /
                               T(6.0);
            else if (rho_u_im < -EPS)
                flux_uw_x_im = rho_u_im *
                               (-w_face(k, i + 1) + T(5.0) * w_face(k, i) + T(2.0) * w_face(k, i - 1)) /
                               T(6.0);
            else
                flux_uw_x_im = rho_u_im * (w_face(k, i - 1) + w_face(k, i)) * T(0.5);
            const T drwudx = (flux_uw_x_ip - flux_uw_x_im) / dx;

            T flux_ww_z_kp;
            if (k == ke - 1) {
                flux_ww_z_kp = T(0.0);
            } else {
                const T rho_w_kp = f2h(rho_w(k, i), rho_w(k + 1, i), dz[k], dz[k + 1]);
                if (rho_w_kp > EPS && k > ks)
                    flux_ww_z_kp = rho_w_kp *
                                   (-w_face(k - 1, i) + T(5.0) * w_face(k, i) + T(2.0) * w_face(k + 1, i)) /
                                   T(6.0);
                else if (rho_w_kp < -EPS && k < ke - 2)
                    flux_ww_z_kp = rho_w_kp *
                                   (-w_face(k + 2, i) + T(5.0) * w_face(k + 1, i) + T(2.0) * w_face(k, i)) /
                                   T(6.0);
                else
                    flux_ww_z_kp = rho_w_kp * f2h(w_face(k, i), w_face(k + 1, i), dz[k], dz[k + 1]);
            }
            T flux_ww_z_km;
            if (k == ks) {
                flux_ww_z_km = T(0.0);
            } else {
                const T rho_w_km = f2h(rho_w(k - 1, i), rho_w(k, i), dz[k - 1], dz[k]);
                if (rho_w_km > EPS && k > ks + 1)
                    flux_ww_z_km = rho_w_km *
                                   (-w_face(k - 2, i) + T(5.0) * w_face(k - 1, i) + T(2.0) * w_face(k, i)) /
                                   T(6.0);
                else if (rho_w_km < -EPS && k < ke - 1)
                    flux_ww_z_km = rho_w_km *
                                   (-w_face(k + 1, i) + T(5.0) * w_face(k, i) + T(2.0) * w_face(k - 1, i)) /
                                   T(6.0);
                else
                    flux_ww_z_km = rho_w_km * f2h(w_face(k - 1, i), w_face(k, i), dz[k - 1], dz[k]);
            }
            const T drwwdz = (flux_ww_z_kp - flux_ww_z_km) / (z[k + 1] - z[k]);
            const T advection = -drwudx - drwwdz;

            const T w_ip = (w_face(k, i + 1) - w_face(k, i)) / dx;
            const T w_im = (w_face(k, i) - w_face(k, i - 1)) / dx;
            const T rho_ip = T(0.25) * (rho(k, i) + rho(k + 1, i) + rho(k, i + 1) + rho(k + 1, i + 1));
            const T rho_im = T(0.25) * (rho(k, i - 1) + rho(k + 1, i - 1) + rho(k, i) + rho(k + 1, i));
            const T w_xx_term = (w_ip * rho_ip - w_im * rho_im) / dx;
            const T w_kp = k == ke - 1 ? T(0.0) : (w_face(k + 1, i) - w_face(k, i)) / dz[k + 1];
            const T w_km = k == ks ? T(0.0) : (w_face(k, i) - w_face(k - 1, i)) / dz[k];
            const T w_zz_term = (w_kp * rho(k + 1, i) - w_km * rho(k, i)) / (z[k + 1] - z[k]);
            const T diffusion = nu * (w_xx_term + w_zz_term);
            T sigma = T(0.0);
            if (zf[k] > (T(1.0) - zf_sponge) * p.H)
                sigma = (GRAV / T(30.0)) * ((zf[k] - (T(1.0) - zf_sponge) * p.H) / (zf_sponge * p.H));
            const T sponge_term = -sigma * rho_w(k, i);
            const T dpdz = (pres(k + 1, i) - pres(k, i)) / (z[k + 1] - z[k]);
            const T buoyancy = -GRAV * (rho(k, i) + rho(k + 1, i)) * T(0.5);
            R_rho_w(k, i) = advection - dpdz + buoyancy + diffusion + sponge_term;
        }

    // --- R_rho_theta (moist.jl:1284-1332)
    OMP_FOR
    for (int i = is; i <= ie; i++)
        for (int k = ks; k <= ke; k++) {
            T flux_ip, flux_im, flux_kp, flux_km;
            if (rho_u(k, i) > EPS)
                flux_ip = rho_u(k, i) * (-theta(k, i - 1) + T(5.0) * theta(k, i) + T(2.0) * theta(k, i + 1)) / T(6.0);
            else if (rho_u(k, i) < -EPS)
                flux_ip = rho_u(k, i) * (-theta(k, i + 2) + T(5.0) * theta(k, i + 1) + T(2.0) * theta(k, i)) / T(6.0);
            else
                flux_ip = rho_u(k, i) * (theta(k, i) + theta(k, i + 1)) * T(0.5);
            if (rho_u(k, i - 1) > EPS)
                flux_im = rho_u(k, i - 1) * (-theta(k, i - 2) + T(5.0) * theta(k, i - 1) + T(2.0) * theta(k, i)) / T(6.0);
            else if (rho_u(k, i - 1) < -EPS)
                flux_im = rho_u(k, i - 1) * (-theta(k, i + 1) + T(5.0) * theta(k, i) + T(2.0) * theta(k, i - 1)) / T(6.0);
            else
                flux_im = rho_u(k, i - 1) * (theta(k, i - 1) + theta(k, i)) * T(0.5);
            if (k == ke) {
                flux_kp = T(0.0);
            } else {
                if (rho_w(k, i) > EPS && k > ks)
                    flux_kp = rho_w(k, i) * (-theta(k - 1, i) + T(5.0) * theta(k, i) + T(2.0) * theta(k + 1, i)) / T(6.0);
                else if (rho_w(k, i) < -EPS && k < ke - 1)
                    flux_kp = rho_w(k, i) * (-theta(k + 2, i) + T(5.0) * theta(k + 1, i) + T(2.0) * theta(k, i)) / T(6.0);
                else
                    flux_kp = rho_w(k, i) * f2h(theta(k, i), theta(k + 1, i), dz[k], dz[k + 1]);
            }
            if (k == ks) {
                flux_km = T(0.0);
            } else {
                if (rho_w(k - 1, i) > EPS && k > ks + 1)
                    flux_km = rho_w(k - 1, i) * (-theta(k - 2, i) + T(5.0) * theta(k - 1, i) + T(2.0) * theta(k, i)) / T(6.0);
                else if (rho_w(k - 1, i) < -EPS && k < ke)
                    flux_km = rho_w(k - 1, i) * (-theta(k + 1, i) + T(5.0) * theta(k, i) + T(2.0) * theta(k - 1, i)) / T(6.0);
                else
                    flux_km = rho_w(k - 1, i) * f2h(theta(k - 1, i), theta(k, i), dz[k - 1], dz[k]);
            }
            const T advection = -((flux_ip - flux_im) / dx + (flux_kp - flux_km) / dz[k]);
            R_rho_theta(k, i) = advection + d_rho_theta_phys(k, i);
        }

    // --- perturbations (moist.jl:1339-1348)
    Field<T> rho_p_f(ka, ia), rho_u_p_f(ka, ia), rho_w_p_f(ka, ia), rho_theta_p_f(ka, ia);
    A2<T> rho_p = rho_p_f.a(), rho_u_p = rho_u_p_f.a(), rho_w_p = rho_w_p_f.a(),
          rho_theta_p = rho_theta_p_f.a();
    OMP_FOR
    for (long j = 0; j < (long)ka * ia; j++) {
        rho_p.d[j] = s0.rho.v[j] - s.rho.v[j];
        rho_u_p.d[j] = s0.rho_u.v[j] - s.rho_u.v[j];
        rho_w_p.d[j] = s0.rho_w.v[j] - s.rho_w.v[j];
        rho_theta_p.d[j] = s0.rho_theta.v[j] - s.rho_theta.v[j];
    }
    exchange_halo(rho_theta_p, p);
    Field<T> rho_theta_p_old_f = rho_theta_p_f;
    A2<T> rho_theta_p_old = rho_theta_p_old_f.a();
    Field<T> mom_flux_x_f = s.rho_u, mom_flux_z_f = s.rho_w;
    A2<T> mom_flux_x = mom_flux_x_f.a(), mom_flux_z = mom_flux_z_f.a();

    // --- acoustic substeps (moist.jl:1351-1461)
    const T dt_s = dt / T(ns);
    for (int n = 1; n <= ns; n++) {
        if (n > 1) exchange_halo(rho_theta_p, p);
        OMP_FOR
        for (int i = is; i <= ie; i++)
            for (int k = ks; k <= ke; k++) {
                T grad_x = (rho_theta_p(k, i + 1) - rho_theta_p(k, i)) / dx;
                const T grad_x_old = (rho_theta_p_old(k, i + 1) - rho_theta_p_old(k, i)) / dx;
                grad_x = grad_x + gamma_d * (grad_x - grad_x_old);
                const T rt2pres_h = (rt2pres(k, i) + rt2pres(k, i + 1)) * T(0.5);
                rho_u_p(k, i) += dt_s * (R_rho_u(k, i) - rt2pres_h * grad_x);
            }
        exchange_halo(rho_u_p, p);
        rho_theta_p_old_f.v = rho_theta_p_f.v;
        // Float64 factor even in Float32 runs: T(0.5) * (1.0 + beta) (moist.jl:1375)
        using W = Wide<T>;
        const W fact_tp = W(T(0.5)) * (W(1.0) + W(p.beta_offcenter));
        OMP_FOR
        for (int i = is; i <= ie; i++) {
            std::vector<T> rho_p_tp(ka), rho_theta_p_tp(ka), drho_w_p(ka, T(0));
            for (int k = ks; k <= ke; k++) {
                T advection = -(rho_u_p(k, i) - rho_u_p(k, i - 1)) / dx;
                T inc = dt_s * (R_rho(k, i) + advection);
                rho_p_tp[k] = (T)(W(rho_p(k, i)) + fact_tp * W(inc));
                rho_p(k, i) += inc;
                const T flux_ip = (theta(k, i + 1) + theta(k, i)) * T(0.5) * rho_u_p(k, i);
                const T flux_im = (theta(k, i) + theta(k, i - 1)) * T(0.5) * rho_u_p(k, i - 1);
                advection = -(flux_ip - flux_im) / dx;
                inc = dt_s * (R_rho_theta(k, i) + advection);
                rho_theta_p_tp[k] = (T)(W(rho_theta_p(k, i)) + fact_tp * W(inc));
                rho_theta_p(k, i) += inc;
            }
            for (int k = ks; k <= ke - 1; k++) {
                const T buoyancy = (rho_theta_p_tp[k + 1] - rho_theta_p_tp[k]) / (z[k + 1] - z[k]);
                const T grav = -GRAV * T(0.5) * (rho_p_tp[k + 1] + rho_p_tp[k]);
                const T rt2pres_h = (rt2pres(k, i) + rt2pres(k + 1, i)) * T(0.5);
                drho_w_p[k] = dt_s * (R_rho_w(k, i) - rt2pres_h * buoyancy + grav);
            }
            implicit_correction<T, TT>(&rho_w_p(0, i), drho_w_p.data(), &theta(0, i), &rt2pres(0, i),
                                       dt_s, p);
            for (int k = ks; k <= ke; k++) {
                const T flux_kp = k == ke ? T(0.0) : rho_w_p(k, i);
                const T flux_km = k == ks ? T(0.0) : rho_w_p(k - 1, i);
                const T advection = -(flux_kp - flux_km) / dz[k];
                rho_p(k, i) += dt_s * advection;
            }
            for (int k = ks; k <= ke; k++) {
                T flux_kp, flux_km;
                if (k == ke) {
                    flux_kp = T(0.0);
                } else {
                    if (rho_w_p(k, i) > EPS && k > ks)
                        flux_kp = rho_w_p(k, i) * (-theta(k - 1, i) + T(5.0) * theta(k, i) + T(2.0) * theta(k + 1, i)) / T(6.0);
                    else if (rho_w(k, i) < -EPS && k < ke - 1)  // s.rho_w selects (moist.jl:1426)
                        flux_kp = rho_w_p(k, i) * (-theta(k + 2, i) + T(5.0) * theta(k + 1, i) + T(2.0) * theta(k, i)) / T(6.0);
                    else
                        flux_kp = rho_w_p(k, i) * f2h(theta(k, i), theta(k + 1, i), dz[k], dz[k + 1]);
                }
                if (k == ks) {
                    flux_km = T(0.0);
                } else {
                    if (rho_w(k - 1, i) > EPS && k > ks + 1)
                        flux_km = rho_w_p(k - 1, i) * (-theta(k - 2, i) + T(5.0) * theta(k - 1, i) + T(2.0) * theta(k, i)) / T(6.0);
                    else if (rho_w(k - 1, i) < -EPS && k < ke)
                        flux_km = rho_w_p(k - 1, i) * (-theta(k + 1, i) + T(5.0) * theta(k, i) + T(2.0) * theta(k - 1, i)) / T(6.0);
                    else
                        flux_km = rho_w_p(k - 1, i) * f2h(theta(k - 1, i), theta(k, i), dz[k - 1], dz[k]);
                }
                const T advection = -(flux_kp - flux_km) / dz[k];
                rho_theta_p(k, i) += dt_s * advection;
            }
        }
        OMP_FOR
        for (int i = is; i <= ie; i++) {
            for (int k = ks; k <= ke; k++) mom_flux_x(k, i) += rho_u_p(k, i) / T(ns);
            for (int k = ks; k <= ke - 1; k++) mom_flux_z(k, i) += rho_w_p(k, i) / T(ns);
        }
    }

    exchange_halo(mom_flux_x, p);
    exchange_halo(s.rho_qv.a(), p);
    exchange_halo(s.rho_qc.a(), p);
    exchange_halo(s.rho_qr.a(), p);

    // --- tracer transport: in-place, lexicographic Gauss-Seidel order (moist.jl:1469-1518)
    A2<T> trs[3] = {s.rho_qv.a(), s.rho_qc.a(), s.rho_qr.a()};
    A2<T> tr0[3] = {s0.rho_qv.a(), s0.rho_qc.a(), s0.rho_qr.a()};
    A2<T> dph[3] = {d_rho_qv_phys, d_rho_qc_phys, d_rho_qr_phys};
#ifndef ORACLE_OMP
    for (int i = is; i <= ie; i++)
        for (int k = ks; k <= ke; k++)
            for (int t = 0; t < 3; t++) tracer_cell(trs[t], trs[t].d, tr0[t], dph[t], rho, mom_flux_x, mom_flux_z, p, dt, k, i);
#else
    // Threads.@threads over i: each thread sweeps a contiguous chunk of columns in order and
    // reads the two columns left of its chunk from the pre-sweep values
    {
        std::vector<std::vector<T>> snap(3);
        for (int t = 0; t < 3; t++) snap[t] = std::vector<T>(trs[t].d, trs[t].d + (size_t)ka * ia);
#pragma omp parallel
        {
            const int nt = omp_get_num_threads(), tid = omp_get_thread_num();
            const int nxi = ie - is + 1;
            const int i0 = is + (int)((long)nxi * tid / nt), i1 = is + (int)((long)nxi * (tid + 1) / nt);
            if (i1 > i0) {
                for (int t = 0; t < 3; t++) {
                    std::vector<T> buf((size_t)ka * (i1 - i0 + 4));
                    for (int i = i0 - 2; i < i1 + 2; i++)
                        for (int k = 0; k < ka; k++) buf[k + (size_t)ka * (i - i0 + 2)] = snap[t][k + (size_t)ka * i];
                    A2<T> loc{buf.data() - (ptrdiff_t)ka * (i0 - 2), ka};
                    for (int i = i0; i < i1; i++)
                        for (int k = ks; k <= ke; k++)
                            tracer_cell(loc, snap[t].data(), tr0[t], dph[t], rho, mom_flux_x, mom_flux_z, p, dt, k, i);
                    for (int i = i0; i < i1; i++)
                        for (int k = 0; k < ka; k++) trs[t](k, i) = loc(k, i);
                }
            }
        }
    }
#endif

    // --- state update (moist.jl:1522-1539)
    OMP_FOR
    for (int i = is; i <= ie; i++) {
        for (int k = ks; k <= ke; k++) {
            rho(k, i) = rho(k, i) + rho_p(k, i);
            rho_u(k, i) = rho_u(k, i) + rho_u_p(k, i);
            rho_theta(k, i) = rho_theta(k, i) + rho_theta_p(k, i);
        }
        for (int k = ks; k <= ke - 1; k++) rho_w(k, i) = rho_w(k, i) + rho_w_p(k, i);
    }

    // --- NaN checks (moist.jl:1542-1578)
    A2<T> chk[12] = {rho, rho_u, rho_w, rho_theta, s.rho_qv.a(), s.rho_qc.a(), s.rho_qr.a(),
                     d_rho_u_phys, d_rho_theta_phys, d_rho_qv_phys, d_rho_qc_phys, d_rho_qr_phys};
    for (int f = 0; f < 12; f++)
        for (int i = is; i <= ie; i++)
            for (int k = ks; k <= ke; k++)
                if (chk[f](k, i) != chk[f](k, i)) return f;
    return -1;
}

// ---------------------------------------------------------------- one large step (1589-1683)

template <class T, class TT>
int rk3_step(State<T>& s, const Par<T>& p) {
    const int ka = p.ka, ia = p.ia, ks = p.ks;
    const T dt = p.dt;
    if (p.do_mp) {
        cloud_microphysics(s.d_rho_qv_mp.a(), s.d_rho_qc_mp.a(), s.d_rho_qr_mp.a(),
                           s.d_rho_theta_mp.a(), s.rho.a(), s.rho_theta.a(), s.rho_qv.a(),
                           s.rho_qc.a(), s.rho_qr.a(), p);
    } else {
        std::fill(s.d_rho_qv_mp.v.begin(), s.d_rho_qv_mp.v.end(), T(0));
        std::fill(s.d_rho_qc_mp.v.begin(), s.d_rho_qc_mp.v.end(), T(0));
        std::fill(s.d_rho_qr_mp.v.begin(), s.d_rho_qr_mp.v.end(), T(0));
        std::fill(s.d_rho_theta_mp.v.begin(), s.d_rho_theta_mp.v.end(), T(0));
    }
    std::vector<T> d_prec(ia, T(0));
    if (p.do_mp && p.do_sed) {
        rain_sedimentation(s.d_rho_qr_sed.a(), d_prec.data(), s.rho_qr.a(), s.rho.a(), p);
    } else {
        std::fill(s.d_rho_qr_sed.v.begin(), s.d_rho_qr_sed.v.end(), T(0));
    }
    if (p.do_sf) {
        surface_fluxes(s.d_rho_u_sf.data(), s.d_rho_theta_sf.data(), s.d_rho_qv_sf.data(),
                       s.mflux.data(), s.shflux.data(), s.lhflux.data(), s.rho.a(), s.rho_u.a(),
                       s.rho_theta.a(), s.rho_qv.a(), s.rho_qc.a(), s.rho_qr.a(), p);
    } else {
        std::fill(s.d_rho_u_sf.begin(), s.d_rho_u_sf.end(), T(0));
        std::fill(s.d_rho_theta_sf.begin(), s.d_rho_theta_sf.end(), T(0));
        std::fill(s.d_rho_qv_sf.begin(), s.d_rho_qv_sf.end(), T(0));
        std::fill(s.mflux.begin(), s.mflux.end(), T(0));
        std::fill(s.shflux.begin(), s.shflux.end(), T(0));
        std::fill(s.lhflux.begin(), s.lhflux.end(), T(0));
    }
    if (p.do_rd) {
        gray_radiation(s.d_rho_theta_rd.a(), s.rho.a(), s.rho_theta.a(), s.rho_qv.a(), s.rho_qc.a(),
                       s.rho_qr.a(), s.theta_ref.data(), p);
    } else {
        std::fill(s.d_rho_theta_rd.v.begin(), s.d_rho_theta_rd.v.end(), T(0));
    }

    // phys tendencies (moist.jl:1633-1644)
    Field<T> d_rho_phys = s.d_rho_qr_sed;
    for (int i = 0; i < ia; i++) d_rho_phys.a()(ks, i) += s.d_rho_qv_sf[i];
    Field<T> d_rho_u_phys(ka, ia);
    for (int i = 0; i < ia; i++) d_rho_u_phys.a()(ks, i) += s.d_rho_u_sf[i];
    Field<T> d_rho_theta_phys(ka, ia);
    for (size_t j = 0; j < (size_t)ka * ia; j++)
        d_rho_theta_phys.v[j] = s.d_rho_theta_mp.v[j] + s.d_rho_theta_rd.v[j] +
                                d_rho_phys.v[j] * s.rho_theta.v[j] / s.rho.v[j];
    for (int i = 0; i < ia; i++) d_rho_theta_phys.a()(ks, i) += s.d_rho_theta_sf[i];
    Field<T> d_rho_qv_phys = s.d_rho_qv_mp;
    for (int i = 0; i < ia; i++) d_rho_qv_phys.a()(ks, i) += s.d_rho_qv_sf[i];
    Field<T> d_rho_qc_phys = s.d_rho_qc_mp;
    Field<T> d_rho_qr_phys(ka, ia);
    for (size_t j = 0; j < (size_t)ka * ia; j++)
        d_rho_qr_phys.v[j] = s.d_rho_qr_mp.v[j] + s.d_rho_qr_sed.v[j];

    State<T> s0 = s;
    int bad;
    const int ns1 = std::max(1, (int)std::ceil(p.ns / 3.0));
    bad = compute_step<T, TT>(d_rho_phys.a(), d_rho_u_phys.a(), d_rho_theta_phys.a(), d_rho_qv_phys.a(),
                              d_rho_qc_phys.a(), d_rho_qr_phys.a(), s, s0, p, dt / T(3), ns1);
    if (bad >= 0) return bad;
    const int ns2 = std::max(1, (int)std::ceil(p.ns / 2.0));
    bad = compute_step<T, TT>(d_rho_phys.a(), d_rho_u_phys.a(), d_rho_theta_phys.a(), d_rho_qv_phys.a(),
                              d_rho_qc_phys.a(), d_rho_qr_phys.a(), s, s0, p, dt / T(2), ns2);
    if (bad >= 0) return bad;
    bad = compute_step<T, TT>(d_rho_phys.a(), d_rho_u_phys.a(), d_rho_theta_phys.a(), d_rho_qv_phys.a(),
                              d_rho_qc_phys.a(), d_rho_qr_phys.a(), s, s0, p, dt, p.ns);
    if (bad >= 0) return bad;
    for (int i = p.is; i <= p.ie; i++) s.prec[i] += d_prec[i] * dt;
    return -1;
}

}  // namespace oracle
