// oracle_capi.cpp - C entry points of the CPU oracle (TEST INFRASTRUCTURE, see moist_oracle.hpp).
//
// The entry points take the same moist_params / moist_state_host structs as the CUDA library
// (include/moist2d.h) and operate directly on host arrays in the reference layout. They return
// -1 on success, the MOIST_FIELD_* index of a field found with a NaN (the reference's
// error("NaN detected in ...")), or -2 for an invalid argument.
#include <cstring>
#include <vector>

#include "moist_oracle.hpp"

using namespace oracle;

namespace {

template <class T>
void copy_in(Field<T>& f, const void* src) {
    if (src) std::memcpy(f.v.data(), src, f.v.size() * sizeof(T));
}
template <class T>
void copy_in(std::vector<T>& f, const void* src) {
    if (src) std::memcpy(f.data(), src, f.size() * sizeof(T));
}
template <class T>
void copy_out(const Field<T>& f, void* dst) {
    if (dst) std::memcpy(dst, f.v.data(), f.v.size() * sizeof(T));
}
template <class T>
void copy_out(const std::vector<T>& f, void* dst) {
    if (dst) std::memcpy(dst, f.data(), f.size() * sizeof(T));
}

template <class T>
void load(State<T>& s, const moist_state_host* h) {
    copy_in(s.rho, h->rho);
    copy_in(s.rho_u, h->rho_u);
    copy_in(s.rho_w, h->rho_w);
    copy_in(s.rho_theta, h->rho_theta);
    copy_in(s.rho_qv, h->rho_qv);
    copy_in(s.rho_qc, h->rho_qc);
    copy_in(s.rho_qr, h->rho_qr);
    copy_in(s.prec, h->prec);
    copy_in(s.mflux, h->mflux);
    copy_in(s.shflux, h->shflux);
    copy_in(s.lhflux, h->lhflux);
    copy_in(s.theta_ref, h->theta_ref);
    copy_in(s.d_rho_theta_mp, h->d_rho_theta_mp);
    copy_in(s.d_rho_qv_mp, h->d_rho_qv_mp);
    copy_in(s.d_rho_qc_mp, h->d_rho_qc_mp);
    copy_in(s.d_rho_qr_mp, h->d_rho_qr_mp);
    copy_in(s.d_rho_qr_sed, h->d_rho_qr_sed);
    copy_in(s.d_rho_u_sf, h->d_rho_u_sf);
    copy_in(s.d_rho_theta_sf, h->d_rho_theta_sf);
    copy_in(s.d_rho_qv_sf, h->d_rho_qv_sf);
    copy_in(s.d_rho_theta_rd, h->d_rho_theta_rd);
}

template <class T>
void store(const State<T>& s, moist_state_host* h) {
    copy_out(s.rho, h->rho);
    copy_out(s.rho_u, h->rho_u);
    copy_out(s.rho_w, h->rho_w);
    copy_out(s.rho_theta, h->rho_theta);
    copy_out(s.rho_qv, h->rho_qv);
    copy_out(s.rho_qc, h->rho_qc);
    copy_out(s.rho_qr, h->rho_qr);
    copy_out(s.prec, h->prec);
    copy_out(s.mflux, h->mflux);
    copy_out(s.shflux, h->shflux);
    copy_out(s.lhflux, h->lhflux);
    copy_out(s.theta_ref, h->theta_ref);
    copy_out(s.d_rho_theta_mp, h->d_rho_theta_mp);
    copy_out(s.d_rho_qv_mp, h->d_rho_qv_mp);
    copy_out(s.d_rho_qc_mp, h->d_rho_qc_mp);
    copy_out(s.d_rho_qr_mp, h->d_rho_qr_mp);
    copy_out(s.d_rho_qr_sed, h->d_rho_qr_sed);
    copy_out(s.d_rho_u_sf, h->d_rho_u_sf);
    copy_out(s.d_rho_theta_sf, h->d_rho_theta_sf);
    copy_out(s.d_rho_qv_sf, h->d_rho_qv_sf);
    copy_out(s.d_rho_theta_rd, h->d_rho_theta_rd);
}

bool params_ok(const moist_params* cp) {
    return cp && cp->nz >= 1 && cp->nx >= 1 && cp->halo >= 0 && cp->zf && cp->dz && cp->z;
}

template <class T, class TT>
int rk3_t(const moist_params* cp, moist_state_host* hs, int nsteps) {
    const Par<T> p = Par<T>::from_c(*cp);
    State<T> s(p);
    load(s, hs);
    int bad = -1;
    for (int n = 0; n < nsteps && bad < 0; n++) bad = rk3_step<T, TT>(s, p);
    store(s, hs);
    return bad;
}

template <class T, class TT>
int compute_step_t(const moist_params* cp, const void* const phys[6], moist_state_host* hs,
                   const moist_state_host* hs0, double dt, int ns) {
    const Par<T> p = Par<T>::from_c(*cp);
    State<T> s(p), s0(p);
    load(s, hs);
    load(s0, hs0);
    Field<T> ph[6];
    for (int j = 0; j < 6; j++) {
        ph[j] = Field<T>(p.ka, p.ia);
        copy_in(ph[j], phys[j]);
    }
    const int bad = compute_step<T, TT>(ph[0].a(), ph[1].a(), ph[2].a(), ph[3].a(), ph[4].a(),
                                        ph[5].a(), s, s0, p, (T)dt, ns);
    store(s, hs);
    return bad;
}

template <class T>
int sf_t(const moist_params* cp, moist_state_host* hs) {
    const Par<T> p = Par<T>::from_c(*cp);
    State<T> s(p);
    load(s, hs);
    surface_fluxes(s.d_rho_u_sf.data(), s.d_rho_theta_sf.data(), s.d_rho_qv_sf.data(), s.mflux.data(),
                   s.shflux.data(), s.lhflux.data(), s.rho.a(), s.rho_u.a(), s.rho_theta.a(), s.rho_qv.a(),
                   s.rho_qc.a(), s.rho_qr.a(), p);
    store(s, hs);
    return -1;
}

template <class T>
int rd_t(const moist_params* cp, moist_state_host* hs) {
    const Par<T> p = Par<T>::from_c(*cp);
    State<T> s(p);
    load(s, hs);
    gray_radiation(s.d_rho_theta_rd.a(), s.rho.a(), s.rho_theta.a(), s.rho_qv.a(), s.rho_qc.a(), s.rho_qr.a(),
                   s.theta_ref.data(), p);
    store(s, hs);
    return -1;
}

template <class T>
int micro_t(const moist_params* cp, moist_state_host* hs) {
    const Par<T> p = Par<T>::from_c(*cp);
    State<T> s(p);
    load(s, hs);
    cloud_microphysics(s.d_rho_qv_mp.a(), s.d_rho_qc_mp.a(), s.d_rho_qr_mp.a(), s.d_rho_theta_mp.a(),
                       s.rho.a(), s.rho_theta.a(), s.rho_qv.a(), s.rho_qc.a(), s.rho_qr.a(), p);
    store(s, hs);
    return -1;
}

template <class T>
int sed_t(const moist_params* cp, moist_state_host* hs, void* d_prec) {
    const Par<T> p = Par<T>::from_c(*cp);
    State<T> s(p);
    load(s, hs);
    std::vector<T> dp(p.ia, T(0));
    rain_sedimentation(s.d_rho_qr_sed.a(), dp.data(), s.rho_qr.a(), s.rho.a(), p);
    store(s, hs);
    copy_out(dp, d_prec);
    return -1;
}

template <class T, class TT>
int implicit_t(const moist_params* cp, void* rho_w, const void* drho_w, const void* theta,
               const void* rt2pres, double dt) {
    const Par<T> p = Par<T>::from_c(*cp);
    implicit_correction<T, TT>((T*)rho_w, (const T*)drho_w, (const T*)theta, (const T*)rt2pres,
                               (T)dt, p);
    return -1;
}

template <class T>
int helper_t(const moist_params* cp, int helper, int n, const double* in, double* out) {
    const Par<T> p = Par<T>::from_c(*cp);
    for (int j = 0; j < n; j++) {
        switch (helper) {
            case MOIST_HELPER_F2H:
                out[j] = (double)f2h((T)in[4 * j], (T)in[4 * j + 1], (T)in[4 * j + 2], (T)in[4 * j + 3]);
                break;
            case MOIST_HELPER_KOREN:
                out[j] = (double)koren_limiter((T)in[j]);
                break;
            case MOIST_HELPER_SAT_VP: {
                T es, d;
                saturation_vapor_pressure((T)in[j], p, &es, &d);
                out[2 * j] = es;
                out[2 * j + 1] = d;
                break;
            }
            case MOIST_HELPER_SAT_Q: {
                T q, d;
                saturation_specific_humidity((T)in[2 * j], (T)in[2 * j + 1], p, &q, &d);
                out[2 * j] = q;
                out[2 * j + 1] = d;
                break;
            }
            case MOIST_HELPER_EXP:
                out[j] = (double)mm::mexp((T)in[j]);
                break;
            case MOIST_HELPER_POW:
                out[j] = (double)mm::mpow((T)in[2 * j], (T)in[2 * j + 1]);
                break;
            default:
                return -2;
        }
    }
    return -1;
}

template <class T>
int flux_t(const moist_params* cp, int dir, const void* scalar_rho, const void* rho,
           const void* vel, int k, int i, double* out) {
    const Par<T> p = Par<T>::from_c(*cp);
    A2<T> sr{(T*)scalar_rho, p.ka}, r{(T*)rho, p.ka}, v{(T*)vel, p.ka};
    *out = dir == 0 ? (double)compute_limited_flux_x(sr, r, v, k, i, p)
                    : (double)compute_limited_flux_z(sr, r, v, k, i, p);
    return -1;
}

// per-cell budget terms (the GPU's k_budget, kernels.cuh): mass and water per cell times
// dz dx, the energy of output_history (moist.jl:1797-1841) formed in T times dz dx, rain per
// column times dx; all as doubles, for an exactly rounded sum in the test
template <class T>
int budget_terms_t(const moist_params* cp, const moist_state_host* hs, double* mass, double* water,
                   double* energy, double* rain) {
    const Par<T> p = Par<T>::from_c(*cp);
    State<T> s(p);
    load(s, hs);
    exchange_halo(s.rho_u.a(), p);  // u at the cell centres reads rho_u[k, i-1] (moist.jl:1799)
    auto rho = s.rho.a(), ru = s.rho_u.a(), rw = s.rho_w.a(), rt = s.rho_theta.a();
    auto rqv = s.rho_qv.a(), rqc = s.rho_qc.a(), rqr = s.rho_qr.a();
    const double dx = (double)p.dx;
    for (int k = 0; k < p.Nz; k++)
        for (int j = 0; j < p.Nx; j++) {
            const int i = p.is + j;
            const size_t o = (size_t)k * p.Nx + j;
            const double vol = (double)p.dz[k] * dx;
            mass[o] = (double)rho(k, i) * vol;
            water[o] = ((double)rqv(k, i) + (double)rqc(k, i) + (double)rqr(k, i)) * vol;
            const T rho_inv = T(1.0) / rho(k, i);
            const T theta = rt(k, i) * rho_inv;
            const T qv = rqv(k, i) * rho_inv, qc = rqc(k, i) * rho_inv, qr = rqr(k, i) * rho_inv;
            const T qt = qv + qc + qr;
            const T qd = T(1.0) - qt;
            const T r = p.Rd * qd + p.Rv * qv;
            const T cp = p.Cpd * qd + p.Cpv * qv + p.Cpl * (qc + qr);
            const T cv = cp - r;
            const T pi = mm::mpow(r * rt(k, i) / p.P0, r / cv);
            const T temp = theta * pi;
            const T u = (ru(k, i) + ru(k, i - 1)) * T(0.5) * rho_inv;
            const T w = k > 0 ? (rw(k, i) + rw(k - 1, i)) * T(0.5) * rho_inv : rw(k, i) * T(0.5) * rho_inv;
            const T eng_k = T(0.5) * rho(k, i) * (u * u + w * w);
            const T eng_p = rho(k, i) * p.GRAV * p.z[k];
            const T eng_i = rho(k, i) * (cv * temp + qv * p.Lv);
            energy[o] = (double)(eng_k + eng_p + eng_i) * vol;
        }
    for (int j = 0; j < p.Nx; j++) rain[j] = (double)s.prec[p.is + j] * dx;
    return -1;
}

// output_history's primitive variables (moist.jl:1795-1835): out[f] is a (Nz, Nx) array,
// z fastest, of u, w, theta, qv, qc, qr, pres, temp, theta_e, RH (the MOIST_DIAG_* order)
template <class T>
int history_diag_t(const moist_params* cp, const moist_state_host* hs, void* const* out) {
    const Par<T> p = Par<T>::from_c(*cp);
    State<T> s(p);
    load(s, hs);
    exchange_halo(s.rho_u.a(), p);  // moist.jl:1798
    auto rho = s.rho.a(), ru = s.rho_u.a(), rw = s.rho_w.a(), rt = s.rho_theta.a();
    auto rqv = s.rho_qv.a(), rqc = s.rho_qc.a(), rqr = s.rho_qr.a();
    T* o[10];
    for (int f = 0; f < 10; f++) o[f] = (T*)out[f];
    for (int j = 0; j < p.Nx; j++)
        for (int k = 0; k < p.Nz; k++) {
            const int i = p.is + j;
            const size_t c = (size_t)k + (size_t)p.Nz * j;
            const T rho_inv = T(1.0) / rho(k, i);
            const T theta = rt(k, i) * rho_inv;
            const T qv = rqv(k, i) * rho_inv, qc = rqc(k, i) * rho_inv, qr = rqr(k, i) * rho_inv;
            const T u = (ru(k, i) + ru(k, i - 1)) * T(0.5) * rho_inv;
            const T w = k > 0 ? (rw(k, i) + rw(k - 1, i)) * T(0.5) * rho_inv : rw(k, i) * T(0.5) * rho_inv;
            const T qt = qv + qc + qr;
            const T qd = T(1.0) - qt;
            const T r = p.Rd * qd + p.Rv * qv;
            T cp = p.Cpd * qd + p.Cpv * qv + p.Cpl * (qc + qr);
            const T cv = cp - r;
            const T pi = mm::mpow(r * rt(k, i) / p.P0, r / cv);
            const T pres = p.P0 * mm::mpow(pi, cp / r);
            const T temp = theta * pi;
            T es, d1, qsat, d2;
            saturation_vapor_pressure(temp, p, &es, &d1);
            saturation_specific_humidity(pres, es, p, &qsat, &d2);
            const T RH = qsat > T(1e-10) ? qv / qsat * T(100.0) : T(0.0);
            const T presv = rho(k, i) * qv * p.Rv * temp;
            const T presd = pres - presv;
            cp = p.Cpd * qd + p.Cpl * qt;
            const T thetae = temp * mm::mpow(presd / p.P0, -p.Rd / cp) * mm::mexp(p.Lv * qv / (cp * temp));
            const T v[10] = {u, w, theta, qv, qc, qr, pres, temp, thetae, RH};
            for (int f = 0; f < 10; f++) o[f][c] = v[f];
        }
    return -1;
}

}  // namespace

extern "C" {

int oracle_history_diag(const moist_params* cp, int prec, const moist_state_host* s, void* const* out) {
    if (!params_ok(cp) || !s || !out) return -2;
    return prec == MOIST_F32 ? history_diag_t<float>(cp, s, out) : history_diag_t<double>(cp, s, out);
}

int oracle_budget_terms(const moist_params* cp, int prec, const moist_state_host* s, double* mass, double* water,
                        double* energy, double* rain) {
    if (!params_ok(cp) || !s || !mass || !water || !energy || !rain) return -2;
    return prec == MOIST_F32 ? budget_terms_t<float>(cp, s, mass, water, energy, rain)
                             : budget_terms_t<double>(cp, s, mass, water, energy, rain);
}


int oracle_rk3_step(const moist_params* cp, int prec, int tri64, moist_state_host* s, int nsteps) {
    if (!params_ok(cp) || !s) return -2;
    if (prec == MOIST_F32)
        return tri64 ? rk3_t<float, double>(cp, s, nsteps) : rk3_t<float, float>(cp, s, nsteps);
    return rk3_t<double, double>(cp, s, nsteps);
}

int oracle_compute_step(const moist_params* cp, int prec, int tri64, const void* const phys[6],
                        moist_state_host* s, const moist_state_host* s0, double dt, int ns) {
    if (!params_ok(cp) || !s || !s0 || !phys) return -2;
    if (prec == MOIST_F32)
        return tri64 ? compute_step_t<float, double>(cp, phys, s, s0, dt, ns)
                     : compute_step_t<float, float>(cp, phys, s, s0, dt, ns);
    return compute_step_t<double, double>(cp, phys, s, s0, dt, ns);
}

int oracle_cloud_microphysics(const moist_params* cp, int prec, moist_state_host* s) {
    if (!params_ok(cp) || !s) return -2;
    return prec == MOIST_F32 ? micro_t<float>(cp, s) : micro_t<double>(cp, s);
}

int oracle_surface_fluxes(const moist_params* cp, int prec, moist_state_host* s) {
    if (!params_ok(cp) || !s || cp->halo < 1) return -2;
    return prec == MOIST_F32 ? sf_t<float>(cp, s) : sf_t<double>(cp, s);
}

int oracle_gray_radiation(const moist_params* cp, int prec, moist_state_host* s) {
    if (!params_ok(cp) || !s) return -2;
    return prec == MOIST_F32 ? rd_t<float>(cp, s) : rd_t<double>(cp, s);
}

int oracle_rain_sedimentation(const moist_params* cp, int prec, moist_state_host* s, void* d_prec) {
    if (!params_ok(cp) || !s) return -2;
    return prec == MOIST_F32 ? sed_t<float>(cp, s, d_prec) : sed_t<double>(cp, s, d_prec);
}

int oracle_implicit_correction(const moist_params* cp, int prec, int tri64, void* rho_w,
                               const void* drho_w, const void* theta, const void* rt2pres,
                               double dt) {
    if (!params_ok(cp) || cp->nz < 2) return -2;
    if (prec == MOIST_F32)
        return tri64 ? implicit_t<float, double>(cp, rho_w, drho_w, theta, rt2pres, dt)
                     : implicit_t<float, float>(cp, rho_w, drho_w, theta, rt2pres, dt);
    return implicit_t<double, double>(cp, rho_w, drho_w, theta, rt2pres, dt);
}

int oracle_eval_helper(const moist_params* cp, int prec, int helper, int n, const double* in,
                       double* out) {
    if (!params_ok(cp)) return -2;
    return prec == MOIST_F32 ? helper_t<float>(cp, helper, n, in, out)
                             : helper_t<double>(cp, helper, n, in, out);
}

// compute_limited_flux_x (dir 0) / compute_limited_flux_z (dir 1) at 0-based (k, i) of
// (nz, nx + 2*halo) column-major arrays
int oracle_limited_flux(const moist_params* cp, int prec, int dir, const void* scalar_rho,
                        const void* rho, const void* vel, int k, int i, double* out) {
    if (!params_ok(cp)) return -2;
    return prec == MOIST_F32 ? flux_t<float>(cp, dir, scalar_rho, rho, vel, k, i, out)
                             : flux_t<double>(cp, dir, scalar_rho, rho, vel, k, i, out);
}

int oracle_exchange_halo(const moist_params* cp, int prec, void* a) {
    if (!params_ok(cp)) return -2;
    if (prec == MOIST_F32) {
        const Par<float> p = Par<float>::from_c(*cp);
        exchange_halo(A2<float>{(float*)a, p.ka}, p);
    } else {
        const Par<double> p = Par<double>::from_c(*cp);
        exchange_halo(A2<double>{(double*)a, p.ka}, p);
    }
    return -1;
}

int oracle_solve_tridiagonal(int prec, int n, void* a, void* b, void* c, void* d) {
    if (n < 1) return -2;
    if (prec == MOIST_F32)
        solve_tridiagonal<float>((float*)a, (float*)b, (float*)c, (float*)d, n);
    else
        solve_tridiagonal<double>((double*)a, (double*)b, (double*)c, (double*)d, n);
    return -1;
}

int oracle_invert_T_for_thetae(const moist_params* cp, int prec, double qt, double theta_e,
                               double p_k, double* out2) {
    if (!params_ok(cp)) return -2;
    if (prec == MOIST_F32) {
        const Par<float> p = Par<float>::from_c(*cp);
        float t, q;
        invert_T_for_thetae((float)qt, (float)theta_e, (float)p_k, p, &t, &q);
        out2[0] = t;
        out2[1] = q;
    } else {
        const Par<double> p = Par<double>::from_c(*cp);
        double t, q;
        invert_T_for_thetae(qt, theta_e, p_k, p, &t, &q);
        out2[0] = t;
        out2[1] = q;
    }
    return -1;
}

// the shared scalar math, for tests/test_math.py
double oracle_exp_d(double x) { return mm::exp_d(x); }
double oracle_log_d(double x) { return mm::log_d(x); }
double oracle_pow_d(double x, double y) { return mm::pow_d(x, y); }

}  // extern "C"
