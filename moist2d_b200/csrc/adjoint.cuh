// adjoint.cuh - discrete adjoint of the large step (moist_adjoint_run), sm_100a.
//
// The reverse sweep handles one large step at a time, last step first. For step n the forward
// step is recomputed from its stored input State with a tape (stage inputs, the perturbations
// after every acoustic substep, R_rho_theta, the time-averaged momentum fluxes, the tracer sweep
// results), then the adjoint of each RK stage runs backwards through the stage:
//   state update -> tracer sweep -> momentum-flux averages -> substeps ns_s .. 1 ->
//   perturbation start -> w-p coefficients -> slow tendencies -> face velocities -> diagnostics
// and after the first stage the physics (phys-tendency assembly, sedimentation, Kessler).
//
// Adjoint variables ("L" fields) are double whatever the state precision. The linear parts of
// the stage (perturbation updates, the tridiagonal w-p solve, the flux averages, the state
// update) are differentiated by hand. The nonlinear cell functions (Kessler, terminal velocity,
// the diagnostics, the tendencies R_rho_u, R_rho_w, R_rho_theta and the tracer cell with its
// limited fluxes) are restated below over a scalar type S with one accessor per input ("slot"),
// and their local partial derivatives come from forward-mode dual numbers (dual.cuh). The
// in-place Gauss-Seidel tracer sweep (moist.jl:1469-1518) is adjoined as a linear recurrence in
// reverse lexicographic order over the stored partials: cell (k, i) read the updated values of
// (k, i-1), (k, i-2), (k-1, i), (k-2, i), so its adjoint collects from (k, i+1), (k, i+2),
// (k+1, i), (k+2, i).
#pragma once

#include "kernels.cuh"

namespace moist {

using mm::Dual;

constexpr int ADJ_THREADS = 128;

// N device pointers, passed to a kernel by value
template <int N>
struct DP {
    double* f[N];
};
constexpr int ADJ_DUAL = 4;  // directions per dual evaluation

template <class S>
__device__ __forceinline__ DevParams<S> params_as(const DevParams<double>& q) {
    DevParams<S> p;
    p.nx = q.nx;
    p.nz = q.nz;
    p.P = q.P;
#define PC(f) p.f = S(q.f);
    PC(dx) PC(dt) PC(H) PC(nu) PC(kappa) PC(gamma_d) PC(beta) PC(zf_sponge)
    PC(EPS) PC(GRAV) PC(Rd) PC(Rv) PC(Cpd) PC(Cpv) PC(Cpl) PC(P0) PC(Lv) PC(SIGMA) PC(EPSvap)
    PC(K_auto) PC(Qc_threshold) PC(K_accr) PC(K_evap) PC(A_term) PC(B_term) PC(T0) PC(ES0) PC(A_SAT) PC(B_SAT)
    PC(Cd) PC(Ch) PC(Ce) PC(uabs_min) PC(temp_surf) PC(k_abs_qv) PC(k_abs_qc) PC(k_abs_qr) PC(surf_emissivity)
    PC(tau_cooling) PC(z_trop)
#undef PC
    p.do_mp = q.do_mp;
    p.do_auto = q.do_auto;
    p.do_accr = q.do_accr;
    p.do_revap = q.do_revap;
    p.do_sed = q.do_sed;
    p.do_rd = q.do_rd;
    p.do_sf = q.do_sf;
    p.dz = nullptr;
    p.z = nullptr;
    p.zf = nullptr;
    return p;
}

// Partial derivatives of f with respect to its NS slots, N directions per evaluation:
// emit(s, df/dslot_s) for every slot with use[s]. val[s] holds the slot values; f(get) is the
// cell function, get(s) returns slot s as a Dual<N> seeded in direction s - s0 of the pass.
template <int N, int NS, class F, class E>
__device__ __forceinline__ void local_jacobian(const double (&val)[NS], F f, E emit) {
#pragma unroll
    for (int s0 = 0; s0 < NS; s0 += N) {
        auto get = [&](int s) {
            Dual<N> d(val[s]);
#pragma unroll
            for (int q = 0; q < N; q++) d.d[q] = (s - s0 == q) ? 1.0 : 0.0;
            return d;
        };
        const Dual<N> r = f(get);
#pragma unroll
        for (int q = 0; q < N; q++)
            if (s0 + q < NS) emit(s0 + q, r.d[q]);
    }
}

// ----------------------------------------------------------------------------- restated cells

// R_rho_u at (k, i) without d_rho_u_phys (moist.jl:1098-1178). Slots:
//  0-2 rho_u (k,i-1) (k,i) (k,i+1); 3-6 rho_w (k,i) (k,i+1) (k-1,i) (k-1,i+1);
//  7-11 u_face (k,i-2..i+2); 12-15 u_face (k-2,i) (k-1,i) (k+1,i) (k+2,i);
//  16-21 rho (k,i) (k,i+1) (k-1,i) (k-1,i+1) (k+1,i) (k+1,i+1); 22-23 pres (k,i) (k,i+1)
template <class S, class G>
__device__ __forceinline__ S gen_R_u(const DevParams<double>& p, int k, const G& v) {
    const int ke = p.nz - 1;
    const S EPS = p.EPS, dx = p.dx;
    const double* dz = p.dz;
    const double* z = p.z;
    const S rho_u_ip = S(0.5) * (v(1) + v(2));
    S f_ip;
    if (rho_u_ip > EPS)
        f_ip = up3(rho_u_ip, v(8), v(9), v(10));
    else if (rho_u_ip < -EPS)
        f_ip = up3(rho_u_ip, v(11), v(10), v(9));
    else
        f_ip = rho_u_ip * (v(9) + v(10)) * S(0.5);
    const S rho_u_im = S(0.5) * (v(0) + v(1));
    S f_im;
    if (rho_u_im > EPS)
        f_im = up3(rho_u_im, v(7), v(8), v(9));
    else if (rho_u_im < -EPS)
        f_im = up3(rho_u_im, v(10), v(9), v(8));
    else
        f_im = rho_u_im * (v(8) + v(9)) * S(0.5);
    const S druudx = (f_ip - f_im) / dx;
    S f_kp = S(0.0);
    if (k < ke) {
        const S rho_w_kp = S(0.5) * (v(3) + v(4));
        if (rho_w_kp > EPS && k > 0)
            f_kp = up3(rho_w_kp, v(13), v(9), v(14));
        else if (rho_w_kp < -EPS && k < ke - 1)
            f_kp = up3(rho_w_kp, v(15), v(14), v(9));
        else
            f_kp = rho_w_kp * f2h(v(9), v(14), S(dz[k]), S(dz[k + 1]));
    }
    S f_km = S(0.0);
    if (k > 0) {
        const S rho_w_km = S(0.5) * (v(5) + v(6));
        if (rho_w_km > EPS && k > 1)
            f_km = up3(rho_w_km, v(12), v(13), v(9));
        else if (rho_w_km < -EPS && k < ke)
            f_km = up3(rho_w_km, v(14), v(9), v(13));
        else
            f_km = rho_w_km * f2h(v(13), v(9), S(dz[k - 1]), S(dz[k]));
    }
    const S drwudz = (f_kp - f_km) / S(dz[k]);
    const S advection = -druudx - drwudz;
    const S u_ip = (v(10) - v(9)) / dx;
    const S u_im = (v(9) - v(8)) / dx;
    const S u_xx = (u_ip * v(17) - u_im * v(16)) / dx;
    const S u_kp = k == ke ? S(0.0) : (v(14) - v(9)) / S(z[k + 1] - z[k]);
    const S u_km = k == 0 ? S(0.0) : (v(9) - v(13)) / S(z[k] - z[k - 1]);
    const S rho_kp = k == ke ? S(0.0) : S(0.25) * (v(16) + v(20) + v(17) + v(21));
    const S rho_km = k == 0 ? S(0.0) : S(0.25) * (v(18) + v(16) + v(19) + v(17));
    const S u_zz = (u_kp * rho_kp - u_km * rho_km) / S(dz[k]);
    const S diffusion = S(p.nu) * (u_xx + u_zz);
    const S dpdx = (v(23) - v(22)) / dx;
    return advection - dpdx + diffusion;
}

// R_rho_w at (k, i), k < nz-1 (moist.jl:1190-1278). Slots:
//  0-3 rho_u (k,i) (k+1,i) (k,i-1) (k+1,i-1); 4-6 rho_w (k-1,i) (k,i) (k+1,i);
//  7-11 w_face (k,i-2..i+2); 12-15 w_face (k-2,i) (k-1,i) (k+1,i) (k+2,i);
//  16-21 rho (k,i) (k+1,i) (k,i-1) (k+1,i-1) (k,i+1) (k+1,i+1); 22-23 pres (k,i) (k+1,i)
template <class S, class G>
__device__ __forceinline__ S gen_R_w(const DevParams<double>& p, int k, const G& v) {
    const int ke = p.nz - 1;
    const S EPS = p.EPS, dx = p.dx;
    const double* dz = p.dz;
    const double* z = p.z;
    const S rho_u_ip = f2h(v(0), v(1), S(z[k]), S(z[k + 1]));  // z weights, as written (1196)
    S f_ip;
    if (rho_u_ip > EPS)
        f_ip = up3(rho_u_ip, v(8), v(9), v(10));
    else if (rho_u_ip < -EPS)
        f_ip = up3(rho_u_ip, v(11), v(10), v(9));
    else
        f_ip = rho_u_ip * (v(9) + v(10)) * S(0.5);
    const S rho_u_im = f2h(v(2), v(3), S(dz[k]), S(dz[k + 1]));
    S f_im;
    if (rho_u_im > EPS)
        f_im = up3(rho_u_im, v(7), v(8), v(9));
    else if (rho_u_im < -EPS)
        f_im = up3(rho_u_im, v(10), v(9), v(8));
    else
        f_im = rho_u_im * (v(8) + v(9)) * S(0.5);
    const S drwudx = (f_ip - f_im) / dx;
    S f_kp = S(0.0);
    if (k < ke - 1) {
        const S rho_w_kp = f2h(v(5), v(6), S(dz[k]), S(dz[k + 1]));
        if (rho_w_kp > EPS && k > 0)
            f_kp = up3(rho_w_kp, v(13), v(9), v(14));
        else if (rho_w_kp < -EPS && k < ke - 2)
            f_kp = up3(rho_w_kp, v(15), v(14), v(9));
        else
            f_kp = rho_w_kp * f2h(v(9), v(14), S(dz[k]), S(dz[k + 1]));
    }
    S f_km = S(0.0);
    if (k > 0) {
        const S rho_w_km = f2h(v(4), v(5), S(dz[k - 1]), S(dz[k]));
        if (rho_w_km > EPS && k > 1)
            f_km = up3(rho_w_km, v(12), v(13), v(9));
        else if (rho_w_km < -EPS && k < ke - 1)
            f_km = up3(rho_w_km, v(14), v(9), v(13));
        else
            f_km = rho_w_km * f2h(v(13), v(9), S(dz[k - 1]), S(dz[k]));
    }
    const S dzc = S(z[k + 1] - z[k]);
    const S drwwdz = (f_kp - f_km) / dzc;
    const S advection = -drwudx - drwwdz;
    const S w_ip = (v(10) - v(9)) / dx;
    const S w_im = (v(9) - v(8)) / dx;
    const S rho_ip = S(0.25) * (v(16) + v(17) + v(20) + v(21));
    const S rho_im = S(0.25) * (v(18) + v(19) + v(16) + v(17));
    const S w_xx = (w_ip * rho_ip - w_im * rho_im) / dx;
    const S w_kp = k == ke - 1 ? S(0.0) : (v(14) - v(9)) / S(dz[k + 1]);
    const S w_km = k == 0 ? S(0.0) : (v(9) - v(13)) / S(dz[k]);
    const S w_zz = (w_kp * v(17) - w_km * v(16)) / dzc;
    const S diffusion = S(p.nu) * (w_xx + w_zz);
    double sigma = 0.0;
    const double zfk = p.zf[k];
    if (zfk > (1.0 - p.zf_sponge) * p.H)
        sigma = (p.GRAV / 30.0) * ((zfk - (1.0 - p.zf_sponge) * p.H) / (p.zf_sponge * p.H));
    const S sponge = S(-sigma) * v(5);
    const S dpdz = (v(23) - v(22)) / dzc;
    const S buoyancy = S(-p.GRAV) * (v(16) + v(17)) * S(0.5);
    return advection - dpdz + buoyancy + diffusion + sponge;
}

// R_rho_theta at (k, i) without d_rho_theta_phys (moist.jl:1284-1331). Slots:
//  0-1 rho_u (k,i) (k,i-1); 2-3 rho_w (k,i) (k-1,i); 4-8 theta (k,i-2..i+2);
//  9-12 theta (k-2,i) (k-1,i) (k+1,i) (k+2,i)
template <class S, class G>
__device__ __forceinline__ S gen_R_t(const DevParams<double>& p, int k, const G& v) {
    const int ke = p.nz - 1;
    const S EPS = p.EPS, dx = p.dx;
    const double* dz = p.dz;
    const S ru_i = v(0), ru_m = v(1);
    S f_ip, f_im, f_kp = S(0.0), f_km = S(0.0);
    if (ru_i > EPS)
        f_ip = up3(ru_i, v(5), v(6), v(7));
    else if (ru_i < -EPS)
        f_ip = up3(ru_i, v(8), v(7), v(6));
    else
        f_ip = ru_i * (v(6) + v(7)) * S(0.5);
    if (ru_m > EPS)
        f_im = up3(ru_m, v(4), v(5), v(6));
    else if (ru_m < -EPS)
        f_im = up3(ru_m, v(7), v(6), v(5));
    else
        f_im = ru_m * (v(5) + v(6)) * S(0.5);
    if (k < ke) {
        const S w = v(2);
        if (w > EPS && k > 0)
            f_kp = up3(w, v(10), v(6), v(11));
        else if (w < -EPS && k < ke - 1)
            f_kp = up3(w, v(12), v(11), v(6));
        else
            f_kp = w * f2h(v(6), v(11), S(dz[k]), S(dz[k + 1]));
    }
    if (k > 0) {
        const S w = v(3);
        if (w > EPS && k > 1)
            f_km = up3(w, v(9), v(10), v(6));
        else if (w < -EPS && k < ke)
            f_km = up3(w, v(11), v(6), v(10));
        else
            f_km = w * f2h(v(10), v(6), S(dz[k - 1]), S(dz[k]));
    }
    return -((f_ip - f_im) / dx + (f_kp - f_km) / S(dz[k]));
}

// The tracer update of one cell (moist.jl:1479-1515) as a function of its reads. Slots:
//  0-8 rho_q at C (k,i), L1 (k,i-1), L2 (k,i-2), R1 (k,i+1), R2 (k,i+2), B1 (k-1,i), B2 (k-2,i),
//      U1 (k+1,i), U2 (k+2,i); 9-10 the linear-index clamp reads rho_q[1, 1] and rho_q[nz, 1]
//      (row 0 and row nz-1 of reference column 1); 11-19 rho at the same nine positions;
//  20-21 mom_flux_x (k,i) (k,i-1); 22-23 mom_flux_z (k,i) (k-1,i)
// The update is q0 + dt (-(adv_x + adv_z) + (diff_x + diff_z) + dph): its x half (adv_x,
// diff_x) reads the slots TR_X, its z half (adv_z, diff_z) the slots TR_Z; only C and rho_C
// are in both.
constexpr int TR_SLOTS = 24;
constexpr int TR_NX = 12, TR_NZ = 14;
__device__ constexpr int TR_X[TR_NX] = {0, 1, 2, 3, 4, 11, 12, 13, 14, 15, 20, 21};
__device__ constexpr int TR_Z[TR_NZ] = {0, 5, 6, 7, 8, 9, 10, 11, 16, 17, 18, 19, 22, 23};

template <class S, class G>
__device__ __forceinline__ void gen_tracer_x(const DevParams<double>& p, const G& v, S& adv_x, S& diff_x) {
    const S EPS = p.EPS, dx = p.dx;
    const S s_c = v(0) / v(11);
    const S s_im1 = v(1) / v(12);
    const S s_im2 = v(2) / v(13);
    const S s_ip1 = v(3) / v(14);
    const S s_ip2 = v(4) / v(15);
    const S fx_ip = limited_flux_x(v(20), s_im1, s_c, s_ip1, s_ip2, EPS);
    const S fx_im = limited_flux_x(v(21), s_im2, s_im1, s_c, s_ip1, EPS);
    adv_x = (fx_ip - fx_im) / dx;
    const S r_c = v(11);
    const S dsdx_ip = (v(14) + r_c) * S(0.5) * (s_ip1 - s_c) / dx;
    const S dsdx_im = (r_c + v(12)) * S(0.5) * (s_c - s_im1) / dx;
    diff_x = S(p.kappa) * (dsdx_ip - dsdx_im) / dx;
}

// limited_flux_z (model.cuh) with its clamp quotient formed only on the two faces that can
// select it (kk = 0 upward, kk = nz-2 downward); the selected operations are the same
template <class S>
__device__ __forceinline__ S gen_flux_z(S vel, S s_m1, S s_0, S s_p1, S s_p2, int kk, int nz, S dz_k, S dz_kp1,
                                        S lin_k, S lin_kp1, S dt_big, S EPS) {
    const bool pos = vel > EPS, neg = vel < -EPS;
    const S f2 = f2h(s_0, s_p1, dz_k, dz_kp1);
    const bool use_clamp = (pos && kk == 0) || (!pos && neg && kk == nz - 2);
    S face;
    if (use_clamp) {
        face = jmin(f2, (pos ? lin_k : lin_kp1) / (pos ? (vel * dt_big) : (-vel * dt_big)));
    } else if (pos || neg) {
        const S r_num = pos ? (s_p1 - s_0) : (s_0 - s_p1);
        const S r_den = pos ? (s_0 - s_m1) : (s_p1 - s_p2);
        const S q = r_num / r_den;
        const S r = mm::mabs(r_den) < EPS ? S(1.0) : q;
        const S half = S(0.5) * koren(r) * r_den;
        face = pos ? (s_0 + half) : (s_p1 - half);
    } else {
        face = f2;
    }
    return face * vel;
}

template <class S, class G>
__device__ __forceinline__ void gen_tracer_z(const DevParams<double>& p, int k, const G& v, S& adv_z, S& diff_z) {
    const int nz = p.nz, ke = nz - 1;
    const S EPS = p.EPS, dtb = p.dt;
    const double* dz = p.dz;
    const double* z = p.z;
    const S s_c = v(0) / v(11);
    const S s_km1 = k >= 1 ? v(5) / v(16) : S(0.0);
    const S s_km2 = k >= 2 ? v(6) / v(17) : S(0.0);
    const S s_kp1 = k + 1 < nz ? v(7) / v(18) : S(0.0);
    const S s_kp2 = k + 2 < nz ? v(8) / v(19) : S(0.0);
    S fz_kp = S(0.0), fz_km = S(0.0);
    if (k < ke)
        fz_kp = gen_flux_z(v(22), s_km1, s_c, s_kp1, s_kp2, k, nz, S(dz[k]), S(dz[k + 1]), v(9), v(10), dtb, EPS);
    if (k > 0)
        fz_km = gen_flux_z(v(23), s_km2, s_km1, s_c, s_kp1, k - 1, nz, S(dz[k - 1]), S(dz[k]), v(9), v(10), dtb, EPS);
    adv_z = (fz_kp - fz_km) / S(dz[k]);
    const S r_c = v(11);
    const S scalar_kp = k == ke ? S(0.0) : s_kp1;
    const S scalar_km = k == 0 ? S(0.0) : s_km1;
    const S dsdz_kp = k == ke ? S(0.0)
                              : f2h(v(18), r_c, S(dz[k + 1]), S(dz[k])) * (scalar_kp - s_c) / S(z[k + 1] - z[k]);
    const S dsdz_km = k == 0 ? S(0.0)
                             : f2h(r_c, v(16), S(dz[k]), S(dz[k - 1])) * (s_c - scalar_km) / S(z[k] - z[k - 1]);
    diff_z = S(p.kappa) * (dsdz_kp - dsdz_km) / S(dz[k]);
}

// Partial derivatives of the two outputs (a, b) of f with respect to the NS slots sl, N
// directions per evaluation: emit(slot, da/dslot, db/dslot). f(get, a, b) evaluates the function;
// get(s) returns slot s as a Dual<N> seeded in its direction of the pass (0 when not in it).
template <int N, int NS, class F, class E>
__device__ __forceinline__ void local_jacobian2(const double (&val)[TR_SLOTS], const int (&sl)[NS], F f, E emit) {
#pragma unroll
    for (int s0 = 0; s0 < NS; s0 += N) {
        auto get = [&](int s) {
            Dual<N> d(val[s]);
#pragma unroll
            for (int q = 0; q < N; q++) d.d[q] = (s0 + q < NS && sl[s0 + q] == s) ? 1.0 : 0.0;
            return d;
        };
        Dual<N> a, b;
        f(get, a, b);
#pragma unroll
        for (int q = 0; q < N; q++)
            if (s0 + q < NS) emit(sl[s0 + q], a.d[q], b.d[q]);
    }
}

// diagnostics pres, theta, rt2pres of one cell (moist.jl:1048-1062). Slots: rho, rho_theta,
// rho_qv, rho_qc, rho_qr; out = 0 pres, 1 theta, 2 rt2pres
template <class S, class G>
__device__ __forceinline__ S gen_diag(const DevParams<double>& p, int out, const G& v) {
    const S rho = v(0), rt = v(1);
    const S qv = v(2) / rho, qc = v(3) / rho, qr = v(4) / rho;
    const S qd = S(1.0) - qv - qc - qr;
    const S r = S(p.Rd) * qd + S(p.Rv) * qv;
    const S cp = S(p.Cpd) * qd + S(p.Cpv) * qv + S(p.Cpl) * (qc + qr);
    const S cv = cp - r;
    const S pr = S(p.P0) * mm::mpow(r * rt / S(p.P0), cp / cv);
    if (out == 0) return pr;
    if (out == 1) return rt / rho;
    return cp / cv * pr / rt;
}

// ----------------------------------------------------------------------------- kernel arguments

template <class T>
struct AdjStage {
    // forward values of the stage (state precision)
    StateP<T> s;                 // stage input
    const T *theta, *rt2, *pres, *uf, *wf;
    const T* rrt;                // R_rho_theta
    const T *mfx, *mfz;          // momentum fluxes after the substeps
    const T* qout[3];            // tracer sweep results
    const T* q0[3];              // s0 tracers
    double dt_stage, dt_s;
    int m;                       // substeps of the stage
    double fact_tp64, fact;      // 0.5 (1 + beta) in double; fact_tm / fact_tp
    // adjoint fields of the stage
    double* Lst[7];              // lambda of the stage input state (rho, ru, rw, rt, qv, qc, qr)
    double* LS0[7];              // lambda of s0 (= the step's input State)
    double* Lph[5];              // lambda of d_rho_phys, d_rho_theta_phys, d_rho_q{v,c,r}_phys
    double *LRrho, *LRu, *LRw, *LRt;
    double *Ltheta, *Lrt2, *Lpres, *Luf, *Lwf;
    double *La, *Lb, *Lc;        // lambda of the w-p coefficients a, b, c
    double *Lmfx, *Lmfz;
    double* Lpend[2];            // pending lambda of rho_theta_p_old
    double* Lqout[3];
    double *Ta, *Tb, *Tc;        // w-p coefficients (double)
    double *Tcp, *Trd;           // elimination of the transposed system: modified super-diagonal, 1 / pivot
    double *Lx, *Ly;             // right-hand side and solution of the transposed solve
    double *Ltp_rho, *Ltp_rt, *Linc_rho, *Linc_rt;
};

template <class T>
struct AdjSub {
    const T *prev_rt, *prev_rw;  // rho_theta_p, rho_w_p at the start of the substep
    const T* old_rt;             // rho_theta_p_old of the substep
    const T *ru, *rw;            // rho_u_p, rho_w_p after the substep
    double* LPn[4];              // lambda of the substep's results (rho_p, ru_p, rw_p, rt_p)
    double* LPo[4];              // lambda of its inputs
    int n;                       // substep number (1-based)
};

#define ADJ_CELL(k, i)                                                  \
    const int i = bid_x * blockDim.x + threadIdx.x;                     \
    const int k = bid_y;                                                \
    const int nx = p.nx, nz = p.nz, P = p.P;                            \
    if (i >= nx || k >= nz) return;                                     \
    const size_t c = MOIST_IDX(k, i);                                   \
    (void)c;

__device__ __forceinline__ void aadd(double* a, double v) { atomicAdd(a, v); }

// ----------------------------------------------------------------------------- stage prologue

// w-p coefficients a, b, c of implicit_correction! (moist.jl:982-1008) in double, per cell
template <class T>
__device__ __forceinline__ void b_adj_tri_coef(const DevParams<double>& p, const AdjStage<T>& a, int bid_x, int bid_y,
                                               int bid_z) {
    ADJ_CELL(k, i);
    const int ke = nz - 1, n = nz - 1;
    if (k >= n) return;
    const double* dz = p.dz;
    const double* z = p.z;
    const double fact_tp = 0.5 * (1.0 + p.beta);
    const double C = (a.dt_s * fact_tp) * (a.dt_s * fact_tp);
    auto TH = [&](int kk) { return (double)a.theta[MOIST_IDX(kk, i)]; };
    auto thh = [&](int kk) { return f2h(TH(kk), TH(kk + 1), dz[kk], dz[kk + 1]); };
    const double r_k = a.rt2[c], r_kp = a.rt2[c + P];
    const double dzc = z[k + 1] - z[k];
    a.Tb[c] = C * (r_k / dz[k] + r_kp / dz[k + 1]) * thh(k) / dzc;
    a.Ta[c] = k > 0 ? -C * (r_k * thh(k - 1) / (dzc * dz[k]) - p.GRAV / (dz[k] + dz[k + 1])) : 0.0;
    a.Tc[c] = k < ke - 1 ? -C * (r_kp * thh(k + 1) / (dzc * dz[k + 1]) + p.GRAV / (dz[k] + dz[k + 1])) : 0.0;
}
template <class T>
__global__ void k_adj_tri_coef(const __grid_constant__ DevParams<double> p, const __grid_constant__ AdjStage<T> a) {
    b_adj_tri_coef(p, a, blockIdx.x, blockIdx.y, blockIdx.z);
}

// elimination of the transposed system A^T (sub-diagonal c_{j-1}, diagonal b_j + 1,
// super-diagonal a_{j+1}), once per stage and column: modified super-diagonal and 1 / pivot
__device__ __forceinline__ void b_adj_tri_fact(int nx, int nz, int P, const double* __restrict__ Ta,
                                               const double* __restrict__ Tb, const double* __restrict__ Tc,
                                               double* __restrict__ Tcp, double* __restrict__ Trd, int bid_x, int bid_y,
                                               int bid_z) {
    const int i = bid_x * blockDim.x + threadIdx.x;
    if (i >= nx) return;
    const int n = nz - 1;
    double cp = 0.0;
    for (int j = 0; j < n; j++) {
        const size_t cj = MOIST_IDX(j, i);
        const double sub = j > 0 ? Tc[cj - P] : 0.0;
        const double rd = 1.0 / (Tb[cj] + 1.0 - sub * cp);
        cp = (j < n - 1 ? Ta[cj + P] : 0.0) * rd;
        Tcp[cj] = cp;
        Trd[cj] = rd;
    }
}
__global__ void k_adj_tri_fact(int nx, int nz, int P, const double* __restrict__ Ta, const double* __restrict__ Tb,
                               const double* __restrict__ Tc, double* __restrict__ Tcp, double* __restrict__ Trd) {
    b_adj_tri_fact(nx, nz, P, Ta, Tb, Tc, Tcp, Trd, blockIdx.x, blockIdx.y, blockIdx.z);
}

// adjoint of the state update (moist.jl:1522-1539): the stage output's lambda goes to the
// stage input (already in Lst) and to the last perturbations; the tracers' lambda moves to
// the sweep results
template <class T>
__device__ __forceinline__ void b_adj_update(const DevParams<double>& p, const AdjStage<T>& a, const DP<4>& LP,
                                             int bid_x, int bid_y, int bid_z) {
    ADJ_CELL(k, i);
    LP.f[0][c] = a.Lst[0][c];
    LP.f[1][c] = a.Lst[1][c];
    LP.f[2][c] = k < nz - 1 ? a.Lst[2][c] : 0.0;
    LP.f[3][c] = a.Lst[3][c];
    for (int t = 0; t < 3; t++) {
        a.Lqout[t][c] = a.Lst[4 + t][c];
        a.Lst[4 + t][c] = 0.0;
    }
}
template <class T>
__global__ void k_adj_update(const __grid_constant__ DevParams<double> p, const __grid_constant__ AdjStage<T> a,
                             const __grid_constant__ DP<4> LP) {
    b_adj_update(p, a, LP, blockIdx.x, blockIdx.y, blockIdx.z);
}

// ----------------------------------------------------------------------------- tracer sweep

// the reads of tracer cell (k, i) from the sweep's stage-start ("old") and result ("new")
// arrays: new values at (k, i-1), (k, i-2) unless they wrap around (periodic halo copies of the
// stage start), new values below, old values at the cell, right and above
template <class T>
__device__ __forceinline__ void tracer_slots(const DevParams<double>& p, const AdjStage<T>& a, int t, int k, int i,
                                             double (&v)[TR_SLOTS]) {
    const int nx = p.nx, nz = p.nz, P = p.P;
    const T* qo = a.s.qv;
    if (t == 1) qo = a.s.qc;
    if (t == 2) qo = a.s.qr;
    const T* qn = a.qout[t];
    const T* rho = a.s.rho;
    const int im = wrapx(i - 1, nx), im2 = wrapx(i - 2, nx), ip = wrapx(i + 1, nx), ip2 = wrapx(i + 2, nx);
    const int hcol = nx - 2;
    v[0] = qo[MOIST_IDX(k, i)];
    v[1] = i >= 1 ? qn[MOIST_IDX(k, im)] : qo[MOIST_IDX(k, im)];
    v[2] = i >= 2 ? qn[MOIST_IDX(k, im2)] : qo[MOIST_IDX(k, im2)];
    v[3] = qo[MOIST_IDX(k, ip)];
    v[4] = qo[MOIST_IDX(k, ip2)];
    v[5] = k >= 1 ? qn[MOIST_IDX(k - 1, i)] : 0.0;
    v[6] = k >= 2 ? qn[MOIST_IDX(k - 2, i)] : 0.0;
    v[7] = k + 1 < nz ? qo[MOIST_IDX(k + 1, i)] : 0.0;
    v[8] = k + 2 < nz ? qo[MOIST_IDX(k + 2, i)] : 0.0;
    v[9] = qo[MOIST_IDX(0, hcol)];
    v[10] = qo[MOIST_IDX(nz - 1, hcol)];
    v[11] = rho[MOIST_IDX(k, i)];
    v[12] = rho[MOIST_IDX(k, im)];
    v[13] = rho[MOIST_IDX(k, im2)];
    v[14] = rho[MOIST_IDX(k, ip)];
    v[15] = rho[MOIST_IDX(k, ip2)];
    v[16] = k >= 1 ? rho[MOIST_IDX(k - 1, i)] : 1.0;
    v[17] = k >= 2 ? rho[MOIST_IDX(k - 2, i)] : 1.0;
    v[18] = k + 1 < nz ? rho[MOIST_IDX(k + 1, i)] : 1.0;
    v[19] = k + 2 < nz ? rho[MOIST_IDX(k + 2, i)] : 1.0;
    v[20] = a.mfx[MOIST_IDX(k, i)];
    v[21] = a.mfx[MOIST_IDX(k, im)];
    v[22] = k < nz - 1 ? a.mfz[MOIST_IDX(k, i)] : 0.0;
    v[23] = k >= 1 ? a.mfz[MOIST_IDX(k - 1, i)] : 0.0;
}

// partial derivatives of every tracer cell with respect to its 24 reads: J[t][slot][cell]
template <class T>
__device__ __forceinline__ void b_adj_tr_jac(const DevParams<double>& p, const AdjStage<T>& a, double* J, int bid_x,
                                             int bid_y, int bid_z) {
    ADJ_CELL(k, i);
    const int t = bid_z;
    double v[TR_SLOTS];
    tracer_slots(p, a, t, k, i, v);
    const size_t fsz = (size_t)nz * P;
    double* Jt = J + (size_t)t * TR_SLOTS * fsz;
    // dq/dslot = dt (-(d adv_x + d adv_z) + (d diff_x + d diff_z)); slots C and rho_C take both
    // halves, the others one
    const double dt = a.dt_stage;
    double ax_c = 0.0, dx_c = 0.0, ax_r = 0.0, dx_r = 0.0;
    using D = Dual<ADJ_DUAL>;
    local_jacobian2<ADJ_DUAL>(
        v, TR_X, [&](const auto& get, D& ax, D& dfx) { gen_tracer_x<D>(p, get, ax, dfx); },
        [&](int s, double ax, double dfx) {
            if (s == 0) {
                ax_c = ax;
                dx_c = dfx;
            } else if (s == 11) {
                ax_r = ax;
                dx_r = dfx;
            } else {
                Jt[(size_t)s * fsz + c] = dt * (-ax + dfx);
            }
        });
    local_jacobian2<ADJ_DUAL>(
        v, TR_Z, [&](const auto& get, D& az, D& dfz) { gen_tracer_z<D>(p, k, get, az, dfz); },
        [&](int s, double az, double dfz) {
            const double ax = s == 0 ? ax_c : (s == 11 ? ax_r : 0.0);
            const double dfx = s == 0 ? dx_c : (s == 11 ? dx_r : 0.0);
            Jt[(size_t)s * fsz + c] = dt * (-(ax + az) + (dfx + dfz));
        });
}
template <class T>
__global__ void __launch_bounds__(ADJ_THREADS) k_adj_tr_jac(const __grid_constant__ DevParams<double> p,
                                  const __grid_constant__ AdjStage<T> a, double* J) {
    b_adj_tr_jac(p, a, J, blockIdx.x, blockIdx.y, blockIdx.z);
}

// reverse sweep: mu(k,i) = lambda_new(k,i) + sum over the later cells that read the new value
// of (k, i): (k, i+1) [slot L1], (k, i+2) [L2], (k+1, i) [B1], (k+2, i) [B2]. One block per
// tracer, thread k owns row k; row k handles column nx-1-(d-(nz-1-k)) at step d, after the rows
// above it, whose results come through a 3-step ring in shared memory.
__device__ __forceinline__ void b_adj_tr_rev(int nx, int nz, int P, const double* __restrict__ J, const DP<3>& lam_new,
                                             const DP<3>& mu, int bid_x, int bid_y, int bid_z) {
    extern __shared__ double ring[];  // [3][nz]
    const int t = bid_x;
    const int k = threadIdx.x;
    const size_t fsz = (size_t)nz * P;
    const double* Jt = J + (size_t)t * TR_SLOTS * fsz;
    const double* JL1 = Jt + 1 * fsz;
    const double* JL2 = Jt + 2 * fsz;
    const double* JB1 = Jt + 5 * fsz;
    const double* JB2 = Jt + 6 * fsz;
    const double* ln = lam_new.f[t];
    double* m = mu.f[t];
    const bool active = k < nz;
    double mp1 = 0.0, mp2 = 0.0;  // mu(k, i+1), mu(k, i+2)
    // the next step's inputs, loaded one step ahead (they do not depend on mu)
    double f_ln = 0.0, f_a1 = 0.0, f_a2 = 0.0, f_b1 = 0.0, f_b2 = 0.0;
    auto fetch = [&](int i) {
        const size_t cc = MOIST_IDX(k, i);
        f_ln = ln[cc];
        f_a1 = i + 1 < nx ? JL1[cc + 1] : 0.0;
        f_a2 = i + 2 < nx ? JL2[cc + 2] : 0.0;
        f_b1 = k + 1 < nz ? JB1[cc + P] : 0.0;
        f_b2 = k + 2 < nz ? JB2[cc + 2 * P] : 0.0;
        // a row walks its arrays backwards, one 128-byte line per 16 steps: ask for the line
        // 16 steps ahead into L1 so that the loads above hit
        if (i >= 16) {
            const size_t cf = cc - 16;
            asm volatile("prefetch.global.L1 [%0];" ::"l"(ln + cf));
            asm volatile("prefetch.global.L1 [%0];" ::"l"(JL1 + cf + 1));
            asm volatile("prefetch.global.L1 [%0];" ::"l"(JL2 + cf + 2));
            if (k + 1 < nz) asm volatile("prefetch.global.L1 [%0];" ::"l"(JB1 + cf + P));
            if (k + 2 < nz) asm volatile("prefetch.global.L1 [%0];" ::"l"(JB2 + cf + 2 * P));
        }
    };
    if (active) fetch(nx - 1);
    const int nsteps = nx + nz - 1;
    for (int d = 0; d < nsteps; d++) {
        const int i = nx - 1 - (d - (nz - 1 - k));
        if (active && i >= 0 && i < nx) {
            const double l = f_ln, a1 = f_a1, a2 = f_a2, b1 = f_b1, b2 = f_b2;
            if (i >= 1) fetch(i - 1);
            double v = l;
            if (i + 1 < nx) v += mp1 * a1;
            if (i + 2 < nx) v += mp2 * a2;
            if (k + 1 < nz) v += ring[((d + 2) % 3) * nz + k + 1] * b1;
            if (k + 2 < nz) v += ring[((d + 1) % 3) * nz + k + 2] * b2;
            m[MOIST_IDX(k, i)] = v;
            ring[(d % 3) * nz + k] = v;
            mp2 = mp1;
            mp1 = v;
        }
        __syncthreads();
    }
}
__global__ void k_adj_tr_rev(int nx, int nz, int P, const double* __restrict__ J, const __grid_constant__ DP<3> lam_new,
                             const __grid_constant__ DP<3> mu) {
    b_adj_tr_rev(nx, nz, P, J, lam_new, mu, blockIdx.x, blockIdx.y, blockIdx.z);
}

// the sweep's lambda contributions to everything read through "old" values, rho, the
// momentum fluxes, s0 tracers and the phys tendencies
template <class T>
__device__ __forceinline__ void b_adj_tr_scatter(const DevParams<double>& p, const AdjStage<T>& a, const double* J,
                                                 const DP<3>& mu, int bid_x, int bid_y, int bid_z) {
    ADJ_CELL(k, i);
    const int t = bid_z;
    const size_t fsz = (size_t)nz * P;
    const double* Jt = J + (size_t)t * TR_SLOTS * fsz;
    const double m = mu.f[t][c];
    if (m == 0.0) return;
    auto Jv = [&](int s) { return m * Jt[(size_t)s * fsz + c]; };
    const int im = wrapx(i - 1, nx), im2 = wrapx(i - 2, nx), ip = wrapx(i + 1, nx), ip2 = wrapx(i + 2, nx);
    const int hcol = nx - 2;
    double* Lq = a.Lst[4 + t];
    double* Lr = a.Lst[0];
    aadd(Lq + c, Jv(0));
    if (i < 1) aadd(Lq + MOIST_IDX(k, im), Jv(1));
    if (i < 2) aadd(Lq + MOIST_IDX(k, im2), Jv(2));
    aadd(Lq + MOIST_IDX(k, ip), Jv(3));
    aadd(Lq + MOIST_IDX(k, ip2), Jv(4));
    if (k + 1 < nz) aadd(Lq + c + P, Jv(7));
    if (k + 2 < nz) aadd(Lq + c + 2 * P, Jv(8));
    aadd(Lq + MOIST_IDX(0, hcol), Jv(9));
    aadd(Lq + MOIST_IDX(nz - 1, hcol), Jv(10));
    aadd(Lr + c, Jv(11));
    aadd(Lr + MOIST_IDX(k, im), Jv(12));
    aadd(Lr + MOIST_IDX(k, im2), Jv(13));
    aadd(Lr + MOIST_IDX(k, ip), Jv(14));
    aadd(Lr + MOIST_IDX(k, ip2), Jv(15));
    if (k >= 1) aadd(Lr + c - P, Jv(16));
    if (k >= 2) aadd(Lr + c - 2 * P, Jv(17));
    if (k + 1 < nz) aadd(Lr + c + P, Jv(18));
    if (k + 2 < nz) aadd(Lr + c + 2 * P, Jv(19));
    aadd(a.Lmfx + c, Jv(20));
    aadd(a.Lmfx + MOIST_IDX(k, im), Jv(21));
    if (k < nz - 1) aadd(a.Lmfz + c, Jv(22));
    if (k >= 1) aadd(a.Lmfz + c - P, Jv(23));
    // rho_q = rho_q0 + dt (... + d_phys)
    aadd(a.LS0[4 + t] + c, m);
    aadd(a.Lph[2 + t] + c, a.dt_stage * m);
}
template <class T>
__global__ void k_adj_tr_scatter(const __grid_constant__ DevParams<double> p, const __grid_constant__ AdjStage<T> a,
                                 const double* J, const __grid_constant__ DP<3> mu) {
    b_adj_tr_scatter(p, a, J, mu, blockIdx.x, blockIdx.y, blockIdx.z);
}

// mom_flux_x = s.rho_u, mom_flux_z = s.rho_w before the averages (moist.jl:1347-1348)
template <class T>
__device__ __forceinline__ void b_adj_mf(const DevParams<double>& p, const AdjStage<T>& a, int bid_x, int bid_y,
                                         int bid_z) {
    ADJ_CELL(k, i);
    a.Lst[1][c] += a.Lmfx[c];
    a.Lst[2][c] += a.Lmfz[c];
}
template <class T>
__global__ void k_adj_mf(const __grid_constant__ DevParams<double> p, const __grid_constant__ AdjStage<T> a) {
    b_adj_mf(p, a, blockIdx.x, blockIdx.y, blockIdx.z);
}

// ----------------------------------------------------------------------------- acoustic substep

// (1) vertical rho_p / rho_theta_p updates (moist.jl:1412-1446) and the momentum-flux average of
// rho_w_p: lambda of the w-p solution x = rho_w_p(k), k < nz-1; theta's share of the vertical
// theta fluxes
template <class T>
__device__ __forceinline__ void b_adj_sub_vert(const DevParams<double>& p, const AdjStage<T>& a, const AdjSub<T>& b,
                                               int bid_x, int bid_y, int bid_z) {
    ADJ_CELL(k, i);
    const int ke = nz - 1;
    if (k >= ke) return;
    const double* dz = p.dz;
    const double EPS = p.EPS, dts = a.dt_s;
    const double x = b.rw[c];
    double lx = b.LPn[2][c] + a.Lmfz[c] / a.m;
    lx += (-dts / dz[k]) * b.LPn[0][c] + (dts / dz[k + 1]) * b.LPn[0][c + P];
    const double al = (-dts / dz[k]) * b.LPn[3][c];      // rho_theta_p(k): kp flux of cell k
    const double be = (dts / dz[k + 1]) * b.LPn[3][c + P];  // rho_theta_p(k+1): km flux of cell k+1
    const T* th = a.theta;
    auto TH = [&](int kk) { return (double)th[MOIST_IDX(kk, i)]; };
    const double sw = a.s.rw[c];
    const double fw1 = dz[k + 1] / (dz[k] + dz[k + 1]), fw2 = dz[k] / (dz[k] + dz[k + 1]);
    double* Lth = a.Ltheta;
    // kp flux of cell k: up3 on (k-1, k, k+1) if x > EPS, k > 0; on (k+2, k+1, k) if
    // s.rho_w < -EPS, k < ke-1 (moist.jl:1426); else f2h
    if (x > EPS && k > 0) {
        lx += al * (-TH(k - 1) + 5.0 * TH(k) + 2.0 * TH(k + 1)) / 6.0;
        aadd(Lth + c - P, -al * x / 6.0);
        aadd(Lth + c, 5.0 * al * x / 6.0);
        aadd(Lth + c + P, 2.0 * al * x / 6.0);
    } else if (sw < -EPS && k < ke - 1) {
        lx += al * (-TH(k + 2) + 5.0 * TH(k + 1) + 2.0 * TH(k)) / 6.0;
        aadd(Lth + c + 2 * P, -al * x / 6.0);
        aadd(Lth + c + P, 5.0 * al * x / 6.0);
        aadd(Lth + c, 2.0 * al * x / 6.0);
    } else {
        lx += al * (TH(k) * fw1 + TH(k + 1) * fw2);
        aadd(Lth + c, al * x * fw1);
        aadd(Lth + c + P, al * x * fw2);
    }
    // km flux of cell k+1, selected by s.rho_w(k)
    if (sw > EPS && k > 0) {
        lx += be * (-TH(k - 1) + 5.0 * TH(k) + 2.0 * TH(k + 1)) / 6.0;
        aadd(Lth + c - P, -be * x / 6.0);
        aadd(Lth + c, 5.0 * be * x / 6.0);
        aadd(Lth + c + P, 2.0 * be * x / 6.0);
    } else if (sw < -EPS && k < ke - 1) {
        lx += be * (-TH(k + 2) + 5.0 * TH(k + 1) + 2.0 * TH(k)) / 6.0;
        aadd(Lth + c + 2 * P, -be * x / 6.0);
        aadd(Lth + c + P, 5.0 * be * x / 6.0);
        aadd(Lth + c, 2.0 * be * x / 6.0);
    } else {
        lx += be * (TH(k) * fw1 + TH(k + 1) * fw2);
        aadd(Lth + c, be * x * fw1);
        aadd(Lth + c + P, be * x * fw2);
    }
    a.Lx[c] = lx;
}
template <class T>
__global__ void k_adj_sub_vert(const __grid_constant__ DevParams<double> p, const __grid_constant__ AdjStage<T> a,
                               const __grid_constant__ AdjSub<T> b) {
    b_adj_sub_vert(p, a, b, blockIdx.x, blockIdx.y, blockIdx.z);
}

// (2a) y = A^-T lambda_x with the stage's elimination (A = tri(a, b + 1, c), the w-p system of
// moist.jl:1009-1018). A block of ADJ_SOLVE_THREADS threads owns `wc` adjacent columns: all of
// them stage the columns' right-hand sides and elimination factors in shared memory with
// coalesced row loads, one thread per column runs the two recurrences from shared memory, and
// all write the solution back by rows.
constexpr int ADJ_SOLVE_THREADS = 256;
__host__ __device__ inline int adj_solve_cols(int nz) {  // widest of 32, 16, 8, 4 within 200 KB
    int w = 32;
    while (w > 4 && (size_t)32 * nz * w > 200 * 1024) w /= 2;
    return w;
}
__host__ __device__ inline size_t adj_solve_smem(int nz) { return (size_t)4 * nz * adj_solve_cols(nz) * sizeof(double); }

__device__ __forceinline__ void b_adj_sub_solve(int nx, int nz, int P, const double* __restrict__ Tc,
                                                const double* __restrict__ Tcp, const double* __restrict__ Trd,
                                                const double* __restrict__ Lx, double* __restrict__ Ly, int bid_x,
                                                int bid_y, int bid_z) {
    extern __shared__ double sm[];
    const int wc = adj_solve_cols(nz);
    const int i0 = bid_x * wc;
    const int n = nz - 1;
    double* sg = sm;                 // [n][wc] right-hand side, then g', then y
    double* ssub = sm + nz * wc;     // c_{j-1}
    double* srd = sm + 2 * nz * wc;  // 1 / pivot
    double* scp = sm + 3 * nz * wc;  // modified super-diagonal
    for (int e = threadIdx.x; e < n * wc; e += blockDim.x) {
        const int j = e / wc, cc = e - j * wc, i = i0 + cc;
        if (i >= nx) continue;
        const size_t cj = MOIST_IDX(j, i);
        sg[e] = Lx[cj];
        ssub[e] = j > 0 ? Tc[cj - P] : 0.0;
        srd[e] = Trd[cj];
        scp[e] = Tcp[cj];
    }
    __syncthreads();
    const int cc = threadIdx.x;
    if (cc < wc && i0 + cc < nx) {
        double g = 0.0;
        for (int j = 0; j < n; j++) {
            const int e = j * wc + cc;
            g = (sg[e] - ssub[e] * g) * srd[e];
            sg[e] = g;
        }
        double y = g;
        for (int j = n - 2; j >= 0; j--) {
            const int e = j * wc + cc;
            y = sg[e] - scp[e] * y;
            sg[e] = y;
        }
    }
    __syncthreads();
    for (int e = threadIdx.x; e < n * wc; e += blockDim.x) {
        const int j = e / wc, c2 = e - j * wc, i = i0 + c2;
        if (i < nx) Ly[MOIST_IDX(j, i)] = sg[e];
    }
}
__global__ void __launch_bounds__(ADJ_SOLVE_THREADS) k_adj_sub_solve(int nx, int nz, int P,
                                  const double* __restrict__ Tc, const double* __restrict__ Tcp,
                                  const double* __restrict__ Trd, const double* __restrict__ Lx,
                                  double* __restrict__ Ly) {
    b_adj_sub_solve(nx, nz, P, Tc, Tcp, Trd, Lx, Ly, blockIdx.x, blockIdx.y, blockIdx.z);
}

// (2b) per cell k, from y of faces k and k-1: the coefficients' lambda -y x^T, the right-hand
// side d = rho_w_p + drho_w - fact (a, b, c) rho_w_p (moist.jl:1009-1018) and
// drho_w = dt_s (R_rho_w - rt2pres_h buoyancy + grav) (1397-1408)
template <class T>
__device__ __forceinline__ void b_adj_sub_rhs(const DevParams<double>& p, const DevParams<T>& pt, const AdjStage<T>& a,
                                              const AdjSub<T>& b, int bid_x, int bid_y, int bid_z) {
    ADJ_CELL(k, i);
    const int n = nz - 1;
    const double* z = p.z;
    const double dts = a.dt_s, fact = a.fact, g2 = -p.GRAV * 0.5;
    const int im = wrapx(i - 1, nx), ip = wrapx(i + 1, nx);
    // rho_theta_p at the off-centred time level, recomputed as the forward substep forms it
    auto rt_tp = [&](int kk) -> double {
        const size_t cc = MOIST_IDX(kk, i);
        const T th_i = a.theta[cc], th_ip = a.theta[MOIST_IDX(kk, ip)], th_im = a.theta[MOIST_IDX(kk, im)];
        const T u_p = b.ru[cc], u_m = b.ru[MOIST_IDX(kk, im)];
        const T flux_ip = (th_ip + th_i) * T(0.5) * u_p;
        const T flux_im = (th_i + th_im) * T(0.5) * u_m;
        const T advection = -(flux_ip - flux_im) / pt.dx;
        const T inc = (T)a.dt_s * (a.rrt[cc] + advection);
        return (double)(T)((double)b.prev_rt[cc] + a.fact_tp64 * (double)inc);
    };
    double lrt2 = 0.0, ltp_rt = 0.0, ltp_rho = 0.0, lpw = 0.0;
    const double tp_k = rt_tp(k);
    if (k < n) {  // face k
        const double y = a.Ly[c];
        const double xk = b.rw[c];
        const double xkm = k > 0 ? (double)b.rw[c - P] : 0.0;
        const double xkp = k < n - 1 ? (double)b.rw[c + P] : 0.0;
        const double wk = b.prev_rw[c];
        const double wkp = k < n - 1 ? (double)b.prev_rw[c + P] : 0.0;
        if (k > 0) a.La[c] += -y * xkm - fact * wk * y;
        a.Lb[c] += -y * xk - fact * wk * y;
        if (k < n - 1) a.Lc[c] += -y * xkp - fact * wkp * y;
        lpw = y * (1.0 - fact * ((k > 0 ? a.Ta[c] : 0.0) + a.Tb[c]));
        a.LRw[c] += dts * y;
        const double dzc = z[k + 1] - z[k];
        const double buoy = (rt_tp(k + 1) - tp_k) / dzc;
        const double rt2h = ((double)a.rt2[c] + (double)a.rt2[c + P]) * 0.5;
        lrt2 += -dts * buoy * 0.5 * y;
        ltp_rt += dts * rt2h * y / dzc;
        ltp_rho += dts * g2 * y;
    }
    if (k >= 1) {  // face k-1
        const double y = a.Ly[c - P];
        const double dzc = z[k] - z[k - 1];
        const double buoy = (tp_k - rt_tp(k - 1)) / dzc;
        const double rt2h = ((double)a.rt2[c - P] + (double)a.rt2[c]) * 0.5;
        lrt2 += -dts * buoy * 0.5 * y;
        ltp_rt += -dts * rt2h * y / dzc;
        ltp_rho += dts * g2 * y;
        if (k < n) lpw += -fact * a.Tc[c - P] * y;
    }
    a.Lrt2[c] += lrt2;
    a.Ltp_rt[c] = ltp_rt;
    a.Ltp_rho[c] = ltp_rho;
    b.LPo[2][c] = lpw;
}
template <class T>
__global__ void k_adj_sub_rhs(const __grid_constant__ DevParams<double> p, const __grid_constant__ DevParams<T> pt,
                              const __grid_constant__ AdjStage<T> a, const __grid_constant__ AdjSub<T> b) {
    b_adj_sub_rhs(p, pt, a, b, blockIdx.x, blockIdx.y, blockIdx.z);
}

// (3) explicit rho_p / rho_theta_p updates and their off-centred values (moist.jl:1367-1396)
template <class T>
__device__ __forceinline__ void b_adj_sub_expl(const DevParams<double>& p, const AdjStage<T>& a, const AdjSub<T>& b,
                                               int bid_x, int bid_y, int bid_z) {
    ADJ_CELL(k, i);
    const double f = a.fact_tp64, dts = a.dt_s;
    const double lrho = b.LPn[0][c], lrt = b.LPn[3][c];
    const double trho = a.Ltp_rho[c], trt = a.Ltp_rt[c];
    const double li_rho = f * trho + lrho, li_rt = f * trt + lrt;
    a.Linc_rho[c] = li_rho;
    a.Linc_rt[c] = li_rt;
    b.LPo[0][c] = trho + lrho;
    double* pend = a.Lpend[(b.n + 1) % 2];
    b.LPo[3][c] = trt + lrt + pend[c];
    pend[c] = 0.0;
    a.LRrho[c] += dts * li_rho;
    a.LRt[c] += dts * li_rt;
}
template <class T>
__global__ void k_adj_sub_expl(const __grid_constant__ DevParams<double> p, const __grid_constant__ AdjStage<T> a,
                               const __grid_constant__ AdjSub<T> b) {
    b_adj_sub_expl(p, a, b, blockIdx.x, blockIdx.y, blockIdx.z);
}

// (4) per face i+1/2: the horizontal forward step of rho_u_p (moist.jl:1355-1366), its
// momentum-flux average and its use in the explicit updates
template <class T>
__device__ __forceinline__ void b_adj_sub_horiz(const DevParams<double>& p, const AdjStage<T>& a, const AdjSub<T>& b,
                                                int bid_x, int bid_y, int bid_z) {
    ADJ_CELL(k, i);
    const int ip = wrapx(i + 1, nx);
    const size_t cp = MOIST_IDX(k, ip);
    const double dts = a.dt_s, dx = p.dx, gam = p.gamma_d;
    double lu = b.LPn[1][c] + a.Lmfx[c] / a.m + dts / dx * (a.Linc_rho[cp] - a.Linc_rho[c]);
    const double lphi = dts / dx * (a.Linc_rt[cp] - a.Linc_rt[c]);
    const double th_i = a.theta[c], th_ip = a.theta[cp];
    const double u = b.ru[c];
    lu += 0.5 * (th_ip + th_i) * lphi;
    aadd(a.Ltheta + c, 0.5 * u * lphi);
    aadd(a.Ltheta + cp, 0.5 * u * lphi);
    b.LPo[1][c] = lu;
    a.LRu[c] += dts * lu;
    const double g = ((double)b.prev_rt[cp] - (double)b.prev_rt[c]) / dx;
    const double g_old = ((double)b.old_rt[cp] - (double)b.old_rt[c]) / dx;
    const double G = g + gam * (g - g_old);
    const double rt2h = ((double)a.rt2[c] + (double)a.rt2[cp]) * 0.5;
    aadd(a.Lrt2 + c, -dts * G * 0.5 * lu);
    aadd(a.Lrt2 + cp, -dts * G * 0.5 * lu);
    const double lG = -dts * rt2h * lu;
    aadd(b.LPo[3] + cp, (1.0 + gam) * lG / dx);
    aadd(b.LPo[3] + c, -(1.0 + gam) * lG / dx);
    double* old = b.n >= 2 ? a.Lpend[b.n % 2] : b.LPo[3];
    aadd(old + cp, -gam * lG / dx);
    aadd(old + c, gam * lG / dx);
}
template <class T>
__global__ void k_adj_sub_horiz(const __grid_constant__ DevParams<double> p, const __grid_constant__ AdjStage<T> a,
                                const __grid_constant__ AdjSub<T> b) {
    b_adj_sub_horiz(p, a, b, blockIdx.x, blockIdx.y, blockIdx.z);
}

// perturbation start rho_p = s0.rho - s.rho etc. (moist.jl:1339-1346)
template <class T>
__device__ __forceinline__ void b_adj_p0(const DevParams<double>& p, const AdjStage<T>& a, const DP<4>& LP, int bid_x,
                                         int bid_y, int bid_z) {
    ADJ_CELL(k, i);
    for (int f = 0; f < 4; f++) {
        const double l = LP.f[f][c];
        a.Lst[f][c] -= l;
        a.LS0[f][c] += l;
    }
}
template <class T>
__global__ void k_adj_p0(const __grid_constant__ DevParams<double> p, const __grid_constant__ AdjStage<T> a,
                         const __grid_constant__ DP<4> LP) {
    b_adj_p0(p, a, LP, blockIdx.x, blockIdx.y, blockIdx.z);
}

// ----------------------------------------------------------------------------- stage tendencies

// lambda of the w-p coefficients -> theta, rt2pres, per cell: theta_h(j) enters b_j, a_{j+1},
// c_{j-1}; rt2pres(k) enters b_k, a_k, b_{k-1}, c_{k-1}
template <class T>
__device__ __forceinline__ void b_adj_tri_coef_T(const DevParams<double>& p, const AdjStage<T>& a, int bid_x, int bid_y,
                                                 int bid_z) {
    ADJ_CELL(k, i);
    const int n = nz - 1;
    const double* dz = p.dz;
    const double* z = p.z;
    const double fact_tp = 0.5 * (1.0 + p.beta);
    const double C = (a.dt_s * fact_tp) * (a.dt_s * fact_tp);
    auto TH = [&](int kk) { return (double)a.theta[MOIST_IDX(kk, i)]; };
    auto R = [&](int kk) { return (double)a.rt2[MOIST_IDX(kk, i)]; };
    auto thh = [&](int kk) { return f2h(TH(kk), TH(kk + 1), dz[kk], dz[kk + 1]); };
    auto dzc = [&](int kk) { return z[kk + 1] - z[kk]; };
    auto LA = [&](int j) { return a.La[MOIST_IDX(j, i)]; };
    auto LB = [&](int j) { return a.Lb[MOIST_IDX(j, i)]; };
    auto LC = [&](int j) { return a.Lc[MOIST_IDX(j, i)]; };
    auto lthh = [&](int j) {
        double l = LB(j) * C * (R(j) / dz[j] + R(j + 1) / dz[j + 1]) / dzc(j);
        if (j + 1 < n) l += LA(j + 1) * (-C * R(j + 1) / (dzc(j + 1) * dz[j + 1]));
        if (j >= 1) l += LC(j - 1) * (-C * R(j) / (dzc(j - 1) * dz[j]));
        return l;
    };
    double lth = 0.0, lr = 0.0;
    if (k < n) {
        lth += lthh(k) * dz[k + 1] / (dz[k] + dz[k + 1]);
        lr += LB(k) * C * thh(k) / (dzc(k) * dz[k]);
        if (k > 0) lr += LA(k) * (-C * thh(k - 1) / (dzc(k) * dz[k]));
    }
    if (k >= 1) {
        lth += lthh(k - 1) * dz[k - 1] / (dz[k - 1] + dz[k]);
        lr += LB(k - 1) * C * thh(k - 1) / (dzc(k - 1) * dz[k]);
        if (k < n) lr += LC(k - 1) * (-C * thh(k) / (dzc(k - 1) * dz[k]));
    }
    a.Ltheta[c] += lth;
    a.Lrt2[c] += lr;
}
template <class T>
__global__ void k_adj_tri_coef_T(const __grid_constant__ DevParams<double> p, const __grid_constant__ AdjStage<T> a) {
    b_adj_tri_coef_T(p, a, blockIdx.x, blockIdx.y, blockIdx.z);
}

// lambda of R_rho, R_rho_u, R_rho_w, R_rho_theta -> their inputs
template <class T>
__device__ __forceinline__ void b_adj_tend_T(const DevParams<double>& p, const AdjStage<T>& a, int bid_x, int bid_y,
                                             int bid_z) {
    ADJ_CELL(k, i);
    const int ke = nz - 1;
    const double dx = p.dx;
    const double* dz = p.dz;
    const int im = wrapx(i - 1, nx), im2 = wrapx(i - 2, nx), ip = wrapx(i + 1, nx), ip2 = wrapx(i + 2, nx);
    double* Lru = a.Lst[1];
    double* Lrw = a.Lst[2];
    double* Lrho = a.Lst[0];
    // R_rho (moist.jl:1079-1086), linear
    {
        const double l = a.LRrho[c];
        if (l != 0.0) {
            aadd(Lru + c, -l / dx);
            aadd(Lru + MOIST_IDX(k, im), l / dx);
            if (k < ke) aadd(Lrw + c, -l / dz[k]);
            if (k > 0) aadd(Lrw + c - P, l / dz[k]);
            a.Lph[0][c] += l;
        }
    }
    const T* ru = a.s.ru;
    const T* rw = a.s.rw;
    const T* rho = a.s.rho;
    auto at = [&](const T* f, int kk, int ii) -> double {
        return (kk >= 0 && kk < nz) ? (double)f[MOIST_IDX(kk, ii)] : 0.0;
    };
    auto tgt = [&](double* f, int kk, int ii, double v) {
        if (kk >= 0 && kk < nz && v != 0.0) aadd(f + MOIST_IDX(kk, ii), v);
    };
    // R_rho_theta
    {
        const double l = a.LRt[c];
        if (l != 0.0) {
            a.Lph[1][c] += l;
            const T* th = a.theta;
            double v[13] = {at(ru, k, i), at(ru, k, im), k < ke ? at(rw, k, i) : 0.0, at(rw, k - 1, i),
                            at(th, k, im2), at(th, k, im), at(th, k, i), at(th, k, ip), at(th, k, ip2),
                            at(th, k - 2, i), at(th, k - 1, i), at(th, k + 1, i), at(th, k + 2, i)};
            local_jacobian<ADJ_DUAL>(
                v, [&](const auto& get) { return gen_R_t<Dual<ADJ_DUAL>>(p, k, get); },
                [&](int s, double d) {
                    const double g = l * d;
                    switch (s) {
                        case 0: tgt(Lru, k, i, g); break;
                        case 1: tgt(Lru, k, im, g); break;
                        case 2: tgt(Lrw, k, i, g); break;
                        case 3: tgt(Lrw, k - 1, i, g); break;
                        case 4: tgt(a.Ltheta, k, im2, g); break;
                        case 5: tgt(a.Ltheta, k, im, g); break;
                        case 6: tgt(a.Ltheta, k, i, g); break;
                        case 7: tgt(a.Ltheta, k, ip, g); break;
                        case 8: tgt(a.Ltheta, k, ip2, g); break;
                        case 9: tgt(a.Ltheta, k - 2, i, g); break;
                        case 10: tgt(a.Ltheta, k - 1, i, g); break;
                        case 11: tgt(a.Ltheta, k + 1, i, g); break;
                        default: tgt(a.Ltheta, k + 2, i, g); break;
                    }
                });
        }
    }
    // R_rho_u
    {
        const double l = a.LRu[c];
        if (l != 0.0) {
            const T* uf = a.uf;
            double v[24] = {at(ru, k, im), at(ru, k, i), at(ru, k, ip),
                            at(rw, k, i), at(rw, k, ip), at(rw, k - 1, i), at(rw, k - 1, ip),
                            at(uf, k, im2), at(uf, k, im), at(uf, k, i), at(uf, k, ip), at(uf, k, ip2),
                            at(uf, k - 2, i), at(uf, k - 1, i), at(uf, k + 1, i), at(uf, k + 2, i),
                            at(rho, k, i), at(rho, k, ip), at(rho, k - 1, i), at(rho, k - 1, ip),
                            at(rho, k + 1, i), at(rho, k + 1, ip), at(a.pres, k, i), at(a.pres, k, ip)};
            local_jacobian<ADJ_DUAL>(
                v, [&](const auto& get) { return gen_R_u<Dual<ADJ_DUAL>>(p, k, get); },
                [&](int s, double d) {
                    const double g = l * d;
                    switch (s) {
                        case 0: tgt(Lru, k, im, g); break;
                        case 1: tgt(Lru, k, i, g); break;
                        case 2: tgt(Lru, k, ip, g); break;
                        case 3: tgt(Lrw, k, i, g); break;
                        case 4: tgt(Lrw, k, ip, g); break;
                        case 5: tgt(Lrw, k - 1, i, g); break;
                        case 6: tgt(Lrw, k - 1, ip, g); break;
                        case 7: tgt(a.Luf, k, im2, g); break;
                        case 8: tgt(a.Luf, k, im, g); break;
                        case 9: tgt(a.Luf, k, i, g); break;
                        case 10: tgt(a.Luf, k, ip, g); break;
                        case 11: tgt(a.Luf, k, ip2, g); break;
                        case 12: tgt(a.Luf, k - 2, i, g); break;
                        case 13: tgt(a.Luf, k - 1, i, g); break;
                        case 14: tgt(a.Luf, k + 1, i, g); break;
                        case 15: tgt(a.Luf, k + 2, i, g); break;
                        case 16: tgt(Lrho, k, i, g); break;
                        case 17: tgt(Lrho, k, ip, g); break;
                        case 18: tgt(Lrho, k - 1, i, g); break;
                        case 19: tgt(Lrho, k - 1, ip, g); break;
                        case 20: tgt(Lrho, k + 1, i, g); break;
                        case 21: tgt(Lrho, k + 1, ip, g); break;
                        case 22: tgt(a.Lpres, k, i, g); break;
                        default: tgt(a.Lpres, k, ip, g); break;
                    }
                });
        }
    }
    // R_rho_w
    if (k < ke) {
        const double l = a.LRw[c];
        if (l != 0.0) {
            const T* wf = a.wf;
            auto atw = [&](int kk,
                           int ii) -> double { return (kk >= 0 && kk < ke) ? (double)wf[MOIST_IDX(kk, ii)] : 0.0; };
            double v[24] = {at(ru, k, i), at(ru, k + 1, i), at(ru, k, im), at(ru, k + 1, im),
                            at(rw, k - 1, i), at(rw, k, i), k + 1 < ke ? at(rw, k + 1, i) : 0.0,
                            atw(k, im2), atw(k, im), atw(k, i), atw(k, ip), atw(k, ip2),
                            atw(k - 2, i), atw(k - 1, i), atw(k + 1, i), atw(k + 2, i),
                            at(rho, k, i), at(rho, k + 1, i), at(rho, k, im), at(rho, k + 1, im),
                            at(rho, k, ip), at(rho, k + 1, ip), at(a.pres, k, i), at(a.pres, k + 1, i)};
            local_jacobian<ADJ_DUAL>(
                v, [&](const auto& get) { return gen_R_w<Dual<ADJ_DUAL>>(p, k, get); },
                [&](int s, double d) {
                    const double g = l * d;
                    switch (s) {
                        case 0: tgt(Lru, k, i, g); break;
                        case 1: tgt(Lru, k + 1, i, g); break;
                        case 2: tgt(Lru, k, im, g); break;
                        case 3: tgt(Lru, k + 1, im, g); break;
                        case 4: tgt(Lrw, k - 1, i, g); break;
                        case 5: tgt(Lrw, k, i, g); break;
                        case 6: tgt(Lrw, k + 1, i, g); break;
                        case 7: tgt(a.Lwf, k, im2, g); break;
                        case 8: tgt(a.Lwf, k, im, g); break;
                        case 9: tgt(a.Lwf, k, i, g); break;
                        case 10: tgt(a.Lwf, k, ip, g); break;
                        case 11: tgt(a.Lwf, k, ip2, g); break;
                        case 12: tgt(a.Lwf, k - 2, i, g); break;
                        case 13: tgt(a.Lwf, k - 1, i, g); break;
                        case 14: tgt(a.Lwf, k + 1, i, g); break;
                        case 15: tgt(a.Lwf, k + 2, i, g); break;
                        case 16: tgt(Lrho, k, i, g); break;
                        case 17: tgt(Lrho, k + 1, i, g); break;
                        case 18: tgt(Lrho, k, im, g); break;
                        case 19: tgt(Lrho, k + 1, im, g); break;
                        case 20: tgt(Lrho, k, ip, g); break;
                        case 21: tgt(Lrho, k + 1, ip, g); break;
                        case 22: tgt(a.Lpres, k, i, g); break;
                        default: tgt(a.Lpres, k + 1, i, g); break;
                    }
                });
        }
    }
}
template <class T>
__global__ void __launch_bounds__(ADJ_THREADS) k_adj_tend_T(const __grid_constant__ DevParams<double> p,
                                  const __grid_constant__ AdjStage<T> a) {
    b_adj_tend_T(p, a, blockIdx.x, blockIdx.y, blockIdx.z);
}

// face velocities u_face = rho_u 2 / (rho_i + rho_i+1), w_face = rho_w / f2h(rho) (moist.jl:1091-1097,
// 1185-1189)
template <class T>
__device__ __forceinline__ void b_adj_face_T(const DevParams<double>& p, const AdjStage<T>& a, int bid_x, int bid_y,
                                             int bid_z) {
    ADJ_CELL(k, i);
    const int ip = wrapx(i + 1, nx);
    const double* dz = p.dz;
    double* Lrho = a.Lst[0];
    {
        const double l = a.Luf[c];
        if (l != 0.0) {
            const double sum = (double)a.s.rho[c] + (double)a.s.rho[MOIST_IDX(k, ip)];
            const double uf = (double)a.s.ru[c] * 2.0 / sum;
            aadd(a.Lst[1] + c, l * 2.0 / sum);
            aadd(Lrho + c, -l * uf / sum);
            aadd(Lrho + MOIST_IDX(k, ip), -l * uf / sum);
        }
    }
    if (k < nz - 1) {
        const double l = a.Lwf[c];
        if (l != 0.0) {
            const double s = dz[k] + dz[k + 1];
            const double f = ((double)a.s.rho[c] * dz[k + 1] + (double)a.s.rho[c + P] * dz[k]) / s;
            const double w = (double)a.s.rw[c];
            aadd(a.Lst[2] + c, l / f);
            aadd(Lrho + c, -l * w / (f * f) * dz[k + 1] / s);
            aadd(Lrho + c + P, -l * w / (f * f) * dz[k] / s);
        }
    }
}
template <class T>
__global__ void k_adj_face_T(const __grid_constant__ DevParams<double> p, const __grid_constant__ AdjStage<T> a) {
    b_adj_face_T(p, a, blockIdx.x, blockIdx.y, blockIdx.z);
}

// diagnostics pres, theta, rt2pres -> rho, rho_theta, rho_q*
template <class T>
__device__ __forceinline__ void b_adj_diag_T(const DevParams<double>& p, const AdjStage<T>& a, int bid_x, int bid_y,
                                             int bid_z) {
    ADJ_CELL(k, i);
    const double lo[3] = {a.Lpres[c], a.Ltheta[c], a.Lrt2[c]};
    if (lo[0] == 0.0 && lo[1] == 0.0 && lo[2] == 0.0) return;
    double v[5] = {(double)a.s.rho[c], (double)a.s.rt[c], (double)a.s.qv[c], (double)a.s.qc[c], (double)a.s.qr[c]};
    const int f_of_slot[5] = {0, 3, 4, 5, 6};
    double acc[5] = {0, 0, 0, 0, 0};
    for (int o = 0; o < 3; o++) {
        if (lo[o] == 0.0) continue;
        local_jacobian<ADJ_DUAL>(v, [&](const auto& get) { return gen_diag<Dual<ADJ_DUAL>>(p, o, get); },
                                 [&](int s, double d) { acc[s] += lo[o] * d; });
    }
    for (int s = 0; s < 5; s++) a.Lst[f_of_slot[s]][c] += acc[s];
}
template <class T>
__global__ void __launch_bounds__(ADJ_THREADS) k_adj_diag_T(const __grid_constant__ DevParams<double> p,
                                  const __grid_constant__ AdjStage<T> a) {
    b_adj_diag_T(p, a, blockIdx.x, blockIdx.y, blockIdx.z);
}

// ----------------------------------------------------------------------------- physics

template <class T>
struct AdjPhys {
    StateP<T> s;              // the step's input State
    const T* sed;             // d_rho_qr_sed of that State
    double* Lst[7];
    double* Lph[5];
    double* Lsed;             // scratch: lambda of d_rho_qr_sed
    const double* prec_w;     // d objective / d prec, per column (or null)
    double* Lpar;             // [2]: d / d K_auto, d / d Qc_threshold
};

// phys assembly (moist.jl:1633-1643) and Kessler microphysics (554-671)
template <class T>
__device__ __forceinline__ void b_adj_kessler(const DevParams<double>& p, const AdjPhys<T>& a, int bid_x, int bid_y,
                                              int bid_z) {
    const int i = bid_x * blockDim.x + threadIdx.x;
    const int k = bid_y;
    const int nx = p.nx, nz = p.nz, P = p.P;
    double par[2] = {0.0, 0.0};
    if (i < nx && k < nz) {
        const size_t c = MOIST_IDX(k, i);
        const double rho = a.s.rho[c], rt = a.s.rt[c], sed = a.sed[c];
        const double l_rho = a.Lph[0][c], l_th = a.Lph[1][c], l_qv = a.Lph[2][c], l_qc = a.Lph[3][c],
                     l_qr = a.Lph[4][c];
        // d_th = dth_mp + th_rd + d_rho * rt / rho; d_qr = dqr_mp + sed; d_rho = sed
        a.Lsed[c] = l_rho + l_qr + l_th * rt / rho;
        double acc[5] = {-l_th * sed * rt / (rho * rho), l_th * sed / rho, 0.0, 0.0, 0.0};
        if (p.do_mp) {
            double v[7] = {rho, rt, (double)a.s.qv[c], (double)a.s.qc[c], (double)a.s.qr[c], p.K_auto, p.Qc_threshold};
            local_jacobian<ADJ_DUAL>(
                v,
                [&](const auto& get) {
                    using S = Dual<ADJ_DUAL>;
                    DevParams<S> q = params_as<S>(p);
                    q.K_auto = get(5);
                    q.Qc_threshold = get(6);
                    S dqv, dqc, dqr, dth;
                    kessler_cell<S>(get(0), get(1), get(2), get(3), get(4), q, dqv, dqc, dqr, dth);
                    return dqv * S(l_qv) + dqc * S(l_qc) + dqr * S(l_qr) + dth * S(l_th);
                },
                [&](int s, double d) {
                    if (s < 5)
                        acc[s] += d;
                    else
                        par[s - 5] += d;
                });
        }
        a.Lst[0][c] += acc[0];
        a.Lst[3][c] += acc[1];
        a.Lst[4][c] += acc[2];
        a.Lst[5][c] += acc[3];
        a.Lst[6][c] += acc[4];
    }
    // block sums of the parameter gradients
    for (int j = 0; j < 2; j++) {
        double v = par[j];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0 && v != 0.0) atomicAdd(a.Lpar + j, v);
    }
}
template <class T>
__global__ void __launch_bounds__(ADJ_THREADS) k_adj_kessler(const __grid_constant__ DevParams<double> p,
                                  const __grid_constant__ AdjPhys<T> a) {
    b_adj_kessler(p, a, blockIdx.x, blockIdx.y, blockIdx.z);
}

// rain sedimentation (moist.jl:674-707): sed(k) = (F(k+1) - F(k)) / dz(k), F = rho_qr Vt,
// d_prec = F(0), prec += d_prec dt
template <class T>
__device__ __forceinline__ void b_adj_sed(const DevParams<double>& p, const AdjPhys<T>& a, int bid_x, int bid_y,
                                          int bid_z) {
    ADJ_CELL(k, i);
    if (!(p.do_mp && p.do_sed)) return;
    const double* dz = p.dz;
    double lF = -a.Lsed[c] / dz[k];
    if (k >= 1) lF += a.Lsed[c - P] / dz[k - 1];
    if (k == 0 && a.prec_w) lF += a.prec_w[i] * p.dt;
    if (lF == 0.0) return;
    double v[2] = {(double)a.s.qr[c], (double)a.s.rho[c]};
    double acc[2] = {0.0, 0.0};
    local_jacobian<2>(v,
                      [&](const auto& get) {
                          using S = Dual<2>;
                          const DevParams<S> q = params_as<S>(p);
                          return get(0) * terminal_velocity<S>(get(0), get(1), q);
                      },
                      [&](int s, double d) { acc[s] = lF * d; });
    a.Lst[6][c] += acc[0];
    a.Lst[0][c] += acc[1];
}
template <class T>
__global__ void __launch_bounds__(ADJ_THREADS) k_adj_sed(const __grid_constant__ DevParams<double> p,
                                  const __grid_constant__ AdjPhys<T> a) {
    b_adj_sed(p, a, blockIdx.x, blockIdx.y, blockIdx.z);
}

// lambda(S^n) = lambda of the first stage's input + lambda of s0
__device__ __forceinline__ void b_adj_step_end(int nx, int nz, int P, const DP<7>& Lst, const DP<7>& LS0,
                                               const DP<5>& Lph, int bid_x, int bid_y, int bid_z) {
    const int i = bid_x * blockDim.x + threadIdx.x;
    const int k = bid_y;
    if (i >= nx || k >= nz) return;
    const size_t c = MOIST_IDX(k, i);
    for (int f = 0; f < 7; f++) {
        Lst.f[f][c] += LS0.f[f][c];
        LS0.f[f][c] = 0.0;
    }
    for (int f = 0; f < 5; f++) Lph.f[f][c] = 0.0;
}
__global__ void k_adj_step_end(int nx, int nz, int P, const __grid_constant__ DP<7> Lst,
                               const __grid_constant__ DP<7> LS0, const __grid_constant__ DP<5> Lph) {
    b_adj_step_end(nx, nz, P, Lst, LS0, Lph, blockIdx.x, blockIdx.y, blockIdx.z);
}

// ----------------------------------------------------------------------------- host layout

// (ka, ia) column-major double -> [nz][P] interior
__global__ void k_adj_from_ref(int nx, int nz, int halo, int P, const double* src, double* dst) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int k = blockIdx.y;
    if (i >= nx || k >= nz) return;
    dst[MOIST_IDX(k, i)] = src ? src[(size_t)(i + halo) * nz + k] : 0.0;
}
// [nz][P] interior -> (ka, ia) column-major double, halo columns zero
__global__ void k_adj_to_ref(int nx, int nz, int halo, int P, const double* src, double* dst) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int k = blockIdx.y;
    const int ia = nx + 2 * halo;
    if (j >= ia || k >= nz) return;
    const int i = j - halo;
    dst[(size_t)j * nz + k] = (i >= 0 && i < nx) ? src[MOIST_IDX(k, i)] : 0.0;
}

// objective J = sum_i w_i prec_i + sum_f <seed_f, state_f> over the interior
template <class T>
__global__ void k_adj_objective(int nx, int nz, int P, StateP<T> s, const T* prec, const double* prec_w, DP<7> seed,
                                double* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int k = blockIdx.y;
    double v = 0.0;
    if (i < nx && k < nz) {
        const size_t c = MOIST_IDX(k, i);
        const T* f[7] = {s.rho, s.ru, s.rw, s.rt, s.qv, s.qc, s.qr};
        for (int j = 0; j < 7; j++)
            if (seed.f[j]) v += seed.f[j][c] * (double)f[j][c];
        if (k == 0 && prec_w) v += prec_w[i] * (double)prec[i];
    }
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0 && v != 0.0) atomicAdd(out, v);
}

// copy of up to 8 fields of n elements (tape and checkpoints)
template <class T>
struct CopyList {
    const T* src[8];
    T* dst[8];
    int nf;
};
template <class T>
__global__ void k_copy_fields(CopyList<T> l, size_t n) {
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (int f = 0; f < l.nf; f++)
        for (size_t j = (size_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += stride) l.dst[f][j] = l.src[f][j];
}

}  // namespace moist
