// oracle_tangent.cpp - forward-mode derivative of the oracle's Float64 large step
// (TEST INFRASTRUCTURE, see moist_oracle.hpp).
//
// The oracle's step is a template over its scalar type. Instantiated with mm::Dual<1> (a Float64
// value and one directional derivative), the same code computes, alongside J, the exact
// directional derivative dJ/dv of an objective of the final State: what ForwardDiff's dual
// numbers give when pushed through the reference's Julia step. Branches (upwind selectors,
// limiter switches, Kessler clamps) select on the value, so dJ/dv is the derivative of the
// piece the run stays on; it is checked against central differences of the Float64 oracle
// (tests/test_tangent.py) and is the exact counterpart of the adjoint's <grad, v>.
//
// The mm:: Dual overloads must be visible before moist_oracle.hpp is parsed: its templates call
// mm::mpow and friends by qualified name, which binds at the template's definition.
#include "../moist2d_b200/csrc/dual.cuh"
#include "moist_oracle.hpp"

using namespace oracle;

namespace {

using D1 = mm::Dual<1>;

// host Float64 array + optional direction -> Dual array
void seed_in(std::vector<D1>& f, const void* src, const double* dir) {
    const double* x = (const double*)src;
    for (size_t j = 0; j < f.size(); j++) {
        f[j] = D1(x ? x[j] : 0.0);
        if (dir) f[j].d[0] = dir[j];
    }
}

double dot_v(const std::vector<D1>& f, const double* w) {
    double s = 0.0;
    if (w)
        for (size_t j = 0; j < f.size(); j++) s += w[j] * f[j].v;
    return s;
}
double dot_d(const std::vector<D1>& f, const double* w) {
    double s = 0.0;
    if (w)
        for (size_t j = 0; j < f.size(); j++) s += w[j] * f[j].d[0];
    return s;
}

}  // namespace

extern "C" {

// Runs nsteps Float64 large steps (rk3_step!, moist.jl:1589-1683; FP64 elimination) from the
// State h (Float64 host arrays) perturbed in direction dir (dir[f], f = rho .. rho_qr in
// MOIST_FIELD order, (ka, ia) or NULL; dir_prec (ia) or NULL; d_k_auto, d_qc_threshold for
// K_auto and Qc_threshold). With the objective
//   J = sum(prec_weight * prec_final) + sum_f sum(state_weight[f] * S_final.f)
// (NULL weights count as 0), writes J and its directional derivative dJ. h is not modified.
// Returns -1, the MOIST_FIELD_* index of a NaN found by the end-of-stage check, or -2.
int oracle_tangent_run(const moist_params* cp, const moist_state_host* h, const double* const dir[7],
                       const double* dir_prec, double d_k_auto, double d_qc_threshold, int nsteps,
                       const double* prec_weight, const double* const state_weight[7], double* J,
                       double* dJ) {
    if (!cp || !h || !J || !dJ || cp->nz < 2 || cp->nx < 1 || !cp->zf || !cp->dz || !cp->z || nsteps < 0)
        return -2;
    Par<D1> p = Par<D1>::from_c(*cp);
    p.K_auto.d[0] = d_k_auto;
    p.Qc_threshold.d[0] = d_qc_threshold;
    State<D1> s(p);
    std::vector<D1>* prog[7] = {&s.rho.v, &s.rho_u.v, &s.rho_w.v, &s.rho_theta.v, &s.rho_qv.v, &s.rho_qc.v,
                                &s.rho_qr.v};
    const void* src[7] = {h->rho, h->rho_u, h->rho_w, h->rho_theta, h->rho_qv, h->rho_qc, h->rho_qr};
    for (int f = 0; f < 7; f++) seed_in(*prog[f], src[f], dir ? dir[f] : nullptr);
    seed_in(s.prec, h->prec, dir_prec);
    seed_in(s.mflux, h->mflux, nullptr);
    seed_in(s.shflux, h->shflux, nullptr);
    seed_in(s.lhflux, h->lhflux, nullptr);
    seed_in(s.theta_ref, h->theta_ref, nullptr);
    seed_in(s.d_rho_theta_mp.v, h->d_rho_theta_mp, nullptr);
    seed_in(s.d_rho_qv_mp.v, h->d_rho_qv_mp, nullptr);
    seed_in(s.d_rho_qc_mp.v, h->d_rho_qc_mp, nullptr);
    seed_in(s.d_rho_qr_mp.v, h->d_rho_qr_mp, nullptr);
    seed_in(s.d_rho_qr_sed.v, h->d_rho_qr_sed, nullptr);
    seed_in(s.d_rho_u_sf, h->d_rho_u_sf, nullptr);
    seed_in(s.d_rho_theta_sf, h->d_rho_theta_sf, nullptr);
    seed_in(s.d_rho_qv_sf, h->d_rho_qv_sf, nullptr);
    seed_in(s.d_rho_theta_rd.v, h->d_rho_theta_rd, nullptr);
    int bad = -1;
    for (int n = 0; n < nsteps && bad < 0; n++) bad = rk3_step<D1, D1>(s, p);
    if (bad >= 0) return bad;
    double j = dot_v(s.prec, prec_weight), dj = dot_d(s.prec, prec_weight);
    for (int f = 0; f < 7; f++) {
        const double* w = state_weight ? state_weight[f] : nullptr;
        j += dot_v(*prog[f], w);
        dj += dot_d(*prog[f], w);
    }
    *J = j;
    *dJ = dj;
    return -1;
}

}  // extern "C"
