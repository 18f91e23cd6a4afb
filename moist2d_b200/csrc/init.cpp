// init.cpp - seeded initial States behind the C-ABI (host code; no device needed).
//
// The reference builds its initial State with init_state! (moist.jl:351-450): a reference theta
// profile, uniform theta noise from per-thread Xoshiro streams (moist.jl:374-375, so the State
// depends on the thread schedule), an RH profile and a per-column Newton iteration for discrete
// hydrostatic balance (moist.jl:387-434). Here the noise comes from the counter-based
// Philox4x32-10 generator (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as
// 1, 2, 3", SC'11), keyed by (seed, stream) and counted by the cell index, so a State depends on
// the seed alone. The benchmark workloads (a warm moist bubble; an analytic sounding with warm
// bubbles) are built the same way as the Python generators of moist2d_b200/init.py: in double
// precision, base columns in the model's discrete hydrostatic balance
//   p_k - p_{k-1} = -g (z_k - z_{k-1}) (rho_{k-1} + rho_k) / 2
// (the pressure-gradient and gravity terms of moist.jl:1271-1274) with p from the equation of
// state p = P0 (r rho theta / P0)^(cp/cv) (moist.jl:1058), bubbles applied at constant
// pressure, then rounded once to the State precision.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../../include/moist2d.h"

namespace {

// ---- Philox4x32-10
void philox4x32_10(uint32_t ctr[4], uint32_t k0, uint32_t k1) {
    const uint64_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
    for (int r = 0; r < 10; r++) {
        const uint64_t p0 = M0 * (uint64_t)ctr[0];
        const uint64_t p1 = M1 * (uint64_t)ctr[2];
        const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        const uint32_t c0 = hi1 ^ ctr[1] ^ k0, c2 = hi0 ^ ctr[3] ^ k1;
        ctr[0] = c0;
        ctr[1] = lo1;
        ctr[2] = c2;
        ctr[3] = lo0;
        k0 += W0;
        k1 += W1;
    }
}

// uniform (0, 1) double of index idx in the stream (seed, stream): the first output word of the
// counter (idx low, idx high, stream, 0) under the key (seed, "mois")
double uniform01(uint32_t seed, uint32_t stream, uint64_t idx) {
    uint32_t c[4] = {(uint32_t)idx, (uint32_t)(idx >> 32), stream, 0u};
    philox4x32_10(c, seed, 0x6D6F6973u);
    return ((double)c[0] + 0.5) * (1.0 / 4294967296.0);
}

struct Consts {
    double GRAV, Rd, Rv, Cpd, Cpv, P0, T0, ES0, A_SAT, B_SAT, EPSvap;
};

Consts consts_of(const moist_params* p) {
    return Consts{p->grav, p->rd, p->rv, p->cpd, p->cpv, p->p0, p->t0, p->es0, p->a_sat, p->b_sat, p->epsvap};
}

// saturation specific humidity (moist.jl:253-273) in double precision
double qsat_of(double pr, double Tk, const Consts& c) {
    const double Tc = Tk - c.T0;
    const double es = c.ES0 * std::exp(c.A_SAT * Tc / (c.B_SAT + Tc));
    const double tmp = pr - (1.0 - c.EPSvap) * es;
    return tmp > 1e-12 ? c.EPSvap * es / std::max(tmp, 1e-12) : 0.0;
}

void gas(double qv, const Consts& c, double& r, double& cp) {
    const double qd = 1.0 - qv;
    r = c.Rd * qd + c.Rv * qv;
    cp = c.Cpd * qd + c.Cpv * qv;
}

// rho, qv, theta at pressure pr for theta = theta_of(Exner) and relative humidity rh
template <class F>
void state_at_pressure(double pr, F theta_of, double rh, const Consts& c, double& rho, double& qv, double& th) {
    qv = 0.0;
    double r, cp;
    for (int it = 0; it < 30; it++) {
        gas(qv, c, r, cp);
        const double Pi = std::pow(pr / c.P0, r / cp);
        const double t = theta_of(Pi);
        qv = std::max(0.0, rh * qsat_of(pr, t * Pi, c));
    }
    gas(qv, c, r, cp);
    const double Pi = std::pow(pr / c.P0, r / cp);
    th = theta_of(Pi);
    rho = pr / (r * th * Pi);
}

// one base column marched up in discrete hydrostatic balance from the surface pressure 1000 hPa:
// rho, qv, theta, p per level. theta_of(k, Exner), rh_of(k).
template <class FT, class FR>
void hydrostatic_column(const std::vector<double>& z, int nz, FT theta_of, FR rh_of, const Consts& c,
                        std::vector<double>& rho, std::vector<double>& qv, std::vector<double>& th,
                        std::vector<double>& pr) {
    const double g = c.GRAV, p_surf = 1e5;
    rho.assign(nz, 0.0);
    qv.assign(nz, 0.0);
    th.assign(nz, 0.0);
    pr.assign(nz, 0.0);
    double p_prev = 0.0, rho_prev = 0.0;
    for (int k = 0; k < nz; k++) {
        const double rh = rh_of(k);
        auto tfn = [&](double Pi) { return theta_of(k, Pi); };
        double p, r_, q_, t_;
        if (k == 0) {
            const double dzk = z[0];
            p = p_surf * std::exp(-g * dzk / (287.0 * 300.0));
            for (int it = 0; it < 60; it++) {  // p0 = p_surf - g z0 rho0
                state_at_pressure(p, tfn, rh, c, r_, q_, t_);
                p = p_surf - g * dzk * r_;
            }
        } else {
            const double dzk = z[k] - z[k - 1];
            p = p_prev * std::exp(-g * dzk / (287.0 * 250.0));
            for (int it = 0; it < 60; it++) {  // p_k = p_{k-1} - g dz (rho_{k-1} + rho_k) / 2
                state_at_pressure(p, tfn, rh, c, r_, q_, t_);
                p = p_prev - g * dzk * 0.5 * (rho_prev + r_);
            }
        }
        state_at_pressure(p, tfn, rh, c, r_, q_, t_);
        rho[k] = r_;
        qv[k] = q_;
        th[k] = t_;
        pr[k] = p;
        p_prev = p;
        rho_prev = r_;
    }
}

// the analytic sounding: theta = 300 + 43 (z/12 km)^1.25 K below 12 km, isothermal above (the
// temperature of the 12 km level); RH = 1 - 0.75 (z/12 km)^1.25, 0.25 above
double sounding_rh(double z) { return 1.0 - 0.75 * std::pow(std::min(z / 12e3, 1.0), 1.25); }

void sounding_column(const std::vector<double>& z, int nz, const Consts& c, std::vector<double>& rho,
                     std::vector<double>& qv, std::vector<double>& th, std::vector<double>& pr) {
    double T12 = 0.0;
    auto theta_of = [&](int k, double Pi) {
        if (z[k] <= 12e3) return 300.0 + 43.0 * std::pow(z[k] / 12e3, 1.25);
        return T12 / Pi;
    };
    auto rh_of = [&](int k) { return sounding_rh(z[k]); };
    int klast = 0;  // levels at or below 12 km
    while (klast < nz && z[klast] <= 12e3) klast++;
    hydrostatic_column(z, std::max(klast, 1), theta_of, rh_of, c, rho, qv, th, pr);
    if (klast < nz) {
        const int kt = std::max(klast, 1) - 1;
        double r, cp;
        gas(qv[kt], c, r, cp);
        const double Pi_top = std::pow(pr[kt] / c.P0, r / cp);
        T12 = th[kt] * Pi_top;
        hydrostatic_column(z, nz, theta_of, rh_of, c, rho, qv, th, pr);
    }
}

double bubble_shape(double x, double z, double xc, double zc, double xr, double zr, double& r) {
    const double a = (x - xc) / xr, b = (z - zc) / zr;
    r = std::sqrt(a * a + b * b);
    if (!(r < 1.0)) return 0.0;
    const double cs = std::cos(3.141592653589793 * r * 0.5);  // numpy.pi
    return cs * cs;
}

// State writer: interior fields given in double (nz, nx), rounded to T, halos periodic
template <class T>
struct Writer {
    const moist_params* p;
    moist_state_host* s;
    int nx, nz, h, ia;
    Writer(const moist_params* p_, moist_state_host* s_) : p(p_), s(s_) {
        nx = p->nx;
        nz = p->nz;
        h = p->halo;
        ia = nx + 2 * h;
    }
    void put(void* dst, const std::vector<double>& f) {  // f[k * nx + i]
        if (!dst) return;
        T* a = (T*)dst;
        for (int i = 0; i < nx; i++)
            for (int k = 0; k < nz; k++) a[(size_t)(i + h) * nz + k] = (T)f[(size_t)k * nx + i];
        halo(a);
    }
    void halo(T* a) {  // exchange_halo! (moist.jl:233-241)
        for (int j = 0; j < h; j++)
            for (int k = 0; k < nz; k++) {
                a[(size_t)j * nz + k] = a[(size_t)(nx + j) * nz + k];
                a[(size_t)(nx + h + j) * nz + k] = a[(size_t)(h + j) * nz + k];
            }
    }
    void zero2(void* dst) {
        if (dst) std::memset(dst, 0, (size_t)nz * ia * sizeof(T));
    }
    void zero1(void* dst) {
        if (dst) std::memset(dst, 0, (size_t)ia * sizeof(T));
    }
    // rho, rho_theta, rho_qv, rho_u from (rho, qv, theta, u); the rest of the State zero
    void fill(const std::vector<double>& rho, const std::vector<double>& qv, const std::vector<double>& th,
              const std::vector<double>& u, const std::vector<double>& theta_ref) {
        const size_t n = (size_t)nz * nx;
        std::vector<double> f(n);
        put(s->rho, rho);
        for (size_t j = 0; j < n; j++) f[j] = rho[j] * th[j];
        put(s->rho_theta, f);
        for (size_t j = 0; j < n; j++) f[j] = rho[j] * qv[j];
        put(s->rho_qv, f);
        for (size_t j = 0; j < n; j++) f[j] = rho[j] * u[j];
        put(s->rho_u, f);
        for (void* z2 : {s->rho_w, s->rho_qc, s->rho_qr, s->d_rho_theta_mp, s->d_rho_qv_mp, s->d_rho_qc_mp,
                         s->d_rho_qr_mp, s->d_rho_qr_sed, s->d_rho_theta_rd})
            zero2(z2);
        for (void* z1 : {s->prec, s->mflux, s->shflux, s->lhflux, s->d_rho_u_sf, s->d_rho_theta_sf, s->d_rho_qv_sf})
            zero1(z1);
        if (s->theta_ref)
            for (int k = 0; k < nz; k++) ((T*)s->theta_ref)[k] = (T)theta_ref[k];
    }
};

template <class T>
std::vector<double> zgrid(const moist_params* p) {
    std::vector<double> z(p->nz);
    for (int k = 0; k < p->nz; k++) z[k] = (double)((const T*)p->z)[k];
    return z;
}

bool valid(const moist_params* p, int precision, const moist_state_host* s) {
    return p && s && p->z && p->nx >= 1 && p->nz >= 1 && p->halo >= 0 && p->halo <= p->nx &&
           (precision == MOIST_F32 || precision == MOIST_F64);
}

template <class T>
int warm_bubble_t(const moist_params* p, uint32_t seed, moist_state_host* s) {
    const Consts c = consts_of(p);
    const int nx = p->nx, nz = p->nz;
    const std::vector<double> z = zgrid<T>(p);
    const double dx = (double)(T)p->dx;
    std::vector<double> rho0, qv0, th0, pr;
    hydrostatic_column(z, nz, [](int, double) { return 300.0; }, [](int) { return 0.2; }, c, rho0, qv0, th0, pr);
    const size_t n = (size_t)nz * nx;
    std::vector<double> rho(n), qv(n), th(n), u(n, 0.0), ref(nz, 300.0);
    for (int k = 0; k < nz; k++)
        for (int i = 0; i < nx; i++) {
            const double x = (i + 0.5) * dx;
            double r;
            const double shape = bubble_shape(x, z[k], 10e3 * nx / 200.0, 2e3, 2e3, 2e3, r);
            const double noise = 0.01 * (uniform01(seed, 0, (uint64_t)i * nz + k) * 2.0 - 1.0);
            const double thp = 2.0 * shape + noise;
            const double rh = r < 1.0 ? 0.95 : 0.2;
            const size_t j = (size_t)k * nx + i;
            state_at_pressure(pr[k], [&](double) { return 300.0 + thp; }, rh, c, rho[j], qv[j], th[j]);
        }
    Writer<T>(p, s).fill(rho, qv, th, u, ref);
    return MOIST_OK;
}

template <class T>
int sounding_t(const moist_params* p, const moist_bubble* b, int nb, moist_state_host* s) {
    const Consts c = consts_of(p);
    const int nx = p->nx, nz = p->nz;
    const std::vector<double> z = zgrid<T>(p);
    const double dx = (double)(T)p->dx;
    const double lx = (double)(T)p->lx;
    std::vector<double> rho0, qv0, th0, pr;
    sounding_column(z, nz, c, rho0, qv0, th0, pr);
    const size_t n = (size_t)nz * nx;
    std::vector<double> rho(n), qv(n), th(n), u(n);
    for (int k = 0; k < nz; k++) {
        const double rh = sounding_rh(z[k]);
        const double uk = 12.0 * std::tanh(z[k] / 3e3);
        for (int i = 0; i < nx; i++) {
            const double x = (i + 0.5) * dx;
            double thp = 0.0;
            for (int j = 0; j < nb; j++) {
                double dxp = std::fabs(x - b[j].xc);
                dxp = std::min(dxp, lx - dxp);  // periodic distance in x
                double r;
                thp += b[j].amp * bubble_shape(dxp, z[k], 0.0, b[j].zc, b[j].radius, b[j].radius, r);
            }
            const size_t jj = (size_t)k * nx + i;
            const double th_env = th0[k];
            state_at_pressure(pr[k], [&](double) { return th_env + thp; }, rh, c, rho[jj], qv[jj], th[jj]);
            u[jj] = uk;
        }
    }
    Writer<T>(p, s).fill(rho, qv, th, u, th0);
    return MOIST_OK;
}

template <class T>
int init_state_t(const moist_params* p, const moist_init_profile* pf, uint32_t seed, moist_state_host* s) {
    const Consts c = consts_of(p);
    const int nx = p->nx, nz = p->nz;
    const std::vector<double> z = zgrid<T>(p);
    const double theta0 = (double)(T)pf->theta0, bl = (double)(T)pf->bndlayer_depth;
    const double zt = (double)(T)pf->z_tropopause, g1 = (double)(T)pf->dtheta_dz_trop;
    const double g2 = (double)(T)pf->dtheta_dz_stra, pert = (double)(T)pf->theta_pert;
    const double RH_surf = (double)(T)pf->rel_hum_surf / 100.0, decay = (double)(T)pf->rel_hum_decay;
    std::vector<double> ref(nz);
    for (int k = 0; k < nz; k++)  // reference theta (moist.jl:358-368)
        ref[k] = z[k] < bl ? theta0 : (z[k] < zt ? theta0 + g1 * (z[k] - bl) : theta0 + g1 * (zt - bl) + g2 * (z[k] - zt));
    const size_t n = (size_t)nz * nx;
    std::vector<double> th(n), rho(n), qv(n), u(n, (double)(T)pf->u0);
    for (int k = 0; k < nz; k++)
        for (int i = 0; i < nx; i++)
            th[(size_t)k * nx + i] = ref[k] + pert * (uniform01(seed, 0, (uint64_t)i * nz + k) * 2.0 - 1.0);
    const double Rd = c.Rd, Rv = c.Rv, Cpd = c.Cpd, Cpv = c.Cpv, P0 = c.P0, g = c.GRAV;
    // per column: the hydrostatic Newton iteration of moist.jl:387-434
    for (int i = 0; i < nx; i++) {
        double Pi = 1.0, p_km = 0.0;
        for (int k = 0; k < nz; k++) {
            const size_t j = (size_t)k * nx + i;
            double theta, zm;
            if (k == 0) {
                theta = (theta0 + th[j]) * 0.5;
                qv[j] = 0.0;
                zm = 0.0;
            } else {
                theta = (th[j - nx] + th[j]) * 0.5;
                qv[j] = qv[j - nx];
                zm = z[k - 1];
            }
            double qd = 1.0 - qv[j];
            double r = Rd * qd + Rv * qv[j];
            double cp = Cpd * qd + Cpv * qv[j];
            Pi = Pi - g * (z[k] - zm) / (cp * theta);
            double p_k = P0 * std::pow(Pi, cp / r);
            double T_k = ref[k] * Pi;
            rho[j] = p_k / (r * T_k);
            for (int it = 0; it < 10; it++) {
                const double qs = qsat_of(p_k, T_k, c);
                const double qv_new = std::max(0.0, RH_surf * std::exp(-z[k] / decay) * qs);
                qv[j] += 0.8 * (qv_new - qv[j]);
                qd = 1.0 - qv[j];
                r = Rd * qd + Rv * qv[j];
                cp = Cpd * qd + Cpv * qv[j];
                const double cv = cp - r;
                Pi = std::pow(rho[j] * r * th[j] / P0, r / cv);
                p_k = P0 * std::pow(Pi, cp / r);
                T_k = ref[k] * Pi;
                if (k > 0) {
                    const double l = p_k - p_km + g * (z[k] - z[k - 1]) * 0.5 * (rho[j - nx] + rho[j]);
                    const double dldr = cp / cv * p_k / rho[j] + g * (z[k] - z[k - 1]) * 0.5;
                    rho[j] -= l / dldr;
                }
            }
            p_km = p_k;
        }
    }
    Writer<T>(p, s).fill(rho, qv, th, u, ref);
    return MOIST_OK;
}

}  // namespace

extern "C" {
#pragma GCC visibility push(default)

int moist_uniform(uint32_t seed, uint32_t stream, int64_t n, const uint64_t* idx, double* out) {
    if (n < 0 || (n > 0 && !out)) return MOIST_ERR_ARG;
    for (int64_t j = 0; j < n; j++) out[j] = uniform01(seed, stream, idx ? idx[j] : (uint64_t)j);
    return MOIST_OK;
}

int moist_init_warm_bubble(const moist_params* p, int precision, uint32_t seed, moist_state_host* s) {
    if (!valid(p, precision, s)) return MOIST_ERR_ARG;
    return precision == MOIST_F64 ? warm_bubble_t<double>(p, seed, s) : warm_bubble_t<float>(p, seed, s);
}

int moist_init_sounding(const moist_params* p, int precision, const moist_bubble* bubbles, int nbubbles,
                        moist_state_host* s) {
    if (!valid(p, precision, s) || nbubbles < 0 || (nbubbles > 0 && !bubbles)) return MOIST_ERR_ARG;
    for (int j = 0; j < nbubbles; j++)
        if (!(bubbles[j].radius > 0.0)) return MOIST_ERR_ARG;
    return precision == MOIST_F64 ? sounding_t<double>(p, bubbles, nbubbles, s)
                                  : sounding_t<float>(p, bubbles, nbubbles, s);
}

int moist_sounding_bubble_row(uint32_t seed, int nbubbles, double lx, double amp_lo, double amp_hi,
                              double rad_lo, double rad_hi, double zc, moist_bubble* out) {
    if (nbubbles < 0 || (nbubbles > 0 && !out)) return MOIST_ERR_ARG;
    for (int j = 0; j < nbubbles; j++) {
        const double ua = uniform01(seed, 1, 2 * (uint64_t)j), ur = uniform01(seed, 1, 2 * (uint64_t)j + 1);
        out[j].xc = (j + 0.5) * lx / nbubbles;
        out[j].zc = zc;
        out[j].radius = rad_lo + (rad_hi - rad_lo) * ur;
        out[j].amp = amp_lo + (amp_hi - amp_lo) * ua;
    }
    return MOIST_OK;
}

int moist_ensemble_member_draw(uint32_t seed, int member, const int* nx_choices, int n_nx, const int* nz_choices,
                               int n_nz, double dx, double amp_lo, double amp_hi, double rad_lo, double rad_hi,
                               double zc, int* nx, int* nz, moist_bubble* bubble) {
    if (member < 0 || !nx_choices || !nz_choices || n_nx < 1 || n_nz < 1 || !nx || !nz || !bubble)
        return MOIST_ERR_ARG;
    double u[5];
    for (int j = 0; j < 5; j++) u[j] = uniform01(seed, 1000u + (uint32_t)member, (uint64_t)j);
    *nx = nx_choices[std::min((int)(u[0] * n_nx), n_nx - 1)];
    *nz = nz_choices[std::min((int)(u[1] * n_nz), n_nz - 1)];
    bubble->xc = u[2] * (*nx * dx);
    bubble->zc = zc;
    bubble->radius = rad_lo + (rad_hi - rad_lo) * u[4];
    bubble->amp = amp_lo + (amp_hi - amp_lo) * u[3];
    return MOIST_OK;
}

int moist_init_state(const moist_params* p, int precision, const moist_init_profile* profile, uint32_t seed,
                     moist_state_host* s) {
    if (!valid(p, precision, s) || !profile) return MOIST_ERR_ARG;
    return precision == MOIST_F64 ? init_state_t<double>(p, profile, seed, s)
                                  : init_state_t<float>(p, profile, seed, s);
}

#pragma GCC visibility pop
}  // extern "C"
