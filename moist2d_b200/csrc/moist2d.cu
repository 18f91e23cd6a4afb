// moist2d.cu - C-ABI of libmoist2d_sm100a.so: contexts, device buffers, step orchestration.
//
// A context owns one device-resident State in the [nz][P] interior layout (model.cuh) and
// every temporary of the large step; nothing is allocated while stepping. Entry points return
// after the work they queued on the context stream has finished.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../include/moist2d.h"
#include "kernels.cuh"
#include "batch.cuh"
#include "adjoint_batch.cuh"

using namespace moist;

namespace {

// the launches of one large step of a context, recorded instead of launched: per slot the
// launch kind and the bytes of its argument struct (batch.cuh)
struct StepRecord {
    std::vector<int> kind;
    std::vector<std::vector<unsigned char>> args;
    template <class A>
    void put(int k, const A& a) {
        kind.push_back(k);
        const unsigned char* b = reinterpret_cast<const unsigned char*>(&a);
        args.emplace_back(b, b + sizeof(A));
    }
};

struct CtxBase {
    virtual ~CtxBase() {}
    virtual int upload(const moist_state_host* s) = 0;
    virtual int download(moist_state_host* s) = 0;
    virtual int rk3(int nsteps) = 0;
    virtual int compute_step(const void* const phys[6], const moist_state_host* s0, double dt, int ns) = 0;
    virtual int microphysics() = 0;
    virtual int sedimentation(void* d_prec) = 0;
    virtual int surface_fluxes() = 0;
    virtual int gray_radiation() = 0;
    virtual int budget(double out[4]) = 0;
    virtual int time_steps(int nsteps, float* ms) = 0;
    virtual int profile(int nsteps, float* total_ms, float* group_ms, long long* group_launches) = 0;
    virtual int rk3_host(moist_state_host* s, int nsteps) = 0;
    virtual int pass_counts(int* counts, int n) = 0;
    virtual int set_wait_limit(long long cycles) = 0;
    virtual int set_tape_mode(int mode) = 0;
    virtual int pass_trace(int nsteps, int maxrec, long long* pass_ns, int* pass_tiles, int* npasses) = 0;
    virtual int adjoint_run(int nsteps, int ckpt, const moist_adjoint_seed* seed, moist_adjoint_grad* out) = 0;
    virtual int autotune(int nsteps, std::string& report) = 0;
    virtual int history(void* const out[MOIST_NDIAG], double summary[6]) = 0;
};

struct BatchBase {
    virtual ~BatchBase() {}
    virtual int step(int nsteps) = 0;
    virtual int adjoint(int nsteps, int ckpt, const moist_adjoint_seed* seeds, moist_adjoint_grad* out,
                        int nthreads) = 0;
    virtual int autotune(int nsteps, std::string& report) = 0;
    virtual int time_steps(int nsteps, float* ms) = 0;
    virtual int profile(int nsteps, float* total_ms, float* group_ms) = 0;
    virtual int set_tape_mode(int mode) = 0;
};

}  // namespace

struct moist_ctx {
    int device = 0;
    int precision = MOIST_F32;
    int flags = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    int nan_field = -1;
    CtxBase* impl = nullptr;
};

struct moist_batch {
    int device = 0;
    int precision = MOIST_F32;
    cudaStream_t stream = nullptr;
    std::vector<moist_ctx*> members;
    std::string err;
    int nan_member = -1, nan_field = -1;
    BatchBase* impl = nullptr;
};

namespace {

int set_err(moist_ctx* c, int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (c) c->err = buf;
    return code;
}

#define CK(call)                                                                                   \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess)                                                                     \
            return set_err(owner, MOIST_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

#define CKL()                                                                                           \
    do {                                                                                                \
        cudaError_t e_ = cudaGetLastError();                                                            \
        if (e_ != cudaSuccess)                                                                          \
            return set_err(owner, MOIST_ERR_CUDA, "kernel launch failed: %s", cudaGetErrorString(e_));  \
    } while (0)

inline unsigned cdiv(int a, int b) { return (unsigned)((a + b - 1) / b); }

#define SINGLE_ARG(...) __VA_ARGS__

template <class T>
DevParams<T> make_params(const moist_params* c, int P) {
    DevParams<T> p{};
    p.nx = c->nx;
    p.nz = c->nz;
    p.P = P;
    p.dx = (T)c->dx;
    p.dt = (T)c->dt;
    p.H = (T)c->h;
    p.nu = (T)c->nu;
    p.kappa = (T)c->kappa;
    p.gamma_d = (T)c->gamma_d;
    p.beta = (T)c->beta_offcenter;
    p.zf_sponge = (T)c->zf_sponge;
    p.EPS = (T)c->eps;
    p.GRAV = (T)c->grav;
    p.Rd = (T)c->rd;
    p.Rv = (T)c->rv;
    p.Cpd = (T)c->cpd;
    p.Cpv = (T)c->cpv;
    p.Cpl = (T)c->cpl;
    p.P0 = (T)c->p0;
    p.Lv = (T)c->lv;
    p.SIGMA = (T)c->sigma;
    p.EPSvap = (T)c->epsvap;
    p.K_auto = (T)c->k_auto;
    p.Qc_threshold = (T)c->qc_threshold;
    p.K_accr = (T)c->k_accr;
    p.K_evap = (T)c->k_evap;
    p.A_term = (T)c->a_term;
    p.B_term = (T)c->b_term;
    p.T0 = (T)c->t0;
    p.ES0 = (T)c->es0;
    p.A_SAT = (T)c->a_sat;
    p.B_SAT = (T)c->b_sat;
    p.Cd = (T)c->cd;
    p.Ch = (T)c->ch;
    p.Ce = (T)c->ce;
    p.uabs_min = (T)c->uabs_min;
    p.temp_surf = (T)c->temp_surf;
    p.k_abs_qv = (T)c->k_abs_qv;
    p.k_abs_qc = (T)c->k_abs_qc;
    p.k_abs_qr = (T)c->k_abs_qr;
    p.surf_emissivity = (T)c->surf_emissivity;
    p.tau_cooling = (T)c->tau_cooling;
    p.z_trop = (T)c->z_tropopause;
    p.do_mp = c->do_mp;
    p.do_auto = c->do_auto;
    p.do_accr = c->do_accr;
    p.do_revap = c->do_revap;
    p.do_sed = c->do_sed;
    p.do_rd = c->do_rd;
    p.do_sf = c->do_sf;
    return p;
}

// the parameters in double, each scalar as the context precision holds it (grid pointers unset)
template <class T>
DevParams<double> params_to_double(const DevParams<T>& q) {
    DevParams<double> p{};
    p.nx = q.nx;
    p.nz = q.nz;
    p.P = q.P;
#define PC(f) p.f = (double)q.f;
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
    return p;
}

template <class T, class TT>
struct Ctx : CtxBase {
    moist_ctx* owner;
    DevParams<T> dp;
    int nx, nz, halo, P, ns;
    size_t fsz;  // elements of one [nz][P] field
    cudaStream_t st;
    std::vector<void*> allocs;

    StateP<T> cur, nxt, s0b;
    T* tmpq[3];
    PhysP<T> ph;
    T *d_th_mp, *d_qv_mp, *d_qc_mp, *d_qr_mp, *d_qr_sed, *d_th_rd, *lw_up, *lw_dn;
    T *pres, *theta, *rt2p, *uface, *wface, *R_rho, *R_ru, *R_rw, *R_rt;
    T *rho_p, *ru_p[2], *rw_p, *rt_p[3], *mfx, *mfz, *ta, *tb, *tc;
    TT *tcp, *tpiv, *dprime;
    T *prec, *d_prec, *mflux, *shflux, *lhflux, *d_u_sf, *d_th_sf, *d_qv_sf, *theta_ref;
    T *halo_vals;  // [0] = rho_u[ks, is-1], [1] = rho[ks, ie+1] as of the last exchange
    T *g_dz, *g_z, *g_zf;
    double* g_trcp = nullptr;  // [nz][TEND_NRCP] reciprocals of the slow tendencies (kernels.cuh)
    T* staging;
    int* err;
    CSum* bud_part;   // [BUDGET_BLOCKS][4] block sums of the budgets
    double* bud_res;  // [4]
    bool rd_dirty = true;
    // tiled tracer sweep (tracer_tiles.cuh)
    bool use_tiles = false;
    bool tiles_df = false;  // the tiled sweep without grid barriers (per-tile versions)
    TileCtl tctl{};
    T* strips = nullptr;
    int* pass_hist = nullptr;  // [64] sweeps that converged after p passes
    size_t tile_smem = 0;
    // when set, launch_step records its launches here instead of launching them
    StepRecord* rec = nullptr;
    // row-streaming tracer sweep (MOIST_FLAG_TRACER_STREAM)
    bool use_stream = false;
    T* s_old[3] = {nullptr, nullptr, nullptr};
    double* rrho = nullptr;
    // column strips of the factorisation and the acoustic substeps
    int strip_wc = 1;
    size_t strip_smem = 0;
    // adjoint tape: when set, run_stage copies the stage internals the reverse sweep needs
    struct Tape {
        T* in[3][7];                           // stage inputs
        std::vector<std::array<T*, 4>> sub[3]; // rho_p, rho_u_p, rho_w_p, rho_theta_p after substep n (0: start)
        T* rrt[3];                             // R_rho_theta
        T* mf[3][2];                           // momentum fluxes after the substeps
        T* qout[3][3];                         // tracer sweep results
        T* sed;                                // d_rho_qr_sed of the step's physics
    };
    Tape* tape = nullptr;
    int tape_stage = 0;
    // buffers of moist_adjoint_run, allocated on its first call
    struct Adj {
        DevParams<double> pd;
        double *dz, *z, *zf;
        double *Lst[7], *LS0[7], *Lph[5], *seed[7];
        double* acc;  // 16 per-stage accumulators, contiguous (one memset)
        double *Lqout[3], *mu[3], *J, *LP[2][4];
        double *Ta, *Tb, *Tc, *Tcp, *Trd, *Lx, *Ly, *Ltp_rho, *Ltp_rt, *Linc_rho, *Linc_rt, *Lsed;
        double *Lpar, *obj, *prec_w, *stage;
        std::vector<Tape> tapes;             // one per step of a segment, or one
        std::vector<std::array<T*, 7>> ck;   // States every ckpt_every steps
        std::vector<std::array<T*, 7>> seg;  // the States of one segment (when one tape is kept)
        std::array<T*, 8> fin;               // the final State and prec
    };
    Adj* adj = nullptr;
    // profiling: events recorded before each kernel group when active
    bool prof_on = false;
    std::vector<cudaEvent_t> ev_pool;
    std::vector<int> ev_group;
    long long launches[MOIST_NGROUPS] = {0};

    // An event opens the interval of each group that follows a different one: consecutive
    // launches of one group (the substeps of a stage) share one interval, because every timing
    // event between kernels costs the stream several microseconds.
    int mark(int group, int nkernels, bool close = false) {
        launches[group] += nkernels;
        if (!prof_on) return MOIST_OK;
        if (!close && !ev_group.empty() && ev_group.back() == group) return MOIST_OK;
        const size_t j = ev_group.size();
        if (j >= ev_pool.size()) {
            cudaEvent_t e;
            CK(cudaEventCreate(&e));
            ev_pool.push_back(e);
        }
        CK(cudaEventRecord(ev_pool[j], st));
        ev_group.push_back(group);
        return MOIST_OK;
    }
#define MARK(g, n)                              \
    do {                                        \
        int m_ = mark((g), (n));                \
        if (m_ != MOIST_OK) return m_;          \
    } while (0)

    explicit Ctx(moist_ctx* o) : owner(o) {}

    ~Ctx() override {
        if (st) cudaStreamSynchronize(st);
        delete adj;
        for (cudaEvent_t e : ev_pool) cudaEventDestroy(e);
        for (void* a : allocs) cudaFree(a);
    }

    template <class U>
    int alloc(U** ptr, size_t n) {
        void* q = nullptr;
        cudaError_t e = cudaMalloc(&q, std::max<size_t>(n, 1) * sizeof(U));
        if (e != cudaSuccess) return set_err(owner, MOIST_ERR_NOMEM, "cudaMalloc of %zu bytes failed: %s", n * sizeof(U), cudaGetErrorString(e));
        allocs.push_back(q);
        *ptr = (U*)q;
        return MOIST_OK;
    }

#define AL(ptr, n)                               \
    do {                                         \
        int r_ = alloc(&(ptr), (n));             \
        if (r_ != MOIST_OK) return r_;           \
        CK(cudaMemsetAsync((ptr), 0, std::max<size_t>((n), 1) * sizeof(*(ptr)), st)); \
    } while (0)

    // device copies of nf whole fields (up to 8) in one launch
    // copies of whole fields (n = fsz) are recorded when rec is set (the adjoint's tape)
    int copyf(const T* const* src, T* const* dst, int nf, size_t n = 0) {
        if (n == 0) n = fsz;
        if (rec && n != fsz) return set_err(owner, MOIST_ERR_ARG, "a recorded copy covers whole fields");
        for (int f0 = 0; f0 < nf; f0 += 8) {
            CopyList<T> l{};
            l.nf = std::min(8, nf - f0);
            for (int j = 0; j < l.nf; j++) {
                l.src[j] = src[f0 + j];
                l.dst[j] = dst[f0 + j];
            }
            if (rec) {
                rec->put(BK_COPY, BCopy<T>{l, n, bz_blocks(fsz)});
                continue;
            }
            k_copy_fields<T><<<std::min<size_t>(1184, (n + 255) / 256), 256, 0, st>>>(l, n);
            CKL();
        }
        return MOIST_OK;
    }

    int init(const moist_params* c) {
        nx = c->nx;
        nz = c->nz;
        halo = c->halo;
        ns = c->ns;
        P = (nx + 31) / 32 * 32;
        fsz = (size_t)nz * P;
        st = owner->stream;
        dp = make_params<T>(c, P);
        for (T** f : {&cur.rho, &cur.ru, &cur.rw, &cur.rt, &cur.qv, &cur.qc, &cur.qr, &nxt.rho, &nxt.ru, &nxt.rw,
                      &nxt.rt, &nxt.qv, &nxt.qc, &nxt.qr, &tmpq[0], &tmpq[1], &tmpq[2], &ph.d_rho, &ph.d_u,
                      &ph.d_th, &ph.d_qv, &ph.d_qc, &ph.d_qr, &d_th_mp, &d_qv_mp, &d_qc_mp, &d_qr_mp, &d_qr_sed,
                      &d_th_rd, &pres, &theta, &rt2p, &uface, &wface, &R_rho, &R_ru, &R_rw, &R_rt, &rho_p,
                      &ru_p[0], &ru_p[1], &rw_p, &rt_p[0], &rt_p[1], &rt_p[2], &mfx, &mfz, &ta, &tb, &tc})
            AL(*f, fsz);
        s0b = StateP<T>{nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
        AL(lw_up, (size_t)(nz + 1) * P);
        AL(lw_dn, (size_t)(nz + 1) * P);
        AL(tcp, fsz);
        AL(tpiv, fsz);
        AL(dprime, fsz);
        for (T** f : {&prec, &d_prec, &mflux, &shflux, &lhflux, &d_u_sf, &d_th_sf, &d_qv_sf}) AL(*f, (size_t)P);
        AL(theta_ref, (size_t)nz);
        AL(halo_vals, 2);
        AL(g_dz, (size_t)nz);
        AL(g_z, (size_t)nz);
        AL(g_zf, (size_t)nz);
        AL(staging, (size_t)nz * (nx + 2 * halo) + 32);
        AL(err, 4);  // [0] halt (NaN field), [1] pending NaN field, [2] timeout, [3] spare
        AL(bud_part, (size_t)BUDGET_BLOCKS * 4);
        AL(bud_res, 4);
        CK(cudaMemcpyAsync(g_dz, c->dz, nz * sizeof(T), cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(g_z, c->z, nz * sizeof(T), cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(g_zf, c->zf, nz * sizeof(T), cudaMemcpyHostToDevice, st));
        dp.dz = g_dz;
        dp.z = g_z;
        dp.zf = g_zf;
        {
            // reciprocals of the slow tendencies' denominators, each formed in T as the kernels
            // form it, then inverted in double (IEEE, as the device would)
            const T* hdz = (const T*)c->dz;
            const T* hz = (const T*)c->z;
            std::vector<double> tab((size_t)nz * TEND_NRCP, 1.0);
            for (int k = 0; k < nz; k++) {
                double* r = &tab[(size_t)k * TEND_NRCP];
                r[TR_DX] = 1.0 / (double)dp.dx;
                r[TR_SIX] = 1.0 / 6.0;
                r[TR_DZ] = 1.0 / (double)hdz[k];
                if (k + 1 < nz) {
                    r[TR_DZ_KP1] = 1.0 / (double)hdz[k + 1];
                    r[TR_SUM_KP] = 1.0 / (double)(T)(hdz[k] + hdz[k + 1]);
                    r[TR_ZD_KP] = 1.0 / (double)(T)(hz[k + 1] - hz[k]);
                    r[TR_ZSUM] = 1.0 / (double)(T)(hz[k] + hz[k + 1]);
                }
                if (k >= 1) {
                    r[TR_SUM_KM] = 1.0 / (double)(T)(hdz[k - 1] + hdz[k]);
                    r[TR_ZD_KM] = 1.0 / (double)(T)(hz[k] - hz[k - 1]);
                }
            }
            AL(g_trcp, tab.size());
            CK(cudaMemcpyAsync(g_trcp, tab.data(), tab.size() * sizeof(double), cudaMemcpyHostToDevice, st));
            CK(cudaStreamSynchronize(st));  // tab is a host temporary
            dp.trcp = g_trcp;
        }
        if (int r = init_strips()) return r;
        if (owner->flags & MOIST_FLAG_TRACER_STREAM) {
            if (nz > STREAM_MAX_ROWS)
                return set_err(owner, MOIST_ERR_UNSUPPORTED, "the streaming tracer sweep needs nz <= %d (got %d)",
                               STREAM_MAX_ROWS, nz);
            for (int t = 0; t < 3; t++) AL(s_old[t], fsz);
            AL(rrho, fsz);
            use_stream = true;
        }
        if (int r = init_tiles()) return r;
        CK(reset_err());
        CK(cudaStreamSynchronize(st));
        return MOIST_OK;
    }

    cudaError_t reset_err() {
        const int v[4] = {INT_MAX, INT_MAX, 0, 0};
        return cudaMemcpyAsync(err, v, sizeof v, cudaMemcpyHostToDevice, st);
    }

    // Strip width: the widest of 8, 4, 2, 1 columns that still gives every SM a block and
    // keeps two blocks' shared memory on an SM; one column always fits (nz <= 1024).
    int init_strips() {
        int dev = 0, nsm = 0;
        CK(cudaGetDevice(&dev));
        CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        strip_wc = 1;
        for (int w : {8, 4, 2}) {
            if (cdiv(nx, w) >= nsm && strip_smem_bytes<T, TT>(nz, w) <= 96 * 1024) {
                strip_wc = w;
                break;
            }
        }
        strip_smem = strip_smem_bytes<T, TT>(nz, strip_wc);
        // the limit is a property of the kernel, shared by every context of the process (whose
        // strips differ, and a batch widens its members' strips): allow the device maximum, the
        // launch's own size sets the occupancy
        int optin = 0;
        CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
        CK(cudaFuncSetAttribute(k_thomas_strip<T, TT>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
        CK(cudaFuncSetAttribute(k_substep_strip<T, TT>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
        return MOIST_OK;
    }

    // The tiled sweep needs every tile resident at once (its passes meet at grid barriers);
    // otherwise, or when MOIST_FLAG_TRACER_WAVEFRONT is set, the exact wavefront runs instead.
    int init_tiles() {
        tctl.tiles_x = (nx + TT_W - 1) / TT_W;
        tctl.tiles_z = (nz + TT_W - 1) / TT_W;
        tctl.ntiles = tctl.tiles_x * tctl.tiles_z;
        tctl.max_pass = tctl.tiles_x + tctl.tiles_z + 2;
        tile_smem = sizeof(TileSmem<T>);
        if (owner->flags & (MOIST_FLAG_TRACER_WAVEFRONT | MOIST_FLAG_TRACER_STREAM)) return MOIST_OK;
        int dev = 0, nsm = 0, coop = 0, nb = 0;
        CK(cudaGetDevice(&dev));
        CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        CK(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
        CK(cudaFuncSetAttribute(k_tracer_tiles<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tile_smem));
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_tracer_tiles<T, false>, 96, tile_smem));
        if (!coop || (long)nb * nsm < tctl.ntiles) return MOIST_OK;
        // the barrier sweep uses two parities of strips, the dataflow sweep TT_RING versions
        AL(strips, (size_t)std::max(2, TT_RING) * 3 * tctl.ntiles * 4 * TT_W);
        AL(tctl.ver, (size_t)3 * tctl.ntiles);
        AL(tctl.bar, 2);
        AL(tctl.changed, (size_t)2 * 3 * tctl.ntiles * 2);
        AL(tctl.any_changed, (size_t)tctl.max_pass + 2);
        AL(tctl.passes, 1);
        AL(pass_hist, 64);
        tctl.pass_ts = nullptr;
        tctl.pass_work = nullptr;
        tctl.timeout = err + 2;
        int clk = 0;
        CK(cudaDeviceGetAttribute(&clk, cudaDevAttrClockRate, dev));  // kHz
        tctl.spin_limit = (long long)clk * 1000LL * 2;                 // about two seconds
        wait_default = tctl.spin_limit;
        use_tiles = true;
        tiles_df = (owner->flags & MOIST_FLAG_TRACER_DATAFLOW) != 0;
        CK(cudaFuncSetAttribute(k_tracer_tiles<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tile_smem));
        return MOIST_OK;
    }

    // finish: wait for the stream, read the NaN word
    int finish() {
        int h[4];
        CK(cudaMemcpyAsync(h, err, sizeof h, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        CKL();
        if (h[2] != 0) {
            // the blocks that gave up left the barrier words mid-count: clear them and the flag
            // so that the context can step again (from a State uploaded anew)
            if (tctl.bar) CK(cudaMemsetAsync(tctl.bar, 0, 2 * sizeof(unsigned), st));
            CK(reset_err());
            CK(cudaStreamSynchronize(st));
            return set_err(owner, MOIST_ERR_TIMEOUT, "a grid barrier of the tiled tracer sweep timed out");
        }
        if (h[0] != INT_MAX) {
            owner->nan_field = h[0];
            static const char* names[12] = {"rho", "rho_u", "rho_w", "rho_theta", "rho_qv", "rho_qc", "rho_qr",
                                            "d_rho_u_phys", "d_rho_theta_phys", "d_rho_qv_phys", "d_rho_qc_phys",
                                            "d_rho_qr_phys"};
            return set_err(owner, MOIST_ERR_NAN, "NaN detected in %s", h[0] >= 0 && h[0] < 12 ? names[h[0]] : "?");
        }
        owner->nan_field = -1;
        return MOIST_OK;
    }

    // ------------------------------------------------------------------ layout moves
    // The device address of a host array the kernels can read and write directly (page-locked
    // and mapped: cudaHostAlloc or cudaHostRegister memory under unified addressing), else null.
    static void* mapped(const void* host) {
        cudaPointerAttributes at;
        if (!host || cudaPointerGetAttributes(&at, host) != cudaSuccess) {
            cudaGetLastError();  // pageable memory may report an error on older runtimes: clear it
            return nullptr;
        }
        return at.type == cudaMemoryTypeHost ? at.devicePointer : nullptr;
    }

    // the prognostic fields of a host State in one launch when every given array is mapped
    // (done = false, and nothing moved, otherwise)
    int put2d_mapped(const void* const host[7], T* const dev[7], bool& done) {
        done = false;
        FieldSet<T> fs{};
        int nf = 0;
        for (int j = 0; j < 7; j++) {
            if (!host[j]) continue;
            const void* hd = mapped(host[j]);
            if (!hd) return MOIST_OK;
            fs.src[nf] = (const T*)hd;
            fs.dst[nf] = dev[j];
            nf++;
        }
        if (nf == 0) return MOIST_OK;
        k_from_ref_n<T><<<dim3(cdiv(nz, 32), cdiv(nx, 32), nf), dim3(32, 8), 0, st>>>(nx, nz, halo, P, fs);
        CKL();
        done = true;
        return MOIST_OK;
    }
    int get2d_mapped(const T* const dev[7], void* const host[7], bool& done) {
        done = false;
        FieldSet<T> fs{};
        int nf = 0;
        for (int j = 0; j < 7; j++) {
            if (!host[j]) continue;
            void* hd = mapped(host[j]);
            if (!hd) return MOIST_OK;
            fs.src[nf] = dev[j];
            fs.dst[nf] = (T*)hd;
            nf++;
        }
        if (nf == 0) return MOIST_OK;
        const int ia = nx + 2 * halo;
        k_to_ref_n<T><<<dim3(cdiv(nz, 32), cdiv(ia, 32), nf), dim3(32, 8), 0, st>>>(nx, nz, halo, P, fs);
        CKL();
        done = true;
        return MOIST_OK;
    }

    int put2d(const void* host, T* dev) {
        if (!host) return MOIST_OK;
        if (const void* hd = mapped(host)) {
            dim3 b(32, 8), g(cdiv(nz, 32), cdiv(nx, 32));
            k_from_ref<T><<<g, b, 0, st>>>(nx, nz, halo, P, (const T*)hd, dev);
            CKL();
            return MOIST_OK;
        }
        const size_t n = (size_t)nz * (nx + 2 * halo);
        CK(cudaMemcpyAsync(staging, host, n * sizeof(T), cudaMemcpyHostToDevice, st));
        dim3 b(32, 8), g(cdiv(nz, 32), cdiv(nx, 32));
        k_from_ref<T><<<g, b, 0, st>>>(nx, nz, halo, P, staging, dev);
        CKL();
        return MOIST_OK;
    }
    int get2d(const T* dev, void* host, bool halos) {
        if (!host) return MOIST_OK;
        const int ia = nx + 2 * halo;
        const size_t n = (size_t)nz * ia;
        if (void* hd = mapped(host)) {  // written in place: the caller's halo columns stay as they are
            dim3 b(32, 8), g(cdiv(nz, 32), cdiv(halos ? ia : nx, 32));
            if (halos)
                k_to_ref<T><<<g, b, 0, st>>>(nx, nz, halo, P, dev, (T*)hd);
            else
                k_to_ref<T><<<g, b, 0, st>>>(nx, nz, 0, P, dev, (T*)hd + (size_t)halo * nz);
            CKL();
            return MOIST_OK;
        }
        if (!halos) {  // keep the caller's halo columns: start from their current values
            CK(cudaMemcpyAsync(staging, host, n * sizeof(T), cudaMemcpyHostToDevice, st));
        }
        dim3 b(32, 8), g(cdiv(nz, 32), cdiv(halos ? ia : nx, 32));
        if (halos) {
            k_to_ref<T><<<g, b, 0, st>>>(nx, nz, halo, P, dev, staging);
        } else {
            // interior only: write columns halo .. halo+nx-1 through an offset view
            k_to_ref<T><<<g, b, 0, st>>>(nx, nz, 0, P, dev, staging + (size_t)halo * nz);
        }
        CKL();
        CK(cudaMemcpyAsync(host, staging, n * sizeof(T), cudaMemcpyDeviceToHost, st));
        return MOIST_OK;
    }
    int put1dx(const void* host, T* dev) {
        if (!host) return MOIST_OK;
        CK(cudaMemcpyAsync(dev, (const T*)host + halo, nx * sizeof(T), cudaMemcpyHostToDevice, st));
        return MOIST_OK;
    }
    int get1dx(const T* dev, void* host) {
        if (!host) return MOIST_OK;
        CK(cudaMemcpyAsync((T*)host + halo, dev, nx * sizeof(T), cudaMemcpyDeviceToHost, st));
        return MOIST_OK;
    }

    int upload(const moist_state_host* s) override {
        int r = queue_upload(s);
        if (r != MOIST_OK) return r;
        CK(cudaStreamSynchronize(st));
        return MOIST_OK;
    }

    // queue the copies and layout moves of a host State on the stream (no synchronisation;
    // stream order keeps the single staging buffer consistent)
    int queue_upload(const moist_state_host* s) {
        int r;
        StateP<T>& d = cur;
        const void* f2[7] = {s->rho, s->rho_u, s->rho_w, s->rho_theta, s->rho_qv, s->rho_qc, s->rho_qr};
        T* dv[7] = {d.rho, d.ru, d.rw, d.rt, d.qv, d.qc, d.qr};
        bool done = false;
        if ((r = put2d_mapped(f2, dv, done)) != MOIST_OK) return r;
        for (int j = 0; j < 7 && !done; j++)
            if ((r = put2d(f2[j], dv[j])) != MOIST_OK) return r;
        const void* g2[6] = {s->d_rho_theta_mp, s->d_rho_qv_mp, s->d_rho_qc_mp, s->d_rho_qr_mp, s->d_rho_qr_sed,
                             s->d_rho_theta_rd};
        T* gv[6] = {d_th_mp, d_qv_mp, d_qc_mp, d_qr_mp, d_qr_sed, d_th_rd};
        for (int j = 0; j < 6; j++)
            if ((r = put2d(g2[j], gv[j])) != MOIST_OK) return r;
        if (s->d_rho_theta_rd) rd_dirty = true;
        const void* f1[8] = {s->prec, s->mflux, s->shflux, s->lhflux, s->d_rho_u_sf, s->d_rho_theta_sf,
                             s->d_rho_qv_sf, nullptr};
        T* d1[8] = {prec, mflux, shflux, lhflux, d_u_sf, d_th_sf, d_qv_sf, nullptr};
        for (int j = 0; j < 7; j++)
            if ((r = put1dx(f1[j], d1[j])) != MOIST_OK) return r;
        if (s->theta_ref) CK(cudaMemcpyAsync(theta_ref, s->theta_ref, nz * sizeof(T), cudaMemcpyHostToDevice, st));
        // halo values the surface fluxes read before the next exchange (moist.jl:723, 736)
        if (halo >= 1) {
            if (s->rho_u) CK(cudaMemcpyAsync(halo_vals, (const T*)s->rho_u + (size_t)(halo - 1) * nz, sizeof(T), cudaMemcpyHostToDevice, st));
            if (s->rho) CK(cudaMemcpyAsync(halo_vals + 1, (const T*)s->rho + (size_t)(nx + halo) * nz, sizeof(T), cudaMemcpyHostToDevice, st));
        }
        return MOIST_OK;
    }

    int download(moist_state_host* s) override {
        int r = queue_download(s);
        if (r != MOIST_OK) return r;
        CK(cudaStreamSynchronize(st));
        return MOIST_OK;
    }

    int queue_download(moist_state_host* s) {
        int r;
        void* f2[7] = {s->rho, s->rho_u, s->rho_w, s->rho_theta, s->rho_qv, s->rho_qc, s->rho_qr};
        const T* dv[7] = {cur.rho, cur.ru, cur.rw, cur.rt, cur.qv, cur.qc, cur.qr};
        bool done = false;
        if ((r = get2d_mapped(dv, f2, done)) != MOIST_OK) return r;
        for (int j = 0; j < 7 && !done; j++) {
            if ((r = get2d(dv[j], f2[j], true)) != MOIST_OK) return r;
        }
        void* g2[6] = {s->d_rho_theta_mp, s->d_rho_qv_mp, s->d_rho_qc_mp, s->d_rho_qr_mp, s->d_rho_qr_sed,
                       s->d_rho_theta_rd};
        T* gv[6] = {d_th_mp, d_qv_mp, d_qc_mp, d_qr_mp, d_qr_sed, d_th_rd};
        for (int j = 0; j < 6; j++) {
            if ((r = get2d(gv[j], g2[j], false)) != MOIST_OK) return r;
        }
        void* f1[7] = {s->prec, s->mflux, s->shflux, s->lhflux, s->d_rho_u_sf, s->d_rho_theta_sf, s->d_rho_qv_sf};
        T* d1[7] = {prec, mflux, shflux, lhflux, d_u_sf, d_th_sf, d_qv_sf};
        for (int j = 0; j < 7; j++)
            if ((r = get1dx(d1[j], f1[j])) != MOIST_OK) return r;
        if (s->theta_ref) CK(cudaMemcpyAsync(s->theta_ref, theta_ref, nz * sizeof(T), cudaMemcpyDeviceToHost, st));
        return MOIST_OK;
    }

    // ------------------------------------------------------------------ the large step
    int launch_physics(int mode) {  // mode bit 1: microphysics, bit 2: sedimentation, 4: full step
        const dim3 b(32, 8), g(cdiv(nx, 32), cdiv(nz, 8));
        const bool full = mode & 4;
        MARK(MOIST_KGROUP_PHYSICS, 1 + (full && dp.do_sf) + (full && dp.do_rd));
        if (full) {
            if (dp.do_sf) {
                if (rec) {
                    rec->put(BK_SF, BSf<T>{dp, cur, halo_vals, halo_vals + 1, d_u_sf, d_th_sf, d_qv_sf, mflux, shflux,
                                           lhflux, err});
                } else {
                    k_surface_fluxes<T><<<cdiv(nx, 128), 128, 0, st>>>(dp, cur, halo_vals, halo_vals + 1, d_u_sf,
                                                                      d_th_sf, d_qv_sf, mflux, shflux, lhflux, err);
                    CKL();
                }
            } else {
                for (T* f : {d_u_sf, d_th_sf, d_qv_sf, mflux, shflux, lhflux}) {
                    if (rec)
                        rec->put(BK_MEMSET, BMemset{f, P * sizeof(T)});
                    else
                        CK(cudaMemsetAsync(f, 0, P * sizeof(T), st));
                }
            }
            if (dp.do_rd) {
                if (rec) {
                    rec->put(BK_RD, BRd<T>{dp, cur, theta_ref, lw_up, lw_dn, d_th_rd, err});
                } else {
                    k_gray_radiation<T><<<cdiv(nx, 128), 128, 0, st>>>(dp, cur, theta_ref, lw_up, lw_dn, d_th_rd, err);
                    CKL();
                }
                rd_dirty = true;
            } else if (rec) {  // a recorded step clears every time: uploads may come between steps
                rec->put(BK_MEMSET, BMemset{d_th_rd, fsz * sizeof(T)});
            } else if (rd_dirty) {
                CK(cudaMemsetAsync(d_th_rd, 0, fsz * sizeof(T), st));
                rd_dirty = false;
            }
        }
        DevParams<T> q = dp;
        if (!full) {  // the unit entry points ignore the process switches checked by rk3_step!
            q.do_mp = 1;
            q.do_sed = 1;
        }
        if (rec) {
            rec->put(BK_PHYS, BPhys<T>{q, cur, d_th_mp, d_qv_mp, d_qc_mp, d_qr_mp, d_qr_sed, d_prec, d_th_rd, d_u_sf,
                                       d_th_sf, d_qv_sf, ph, err});
            return MOIST_OK;
        }
        k_physics<T><<<g, b, 0, st>>>(q, cur, d_th_mp, d_qv_mp, d_qc_mp, d_qr_mp, d_qr_sed, d_prec, d_th_rd, d_u_sf,
                                      d_th_sf, d_qv_sf, ph, err);
        CKL();
        return MOIST_OK;
    }

    int run_stage(StateP<T> s_in, StateP<T> s0, T* const qout[3], StateP<T> s_out, T dt_stage, int ns_s) {
        const dim3 b2(32, 8), g2(cdiv(nx, 32), cdiv(nz, 8));
        const int js = tape_stage;
        if (tape) {
            const T* src[7] = {s_in.rho, s_in.ru, s_in.rw, s_in.rt, s_in.qv, s_in.qc, s_in.qr};
            if (int r = copyf(src, tape->in[js], 7)) return r;
        }
        MARK(MOIST_KGROUP_PROLOGUE, 3);
        TendArgs<T> ta_{s_in, s0, ph, pres, theta, uface, wface, R_rho, R_ru, R_rw, R_rt, rho_p, ru_p[0], rw_p,
                        rt_p[0], mfx, mfz, halo_vals, halo_vals + 1};
        const T dt_s = dt_stage / T(ns_s);
        const unsigned gs = cdiv(nx, strip_wc);
        if (rec) {
            rec->put(BK_DIAG, BDiag<T>{dp, s_in, pres, theta, rt2p, uface, wface, err});
            rec->put(BK_TEND, BTend<T>{dp, ta_, err});
            rec->put(BK_THOMAS, BThomas<T, TT>{dp, theta, rt2p, dt_s, strip_wc, ta, tb, tc, tcp, tpiv, err});
        } else {
            k_diag<T><<<g2, b2, 0, st>>>(dp, s_in, pres, theta, rt2p, uface, wface, err);
            CKL();
            k_tend<T><<<g2, b2, 0, st>>>(dp, ta_, err);
            CKL();
            k_thomas_strip<T, TT><<<gs, STRIP_THREADS, strip_smem, st>>>(dp, theta, rt2p, dt_s, strip_wc, ta, tb, tc,
                                                                         tcp, tpiv, err);
            CKL();
        }
        if (tape) {
            const T* src[5] = {rho_p, ru_p[0], rw_p, rt_p[0], R_rt};
            T* dst[5] = {tape->sub[js][0][0], tape->sub[js][0][1], tape->sub[js][0][2], tape->sub[js][0][3],
                         tape->rrt[js]};
            if (int r = copyf(src, dst, 5)) return r;
        }
        const double fact_tp64 = (double)T(0.5) * (1.0 + (double)dp.beta);
        for (int n = 1; n <= ns_s; n++) {
            MARK(MOIST_KGROUP_SUBSTEP, 1);
            SubArgs<T, TT> sa;
            sa.R_rho = R_rho;
            sa.R_ru = R_ru;
            sa.R_rw = R_rw;
            sa.R_rt = R_rt;
            sa.theta = theta;
            sa.rt2pres = rt2p;
            sa.s_rw = s_in.rw;
            sa.ru_in = ru_p[(n - 1) % 2];
            sa.ru_out = ru_p[n % 2];
            sa.rt_in = rt_p[(n - 1) % 3];
            sa.rt_old = rt_p[n >= 2 ? (n - 2) % 3 : 0];
            sa.rt_out = rt_p[n % 3];
            sa.rho_p = rho_p;
            sa.rw_p = rw_p;
            sa.mfx = mfx;
            sa.mfz = mfz;
            sa.ta = ta;
            sa.tb = tb;
            sa.tc = tc;
            sa.tcp = tcp;
            sa.tpiv = tpiv;
            sa.dprime = dprime;
            if (rec) {
                rec->put(BK_SUB, BSub<T, TT>{dp, sa, dt_s, T(ns_s), fact_tp64, strip_wc, err});
            } else {
                k_substep_strip<T, TT><<<gs, STRIP_THREADS, strip_smem, st>>>(dp, sa, dt_s, T(ns_s), fact_tp64,
                                                                              strip_wc, err);
                CKL();
            }
            if (tape) {
                const T* src[4] = {rho_p, ru_p[n % 2], rw_p, rt_p[n % 3]};
                if (int r = copyf(src, tape->sub[js][n].data(), 4)) return r;
            }
        }
        if (tape) {
            const T* src[2] = {mfx, mfz};
            if (int r = copyf(src, tape->mf[js], 2)) return r;
        }
        TracerArgs<T> tr;
        const T* qin[3] = {s_in.qv, s_in.qc, s_in.qr};
        const T* q0[3] = {s0.qv, s0.qc, s0.qr};
        const T* dq[3] = {ph.d_qv, ph.d_qc, ph.d_qr};
        for (int j = 0; j < 3; j++) {
            tr.q_old[j] = qin[j];
            tr.q_new[j] = qout[j];
            tr.q0[j] = q0[j];
            tr.dphys[j] = dq[j];
        }
        tr.rho = s_in.rho;
        tr.mfx = mfx;
        tr.mfz = mfz;
        tr.dt = dt_stage;
        MARK(MOIST_KGROUP_TRACER, (use_stream || use_tiles) ? 2 : 1);
        if (use_stream) {
            StreamArgs<T> sa{tr, {s_old[0], s_old[1], s_old[2]}, rrho};
            if (rec) {
                rec->put(BK_PREP, BPrep<T>{dp, tr, s_old[0], s_old[1], s_old[2], rrho, err});
                rec->put(BK_STREAM, BStream<T>{dp, sa, err});
            } else {
                k_stream_prep<T><<<g2, b2, 0, st>>>(dp, tr, s_old[0], s_old[1], s_old[2], rrho, err);
                CKL();
                k_tracer_stream<T><<<3, (nz + 31) / 32 * 32, 0, st>>>(dp, sa, err);
                CKL();
            }
        } else if (rec) {
            return set_err(owner, MOIST_ERR_UNSUPPORTED, "a recorded step needs the streaming tracer sweep");
        } else if (use_tiles) {
            CK(cudaMemsetAsync(tctl.any_changed, 0, (tctl.max_pass + 2) * sizeof(int), st));
            TileCtl c = tctl;
            if (trace_ts && trace_n < trace_cap) {  // moist_tracer_pass_trace
                const size_t stride = (size_t)tctl.max_pass + 3;
                c.pass_ts = trace_ts + trace_n * stride;
                c.pass_work = trace_work + trace_n * stride;
                trace_n++;
            }
            T* sp = strips;
            int* e = err;
            void* args[] = {&dp, &tr, &c, &sp, &e};
            if (tiles_df) {
                CK(cudaMemsetAsync(tctl.ver, 0, (size_t)3 * tctl.ntiles * sizeof(int), st));
                CK(cudaMemsetAsync(tctl.passes, 0, sizeof(int), st));
                CK(cudaLaunchCooperativeKernel((void*)k_tracer_tiles<T, true>, dim3(tctl.ntiles), dim3(96), args,
                                               tile_smem, st));
            } else {
                CK(cudaLaunchCooperativeKernel((void*)k_tracer_tiles<T, false>, dim3(tctl.ntiles), dim3(96), args,
                                               tile_smem, st));
            }
            k_pass_count<<<1, 1, 0, st>>>(tctl.passes, pass_hist);
            CKL();
        } else {
            const int nthr = (nz + 31) / 32 * 32;
            k_tracer_wavefront<T><<<3, nthr, 3 * nz * sizeof(T), st>>>(dp, tr, err);
            CKL();
        }
        if (tape) {
            const T* src[3] = {qout[0], qout[1], qout[2]};
            if (int r = copyf(src, tape->qout[js], 3)) return r;
        }
        MARK(MOIST_KGROUP_UPDATE, 2);
        UpdArgs<T> ua{s_in, s_out, rho_p, ru_p[ns_s % 2], rw_p, rt_p[ns_s % 3], ph};
        if (rec) {
            rec->put(BK_UPD, BUpd<T>{dp, ua, err});
            rec->put(BK_STAGE_END, BStageEnd{err});
            return MOIST_OK;
        }
        k_update<T><<<g2, b2, 0, st>>>(dp, ua, err);
        CKL();
        k_stage_end<<<1, 1, 0, st>>>(err);
        CKL();
        return MOIST_OK;
    }

    static StateP<T> with_q(StateP<T> s, T* const q[3]) {
        s.qv = q[0];
        s.qc = q[1];
        s.qr = q[2];
        return s;
    }

    int launch_step() {
        int r;
        if ((r = launch_physics(4)) != MOIST_OK) return r;
        if (tape) {
            const T* src[1] = {d_qr_sed};
            if ((r = copyf(src, &tape->sed, 1)) != MOIST_OK) return r;
        }
        const T dt = dp.dt;
        const int ns1 = std::max(1, (int)std::ceil(ns / 3.0));
        const int ns2 = std::max(1, (int)std::ceil(ns / 2.0));
        T* const nq[3] = {nxt.qv, nxt.qc, nxt.qr};
        tape_stage = 0;
        if ((r = run_stage(cur, cur, nq, nxt, dt / T(3), ns1)) != MOIST_OK) return r;
        tape_stage = 1;
        if ((r = run_stage(nxt, cur, tmpq, with_q(nxt, tmpq), dt / T(2), ns2)) != MOIST_OK) return r;
        tape_stage = 2;
        if ((r = run_stage(with_q(nxt, tmpq), cur, nq, nxt, dt, ns)) != MOIST_OK) return r;
        MARK(MOIST_KGROUP_OTHER, 1);
        if (rec) {
            rec->put(BK_PREC, BPrec<T>{dp, prec, d_prec, err});
        } else {
            k_prec<T><<<cdiv(nx, 128), 128, 0, st>>>(dp, prec, d_prec, err);
            CKL();
        }
        std::swap(cur, nxt);
        return MOIST_OK;
    }

    int check_stage_shape() {
        if (halo != 2 || nx < 2)
            return set_err(owner, MOIST_ERR_ARG, "the RK stages need halo = 2 and nx >= 2 (got halo = %d, nx = %d)",
                           halo, nx);
        return MOIST_OK;
    }

    int rk3(int nsteps) override {
        if (int r = check_stage_shape()) return r;
        CK(reset_err());
        for (int n = 0; n < nsteps; n++) {
            int r = launch_step();
            if (r != MOIST_OK) return r;
        }
        return finish();
    }

    int time_steps(int nsteps, float* ms) override {
        if (int r = check_stage_shape()) return r;
        cudaEvent_t e0, e1;
        CK(cudaEventCreate(&e0));
        CK(cudaEventCreate(&e1));
        CK(reset_err());
        CK(cudaEventRecord(e0, st));
        for (int n = 0; n < nsteps; n++) {
            int r = launch_step();
            if (r != MOIST_OK) return r;
        }
        CK(cudaEventRecord(e1, st));
        CK(cudaEventSynchronize(e1));
        CK(cudaEventElapsedTime(ms, e0, e1));
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        return finish();
    }

    int profile(int nsteps, float* total_ms, float* group_ms, long long* group_launches) override {
        if (int r = check_stage_shape()) return r;
        CK(reset_err());
        for (int g = 0; g < MOIST_NGROUPS; g++) launches[g] = 0;
        ev_group.clear();
        prof_on = true;
        int r = MOIST_OK;
        for (int n = 0; n < nsteps && r == MOIST_OK; n++) r = launch_step();
        if (r == MOIST_OK) r = mark(MOIST_KGROUP_OTHER, 0, true);  // closes the last interval
        prof_on = false;
        if (r != MOIST_OK) return r;
        CK(cudaStreamSynchronize(st));
        for (int g = 0; g < MOIST_NGROUPS; g++) {
            if (group_ms) group_ms[g] = 0.f;
            if (group_launches) group_launches[g] = launches[g];
        }
        float tot = 0.f;
        for (size_t j = 0; j + 1 < ev_group.size(); j++) {
            float ms = 0.f;
            CK(cudaEventElapsedTime(&ms, ev_pool[j], ev_pool[j + 1]));
            if (group_ms) group_ms[ev_group[j]] += ms;
            tot += ms;
        }
        if (total_ms) *total_ms = tot;
        return finish();
    }

    // moist_tracer_pass_trace: per-sweep pass timestamps and working tiles
    unsigned long long* trace_ts = nullptr;
    int* trace_work = nullptr;
    int trace_n = 0, trace_cap = 0;
    int pass_trace(int nsteps, int maxrec, long long* pass_ns, int* pass_tiles, int* npasses) override {
        if (int r = check_stage_shape()) return r;
        if (!use_tiles) return set_err(owner, MOIST_ERR_UNSUPPORTED, "the tiled tracer sweep is not in use");
        const size_t stride = (size_t)tctl.max_pass + 3, nsw = (size_t)3 * nsteps;
        unsigned long long* ts = nullptr;
        int* wk = nullptr;
        CK(cudaMalloc(&ts, nsw * stride * sizeof(unsigned long long)));
        CK(cudaMalloc(&wk, nsw * stride * sizeof(int)));
        CK(cudaMemsetAsync(ts, 0, nsw * stride * sizeof(unsigned long long), st));
        CK(cudaMemsetAsync(wk, 0, nsw * stride * sizeof(int), st));
        trace_ts = ts;
        trace_work = wk;
        trace_n = 0;
        trace_cap = (int)nsw;
        CK(reset_err());
        int r = MOIST_OK;
        for (int n = 0; n < nsteps && r == MOIST_OK; n++) r = launch_step();
        trace_ts = nullptr;
        trace_work = nullptr;
        std::vector<unsigned long long> hts(nsw * stride);
        std::vector<int> hwk(nsw * stride);
        CK(cudaMemcpyAsync(hts.data(), ts, hts.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(hwk.data(), wk, hwk.size() * sizeof(int), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        cudaFree(ts);
        cudaFree(wk);
        if (r != MOIST_OK) return r;
        // per sweep: the passes run, each pass's duration (start of the next pass, or block 0
        // leaving, minus its start) and the tile-tracer warps that recomputed in it
        for (size_t w = 0; w < nsw; w++) {
            const unsigned long long* t = &hts[w * stride];
            const int* k = &hwk[w * stride];
            int np = 0;
            while (np + 1 <= tctl.max_pass && t[np + 1] != 0) np++;
            if (npasses) npasses[w] = np;
            for (int q = 0; q < maxrec; q++) {
                long long d = 0;
                if (q + 1 <= np) {
                    const unsigned long long t1 = (q + 2 <= np) ? t[q + 2] : t[tctl.max_pass + 2];
                    d = (long long)(t1 - t[q + 1]);
                }
                if (pass_ns) pass_ns[w * maxrec + q] = d;
                if (pass_tiles) pass_tiles[w * maxrec + q] = (q + 1 <= np) ? k[q + 1] : 0;
            }
        }
        return finish();
    }

    // bound of every device-side wait of the context's kernels, in SM clock cycles (<= 0: the
    // default of about two seconds)
    long long wait_default = 0;
    int tape_mode = -1;  // moist_set_adjoint_tapes
    int set_tape_mode(int mode) override {
        tape_mode = mode;
        return MOIST_OK;
    }

    int set_wait_limit(long long cycles) override {
        if (!use_tiles)
            return set_err(owner, MOIST_ERR_UNSUPPORTED, "the context runs no kernel that waits on other blocks");
        tctl.spin_limit = cycles > 0 ? cycles : wait_default;
        return MOIST_OK;
    }

    int pass_counts(int* counts, int n) override {
        int h[64] = {0};
        if (use_tiles) {
            CK(cudaMemcpyAsync(h, pass_hist, sizeof h, cudaMemcpyDeviceToHost, st));
            CK(cudaMemsetAsync(pass_hist, 0, sizeof h, st));
            CK(cudaStreamSynchronize(st));
        }
        for (int j = 0; j < n; j++) counts[j] = j < 64 ? h[j] : 0;
        return use_tiles ? MOIST_OK : set_err(owner, MOIST_ERR_UNSUPPORTED, "the tiled tracer sweep is not in use");
    }

    int rk3_host(moist_state_host* s, int nsteps) override {
        if (int r = check_stage_shape()) return r;
        int r = queue_upload(s);
        if (r != MOIST_OK) return r;
        CK(reset_err());
        for (int n = 0; n < nsteps && r == MOIST_OK; n++) r = launch_step();
        if (r != MOIST_OK) return r;
        r = queue_download(s);
        if (r != MOIST_OK) return r;
        return finish();
    }

    int compute_step(const void* const phys[6], const moist_state_host* s0, double dt, int ns_s) override {
        if (ns_s < 1) return set_err(owner, MOIST_ERR_ARG, "ns must be >= 1");
        if (int r0 = check_stage_shape()) return r0;
        int r;
        if (!s0b.rho) {
            for (T** f : {&s0b.rho, &s0b.ru, &s0b.rw, &s0b.rt, &s0b.qv, &s0b.qc, &s0b.qr}) AL(*f, fsz);
        }
        const void* f2[7] = {s0->rho, s0->rho_u, s0->rho_w, s0->rho_theta, s0->rho_qv, s0->rho_qc, s0->rho_qr};
        T* dv[7] = {s0b.rho, s0b.ru, s0b.rw, s0b.rt, s0b.qv, s0b.qc, s0b.qr};
        for (int j = 0; j < 7; j++) {
            if (!f2[j]) return set_err(owner, MOIST_ERR_ARG, "s0 field %d is NULL", j);
            if ((r = put2d(f2[j], dv[j])) != MOIST_OK) return r;
        }
        T* pv[6] = {ph.d_rho, ph.d_u, ph.d_th, ph.d_qv, ph.d_qc, ph.d_qr};
        for (int j = 0; j < 6; j++) {
            if (!phys[j]) return set_err(owner, MOIST_ERR_ARG, "phys field %d is NULL", j);
            if ((r = put2d(phys[j], pv[j])) != MOIST_OK) return r;
        }
        CK(reset_err());
        T* const nq[3] = {nxt.qv, nxt.qc, nxt.qr};
        if ((r = run_stage(cur, s0b, nq, nxt, (T)dt, ns_s)) != MOIST_OK) return r;
        std::swap(cur, nxt);
        return finish();
    }

    int microphysics() override {
        CK(reset_err());
        int r = launch_physics(1);
        if (r != MOIST_OK) return r;
        return finish();
    }

    int sedimentation(void* host_d_prec) override {
        CK(reset_err());
        int r = launch_physics(2);
        if (r != MOIST_OK) return r;
        if (host_d_prec) {
            std::vector<T> tmp(nx + 2 * halo, T(0));
            CK(cudaMemcpyAsync(tmp.data() + halo, d_prec, nx * sizeof(T), cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            std::memcpy((T*)host_d_prec + halo, tmp.data() + halo, nx * sizeof(T));
        }
        return finish();
    }

    // surface_fluxes! (moist.jl:710-752) on the current state alone: the halo reads
    // rho_u[ks, is-1] and rho[ks, ie+1] are the uploaded halo columns (or the last exchange's)
    int surface_fluxes() override {
        if (halo < 1) return set_err(owner, MOIST_ERR_ARG, "surface_fluxes! reads one halo column: halo >= 1");
        CK(reset_err());
        k_surface_fluxes<T><<<cdiv(nx, 128), 128, 0, st>>>(dp, cur, halo_vals, halo_vals + 1, d_u_sf, d_th_sf,
                                                          d_qv_sf, mflux, shflux, lhflux, err);
        CKL();
        return finish();
    }

    // gray_radiation! (moist.jl:776-840) on the current state alone, with the uploaded theta_ref
    int gray_radiation() override {
        CK(reset_err());
        k_gray_radiation<T><<<cdiv(nx, 128), 128, 0, st>>>(dp, cur, theta_ref, lw_up, lw_dn, d_th_rd, err);
        CKL();
        rd_dirty = true;
        return finish();
    }

    // compensated FP64 domain budgets of the current state (kernels.cuh, k_budget)
    int budget(double out[4]) override {
        k_budget<T><<<BUDGET_BLOCKS, BUDGET_THREADS, 0, st>>>(dp, cur, prec, bud_part);
        CKL();
        k_budget_final<<<1, 32, 0, st>>>(bud_part, bud_res);
        CKL();
        CK(cudaMemcpyAsync(out, bud_res, 4 * sizeof(double), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        return MOIST_OK;
    }

    // hash of the current State's bit patterns (7 fields and prec), queued on the stream
    unsigned long long* hash_buf = nullptr;
    int queue_state_hash(unsigned long long* dst_slot) {
        if (!hash_buf) AL(hash_buf, 64);
        CK(cudaMemsetAsync(dst_slot, 0, sizeof(unsigned long long), st));
        const auto cf = cur_fields();
        for (int f = 0; f < 7; f++) k_hash<T><<<64, 256, 0, st>>>(cf[f], fsz, dst_slot);
        k_hash<T><<<1, 256, 0, st>>>(prec, (size_t)P, dst_slot);
        CKL();
        return MOIST_OK;
    }

    // ------------------------------------------------------------------ history diagnostics
    // output_history's primitive variables on the device (k_history_diag); only the requested
    // fields travel to the host
    int history(void* const out[MOIST_NDIAG], double summary[6]) override {
        const size_t ncell = (size_t)nx * nz;
        const unsigned nb = (unsigned)((ncell + HIST_THREADS - 1) / HIST_THREADS);
        if (!hist) {
            AL(hist, (size_t)MOIST_NDIAG * ncell);
            AL(hist_part, (size_t)nb * 6);
        }
        k_history_diag<T><<<nb, HIST_THREADS, 0, st>>>(dp, cur, hist, hist_part);
        CKL();
        for (int f = 0; f < MOIST_NDIAG; f++)
            if (out && out[f])
                CK(cudaMemcpyAsync(out[f], hist + (size_t)f * ncell, ncell * sizeof(T), cudaMemcpyDeviceToHost, st));
        std::vector<double> part;
        if (summary) {
            part.resize((size_t)nb * 6);
            CK(cudaMemcpyAsync(part.data(), hist_part, part.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
        }
        CK(cudaStreamSynchronize(st));
        if (summary) {
            double r[6] = {1e300, -1e300, -1e300, -1e300, 1e300, -1e300};
            for (unsigned b = 0; b < nb; b++)
                for (int j = 0; j < 6; j++) {
                    const double x = part[(size_t)b * 6 + j];
                    r[j] = (j == 0 || j == 4) ? std::min(r[j], x) : std::max(r[j], x);
                }
            summary[0] = r[0];           // w min (m/s)
            summary[1] = r[1];           // w max
            summary[2] = r[2] * 1000.0;  // qc max (g/kg)
            summary[3] = r[3] * 1000.0;  // qr max (g/kg)
            summary[4] = r[4];           // RH min (%)
            summary[5] = r[5];           // RH max
        }
        return MOIST_OK;
    }

    // ------------------------------------------------------------------ autotuner
    // Times nsteps large steps for every strip width of the factorisation and substep kernels
    // (1, 2, 4, 8 columns) and every tracer sweep this context can run (tiled, row-streaming),
    // each from the same saved State, keeps the fastest and restores the State. All candidates
    // give the same results bit for bit, so the choice changes only the speed.
    int autotune(int nsteps, std::string& report) override {
        if (int r = check_stage_shape()) return r;
        if (nsteps < 1) return set_err(owner, MOIST_ERR_ARG, "moist_autotune needs nsteps >= 1");
        int dev = 0, optin = 0;
        CK(cudaGetDevice(&dev));
        CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
        if (nz <= STREAM_MAX_ROWS && !s_old[0]) {  // buffers of the streaming sweep
            for (int t = 0; t < 3; t++) AL(s_old[t], fsz);
            AL(rrho, fsz);
        }
        std::array<T*, 8>& save = tune_save;
        if (!save[0]) {  // kept for later calls
            for (int f = 0; f < 7; f++) AL(save[f], fsz);
            AL(save[7], (size_t)P);
            AL(tune_halo, 2);
        }
        // the State: prognostic fields, accumulated rain and the two halo values the surface
        // fluxes carry across steps
        auto restore = [&]() -> int {
            const auto dst = cur_fields();
            if (int r = copyf(save.data(), dst.data(), 7)) return r;
            CK(cudaMemcpyAsync(prec, save[7], P * sizeof(T), cudaMemcpyDeviceToDevice, st));
            CK(cudaMemcpyAsync(halo_vals, tune_halo, 2 * sizeof(T), cudaMemcpyDeviceToDevice, st));
            return MOIST_OK;
        };
        {
            const auto src = cur_fields();
            if (int r = copyf(src.data(), save.data(), 7)) return r;
            CK(cudaMemcpyAsync(save[7], prec, P * sizeof(T), cudaMemcpyDeviceToDevice, st));
            CK(cudaMemcpyAsync(tune_halo, halo_vals, 2 * sizeof(T), cudaMemcpyDeviceToDevice, st));
        }
        struct Cand {
            int wc;
            int tracer;  // 0 tiles, 1 stream, 2 tiles without grid barriers
        };
        std::vector<Cand> cands;
        for (int tr = 0; tr < 3; tr++) {
            if (tr != 1 && !strips) continue;  // the tiles need all of them resident (init_tiles)
            if (tr == 1 && !s_old[0]) continue;
            for (int w : {1, 2, 4, 8})
                if (w <= nx && strip_smem_bytes<T, TT>(nz, w) <= (size_t)optin) cands.push_back({w, tr});
        }
        const int wc0 = strip_wc, str0 = use_stream, til0 = use_tiles, df0 = tiles_df;
        auto tracer_name = [](int tr) { return tr == 1 ? "stream" : tr == 2 ? "tiles dataflow" : "tiles"; };
        cudaEvent_t e0, e1;
        CK(cudaEventCreate(&e0));
        CK(cudaEventCreate(&e1));
        float best = 1e30f;
        Cand bc{wc0, str0 ? 1 : (df0 ? 2 : 0)};
        char buf[128];
        if (!hash_buf) AL(hash_buf, 64);
        std::vector<unsigned long long> hashes(cands.size());
        for (size_t ci = 0; ci < cands.size(); ci++) {
            const Cand& c = cands[ci];
            strip_wc = c.wc;
            strip_smem = strip_smem_bytes<T, TT>(nz, c.wc);
            use_tiles = c.tracer != 1;
            use_stream = c.tracer == 1;
            tiles_df = c.tracer == 2;
            if (int rr = restore()) return rr;
            CK(reset_err());
            int r = launch_step();  // warm-up
            CK(cudaEventRecord(e0, st));
            for (int n = 0; n < nsteps && r == MOIST_OK; n++) r = launch_step();
            CK(cudaEventRecord(e1, st));
            if (r != MOIST_OK) return r;
            if (int rh = queue_state_hash(hash_buf)) return rh;
            CK(cudaMemcpyAsync(&hashes[ci], hash_buf, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
            CK(cudaEventSynchronize(e1));
            CK(cudaStreamSynchronize(st));
            if (hashes[ci] != hashes[0])
                return set_err(owner, MOIST_ERR_CUDA,
                               "autotune: strip %d / %s gives another State than the first candidate", c.wc,
                               tracer_name(c.tracer));
            float ms = 0.f;
            CK(cudaEventElapsedTime(&ms, e0, e1));
            ms /= nsteps;
            snprintf(buf, sizeof buf, "%sstrip %d, %s: %.3f ms", report.empty() ? "" : "; ", c.wc,
                     tracer_name(c.tracer), ms);
            report += buf;
            if (ms < best) {
                best = ms;
                bc = c;
            }
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (cands.empty()) {
            strip_wc = wc0;
            use_stream = str0;
            use_tiles = til0;
            tiles_df = df0;
        } else {
            strip_wc = bc.wc;
            use_tiles = bc.tracer != 1;
            use_stream = bc.tracer == 1;
            tiles_df = bc.tracer == 2;
        }
        strip_smem = strip_smem_bytes<T, TT>(nz, strip_wc);
        snprintf(buf, sizeof buf, " -> strip %d, %s (%.3f ms per step)", strip_wc,
                 tracer_name(use_stream ? 1 : (tiles_df ? 2 : 0)), best);
        report += buf;
        if (int rr = restore()) return rr;
        CK(reset_err());
        return finish();
    }

    // ------------------------------------------------------------------ adjoint (adjoint.cuh)
    int stage_substeps(int j) const {
        return j == 0 ? std::max(1, (int)std::ceil(ns / 3.0)) : (j == 1 ? std::max(1, (int)std::ceil(ns / 2.0)) : ns);
    }

    // seg_mode: -1 decides the tape mode from the free memory; 0 / 1 sets one tape / a tape per
    // step of a segment (the packed batch adjoint runs every member in the same mode)
    int adj_alloc(int nsteps, int ckpt, int seg_mode = -1) {
        if (!adj) {
            adj = new Adj();
            Adj& A = *adj;
            std::vector<T> h(nz);
            std::vector<double> hd(nz);
            double** g[3] = {&A.dz, &A.z, &A.zf};
            const T* src[3] = {g_dz, g_z, g_zf};
            for (int j = 0; j < 3; j++) {
                AL(*g[j], (size_t)nz);
                CK(cudaMemcpyAsync(h.data(), src[j], nz * sizeof(T), cudaMemcpyDeviceToHost, st));
                CK(cudaStreamSynchronize(st));
                for (int k = 0; k < nz; k++) hd[k] = (double)h[k];
                CK(cudaMemcpyAsync(*g[j], hd.data(), nz * sizeof(double), cudaMemcpyHostToDevice, st));
                CK(cudaStreamSynchronize(st));
            }
            int dev = 0, optin = 0;  // shared by all contexts (other nz): the device maximum
            CK(cudaGetDevice(&dev));
            CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
            CK(cudaFuncSetAttribute(k_adj_sub_solve, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
            A.pd = params_to_double(dp);
            A.pd.dz = A.dz;
            A.pd.z = A.z;
            A.pd.zf = A.zf;
            for (int f = 0; f < 7; f++) {
                AL(A.Lst[f], fsz);
                AL(A.LS0[f], fsz);
                AL(A.seed[f], fsz);
            }
            for (int f = 0; f < 5; f++) AL(A.Lph[f], fsz);
            AL(A.acc, 16 * fsz);
            for (int t = 0; t < 3; t++) {
                AL(A.Lqout[t], fsz);
                AL(A.mu[t], fsz);
            }
            AL(A.J, 3 * TR_SLOTS * fsz);
            for (int q = 0; q < 2; q++)
                for (int f = 0; f < 4; f++) AL(A.LP[q][f], fsz);
            for (double** f : {&A.Ta, &A.Tb, &A.Tc, &A.Tcp, &A.Trd, &A.Lx, &A.Ly, &A.Ltp_rho, &A.Ltp_rt,
                               &A.Linc_rho, &A.Linc_rt, &A.Lsed})
                AL(*f, fsz);
            AL(A.Lpar, 2);
            AL(A.obj, 1);
            AL(A.prec_w, (size_t)P);
            AL(A.stage, (size_t)nz * (nx + 2 * halo));
            for (int f = 0; f < 7; f++) AL(A.fin[f], fsz);
            AL(A.fin[7], (size_t)P);
        }
        Adj& A = *adj;
        // a tape per step of a segment when that fits in half the free device memory (the
        // segment is then recomputed once), else one tape and the segment's States
        if (seg_mode >= 0) {
            seg_tapes = seg_mode == 1;
            adj_ckpt = -1;  // a later moist_adjoint_run decides again
        } else if (ckpt != adj_ckpt) {  // decided once per checkpoint interval
            size_t free_b = 0, total_b = 0;
            CK(cudaMemGetInfo(&free_b, &total_b));
            const size_t need =
                (size_t)std::max<long>(0, (long)ckpt - (long)A.tapes.size()) * tape_fields() * fsz * sizeof(T);
            seg_tapes = A.tapes.size() >= (size_t)ckpt || need <= free_b / 2;
            adj_ckpt = ckpt;
        }
        const size_t ntapes = seg_tapes ? (size_t)ckpt : 1;
        while (A.tapes.size() < ntapes) {
            A.tapes.emplace_back();
            if (int r = alloc_tape(A.tapes.back())) return r;
        }
        const size_t nck = (size_t)((nsteps + ckpt - 1) / ckpt);
        while (A.ck.size() < nck) {
            std::array<T*, 7> a;
            for (int f = 0; f < 7; f++) AL(a[f], fsz);
            A.ck.push_back(a);
        }
        while (!seg_tapes && A.seg.size() < (size_t)ckpt) {
            std::array<T*, 7> a;
            for (int f = 0; f < 7; f++) AL(a[f], fsz);
            A.seg.push_back(a);
        }
        return MOIST_OK;
    }

    bool seg_tapes = false;
    T* hist = nullptr;         // history diagnostics, [MOIST_NDIAG][nz * nx]
    double* hist_part = nullptr;
    std::array<T*, 8> tune_save{};  // the State saved by autotune
    T* tune_halo = nullptr;
    int adj_ckpt = -1;  // checkpoint interval the tape mode was chosen for

    size_t tape_fields() const {
        size_t n = 21 + 3 + 6 + 9 + 1;
        for (int j = 0; j < 3; j++) n += 4 * (size_t)(stage_substeps(j) + 1);
        return n;
    }

    int alloc_tape(Tape& tp) {
        for (int j = 0; j < 3; j++) {
            for (int f = 0; f < 7; f++) AL(tp.in[j][f], fsz);
            tp.sub[j].resize(stage_substeps(j) + 1);
            for (auto& a : tp.sub[j])
                for (int f = 0; f < 4; f++) AL(a[f], fsz);
            AL(tp.rrt[j], fsz);
            AL(tp.mf[j][0], fsz);
            AL(tp.mf[j][1], fsz);
            for (int t = 0; t < 3; t++) AL(tp.qout[j][t], fsz);
        }
        AL(tp.sed, fsz);
        return MOIST_OK;
    }

    std::array<T*, 7> cur_fields() const { return {cur.rho, cur.ru, cur.rw, cur.rt, cur.qv, cur.qc, cur.qr}; }

    // the adjoint of one large step: lambda of the step's output State in A.Lst becomes the
    // lambda of its input State; the tape holds the step's internals. With rec set, every
    // launch is recorded for a packed batch launch (adjoint_batch.cuh) instead.
    int adj_step(const Tape& tp) {
        Adj& A = *adj;
        const dim3 b(ADJ_THREADS), gc(cdiv(nx, ADJ_THREADS), nz), gc3(cdiv(nx, ADJ_THREADS), nz, 3);
        const unsigned gcol = cdiv(nx, 32);
        const dim3 b2(32, 8), g2(cdiv(nx, 32), cdiv(nz, 8));
        const T dtT = dp.dt;
        const T dst[3] = {dtT / T(3), dtT / T(2), dtT};
        const T fact_tpT = T(0.5) * (T(1.0) + dp.beta), fact_tmT = T(0.5) * (T(1.0) - dp.beta);
        int lp = 0;
        for (int j = 2; j >= 0; j--) {
            const int m = stage_substeps(j);
            const StateP<T> s{tp.in[j][0], tp.in[j][1], tp.in[j][2], tp.in[j][3], tp.in[j][4], tp.in[j][5], tp.in[j][6]};
            if (rec)
                rec->put(BK_DIAG, BDiag<T>{dp, s, pres, theta, rt2p, uface, wface, err});
            else
                k_diag<T><<<g2, b2, 0, st>>>(dp, s, pres, theta, rt2p, uface, wface, err);
            AdjStage<T> a{};
            a.s = s;
            a.theta = theta;
            a.rt2 = rt2p;
            a.pres = pres;
            a.uf = uface;
            a.wf = wface;
            a.rrt = tp.rrt[j];
            a.mfx = tp.mf[j][0];
            a.mfz = tp.mf[j][1];
            for (int t = 0; t < 3; t++) {
                a.qout[t] = tp.qout[j][t];
                a.q0[t] = tp.in[0][4 + t];
                a.Lqout[t] = A.Lqout[t];
            }
            a.dt_stage = (double)dst[j];
            a.dt_s = (double)(dst[j] / T(m));
            a.m = m;
            a.fact_tp64 = (double)T(0.5) * (1.0 + (double)dp.beta);
            a.fact = (double)(fact_tmT / fact_tpT);
            for (int f = 0; f < 7; f++) {
                a.Lst[f] = A.Lst[f];
                a.LS0[f] = A.LS0[f];
            }
            for (int f = 0; f < 5; f++) a.Lph[f] = A.Lph[f];
            double* acc[16];
            for (int q = 0; q < 16; q++) acc[q] = A.acc + (size_t)q * fsz;
            a.LRrho = acc[0];
            a.LRu = acc[1];
            a.LRw = acc[2];
            a.LRt = acc[3];
            a.Ltheta = acc[4];
            a.Lrt2 = acc[5];
            a.Lpres = acc[6];
            a.Luf = acc[7];
            a.Lwf = acc[8];
            a.La = acc[9];
            a.Lb = acc[10];
            a.Lc = acc[11];
            a.Lmfx = acc[12];
            a.Lmfz = acc[13];
            a.Lpend[0] = acc[14];
            a.Lpend[1] = acc[15];
            a.Ta = A.Ta;
            a.Tb = A.Tb;
            a.Tc = A.Tc;
            a.Tcp = A.Tcp;
            a.Trd = A.Trd;
            a.Lx = A.Lx;
            a.Ly = A.Ly;
            a.Ltp_rho = A.Ltp_rho;
            a.Ltp_rt = A.Ltp_rt;
            a.Linc_rho = A.Linc_rho;
            a.Linc_rt = A.Linc_rt;
            DP<4> LPc{{A.LP[lp][0], A.LP[lp][1], A.LP[lp][2], A.LP[lp][3]}};
            const DP<3> lq{{A.Lqout[0], A.Lqout[1], A.Lqout[2]}}, mu{{A.mu[0], A.mu[1], A.mu[2]}};
            if (rec) {
                rec->put(BK_ZERO, BZero{A.acc, 16 * fsz, bz_blocks(fsz)});
                rec->put(AK_TRI_COEF, AStage<T>{A.pd, a});
                rec->put(AK_TRI_FACT, ATriFact{nx, nz, P, A.Ta, A.Tb, A.Tc, A.Tcp, A.Trd});
                rec->put(AK_UPDATE, AStageLP<T>{A.pd, a, LPc});
                rec->put(AK_TR_JAC, ATrJac<T>{A.pd, a, A.J});
                rec->put(AK_TR_REV, ATrRev{nx, nz, P, A.J, lq, mu});
                rec->put(AK_TR_SCATTER, ATrScatter<T>{A.pd, a, A.J, mu});
                rec->put(AK_MF, AStage<T>{A.pd, a});
            } else {
                CK(cudaMemsetAsync(A.acc, 0, 16 * fsz * sizeof(double), st));
                k_adj_tri_coef<T><<<gc, b, 0, st>>>(A.pd, a);
                k_adj_tri_fact<<<gcol, 32, 0, st>>>(nx, nz, P, A.Ta, A.Tb, A.Tc, A.Tcp, A.Trd);
                k_adj_update<T><<<gc, b, 0, st>>>(A.pd, a, LPc);
                k_adj_tr_jac<T><<<gc3, b, 0, st>>>(A.pd, a, A.J);
                k_adj_tr_rev<<<3, (nz + 31) / 32 * 32, 3 * nz * sizeof(double), st>>>(nx, nz, P, A.J, lq, mu);
                k_adj_tr_scatter<T><<<gc3, b, 0, st>>>(A.pd, a, A.J, mu);
                k_adj_mf<T><<<gc, b, 0, st>>>(A.pd, a);
            }
            for (int n = m; n >= 1; n--) {
                AdjSub<T> sb;
                sb.prev_rt = tp.sub[j][n - 1][3];
                sb.prev_rw = tp.sub[j][n - 1][2];
                sb.old_rt = tp.sub[j][std::max(n - 2, 0)][3];
                sb.ru = tp.sub[j][n][1];
                sb.rw = tp.sub[j][n][2];
                for (int f = 0; f < 4; f++) {
                    sb.LPn[f] = A.LP[lp][f];
                    sb.LPo[f] = A.LP[1 - lp][f];
                }
                sb.n = n;
                if (rec) {
                    const ASub<T> as{A.pd, dp, a, sb};
                    rec->put(AK_SUB_VERT, as);
                    rec->put(AK_SUB_SOLVE, ASolve{nx, nz, P, A.Tc, A.Tcp, A.Trd, A.Lx, A.Ly});
                    rec->put(AK_SUB_RHS, as);
                    rec->put(AK_SUB_EXPL, as);
                    rec->put(AK_SUB_HORIZ, as);
                } else {
                    k_adj_sub_vert<T><<<gc, b, 0, st>>>(A.pd, a, sb);
                    k_adj_sub_solve<<<cdiv(nx, adj_solve_cols(nz)), ADJ_SOLVE_THREADS, adj_solve_smem(nz), st>>>(
                        nx, nz, P, A.Tc, A.Tcp, A.Trd, A.Lx, A.Ly);
                    k_adj_sub_rhs<T><<<gc, b, 0, st>>>(A.pd, dp, a, sb);
                    k_adj_sub_expl<T><<<gc, b, 0, st>>>(A.pd, a, sb);
                    k_adj_sub_horiz<T><<<gc, b, 0, st>>>(A.pd, a, sb);
                }
                lp = 1 - lp;
            }
            DP<4> LP0{{A.LP[lp][0], A.LP[lp][1], A.LP[lp][2], A.LP[lp][3]}};
            if (rec) {
                rec->put(AK_P0, AStageLP<T>{A.pd, a, LP0});
                rec->put(AK_TRI_COEF_T, AStage<T>{A.pd, a});
                rec->put(AK_TEND_T, AStage<T>{A.pd, a});
                rec->put(AK_FACE_T, AStage<T>{A.pd, a});
                rec->put(AK_DIAG_T, AStage<T>{A.pd, a});
            } else {
                k_adj_p0<T><<<gc, b, 0, st>>>(A.pd, a, LP0);
                k_adj_tri_coef_T<T><<<gc, b, 0, st>>>(A.pd, a);
                k_adj_tend_T<T><<<gc, b, 0, st>>>(A.pd, a);
                k_adj_face_T<T><<<gc, b, 0, st>>>(A.pd, a);
                k_adj_diag_T<T><<<gc, b, 0, st>>>(A.pd, a);
                CKL();
            }
        }
        AdjPhys<T> ph;
        ph.s = StateP<T>{tp.in[0][0], tp.in[0][1], tp.in[0][2], tp.in[0][3], tp.in[0][4], tp.in[0][5], tp.in[0][6]};
        ph.sed = tp.sed;
        for (int f = 0; f < 7; f++) ph.Lst[f] = A.Lst[f];
        for (int f = 0; f < 5; f++) ph.Lph[f] = A.Lph[f];
        ph.Lsed = A.Lsed;
        ph.prec_w = A.prec_w;
        ph.Lpar = A.Lpar;
        DP<7> L7, S7;
        DP<5> L5;
        for (int f = 0; f < 7; f++) {
            L7.f[f] = A.Lst[f];
            S7.f[f] = A.LS0[f];
        }
        for (int f = 0; f < 5; f++) L5.f[f] = A.Lph[f];
        if (rec) {
            rec->put(AK_KESSLER, APhys<T>{A.pd, ph});
            rec->put(AK_SED, APhys<T>{A.pd, ph});
            rec->put(AK_STEP_END, AStepEnd{nx, nz, P, L7, S7, L5});
            return MOIST_OK;
        }
        k_adj_kessler<T><<<gc, b, 0, st>>>(A.pd, ph);
        k_adj_sed<T><<<gc, b, 0, st>>>(A.pd, ph);
        k_adj_step_end<<<gc, b, 0, st>>>(nx, nz, P, L7, S7, L5);
        CKL();
        return MOIST_OK;
    }

    // moist_adjoint_run in phases; the packed batch adjoint runs the same phases around its
    // packed forward and reverse steps
    bool adj_seed_on[7] = {false, false, false, false, false, false, false};
    bool adj_prec_on = false;

    int adj_check(int nsteps, int ckpt, const void* out) {
        if (int r = check_stage_shape()) return r;
        if (!out || nsteps < 1 || ckpt < 1)
            return set_err(owner, MOIST_ERR_ARG, "moist_adjoint_run needs out != NULL, nsteps >= 1 and ckpt_every >= 1");
        if (dp.do_sf || dp.do_rd)
            return set_err(owner, MOIST_ERR_UNSUPPORTED,
                           "moist_adjoint_run covers do_sf = do_rd = 0 (surface fluxes and radiation are not differentiated)");
        return MOIST_OK;
    }

    // the seeds on the device, the error words reset
    int adj_seeds(const moist_adjoint_seed* seed) {
        Adj& A = *adj;
        const dim3 b(ADJ_THREADS), gc(cdiv(nx, ADJ_THREADS), nz);
        const int ia = nx + 2 * halo;
        for (int f = 0; f < 7; f++) {
            const double* h = seed ? seed->state[f] : nullptr;
            adj_seed_on[f] = h != nullptr;
            if (h) {
                CK(cudaMemcpyAsync(A.stage, h, (size_t)nz * ia * sizeof(double), cudaMemcpyHostToDevice, st));
                k_adj_from_ref<<<gc, b, 0, st>>>(nx, nz, halo, P, A.stage, A.seed[f]);
                CKL();
            }
        }
        adj_prec_on = seed && seed->prec_weight;
        if (adj_prec_on)
            CK(cudaMemcpyAsync(A.prec_w, seed->prec_weight + halo, nx * sizeof(double), cudaMemcpyHostToDevice, st));
        CK(reset_err());
        return MOIST_OK;
    }

    // after the forward run: the objective, the final State kept, lambda of the final State
    int adj_begin() {
        Adj& A = *adj;
        const dim3 b(ADJ_THREADS), gc(cdiv(nx, ADJ_THREADS), nz);
        CK(cudaMemsetAsync(A.obj, 0, sizeof(double), st));
        DP<7> sd;
        for (int f = 0; f < 7; f++) sd.f[f] = adj_seed_on[f] ? A.seed[f] : nullptr;
        k_adj_objective<T><<<gc, b, 0, st>>>(nx, nz, P, cur, prec, adj_prec_on ? A.prec_w : nullptr, sd, A.obj);
        CKL();
        int r;
        {
            const auto src = cur_fields();
            if ((r = copyf(src.data(), A.fin.data(), 7)) != MOIST_OK) return r;
            CK(cudaMemcpyAsync(A.fin[7], prec, P * sizeof(T), cudaMemcpyDeviceToDevice, st));
        }
        for (int f = 0; f < 7; f++) {
            if (adj_seed_on[f])
                CK(cudaMemcpyAsync(A.Lst[f], A.seed[f], fsz * sizeof(double), cudaMemcpyDeviceToDevice, st));
            else
                CK(cudaMemsetAsync(A.Lst[f], 0, fsz * sizeof(double), st));
            CK(cudaMemsetAsync(A.LS0[f], 0, fsz * sizeof(double), st));
        }
        for (int f = 0; f < 5; f++) CK(cudaMemsetAsync(A.Lph[f], 0, fsz * sizeof(double), st));
        CK(cudaMemsetAsync(A.Lpar, 0, 2 * sizeof(double), st));
        if (!adj_prec_on) CK(cudaMemsetAsync(A.prec_w, 0, P * sizeof(double), st));
        return MOIST_OK;
    }

    // after the reverse sweep: the gradients to the host, the context back at the final State
    int adj_results(const moist_adjoint_seed* seed, moist_adjoint_grad* out, double forward_ms, double reverse_ms) {
        Adj& A = *adj;
        const int ia = nx + 2 * halo;
        const dim3 b(ADJ_THREADS), gr(cdiv(ia, ADJ_THREADS), nz);
        int r;
        for (int f = 0; f < 7; f++) {
            if (!out->state[f]) continue;
            k_adj_to_ref<<<gr, b, 0, st>>>(nx, nz, halo, P, A.Lst[f], A.stage);
            CKL();
            CK(cudaMemcpyAsync(out->state[f], A.stage, (size_t)nz * ia * sizeof(double), cudaMemcpyDeviceToHost, st));
        }
        double hp[3];
        CK(cudaMemcpyAsync(hp, A.Lpar, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(hp + 2, A.obj, sizeof(double), cudaMemcpyDeviceToHost, st));
        {
            const auto dstf = cur_fields();
            if ((r = copyf(A.fin.data(), dstf.data(), 7)) != MOIST_OK) return r;
            CK(cudaMemcpyAsync(prec, A.fin[7], P * sizeof(T), cudaMemcpyDeviceToDevice, st));
        }
        CK(cudaStreamSynchronize(st));
        if (out->prec) {
            for (int j = 0; j < ia; j++) {
                const int i = j - halo;
                out->prec[j] = (adj_prec_on && i >= 0 && i < nx) ? seed->prec_weight[j] : 0.0;
            }
        }
        out->k_auto = hp[0];
        out->qc_threshold = hp[1];
        out->objective = hp[2];
        out->forward_ms = forward_ms;
        out->reverse_ms = reverse_ms;
        return finish();
    }

    int adjoint_run(int nsteps, int ckpt, const moist_adjoint_seed* seed, moist_adjoint_grad* out) override {
        if (int r = adj_check(nsteps, ckpt, out)) return r;
        ckpt = std::min(ckpt, nsteps);
        if (int r = adj_alloc(nsteps, ckpt, tape_mode)) return r;
        Adj& A = *adj;
        int r;
        if ((r = adj_seeds(seed)) != MOIST_OK) return r;
        // forward run, keeping the State every ckpt steps
        const auto t0 = std::chrono::steady_clock::now();
        for (int n = 0; n < nsteps; n++) {
            if (n % ckpt == 0) {
                const auto src = cur_fields();
                if ((r = copyf(src.data(), A.ck[n / ckpt].data(), 7)) != MOIST_OK) return r;
            }
            if ((r = launch_step()) != MOIST_OK) return r;
        }
        CK(cudaStreamSynchronize(st));
        const auto t1 = std::chrono::steady_clock::now();
        if ((r = adj_begin()) != MOIST_OK) return r;
        // reverse sweep, one segment of ckpt steps at a time
        const int nck = (nsteps + ckpt - 1) / ckpt;
        for (int sg = nck - 1; sg >= 0; sg--) {
            const int n0 = sg * ckpt, n1 = std::min(n0 + ckpt, nsteps);
            if (seg_tapes) {  // recompute the segment once, taping every step
                const auto dstf = cur_fields();
                if ((r = copyf(A.ck[sg].data(), dstf.data(), 7)) != MOIST_OK) return r;
                for (int n = n0; n < n1; n++) {
                    tape = &A.tapes[n - n0];
                    r = launch_step();
                    tape = nullptr;
                    if (r != MOIST_OK) return r;
                }
                for (int n = n1 - 1; n >= n0; n--)
                    if ((r = adj_step(A.tapes[n - n0])) != MOIST_OK) return r;
                continue;
            }
            {
                const auto dstf = cur_fields();
                if ((r = copyf(A.ck[sg].data(), dstf.data(), 7)) != MOIST_OK) return r;
                if ((r = copyf(A.ck[sg].data(), A.seg[0].data(), 7)) != MOIST_OK) return r;
            }
            for (int n = n0; n < n1 - 1; n++) {
                if ((r = launch_step()) != MOIST_OK) return r;
                const auto src = cur_fields();
                if ((r = copyf(src.data(), A.seg[n - n0 + 1].data(), 7)) != MOIST_OK) return r;
            }
            for (int n = n1 - 1; n >= n0; n--) {
                const auto dstf = cur_fields();
                if ((r = copyf(A.seg[n - n0].data(), dstf.data(), 7)) != MOIST_OK) return r;
                tape = &A.tapes[0];
                r = launch_step();
                tape = nullptr;
                if (r != MOIST_OK) return r;
                if ((r = adj_step(A.tapes[0])) != MOIST_OK) return r;
            }
        }
        CK(cudaStreamSynchronize(st));
        const auto t2 = std::chrono::steady_clock::now();
        return adj_results(seed, out, std::chrono::duration<double, std::milli>(t1 - t0).count(),
                           std::chrono::duration<double, std::milli>(t2 - t1).count());
    }
};

// device helper evaluation and single-column implicit correction (unit-test entry points)
template <class T>
__global__ void k_eval_helper(DevParams<T> p, int helper, int n, const double* in, double* out) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    switch (helper) {
        case MOIST_HELPER_F2H:
            out[j] = (double)f2h((T)in[4 * j], (T)in[4 * j + 1], (T)in[4 * j + 2], (T)in[4 * j + 3]);
            break;
        case MOIST_HELPER_KOREN:
            out[j] = (double)koren((T)in[j]);
            break;
        case MOIST_HELPER_SAT_VP: {
            T es, d;
            sat_vp((T)in[j], p, es, d);
            out[2 * j] = es;
            out[2 * j + 1] = d;
            break;
        }
        case MOIST_HELPER_SAT_Q: {
            T q, d;
            sat_q((T)in[2 * j], (T)in[2 * j + 1], p, q, d);
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
    }
}

// implicit_correction! for one column: the per-stage factorisation followed by one substep's
// right-hand side, elimination and back substitution, exactly as k_thomas_factors + k_substep
template <class T, class TT>
__global__ void k_implicit_column(DevParams<T> p, T* rho_w, const T* drho_w, const T* theta, const T* rt2pres,
                                  T dt) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const int nz = p.nz, n = nz - 1, ke = nz - 1;
    const T* dz = p.dz;
    const T* z = p.z;
    const T fact_tp = T(0.5) * (T(1.0) + p.beta);
    const T fact_tm = T(0.5) * (T(1.0) - p.beta);
    const T dt_tp2 = (dt * fact_tp) * (dt * fact_tp);
    const T fact = fact_tm / fact_tp;
    TT cp_prev = TT(0), d_prev = TT(0);
    extern __shared__ unsigned char sm[];
    TT* cps = reinterpret_cast<TT*>(sm);
    TT* dps = cps + n;
    for (int j = 0; j < n; j++) {
        const int k = j;
        const T th_cur = f2h(theta[k], theta[k + 1], dz[k], dz[k + 1]);
        const T th_prev = k > 0 ? f2h(theta[k - 1], theta[k], dz[k - 1], dz[k]) : T(0);
        const T th_next = (k + 1 <= ke - 1) ? f2h(theta[k + 1], theta[k + 2], dz[k + 1], dz[k + 2]) : T(0);
        const T b = dt_tp2 * (rt2pres[k] / dz[k] + rt2pres[k + 1] / dz[k + 1]) * th_cur / (z[k + 1] - z[k]);
        const T a = (k > 0) ? -dt_tp2 * (rt2pres[k] * th_prev / ((z[k + 1] - z[k]) * dz[k]) - p.GRAV / (dz[k] + dz[k + 1])) : T(0);
        const T c = (k < ke - 1) ? -dt_tp2 * (rt2pres[k + 1] * th_next / ((z[k + 1] - z[k]) * dz[k + 1]) + p.GRAV / (dz[k] + dz[k + 1])) : T(0);
        T d = rho_w[k] + drho_w[k];
        if (k > 0) d -= a * fact * rho_w[k];
        d -= b * fact * rho_w[k];
        const T bb = b + T(1.0);
        if (k < ke - 1) d -= c * fact * rho_w[k + 1];
        TT piv, cpj, dpj;
        if (j == 0) {
            piv = (TT)bb;
            cpj = (TT)c / piv;
            dpj = (TT)d / piv;
        } else {
            piv = (TT)bb - (TT)a * cp_prev;
            cpj = (TT)c / piv;
            dpj = ((TT)d - (TT)a * d_prev) / piv;
        }
        cps[j] = cpj;
        dps[j] = dpj;
        cp_prev = cpj;
        d_prev = dpj;
    }
    TT x = dps[n - 1];
    rho_w[n - 1] = (T)x;
    for (int j = n - 2; j >= 0; j--) {
        x = dps[j] - cps[j] * x;
        rho_w[j] = (T)x;
    }
}

template <class T>
int eval_helper_t(const moist_params* c, int helper, int n, const double* in, double* out) {
    moist_ctx* owner = nullptr;
    DevParams<T> p = make_params<T>(c, 0);
    int nin = (helper == MOIST_HELPER_F2H) ? 4 : (helper == MOIST_HELPER_SAT_Q || helper == MOIST_HELPER_POW) ? 2 : 1;
    int nout = (helper == MOIST_HELPER_SAT_VP || helper == MOIST_HELPER_SAT_Q) ? 2 : 1;
    if (helper < 0 || helper > MOIST_HELPER_POW) return MOIST_ERR_ARG;
    double *din = nullptr, *dout = nullptr;
    CK(cudaMalloc(&din, std::max(1, n * nin) * sizeof(double)));
    CK(cudaMalloc(&dout, std::max(1, n * nout) * sizeof(double)));
    CK(cudaMemcpy(din, in, n * nin * sizeof(double), cudaMemcpyHostToDevice));
    if (n > 0) k_eval_helper<T><<<cdiv(n, 128), 128>>>(p, helper, n, din, dout);
    CKL();
    CK(cudaMemcpy(out, dout, n * nout * sizeof(double), cudaMemcpyDeviceToHost));
    cudaFree(din);
    cudaFree(dout);
    return MOIST_OK;
}

template <class T, class TT>
int implicit_t(const moist_params* c, void* rho_w, const void* drho_w, const void* theta, const void* rt2pres,
               double dt) {
    moist_ctx* owner = nullptr;
    const int nz = c->nz;
    DevParams<T> p = make_params<T>(c, 0);
    T* buf = nullptr;
    CK(cudaMalloc(&buf, 6 * nz * sizeof(T)));
    T *w = buf, *dw = buf + nz, *th = buf + 2 * nz, *r2 = buf + 3 * nz, *gdz = buf + 4 * nz, *gz = buf + 5 * nz;
    CK(cudaMemcpy(w, rho_w, nz * sizeof(T), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(dw, drho_w, nz * sizeof(T), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(th, theta, nz * sizeof(T), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(r2, rt2pres, nz * sizeof(T), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(gdz, c->dz, nz * sizeof(T), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(gz, c->z, nz * sizeof(T), cudaMemcpyHostToDevice));
    p.dz = gdz;
    p.z = gz;
    k_implicit_column<T, TT><<<1, 32, 2 * nz * sizeof(TT)>>>(p, w, dw, th, r2, (T)dt);
    CKL();
    CK(cudaMemcpy(rho_w, w, nz * sizeof(T), cudaMemcpyDeviceToHost));
    cudaFree(buf);
    return MOIST_OK;
}


// ---------------------------------------------------------------------------- ensembles

int set_berr(moist_batch* b, int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (b) b->err = buf;
    return code;
}

#define BCK(call)                                                                                    \
    do {                                                                                             \
        cudaError_t e_ = (call);                                                                     \
        if (e_ != cudaSuccess)                                                                       \
            return set_berr(owner, MOIST_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_));  \
    } while (0)

// The members' recorded steps turned into packed launches (batch.cuh). Two steps are recorded
// because the current and next States swap every step; each is captured as a CUDA graph.
template <class T, class TT>
struct BatchImpl : BatchBase {
    moist_batch* owner;
    cudaStream_t st;
    std::vector<Ctx<T, TT>*> m;
    struct Slot {
        int kind;
        unsigned nitems;
        dim3 block;
        size_t smem;
        const BItem* items;
        const void* args;
        int group;
    };
    // the packed launches of the even and odd step: kind and the members' argument structs
    struct Launch {
        int kind;
        const void* args;
    };
    std::vector<Launch> launches[2];
    // per parity: the launches of member group 0, then of group 1, ...; the groups' chains are
    // parallel branches of the step graph, so one group's kernels fill the SMs that another
    // group's long members leave idle at the end of a launch
    std::vector<Slot> slots[2];
    static constexpr int MAX_GROUPS = 4;
    int ngroups = 1;
    std::vector<int> grp;  // group of each member
    cudaStream_t gstream[MAX_GROUPS] = {nullptr, nullptr, nullptr, nullptr};
    cudaEvent_t gfork = nullptr, gjoin[MAX_GROUPS] = {nullptr, nullptr, nullptr, nullptr};
    std::vector<void*> allocs;
    int col_threads = BATCH_COL_THREADS;  // threads per block of the per-column kernels
    bool sub_strips = false;               // factorisation and substep over column strips instead
    int stream_minb = 1;                   // register bound of the streaming tracer sweep: 1 or 2 blocks of
                                           // 256 threads per SM, or 3 blocks of 128 (rows <= 128)
    // per-column substep body: 0 b_substep_col (64 registers), 1 and 2 b_substep_col_pf (loads one
    // level ahead; 128 and 85 registers), 3 and 4 b_substep_col_async (the next level copied into
    // shared memory; 85 and 128 registers), 5 the same two levels ahead (128 registers)
    int sub_form = 4;
    std::vector<std::array<T*, 8>> tune_save;  // the members' States saved by autotune
    std::vector<T*> tune_halo;
    cudaGraphExec_t exec[2] = {nullptr, nullptr};
    int parity = 0;
    int** errs = nullptr;  // device: the members' error words
    int* err_all = nullptr;
    size_t max_strip_smem = 0;
    int max_rows = 32;

    BatchImpl(moist_batch* o, std::vector<Ctx<T, TT>*> members) : owner(o), st(o->stream), m(std::move(members)) {}
    ~BatchImpl() override {
        if (st) cudaStreamSynchronize(st);
        for (auto& e : exec)
            if (e) cudaGraphExecDestroy(e);
        for (int g = 1; g < MAX_GROUPS; g++) {
            if (gstream[g]) cudaStreamDestroy(gstream[g]);
            if (gjoin[g]) cudaEventDestroy(gjoin[g]);
        }
        if (gfork) cudaEventDestroy(gfork);
        for (void* a : item_allocs) cudaFree(a);
        for (void* a : allocs) cudaFree(a);
    }

    template <class U>
    int dalloc(U** p, size_t n) {
        void* q = nullptr;
        cudaError_t e = cudaMalloc(&q, std::max<size_t>(n, 1) * sizeof(U));
        if (e != cudaSuccess) return set_berr(owner, MOIST_ERR_NOMEM, "cudaMalloc of %zu bytes failed", n * sizeof(U));
        allocs.push_back(q);
        *p = (U*)q;
        return MOIST_OK;
    }

    // (member, block) items of one launch kind
    void items_of(int kind, std::vector<BItem>& it, dim3& block, size_t& smem, int group) {
        const int n = (int)m.size();
        smem = 0;
        auto in_group = [&](int i) { return group < 0 || grp[i] == group; };  // group < 0: every member
        auto cells = [&](int i) {
            for (unsigned by = 0; by < cdiv(m[i]->nz, 8); by++)
                for (unsigned bx = 0; bx < cdiv(m[i]->nx, 32); bx++) it.push_back({i, (int)bx, (int)by});
        };
        switch (kind) {
            case BK_MEMSET:
                block = dim3(256);
                for (int i = 0; i < n; i++)
                    if (in_group(i)) it.push_back({i, 0, 0});
                break;
            case BK_SF:
            case BK_RD:
            case BK_PREC:
                block = dim3(128);
                for (int i = 0; i < n; i++)
                    if (in_group(i))
                        for (unsigned bx = 0; bx < cdiv(m[i]->nx, 128); bx++) it.push_back({i, (int)bx, 0});
                break;
            case BK_PHYS:
            case BK_DIAG:
            case BK_TEND:
            case BK_UPD:
            case BK_PREP:
                block = dim3(32, 8);
                for (int i = 0; i < n; i++)
                    if (in_group(i)) cells(i);
                break;
            case BK_THOMAS:
            case BK_SUB:
                if (sub_strips) {  // column strips of each member's recorded width
                    block = dim3(STRIP_THREADS);
                    smem = max_strip_smem;
                    for (int i = 0; i < n; i++)
                        if (in_group(i))
                            for (unsigned bx = 0; bx < cdiv(m[i]->nx, m[i]->strip_wc); bx++) it.push_back({i, (int)bx, 0});
                } else {
                    block = dim3(col_threads);
                    if (kind == BK_SUB && sub_form >= 3)
                        smem = (size_t)col_threads * sub_async_bytes_per_thread<T, TT>(sub_form == 5 ? 3 : 2);
                    for (int i = 0; i < n; i++)
                        if (in_group(i))
                            for (unsigned bx = 0; bx < cdiv(m[i]->nx, col_threads); bx++) it.push_back({i, (int)bx, 0});
                }
                break;
            case BK_STREAM: {
                // the longest sweeps (nx + nz steps) first, so that the short ones fill the tail
                block = dim3(max_rows);
                std::vector<int> order(n);
                for (int i = 0; i < n; i++) order[i] = i;
                order.erase(std::remove_if(order.begin(), order.end(), [&](int i) { return !in_group(i); }), order.end());
                std::stable_sort(order.begin(), order.end(),
                                 [&](int a, int b) { return m[a]->nx + m[a]->nz > m[b]->nx + m[b]->nz; });
                for (int i : order)
                    for (int t = 0; t < 3; t++) it.push_back({i, t, 0});
                break;
            }
            case BK_STAGE_END:
                block = dim3(32);
                for (int i = 0; i < n; i++)
                    if (in_group(i)) it.push_back({i, 0, 0});
                break;
            // the adjoint's launches (adjoint_batch.cuh)
            case BK_ZERO:
            case BK_COPY:
                block = dim3(256);
                for (int i = 0; i < n; i++)
                    if (in_group(i))
                        for (unsigned bx = 0; bx < bz_blocks(m[i]->fsz); bx++) it.push_back({i, (int)bx, 0});
                break;
            case AK_TRI_FACT:
                block = dim3(32);
                for (int i = 0; i < n; i++)
                    if (in_group(i))
                        for (unsigned bx = 0; bx < cdiv(m[i]->nx, 32); bx++) it.push_back({i, (int)bx, 0});
                break;
            case AK_TR_REV: {  // one block per member and tracer, the longest sweeps first
                block = dim3(max_rows);
                int maxnz = 1;
                std::vector<int> order;
                for (int i = 0; i < n; i++)
                    if (in_group(i)) {
                        order.push_back(i);
                        maxnz = std::max(maxnz, m[i]->nz);
                    }
                smem = (size_t)3 * maxnz * sizeof(double);
                std::stable_sort(order.begin(), order.end(),
                                 [&](int a, int b) { return m[a]->nx + m[a]->nz > m[b]->nx + m[b]->nz; });
                for (int i : order)
                    for (int t = 0; t < 3; t++) it.push_back({i, t, 0});
                break;
            }
            case AK_SUB_SOLVE:
                block = dim3(ADJ_SOLVE_THREADS);
                for (int i = 0; i < n; i++)
                    if (in_group(i)) {
                        smem = std::max(smem, adj_solve_smem(m[i]->nz));
                        for (unsigned bx = 0; bx < cdiv(m[i]->nx, adj_solve_cols(m[i]->nz)); bx++)
                            it.push_back({i, (int)bx, 0});
                    }
                break;
            case AK_TR_JAC:
            case AK_TR_SCATTER:  // by = row + nz * tracer
                block = dim3(ADJ_THREADS);
                for (int i = 0; i < n; i++)
                    if (in_group(i))
                        for (int by = 0; by < 3 * m[i]->nz; by++)
                            for (unsigned bx = 0; bx < cdiv(m[i]->nx, ADJ_THREADS); bx++) it.push_back({i, (int)bx, by});
                break;
            default:  // the adjoint's cell kernels: (x block of ADJ_THREADS cells, row)
                if (kind >= AK_TRI_COEF && kind < AK_NKINDS) {
                    block = dim3(ADJ_THREADS);
                    for (int i = 0; i < n; i++)
                        if (in_group(i))
                            for (int by = 0; by < m[i]->nz; by++)
                                for (unsigned bx = 0; bx < cdiv(m[i]->nx, ADJ_THREADS); bx++)
                                    it.push_back({i, (int)bx, by});
                }
                break;
        }
    }

#define BATCH_LAUNCH(KIND, A, F, MINB)                                                                 \
    case KIND:                                                                                         \
        k_batched<A, F, MINB><<<s.nitems, s.block, s.smem, ls>>>(s.items, (const A*)s.args, F{});     \
        break;
    int launch(const Slot& s, cudaStream_t ls) {
        switch (s.kind) {
            BATCH_LAUNCH(BK_MEMSET, BMemset, FMemset, 1)
            BATCH_LAUNCH(BK_SF, BSf<T>, FSf<T>, 1)
            BATCH_LAUNCH(BK_RD, BRd<T>, FRd<T>, 1)
            BATCH_LAUNCH(BK_PHYS, BPhys<T>, FPhys<T>, 3)
            BATCH_LAUNCH(BK_DIAG, BDiag<T>, FDiag<T>, 4)
            BATCH_LAUNCH(BK_TEND, BTend<T>, FTend<T>, 4)
            case BK_THOMAS:
                if (sub_strips)
                    k_batched<BThomas<T, TT>, FThomasStrip<T, TT>, 4><<<s.nitems, s.block, s.smem, ls>>>(
                        s.items, (const BThomas<T, TT>*)s.args, FThomasStrip<T, TT>{});
                else
                    k_batched<BThomas<T, TT>, FThomas<T, TT>, 4><<<s.nitems, s.block, s.smem, ls>>>(
                        s.items, (const BThomas<T, TT>*)s.args, FThomas<T, TT>{});
                break;
            case BK_SUB:
                if (sub_strips)
                    k_batched<BSub<T, TT>, FSubStrip<T, TT>, 4><<<s.nitems, s.block, s.smem, ls>>>(
                        s.items, (const BSub<T, TT>*)s.args, FSubStrip<T, TT>{});
                else if (sub_form == 1)
                    k_batched<BSub<T, TT>, FSubPf<T, TT>, 2><<<s.nitems, s.block, s.smem, ls>>>(
                        s.items, (const BSub<T, TT>*)s.args, FSubPf<T, TT>{});
                else if (sub_form == 2)
                    k_batched<BSub<T, TT>, FSubPf<T, TT>, 3><<<s.nitems, s.block, s.smem, ls>>>(
                        s.items, (const BSub<T, TT>*)s.args, FSubPf<T, TT>{});
                else if (sub_form == 3)
                    k_batched<BSub<T, TT>, SINGLE_ARG(FSubAsync<T, TT, 2>), 3><<<s.nitems, s.block, s.smem, ls>>>(
                        s.items, (const BSub<T, TT>*)s.args, FSubAsync<T, TT, 2>{});
                else if (sub_form == 4)
                    k_batched<BSub<T, TT>, SINGLE_ARG(FSubAsync<T, TT, 2>), 2><<<s.nitems, s.block, s.smem, ls>>>(
                        s.items, (const BSub<T, TT>*)s.args, FSubAsync<T, TT, 2>{});
                else if (sub_form == 5)
                    k_batched<BSub<T, TT>, SINGLE_ARG(FSubAsync<T, TT, 3>), 2><<<s.nitems, s.block, s.smem, ls>>>(
                        s.items, (const BSub<T, TT>*)s.args, FSubAsync<T, TT, 3>{});
                else
                    k_batched<BSub<T, TT>, FSub<T, TT>, 4><<<s.nitems, s.block, s.smem, ls>>>(
                        s.items, (const BSub<T, TT>*)s.args, FSub<T, TT>{});
                break;
            BATCH_LAUNCH(BK_PREP, BPrep<T>, FPrep<T>, 4)
            case BK_STREAM:
                if (stream_minb == 2)  // registers bounded so that twice the blocks fit on an SM
                    k_batched<BStream<T>, FStream<T>, 2><<<s.nitems, s.block, s.smem, ls>>>(
                        s.items, (const BStream<T>*)s.args, FStream<T>{});
                else if (stream_minb == 3)  // blocks of at most 128 threads, three of them per SM
                    k_batched_b<BStream<T>, FStream<T>, 128, 3><<<s.nitems, s.block, s.smem, ls>>>(
                        s.items, (const BStream<T>*)s.args, FStream<T>{});
                else
                    k_batched<BStream<T>, FStream<T>, 1><<<s.nitems, s.block, s.smem, ls>>>(
                        s.items, (const BStream<T>*)s.args, FStream<T>{});
                break;
            BATCH_LAUNCH(BK_UPD, BUpd<T>, FUpd<T>, 4)
            BATCH_LAUNCH(BK_STAGE_END, BStageEnd, FStageEnd, 1)
            BATCH_LAUNCH(BK_PREC, BPrec<T>, FPrec<T>, 1)
            BATCH_LAUNCH(BK_ZERO, BZero, FZero, 1)
            BATCH_LAUNCH(BK_COPY, BCopy<T>, FCopy<T>, 1)
            BATCH_LAUNCH(AK_TRI_COEF, AStage<T>, FATriCoef<T>, 1)
            BATCH_LAUNCH(AK_TRI_FACT, ATriFact, FATriFact, 1)
            BATCH_LAUNCH(AK_UPDATE, AStageLP<T>, FAUpdate<T>, 1)
            BATCH_LAUNCH(AK_TR_REV, ATrRev, FATrRev, 1)
            BATCH_LAUNCH(AK_TR_SCATTER, ATrScatter<T>, FATrScatter<T>, 1)
            BATCH_LAUNCH(AK_MF, AStage<T>, FAMf<T>, 1)
            BATCH_LAUNCH(AK_SUB_VERT, ASub<T>, FASubVert<T>, 1)
            BATCH_LAUNCH(AK_SUB_RHS, ASub<T>, FASubRhs<T>, 1)
            BATCH_LAUNCH(AK_SUB_EXPL, ASub<T>, FASubExpl<T>, 1)
            BATCH_LAUNCH(AK_SUB_HORIZ, ASub<T>, FASubHoriz<T>, 1)
            BATCH_LAUNCH(AK_P0, AStageLP<T>, FAP0<T>, 1)
            BATCH_LAUNCH(AK_TRI_COEF_T, AStage<T>, FATriCoefT<T>, 1)
            BATCH_LAUNCH(AK_FACE_T, AStage<T>, FAFaceT<T>, 1)
            BATCH_LAUNCH(AK_STEP_END, AStepEnd, FAStepEnd, 1)
#define BATCH_LAUNCH_B(KIND, A, F, MAXT)                                                               \
    case KIND:                                                                                         \
        k_batched_b<A, F, MAXT, 1><<<s.nitems, s.block, s.smem, ls>>>(s.items, (const A*)s.args, F{}); \
        break;
#define BATCH_LAUNCH_B3(KIND, A, F, MAXT)                                                              \
    case KIND:                                                                                         \
        k_batched_b<A, F, MAXT, 3><<<s.nitems, s.block, s.smem, ls>>>(s.items, (const A*)s.args, F{}); \
        break;
            BATCH_LAUNCH_B3(AK_TR_JAC, ATrJac<T>, FATrJac<T>, ADJ_THREADS)  // registers for 3 blocks per SM
#undef BATCH_LAUNCH_B3
            BATCH_LAUNCH_B(AK_SUB_SOLVE, ASolve, FASubSolve, ADJ_SOLVE_THREADS)
            BATCH_LAUNCH_B(AK_TEND_T, AStage<T>, FATendT<T>, ADJ_THREADS)
            BATCH_LAUNCH_B(AK_DIAG_T, AStage<T>, FADiagT<T>, ADJ_THREADS)
            BATCH_LAUNCH_B(AK_KESSLER, APhys<T>, FAKessler<T>, ADJ_THREADS)
            BATCH_LAUNCH_B(AK_SED, APhys<T>, FASed<T>, ADJ_THREADS)
#undef BATCH_LAUNCH_B
            default:
                return set_berr(owner, MOIST_ERR_ARG, "unknown launch kind %d", s.kind);
        }
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return set_berr(owner, MOIST_ERR_CUDA, "batched launch failed: %s", cudaGetErrorString(e));
        return MOIST_OK;
    }
#undef BATCH_LAUNCH

    // the members' State buffers the two step graphs read at parity 0 (cur0) and 1 (nxt0)
    std::vector<StateP<T>> cur0, nxt0;

    // A member stepped on its own (its moist_rk3_step, moist_adjoint_run, ...) swaps its current
    // and next State; the graphs read the buffers of their parity, so move such a member's State
    // back into the buffer the next graph reads.
    int sync_members() {
        for (size_t i = 0; i < m.size(); i++) {
            const StateP<T>& want = parity == 0 ? cur0[i] : nxt0[i];
            const StateP<T>& other = parity == 0 ? nxt0[i] : cur0[i];
            if (m[i]->cur.rho == want.rho) continue;
            const T* src[7] = {m[i]->cur.rho, m[i]->cur.ru, m[i]->cur.rw, m[i]->cur.rt,
                               m[i]->cur.qv, m[i]->cur.qc, m[i]->cur.qr};
            T* dst[7] = {want.rho, want.ru, want.rw, want.rt, want.qv, want.qc, want.qr};
            for (int f = 0; f < 7; f++)
                BCK(cudaMemcpyAsync(dst[f], src[f], m[i]->fsz * sizeof(T), cudaMemcpyDeviceToDevice, st));
            m[i]->cur = want;
            m[i]->nxt = other;
        }
        return MOIST_OK;
    }

    // moist_batch_adjoint_run. nthreads <= 0: packed, every kernel of the members' forward,
    // recomputation and reverse steps one launch for all members (adjoint_packed); nthreads > 0:
    // every member's own moist_adjoint_run from up to nthreads host threads (adjoint_threads)
    int adjoint(int nsteps, int ckpt, const moist_adjoint_seed* seeds, moist_adjoint_grad* out,
                int nthreads) override {
        if (!out || nsteps < 1 || ckpt < 1)
            return set_berr(owner, MOIST_ERR_ARG, "moist_batch_adjoint_run needs out != NULL, nsteps >= 1, ckpt_every >= 1");
        return nthreads > 0 ? adjoint_threads(nsteps, ckpt, seeds, out, nthreads) : adjoint_packed(nsteps, ckpt, seeds, out);
    }

    // the members' device buffers allocated one member at a time first, then the members' runs
    // from up to nthreads host threads (each member works on its own stream, so their kernels
    // overlap on the GPU)
    int adjoint_threads(int nsteps, int ckpt, const moist_adjoint_seed* seeds, moist_adjoint_grad* out,
                        int nthreads) {
        const int n = (int)m.size();
        BCK(cudaStreamSynchronize(st));
        const int ck = std::min(ckpt, nsteps);
        for (int i = 0; i < n; i++) {
            if (m[i]->dp.do_sf || m[i]->dp.do_rd) break;  // reported by the member's own call
            if (int r = m[i]->adj_alloc(nsteps, ck))
                return set_berr(owner, r, "member %d: %s", i, m[i]->owner->err.c_str());
        }
        std::atomic<int> next{0};
        std::vector<int> rc(n, MOIST_OK);
        const int dev = owner->device;
        auto work = [&]() {
            cudaSetDevice(dev);
            for (int i; (i = next.fetch_add(1)) < n;)
                rc[i] = m[i]->adjoint_run(nsteps, ckpt, seeds ? seeds + i : nullptr, out + i);
        };
        const int nt = std::max(1, std::min(nthreads, n));
        std::vector<std::thread> th;
        for (int t = 1; t < nt; t++) th.emplace_back(work);
        work();
        for (auto& t : th) t.join();
        for (int i = 0; i < n; i++)
            if (rc[i] != MOIST_OK) {
                if (rc[i] == MOIST_ERR_NAN) owner->nan_member = i;
                return set_berr(owner, rc[i], "member %d: %s", i, m[i]->owner->err.c_str());
            }
        return MOIST_OK;
    }

    int tape_mode = -1;  // moist_batch_set_adjoint_tapes
    int set_tape_mode(int mode) override {
        tape_mode = mode;
        for (auto* c : m) c->tape_mode = mode;
        return MOIST_OK;
    }

    // ------------------------------------------------------------------ packed adjoint
    // Work lists per launch kind (built once per packed adjoint run) and the argument arrays of
    // its recorded phases, released when the run ends.
    std::vector<Slot> adj_kslot;
    std::vector<void*> adj_mem;

    void adj_release() {
        cudaStreamSynchronize(st);
        for (void* a : adj_mem) cudaFree(a);
        adj_mem.clear();
        adj_kslot.clear();
    }

    // the members' records of one phase as packed launches: every launch's argument structs
    // side by side in one device allocation, its work list shared by the launches of its kind
    int adj_pack(std::vector<StepRecord>& rec, std::vector<Slot>& out) {
        const int n = (int)m.size();
        for (int i = 1; i < n; i++)
            if (rec[i].kind != rec[0].kind)
                return set_berr(owner, MOIST_ERR_ARG, "member %d takes other adjoint launches than member 0", i);
        std::vector<size_t> off(rec[0].kind.size());
        size_t total = 0;
        for (size_t j = 0; j < rec[0].kind.size(); j++) {
            off[j] = total;
            total += (rec[0].args[j].size() * n + 255) / 256 * 256;
        }
        std::vector<unsigned char> h(std::max<size_t>(total, 1));
        for (size_t j = 0; j < rec[0].kind.size(); j++) {
            const size_t sz = rec[0].args[j].size();
            for (int i = 0; i < n; i++) std::memcpy(h.data() + off[j] + sz * i, rec[i].args[j].data(), sz);
        }
        void* d = nullptr;
        if (cudaMalloc(&d, h.size()) != cudaSuccess)
            return set_berr(owner, MOIST_ERR_NOMEM, "cudaMalloc of %zu bytes of adjoint launch arguments failed", h.size());
        adj_mem.push_back(d);
        BCK(cudaMemcpy(d, h.data(), h.size(), cudaMemcpyHostToDevice));
        if (adj_kslot.empty()) adj_kslot.resize(AK_NKINDS);
        for (size_t j = 0; j < rec[0].kind.size(); j++) {
            const int kind = rec[0].kind[j];
            Slot& ks = adj_kslot[kind];
            if (!ks.items) {
                std::vector<BItem> it;
                ks.kind = kind;
                items_of(kind, it, ks.block, ks.smem, -1);
                void* di = nullptr;
                if (cudaMalloc(&di, std::max<size_t>(it.size(), 1) * sizeof(BItem)) != cudaSuccess)
                    return set_berr(owner, MOIST_ERR_NOMEM, "cudaMalloc of an adjoint work list failed");
                adj_mem.push_back(di);
                BCK(cudaMemcpy(di, it.data(), it.size() * sizeof(BItem), cudaMemcpyHostToDevice));
                ks.items = (const BItem*)di;
                ks.nitems = (unsigned)it.size();
            }
            Slot sl = ks;
            sl.args = (const unsigned char*)d + off[j];
            sl.group = 0;
            if (sl.nitems) out.push_back(sl);
        }
        return MOIST_OK;
    }

    int run_slots(const std::vector<Slot>& sl) {
        for (const Slot& s : sl)
            if (int r = launch(s, st)) return r;
        return MOIST_OK;
    }

    // the members' current State in the buffers the graph of parity 0 reads
    void at_parity0() {
        for (size_t i = 0; i < m.size(); i++) {
            m[i]->cur = cur0[i];
            m[i]->nxt = nxt0[i];
        }
        parity = 0;
    }

    int adjoint_packed(int nsteps, int ckpt, const moist_adjoint_seed* seeds, moist_adjoint_grad* out) {
        const int n = (int)m.size();
        for (int i = 0; i < n; i++)
            if (int r = m[i]->adj_check(nsteps, ckpt, out + i))
                return set_berr(owner, r, "member %d: %s", i, m[i]->owner->err.c_str());
        if (int r = sync_members()) return r;
        BCK(cudaStreamSynchronize(st));
        const int ck = std::min(ckpt, nsteps);
        // one tape mode for every member: a tape per step of a segment when all of them fit in
        // half the free device memory, else one tape and the segment's States
        size_t free_b = 0, total_b = 0;
        BCK(cudaMemGetInfo(&free_b, &total_b));
        size_t need = 0;
        for (int i = 0; i < n; i++) {
            const size_t have = m[i]->adj ? m[i]->adj->tapes.size() : 0;
            if (have < (size_t)ck) need += (ck - have) * m[i]->tape_fields() * m[i]->fsz * sizeof(T);
        }
        const bool seg = tape_mode >= 0 ? tape_mode == 1 : need <= free_b / 2;
        for (int i = 0; i < n; i++)
            if (int r = m[i]->adj_alloc(nsteps, ck, seg ? 1 : 0))
                return set_berr(owner, r, "member %d: %s", i, m[i]->owner->err.c_str());
        // every member's work on the batch stream for the run
        std::vector<cudaStream_t> own(n);
        for (int i = 0; i < n; i++) {
            own[i] = m[i]->st;
            m[i]->st = st;
        }
        int r = adjoint_packed_run(nsteps, ck, seg, seeds, out);
        for (int i = 0; i < n; i++) {
            m[i]->rec = nullptr;
            m[i]->tape = nullptr;
            m[i]->st = own[i];
        }
        adj_release();
        return r;
    }

    int adjoint_packed_run(int nsteps, int ck, bool seg, const moist_adjoint_seed* seeds, moist_adjoint_grad* out) {
        const int n = (int)m.size();
        int r;
        auto member_err = [&](int i, int rc) {
            if (rc == MOIST_ERR_NAN) owner->nan_member = i;
            return set_berr(owner, rc, "member %d: %s", i, m[i]->owner->err.c_str());
        };
        for (int i = 0; i < n; i++)
            if ((r = m[i]->adj_seeds(seeds ? seeds + i : nullptr)) != MOIST_OK) return member_err(i, r);
        // the recomputed (taped) forward steps and the reverse steps, per tape: with a tape per
        // step of a segment, step j of a segment starts from the States of parity j % 2
        const int ntapes = seg ? ck : 1;
        std::vector<std::vector<Slot>> taped(ntapes), rev(ntapes);
        for (int j = 0; j < ntapes; j++) {
            std::vector<StepRecord> rf(n), ra(n);
            const int pj = seg ? j % 2 : 0;
            for (int i = 0; i < n; i++) {
                m[i]->cur = pj == 0 ? cur0[i] : nxt0[i];
                m[i]->nxt = pj == 0 ? nxt0[i] : cur0[i];
                m[i]->tape = &m[i]->adj->tapes[j];
                m[i]->rec = &rf[i];
                r = m[i]->launch_step();
                m[i]->tape = nullptr;
                if (r == MOIST_OK) {
                    m[i]->rec = &ra[i];
                    r = m[i]->adj_step(m[i]->adj->tapes[j]);
                }
                m[i]->rec = nullptr;
                if (r != MOIST_OK) return member_err(i, r);
            }
            if ((r = adj_pack(rf, taped[j])) != MOIST_OK) return r;
            if ((r = adj_pack(ra, rev[j])) != MOIST_OK) return r;
        }
        for (int i = 0; i < n; i++) {  // back to the members' current States
            m[i]->cur = parity == 0 ? cur0[i] : nxt0[i];
            m[i]->nxt = parity == 0 ? nxt0[i] : cur0[i];
        }
        auto copy_to = [&](int i, const std::array<T*, 7>& src, const std::array<T*, 7>& dst) {
            return m[i]->copyf(src.data(), dst.data(), 7);
        };
        // forward run through the step graphs, keeping the States every ck steps
        const auto t0 = std::chrono::steady_clock::now();
        for (int s = 0; s < nsteps; s++) {
            if (s % ck == 0)
                for (int i = 0; i < n; i++)
                    if ((r = copy_to(i, m[i]->cur_fields(), m[i]->adj->ck[s / ck])) != MOIST_OK) return member_err(i, r);
            if ((r = launch_steps(1)) != MOIST_OK) return r;
        }
        BCK(cudaStreamSynchronize(st));
        const auto t1 = std::chrono::steady_clock::now();
        for (int i = 0; i < n; i++)
            if ((r = m[i]->adj_begin()) != MOIST_OK) return member_err(i, r);
        // reverse sweep, one segment of ck steps at a time
        const int nck = (nsteps + ck - 1) / ck;
        for (int sg = nck - 1; sg >= 0; sg--) {
            const int n0 = sg * ck, n1 = std::min(n0 + ck, nsteps);
            at_parity0();
            for (int i = 0; i < n; i++) {
                if ((r = copy_to(i, m[i]->adj->ck[sg], m[i]->cur_fields())) != MOIST_OK) return member_err(i, r);
                if (!seg && (r = copy_to(i, m[i]->adj->ck[sg], m[i]->adj->seg[0])) != MOIST_OK) return member_err(i, r);
            }
            if (seg) {  // recompute the segment once, taping every step
                for (int s = n0; s < n1; s++) {
                    if ((r = run_slots(taped[s - n0])) != MOIST_OK) return r;
                    parity ^= 1;
                    for (auto* c : m) std::swap(c->cur, c->nxt);
                }
                for (int s = n1 - 1; s >= n0; s--)
                    if ((r = run_slots(rev[s - n0])) != MOIST_OK) return r;
                continue;
            }
            for (int s = n0; s < n1 - 1; s++) {
                if ((r = launch_steps(1)) != MOIST_OK) return r;
                for (int i = 0; i < n; i++)
                    if ((r = copy_to(i, m[i]->cur_fields(), m[i]->adj->seg[s - n0 + 1])) != MOIST_OK)
                        return member_err(i, r);
            }
            for (int s = n1 - 1; s >= n0; s--) {
                at_parity0();
                for (int i = 0; i < n; i++)
                    if ((r = copy_to(i, m[i]->adj->seg[s - n0], m[i]->cur_fields())) != MOIST_OK) return member_err(i, r);
                if ((r = run_slots(taped[0])) != MOIST_OK) return r;
                parity = 1;
                for (auto* c : m) std::swap(c->cur, c->nxt);
                if ((r = run_slots(rev[0])) != MOIST_OK) return r;
            }
        }
        BCK(cudaStreamSynchronize(st));
        const auto t2 = std::chrono::steady_clock::now();
        const double fwd = std::chrono::duration<double, std::milli>(t1 - t0).count();
        const double rv = std::chrono::duration<double, std::milli>(t2 - t1).count();
        for (int i = 0; i < n; i++)
            if ((r = m[i]->adj_results(seeds ? seeds + i : nullptr, out + i, fwd, rv)) != MOIST_OK)
                return member_err(i, r);
        return MOIST_OK;
    }

    int build() {
        const int n = (int)m.size();
        for (auto* c : m) {
            cur0.push_back(c->cur);
            nxt0.push_back(c->nxt);
            // a batch has blocks enough for every SM without narrow strips: take the widest
            // strip whose shared memory leaves room for several blocks per SM
            for (int w : {8, 4, 2, 1}) {
                if (w == 1 || strip_smem_bytes<T, TT>(c->nz, w) <= 64 * 1024) {
                    c->strip_wc = w;
                    c->strip_smem = strip_smem_bytes<T, TT>(c->nz, w);
                    break;
                }
            }
            max_strip_smem = std::max(max_strip_smem, c->strip_smem);
            max_rows = std::max(max_rows, (c->nz + 31) / 32 * 32);
        }
        {  // the limit is shared by every batch of the process: allow the device maximum
            int optin = 0;
            BCK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, owner->device));
            BCK(cudaFuncSetAttribute(k_batched<SINGLE_ARG(BThomas<T, TT>), SINGLE_ARG(FThomasStrip<T, TT>), 4>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
            BCK(cudaFuncSetAttribute(k_batched<SINGLE_ARG(BSub<T, TT>), SINGLE_ARG(FSubStrip<T, TT>), 4>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
            BCK(cudaFuncSetAttribute(k_batched<SINGLE_ARG(BSub<T, TT>), SINGLE_ARG(FSubAsync<T, TT, 2>), 3>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
            BCK(cudaFuncSetAttribute(k_batched<SINGLE_ARG(BSub<T, TT>), SINGLE_ARG(FSubAsync<T, TT, 2>), 2>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
            BCK(cudaFuncSetAttribute(k_batched<SINGLE_ARG(BSub<T, TT>), SINGLE_ARG(FSubAsync<T, TT, 3>), 2>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
            BCK(cudaFuncSetAttribute(k_batched_b<ASolve, FASubSolve, ADJ_SOLVE_THREADS, 1>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
        }
        for (int q = 0; q < 2; q++) {
            std::vector<StepRecord> rec(n);
            for (int i = 0; i < n; i++) {
                m[i]->rec = &rec[i];
                const int r = m[i]->launch_step();  // records; swaps the member's current and next State
                m[i]->rec = nullptr;
                if (r != MOIST_OK)
                    return set_berr(owner, r, "member %d: %s", i, m[i]->owner->err.c_str());
            }
            for (int i = 1; i < n; i++)
                if (rec[i].kind != rec[0].kind)
                    return set_berr(owner, MOIST_ERR_ARG,
                                    "member %d takes other launches than member 0 (ns, do_sf and do_rd must agree)", i);
            for (size_t j = 0; j < rec[0].kind.size(); j++) {
                const size_t sz = rec[0].args[j].size();
                std::vector<unsigned char> packed(sz * n);
                for (int i = 0; i < n; i++) std::memcpy(packed.data() + sz * i, rec[i].args[j].data(), sz);
                unsigned char* dargs;
                if (int r = dalloc(&dargs, packed.size())) return r;
                BCK(cudaMemcpy(dargs, packed.data(), packed.size(), cudaMemcpyHostToDevice));
                launches[q].push_back(Launch{rec[0].kind[j], dargs});
            }
        }
        for (int g = 1; g < MAX_GROUPS; g++) {
            BCK(cudaStreamCreateWithFlags(&gstream[g], cudaStreamNonBlocking));
            BCK(cudaEventCreateWithFlags(&gjoin[g], cudaEventDisableTiming));
        }
        BCK(cudaEventCreateWithFlags(&gfork, cudaEventDisableTiming));
        assign_groups(1);
        std::vector<int*> ev(n);
        for (int i = 0; i < n; i++) ev[i] = m[i]->err;
        if (int r = dalloc(&errs, n)) return r;
        if (int r = dalloc(&err_all, 4 * n)) return r;
        BCK(cudaMemcpy(errs, ev.data(), n * sizeof(int*), cudaMemcpyHostToDevice));
        return rebuild_slots();
    }

    // G groups of members, dealt in turn from the longest sweeps (nx + nz) down, so that every
    // group holds long and short members
    void assign_groups(int G) {
        const int n = (int)m.size();
        ngroups = std::max(1, std::min(G, n));
        std::vector<int> order(n);
        for (int i = 0; i < n; i++) order[i] = i;
        std::stable_sort(order.begin(), order.end(),
                         [&](int a, int b) { return m[a]->nx + m[a]->nz > m[b]->nx + m[b]->nz; });
        grp.assign(n, 0);
        for (int r = 0; r < n; r++) grp[order[r]] = r % ngroups;
    }

    // the work lists of every launch for the current groups, forms and block sizes, and new graphs
    std::vector<void*> item_allocs;
    int rebuild_slots() {
        BCK(cudaStreamSynchronize(st));  // no graph that reads the old work lists is in flight
        for (void* a : item_allocs) cudaFree(a);
        item_allocs.clear();
        for (int q = 0; q < 2; q++) {
            slots[q].clear();
            for (int g = 0; g < ngroups; g++)
                for (const Launch& L : launches[q]) {
                    Slot sl{};
                    sl.kind = L.kind;
                    sl.args = L.args;
                    sl.group = g;
                    std::vector<BItem> it;
                    items_of(sl.kind, it, sl.block, sl.smem, g);
                    if (it.empty()) continue;
                    void* d = nullptr;
                    cudaError_t e = cudaMalloc(&d, it.size() * sizeof(BItem));
                    if (e != cudaSuccess) return set_berr(owner, MOIST_ERR_NOMEM, "cudaMalloc of a work list failed");
                    item_allocs.push_back(d);
                    BCK(cudaMemcpy(d, it.data(), it.size() * sizeof(BItem), cudaMemcpyHostToDevice));
                    sl.items = (const BItem*)d;
                    sl.nitems = (unsigned)it.size();
                    slots[q].push_back(sl);
                }
        }
        return capture();
    }

    // the two step graphs (even and odd step) from the packed slots
    int capture() {
        for (int q = 0; q < 2; q++) {
            if (exec[q]) {
                cudaGraphExecDestroy(exec[q]);
                exec[q] = nullptr;
            }
            cudaGraph_t g;
            BCK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
            int r = MOIST_OK;
            cudaError_t ef = cudaSuccess;
            if (ngroups > 1) {  // fork: the groups' chains become parallel branches of the graph
                ef = cudaEventRecord(gfork, st);
                for (int g2 = 1; g2 < ngroups && ef == cudaSuccess; g2++) ef = cudaStreamWaitEvent(gstream[g2], gfork, 0);
            }
            for (const Slot& sl : slots[q]) {
                if (ef != cudaSuccess) break;
                if ((r = launch(sl, sl.group == 0 ? st : gstream[sl.group])) != MOIST_OK) break;
            }
            for (int g2 = 1; g2 < ngroups; g2++) {  // join every branch back before the capture ends
                cudaEventRecord(gjoin[g2], gstream[g2]);
                cudaStreamWaitEvent(st, gjoin[g2], 0);
            }
            cudaError_t e = cudaStreamEndCapture(st, &g);
            if (ef != cudaSuccess && e == cudaSuccess) e = ef;
            if (r != MOIST_OK) return r;
            if (e != cudaSuccess) return set_berr(owner, MOIST_ERR_CUDA, "stream capture failed: %s", cudaGetErrorString(e));
            e = cudaGraphInstantiate(&exec[q], g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) return set_berr(owner, MOIST_ERR_CUDA, "graph instantiation failed: %s", cudaGetErrorString(e));
        }
        return MOIST_OK;
    }

    // new work lists for the per-column kernels (ct threads per block, or column strips when
    // ct == 0) and new graphs
    int set_col_threads(int ct) {
        sub_strips = ct == 0;
        if (ct > 0) col_threads = ct;
        return rebuild_slots();
    }

    // Times nsteps batch steps for the factorisation and acoustic substep over column strips and
    // one thread per column with 32, 64, 128 and 256 threads per block, each from the same saved
    // States, keeps the fastest and restores the States (same results for every choice).
    int autotune(int nsteps, std::string& report) override {
        if (nsteps < 1) return set_berr(owner, MOIST_ERR_ARG, "moist_batch_autotune needs nsteps >= 1");
        if (int r = sync_members()) return r;
        const int n = (int)m.size();
        std::vector<std::array<T*, 8>>& save = tune_save;
        if (save.empty()) {  // kept for later calls
            save.resize(n);
            tune_halo.resize(n);
            for (int i = 0; i < n; i++)
                if (int r = dalloc(&tune_halo[i], 2)) return r;
            for (int i = 0; i < n; i++) {
                for (int f = 0; f < 7; f++)
                    if (int r = dalloc(&save[i][f], m[i]->fsz)) return r;
                if (int r = dalloc(&save[i][7], (size_t)m[i]->P)) return r;
            }
        }
        auto copy_all = [&](bool to_save) -> int {
            for (int i = 0; i < n; i++) {
                const auto cf = m[i]->cur_fields();
                for (int f = 0; f < 7; f++) {
                    T* a = to_save ? save[i][f] : cf[f];
                    const T* b = to_save ? cf[f] : save[i][f];
                    BCK(cudaMemcpyAsync(a, b, m[i]->fsz * sizeof(T), cudaMemcpyDeviceToDevice, st));
                }
                T* a = to_save ? save[i][7] : m[i]->prec;
                const T* b = to_save ? m[i]->prec : save[i][7];
                BCK(cudaMemcpyAsync(a, b, m[i]->P * sizeof(T), cudaMemcpyDeviceToDevice, st));
                T* ha = to_save ? tune_halo[i] : m[i]->halo_vals;  // carried by the surface fluxes
                const T* hb = to_save ? m[i]->halo_vals : tune_halo[i];
                BCK(cudaMemcpyAsync(ha, hb, 2 * sizeof(T), cudaMemcpyDeviceToDevice, st));
            }
            return MOIST_OK;
        };
        if (int r = copy_all(true)) return r;
        float best = 1e30f;
        int bct = sub_strips ? 0 : col_threads;
        char buf[96];
        unsigned long long* hb;
        if (int r = dalloc(&hb, 1)) return r;
        unsigned long long h0 = 0;
        bool first = true;
        int bform = sub_form;
        struct SubCand {
            int ct, form;
        };
        std::vector<SubCand> sub_cands{{0, 0}};
        for (int form : {4, 5, 3, 1, 2, 0})
            for (int ct : {32, 64, 128, 256}) sub_cands.push_back({ct, form});
        for (const SubCand& sc : sub_cands) {
            const int ct = sc.ct;
            sub_form = sc.form;
            if (int r = set_col_threads(ct)) return r;
            if (int r = copy_all(false)) return r;
            float ms = 0.f;
            if (int r = launch_steps(1)) return r;  // warm-up
            if (int r = time_steps(nsteps, &ms)) return r;
            // every candidate starts from the same States: their results must agree bit for bit
            BCK(cudaMemsetAsync(hb, 0, sizeof(unsigned long long), st));
            for (int i = 0; i < n; i++) {
                const auto cf = m[i]->cur_fields();
                for (int f = 0; f < 7; f++) k_hash<T><<<64, 256, 0, st>>>(cf[f], m[i]->fsz, hb);
                k_hash<T><<<1, 256, 0, st>>>(m[i]->prec, (size_t)m[i]->P, hb);
            }
            unsigned long long h = 0;
            BCK(cudaMemcpyAsync(&h, hb, sizeof h, cudaMemcpyDeviceToHost, st));
            BCK(cudaStreamSynchronize(st));
            if (first) {
                h0 = h;
                first = false;
            } else if (h != h0) {
                return set_berr(owner, MOIST_ERR_CUDA,
                                "autotune: column block %d form %d gives other States than column strips", ct, sc.form);
            }
            ms /= nsteps;
            if (ct == 0)
                snprintf(buf, sizeof buf, "%scolumn strips: %.2f ms", report.empty() ? "" : "; ", ms);
            else
                snprintf(buf, sizeof buf, "%scolumn block %d form %d: %.2f ms", report.empty() ? "" : "; ", ct,
                         sc.form, ms);
            report += buf;
            if (ms < best) {
                best = ms;
                bct = ct;
                bform = sc.form;
            }
        }
        sub_form = bform;
        // then, with that form, the register bound of the streaming tracer sweep
        int bmb = stream_minb;
        float best_mb = 1e30f;
        for (int mb : {1, 2, 3}) {
            if (mb == 3 && max_rows > 128) continue;  // the 128-thread bound needs rows <= 128
            stream_minb = mb;
            if (int r = set_col_threads(bct)) return r;  // recaptures the graphs
            if (int r = copy_all(false)) return r;
            float ms = 0.f;
            if (int r = launch_steps(1)) return r;
            if (int r = time_steps(nsteps, &ms)) return r;
            BCK(cudaMemsetAsync(hb, 0, sizeof(unsigned long long), st));
            for (int i = 0; i < n; i++) {
                const auto cf = m[i]->cur_fields();
                for (int f = 0; f < 7; f++) k_hash<T><<<64, 256, 0, st>>>(cf[f], m[i]->fsz, hb);
                k_hash<T><<<1, 256, 0, st>>>(m[i]->prec, (size_t)m[i]->P, hb);
            }
            unsigned long long h = 0;
            BCK(cudaMemcpyAsync(&h, hb, sizeof h, cudaMemcpyDeviceToHost, st));
            BCK(cudaStreamSynchronize(st));
            if (h != h0)
                return set_berr(owner, MOIST_ERR_CUDA, "autotune: tracer register bound %d gives other States", mb);
            ms /= nsteps;
            snprintf(buf, sizeof buf, "; tracer bound %d: %.2f ms", mb, ms);
            report += buf;
            if (ms < best_mb) {
                best_mb = ms;
                bmb = mb;
            }
        }
        best = best_mb;
        stream_minb = bmb;
        // then the number of member groups whose chains run as parallel branches of the graph
        int bg = 1;
        float best_g = best;
        for (int G : {2, 4}) {
            if (G > (int)m.size()) continue;
            assign_groups(G);
            if (int r = set_col_threads(bct)) return r;  // new work lists and graphs
            if (int r = copy_all(false)) return r;
            float ms = 0.f;
            if (int r = launch_steps(1)) return r;
            if (int r = time_steps(nsteps, &ms)) return r;
            BCK(cudaMemsetAsync(hb, 0, sizeof(unsigned long long), st));
            for (int i = 0; i < n; i++) {
                const auto cf = m[i]->cur_fields();
                for (int f = 0; f < 7; f++) k_hash<T><<<64, 256, 0, st>>>(cf[f], m[i]->fsz, hb);
                k_hash<T><<<1, 256, 0, st>>>(m[i]->prec, (size_t)m[i]->P, hb);
            }
            unsigned long long h = 0;
            BCK(cudaMemcpyAsync(&h, hb, sizeof h, cudaMemcpyDeviceToHost, st));
            BCK(cudaStreamSynchronize(st));
            if (h != h0) return set_berr(owner, MOIST_ERR_CUDA, "autotune: %d member groups give other States", G);
            ms /= nsteps;
            snprintf(buf, sizeof buf, "; %d groups: %.2f ms", G, ms);
            report += buf;
            if (ms < best_g) {
                best_g = ms;
                bg = G;
            }
        }
        best = best_g;
        assign_groups(bg);
        if (int r = set_col_threads(bct)) return r;
        if (int r = copy_all(false)) return r;
        BCK(cudaStreamSynchronize(st));
        if (bct == 0)
            snprintf(buf, sizeof buf, " -> column strips, tracer bound %d, %d groups (%.2f ms per step)", bmb, ngroups,
                     best);
        else
            snprintf(buf, sizeof buf, " -> column block %d form %d, tracer bound %d, %d groups (%.2f ms per step)", bct,
                     sub_form, bmb, ngroups, best);
        report += buf;
        return MOIST_OK;
    }

    int launch_steps(int nsteps) {
        for (int j = 0; j < nsteps; j++) {
            BCK(cudaGraphLaunch(exec[parity], st));
            parity ^= 1;
            for (auto* c : m) std::swap(c->cur, c->nxt);
        }
        return MOIST_OK;
    }

    int step(int nsteps) override {
        const int n = (int)m.size();
        if (int r = sync_members()) return r;
        k_reset_err<<<cdiv(n, 128), 128, 0, st>>>(errs, n);
        if (int r = launch_steps(nsteps)) return r;
        k_gather_err<<<cdiv(n, 128), 128, 0, st>>>(errs, n, err_all);
        std::vector<int> h(4 * (size_t)n);
        BCK(cudaMemcpyAsync(h.data(), err_all, h.size() * sizeof(int), cudaMemcpyDeviceToHost, st));
        BCK(cudaStreamSynchronize(st));
        BCK(cudaGetLastError());
        owner->nan_member = -1;
        owner->nan_field = -1;
        for (int i = 0; i < n; i++) {
            if (h[4 * i] != INT_MAX) {
                static const char* names[12] = {"rho", "rho_u", "rho_w", "rho_theta", "rho_qv", "rho_qc", "rho_qr",
                                                "d_rho_u_phys", "d_rho_theta_phys", "d_rho_qv_phys", "d_rho_qc_phys",
                                                "d_rho_qr_phys"};
                owner->nan_member = i;
                owner->nan_field = h[4 * i];
                m[i]->owner->nan_field = h[4 * i];
                const char* nm = h[4 * i] >= 0 && h[4 * i] < 12 ? names[h[4 * i]] : "?";
                m[i]->owner->err = std::string("NaN detected in ") + nm;
                return set_berr(owner, MOIST_ERR_NAN, "member %d: NaN detected in %s", i, nm);
            }
        }
        return MOIST_OK;
    }

    // nsteps without the graphs: events around every packed launch, summed per kernel group
    int profile(int nsteps, float* total_ms, float* group_ms) override {
        if (int r = sync_members()) return r;
        static const int group_of[BK_NKINDS] = {MOIST_KGROUP_PHYSICS,  MOIST_KGROUP_PHYSICS, MOIST_KGROUP_PHYSICS,
                                                MOIST_KGROUP_PHYSICS,  MOIST_KGROUP_PROLOGUE, MOIST_KGROUP_PROLOGUE,
                                                MOIST_KGROUP_PROLOGUE, MOIST_KGROUP_SUBSTEP, MOIST_KGROUP_TRACER,
                                                MOIST_KGROUP_TRACER,   MOIST_KGROUP_UPDATE,  MOIST_KGROUP_UPDATE,
                                                MOIST_KGROUP_OTHER};
        size_t per = slots[0].size() + slots[1].size();
        std::vector<cudaEvent_t> ev(nsteps * (per + 2) + 1);
        for (auto& e : ev) BCK(cudaEventCreate(&e));
        std::vector<int> kinds;
        size_t j = 0;
        BCK(cudaEventRecord(ev[j++], st));
        for (int n = 0; n < nsteps; n++) {
            for (const Slot& sl : slots[parity]) {
                if (int r = launch(sl, st)) return r;
                kinds.push_back(sl.kind);
                BCK(cudaEventRecord(ev[j++], st));
            }
            parity ^= 1;
            for (auto* c : m) std::swap(c->cur, c->nxt);
        }
        BCK(cudaEventSynchronize(ev[j - 1]));
        for (int g = 0; g < MOIST_NGROUPS; g++) group_ms[g] = 0.f;
        for (size_t q = 0; q < kinds.size(); q++) {
            float t;
            BCK(cudaEventElapsedTime(&t, ev[q], ev[q + 1]));
            group_ms[group_of[kinds[q]]] += t;
        }
        BCK(cudaEventElapsedTime(total_ms, ev[0], ev[j - 1]));
        for (auto& e : ev) cudaEventDestroy(e);
        return MOIST_OK;
    }

    int time_steps(int nsteps, float* ms) override {
        if (int r = sync_members()) return r;
        cudaEvent_t e0, e1;
        BCK(cudaEventCreate(&e0));
        BCK(cudaEventCreate(&e1));
        BCK(cudaEventRecord(e0, st));
        int r = launch_steps(nsteps);
        BCK(cudaEventRecord(e1, st));
        BCK(cudaEventSynchronize(e1));
        BCK(cudaEventElapsedTime(ms, e0, e1));
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        return r;
    }
};

}  // namespace

// ============================================================================ C-ABI

extern "C" {
#pragma GCC visibility push(default)

int moist_abi_version(void) { return MOIST2D_ABI_VERSION; }

const char* moist_status_string(int s) {
    switch (s) {
        case MOIST_OK: return "ok";
        case MOIST_ERR_NAN: return "NaN detected";
        case MOIST_ERR_ARG: return "invalid argument";
        case MOIST_ERR_CUDA: return "CUDA error";
        case MOIST_ERR_TIMEOUT: return "device wait timed out";
        case MOIST_ERR_UNSUPPORTED: return "unsupported";
        case MOIST_ERR_NOMEM: return "out of device memory";
        case MOIST_ERR_IO: return "file error";
        default: return "unknown status";
    }
}

int moist_ctx_create(const moist_params* p, int precision, int flags, moist_ctx** out) {
    if (!out) return MOIST_ERR_ARG;
    *out = nullptr;
    if (!p || !p->zf || !p->dz || !p->z) return MOIST_ERR_ARG;
    // any halo / nx >= 1 is accepted for the physics entry points (the reference's own
    // microphysics testset uses halo = 0, Nx = 1); the RK stages need halo = 2 and nx >= 2
    if (p->nx < 1 || p->nz < 2 || p->halo < 0 || p->ns < 1 || p->nz > 1024) return MOIST_ERR_ARG;
    if (precision != MOIST_F32 && precision != MOIST_F64) return MOIST_ERR_ARG;
    moist_ctx* c = new moist_ctx();
    if (cudaGetDevice(&c->device) != cudaSuccess) {
        delete c;
        return MOIST_ERR_CUDA;
    }
    c->precision = precision;
    c->flags = flags;
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete c;
        return MOIST_ERR_CUDA;
    }
    int r;
    if (precision == MOIST_F64) {
        auto* x = new Ctx<double, double>(c);
        c->impl = x;
        r = x->init(p);
    } else if (flags & MOIST_FLAG_TRI_NATIVE) {
        auto* x = new Ctx<float, float>(c);
        c->impl = x;
        r = x->init(p);
    } else {
        auto* x = new Ctx<float, double>(c);
        c->impl = x;
        r = x->init(p);
    }
    if (r != MOIST_OK) {
        delete c->impl;
        cudaStreamDestroy(c->stream);
        delete c;
        return r;
    }
    *out = c;
    return MOIST_OK;
}

int moist_ctx_destroy(moist_ctx* c) {
    if (!c) return MOIST_ERR_ARG;
    cudaSetDevice(c->device);  // best effort: the context is released either way
    delete c->impl;
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return MOIST_OK;
}

const char* moist_last_error(const moist_ctx* c) { return c ? c->err.c_str() : "null context"; }

// ------------------------------------------------------------------------- ensembles

int moist_batch_destroy(moist_batch* b) {
    if (!b) return MOIST_ERR_ARG;
    cudaSetDevice(b->device);  // best effort: the batch is released either way
    delete b->impl;
    for (moist_ctx* c : b->members) moist_ctx_destroy(c);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return MOIST_OK;
}

int moist_batch_create(const moist_params* members, int nmembers, int precision, int flags, moist_batch** out) {
    if (!out) return MOIST_ERR_ARG;
    *out = nullptr;
    if (!members || nmembers < 1 || (precision != MOIST_F32 && precision != MOIST_F64)) return MOIST_ERR_ARG;
    for (int i = 0; i < nmembers; i++) {
        if (members[i].halo != 2 || members[i].nx < 2) return MOIST_ERR_ARG;
        if (members[i].nz > STREAM_MAX_ROWS) return MOIST_ERR_UNSUPPORTED;
        if (members[i].ns != members[0].ns) return MOIST_ERR_ARG;
    }
    moist_batch* b = new moist_batch();
    b->precision = precision;
    if (cudaGetDevice(&b->device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete b;
        return MOIST_ERR_CUDA;
    }
    const int mflags = (flags & MOIST_FLAG_TRI_NATIVE) | MOIST_FLAG_TRACER_STREAM;
    for (int i = 0; i < nmembers; i++) {
        moist_ctx* c = nullptr;
        const int r = moist_ctx_create(&members[i], precision, mflags, &c);
        if (r != MOIST_OK) {
            moist_batch_destroy(b);
            return r;
        }
        b->members.push_back(c);
    }
    int r;
    if (precision == MOIST_F64) {
        std::vector<Ctx<double, double>*> v;
        for (auto* c : b->members) v.push_back(static_cast<Ctx<double, double>*>(c->impl));
        auto* x = new BatchImpl<double, double>(b, v);
        b->impl = x;
        r = x->build();
    } else if (flags & MOIST_FLAG_TRI_NATIVE) {
        std::vector<Ctx<float, float>*> v;
        for (auto* c : b->members) v.push_back(static_cast<Ctx<float, float>*>(c->impl));
        auto* x = new BatchImpl<float, float>(b, v);
        b->impl = x;
        r = x->build();
    } else {
        std::vector<Ctx<float, double>*> v;
        for (auto* c : b->members) v.push_back(static_cast<Ctx<float, double>*>(c->impl));
        auto* x = new BatchImpl<float, double>(b, v);
        b->impl = x;
        r = x->build();
    }
    if (r != MOIST_OK) {
        moist_batch_destroy(b);
        return r;
    }
    *out = b;
    return MOIST_OK;
}

moist_ctx* moist_batch_member(moist_batch* b, int member) {
    return (b && member >= 0 && member < (int)b->members.size()) ? b->members[member] : nullptr;
}

int moist_batch_upload(moist_batch* b, int member, const moist_state_host* s) {
    moist_ctx* c = moist_batch_member(b, member);
    return c ? moist_upload_state(c, s) : MOIST_ERR_ARG;
}

int moist_batch_download(moist_batch* b, int member, moist_state_host* s) {
    moist_ctx* c = moist_batch_member(b, member);
    return c ? moist_download_state(c, s) : MOIST_ERR_ARG;
}

int moist_batch_adjoint_run(moist_batch* b, int nsteps, int ckpt_every, const moist_adjoint_seed* seeds,
                            moist_adjoint_grad* out, int nthreads) {
    if (!b) return MOIST_ERR_ARG;
    if (cudaSetDevice(b->device) != cudaSuccess) return MOIST_ERR_CUDA;
    return b->impl->adjoint(nsteps, ckpt_every, seeds, out, nthreads);
}

int moist_history_diagnostics(moist_ctx* c, void* const out[MOIST_NDIAG], double summary[6]) {
    if (!c) return MOIST_ERR_ARG;
    if (cudaSetDevice(c->device) != cudaSuccess) return MOIST_ERR_CUDA;
    return c->impl->history(out, summary);
}

int moist_autotune(moist_ctx* c, int nsteps, char* report, size_t report_len) {
    if (!c) return MOIST_ERR_ARG;
    if (cudaSetDevice(c->device) != cudaSuccess) return MOIST_ERR_CUDA;
    std::string rep;
    const int r = c->impl->autotune(nsteps, rep);
    if (report && report_len) snprintf(report, report_len, "%s", rep.c_str());
    return r;
}

int moist_batch_autotune(moist_batch* b, int nsteps, char* report, size_t report_len) {
    if (!b) return MOIST_ERR_ARG;
    if (cudaSetDevice(b->device) != cudaSuccess) return MOIST_ERR_CUDA;
    std::string rep;
    const int r = b->impl->autotune(nsteps, rep);
    if (report && report_len) snprintf(report, report_len, "%s", rep.c_str());
    return r;
}

int moist_batch_step(moist_batch* b, int nsteps) {
    if (!b || nsteps < 0) return MOIST_ERR_ARG;
    if (cudaSetDevice(b->device) != cudaSuccess) return MOIST_ERR_CUDA;
    return b->impl->step(nsteps);
}

int moist_batch_time_steps(moist_batch* b, int nsteps, float* ms) {
    if (!b || nsteps < 0 || !ms) return MOIST_ERR_ARG;
    if (cudaSetDevice(b->device) != cudaSuccess) return MOIST_ERR_CUDA;
    return b->impl->time_steps(nsteps, ms);
}

int moist_batch_profile(moist_batch* b, int nsteps, float* total_ms, float* group_ms) {
    if (!b || nsteps < 1 || !total_ms || !group_ms) return MOIST_ERR_ARG;
    if (cudaSetDevice(b->device) != cudaSuccess) return MOIST_ERR_CUDA;
    return b->impl->profile(nsteps, total_ms, group_ms);
}

const char* moist_batch_last_error(const moist_batch* b) { return b ? b->err.c_str() : "null batch"; }
int moist_batch_nan_member(const moist_batch* b) { return b ? b->nan_member : -1; }

int moist_nan_field(const moist_ctx* c) { return c ? c->nan_field : -1; }

// the context's device is made current for the calling thread at every entry point
#define CTX_DEVICE(c)                                                   \
    do {                                                                \
        if (cudaSetDevice((c)->device) != cudaSuccess) return MOIST_ERR_CUDA; \
    } while (0)

int moist_set_device(int device) {
    return cudaSetDevice(device) == cudaSuccess ? MOIST_OK : MOIST_ERR_CUDA;
}

int moist_upload_state(moist_ctx* c, const moist_state_host* s) {
    if (!c || !s) return MOIST_ERR_ARG;
    CTX_DEVICE(c);
    return c->impl->upload(s);
}
int moist_download_state(moist_ctx* c, moist_state_host* s) {
    if (!c || !s) return MOIST_ERR_ARG;
    CTX_DEVICE(c);
    return c->impl->download(s);
}
int moist_rk3_step(moist_ctx* c, int nsteps) {
    if (!c || nsteps < 0) return MOIST_ERR_ARG;
    CTX_DEVICE(c);
    return c->impl->rk3(nsteps);
}
int moist_compute_step(moist_ctx* c, const void* const phys[6], const moist_state_host* s0, double dt, int ns) {
    if (!c || !phys || !s0) return MOIST_ERR_ARG;
    CTX_DEVICE(c);
    return c->impl->compute_step(phys, s0, dt, ns);
}
int moist_cloud_microphysics(moist_ctx* c) {
    if (!c) return MOIST_ERR_ARG;
    CTX_DEVICE(c);
    return c->impl->microphysics();
}
int moist_rain_sedimentation(moist_ctx* c, void* d_prec) {
    if (!c) return MOIST_ERR_ARG;
    CTX_DEVICE(c);
    return c->impl->sedimentation(d_prec);
}
int moist_surface_fluxes(moist_ctx* c) {
    if (!c) return MOIST_ERR_ARG;
    CTX_DEVICE(c);
    return c->impl->surface_fluxes();
}
int moist_gray_radiation(moist_ctx* c) {
    if (!c) return MOIST_ERR_ARG;
    CTX_DEVICE(c);
    return c->impl->gray_radiation();
}
int moist_budget(moist_ctx* c, double out[4]) {
    if (!c || !out) return MOIST_ERR_ARG;
    CTX_DEVICE(c);
    return c->impl->budget(out);
}
int moist_adjoint_run(moist_ctx* c, int nsteps, int ckpt_every, const moist_adjoint_seed* seed,
                      moist_adjoint_grad* out) {
    if (!c) return MOIST_ERR_ARG;
    CTX_DEVICE(c);
    return c->impl->adjoint_run(nsteps, ckpt_every, seed, out);
}
void* moist_stream(moist_ctx* c) { return c ? (void*)c->stream : nullptr; }
int moist_synchronize(moist_ctx* c) {
    if (!c) return MOIST_ERR_ARG;
    return cudaStreamSynchronize(c->stream) == cudaSuccess ? MOIST_OK : MOIST_ERR_CUDA;
}
int moist_time_steps(moist_ctx* c, int nsteps, float* ms) {
    if (!c || !ms || nsteps < 0) return MOIST_ERR_ARG;
    CTX_DEVICE(c);
    return c->impl->time_steps(nsteps, ms);
}

int moist_rk3_step_host(moist_ctx* c, moist_state_host* s, int nsteps) {
    if (!c || !s || nsteps < 0) return MOIST_ERR_ARG;
    CTX_DEVICE(c);
    return c->impl->rk3_host(s, nsteps);
}

int moist_tracer_pass_counts(moist_ctx* c, int* counts, int n) {
    if (!c || !counts || n < 0) return MOIST_ERR_ARG;
    CTX_DEVICE(c);
    return c->impl->pass_counts(counts, n);
}

int moist_tracer_pass_trace(moist_ctx* c, int nsteps, int maxrec, long long* pass_ns, int* pass_tiles,
                            int* npasses) {
    if (!c || nsteps < 1 || maxrec < 0) return MOIST_ERR_ARG;
    CTX_DEVICE(c);
    return c->impl->pass_trace(nsteps, maxrec, pass_ns, pass_tiles, npasses);
}

int moist_set_adjoint_tapes(moist_ctx* c, int mode) {
    if (!c || mode < -1 || mode > 1) return MOIST_ERR_ARG;
    return c->impl->set_tape_mode(mode);
}

int moist_batch_set_adjoint_tapes(moist_batch* b, int mode) {
    if (!b || mode < -1 || mode > 1) return MOIST_ERR_ARG;
    return b->impl->set_tape_mode(mode);
}

int moist_set_wait_limit(moist_ctx* c, long long cycles) {
    if (!c) return MOIST_ERR_ARG;
    CTX_DEVICE(c);
    return c->impl->set_wait_limit(cycles);
}

int moist_step_profile(moist_ctx* c, int nsteps, float* total_ms, float* group_ms, long long* group_launches) {
    if (!c || nsteps < 0) return MOIST_ERR_ARG;
    CTX_DEVICE(c);
    return c->impl->profile(nsteps, total_ms, group_ms, group_launches);
}

int moist_implicit_correction(const moist_params* p, int precision, int flags, void* rho_w, const void* drho_w,
                              const void* theta, const void* rt2pres, double dt) {
    if (!p || !p->dz || !p->z || p->nz < 2 || !rho_w || !drho_w || !theta || !rt2pres) return MOIST_ERR_ARG;
    if (precision == MOIST_F64) return implicit_t<double, double>(p, rho_w, drho_w, theta, rt2pres, dt);
    if (flags & MOIST_FLAG_TRI_NATIVE) return implicit_t<float, float>(p, rho_w, drho_w, theta, rt2pres, dt);
    return implicit_t<float, double>(p, rho_w, drho_w, theta, rt2pres, dt);
}

int moist_eval_helper(const moist_params* p, int precision, int helper, int n, const double* in, double* out) {
    if (!p || n < 0 || (n > 0 && (!in || !out))) return MOIST_ERR_ARG;
    return precision == MOIST_F64 ? eval_helper_t<double>(p, helper, n, in, out)
                                  : eval_helper_t<float>(p, helper, n, in, out);
}

}  // extern "C"
