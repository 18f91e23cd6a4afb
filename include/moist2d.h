/*
 * moist2d.h - C-ABI of libmoist2d_sm100a.so, the B200 (sm_100a) implementation of
 * moist2d's large time step.
 *
 * The entry points replace the Julia methods of moist.jl (seiya/moist2d):
 *   rk3_step!(s::State, p::Params{T})               moist.jl:1589-1683  -> moist_rk3_step
 *   compute_step!(d_phys x6, s, s0, p, dt, ns)       moist.jl:1039-1580  -> moist_compute_step
 *   cloud_microphysics!(...)                         moist.jl:554-671    -> moist_cloud_microphysics
 *   rain_sedimentation!(...)                         moist.jl:674-707    -> moist_rain_sedimentation
 *   implicit_correction!(rho_w, drho_w, theta, rt2pres, dt, p)
 *                                                    moist.jl:974-1030   -> moist_implicit_correction
 *   device(x)  (the CuArray hook)                    moist.jl:227-228    -> moist_ctx_create + moist_upload_state
 *   output_history(...) field computation            moist.jl:1795-1843  -> moist_history_diagnostics
 * A Julia caller binds them with ccall; Python binds them with ctypes (moist2d_b200/_lib.py).
 *
 * Conventions
 *  - Every call returns an int status (MOIST_OK = 0). Errors the reference raises as Julia
 *    exceptions (error("NaN detected in rho"), moist.jl:1543-1577) become MOIST_ERR_NAN, with
 *    the field index from moist_nan_field() and the text from moist_last_error().
 *  - Precision is chosen per context (MOIST_F32 / MOIST_F64), the counterpart of Params{T}
 *    and the global FT (moist.jl:22-24). Every host array passed to a context holds elements
 *    of that type.
 *  - Host state arrays use the reference layout: 2-D fields are Julia column-major (ka, ia)
 *    arrays, z (k) fastest, ka = nz, ia = nx + 2*halo, with `halo` periodic columns on each
 *    side (moist.jl:82-88, 319-345). 1-D x fields have length ia, theta_ref has length ka.
 *  - Device buffers belong to the context. One context = one CUDA stream. Calls on one
 *    context are not thread-safe; different contexts may be driven from different threads.
 *    Calls return after the work they queued has finished, unless stated otherwise.
 */
#ifndef MOIST2D_H
#define MOIST2D_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MOIST2D_ABI_VERSION 1

/* precision of a context (Params{Float32} / Params{Float64}) */
enum { MOIST_F32 = 0, MOIST_F64 = 1 };

/* status codes */
enum {
    MOIST_OK = 0,
    MOIST_ERR_NAN = 1,          /* a NaN was found by the end-of-stage check (moist.jl:1542-1578) */
    MOIST_ERR_ARG = 2,          /* invalid argument (null pointer, nz < 2, nx < 2, ns < 1, ...) */
    MOIST_ERR_CUDA = 3,         /* a CUDA runtime call failed; text in moist_last_error */
    MOIST_ERR_TIMEOUT = 4,      /* a bounded device-side wait ran out */
    MOIST_ERR_UNSUPPORTED = 5,  /* valid in the reference but not provided by this library */
    MOIST_ERR_NOMEM = 6,        /* device allocation failed */
    MOIST_ERR_IO = 7            /* a history or restart file could not be written or read;
                                   text in moist_io_last_error */
};

/* field indices reported by moist_nan_field(), in the order compute_step! checks them */
enum {
    MOIST_FIELD_RHO = 0,
    MOIST_FIELD_RHO_U = 1,
    MOIST_FIELD_RHO_W = 2,
    MOIST_FIELD_RHO_THETA = 3,
    MOIST_FIELD_RHO_QV = 4,
    MOIST_FIELD_RHO_QC = 5,
    MOIST_FIELD_RHO_QR = 6,
    MOIST_FIELD_D_RHO_U_PHYS = 7,
    MOIST_FIELD_D_RHO_THETA_PHYS = 8,
    MOIST_FIELD_D_RHO_QV_PHYS = 9,
    MOIST_FIELD_D_RHO_QC_PHYS = 10,
    MOIST_FIELD_D_RHO_QR_PHYS = 11
};

/* context creation flags */
enum {
    /* In a MOIST_F32 context the w-p tridiagonal elimination runs in FP64 by default; this flag
     * selects the reference's literal Float32 elimination (moist.jl:952-971) instead. */
    MOIST_FLAG_TRI_NATIVE = 1,
    /* Run the tracer transport as one exact wavefront per tracer instead of the tiled sweep
     * (same results bit for bit, much slower; kept for cross-checking). */
    MOIST_FLAG_TRACER_WAVEFRONT = 2,
    /* Run the tracer transport as one exact row-streaming wavefront per tracer (one thread per
     * row; no repair passes; same results bit for bit). Needs nz <= 256. */
    MOIST_FLAG_TRACER_STREAM = 4,
    /* Run the tiled tracer sweep without grid-wide passes: each tile publishes numbered versions
     * of its boundary strips and recomputes as soon as its left or lower neighbour publishes a
     * new one (same results bit for bit). */
    MOIST_FLAG_TRACER_DATAFLOW = 8
};

/*
 * Params{T} (moist.jl:70-222) plus the global physical constants of set_constants!
 * (moist.jl:26-60). Scalars are passed as double and converted to the context precision
 * (exact for values that are already of type T, which is how the Julia and Python mirrors
 * fill them). The grid vectors are arrays of the context type T, length nz, as produced by
 * the Params constructor (moist.jl:198-216); they are copied at context creation.
 */
typedef struct moist_params {
    /* grid */
    int32_t nx, nz, halo;      /* Nx, Nz, halo; ia = nx + 2*halo, ka = nz */
    int32_t ns;                /* acoustic substeps of the last RK stage (Params.ns) */
    double lx, h, dx;          /* Lx, H, dx */
    const void* zf;            /* face heights zf[k]   (T, nz) */
    const void* dz;            /* layer depths dz[k]   (T, nz) */
    const void* z;             /* centre heights z[k]  (T, nz) */
    double dt;                 /* large time step */
    /* dynamics */
    double nu, kappa, gamma_d, beta_offcenter, zf_sponge;
    /* process switches (moist.jl:107-120) */
    int32_t do_mp, do_auto, do_accr, do_revap, do_sed, do_rd, do_sf;
    /* surface-flux and radiation coefficients (moist.jl:121-135) */
    double cd, ch, ce, uabs_min, temp_surf;
    double k_abs_qv, k_abs_qc, k_abs_qr, surf_emissivity, tau_cooling, z_tropopause;
    /* physical constants (moist.jl:30-59) */
    double grav, rd, rv, cpd, cpv, cpl, cvd, p0, lv, sigma, epsvap;
    double k_auto, qc_threshold, k_accr, k_evap, a_term, b_term;
    double t0, es0, a_sat, b_sat, eps;
} moist_params;

/*
 * Host view of State (moist.jl:294-317). Every pointer may be NULL, which means "skip this
 * field" on upload and download. Element type = context precision.
 */
typedef struct moist_state_host {
    void* rho;            /* (ka, ia) */
    void* rho_u;          /* (ka, ia)  at (k, i+1/2) */
    void* rho_w;          /* (ka, ia)  at (k+1/2, i); rho_w[ke] is the rigid lid */
    void* rho_theta;      /* (ka, ia) */
    void* rho_qv;         /* (ka, ia) */
    void* rho_qc;         /* (ka, ia) */
    void* rho_qr;         /* (ka, ia) */
    void* prec;           /* (ia) accumulated precipitation */
    void* mflux;          /* (ia) */
    void* shflux;         /* (ia) */
    void* lhflux;         /* (ia) */
    void* theta_ref;      /* (ka) */
    void* d_rho_theta_mp; /* (ka, ia) */
    void* d_rho_qv_mp;    /* (ka, ia) */
    void* d_rho_qc_mp;    /* (ka, ia) */
    void* d_rho_qr_mp;    /* (ka, ia) */
    void* d_rho_qr_sed;   /* (ka, ia) */
    void* d_rho_u_sf;     /* (ia) */
    void* d_rho_theta_sf; /* (ia) */
    void* d_rho_qv_sf;    /* (ia) */
    void* d_rho_theta_rd; /* (ka, ia) */
} moist_state_host;

typedef struct moist_ctx moist_ctx;

/* library identification */
int moist_abi_version(void);
const char* moist_status_string(int status);

/* Select the CUDA device on which this host thread creates contexts (cudaSetDevice in the
 * library's runtime; the default is device 0). A context remembers its device and makes it
 * current at each of its entry points. */
int moist_set_device(int device);

/* Context = one device-resident State plus Params (replaces device(), moist.jl:227-228).
 * Fails with MOIST_ERR_ARG for nx < 1, nz < 2 (or > 1024), halo < 0, ns < 1 or a NULL grid
 * vector. The RK-stage entry points (rk3_step, compute_step, time_steps) further need
 * halo = 2 and nx >= 2, the shapes on which the reference's stencils stay inside the array. */
int moist_ctx_create(const moist_params* p, int precision, int flags, moist_ctx** out);
int moist_ctx_destroy(moist_ctx* ctx);
const char* moist_last_error(const moist_ctx* ctx);
int moist_nan_field(const moist_ctx* ctx);

/* Copy a host State into the context (reference layout, halos included in the host arrays).
 * The library keeps interior columns; halo columns are re-derived periodically, as every
 * reference code path on the large step does before reading them. Host arrays in page-locked,
 * mapped memory (cudaHostAlloc, cudaHostRegister) are read in place by the layout kernels, the
 * seven prognostic fields in one launch; pageable arrays go through a staging copy. */
int moist_upload_state(moist_ctx* ctx, const moist_state_host* s);
/* Copy the context State to host arrays; halo columns are written as periodic copies (the
 * phys tendencies keep the caller's halo columns). Page-locked, mapped host arrays are written
 * in place, as moist_upload_state reads them. */
int moist_download_state(moist_ctx* ctx, moist_state_host* s);

/* rk3_step!(s, p) applied nsteps times (moist.jl:1589-1683). */
int moist_rk3_step(moist_ctx* ctx, int nsteps);

/* rk3_step!(s, p) on a host State, the reference's calling convention (moist.jl:1589): copy s
 * to the device, apply nsteps large steps, copy the State back into s. Equivalent to
 * moist_upload_state + moist_rk3_step + moist_download_state with one synchronisation. Host
 * arrays in page-locked memory are read and written in place by the layout kernels over the
 * bus, without staging copies. */
int moist_rk3_step_host(moist_ctx* ctx, moist_state_host* s, int nsteps);

/* compute_step!(d_rho_phys, d_rho_u_phys, d_rho_theta_phys, d_rho_qv_phys, d_rho_qc_phys,
 * d_rho_qr_phys, s, s0, p, dt, ns) (moist.jl:1039-1580): one RK stage on the context state s,
 * with s0 given as a host State (its rho, rho_u, rho_w, rho_theta, rho_qv, rho_qc, rho_qr are
 * read) and the six tendency fields given as host (ka, ia) arrays in that order. */
int moist_compute_step(moist_ctx* ctx, const void* const phys[6], const moist_state_host* s0,
                       double dt, int ns);

/* cloud_microphysics!(...) (moist.jl:554-671) on the context state: fills d_rho_{theta,qv,qc,qr}_mp
 * (download them with moist_download_state). */
int moist_cloud_microphysics(moist_ctx* ctx);

/* rain_sedimentation!(d_rho_qr_sed, d_prec, rho_qr, rho, p) (moist.jl:674-707): fills
 * d_rho_qr_sed in the context and, if d_prec is not NULL, the host array d_prec (ia, type T). */
int moist_rain_sedimentation(moist_ctx* ctx, void* d_prec);

/* surface_fluxes!(d_rho_u_sf, d_rho_theta_sf, d_rho_qv_sf, mflux, shflux, lhflux, rho, rho_u,
 * rho_theta, rho_qv, rho_qc, rho_qr, p) (moist.jl:710-752) on the context state: fills
 * d_rho_{u,theta,qv}_sf, mflux, shflux and lhflux (download them with moist_download_state).
 * Its reads of rho_u[ks, is-1] and rho[ks, ie+1] see the halo columns of the last upload (or
 * of the last RK stage's exchange). Needs halo >= 1. */
int moist_surface_fluxes(moist_ctx* ctx);

/* gray_radiation!(d_rho_theta_rd, rho, rho_theta, rho_qv, rho_qc, rho_qr, theta_ref, p)
 * (moist.jl:776-840) on the context state with its uploaded theta_ref: fills d_rho_theta_rd. */
int moist_gray_radiation(moist_ctx* ctx);

/* implicit_correction!(rho_w, drho_w, theta, rt2pres, dt, p) (moist.jl:974-1030) for one
 * column on the device: host arrays of length nz and type T; rho_w is updated in place.
 * Only p->nz, p->dz, p->z, p->grav and p->beta_offcenter are read. */
int moist_implicit_correction(const moist_params* p, int precision, int flags, void* rho_w,
                              const void* drho_w, const void* theta, const void* rt2pres,
                              double dt);

/* Allocation-free variant of moist_implicit_correction. It has no counterpart in the
 * reference; it is for callers that must not have a library allocate device memory behind
 * them: a host whose device memory all comes from its own pool (Julia's CUDA.jl, which
 * reclaims pool memory under pressure), a host that reserves a fixed device-memory budget up
 * front and cannot meet an out-of-memory failure mid-run, and a host that keeps other streams
 * busy and cannot afford cudaFree, which waits for the whole device.
 * Solves implicit_correction! for ncols columns at once. rho_w (updated in place), drho_w,
 * theta and rt2pres are DEVICE arrays of type T laid out (nz, ncols) with z fastest (column j
 * starts at element j*nz); p->dz, p->z (host) give the grid and travel in the kernel's
 * parameter block; p->grav and p->beta_offcenter are read. The work is queued on `stream` (a
 * cudaStream_t, NULL = default stream) and the call returns without waiting; it issues no
 * memory copy. It calls no cudaMalloc or cudaFree: its scratch is one fixed array of
 * MOIST_NOALLOC_SCRATCH_BYTES per device, held by every GPU that loads the library until exit.
 * Limits: nz <= MOIST_NOALLOC_MAX_NZ, and 2*(nz-1)*ncols*sizeof(elimination type) <=
 * MOIST_NOALLOC_SCRATCH_BYTES (e.g. 2048 columns of 128 levels with the FP64 elimination);
 * larger calls return MOIST_ERR_ARG before queuing anything and write the reason to err (if not
 * NULL). The first call on a device looks up the scratch array's device address with that
 * device current and keeps it for the life of the process, so make no call after a
 * cudaDeviceReset of the device. All calls share the array and keep the last call's contents;
 * nothing in it needs to start at zero (every element is written before it is read). Calls that
 * overlap on the same GPU (for example on two streams) race on it, so serialise them. */
#define MOIST_NOALLOC_MAX_NZ 1024
#define MOIST_NOALLOC_SCRATCH_BYTES (4 * 1024 * 1024)
int moist_implicit_correction_noalloc(const moist_params* p, int precision, int flags, int ncols,
                                      void* rho_w, const void* drho_w, const void* theta,
                                      const void* rt2pres, double dt, void* stream, char* err,
                                      size_t errlen);

/* Device evaluation of the scalar helpers, for the restated unit tests (runtests.jl:25-80,
 * 377-401): out[j] = helper(in[j*nin ...]) for j < n, computed by the same device functions
 * the kernels use. Values are passed as double and rounded to the precision first. */
enum {
    MOIST_HELPER_F2H = 0,          /* in: vf1, vf2, dz1, dz2          out: 1 (moist.jl:243-251) */
    MOIST_HELPER_KOREN = 1,        /* in: r                           out: 1 (moist.jl:844-847) */
    MOIST_HELPER_SAT_VP = 2,       /* in: T                           out: es, des/dT (253-260) */
    MOIST_HELPER_SAT_Q = 3,        /* in: p, es                       out: qsat, dqsat/des (263-273) */
    MOIST_HELPER_EXP = 4,          /* in: x                           out: exp(x) */
    MOIST_HELPER_POW = 5           /* in: x, y                        out: x^y */
};
int moist_eval_helper(const moist_params* p, int precision, int helper, int n, const double* in,
                      double* out);

/* Domain budgets (compensated FP64 sums on the device, deterministic order):
 * out[0] = mass  sum(rho*dz*dx), out[1] = water sum((rho_qv+rho_qc+rho_qr)*dz*dx) + sum(prec*dx),
 * out[2] = total energy (kinetic + potential + internal, the terms of moist.jl:1839-1852)*dx*dz,
 * out[3] = accumulated surface rain sum(prec*dx). */
int moist_budget(moist_ctx* ctx, double out[4]);

/* ---- Ensembles (no counterpart in the reference, which advances one domain per process).
 * A batch advances nmembers independent domains together: members[i] are the members'
 * parameters (each its own nx, nz, grid, dt and physics switches; ns, do_sf and do_rd must
 * agree; halo = 2, nx >= 2, nz <= 256). Each large step is one launch per kernel of the step
 * for all members, from a packed (member, block) work list, captured once as a CUDA graph; the
 * tracer transport runs as the row-streaming wavefront (MOIST_FLAG_TRACER_STREAM). Every
 * member's results equal those of a context stepping that member alone, bit for bit.
 * flags: MOIST_FLAG_TRI_NATIVE as for moist_ctx_create. */
typedef struct moist_batch moist_batch;
int moist_batch_create(const moist_params* members, int nmembers, int precision, int flags, moist_batch** out);
int moist_batch_destroy(moist_batch* b);
/* the member's own context: upload, download, budget and the other per-context calls apply
 * to it (its moist_rk3_step advances that member alone) */
moist_ctx* moist_batch_member(moist_batch* b, int member);
int moist_batch_upload(moist_batch* b, int member, const moist_state_host* s);
int moist_batch_download(moist_batch* b, int member, moist_state_host* s);
/* nsteps large steps of every member; a NaN in a member stops that member's work (the others
 * continue) and returns MOIST_ERR_NAN, with the member in moist_batch_nan_member and the field
 * in moist_nan_field(moist_batch_member(b, m)) */
int moist_batch_step(moist_batch* b, int nsteps);
/* nsteps large steps timed with CUDA events on the batch stream (no error check) */
int moist_batch_time_steps(moist_batch* b, int nsteps, float* ms);
/* nsteps large steps launched without the graphs, with CUDA events around every packed launch:
 * total device time and its split over the MOIST_KGROUP_* groups (group_ms[MOIST_NGROUPS]) */
int moist_batch_profile(moist_batch* b, int nsteps, float* total_ms, float* group_ms);
const char* moist_batch_last_error(const moist_batch* b);
int moist_batch_nan_member(const moist_batch* b);

/* ---- Adjoint (no counterpart in the reference, which has no derivatives; a Julia caller
 * exposes it as the pullback of a ChainRulesCore.rrule around rk3_step!).
 *
 * moist_adjoint_run advances the context State nsteps large steps (as moist_rk3_step does, the
 * context is left at the final State) and returns the gradient of the objective
 *   J = sum_i prec_weight[i] * prec_final[i] + sum_f sum_(k,i) state[f](k,i) * S_final_f(k,i)
 * with respect to the initial State's seven prognostic fields, the initial prec and the Kessler
 * parameters K_auto and Qc_threshold. The gradient is the discrete adjoint of the computed step:
 * the reverse sweep goes step by step from the last step, each step recomputed from its input
 * State (kept every ckpt_every steps and recomputed in between) with its stage internals
 * taped, and adjoint variables in double whatever the context precision. Branch points
 * (upwind and limiter switches, Kessler clamps) contribute the derivative of the branch taken.
 * Needs do_sf = do_rd = 0 (MOIST_ERR_UNSUPPORTED otherwise). Device memory: about
 * (nsteps / ckpt_every + ckpt_every) States plus 3*ns + 40 fields of one step. */
typedef struct moist_adjoint_seed {
    const double* prec_weight; /* (ia) d J / d prec_final, or NULL */
    const double* state[7];    /* (ka, ia) d J / d S_final of rho, rho_u, rho_w, rho_theta,
                                  rho_qv, rho_qc, rho_qr, or NULL */
} moist_adjoint_seed;
typedef struct moist_adjoint_grad {
    double* state[7];          /* (ka, ia) d J / d S_initial (halo columns 0), or NULL to skip */
    double* prec;              /* (ia) d J / d prec_initial, or NULL */
    double k_auto;             /* d J / d K_auto */
    double qc_threshold;       /* d J / d Qc_threshold */
    double objective;          /* J */
    double forward_ms;         /* wall time of the forward run */
    double reverse_ms;         /* wall time of the reverse sweep (recomputation included) */
} moist_adjoint_grad;
int moist_adjoint_run(moist_ctx* ctx, int nsteps, int ckpt_every, const moist_adjoint_seed* seed,
                      moist_adjoint_grad* out);

/* moist_adjoint_run for every member of a batch (no counterpart in the reference): seeds[m] and
 * out[m] belong to member m (seeds may be NULL: J = 0). nthreads <= 0: the members' kernels run
 * packed, one launch per kernel of the forward step, of the recomputed (taped) step and of the
 * reverse step for all members (the forward through the batch's step graphs); every member gets
 * the gradient of its own moist_adjoint_run (atomic sums may round in another order).
 * forward_ms and reverse_ms are the batch's. nthreads > 0: every member's own
 * moist_adjoint_run from up to nthreads host threads, each on its member context's stream.
 * Each member is left at its final State; the next moist_batch_step continues from there. The
 * first failing member's status is returned, its index in moist_batch_last_error. */
int moist_batch_adjoint_run(moist_batch* b, int nsteps, int ckpt_every, const moist_adjoint_seed* seeds,
                            moist_adjoint_grad* out, int nthreads);

/* Tape mode of moist_adjoint_run (no counterpart in the reference). The reverse sweep
 * recomputes each segment of ckpt_every steps from its checkpoint. mode 1: a tape of every step
 * of the segment, the segment recomputed once; mode 0: the segment's States and one tape, every
 * step recomputed from its State (one more forward step per step, ckpt_every - 1 States instead
 * of ckpt_every tapes of 3*ns + 40 fields); mode -1 (the default): mode 1 when the tapes fit in
 * half the free device memory. The gradients do not depend on the mode. */
int moist_set_adjoint_tapes(moist_ctx* ctx, int mode);
/* The same for moist_batch_adjoint_run: every member runs in one mode (-1: decided from the
 * members' tapes together). */
int moist_batch_set_adjoint_tapes(moist_batch* b, int mode);

/* output_history's primitive variables (moist.jl:1795-1835) computed on the device from the
 * context State, so that a run_sim-style driver reads only what it writes to its history file:
 * out[f] (f = MOIST_DIAG_*, NULL to skip) receives field f as a host (Nz, Nx) array of the
 * context precision, z fastest, interior only (output_history's arrays before the transpose
 * of its writes; moist_history_append puts them in the file's x-fastest order); summary (if not NULL)
 * receives the run log's min w, max w (m/s), max qc, max qr (g/kg), min RH, max RH (%)
 * (moist.jl:1838-1843). The energy sums of the log come from moist_budget. */
enum {
    MOIST_DIAG_U = 0,       /* u at cell centres, (rho_u[i] + rho_u[i-1]) / 2 / rho */
    MOIST_DIAG_W = 1,       /* w at cell centres */
    MOIST_DIAG_THETA = 2,
    MOIST_DIAG_QV = 3,
    MOIST_DIAG_QC = 4,
    MOIST_DIAG_QR = 5,
    MOIST_DIAG_PRES = 6,
    MOIST_DIAG_TEMP = 7,
    MOIST_DIAG_THETAE = 8,  /* equivalent potential temperature */
    MOIST_DIAG_RH = 9,      /* relative humidity (%) */
    MOIST_NDIAG = 10
};
int moist_history_diagnostics(moist_ctx* ctx, void* const out[MOIST_NDIAG], double summary[6]);

/* History and restart files: init_history / output_history (moist.jl:1686-1891) and the
 * restart read of run_sim (moist.jl:1905-1919). The reference writes through NCDatasets; this
 * library writes the NetCDF classic format with 64-bit offsets (CDF-2) itself, which every
 * NetCDF reader opens: dimensions x (Nx), z (Nz) and the unlimited time; the variables of
 * init_history in its order (x, z, zf, time, rho, rhou, rhow, u, w, theta, qv, qc, qr, RH,
 * temp, pres, thetae, prec, mflux, shflux, lhflux, d_rho_theta_mp, d_rho_qv_mp, d_rho_qc_mp,
 * d_rho_qr_mp, d_rho_qr_sed, d_rho_u_sf, d_rho_theta_sf, d_rho_qv_sf, d_rho_theta_rd), each of
 * the context precision with its "units" attribute; a Julia (x, z, time) variable is
 * (time, z, x) in the file. Failures return MOIST_ERR_IO with the reason in
 * moist_io_last_error (per host thread). */
typedef struct moist_history moist_history;
const char* moist_io_last_error(void);
/* init_history (moist.jl:1716-1793): creates (replaces) path and writes the header and x, z,
 * zf. precision: MOIST_F32 or MOIST_F64. */
int moist_history_create(const char* path, const moist_params* p, int precision, moist_history** out);
/* output_history (moist.jl:1795-1889): appends one record at time t from the context's State,
 * with the diagnostics computed on the device (moist_history_diagnostics); pres in hPa. For
 * member m of an ensemble pass moist_batch_member(b, m) (moist_batch_step returns with the
 * batch's work finished, so the member context holds its current State). */
int moist_history_append(moist_history* h, double t, moist_ctx* ctx);
/* The same record from host arrays: s in the reference layout (NULL fields are written as 0),
 * diag[f] as moist_history_diagnostics returns them. Needs no device. */
int moist_history_append_host(moist_history* h, double t, const moist_state_host* s,
                              const void* const diag[MOIST_NDIAG]);
int moist_history_close(moist_history* h);
/* The restart of run_sim (moist.jl:1905-1919): from the last record of a history file, fills
 * the interior of s->rho, rho_u, rho_w (as stored), rho_theta, rho_qv, rho_qc, rho_qr (theta,
 * qv, qc, qr times rho in the file's type, then rounded to the context precision) and prec,
 * and the halo columns of the seven prognostic fields periodically (exchange_halo!). NULL
 * fields are skipped. rho_qr is read from "qr" (the reference reads "qc" there,
 * moist.jl:1917). Needs no device. */
int moist_restart_read(const char* path, const moist_params* p, int precision, moist_state_host* s);

/* ---- Seeded initial States (host only: no device is needed). The reference builds its State
 * with init_state! (moist.jl:351-450), whose theta noise comes from per-thread Xoshiro streams
 * (moist.jl:374-375) and so depends on the thread schedule. These generators draw from the
 * counter-based Philox4x32-10 generator keyed by (seed, stream), so a State depends on the seed
 * alone, and build the base columns in the model's discrete hydrostatic balance (the iteration of
 * moist.jl:413-431), in double precision, rounded once to the State precision. They fill the
 * seven prognostic fields (halo columns periodic), theta_ref, and zero the rest of the State
 * (NULL fields are skipped). The Python mirror is moist2d_b200/init.py (the same algorithms in
 * numpy; states agree to the last bits of double-precision exp/pow). */
typedef struct moist_bubble {
    double xc, zc;   /* centre (m); the x distance is periodic in moist_init_sounding */
    double radius;   /* m */
    double amp;      /* theta perturbation (K) at the centre, cos^2 shape */
} moist_bubble;
/* the fields of Params{T} that init_state! reads (moist.jl:136-148) */
typedef struct moist_init_profile {
    double theta0, bndlayer_depth, z_tropopause, dtheta_dz_trop, dtheta_dz_stra, theta_pert;
    double rel_hum_surf, rel_hum_decay, u0;
} moist_init_profile;
/* out[j] = uniform (0, 1) double of index idx[j] (or j when idx is NULL) in stream
 * (seed, stream): Philox4x32-10 of the counter (idx low, idx high, stream, 0) and the key
 * (seed, 0x6D6F6973), first word + 1/2 over 2^32 */
int moist_uniform(uint32_t seed, uint32_t stream, int64_t n, const uint64_t* idx, double* out);
/* init_state!(s, p, rngs) (moist.jl:351-450) with the noise of stream 0, index i*nz + k */
int moist_init_state(const moist_params* p, int precision, const moist_init_profile* profile, uint32_t seed,
                     moist_state_host* s);
/* warm moist bubble: theta = 300 K neutral, surface pressure 1000 hPa, RH 20 % outside and 95 %
 * inside a cos^2 bubble of 2 K, radius 2 km, centred at x = 10 km * nx / 200, z = 2 km, uniform
 * +-0.01 K theta noise (stream 0, index i*nz + k), u = 0 */
int moist_init_warm_bubble(const moist_params* p, int precision, uint32_t seed, moist_state_host* s);
/* analytic sounding: theta = 300 + 43 (z/12 km)^1.25 K below 12 km, isothermal above; RH =
 * 1 - 0.75 (z/12 km)^1.25, 0.25 above; u = 12 tanh(z / 3 km) m/s; plus the given warm bubbles
 * applied at constant pressure */
int moist_init_sounding(const moist_params* p, int precision, const moist_bubble* bubbles, int nbubbles,
                        moist_state_host* s);
/* the seeded bubble row of the sounding workload: bubble j at x = (j + 1/2) lx / n, z = zc,
 * amplitude and radius uniform in the ranges (stream 1, indices 2j and 2j + 1) */
int moist_sounding_bubble_row(uint32_t seed, int nbubbles, double lx, double amp_lo, double amp_hi,
                              double rad_lo, double rad_hi, double zc, moist_bubble* out);
/* member `member` of the uneven ensemble: nx and nz drawn from the choices, one bubble at a
 * seeded x in (0, nx*dx), z = zc, amplitude and radius uniform in the ranges (stream
 * 1000 + member, indices 0..4) */
int moist_ensemble_member_draw(uint32_t seed, int member, const int* nx_choices, int n_nx, const int* nz_choices,
                               int n_nz, double dx, double amp_lo, double amp_hi, double rad_lo, double rad_hi,
                               double zc, int* nx, int* nz, moist_bubble* bubble);

/* ---- Autotuner (no counterpart in the reference). moist_autotune times nsteps large steps of
 * the context for every strip width of the factorisation and acoustic-substep kernels (1, 2, 4
 * or 8 columns per block) and every exact tracer sweep the context can run (tiled; streaming
 * when nz <= 256), each from the same saved State, keeps the fastest for the context's later
 * steps and restores the State: results are the same bit for bit whatever it picks.
 * moist_batch_autotune does the same for a batch over the threads per block (32, 64, 128,
 * 256) of its per-column kernels and rebuilds the batch's step graphs. report (if not NULL)
 * receives the timings and the choice. */
int moist_autotune(moist_ctx* ctx, int nsteps, char* report, size_t report_len);
int moist_batch_autotune(moist_batch* b, int nsteps, char* report, size_t report_len);

/* Kernel groups of one large step, for moist_step_profile. */
enum {
    MOIST_KGROUP_PHYSICS = 0,   /* surface fluxes, radiation, Kessler + sedimentation + phys assembly */
    MOIST_KGROUP_PROLOGUE = 1,  /* per stage: diagnostics, slow tendencies, w-p factorisation */
    MOIST_KGROUP_SUBSTEP = 2,   /* per acoustic substep */
    MOIST_KGROUP_TRACER = 3,    /* per stage: Koren tracer transport (Gauss-Seidel order) */
    MOIST_KGROUP_UPDATE = 4,    /* per stage: state update and NaN check */
    MOIST_KGROUP_OTHER = 5,     /* precipitation accumulation */
    MOIST_NGROUPS = 6
};
/* Run nsteps large steps with CUDA events recorded on the context stream wherever the kernel
 * group changes (consecutive launches of one group, such as the substeps of a stage, share one
 * interval): *total_ms = device time from the first to the last event, group_ms[g] = time
 * spent in group g, group_launches[g] = kernels launched in group g (arrays of MOIST_NGROUPS;
 * any pointer may be NULL). Every event between two kernels costs the stream a few
 * microseconds, so *total_ms is somewhat above the time moist_time_steps gives. */
int moist_step_profile(moist_ctx* ctx, int nsteps, float* total_ms, float* group_ms,
                       long long* group_launches);

/* Diagnostic of the tiled tracer sweep: counts[p] (p < n, p < 64) = sweeps since the last call
 * that reached their bitwise fixed point after p passes; the counters are reset.
 * MOIST_ERR_UNSUPPORTED when the context runs the wavefront sweep. */
int moist_tracer_pass_counts(moist_ctx* ctx, int* counts, int n);

/* Bound of the device-side waits of the context's kernels (no counterpart in the reference,
 * whose threads never wait on one another). The tiled tracer sweep's blocks wait for each
 * other between repair passes, or in its dataflow form (MOIST_FLAG_TRACER_DATAFLOW) for their
 * left and lower neighbours' new strips; every such wait gives up after `cycles` SM clock cycles
 * (cycles <= 0 restores the default, about two seconds), and the step then returns
 * MOIST_ERR_TIMEOUT, leaving the context's State undefined (upload a State before stepping
 * again). Meant for tests of that path. MOIST_ERR_UNSUPPORTED when the context's tracer sweep
 * does not wait (the streaming or wavefront sweep). */
int moist_set_wait_limit(moist_ctx* ctx, long long cycles);

/* Diagnostic of the tiled tracer sweep (no counterpart in the reference): runs nsteps large
 * steps (3 sweeps each) with every pass timed on the device. For sweep w (0 .. 3*nsteps-1):
 * npasses[w] = passes run; pass_ns[w*maxrec + q] = duration of pass q+1 in ns (from its start to
 * the next pass's start, the last one to the moment block 0 leaves the sweep);
 * pass_tiles[w*maxrec + q] = tile-tracer warps that recomputed in that pass (3 per tile at most).
 * In the dataflow form a "pass" is a tile's q-th computation: npasses is the largest count of
 * any tile, pass_tiles counts the tile-tracer warps that computed a q-th time, and pass_ns is the
 * difference between the latest starts of computations q+1 and q+2 (or the end). Any output
 * pointer may be NULL. Allocates its timing buffers per call. */
int moist_tracer_pass_trace(moist_ctx* ctx, int nsteps, int maxrec, long long* pass_ns, int* pass_tiles,
                            int* npasses);

/* Stream of the context (a cudaStream_t), for callers that order their own work after it. */
void* moist_stream(moist_ctx* ctx);
/* Block until the context stream is idle. */
int moist_synchronize(moist_ctx* ctx);
/* Run nsteps large steps, timed with CUDA events recorded on the context stream around them;
 * *ms receives the elapsed device time. */
int moist_time_steps(moist_ctx* ctx, int nsteps, float* ms);

#ifdef __cplusplus
}
#endif

#endif /* MOIST2D_H */
