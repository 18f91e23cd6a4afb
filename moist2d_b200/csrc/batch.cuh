// batch.cuh - ensembles of independent domains advanced together: one launch per kernel of the
// large step for all members, from a packed work list.
//
// Every kernel of the step is a device body with explicit block coordinates (kernels.cuh,
// tracer_stream.cuh). A member context records, instead of launching, the argument struct of
// each launch of one step (a "slot"); the batch concatenates the members' structs of a slot
// into one device array and builds a work list of (member, block) items, so that one launch of
// k_batched runs that kernel for every member, each block reading its member's arguments. The
// tracer transport uses the row-streaming sweep, whose blocks are independent (the tiled sweep
// needs all of one domain's tiles resident at once).
#pragma once

#include "tracer_stream.cuh"

namespace moist {

// launch kinds of the large step
enum BatchKind {
    BK_MEMSET = 0,
    BK_SF,
    BK_RD,
    BK_PHYS,
    BK_DIAG,
    BK_TEND,
    BK_THOMAS,
    BK_SUB,
    BK_PREP,
    BK_STREAM,
    BK_UPD,
    BK_STAGE_END,
    BK_PREC,
    BK_NKINDS
};

struct BItem {
    int m, bx, by;  // member, block coordinates within the member's grid
};

// argument structs, one per member and launch
struct BMemset {
    void* ptr;
    size_t bytes;
};
template <class T>
struct BSf {
    DevParams<T> p;
    StateP<T> s;
    const T *ru_left, *rho_right;
    T *d_u_sf, *d_th_sf, *d_qv_sf, *mflux, *shflux, *lhflux;
    const int* err;
};
template <class T>
struct BRd {
    DevParams<T> p;
    StateP<T> s;
    const T* theta_ref;
    T *lw_up, *lw_dn, *d_th_rd;
    const int* err;
};
template <class T>
struct BPhys {
    DevParams<T> p;
    StateP<T> s;
    T *d_th_mp, *d_qv_mp, *d_qc_mp, *d_qr_mp, *d_qr_sed, *d_prec;
    const T *d_th_rd, *d_u_sf, *d_th_sf, *d_qv_sf;
    PhysP<T> ph;
    const int* err;
};
template <class T>
struct BDiag {
    DevParams<T> p;
    StateP<T> s;
    T *pres, *theta, *rt2pres, *u_face, *w_face;
    const int* err;
};
template <class T>
struct BTend {
    DevParams<T> p;
    TendArgs<T> a;
    const int* err;
};
template <class T, class TT>
struct BThomas {
    DevParams<T> p;
    const T *theta, *rt2pres;
    T dt_s;
    int wc;
    T *ta, *tb, *tc;
    TT *tcp, *tpiv;
    const int* err;
};
template <class T, class TT>
struct BSub {
    DevParams<T> p;
    SubArgs<T, TT> a;
    T dt_s, ns_T;
    double fact_tp64;
    int wc;
    const int* err;
};
template <class T>
struct BPrep {
    DevParams<T> p;
    TracerArgs<T> tr;
    T *s0, *s1, *s2;
    double* rrho;
    const int* err;
};
template <class T>
struct BStream {
    DevParams<T> p;
    StreamArgs<T> a;
    const int* err;
};
template <class T>
struct BUpd {
    DevParams<T> p;
    UpdArgs<T> a;
    int* err;
};
struct BStageEnd {
    int* err;
};
template <class T>
struct BPrec {
    DevParams<T> p;
    T* prec;
    const T* d_prec;
    const int* err;
};

// the bodies behind each kind
struct FMemset {
    __device__ void operator()(const BMemset& a, int, int) const {
        unsigned char* d = (unsigned char*)a.ptr;
        for (size_t j = threadIdx.x; j < a.bytes; j += blockDim.x) d[j] = 0;
    }
};
template <class T>
struct FSf {
    __device__ void operator()(const BSf<T>& a, int bx, int by) const {
        b_surface_fluxes(a.p, a.s, a.ru_left, a.rho_right, a.d_u_sf, a.d_th_sf, a.d_qv_sf, a.mflux, a.shflux,
                         a.lhflux, a.err, bx, by);
    }
};
template <class T>
struct FRd {
    __device__ void operator()(const BRd<T>& a, int bx, int by) const {
        b_gray_radiation(a.p, a.s, a.theta_ref, a.lw_up, a.lw_dn, a.d_th_rd, a.err, bx, by);
    }
};
template <class T>
struct FPhys {
    __device__ void operator()(const BPhys<T>& a, int bx, int by) const {
        b_physics(a.p, a.s, a.d_th_mp, a.d_qv_mp, a.d_qc_mp, a.d_qr_mp, a.d_qr_sed, a.d_prec, a.d_th_rd, a.d_u_sf,
                  a.d_th_sf, a.d_qv_sf, a.ph, a.err, bx, by);
    }
};
template <class T>
struct FDiag {
    __device__ void operator()(const BDiag<T>& a, int bx, int by) const {
        b_diag(a.p, a.s, a.pres, a.theta, a.rt2pres, a.u_face, a.w_face, a.err, bx, by);
    }
};
template <class T>
struct FTend {
    __device__ void operator()(const BTend<T>& a, int bx, int by) const { b_tend(a.p, a.a, a.err, bx, by); }
};
// The factorisation and the acoustic substep run one thread per column in the batch: the
// ensemble's columns give every SM enough warps to overlap their recurrences, which the column
// strips of a single domain have to stage through shared memory instead (same values).
template <class T, class TT>
struct FThomas {
    __device__ void operator()(const BThomas<T, TT>& a, int bx, int) const {
        b_thomas_col<T, TT>(a.p, a.theta, a.rt2pres, a.dt_s, a.ta, a.tb, a.tc, a.tcp, a.tpiv, a.err, bx);
    }
};
template <class T, class TT>
struct FSub {
    __device__ void operator()(const BSub<T, TT>& a, int bx, int) const {
        b_substep_col<T, TT>(a.p, a.a, a.dt_s, a.ns_T, a.fact_tp64, a.err, bx);
    }
};
template <class T, class TT>
struct FSubPf {
    __device__ void operator()(const BSub<T, TT>& a, int bx, int) const {
        b_substep_col_pf<T, TT>(a.p, a.a, a.dt_s, a.ns_T, a.fact_tp64, a.err, bx);
    }
};
template <class T, class TT, int NBUF>
struct FSubAsync {
    __device__ void operator()(const BSub<T, TT>& a, int bx, int) const {
        b_substep_col_async<T, TT, NBUF>(a.p, a.a, a.dt_s, a.ns_T, a.fact_tp64, a.err, bx);
    }
};
// the same two kernels over column strips (for ensembles too small to fill the GPU with columns)
template <class T, class TT>
struct FThomasStrip {
    __device__ void operator()(const BThomas<T, TT>& a, int bx, int by) const {
        b_thomas_strip<T, TT>(a.p, a.theta, a.rt2pres, a.dt_s, a.wc, a.ta, a.tb, a.tc, a.tcp, a.tpiv, a.err, bx, by);
    }
};
template <class T, class TT>
struct FSubStrip {
    __device__ void operator()(const BSub<T, TT>& a, int bx, int by) const {
        b_substep_strip<T, TT>(a.p, a.a, a.dt_s, a.ns_T, a.fact_tp64, a.wc, a.err, bx, by);
    }
};
constexpr int BATCH_COL_THREADS = 64;
template <class T>
struct FPrep {
    __device__ void operator()(const BPrep<T>& a, int bx, int by) const {
        b_stream_prep(a.p, a.tr, a.s0, a.s1, a.s2, a.rrho, a.err, bx, by);
    }
};
template <class T>
struct FStream {
    __device__ void operator()(const BStream<T>& a, int bx, int) const { b_tracer_stream(a.p, a.a, a.err, bx); }
};
template <class T>
struct FUpd {
    __device__ void operator()(const BUpd<T>& a, int bx, int by) const { b_update(a.p, a.a, a.err, bx, by); }
};
struct FStageEnd {
    __device__ void operator()(const BStageEnd& a, int, int) const {
        if (threadIdx.x == 0 && a.err[1] != INT_MAX && a.err[0] == INT_MAX) a.err[0] = a.err[1];
    }
};
template <class T>
struct FPrec {
    __device__ void operator()(const BPrec<T>& a, int bx, int by) const {
        b_prec(a.p, a.prec, a.d_prec, a.err, bx, by);
    }
};

// one launch for all members: block b runs item b with its member's arguments. MINB bounds
// the registers so that MINB blocks of 256 threads fit on an SM.
template <class A, class F, int MINB = 1>
__global__ void __launch_bounds__(256, MINB) k_batched(const BItem* __restrict__ items, const A* __restrict__ args,
                                                        F f) {
    const BItem it = items[blockIdx.x];
    f(args[it.m], it.bx, it.by);
}

// the same with a block of at most MAXT threads, MINB of them per SM
template <class A, class F, int MAXT, int MINB>
__global__ void __launch_bounds__(MAXT, MINB) k_batched_b(const BItem* __restrict__ items,
                                                           const A* __restrict__ args, F f) {
    const BItem it = items[blockIdx.x];
    f(args[it.m], it.bx, it.by);
}

// the members' error words gathered into one array: out[m][4]
__global__ void k_gather_err(int* const* errs, int n, int* out) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= n) return;
    for (int j = 0; j < 4; j++) out[4 * m + j] = errs[m][j];
}
__global__ void k_reset_err(int* const* errs, int n) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= n) return;
    errs[m][0] = INT_MAX;
    errs[m][1] = INT_MAX;
    errs[m][2] = 0;
    errs[m][3] = 0;
}

}  // namespace moist
