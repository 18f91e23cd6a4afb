// adjoint_batch.cuh - the adjoint of an ensemble as packed launches: one launch per kernel of
// the reverse step (and of the taped forward step it recomputes) for all members.
//
// Every adjoint kernel of adjoint.cuh is a device body with explicit block coordinates; a
// member context records, instead of launching, the argument struct of each launch, and the
// batch concatenates the members' structs and builds (member, block) work lists as for the
// forward step (batch.cuh). The members' arithmetic is that of their own moist_adjoint_run.
#pragma once

#include "adjoint.cuh"
#include "batch.cuh"

namespace moist {

// launch kinds of the adjoint, numbered after the forward step's
enum AdjBatchKind {
    BK_ZERO = BK_NKINDS,  // zero n doubles
    BK_COPY,              // copy up to 8 fields
    AK_TRI_COEF,
    AK_TRI_FACT,
    AK_UPDATE,
    AK_TR_JAC,
    AK_TR_REV,
    AK_TR_SCATTER,
    AK_MF,
    AK_SUB_VERT,
    AK_SUB_SOLVE,
    AK_SUB_RHS,
    AK_SUB_EXPL,
    AK_SUB_HORIZ,
    AK_P0,
    AK_TRI_COEF_T,
    AK_TEND_T,
    AK_FACE_T,
    AK_DIAG_T,
    AK_KESSLER,
    AK_SED,
    AK_STEP_END,
    AK_NKINDS
};

// zero and copy launches: blocks of 256 threads, nblk = ceil(fsz / BZ_CHUNK) blocks per member
// striding over the member's n elements
constexpr int BZ_CHUNK = 2048;
__host__ __device__ inline unsigned bz_blocks(size_t fsz) { return (unsigned)((fsz + BZ_CHUNK - 1) / BZ_CHUNK); }

struct BZero {
    double* ptr;
    size_t n;
    unsigned nblk;
};
template <class T>
struct BCopy {
    CopyList<T> l;
    size_t n;
    unsigned nblk;
};
template <class T>
struct AStage {
    DevParams<double> p;
    AdjStage<T> a;
};
template <class T>
struct AStageLP {
    DevParams<double> p;
    AdjStage<T> a;
    DP<4> LP;
};
template <class T>
struct ATrJac {
    DevParams<double> p;
    AdjStage<T> a;
    double* J;
};
template <class T>
struct ATrScatter {
    DevParams<double> p;
    AdjStage<T> a;
    const double* J;
    DP<3> mu;
};
struct ATriFact {
    int nx, nz, P;
    const double *Ta, *Tb, *Tc;
    double *Tcp, *Trd;
};
struct ATrRev {
    int nx, nz, P;
    const double* J;
    DP<3> lam, mu;
};
struct ASolve {
    int nx, nz, P;
    const double *Tc, *Tcp, *Trd, *Lx;
    double* Ly;
};
template <class T>
struct ASub {
    DevParams<double> p;
    DevParams<T> pt;
    AdjStage<T> a;
    AdjSub<T> b;
};
template <class T>
struct APhys {
    DevParams<double> p;
    AdjPhys<T> a;
};
struct AStepEnd {
    int nx, nz, P;
    DP<7> L7, S7;
    DP<5> L5;
};

struct FZero {
    __device__ void operator()(const BZero& x, int bx, int) const {
        const size_t stride = (size_t)x.nblk * blockDim.x;
        for (size_t j = (size_t)bx * blockDim.x + threadIdx.x; j < x.n; j += stride) x.ptr[j] = 0.0;
    }
};
template <class T>
struct FCopy {
    __device__ void operator()(const BCopy<T>& x, int bx, int) const {
        const size_t stride = (size_t)x.nblk * blockDim.x;
        for (int f = 0; f < x.l.nf; f++) {
            const T* __restrict__ s = x.l.src[f];
            T* __restrict__ d = x.l.dst[f];
            for (size_t j = (size_t)bx * blockDim.x + threadIdx.x; j < x.n; j += stride) d[j] = s[j];
        }
    }
};

// cell kernels: block (bx, by) = (x block of 128 cells, row); the two tracer-sweep kernels
// take by = row + nz * tracer
template <class T>
struct FATriCoef {
    __device__ void operator()(const AStage<T>& x, int bx, int by) const { b_adj_tri_coef(x.p, x.a, bx, by, 0); }
};
struct FATriFact {
    __device__ void operator()(const ATriFact& x, int bx, int) const {
        b_adj_tri_fact(x.nx, x.nz, x.P, x.Ta, x.Tb, x.Tc, x.Tcp, x.Trd, bx, 0, 0);
    }
};
template <class T>
struct FAUpdate {
    __device__ void operator()(const AStageLP<T>& x, int bx, int by) const { b_adj_update(x.p, x.a, x.LP, bx, by, 0); }
};
template <class T>
struct FATrJac {
    __device__ void operator()(const ATrJac<T>& x, int bx, int by) const {
        b_adj_tr_jac(x.p, x.a, x.J, bx, by % x.p.nz, by / x.p.nz);
    }
};
struct FATrRev {
    __device__ void operator()(const ATrRev& x, int bx, int) const {
        b_adj_tr_rev(x.nx, x.nz, x.P, x.J, x.lam, x.mu, bx, 0, 0);
    }
};
template <class T>
struct FATrScatter {
    __device__ void operator()(const ATrScatter<T>& x, int bx, int by) const {
        b_adj_tr_scatter(x.p, x.a, x.J, x.mu, bx, by % x.p.nz, by / x.p.nz);
    }
};
template <class T>
struct FAMf {
    __device__ void operator()(const AStage<T>& x, int bx, int by) const { b_adj_mf(x.p, x.a, bx, by, 0); }
};
template <class T>
struct FASubVert {
    __device__ void operator()(const ASub<T>& x, int bx, int by) const { b_adj_sub_vert(x.p, x.a, x.b, bx, by, 0); }
};
struct FASubSolve {
    __device__ void operator()(const ASolve& x, int bx, int) const {
        b_adj_sub_solve(x.nx, x.nz, x.P, x.Tc, x.Tcp, x.Trd, x.Lx, x.Ly, bx, 0, 0);
    }
};
template <class T>
struct FASubRhs {
    __device__ void operator()(const ASub<T>& x, int bx, int by) const {
        b_adj_sub_rhs(x.p, x.pt, x.a, x.b, bx, by, 0);
    }
};
template <class T>
struct FASubExpl {
    __device__ void operator()(const ASub<T>& x, int bx, int by) const { b_adj_sub_expl(x.p, x.a, x.b, bx, by, 0); }
};
template <class T>
struct FASubHoriz {
    __device__ void operator()(const ASub<T>& x, int bx, int by) const { b_adj_sub_horiz(x.p, x.a, x.b, bx, by, 0); }
};
template <class T>
struct FAP0 {
    __device__ void operator()(const AStageLP<T>& x, int bx, int by) const { b_adj_p0(x.p, x.a, x.LP, bx, by, 0); }
};
template <class T>
struct FATriCoefT {
    __device__ void operator()(const AStage<T>& x, int bx, int by) const { b_adj_tri_coef_T(x.p, x.a, bx, by, 0); }
};
template <class T>
struct FATendT {
    __device__ void operator()(const AStage<T>& x, int bx, int by) const { b_adj_tend_T(x.p, x.a, bx, by, 0); }
};
template <class T>
struct FAFaceT {
    __device__ void operator()(const AStage<T>& x, int bx, int by) const { b_adj_face_T(x.p, x.a, bx, by, 0); }
};
template <class T>
struct FADiagT {
    __device__ void operator()(const AStage<T>& x, int bx, int by) const { b_adj_diag_T(x.p, x.a, bx, by, 0); }
};
template <class T>
struct FAKessler {
    __device__ void operator()(const APhys<T>& x, int bx, int by) const { b_adj_kessler(x.p, x.a, bx, by, 0); }
};
template <class T>
struct FASed {
    __device__ void operator()(const APhys<T>& x, int bx, int by) const { b_adj_sed(x.p, x.a, bx, by, 0); }
};
struct FAStepEnd {
    __device__ void operator()(const AStepEnd& x, int bx, int by) const {
        b_adj_step_end(x.nx, x.nz, x.P, x.L7, x.S7, x.L5, bx, by, 0);
    }
};

}  // namespace moist
