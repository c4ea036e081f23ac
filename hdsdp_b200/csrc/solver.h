// Internal structures of the B200 HDSDP solver.
//
// The host side holds the interior-point control flow and all m-vectors
// (y, dy, Schur right-hand sides); n x n and m x m matrices live on the GPU.
// Every cone / KKT operation mirrors one hook of the reference's conic
// callback interface (interface/def_hdsdp_conic.h:56-104) and KKT manager
// (interface/hdsdp_schur.h:10-21) with the same buffer semantics:
// BUFFER_DUALVAR (S and its factor), BUFFER_DUALCHECK (trial S and its
// factor), BUFFER_DUALSTEP (dS).
#pragma once
#include <vector>
#include <string>
#include <cuda_runtime.h>
#include "la.h"
#include "sdp.h"
#include "sparse_chol.h"
#include "../../include/hdsdp.h"
#include "../../include/hdsdp_user_data.h"

struct hdsdp_user_data {
    cone_type cone;
    int nConicRow;
    int nConicCol;
    int *coneMatBeg;
    int *coneMatIdx;
    double *coneMatElem;
};

namespace hb {

enum { BUFFER_DUALVAR = 0, BUFFER_DUALCHECK = 1, BUFFER_DUALSTEP = 2 };
enum { KKT_TYPE_INFEASIBLE = 0, KKT_TYPE_CORRECTOR = 1, KKT_TYPE_HOMOGENEOUS = 2, KKT_TYPE_PRIMAL = 3 };
enum { REF_ZERO = 0, REF_SPARSE = 1, REF_DENSE = 2, REF_SPR1 = 3, REF_DSR1 = 4 };
enum { ABS_NORM = 1, FRO_NORM = 2 };

// Per-solve timing split (seconds, device-synchronised at each phase edge).
struct Timers {
    double schur = 0, schur_factor = 0, schur_solve = 0, s_factor = 0, s_inverse = 0, lanczos = 0,
           assemble = 0, primal = 0, total = 0;
    long n_schur = 0, n_sfactor = 0, n_lanczos = 0, n_lanczos_mv = 0, n_schur_solve = 0;
    // finer split (seconds)
    double lz_inverse = 0, lz_host = 0, lz_wait = 0, sch_matrix = 0, sch_inner = 0, sch_innersq = 0;
    // presolve + upload (host wall) and the device-timed iterations + final check (CUDA events)
    double setup = 0, ipm_device = 0;
};

// Lanczos maximum-step estimator (linalg/hdsdp_lanczos.c:161-292) on the GPU.
constexpr int kLanczosMaxBlocks = 1024;   // grid bound of the fused Lanczos steps
struct Lanczos {
    int n = 0, maxdim = 30;
    long ld = 0;
    cudaStream_t s = nullptr;
    double *V = nullptr, *w = nullptr, *z1 = nullptr, *z2 = nullptr, *t1 = nullptr, *u = nullptr, *warm = nullptr;
    double *d_ab = nullptr;   // alpha[0..maxdim), beta[maxdim..2*maxdim+1)
    double *h_ab = nullptr;   // pinned
    double *d_y = nullptr;    // 2 * (maxdim + 1)
    double *d_scal = nullptr, *h_scal = nullptr;
    double *init_vec = nullptr, *pert_vec = nullptr;  // device, deterministic per n
    double *part = nullptr;   // per-block partial sums of the fused steps (2 x kLanczosMaxBlocks)
    // pinned Ritz coefficients, and the device addresses of the pinned h_ab, h_scal and h_yv
    // (null where the memory is not mapped), for the batched small-block runs
    double *h_yv = nullptr;
    double *dm_ab = nullptr, *dm_scal = nullptr, *dm_yv = nullptr;
    int nComputed = 0;
    // when set, the operator is built from this sparse factor of S instead of F
    HybridFactor *hyOp = nullptr;
    void init(int n_, cudaStream_t s_);
    void release();
    // Max alpha with  I + alpha * K (-D) K^T  psd, where K = L^-1 of the factor.
    hdsdp_retcode solve(DenseFactor &F, const double *D, long ldD, double *maxStep, Timers *tm);
};

// One cone's small-block Lanczos bound (order <= 96, dense factor) for lanczos_small_batch:
// the operator I + alpha K (-D) K^T of its factor F and step matrix D, the bound into
// *maxStep, the outcome in ret.
struct LzTask {
    Lanczos *lz;
    DenseFactor *F;
    const double *D;
    long ldD;
    double *maxStep;
    Timers *tm;
    hdsdp_retcode ret;
};
// The bounds of several tasks (one stream), the launches shared; each task's result is
// the one Lanczos::solve gives.
void lanczos_small_batch(std::vector<LzTask> &tasks);
constexpr int kSmallLanczosMaxN = 96;

// Inputs that produced a dual-slack buffer (dC*C + dAs*sum y_i A_i + dEye*I); a
// factorisation of a buffer rebuilt from identical inputs is reused, which gives
// bit-identical results because the factor kernels are deterministic.
struct SlackSig {
    bool valid = false;
    double dC = 0, dAs = 0, dEye = 0;
    std::vector<double> y;
    bool same(const SlackSig &o) const {
        return valid && o.valid && dC == o.dC && dAs == o.dAs && dEye == o.dEye && y == o.y;
    }
};

// SDP cone on the device (interface/hdsdp_conic_sdp.c). A dense cone holds every
// constraint of the problem; a sparse cone (at most 30% of the constraints have a
// coefficient in the block, interface/hdsdp_user_data.c:73-86) holds only those,
// listed in `rows`, and works on that subset: m is then the number of rows it holds,
// its m-vectors are gathered from and scattered into the problem's by `rows`.
struct SdpCone {
    int n = 0, m = 0;
    int mAll = 0;                // constraints of the problem
    bool sparse = false;
    std::vector<int> rows;       // sparse cone: problem row of each local row (increasing)
    int *d_rows = nullptr;       // device copy of rows
    std::vector<double> ybuf;    // gathered coefficient vector
    long ld = 0;
    cudaStream_t s = nullptr;
    SdpDevice dev;
    HostCoeff C;
    std::vector<HostCoeff> A;
    std::vector<int> refType;    // reference coefficient type per row after presolve
    int refTypeC = REF_ZERO;
    int stats[5] = {0, 0, 0, 0, 0};
    double *Svar = nullptr, *Scheck = nullptr, *dS = nullptr, *W = nullptr;
    DenseFactor Fvar, Fcheck;
    SlackSig sigVar, sigCheck;   // inputs of the current Svar / Scheck contents
    SlackSig facVar, facCheck;   // inputs of the matrices factored in Fvar / Fcheck
    bool facVarOk = false, facCheckOk = false;
    long nFactorReuse = 0;
    // The factor of the slack at the point of the last Schur build (the accepted iterate) is
    // set aside (Fkeep) when a trial point's factorisation is about to overwrite Fvar, and handed
    // back when that point is factored again, as after a line search that found no better point.
    // Dense factors only (no sparse slack factorisation on the cone).
    DenseFactor Fkeep;
    SlackSig facKeep;
    bool facKeepOk = false;
    bool pinVar = false;
    void keep_var();       // before a factorisation into Fvar
    bool restore_var();    // the kept factor is that of Svar's inputs: back into Fvar
    // Factor the buffer `which` (Svar into Fvar, Scheck into Fcheck), reusing a
    // factor of the same inputs held by either factor object.
    bool factor_buffer(int which);
    void invalidate_check_factor() { facCheck.valid = false; }
    // Sparse dual pattern: positive-definiteness checks and log det go through the
    // hybrid sparse factorisation; Fvar / Fcheck then hold no dense factor of their
    // buffer (hyVar / hyCheck) until ensure_dense() forms it for a consumer of L.
    // -1 trial points only (BUFFER_DUALCHECK; the accepted point's S^-1 feeds the Schur
    // build, which needs the dense factor), 0 off, 1 both buffers
    int sparseMode = -1;
    HybridFactor *hy = nullptr;
    bool hyVar = false, hyCheck = false;
    double hyLogdetVar = 0.0, hyLogdetCheck = 0.0;
    long hySeqVar = -1, hySeqCheck = -1;  // the sparse factorisation each buffer's result came from
    long nHybrid = 0, nHybridCheck = 0, nDenseAfter[2] = {0, 0};
    bool use_hybrid(int which) const {
        return hy && (sparseMode == 1 || which != BUFFER_DUALVAR);
    }
    bool hybrid_factor(int which);
    bool ensure_dense(int which);
    enum { FP_DONE = 0, FP_SMALL = 1, FP_ASYNC = 2 };
    int factor_plan(int which, bool *ok);
    bool factor_finish(int which, bool synced = false);
    // the step S += step * dS of add_step_and_check, without the factorisation
    void add_step(double step, int which);
    // ratio_test takes the small-block Lanczos path (order 2 .. kSmallLanczosMaxN, no
    // sparse factor), which several cones can share (lanczos_small_batch)
    bool small_lanczos() const { return n > 1 && n <= kSmallLanczosMaxN && !hy; }
    Lanczos lz;
    double dualResidual = 0.0, dualPerturb = 0.0;
    double *d_y = nullptr;       // device copy of the current coefficient vector
    double *d_vec = nullptr;     // device m scratch
    double *h_vec = nullptr;     // pinned m scratch
    double *d_vec2 = nullptr, *h_vec2 = nullptr;   // second pair (batched Schur builds)
    double *Mown = nullptr;      // the cone's own Schur-block scratch (batched Schur builds)
    double *d_scal = nullptr, *h_scal = nullptr;
    double objScal = 1.0;
    Timers *tm = nullptr;
    int precision = 0;

    hdsdp_retcode proc_data(int nRow, int nCol, const int *Ap, const int *Ai, const double *Ax,
                            bool sparseCone = false);
    hdsdp_retcode presolve();
    // problem m-vector -> the cone's rows (the input itself for a dense cone)
    const double *local(const double *v);
    hdsdp_retcode setup_device(cudaStream_t stream, Timers *t);
    void release();

    double obj_norm(int type) const;
    double coeff_norm(int type) const;
    void scal(double a);
    void detect_feature(const double *rowRHS, int intF[20], double dblF[20]) const;

    void update_buffer(double dC, double dAs, const double *y, double dEye, int which);
    bool buffer_plan(double dC, double dAs, const double *y, double &dEye, int which, double **target,
                     const double **ly);
    void set_start(double r) { dualResidual = r; }
    void reduce_resi(double r) { dualResidual = r; }
    void set_perturb(double p) { dualPerturb = p; }
    hdsdp_retcode update(double tau, const double *y);
    hdsdp_retcode ratio_test(double dtau, const double *dy, double ada, int which, double *step);
    hdsdp_retcode interior_check(double tau, const double *y, int *interior);
    hdsdp_retcode interior_check_expert(double dC, double dAs, const double *y, double dEye, int which, int *interior);
    hdsdp_retcode get_barrier(double tau, const double *y, int which, double *logdet);
    hdsdp_retcode add_step_and_check(double step, int which, int *interior);
    void get_primal(double mu, const double *y, const double *dy, double *X);   // device X (ld)
    void get_dual(double *S);                                                  // device S (ld)
    void atimesx(const double *X, double *out);                                // host out (problem m), accumulated
    double trace_cx(const double *X);
};

// update_buffer(dC, dAs, y, dEye[q], which) of several cones (all on one stream): y in problem
// order, uploaded once into d_yall (mAll doubles, pinned staging h_yall); small cones whose
// coefficients all sit in the gather map assembled in shared launches
void assemble_buffers(const std::vector<SdpCone *> &cones, double dC, double dAs, const double *y,
                      const std::vector<double> &dEye, int which, double *d_yall, double *h_yall);

// factor_buffer(which) of several cones (all on one stream), small dense factorisations
// batched: ok[q] = positive definite
void factor_buffers(const std::vector<SdpCone *> &cones, int which, std::vector<char> &ok);

// Scalar dual box l <= y <= u (interface/hdsdp_conic_bound.c), host-side O(m).
struct BoundCone {
    int m = 0;
    double lo = -1e7, up = 1e7;
    std::vector<double> dl, du, dlInv, duInv, dlStep, duStep, dlChk, duChk;
    void proc(int m_, double l, double u);
    void update_buffer(double dC, double dAs, const double *y, int which);
    void update(double tau, const double *y) { update_buffer(tau, -1.0, y, BUFFER_DUALVAR); }
    double ratio_test(double dtau, const double *dy, int which);
    int interior_check(double tau, const double *y);
    int interior_check_expert(double dC, double dAs, const double *y, int which);
    hdsdp_retcode get_barrier(double tau, const double *y, int which, double *logdet);
    int add_step_and_check(double step, int which);
    void get_primal(double mu, const double *y, const double *dy, double *lower, double *upper) const;
};

// LP cone s = c - A^T y - r >= 0 (interface/hdsdp_conic_lp.c), host-side O(nnz)
// except its Schur block, added on the device. A is stored by constraint: column i
// (0 .. m-1) lists the LP columns k with A_ki, in the user's order.
struct LpCone {
    int m = 0, nCol = 0;
    std::vector<double> obj;                  // c
    std::vector<int> beg, idx;
    std::vector<double> val;
    std::vector<double> s, sChk, sStep, sInv, buf;
    double dualResidual = 0.0, dualPerturb = 0.0;
    // Schur block: the lower pairs (i >= j) of constraints that share an LP column, and
    // the per-build values added to M there
    std::vector<int> pairI, pairJ;
    std::vector<double> pairVal;
    int *d_pi = nullptr, *d_pj = nullptr;
    double *d_pv = nullptr;
    cudaStream_t st = nullptr;

    hdsdp_retcode proc_data(int nRow, int nCol_, const int *Ap, const int *Ai, const double *Ax, cudaStream_t stream);
    void release();
    double obj_norm(int type) const;
    double coeff_norm(int type) const;
    void scal(double a);
    void detect_feature(int intF[20], double dblF[20]) const;
    void update_buffer(double dC, double dAs, const double *y, double dEye, int which);
    void set_start(double r) { dualResidual = r; }
    void reduce_resi(double r) { dualResidual = r; }
    void set_perturb(double p) { dualPerturb = p; }
    void update(double tau, const double *y) { update_buffer(tau, -1.0, y, -dualResidual, BUFFER_DUALVAR); }
    double ratio_test(double dtau, const double *dy, double ada, int which);
    int interior_check(double tau, const double *y);
    int interior_check_expert(double dC, double dAs, const double *y, double dEye, int which);
    double get_barrier(double tau, const double *y, int which);
    int add_step_and_check(double step, int which);
    void get_primal(double mu, const double *y, const double *dy, double *x);   // host x (nCol)
    void get_dual(double *out) const;                                         // host (nCol)
    void atimesx(const double *x, double *out) const;                         // out (m) accumulated
    double trace_cx(const double *x) const;
};

// Up to this order the Schur solves use K = L^-1 (formed inside the factorisation); above
// it they are triangular solves with L, which read L once instead of forming K.
constexpr int kTriSolveMinM = 6000;

struct ArrowSchur;
// Whether the block-arrow Schur complement is used for these sparse SDP cones (the whole
// problem; mode -1 automatic, 0 never, 1 always).
bool arrow_chosen(int mode, int m, const std::vector<SdpCone *> &cones);

// Schur complement system (interface/hdsdp_schur.c).
struct KKT {
    int m = 0;
    long ldm = 0;
    cudaStream_t s = nullptr;
    double *M = nullptr;          // device m x m
    DenseFactor F;
    std::vector<double> asinv, asinvrd, asinvcs;
    double dCSinv = 0, dCSinvCSinv = 0, dCSinvRdSinv = 0, dTraceSinv = 0;
    double *d_rhs = nullptr, *d_x = nullptr, *d_r = nullptr, *d_t = nullptr, *d_diag = nullptr;
    double *h_buf = nullptr;
    std::vector<double> diag_add;     // bound-cone diagonal accumulated before factorisation
    double shift = 0.0;               // diagonal shift applied if the Cholesky of M failed
    // LDL^T (Bunch-Kaufman) factor of M: taken when the Cholesky fails even with the shift
    // retries (ldlMode 0) or for every factorisation (ldlMode 1); ldlActive while the current
    // factor is this one
    LdlFactor ldl;
    int ldlMode = 0;
    bool ldlActive = false;
    const double *primalX = nullptr;  // device X for KKT_TYPE_PRIMAL
    Timers *tm = nullptr;
    // M holds a partial sum of the current build (false after clean: the first dense SDP
    // cone writes M outright, any other contribution zeroes it first)
    bool mOpen = false;
    double *Msub = nullptr;           // Schur block of a cone added into M (sparse or not first)
    size_t msubCap = 0;
    // descriptors of the batched Schur builds (add_sdp_batch): the grouped W = K^T K and the
    // per-cone build jobs
    GemmDesc *d_wdesc = nullptr;
    SchurBuildJob *d_jobs = nullptr;
    size_t fusedCap = 0;
    // dense M and F are allocated unless denseM is false (the block-arrow form is used)
    void init(int m_, cudaStream_t stream, Timers *t, bool denseM = true);
    void release();
    // Block-arrow sparse Schur complement (arrow.cu) for problems whose cones are all sparse
    // SDP cones: M kept as per-cone local blocks, their coupling rows and a coupling block.
    // Engaged by setup_arrow after init(..., false); the methods below then route to it.
    ArrowSchur *arrow = nullptr;
    bool setup_arrow(const std::vector<SdpCone *> &cones);
    void release_arrow();
    void arrow_open();
    void arrow_add(const SdpCone &cone, const double *Msub, long ldsub);
    void arrow_add_diag(const double *h_diag);
    void arrow_regularize(double reg);
    bool arrow_factorize();
    bool arrow_solve(const double *rhs, double *lhs);
    // {engaged, coupling rows, cones, largest local block, device bytes of the block arrow,
    // device bytes the dense M and its factor take}
    void arrow_info(double out[6]) const;
    void clean(int type);
    void open_m();
    hdsdp_retcode add_sdp(SdpCone &cone, int type);
    // add_sdp for several SDP cones (types KKT_TYPE_INFEASIBLE and KKT_TYPE_CORRECTOR), one
    // wait for all
    hdsdp_retcode add_sdp_batch(const std::vector<SdpCone *> &cones, int type);
    hdsdp_retcode build(SdpCone &cone, int type) {  // a build with this single cone
        clean(type);
        return add_sdp(cone, type);
    }
    void add_lp(LpCone &lp, int type);
    void add_bound(BoundCone &b, int type);
    void regularize(double reg);
    hdsdp_retcode factorize();
    hdsdp_retcode solve(const double *rhs, double *lhs);   // host vectors; lhs may alias rhs
};

struct AdjointState;
void adjoint_release(AdjointState *&a);

// Per-iteration record for time-to-gap reporting.
struct IterRecord {
    double t, pobj, dobj, mu, gap;
    int phase;
};

}  // namespace hb

namespace hb {
// One cone of the problem in the user's order (interface/hdsdp.c:571-578): an SDP
// block (dense or sparse cone) or an LP cone.
struct ConeSlot {
    user_data *usr = nullptr;
    cone_type type = HDSDP_CONETYPE_UNKNOWN;
    SdpCone *sdp = nullptr;
    LpCone *lp = nullptr;
};
}  // namespace hb

struct hdsdp_solver_internal {
    int nRows = 0;
    int nCones = 0;
    std::vector<double> rowRHS;
    std::vector<hb::ConeSlot> cones;
    hb::SdpCone *cone = nullptr;   // the first SDP cone (the only one for primal refinement and the adjoint)
    hb::BoundCone bnd;
    hb::KKT kkt;
    cudaStream_t stream = nullptr;
    hb::Timers timers;

    std::vector<double> y, dy, d1, d2, d3, d4, aux1, aux2, pInfUp, pInfLow;
    std::vector<double> accY, accDy, inaccY, inaccDy;
    double tau = 1.0, dtau = 0.0;
    double dTraceSinv = 0.0;
    int whichMethod = 0;
    int nIterCount = 0;
    int nSmallStep = 0;
    double mu = 1e10, proxNorm = 0, potentialVal = 0, barrierVal = 0, dStep = 0, resi = 0, perturb = 0;
    double allConeDims = 0;
    double pObjVal = 0, dObjVal = 0, pObjInternal = 0, dObjInternal = 0, dObjImprove = 0;
    double pInfeas = 0, dInfeas = 0, comp = HDSDP_INFINITY;
    double accMu = -1.0, inaccMu = -1.0;
    double timeBegin = 0;
    hdsdp_status HStatus = HDSDP_UNKNOWN;
    int HIntParams[20] = {0};
    double HDblParams[20] = {0};
    int HIntFeatures[20] = {0};
    double HDblFeatures[20] = {0};
    double dErrs[6] = {0};
    bool optimized = false;
    int precision = 0;
    int sparseSlack = -1;          // factorisation of S in PSD checks: -1 trial points sparse (automatic), 0 dense, 1 sparse
    int sparseSchur = -1;          // Schur complement form: -1 automatic, 0 dense, 1 block arrow when every cone is a sparse SDP cone
    int schurLdl = 0;              // Schur factorisation: 0 Cholesky (LDL^T when it fails), 1 LDL^T
    int verbose = 0;
    std::vector<hb::IterRecord> log;
    std::string modelFeatures;
    hb::AdjointState *adj = nullptr;  // cached adjoint factors of the last solve
    double *d_yall = nullptr, *h_yall = nullptr;   // y of the batched cone updates (device, pinned)
};
