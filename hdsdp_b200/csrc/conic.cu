// The conic callback interface and the KKT manager as a C ABI (include/hdsdp_conic.h).
//
// The reference drives its cones through a table of function pointers (the hdsdp_cone
// struct, interface/def_hdsdp_conic.h:56-104) filled by HConeSetData
// (interface/hdsdp_conic.c:50-188), and builds the Schur complement through HKKT*
// (interface/hdsdp_schur.c). This file gives the same table and the same dispatch over
// this library's cones: SdpCone (dense and sparse SDP blocks, matrices on the GPU),
// LpCone and BoundCone (host O(nnz) slacks), and KKT (M on the GPU). The solver in
// solver.cu calls those classes directly; this interface serves hosts that run their own
// iteration over the cones.
//
// Every cone and KKT object made here on a device shares one non-blocking CUDA stream of
// the library (one per device), so their device work is ordered as the host calls it.
// An SDP cone allocates its device buffers on its first numeric hook, after the host has
// had the chance to scale its objective (coneScal); a later coneScal re-uploads them.
#include "solver.h"
#include "../../include/hdsdp_conic.h"
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>

struct hdsdp_kkt_internal {
    hb::KKT kkt;
    hb::Timers tm;
    int nRow = 0;
    int nCones = 0;
    hdsdp_cone **cones = nullptr;
    bool ready = false;
};

namespace hb {
namespace {

cudaStream_t conic_stream() {
    static std::mutex mu;
    static cudaStream_t streams[kMaxDevices] = {nullptr};
    std::lock_guard<std::mutex> g(mu);
    cudaStream_t &s = streams[current_device()];
    if (!s) HB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    return s;
}

// The object behind hdsdp_cone::coneData.
struct ConeObj {
    cone_type type = HDSDP_CONETYPE_UNKNOWN;
    SdpCone *sdp = nullptr;
    LpCone *lp = nullptr;
    BoundCone *bnd = nullptr;
    Timers tm;
    bool deviceReady = false;
    double *dX = nullptr;      // device n x ld scratch for primal recovery and A X
};

ConeObj *obj(void *p) { return static_cast<ConeObj *>(p); }

// device buffers of an SDP cone, allocated at the first numeric hook
bool sdp_ready(ConeObj *c) {
    if (!c->sdp) return false;
    if (c->deviceReady) return true;
    if (c->sdp->setup_device(conic_stream(), &c->tm) != HDSDP_RETCODE_OK) return false;
    c->deviceReady = true;
    return true;
}

hdsdp_retcode create_of(void **pp, cone_type t) {
    if (!pp) return HDSDP_RETCODE_FAILED;
    ConeObj *c = new (std::nothrow) ConeObj();
    if (!c) return HDSDP_RETCODE_MEMORY;
    c->type = t;
    *pp = c;
    return HDSDP_RETCODE_OK;
}

// ---------------------------------------------------------------- SDP cones
hdsdp_retcode sdp_dense_create(void **pp) { return create_of(pp, HDSDP_CONETYPE_DENSE_SDP); }
hdsdp_retcode sdp_sparse_create(void **pp) { return create_of(pp, HDSDP_CONETYPE_SPARSE_SDP); }

hdsdp_retcode sdp_proc(void *p, int nRow, int nCol, int *Ap, int *Ai, double *Ax) {
    ConeObj *c = obj(p);
    c->sdp = new (std::nothrow) SdpCone();
    if (!c->sdp) return HDSDP_RETCODE_MEMORY;
    return c->sdp->proc_data(nRow, nCol, Ap, Ai, Ax, c->type == HDSDP_CONETYPE_SPARSE_SDP);
}

hdsdp_retcode sdp_presolve(void *p) { return obj(p)->sdp->presolve(); }

void sdp_destroy(void **pp) {
    if (!pp || !*pp) return;
    ConeObj *c = obj(*pp);
    if (c->sdp) {
        if (c->deviceReady) {
            HB_CUDA(cudaStreamSynchronize(c->sdp->s));
            c->sdp->release();
        }
        delete c->sdp;
    }
    if (c->dX) cache_free(c->dX);
    delete c;
    *pp = nullptr;
}

void sdp_set_start(void *p, double r) { obj(p)->sdp->set_start(r); }

void sdp_update(void *p, double tau, double *y) {
    if (sdp_ready(obj(p))) obj(p)->sdp->update(tau, y);
}

hdsdp_retcode sdp_ratio(void *p, double dtau, double *dy, double ada, int which, double *step) {
    if (!sdp_ready(obj(p))) return HDSDP_RETCODE_FAILED;
    return obj(p)->sdp->ratio_test(dtau, dy, ada, which, step);
}

int64_t sdp_sym_nnz(void *p) {
    const int64_t k = obj(p)->sdp->m;
    return k * k;
}

int sdp_dim(void *p) { return obj(p)->sdp->n; }

// Column iCol of the Schur pattern: every row for a dense cone; for a sparse cone, its
// rows at and below iCol when iCol is one of them (the dense M of this library needs no
// mapping, so the pattern only informs the host).
void sdp_add_sym_nz(void *p, int iCol, int *col) {
    SdpCone &s = *obj(p)->sdp;
    if (!s.sparse) {
        for (int i = 0; i < s.mAll; ++i) col[i] = 1;
        return;
    }
    auto it = std::lower_bound(s.rows.begin(), s.rows.end(), iCol);
    if (it == s.rows.end() || *it != iCol) return;
    for (; it != s.rows.end(); ++it) col[*it] = 1;
}

void sym_map_none(void *, int, int *) {}

hdsdp_retcode sdp_build_schur(void *p, void *kkt, int type) {
    ConeObj *c = obj(p);
    hdsdp_kkt_internal *k = static_cast<hdsdp_kkt_internal *>(kkt);
    if (!k || !k->ready || !sdp_ready(c)) return HDSDP_RETCODE_FAILED;
    return k->kkt.add_sdp(*c->sdp, type);
}

// The reference's fixed strategies choose among formulas of the same M (M1-M5,
// interface/hdsdp_conic_sdp.c:1806-1872); this library has one build per coefficient
// class, so the strategy does not change the result.
hdsdp_retcode sdp_build_schur_fixed(void *p, void *kkt, int type, int strategy) {
    (void) strategy;
    return sdp_build_schur(p, kkt, type);
}

hdsdp_retcode sdp_interior(void *p, double tau, double *y, int *interior) {
    if (!sdp_ready(obj(p))) return HDSDP_RETCODE_FAILED;
    return obj(p)->sdp->interior_check(tau, y, interior);
}

hdsdp_retcode sdp_interior_expert(void *p, double dC, double dA, double *y, double dEye, int which, int *interior) {
    if (!sdp_ready(obj(p))) return HDSDP_RETCODE_FAILED;
    return obj(p)->sdp->interior_check_expert(dC, dA, y, dEye, which, interior);
}

hdsdp_retcode sdp_barrier(void *p, double tau, double *y, int which, double *logdet) {
    if (!sdp_ready(obj(p))) return HDSDP_RETCODE_FAILED;
    return obj(p)->sdp->get_barrier(tau, y, which, logdet);
}

hdsdp_retcode sdp_axpy_check(void *p, double step, int which, int *interior) {
    if (!sdp_ready(obj(p))) return HDSDP_RETCODE_FAILED;
    return obj(p)->sdp->add_step_and_check(step, which, interior);
}

void sdp_reduce_resi(void *p, double r) { obj(p)->sdp->reduce_resi(r); }
void sdp_set_perturb(void *p, double v) { obj(p)->sdp->set_perturb(v); }

double *sdp_scratch(ConeObj *c) {
    if (!c->dX) HB_CUDA(cmalloc(&c->dX, sizeof(double) * c->sdp->ld * c->sdp->n));
    return c->dX;
}

// X = mu (S^-1 + S^-1 (A^* dy) S^-1) at S = C - A^T y into the host n x n array X; X is
// left as it was when that S is not interior (interface/hdsdp_conic_sdp.c:2328-2379).
void sdp_primal(void *p, double mu, double *y, double *dy, double *X, double *aux) {
    (void) aux;
    ConeObj *c = obj(p);
    if (!X || !sdp_ready(c)) return;
    SdpCone &s = *c->sdp;
    double *dX = sdp_scratch(c);
    if (!dX) return;
    HB_CUDA(cudaMemcpy2DAsync(dX, sizeof(double) * s.ld, X, sizeof(double) * s.n, sizeof(double) * s.n, s.n,
                              cudaMemcpyHostToDevice, s.s));
    s.get_primal(mu, y, dy, dX);
    HB_CUDA(cudaMemcpy2DAsync(X, sizeof(double) * s.n, dX, sizeof(double) * s.ld, sizeof(double) * s.n, s.n,
                              cudaMemcpyDeviceToHost, s.s));
    HB_CUDA(cudaStreamSynchronize(s.s));
}

// S of the current dual buffer as a full symmetric host n x n array.
void sdp_dual(void *p, double *S, double *aux) {
    (void) aux;
    ConeObj *c = obj(p);
    if (!S || !sdp_ready(c)) return;
    SdpCone &s = *c->sdp;
    double *dS = sdp_scratch(c);
    if (!dS) return;
    s.get_dual(dS);
    HB_CUDA(cudaMemcpy2DAsync(S, sizeof(double) * s.n, dS, sizeof(double) * s.ld, sizeof(double) * s.n, s.n,
                              cudaMemcpyDeviceToHost, s.s));
    HB_CUDA(cudaStreamSynchronize(s.s));
}

// out[i] += <A_i, X> for the host n x n array X (full, symmetric)
void sdp_atimesx(void *p, double *X, double *out) {
    ConeObj *c = obj(p);
    if (!sdp_ready(c)) return;
    SdpCone &s = *c->sdp;
    double *dX = sdp_scratch(c);
    if (!dX) return;
    HB_CUDA(cudaMemcpy2DAsync(dX, sizeof(double) * s.ld, X, sizeof(double) * s.n, sizeof(double) * s.n, s.n,
                              cudaMemcpyHostToDevice, s.s));
    s.atimesx(dX, out);
}

double sdp_trace_cx(void *p, double *X) {
    ConeObj *c = obj(p);
    if (!sdp_ready(c)) return NAN;
    SdpCone &s = *c->sdp;
    double *dX = sdp_scratch(c);
    if (!dX) return NAN;
    HB_CUDA(cudaMemcpy2DAsync(dX, sizeof(double) * s.ld, X, sizeof(double) * s.n, sizeof(double) * s.n, s.n,
                              cudaMemcpyHostToDevice, s.s));
    return s.trace_cx(dX);
}

double sdp_coeff_norm(void *p, int which) { return obj(p)->sdp->coeff_norm(which); }
double sdp_obj_norm(void *p, int which) { return obj(p)->sdp->obj_norm(which); }

void sdp_scal(void *p, double a) {
    ConeObj *c = obj(p);
    c->sdp->scal(a);
    if (c->deviceReady) {
        // the device copy of C was made with the old scale: rebuild it at the next hook
        HB_CUDA(cudaStreamSynchronize(c->sdp->s));
        c->sdp->release();
        c->deviceReady = false;
    }
}

void sdp_view(void *p) {
    const SdpCone &s = *obj(p)->sdp;
    printf("%s SDP cone of order %d with %d constraints (zero %d, sparse %d, dense %d, sparse rank-one %d, "
           "dense rank-one %d)\n",
           s.sparse ? "Sparse" : "Dense", s.n, s.m, s.stats[REF_ZERO], s.stats[REF_SPARSE], s.stats[REF_DENSE],
           s.stats[REF_SPR1], s.stats[REF_DSR1]);
}

void sdp_getstat(void *p, double *rowRHS, int intF[20], double dblF[20]) {
    obj(p)->sdp->detect_feature(rowRHS, intF, dblF);
}

// ---------------------------------------------------------------- LP cone
hdsdp_retcode lp_create(void **pp) { return create_of(pp, HDSDP_CONETYPE_LP); }

hdsdp_retcode lp_proc(void *p, int nRow, int nCol, int *Ap, int *Ai, double *Ax) {
    ConeObj *c = obj(p);
    c->lp = new (std::nothrow) LpCone();
    if (!c->lp) return HDSDP_RETCODE_MEMORY;
    return c->lp->proc_data(nRow, nCol, Ap, Ai, Ax, conic_stream());
}

hdsdp_retcode presolve_none(void *) { return HDSDP_RETCODE_OK; }

void lp_destroy(void **pp) {
    if (!pp || !*pp) return;
    ConeObj *c = obj(*pp);
    if (c->lp) {
        HB_CUDA(cudaStreamSynchronize(conic_stream()));
        c->lp->release();
        delete c->lp;
    }
    delete c;
    *pp = nullptr;
}

void lp_set_start(void *p, double r) { obj(p)->lp->set_start(r); }
void lp_update(void *p, double tau, double *y) { obj(p)->lp->update(tau, y); }

hdsdp_retcode lp_ratio(void *p, double dtau, double *dy, double ada, int which, double *step) {
    *step = obj(p)->lp->ratio_test(dtau, dy, ada, which);
    return HDSDP_RETCODE_OK;
}

int64_t lp_sym_nnz(void *p) {
    const int64_t m = obj(p)->lp->m;
    return m * m;
}

int lp_dim(void *p) { return obj(p)->lp->nCol; }

hdsdp_retcode lp_build_schur(void *p, void *kkt, int type) {
    hdsdp_kkt_internal *k = static_cast<hdsdp_kkt_internal *>(kkt);
    if (!k || !k->ready) return HDSDP_RETCODE_FAILED;
    k->kkt.add_lp(*obj(p)->lp, type);
    return device_error_flag() ? HDSDP_RETCODE_FAILED : HDSDP_RETCODE_OK;
}

hdsdp_retcode lp_build_schur_fixed(void *p, void *kkt, int type, int strategy) {
    (void) strategy;
    return lp_build_schur(p, kkt, type);
}

hdsdp_retcode lp_interior(void *p, double tau, double *y, int *interior) {
    *interior = obj(p)->lp->interior_check(tau, y);
    return HDSDP_RETCODE_OK;
}

hdsdp_retcode lp_interior_expert(void *p, double dC, double dA, double *y, double dEye, int which, int *interior) {
    *interior = obj(p)->lp->interior_check_expert(dC, dA, y, dEye, which);
    return HDSDP_RETCODE_OK;
}

hdsdp_retcode lp_barrier(void *p, double tau, double *y, int which, double *logdet) {
    *logdet = obj(p)->lp->get_barrier(tau, y, which);
    return HDSDP_RETCODE_OK;
}

hdsdp_retcode lp_axpy_check(void *p, double step, int which, int *interior) {
    *interior = obj(p)->lp->add_step_and_check(step, which);
    return HDSDP_RETCODE_OK;
}

void lp_reduce_resi(void *p, double r) { obj(p)->lp->reduce_resi(r); }
void lp_set_perturb(void *p, double v) { obj(p)->lp->set_perturb(v); }
void lp_primal(void *p, double mu, double *y, double *dy, double *x, double *aux) {
    (void) aux;
    obj(p)->lp->get_primal(mu, y, dy, x);
}
void lp_dual(void *p, double *s, double *aux) {
    (void) aux;
    obj(p)->lp->get_dual(s);
}
void lp_atimesx(void *p, double *x, double *out) { obj(p)->lp->atimesx(x, out); }
double lp_trace_cx(void *p, double *x) { return obj(p)->lp->trace_cx(x); }
double lp_coeff_norm(void *p, int which) { return obj(p)->lp->coeff_norm(which); }
double lp_obj_norm(void *p, int which) { return obj(p)->lp->obj_norm(which); }
void lp_scal(void *p, double a) { obj(p)->lp->scal(a); }
void lp_view(void *p) { printf("LP cone with %d columns and %d constraints\n", obj(p)->lp->nCol, obj(p)->lp->m); }
void lp_getstat(void *p, double *rowRHS, int intF[20], double dblF[20]) {
    (void) rowRHS;
    obj(p)->lp->detect_feature(intF, dblF);
}

// ---------------------------------------------------------------- scalar bound cone
// user data: nConicRow constraints, coneMatElem = {lower, upper}
// (interface/hdsdp_conic_bound.c:78-118)
hdsdp_retcode bnd_create(void **pp) { return create_of(pp, HDSDP_CONETYPE_SCALAR_BOUND); }

hdsdp_retcode bnd_proc(void *p, int nRow, int nCol, int *Ap, int *Ai, double *Ax) {
    (void) nCol;
    (void) Ap;
    (void) Ai;
    if (!Ax || !(Ax[0] < Ax[1])) return HDSDP_RETCODE_FAILED;
    ConeObj *c = obj(p);
    c->bnd = new (std::nothrow) BoundCone();
    if (!c->bnd) return HDSDP_RETCODE_MEMORY;
    c->bnd->proc(nRow, Ax[0], Ax[1]);
    return HDSDP_RETCODE_OK;
}

void bnd_destroy(void **pp) {
    if (!pp || !*pp) return;
    ConeObj *c = obj(*pp);
    delete c->bnd;
    delete c;
    *pp = nullptr;
}

void bnd_set_start(void *, double) {}
void bnd_update(void *p, double tau, double *y) { obj(p)->bnd->update(tau, y); }

hdsdp_retcode bnd_ratio(void *p, double dtau, double *dy, double ada, int which, double *step) {
    (void) ada;
    *step = obj(p)->bnd->ratio_test(dtau, dy, which);
    return HDSDP_RETCODE_OK;
}

int64_t bnd_sym_nnz(void *p) { return obj(p)->bnd->m; }
int bnd_dim(void *p) { return obj(p)->bnd->m; }
void bnd_add_sym_nz(void *, int iCol, int *col) { col[iCol] = 1; }

hdsdp_retcode bnd_build_schur(void *p, void *kkt, int type) {
    hdsdp_kkt_internal *k = static_cast<hdsdp_kkt_internal *>(kkt);
    if (!k || !k->ready) return HDSDP_RETCODE_FAILED;
    k->kkt.add_bound(*obj(p)->bnd, type);
    return device_error_flag() ? HDSDP_RETCODE_FAILED : HDSDP_RETCODE_OK;
}

hdsdp_retcode bnd_build_schur_fixed(void *p, void *kkt, int type, int strategy) {
    (void) strategy;
    return bnd_build_schur(p, kkt, type);
}

hdsdp_retcode bnd_interior(void *p, double tau, double *y, int *interior) {
    *interior = obj(p)->bnd->interior_check(tau, y);
    return HDSDP_RETCODE_OK;
}

hdsdp_retcode bnd_interior_expert(void *p, double dC, double dA, double *y, double dEye, int which, int *interior) {
    (void) dEye;
    *interior = obj(p)->bnd->interior_check_expert(dC, dA, y, which);
    return HDSDP_RETCODE_OK;
}

hdsdp_retcode bnd_barrier(void *p, double tau, double *y, int which, double *logdet) {
    return obj(p)->bnd->get_barrier(tau, y, which, logdet);
}

hdsdp_retcode bnd_axpy_check(void *p, double step, int which, int *interior) {
    *interior = obj(p)->bnd->add_step_and_check(step, which);
    return HDSDP_RETCODE_OK;
}

void bnd_reduce_resi(void *, double) {}
void bnd_set_perturb(void *, double) {}
void bnd_primal(void *p, double mu, double *y, double *dy, double *lower, double *upper) {
    obj(p)->bnd->get_primal(mu, y, dy, lower, upper);
}
double norm_none(void *, int) { return 0.0; }
void scal_none(void *, double) {}
void bnd_view(void *p) {
    printf("Bound cone %g <= y <= %g over %d rows\n", obj(p)->bnd->lo, obj(p)->bnd->up, obj(p)->bnd->m);
}

}  // namespace
}  // namespace hb

using namespace hb;

extern "C" {

hdsdp_retcode HConeCreate(hdsdp_cone **pHCone) {
    if (!pHCone) return HDSDP_RETCODE_FAILED;
    hdsdp_cone *c = (hdsdp_cone *) calloc(1, sizeof(hdsdp_cone));
    if (!c) return HDSDP_RETCODE_MEMORY;
    *pHCone = c;
    return HDSDP_RETCODE_OK;
}

int HConeGetVarBufferDim(hdsdp_cone *HCone) {
    const int d = HCone->coneGetDim(HCone->coneData);
    if (HCone->cone == HDSDP_CONETYPE_DENSE_SDP || HCone->cone == HDSDP_CONETYPE_SPARSE_SDP) return d * d;
    return d;
}

hdsdp_retcode HConeSetData(hdsdp_cone *c, user_data *usrData) {
    c->usrData = usrData;
    c->cone = HUserDataChooseCone(usrData);
    switch (c->cone) {
        case HDSDP_CONETYPE_DENSE_SDP:
        case HDSDP_CONETYPE_SPARSE_SDP:
            c->coneCreate = (c->cone == HDSDP_CONETYPE_DENSE_SDP) ? sdp_dense_create : sdp_sparse_create;
            c->coneProcData = sdp_proc;
            c->conePresolveData = sdp_presolve;
            c->coneDestroyData = sdp_destroy;
            c->coneSetStart = sdp_set_start;
            c->coneUpdate = sdp_update;
            c->coneRatioTest = sdp_ratio;
            c->coneGetSymNnz = sdp_sym_nnz;
            c->coneGetDim = sdp_dim;
            c->coneAddSymNz = sdp_add_sym_nz;
            c->coneGetKKTMap = sym_map_none;
            c->coneBuildSchur = sdp_build_schur;
            c->coneBuildSchurFixed = sdp_build_schur_fixed;
            c->coneInteriorCheck = sdp_interior;
            c->coneInteriorCheckExpert = sdp_interior_expert;
            c->coneGetBarrier = sdp_barrier;
            c->coneAxpyBufferAndCheck = sdp_axpy_check;
            c->coneReduceResi = sdp_reduce_resi;
            c->coneSetPerturb = sdp_set_perturb;
            c->conePRecover = sdp_primal;
            c->coneDRecover = sdp_dual;
            c->coneATimesX = sdp_atimesx;
            c->coneTraceCX = sdp_trace_cx;
            c->coneGetCoeffNorm = sdp_coeff_norm;
            c->coneGetObjNorm = sdp_obj_norm;
            c->coneScal = sdp_scal;
            c->coneView = sdp_view;
            c->getstat = sdp_getstat;
            return HDSDP_RETCODE_OK;
        case HDSDP_CONETYPE_LP:
            c->coneCreate = lp_create;
            c->coneProcData = lp_proc;
            c->conePresolveData = presolve_none;
            c->coneDestroyData = lp_destroy;
            c->coneSetStart = lp_set_start;
            c->coneUpdate = lp_update;
            c->coneRatioTest = lp_ratio;
            c->coneGetSymNnz = lp_sym_nnz;
            c->coneGetDim = lp_dim;
            c->coneAddSymNz = sym_map_none;
            c->coneGetKKTMap = sym_map_none;
            c->coneBuildSchur = lp_build_schur;
            c->coneBuildSchurFixed = lp_build_schur_fixed;
            c->coneInteriorCheck = lp_interior;
            c->coneInteriorCheckExpert = lp_interior_expert;
            c->coneGetBarrier = lp_barrier;
            c->coneAxpyBufferAndCheck = lp_axpy_check;
            c->coneReduceResi = lp_reduce_resi;
            c->coneSetPerturb = lp_set_perturb;
            c->conePRecover = lp_primal;
            c->coneDRecover = lp_dual;
            c->coneATimesX = lp_atimesx;
            c->coneTraceCX = lp_trace_cx;
            c->coneGetCoeffNorm = lp_coeff_norm;
            c->coneGetObjNorm = lp_obj_norm;
            c->coneScal = lp_scal;
            c->coneView = lp_view;
            c->getstat = lp_getstat;
            return HDSDP_RETCODE_OK;
        case HDSDP_CONETYPE_SCALAR_BOUND:
            c->coneCreate = bnd_create;
            c->coneProcData = bnd_proc;
            c->conePresolveData = presolve_none;
            c->coneDestroyData = bnd_destroy;
            c->coneSetStart = bnd_set_start;
            c->coneUpdate = bnd_update;
            c->coneRatioTest = bnd_ratio;
            c->coneGetSymNnz = bnd_sym_nnz;
            c->coneGetDim = bnd_dim;
            c->coneAddSymNz = bnd_add_sym_nz;
            c->coneGetKKTMap = sym_map_none;
            c->coneBuildSchur = bnd_build_schur;
            c->coneBuildSchurFixed = bnd_build_schur_fixed;
            c->coneInteriorCheck = bnd_interior;
            c->coneInteriorCheckExpert = bnd_interior_expert;
            c->coneGetBarrier = bnd_barrier;
            c->coneAxpyBufferAndCheck = bnd_axpy_check;
            c->coneReduceResi = bnd_reduce_resi;
            c->coneSetPerturb = bnd_set_perturb;
            c->conePRecover = bnd_primal;
            c->coneDRecover = nullptr;
            c->coneATimesX = nullptr;
            c->coneTraceCX = nullptr;
            c->coneGetCoeffNorm = norm_none;
            c->coneGetObjNorm = norm_none;
            c->coneScal = scal_none;
            c->coneView = bnd_view;
            c->getstat = nullptr;
            return HDSDP_RETCODE_OK;
        default:
            return HDSDP_RETCODE_FAILED;
    }
}

void HConeClear(hdsdp_cone *c) {
    if (!c) return;
    if (c->coneDestroyData) c->coneDestroyData(&c->coneData);
    memset(c, 0, sizeof(hdsdp_cone));
}

void HConeDestroy(hdsdp_cone **pHCone) {
    if (!pHCone) return;
    HConeClear(*pHCone);
    free(*pHCone);
    *pHCone = nullptr;
}

void HConeView(hdsdp_cone *c) { c->coneView(c->coneData); }

hdsdp_retcode HConeProcData(hdsdp_cone *c) {
    user_data *u = (user_data *) c->usrData;
    if (!c->coneCreate || !u) return HDSDP_RETCODE_FAILED;
    hdsdp_retcode r = c->coneCreate(&c->coneData);
    if (r != HDSDP_RETCODE_OK) return r;
    return c->coneProcData(c->coneData, u->nConicRow, u->nConicCol, u->coneMatBeg, u->coneMatIdx, u->coneMatElem);
}

hdsdp_retcode HConePresolveData(hdsdp_cone *c) { return c->conePresolveData(c->coneData); }

void HConeSetStart(hdsdp_cone *c, double v) { c->coneSetStart(c->coneData, v); }
void HConeUpdate(hdsdp_cone *c, double tau, double *y) { c->coneUpdate(c->coneData, tau, y); }

hdsdp_retcode HConeRatioTest(hdsdp_cone *c, double dtau, double *dy, double ada, int which, double *maxStep) {
    return c->coneRatioTest(c->coneData, dtau, dy, ada, which, maxStep);
}

int64_t HConeGetSymNnz(hdsdp_cone *c) { return c->coneGetSymNnz(c->coneData); }
void HConeAddSymNz(hdsdp_cone *c, int iCol, int *col) { c->coneAddSymNz(c->coneData, iCol, col); }
void HConeGetSymMapping(hdsdp_cone *c, int iCol, int *col) { c->coneGetKKTMap(c->coneData, iCol, col); }
int HConeGetDim(hdsdp_cone *c) { return c->coneGetDim(c->coneData); }
double HConeGetCoeffNorm(hdsdp_cone *c, int which) { return c->coneGetCoeffNorm(c->coneData, which); }
double HConeGetObjNorm(hdsdp_cone *c, int which) { return c->coneGetObjNorm(c->coneData, which); }

hdsdp_retcode HConeBuildSchurComplement(hdsdp_cone *c, void *schurMat, int typeKKT) {
    return c->coneBuildSchur(c->coneData, schurMat, typeKKT);
}

hdsdp_retcode HConeBuildSchurComplementFixed(hdsdp_cone *c, void *schurMat, int typeKKT, int kktStrategy) {
    return c->coneBuildSchurFixed(c->coneData, schurMat, typeKKT, kktStrategy);
}

hdsdp_retcode HConeGetLogBarrier(hdsdp_cone *c, double tau, double *y, int which, double *logdet) {
    return c->coneGetBarrier(c->coneData, tau, y, which, logdet);
}

hdsdp_retcode HConeAddStepToBufferAndCheck(hdsdp_cone *c, double step, int which, int *interior) {
    return c->coneAxpyBufferAndCheck(c->coneData, step, which, interior);
}

hdsdp_retcode HConeCheckIsInterior(hdsdp_cone *c, double tau, double *y, int *interior) {
    return c->coneInteriorCheck(c->coneData, tau, y, interior);
}

hdsdp_retcode HConeCheckIsInteriorExpert(hdsdp_cone *c, double dC, double dA, double *y, double dEye, int which,
                                         int *interior) {
    return c->coneInteriorCheckExpert(c->coneData, dC, dA, y, dEye, which, interior);
}

void HConeReduceResi(hdsdp_cone *c, double r) { c->coneReduceResi(c->coneData, r); }
void HConeSetPerturb(hdsdp_cone *c, double v) { c->coneSetPerturb(c->coneData, v); }

void HConeGetPrimal(hdsdp_cone *c, double mu, double *y, double *dy, double *X, double *X2) {
    c->conePRecover(c->coneData, mu, y, dy, X, X2);
}

void HConeGetDual(hdsdp_cone *c, double *S, double *S2) {
    if (c->coneDRecover) c->coneDRecover(c->coneData, S, S2);
}

void HConeComputeATimesX(hdsdp_cone *c, double *X, double *out) {
    if (c->coneATimesX) c->coneATimesX(c->coneData, X, out);
}

double HConeComputeTraceCX(hdsdp_cone *c, double *X) {
    return c->coneTraceCX ? c->coneTraceCX(c->coneData, X) : 0.0;
}

void HConeScalByConstant(hdsdp_cone *c, double a) { c->coneScal(c->coneData, a); }

void HConeDetectFeature(hdsdp_cone *c, double *rowRHS, int intF[20], double dblF[20]) {
    if (c->getstat) c->getstat(c->coneData, rowRHS, intF, dblF);
}

// ---------------------------------------------------------------- KKT manager
hdsdp_retcode HKKTCreate(hdsdp_kkt **pHKKT) {
    if (!pHKKT) return HDSDP_RETCODE_FAILED;
    hdsdp_kkt *k = new (std::nothrow) hdsdp_kkt_internal();
    if (!k) return HDSDP_RETCODE_MEMORY;
    *pHKKT = k;
    return HDSDP_RETCODE_OK;
}

hdsdp_retcode HKKTInit(hdsdp_kkt *k, int nRow, int nCones, hdsdp_cone **cones) {
    if (!k || nRow <= 0 || nCones < 0 || (nCones > 0 && !cones)) return HDSDP_RETCODE_FAILED;
    if (k->ready) {
        HB_CUDA(cudaStreamSynchronize(k->kkt.s));
        k->kkt.release();
        k->ready = false;
    }
    k->nRow = nRow;
    k->nCones = nCones;
    k->cones = cones;
    k->kkt.init(nRow, conic_stream(), &k->tm);
    HB_CUDA(cudaStreamSynchronize(k->kkt.s));
    if (device_error_flag()) return HDSDP_RETCODE_MEMORY;
    k->ready = true;
    return HDSDP_RETCODE_OK;
}

hdsdp_retcode HKKTBuildUp(hdsdp_kkt *k, int typeKKT) {
    if (!k || !k->ready) return HDSDP_RETCODE_FAILED;
    k->kkt.clean(typeKKT);
    for (int i = 0; i < k->nCones; ++i) {
        hdsdp_retcode r = HConeBuildSchurComplement(k->cones[i], k, typeKKT);
        if (r != HDSDP_RETCODE_OK) return r;
    }
    return HDSDP_RETCODE_OK;
}

hdsdp_retcode HKKTBuildUpExtraCone(hdsdp_kkt *k, hdsdp_cone *cone, int typeKKT) {
    if (!k || !k->ready || !cone) return HDSDP_RETCODE_FAILED;
    return HConeBuildSchurComplement(cone, k, typeKKT);
}

hdsdp_retcode HKKTBuildUpFixed(hdsdp_kkt *k, int typeKKT, int kktStrategy) {
    if (!k || !k->ready) return HDSDP_RETCODE_FAILED;
    k->kkt.clean(typeKKT);
    for (int i = 0; i < k->nCones; ++i) {
        hdsdp_retcode r = HConeBuildSchurComplementFixed(k->cones[i], k, typeKKT, kktStrategy);
        if (r != HDSDP_RETCODE_OK) return r;
    }
    return HDSDP_RETCODE_OK;
}

void HKKTExport(hdsdp_kkt *k, double *asinv, double *asinvrd, double *asinvcs, double *csinvcsinv, double *csinv,
                double *csinvrdcsinv, double *tracesinv) {
    if (!k || !k->ready) return;
    const size_t bytes = sizeof(double) * k->nRow;
    if (asinv) memcpy(asinv, k->kkt.asinv.data(), bytes);
    if (asinvrd) memcpy(asinvrd, k->kkt.asinvrd.data(), bytes);
    if (asinvcs) memcpy(asinvcs, k->kkt.asinvcs.data(), bytes);
    if (csinvcsinv) *csinvcsinv = k->kkt.dCSinvCSinv;
    if (csinv) *csinv = k->kkt.dCSinv;
    if (csinvrdcsinv) *csinvrdcsinv = k->kkt.dCSinvRdSinv;
    if (tracesinv) *tracesinv = k->kkt.dTraceSinv;
}

hdsdp_retcode HKKTFactorize(hdsdp_kkt *k) {
    if (!k || !k->ready) return HDSDP_RETCODE_FAILED;
    return k->kkt.factorize();
}

hdsdp_retcode HKKTSolve(hdsdp_kkt *k, double *rhs, double *lhs) {
    if (!k || !k->ready || !rhs) return HDSDP_RETCODE_FAILED;
    return k->kkt.solve(rhs, lhs ? lhs : rhs);
}

void HKKTRegularize(hdsdp_kkt *k, double reg) {
    if (k && k->ready) k->kkt.regularize(reg);
}

void HKKTClear(hdsdp_kkt *k) {
    if (!k) return;
    if (k->ready) {
        HB_CUDA(cudaStreamSynchronize(k->kkt.s));
        k->kkt.release();
    }
    k->ready = false;
    k->nRow = k->nCones = 0;
    k->cones = nullptr;
}

void HKKTDestroy(hdsdp_kkt **pHKKT) {
    if (!pHKKT || !*pHKKT) return;
    HKKTClear(*pHKKT);
    delete *pHKKT;
    *pHKKT = nullptr;
}

hdsdp_retcode HKKTGetMatrix(hdsdp_kkt *k, double *M) {
    if (!k || !k->ready || !M) return HDSDP_RETCODE_FAILED;
    const int m = k->nRow;
    std::vector<double> full((size_t) m * m);
    HB_CUDA(cudaMemcpy2DAsync(full.data(), sizeof(double) * m, k->kkt.M, sizeof(double) * k->kkt.ldm,
                              sizeof(double) * m, m, cudaMemcpyDeviceToHost, k->kkt.s));
    HB_CUDA(cudaStreamSynchronize(k->kkt.s));
    if (device_error_flag()) return HDSDP_RETCODE_FAILED;
    for (int j = 0; j < m; ++j)
        for (int i = j; i < m; ++i) M[(size_t) i + (size_t) j * m] = full[(size_t) i + (size_t) j * m];
    return HDSDP_RETCODE_OK;
}

}  // extern "C"
