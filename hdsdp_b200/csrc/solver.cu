// Interior-point driver and public C API of the B200 HDSDP library.
//
// Control flow, constants and heuristics restate the reference's dual-scaling
// method so that iterates, iteration counts and statuses match it:
//   presolve / parameters  interface/hdsdp.c:29-402, :617-689
//   Phase A (infeasible)   interface/hdsdp_algo.c:547-1203
//   Phase A' (embedding)   interface/hdsdp_algo.c:262-545
//   Phase B (potential)    interface/hdsdp_algo.c:1205-1846
//   primal refinement      interface/hdsdp_psdp.c:81-295
//   solution check         interface/hdsdp.c:711-906
// The numerical work of every step runs on the GPU through SdpCone and KKT.
#include "solver.h"
#include <cmath>
#include <cstring>
#include <cstdio>
#include <algorithm>
#include <chrono>

using namespace hb;

namespace {

enum {
    I_NULLOBJ = 0, I_MANYCONES = 1, I_NOPINTERIOR = 2, I_NODINTERIOR = 3, I_VERYDENSE = 4, I_IMPTRACE = 5,
    I_IMPYBOUND = 6, N_SUMCONEDIMS = 7, N_MAXCONEDIM = 8, N_CONES = 9, N_ROWS = 10, N_SPSDPCONES = 11,
    N_DSSDPCONES = 12, N_LPCONES = 13, N_BNDCONES = 14
};
enum {
    D_OBJFRONORM = 0, D_OBJONENORM = 1, D_RHSFRONORM = 2, D_RHSONENORM = 3, D_RHSINFNORM = 4, D_OBJSCALING = 5,
    D_RHSSCALING = 6, D_DATAFRONORM = 7, D_DATAONENORM = 8, D_IMPYBOUNDUP = 9, D_IMPYBOUNDLOW = 10, D_IMPTRACEX = 11
};
enum { METHOD_INFEAS = 0, METHOD_HSD = 1, METHOD_POTENTIAL = 2 };

double wall() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

#define CALL(x)                                  \
    do {                                         \
        retcode = (x);                           \
        if (retcode != HDSDP_RETCODE_OK) goto exit_cleanup; \
    } while (0)

inline int &ip(hdsdp *h, int i) { return h->HIntParams[i]; }
inline double &dp(hdsdp *h, int i) { return h->HDblParams[i]; }
inline int &fi(hdsdp *h, int i) { return h->HIntFeatures[i]; }
inline double &fd(hdsdp *h, int i) { return h->HDblFeatures[i]; }

void default_params(hdsdp *h) {
    ip(h, INT_PARAM_MAXITER) = 500;
    ip(h, INT_PARAM_CORRECTORA) = 12;
    ip(h, INT_PARAM_CORRECTORB) = 12;
    ip(h, INT_PARAM_THREADS) = 12;
    ip(h, INT_PARAM_PSDP) = 1;
    dp(h, DBL_PARAM_ABSOPTTOL) = 1e-08;
    dp(h, DBL_PARAM_ABSFEASTOL) = 1e-08;
    dp(h, DBL_PARAM_RELOPTTOL) = 1e-10;
    dp(h, DBL_PARAM_RELFEASTOL) = 1e-10;
    dp(h, DBL_PARAM_TIMELIMIT) = 3600.0;
    dp(h, DBL_PARAM_POTRHOVAL) = 4.0;
    dp(h, DBL_PARAM_HSDGAMMA) = 0.5;
    dp(h, DBL_PARAM_DUALBOX_UP) = 1e+07;
    dp(h, DBL_PARAM_DUALBOX_LOW) = -1e+07;
    dp(h, DBL_PARAM_BARMUSTART) = 1e+05;
    dp(h, DBL_PARAM_POBJSTART) = 1e+10;
    dp(h, DBL_PARAM_DUALSTART) = 1e+05;
    dp(h, DBL_PARAM_TRXESTIMATE) = 1e+08;
    dp(h, DBL_PARAM_PRECORDACC) = 1e-08;
}

// ---------------------------------------------------------------- statistics / tuning
void get_statistics(hdsdp *h) {
    int sumDims = 0, maxDim = 0, nDense = 0, nSparse = 0, nLp = 0;
    // sums over the cones in the user's order, as the reference adds them
    double objOne = 0.0, dataOne = 0.0, objFro2 = 0.0, dataFro2 = 0.0;
    for (ConeSlot &k : h->cones) {
        double of, df;
        if (k.sdp) {
            maxDim = std::max(maxDim, k.sdp->n);
            sumDims += k.sdp->n;
            objOne += k.sdp->obj_norm(ABS_NORM);
            dataOne += k.sdp->coeff_norm(ABS_NORM);
            of = k.sdp->obj_norm(FRO_NORM);
            df = k.sdp->coeff_norm(FRO_NORM);
            (k.sdp->sparse ? nSparse : nDense) += 1;
        } else {
            sumDims += k.lp->nCol;
            objOne += k.lp->obj_norm(ABS_NORM);
            dataOne += k.lp->coeff_norm(ABS_NORM);
            of = k.lp->obj_norm(FRO_NORM);
            df = k.lp->coeff_norm(FRO_NORM);
            nLp += 1;
        }
        objFro2 += of * of;
        dataFro2 += df * df;
    }
    fi(h, N_MAXCONEDIM) = maxDim;
    fi(h, N_SUMCONEDIMS) = sumDims;
    fi(h, N_ROWS) = h->nRows;
    fi(h, N_CONES) = h->nCones;
    h->allConeDims = (double) sumDims + 2.0 * h->nRows;
    fd(h, D_OBJFRONORM) = std::sqrt(objFro2);
    fd(h, D_DATAFRONORM) = std::sqrt(dataFro2);
    fd(h, D_OBJONENORM) = objOne;
    fd(h, D_DATAONENORM) = dataOne;
    double one = 0, fro = 0, inf = 0;
    for (int i = 0; i < h->nRows; ++i) {
        one += std::fabs(h->rowRHS[i]);
        fro += h->rowRHS[i] * h->rowRHS[i];
        inf = std::max(inf, std::fabs(h->rowRHS[i]));
    }
    fd(h, D_RHSONENORM) = one;
    fd(h, D_RHSFRONORM) = std::sqrt(fro);
    fd(h, D_RHSINFNORM) = inf;
    if (fd(h, D_OBJFRONORM) == 0.0) fi(h, I_NULLOBJ) = 1;
    if (h->nCones >= 100) fi(h, I_MANYCONES) = 1;
    fi(h, N_DSSDPCONES) = nDense;
    fi(h, N_SPSDPCONES) = nSparse;
    fi(h, N_LPCONES) = nLp;
}

// HConeDetectFeature of one cone: the dense SDP cone's structure tests
// (conic_sdp.c:2560-2654), only the coefficient counts for a sparse SDP cone
// (conic_sdp.c:2656-2667), the LP cone's tests (conic_lp.c)
void detect_feature_of(hdsdp *h, ConeSlot &k) {
    if (k.lp) {
        k.lp->detect_feature(h->HIntFeatures, h->HDblFeatures);
    } else if (!k.sdp->sparse) {
        k.sdp->detect_feature(h->rowRHS.data(), h->HIntFeatures, h->HDblFeatures);
    } else {
        const int *st = k.sdp->stats;
        h->HIntFeatures[15] = st[REF_ZERO];
        h->HIntFeatures[17] = st[REF_DENSE];
        h->HIntFeatures[16] = st[REF_SPARSE];
        h->HIntFeatures[18] = st[REF_SPR1];
        h->HIntFeatures[19] = st[REF_DSR1];
    }
}

// HDSDPIAdjustConeParams (interface/hdsdp.c:136-152): structure detection on the first
// cone when there is one SDP cone, on the last cone when LP cones are present (fewer
// than ten cones); primal refinement only with a single SDP cone
void adjust_cone_params(hdsdp *h) {
    const bool oneCone = fi(h, N_DSSDPCONES) + fi(h, N_SPSDPCONES) <= 1;
    if (!oneCone) ip(h, INT_PARAM_PSDP) = 0;
    if (oneCone) detect_feature_of(h, h->cones[0]);
    if (fi(h, N_LPCONES) && fi(h, N_CONES) < 10) detect_feature_of(h, h->cones[h->nCones - 1]);
    const int impTrace = fi(h, I_IMPTRACE), noPInt = fi(h, I_NOPINTERIOR), noDInt = fi(h, I_NODINTERIOR);
    const int dense = fi(h, I_VERYDENSE), impDual = fi(h, I_IMPYBOUND), noObj = fi(h, I_NULLOBJ);
    h->modelFeatures.clear();
    const bool hit = (impTrace + noPInt + noDInt + dense + noObj) || impDual;
    if (hit) h->modelFeatures += "This is a ";
    if (dense) {
        ip(h, INT_PARAM_CORRECTORA) = 4;
        dp(h, DBL_PARAM_DUALSTART) = 1.0;
        dp(h, DBL_PARAM_DUALBOX_UP) = 1e+04;
        dp(h, DBL_PARAM_DUALBOX_LOW) = -1e+04;
        h->modelFeatures += "dense ";
    }
    if (impTrace) {
        dp(h, DBL_PARAM_DUALSTART) = 1e+03;
        dp(h, DBL_PARAM_TRXESTIMATE) = fd(h, D_IMPTRACEX);
        dp(h, DBL_PARAM_POBJSTART) = 1e+08;
        dp(h, DBL_PARAM_POTRHOVAL) = 5.0;
        dp(h, DBL_PARAM_DUALBOX_UP) = 1e+06;
        dp(h, DBL_PARAM_DUALBOX_LOW) = -1e+06;
        h->modelFeatures += "trace-implied ";
    }
    if (noPInt) {
        dp(h, DBL_PARAM_DUALBOX_UP) = 1e+04;
        dp(h, DBL_PARAM_DUALBOX_LOW) = -1e+04;
        dp(h, DBL_PARAM_DUALSTART) = 1e+03;
        dp(h, DBL_PARAM_PRECORDACC) = 1e-07;
        h->modelFeatures += "no-primal interior ";
    }
    if (impDual) {
        double bu = dp(h, DBL_PARAM_DUALBOX_UP), bl = dp(h, DBL_PARAM_DUALBOX_LOW);
        int isU = 0, isL = 0;
        if (fd(h, D_IMPYBOUNDUP)) {
            isU = 1;
            bu = std::min(bu, fd(h, D_IMPYBOUNDUP));
            dp(h, DBL_PARAM_DUALBOX_UP) = bu;
        }
        if (fd(h, D_IMPYBOUNDLOW)) {
            isL = 1;
            bl = std::max(bl, fd(h, D_IMPYBOUNDLOW));
            dp(h, DBL_PARAM_DUALBOX_LOW) = bl;
        }
        if (isU && isL) {
            dp(h, DBL_PARAM_DUALSTART) = 1e+02;
            dp(h, DBL_PARAM_POBJSTART) = 1e+05;
        } else {
            dp(h, DBL_PARAM_DUALSTART) = 1e+05;
            dp(h, DBL_PARAM_POBJSTART) = 1e+10;
            ip(h, INT_PARAM_CORRECTORA) = 12;
            ip(h, INT_PARAM_CORRECTORB) = 12;
        }
        dp(h, DBL_PARAM_ABSOPTTOL) = 1e-01;
        dp(h, DBL_PARAM_RELOPTTOL) = 1e-04;
        dp(h, DBL_PARAM_PRECORDACC) = 1e-05;
        h->modelFeatures += "dual-bounded ";
    }
    if (noDInt) {
        dp(h, DBL_PARAM_DUALBOX_UP) = 1.0;
        dp(h, DBL_PARAM_DUALBOX_LOW) = -1.0;
        if (h->allConeDims > 100000) {
            dp(h, DBL_PARAM_DUALSTART) = 1e+00;
            dp(h, DBL_PARAM_ABSFEASTOL) = 1e-04;
            dp(h, DBL_PARAM_RELFEASTOL) = 1e-05;
        } else {
            dp(h, DBL_PARAM_DUALBOX_UP) = 1e+01;
            dp(h, DBL_PARAM_DUALBOX_LOW) = -1e+01;
            dp(h, DBL_PARAM_ABSFEASTOL) = 1e-05;
            dp(h, DBL_PARAM_RELFEASTOL) = 1e-07;
        }
        dp(h, DBL_PARAM_PRECORDACC) = 1e-05;
        h->modelFeatures += "no-dual interior ";
    }
    if (noObj) {
        dp(h, DBL_PARAM_DUALSTART) = 1.0;
        dp(h, DBL_PARAM_DUALBOX_UP) = 1.0;
        dp(h, DBL_PARAM_DUALBOX_LOW) = -1.0;
        h->modelFeatures += "no objective ";
    }
    if (hit) h->modelFeatures += "SDP problem\n";
}

void adjust_params(hdsdp *h) {
    const double objOne = fd(h, D_OBJONENORM), rhsInf = fd(h, D_RHSINFNORM);
    double objScal = 1.0, rhsScal = 1.0;
    if (objOne > 1e+10) objScal = 1e-08;
    else if (objOne > 1e+08) objScal = 1e-06;
    else if (objOne > 1e+05) objScal = 1e-05;
    if (rhsInf > 1e+10) rhsScal = 1e-08;
    else if (rhsInf > 1e+08) rhsScal = 1e-06;
    else rhsScal = 1.0;
    fd(h, D_OBJSCALING) = objScal;
    fd(h, D_RHSSCALING) = rhsScal;
    for (ConeSlot &k : h->cones) {
        if (k.sdp) k.sdp->scal(objScal);
        else k.lp->scal(objScal);
    }
    for (int i = 0; i < h->nRows; ++i) h->rowRHS[i] *= rhsScal;
    // thread count: the GPU build records the host default
    ip(h, INT_PARAM_THREADS) = std::min(ip(h, INT_PARAM_THREADS), 12);

    const int maxDim = fi(h, N_MAXCONEDIM);
    int nCorrA = (h->nRows - 2) / maxDim;
    if (fi(h, N_SUMCONEDIMS) < 100 && nCorrA == 0) nCorrA = 1;
    if (nCorrA >= 1) nCorrA += 1;
    nCorrA = nCorrA * nCorrA;
    if (h->nRows < 2000 && nCorrA > 10) nCorrA = 10;
    int nCorrB = nCorrA;
    if (maxDim >= 5 * h->nRows) {
        nCorrB = 0;
        nCorrA = 2;
    } else if (maxDim >= h->nRows) {
        nCorrB = std::min(nCorrB, 2);
        nCorrA = 4;
    } else {
        nCorrA = 6;
    }
    if (h->nRows > 20 * maxDim) {
        nCorrB = std::max(nCorrB, 12);
        nCorrA = 12;
    } else if (h->nRows > 5 * maxDim) {
        nCorrB = std::max(nCorrB, 10);
        nCorrA = 10;
    } else if (h->nRows > 2 * maxDim) {
        nCorrB = std::max(nCorrB, 8);
        nCorrA = 8;
    }
    nCorrB = std::min(nCorrB, 12);
    nCorrA = std::max(nCorrA, 2);
    ip(h, INT_PARAM_CORRECTORA) = nCorrA;
    ip(h, INT_PARAM_CORRECTORB) = nCorrB;
    if (fi(h, I_MANYCONES)) {
        ip(h, INT_PARAM_CORRECTORA) = 6;
        ip(h, INT_PARAM_CORRECTORB) = 0;
        dp(h, DBL_PARAM_DUALSTART) = 1.0;
        dp(h, DBL_PARAM_POBJSTART) = 1e+10;
    }
    adjust_cone_params(h);
}

// ---------------------------------------------------------------- algorithm helpers
void cones_set_start(hdsdp *h, double r);

void set_start(hdsdp *h, int method, int dOnly) {
    std::fill(h->y.begin(), h->y.end(), 0.0);
    h->tau = 1.0;
    double objFro = fd(h, D_OBJFRONORM) * fd(h, D_OBJSCALING);
    objFro = std::max(objFro, 100.0);
    if (method == METHOD_HSD) {
        h->mu = 1e+08;
        h->resi = dOnly ? -objFro * dp(h, DBL_PARAM_DUALSTART) : -objFro * 1e+01;
    } else {
        h->resi = -objFro * dp(h, DBL_PARAM_DUALSTART);
        h->pInfeas = 1.0 + fd(h, D_RHSFRONORM);
        h->pObjInternal = dp(h, DBL_PARAM_POBJSTART);
        h->mu = h->pObjInternal - h->dObjInternal - h->resi * dp(h, DBL_PARAM_TRXESTIMATE);
        h->mu = h->mu / h->allConeDims;
    }
    if (h->verbose) printf("Initialize with dual residual %3.1e\n", -h->resi);
    cones_set_start(h, h->resi);
}

void reset_start(hdsdp *h) {
    std::fill(h->y.begin(), h->y.end(), 0.0);
    h->tau = 1.0;
    const double objFro = fd(h, D_OBJFRONORM);
    h->pObjInternal = 1e+15;
    h->resi = -std::max(objFro, 1e+02) * 1e+06;
    h->resi = std::max(h->resi, -1e+15);
    if (h->verbose) printf("Reset with dual residual %3.1e\n", -h->resi);
    cones_set_start(h, h->resi);
}

void print_log(hdsdp *h, int method) {
    const double rhsScal = fd(h, D_RHSSCALING), objScal = fd(h, D_OBJSCALING);
    const double elapsed = wall() - h->timeBegin;
    const double nSum = (double) fi(h, N_SUMCONEDIMS);
    const double pdScal = 1.0 / (rhsScal * objScal * h->tau);
    h->dInfeas = std::sqrt(nSum) * std::fabs(h->resi) / (rhsScal * h->tau);
    h->dObjInternal = 0.0;
    for (int i = 0; i < h->nRows; ++i) h->dObjInternal += h->rowRHS[i] * h->y[i];
    h->dObjVal = h->dObjInternal * pdScal;
    h->pObjVal = h->pObjInternal * pdScal;
    h->comp = h->pObjVal - h->dObjVal;
    const double gap = h->comp / (std::fabs(h->pObjVal) + std::fabs(h->dObjVal) + 1.0);
    h->log.push_back({elapsed, h->pObjVal, h->dObjVal, h->mu, gap, method});
    if (!h->verbose) return;
    const double third = (method == METHOD_HSD) ? h->tau : h->proxNorm;
    const double infv = (method == METHOD_POTENTIAL) ? h->pInfeas : h->dInfeas;
    printf("    %5d  %+15.8e  %+15.8e  %8.2e  %8.2e  %5.2f  %5.1e  %4.1f\n", h->nIterCount + 1,
           (method == METHOD_HSD) ? HDSDP_INFINITY : h->pObjVal, h->dObjVal, infv, h->mu, h->dStep, third, elapsed);
}

// Arithmetic of the next full Schur build: mode 0 FP64; 1 split precision
// throughout; 2 split precision while the relative gap is above 1e-3 (or not
// yet defined), FP64 for the final iterations.
void schur_precision(hdsdp *h) {
    int p = 0;
    if (h->precision == 1) {
        p = 1;
    } else if (h->precision == 2) {
        const double gap = h->log.empty() ? HDSDP_INFINITY : std::fabs(h->log.back().gap);
        p = (std::isfinite(gap) && gap < 1e-3) ? 0 : 1;
    }
    for (ConeSlot &k : h->cones)
        if (k.sdp) k.sdp->dev.precision = p;
}

// ---- the cones in the user's order (interface/hdsdp_algo.c: every loop over HCones)
//
// With several SDP cones, the checks first bring every SDP cone's buffer up to date and
// factor them together (factor_buffers: the small blocks in one launch, one wait), then
// read the answers in the user's order with the reference's early exit. The cones after
// the first failing one have then been factored too, which changes no result: every later
// use of a buffer rebuilds it from its inputs.
static std::vector<SdpCone *> sdp_cones(hdsdp *h) {
    std::vector<SdpCone *> v;
    for (ConeSlot &k : h->cones)
        if (k.sdp) v.push_back(k.sdp);
    return v;
}

// SdpCone::update(tau, y) of every cone of sc, batched
static void update_cones(hdsdp *h, const std::vector<SdpCone *> &sc, double tau, const double *y) {
    std::vector<double> eye;
    for (SdpCone *c : sc) eye.push_back(-c->dualResidual);
    assemble_buffers(sc, tau, -1.0, y, eye, BUFFER_DUALVAR, h->d_yall, h->h_yall);
}

static bool batched_cones(hdsdp *h) {
    int nSdp = 0;
    for (ConeSlot &k : h->cones) nSdp += k.sdp ? 1 : 0;
    return nSdp > 1;
}

// the answers of the batched checks in the user's order: SDP cones from ok, LP cones by
// their own check; stops at the first cone that is not interior
template <class LpCheck>
static int cones_first_failure(hdsdp *h, const std::vector<char> &ok, LpCheck lpCheck) {
    size_t q = 0;
    for (ConeSlot &k : h->cones) {
        const int in = k.sdp ? (int) ok[q++] : lpCheck(*k.lp);
        if (!in) return 0;
    }
    return 1;
}

hdsdp_retcode cones_interior(hdsdp *h, double tau, const double *y, int *interior) {
    *interior = 1;
    if (batched_cones(h)) {
        std::vector<SdpCone *> sc = sdp_cones(h);
        update_cones(h, sc, tau, y);
        std::vector<char> ok;
        factor_buffers(sc, BUFFER_DUALVAR, ok);
        *interior = cones_first_failure(h, ok, [&](LpCone &lp) { return lp.interior_check(tau, y); });
        return device_error_flag() ? HDSDP_RETCODE_FAILED : HDSDP_RETCODE_OK;
    }
    for (ConeSlot &k : h->cones) {
        if (k.sdp) {
            hdsdp_retcode r = k.sdp->interior_check(tau, y, interior);
            if (r != HDSDP_RETCODE_OK) return r;
        } else {
            *interior = k.lp->interior_check(tau, y);
        }
        if (!*interior) break;
    }
    return HDSDP_RETCODE_OK;
}

hdsdp_retcode cones_interior_expert(hdsdp *h, double dC, double dAs, const double *y, double dEye, int which,
                                    int *interior) {
    *interior = 1;
    if (batched_cones(h)) {
        std::vector<SdpCone *> sc = sdp_cones(h);
        assemble_buffers(sc, dC, dAs, y, std::vector<double>(sc.size(), dEye), which, h->d_yall, h->h_yall);
        std::vector<char> ok;
        factor_buffers(sc, which == BUFFER_DUALVAR ? BUFFER_DUALVAR : BUFFER_DUALCHECK, ok);
        *interior = cones_first_failure(
            h, ok, [&](LpCone &lp) { return lp.interior_check_expert(dC, dAs, y, dEye, which); });
        return device_error_flag() ? HDSDP_RETCODE_FAILED : HDSDP_RETCODE_OK;
    }
    for (ConeSlot &k : h->cones) {
        if (k.sdp) {
            hdsdp_retcode r = k.sdp->interior_check_expert(dC, dAs, y, dEye, which, interior);
            if (r != HDSDP_RETCODE_OK) return r;
        } else {
            *interior = k.lp->interior_check_expert(dC, dAs, y, dEye, which);
        }
        if (!*interior) break;
    }
    return HDSDP_RETCODE_OK;
}

// running minimum of the cones' step bounds
hdsdp_retcode cones_ratio(hdsdp *h, double dtau, const double *dy, double ada, int which, double *mx) {
    if (batched_cones(h)) {
        // the small blocks' Lanczos bounds share their launches (lanczos_small_batch)
        std::vector<double> st(h->cones.size(), HDSDP_INFINITY);
        std::vector<LzTask> tasks;
        std::vector<SdpCone *> small;
        size_t q = 0;
        for (ConeSlot &k : h->cones) {
            double *sq = &st[q++];
            if (k.sdp && k.sdp->small_lanczos()) {
                SdpCone &c = *k.sdp;
                small.push_back(&c);
                tasks.push_back(LzTask{&c.lz, which == BUFFER_DUALVAR ? &c.Fvar : &c.Fcheck, c.dS, c.ld, sq, c.tm,
                                       HDSDP_RETCODE_OK});
            } else if (k.sdp) {
                hdsdp_retcode r = k.sdp->ratio_test(dtau, dy, ada, which, sq);
                if (r != HDSDP_RETCODE_OK) return r;
            } else {
                *sq = k.lp->ratio_test(dtau, dy, ada, which);
            }
        }
        {
            std::vector<double> eye;
            for (SdpCone *c : small) eye.push_back(ada * c->dualResidual);
            assemble_buffers(small, dtau, -1.0, dy, eye, BUFFER_DUALSTEP, h->d_yall, h->h_yall);
        }
        lanczos_small_batch(tasks);
        for (const LzTask &t : tasks)
            if (t.ret != HDSDP_RETCODE_OK) return t.ret;
        for (double v : st) *mx = std::min(*mx, v);
        return HDSDP_RETCODE_OK;
    }
    for (ConeSlot &k : h->cones) {
        double st = 0.0;
        if (k.sdp) {
            hdsdp_retcode r = k.sdp->ratio_test(dtau, dy, ada, which, &st);
            if (r != HDSDP_RETCODE_OK) return r;
        } else {
            st = k.lp->ratio_test(dtau, dy, ada, which);
        }
        *mx = std::min(*mx, st);
    }
    return HDSDP_RETCODE_OK;
}

hdsdp_retcode cones_add_step(hdsdp *h, double step, int which, int *interior) {
    *interior = 1;
    if (batched_cones(h)) {
        std::vector<SdpCone *> sc = sdp_cones(h);
        for (SdpCone *c : sc) c->add_step(step, which);
        std::vector<char> ok;
        factor_buffers(sc, which == BUFFER_DUALVAR ? BUFFER_DUALVAR : BUFFER_DUALCHECK, ok);
        *interior = cones_first_failure(h, ok, [&](LpCone &lp) { return lp.add_step_and_check(step, which); });
        return device_error_flag() ? HDSDP_RETCODE_FAILED : HDSDP_RETCODE_OK;
    }
    for (ConeSlot &k : h->cones) {
        if (k.sdp) {
            hdsdp_retcode r = k.sdp->add_step_and_check(step, which, interior);
            if (r != HDSDP_RETCODE_OK) return r;
        } else {
            *interior = k.lp->add_step_and_check(step, which);
        }
        if (!*interior) break;
    }
    return HDSDP_RETCODE_OK;
}

void cones_set_start(hdsdp *h, double r) {
    for (ConeSlot &k : h->cones) {
        if (k.sdp) k.sdp->set_start(r);
        else k.lp->set_start(r);
    }
}

// sum of the cones' log det (SDP) or sum log s (LP) at the buffer `which`
hdsdp_retcode cones_barrier(hdsdp *h, double tau, const double *y, int which, double *sum) {
    *sum = 0.0;
    if (y && batched_cones(h)) {
        std::vector<SdpCone *> sc = sdp_cones(h);
        update_cones(h, sc, tau, y);
        std::vector<char> ok;
        factor_buffers(sc, BUFFER_DUALVAR, ok);
        for (char o : ok)
            if (!o) return HDSDP_RETCODE_FAILED;
        // every factor is in place: the log dets are read without a new factorisation
        for (ConeSlot &k : h->cones) {
            if (k.sdp) {
                double ld = 0.0;
                hdsdp_retcode r = k.sdp->get_barrier(tau, nullptr, which, &ld);
                if (r != HDSDP_RETCODE_OK) return r;
                *sum += ld;
            } else {
                *sum += k.lp->get_barrier(tau, y, which);
            }
        }
        return HDSDP_RETCODE_OK;
    }
    for (ConeSlot &k : h->cones) {
        if (k.sdp) {
            double ld = 0.0;
            hdsdp_retcode r = k.sdp->get_barrier(tau, y, which, &ld);
            if (r != HDSDP_RETCODE_OK) return r;
            *sum += ld;
        } else {
            *sum += k.lp->get_barrier(tau, y, which);
        }
    }
    return HDSDP_RETCODE_OK;
}

// HKKTBuildUp (interface/hdsdp_schur.c:256-268): clean, then every cone in order
hdsdp_retcode build_kkt(hdsdp *h, int type) {
    h->kkt.clean(type);
    if (batched_cones(h) && (type == KKT_TYPE_INFEASIBLE || type == KKT_TYPE_CORRECTOR)) {
        bool lp = false;
        for (ConeSlot &k : h->cones) lp = lp || (k.lp != nullptr);
        if (!lp) return h->kkt.add_sdp_batch(sdp_cones(h), type);
    }
    for (ConeSlot &k : h->cones) {
        if (k.sdp) {
            hdsdp_retcode r = h->kkt.add_sdp(*k.sdp, type);
            if (r != HDSDP_RETCODE_OK) return r;
        } else {
            h->kkt.add_lp(*k.lp, type);
        }
    }
    return HDSDP_RETCODE_OK;
}

hdsdp_retcode check_interior(hdsdp *h, double tau, const double *y, int *interior) {
    (void) tau;
    hdsdp_retcode r = cones_interior(h, 1.0, y, interior);
    if (r != HDSDP_RETCODE_OK) return r;
    if (!*interior) return HDSDP_RETCODE_OK;
    if (h->whichMethod != METHOD_HSD) *interior = h->bnd.interior_check(1.0, y);
    return HDSDP_RETCODE_OK;
}

int is_interior(hdsdp *h, const double *y) {
    int in = 0;
    check_interior(h, 1.0, y, &in);
    return in;
}

hdsdp_retcode get_log_barrier(hdsdp *h, double tau, const double *y, int which, double *val) {
    double ld = 0.0, bv = 0.0;
    hdsdp_retcode r = cones_barrier(h, tau, y, which, &ld);
    if (r != HDSDP_RETCODE_OK) return r;
    bv -= ld;
    if (h->whichMethod != METHOD_HSD) {
        r = h->bnd.get_barrier(tau, y, which, &ld);
        if (r != HDSDP_RETCODE_OK) return r;
        bv -= ld;
    }
    *val = bv;
    return HDSDP_RETCODE_OK;
}

void set_residual(hdsdp *h, double r) {
    for (ConeSlot &k : h->cones) {
        if (k.sdp) k.sdp->reduce_resi(r);
        else k.lp->reduce_resi(r);
    }
}

hdsdp_retcode kkt_solve(hdsdp *h, std::vector<double> &rhs, std::vector<double> *lhs) {
    return h->kkt.solve(rhs.data(), lhs ? lhs->data() : rhs.data());
}

// ---------------------------------------------------------------- Phase A': embedding
void hsd_build_step(hdsdp *h) {
    double dCSinvCSinv = h->kkt.dCSinvCSinv, dCSinv = h->kkt.dCSinv, dCSinvRd = h->kkt.dCSinvRdSinv;
    h->dtau = 0.0;
    const double old = h->dObjInternal;
    double bTy = 0.0;
    for (int i = 0; i < h->nRows; ++i) bTy += h->rowRHS[i] * h->y[i];
    h->dObjInternal = bTy;
    h->dObjImprove = bTy - old;
    std::vector<double> &dd1 = h->aux1;
    for (int i = 0; i < h->nRows; ++i) dd1[i] = h->rowRHS[i] - h->mu * h->kkt.asinvcs[i];
    double num = -bTy + h->mu / h->tau + h->mu * (dCSinv - dCSinvRd);
    double den = h->mu * dCSinvCSinv + h->mu / (h->tau * h->tau);
    const double tauOverMu = h->tau / h->mu;
    for (int i = 0; i < h->nRows; ++i) {
        num -= dd1[i] * (h->d1[i] * tauOverMu - h->d2[i] + h->d3[i]);
        den += dd1[i] * (h->d1[i] / h->mu + h->d4[i]);
    }
    h->dtau = (std::fabs(den) < 1e-12) ? 0.0 : num / den;
    for (int i = 0; i < h->nRows; ++i)
        h->dy[i] = h->d1[i] * (h->tau + h->dtau) / h->mu + h->d4[i] * h->dtau - h->d2[i] + h->d3[i];
}

hdsdp_retcode hsd_ratio_test(hdsdp *h, double *maxDist) {
    hdsdp_retcode retcode = HDSDP_RETCODE_OK;
    double mx = HDSDP_INFINITY, st = 0.0;
    st = h->tau / h->dtau;
    if (st < 0.0) mx = std::min(mx, -st);
    CALL(cones_ratio(h, h->dtau, h->dy.data(), 1.0, BUFFER_DUALVAR, &mx));
    if (h->whichMethod != METHOD_HSD) st = h->bnd.ratio_test(h->dtau, h->dy.data(), BUFFER_DUALVAR);
    if (mx < 1e-02) {
        h->nSmallStep += 1;
        if (h->nSmallStep > 2 && h->verbose) printf("HDSDP stagates at the cone boundary. \n");
    }
exit_cleanup:
    *maxDist = mx;
    return retcode;
}

hdsdp_retcode phaseA_hsd(hdsdp *h, int dOnly) {
    hdsdp_retcode retcode = HDSDP_RETCODE_OK;
    h->whichMethod = METHOD_HSD;
    const int maxIter = ip(h, INT_PARAM_MAXITER);
    const double gamma = dp(h, DBL_PARAM_HSDGAMMA);
    double absFeas = dp(h, DBL_PARAM_ABSFEASTOL), absOpt = dp(h, DBL_PARAM_ABSOPTTOL);
    double relFeas = dp(h, DBL_PARAM_RELFEASTOL), relOpt = dp(h, DBL_PARAM_RELOPTTOL);
    const double timeLimit = dp(h, DBL_PARAM_TIMELIMIT);
    const double objOne = fd(h, D_OBJONENORM), objScal = fd(h, D_OBJSCALING);
    const double nSum = (double) fi(h, N_SUMCONEDIMS);
    if (!dOnly) {
        absOpt = 1e+20;
        relOpt = 1e+20;
    }
    double feasTol = std::min(absFeas, relFeas * (1.0 + objOne)) * objScal / std::sqrt(nSum);
    absOpt = absOpt * 1e-04;
    relOpt = absOpt * 1e-04;
    if (h->HStatus == HDSDP_UNKNOWN) set_start(h, METHOD_HSD, dOnly);
    if (h->verbose) printf("HDSDP starts. Using self-dual method \n\n");
    while (true) {
        int interior = 0;
        CALL(cones_interior(h, h->tau, h->y.data(), &interior));
        if (!interior) {
            if (h->nIterCount == 0) {
                if (h->verbose) printf("Initial point is not in the cone. Adding slack value.\n");
                h->resi *= 100.0;
                reset_start(h);
                h->nIterCount += 1;
                continue;
            }
            if (h->verbose) printf("Iteration %d is not in the cone. \n", h->nIterCount);
            retcode = HDSDP_RETCODE_FAILED;
            goto exit_cleanup;
        }
        schur_precision(h);
        CALL(build_kkt(h, KKT_TYPE_HOMOGENEOUS));
        h->kkt.regularize(0.0);
        h->d2 = h->kkt.asinv;
        h->d3 = h->kkt.asinvrd;
        h->d4 = h->kkt.asinvcs;
        CALL(h->kkt.factorize());
        CALL(kkt_solve(h, h->rowRHS, &h->d1));
        CALL(kkt_solve(h, h->d2, nullptr));
        CALL(kkt_solve(h, h->d3, nullptr));
        CALL(kkt_solve(h, h->d4, nullptr));
        hsd_build_step(h);
        CALL(hsd_ratio_test(h, &h->dStep));
        if (h->dStep > 1.0) h->dStep = std::min(0.7 * h->dStep, 1.0);
        else if (h->dStep > 0.5) h->dStep = std::min(0.5 * h->dStep, 1.0);
        else if (h->dStep > 0.2) h->dStep = std::min(0.3 * h->dStep, 1.0);
        else h->dStep = std::min(0.2 * h->dStep, 1.0);
        print_log(h, METHOD_HSD);
        h->tau += h->dStep * h->dtau;
        for (int i = 0; i < h->nRows; ++i) h->y[i] += h->dStep * h->dy[i];
        h->resi = h->resi * (1.0 - h->dStep);
        set_residual(h, h->resi);
        double target = 0.0;
        if (h->mu > 1e-12) {
            if (h->dStep > 0.8 && h->tau > 1.0) {
                target = std::max(0.1 * h->mu, -0.1 * h->resi / h->tau);
                h->mu = std::min(h->mu, target);
            } else {
                target = std::max(gamma * h->mu, -0.1 * h->resi / h->tau);
                h->mu = std::min(h->mu, target);
            }
        } else {
            h->mu = std::min(h->mu, 0.8 * h->mu);
        }
        if (std::fabs(h->resi) < feasTol * h->tau && h->mu < absOpt &&
            (h->mu < relOpt * (1 + 2.0 * std::fabs(h->dObjVal)) &&
             std::fabs(h->dObjImprove) < 1e-05 * (std::fabs(h->dObjInternal) + 1.0))) {
            h->HStatus = dOnly ? HDSDP_DUAL_OPTIMAL : HDSDP_DUAL_FEASIBLE;
            break;
        }
        if (h->tau <= 1e-10) {
            h->HStatus = HDSDP_SUSPECT_INFEAS_OR_UNBOUNDED;
            break;
        }
        if (wall() - h->timeBegin >= timeLimit) {
            h->HStatus = HDSDP_TIMELIMIT;
            break;
        }
        h->nIterCount += 1;
        if (h->nIterCount >= maxIter) {
            h->HStatus = HDSDP_MAXITER;
            break;
        }
    }
exit_cleanup:
    if (retcode != HDSDP_RETCODE_OK) h->HStatus = HDSDP_NUMERICAL;
    return retcode;
}

// ---------------------------------------------------------------- Phase A: infeasible start
int prox_measure(hdsdp *h) {
    int isPFeasible = 0;
    const double dTraceSinv = h->kkt.dTraceSinv;
    double pObjNew = h->dObjInternal;
    const double pAcc = dp(h, DBL_PARAM_PRECORDACC);
    for (int i = 0; i < h->nRows; ++i) {
        h->aux1[i] = h->d1[i] / h->mu - h->d2[i];
        h->aux2[i] = h->rowRHS[i] / h->mu - h->kkt.asinv[i];
    }
    h->proxNorm = 0.0;
    for (int i = 0; i < h->nRows; ++i) h->proxNorm += h->aux1[i] * h->aux2[i];
    if (h->proxNorm < 0.0) {
        h->proxNorm = 1.0;
        return 0;
    }
    h->proxNorm = std::sqrt(h->proxNorm);
    for (int i = 0; i < h->nRows; ++i) h->aux2[i] = h->aux1[i] - h->y[i];
    isPFeasible = h->bnd.interior_check_expert(1.0, 1.0, h->aux2.data(), BUFFER_DUALCHECK);
    if (isPFeasible) {
        int in = 0;
        cones_interior_expert(h, 1.0, 1.0, h->aux2.data(), -h->resi, BUFFER_DUALCHECK, &in);
        isPFeasible = in;
    }
    if (isPFeasible) {
        double relGap = 0.0;
        if (h->whichMethod == METHOD_INFEAS) {
            for (int i = 0; i < h->nRows; ++i) relGap += h->aux1[i] * (h->kkt.asinvrd[i] + h->kkt.asinv[i]);
            relGap += dTraceSinv * h->resi;
        } else {
            for (int i = 0; i < h->nRows; ++i) relGap += h->aux1[i] * h->kkt.asinv[i];
        }
        relGap += h->allConeDims;
        pObjNew += relGap * h->mu;
        if (relGap < 0) {
            isPFeasible = (relGap < -1.0) ? -1 : 0;
        } else {
            h->pObjInternal = pObjNew;
            double inAcc = std::min(pAcc * 1000, 5e-03);
            inAcc = std::max(pAcc, 1e-04);
            h->bnd.get_primal(h->mu, h->y.data(), h->aux1.data(), h->pInfLow.data(), h->pInfUp.data());
            double pinf = 0.0;
            for (int i = 0; i < h->nRows; ++i) pinf = std::max(pinf, std::fabs(h->pInfUp[i] - h->pInfLow[i]));
            h->pInfeas = (pinf < 1e-16) ? 0.0 : pinf;
            if (pinf < 1.0) {
                if (relGap * h->mu > inAcc * (std::fabs(h->dObjInternal) + 1.0)) {
                    h->inaccMu = h->mu;
                    h->inaccY = h->y;
                    h->inaccDy = h->aux1;
                } else if (relGap * h->mu > pAcc * (std::fabs(h->dObjInternal) + 1.0)) {
                    h->accMu = h->mu;
                    h->accY = h->y;
                    h->accDy = h->aux1;
                }
            }
        }
    }
    return isPFeasible;
}

hdsdp_retcode phaseA_adaptive_resi(hdsdp *h, double *rate) {
    hdsdp_retcode retcode = HDSDP_RETCODE_OK;
    double alphaC = 0, alphaInf = 0, ada = 0, mx = HDSDP_INFINITY, st = 0;
    int interior = 0;
    for (int i = 0; i < h->nRows; ++i) h->aux1[i] = -h->d2[i];
    CALL(cones_ratio(h, 0.0, h->aux1.data(), 0.0, BUFFER_DUALVAR, &mx));
    st = h->bnd.ratio_test(0.0, h->aux1.data(), BUFFER_DUALVAR);
    mx = std::min(mx, st);
    alphaC = std::min(0.98 * mx, 1.0);
    mx = alphaC;
    while (!interior && alphaC > 1e-02 * mx) {
        CALL(cones_add_step(h, alphaC, BUFFER_DUALCHECK, &interior));
        // the bound-cone result replaces the cones' result here, as in the reference
        interior = h->bnd.add_step_and_check(alphaC, BUFFER_DUALCHECK);
        if (!interior) alphaC *= 0.8;
    }
    mx = HDSDP_INFINITY;
    CALL(cones_ratio(h, 0.0, h->d3.data(), 1.0, BUFFER_DUALCHECK, &mx));
    alphaInf = mx;
    ada = alphaInf / alphaC;
    ada = std::min(0.98 * ada, 1.0);
    if (h->proxNorm < 1.0) ada = std::max(0.9, ada);
    else if (h->proxNorm < 10.0) ada = std::max(0.3, ada);
    else if (h->proxNorm < 50.0) ada = std::max(0.1, ada);
    *rate = ada;
exit_cleanup:
    return retcode;
}

void infeasible_build_step(hdsdp *h, double ada) {
    for (int i = 0; i < h->nRows; ++i) h->dy[i] = h->d1[i] / h->mu - h->d2[i] + ada * h->d3[i];
}

hdsdp_retcode ratio_test_all(hdsdp *h, double ada, double *maxDist) {
    hdsdp_retcode retcode = HDSDP_RETCODE_OK;
    double mx = HDSDP_INFINITY, st = 0.0;
    CALL(cones_ratio(h, 0.0, h->dy.data(), ada, BUFFER_DUALVAR, &mx));
    st = h->bnd.ratio_test(0.0, h->dy.data(), BUFFER_DUALVAR);
    mx = std::min(mx, st);
exit_cleanup:
    *maxDist = mx;
    return retcode;
}

hdsdp_retcode infeasible_corrector(hdsdp *h) {
    hdsdp_retcode retcode = HDSDP_RETCODE_OK;
    const int nMaxCorr = ip(h, INT_PARAM_CORRECTORA);
    int interior = is_interior(h, h->y.data());
    double barrier = 0, newBarrier = 0, mx = 0, st = 0, alphaC = 0, alphaInf = 0, ada = 0, adaMax = 0.8;
    if (!interior) {
        retcode = HDSDP_RETCODE_FAILED;
        goto exit_cleanup;
    }
    CALL(get_log_barrier(h, 0.0, nullptr, BUFFER_DUALVAR, &barrier));
    for (int nCorr = 0; nCorr < nMaxCorr; ++nCorr) {
        if (!h->resi) break;
        CALL(build_kkt(h, KKT_TYPE_CORRECTOR));
        h->kkt.add_bound(h->bnd, KKT_TYPE_CORRECTOR);
        h->d2 = h->kkt.asinv;
        h->d3 = h->kkt.asinvrd;
        CALL(kkt_solve(h, h->d2, nullptr));
        if (adaMax) CALL(kkt_solve(h, h->d3, nullptr));
        for (int i = 0; i < h->nRows; ++i) h->dy[i] = -h->d2[i];
        ratio_test_all(h, 0.0, &mx);
        mx = std::min(0.8 * mx, 1.0);
        while (true) {
            for (int i = 0; i < h->nRows; ++i) h->aux1[i] = h->y[i] + mx * h->dy[i];
            interior = is_interior(h, h->aux1.data());
            if (!interior) mx *= 0.5;
            if (interior || mx < 5e-03) break;
        }
        if (mx < 5e-03) {
            interior = is_interior(h, h->y.data());
            break;
        }
        CALL(get_log_barrier(h, 0.0, nullptr, BUFFER_DUALVAR, &newBarrier));
        if (newBarrier > barrier) {
            mx *= 0.5;
            for (int i = 0; i < h->nRows; ++i) h->aux1[i] = h->y[i] + mx * h->dy[i];
            interior = is_interior(h, h->aux1.data());
            barrier = -HDSDP_INFINITY;
        }
        alphaC = mx;
        mx = HDSDP_INFINITY;
        CALL(cones_ratio(h, 0.0, h->d3.data(), 1.0, BUFFER_DUALVAR, &mx));
        st = h->bnd.ratio_test(0.0, h->d3.data(), BUFFER_DUALVAR);
        mx = std::min(mx, st);
        alphaInf = mx;
        ada = alphaInf / alphaC;
        ada = std::min(1.0, adaMax * ada);
        {
            const double r0 = h->resi;
            for (int iTry = 0;; ++iTry) {
                h->resi = r0 * (1 - alphaC * ada);
                set_residual(h, r0 * (1 - alphaC * ada));
                for (int i = 0; i < h->nRows; ++i) h->aux1[i] = h->y[i] + alphaC * (ada * h->d3[i] - h->d2[i]);
                interior = is_interior(h, h->aux1.data());
                if (interior) break;
                ada *= 0.8;
                if (iTry > 2000) {  // the reference loops until interior; bound the host loop
                    retcode = HDSDP_RETCODE_FAILED;
                    goto exit_cleanup;
                }
            }
        }
        if (alphaC * ada < 5e-04) adaMax = 0.0;
        else if (alphaC * ada < 0.1) adaMax = adaMax * 0.9;
        if (alphaC * ada > 0.8) {
            h->mu *= 0.8;
            adaMax = std::min(adaMax * 2.0, 0.9);
        } else if (alphaC * ada > 0.3) {
            h->mu *= 0.95;
            adaMax = std::min(adaMax * 2.0, 0.8);
        }
        h->y = h->aux1;
        if (adaMax == 0.0) break;
        barrier = newBarrier;
    }
exit_cleanup:
    return retcode;
}

hdsdp_retcode phaseA_infeasible(hdsdp *h, int dOnly) {
    (void) dOnly;
    hdsdp_retcode retcode = HDSDP_RETCODE_OK;
    h->whichMethod = METHOD_INFEAS;
    const int maxIter = ip(h, INT_PARAM_MAXITER);
    int allowReset = 1;
    if (fi(h, I_MANYCONES) || fi(h, I_IMPTRACE) || fi(h, I_VERYDENSE)) allowReset = 0;
    const double absFeas = dp(h, DBL_PARAM_ABSFEASTOL), relFeas = dp(h, DBL_PARAM_RELFEASTOL);
    const double timeLimit = dp(h, DBL_PARAM_TIMELIMIT);
    const double nSum = (double) fi(h, N_SUMCONEDIMS);
    const double objScal = fd(h, D_OBJSCALING), objOne = fd(h, D_OBJONENORM);
    double feasTol = std::max(absFeas, relFeas * (1 + objOne)) * objScal / std::sqrt(nSum);
    double ada = 0.0;
    int interior = 0, pObjFound = 0, pObjType = 0;
    set_start(h, METHOD_INFEAS, 0);
    CALL(cones_interior(h, h->tau, h->y.data(), &interior));
    if (interior) interior = h->bnd.interior_check(h->tau, h->y.data());
    if (!interior) {
        if (h->verbose) printf("Initial point is not in the cone. Adding slack value.\n");
        reset_start(h);
    }
    if (h->verbose) printf("HDSDP starts. Using infeasible dual method \n\n");
    while (true) {
        if (h->nIterCount == 3 && !pObjFound && allowReset) {
            if (h->verbose) printf("Increasing dual infeasibility \n");
            reset_start(h);
            CALL(cones_interior(h, h->tau, h->y.data(), &interior));
            if (!interior) {
                retcode = HDSDP_RETCODE_FAILED;
                goto exit_cleanup;
            }
        }
        schur_precision(h);
        CALL(build_kkt(h, KKT_TYPE_INFEASIBLE));
        h->kkt.add_bound(h->bnd, KKT_TYPE_INFEASIBLE);
        h->d2 = h->kkt.asinv;
        h->d3 = h->kkt.asinvrd;
        CALL(h->kkt.factorize());
        CALL(kkt_solve(h, h->rowRHS, &h->d1));
        CALL(kkt_solve(h, h->d2, nullptr));
        CALL(kkt_solve(h, h->d3, nullptr));
        pObjType = prox_measure(h);
        if (pObjType < 0) h->HStatus = HDSDP_SUSPECT_INFEAS_OR_UNBOUNDED;
        else pObjFound += pObjType;
        if (pObjType == 1 && h->proxNorm < 2.0) h->mu *= 0.7;
        {
            double target = h->pObjInternal - h->dObjInternal;
            target = target - h->resi * dp(h, DBL_PARAM_TRXESTIMATE);
            target = target / (5.0 * h->allConeDims);
            if (h->proxNorm < 1.0) h->mu = h->mu * 0.005;
            else if (h->proxNorm < 5.0) h->mu = std::max(h->mu * 0.01, target * 0.1);
            else if (h->proxNorm < 10.0) h->mu = std::max(h->mu * 0.1, target * 0.8);
            else h->mu = std::max(h->mu * 0.95, target);
        }
        CALL(phaseA_adaptive_resi(h, &ada));
        infeasible_build_step(h, ada);
        CALL(ratio_test_all(h, ada, &h->dStep));
        h->dStep = std::min(0.95 * h->dStep, 1.0);
        if (h->dStep < 1e-03) h->nSmallStep += 1;
        for (int i = 0; i < h->nRows; ++i) h->y[i] += h->dStep * h->dy[i];
        h->resi = h->resi * (1.0 - ada * h->dStep);
        set_residual(h, h->resi);
        CALL(infeasible_corrector(h));
        print_log(h, METHOD_INFEAS);
        if (std::fabs(h->resi) < feasTol) {
            h->HStatus = HDSDP_DUAL_FEASIBLE;
            break;
        }
        if (h->nSmallStep > 3) {
            h->HStatus = HDSDP_SUSPECT_INFEAS_OR_UNBOUNDED;
            break;
        }
        if (h->HStatus == HDSDP_SUSPECT_INFEAS_OR_UNBOUNDED) break;
        if (wall() - h->timeBegin >= timeLimit) {
            h->HStatus = HDSDP_TIMELIMIT;
            break;
        }
        h->nIterCount += 1;
        if (h->nIterCount >= maxIter) {
            h->HStatus = HDSDP_MAXITER;
            break;
        }
    }
exit_cleanup:
    return retcode;
}

// ---------------------------------------------------------------- Phase B: potential reduction
hdsdp_retcode phaseB_choose_barrier(hdsdp *h, int pObjType) {
    hdsdp_retcode retcode = HDSDP_RETCODE_OK;
    const double rho = dp(h, DBL_PARAM_POTRHOVAL);
    const double absGap = h->pObjInternal - h->dObjInternal;
    const double upper = absGap / h->allConeDims, lower = upper / rho;
    double mx = HDSDP_INFINITY, pst = 0.0, st = 0.0;
    if (pObjType > 0) {
        for (int i = 0; i < h->nRows; ++i) h->aux1[i] = -h->d1[i] / h->mu;
        CALL(cones_ratio(h, 0.0, h->aux1.data(), 0.0, BUFFER_DUALCHECK, &mx));
        st = h->bnd.ratio_test(0.0, h->aux1.data(), BUFFER_DUALCHECK);
        mx = std::min(mx, st);
        mx = std::min(mx * 0.97, 1e+05);
        h->mu = h->mu / (1.0 + mx);
    } else {
        for (int i = 0; i < h->nRows; ++i) h->aux2[i] = -h->d1[i] / h->mu + h->d2[i];
        CALL(cones_ratio(h, 0.0, h->aux2.data(), 0.0, BUFFER_DUALVAR, &mx));
        st = h->bnd.ratio_test(0.0, h->aux2.data(), BUFFER_DUALVAR);
        pst = std::min(mx, st);
        if (pst < 1.0) pst = 0.97 * pst;
        int interior = 0;
        for (int iTry = 0;; ++iTry) {
            CALL(cones_add_step(h, pst, BUFFER_DUALCHECK, &interior));
            interior = h->bnd.add_step_and_check(pst, BUFFER_DUALCHECK);
            if (!interior) pst = (iTry > 2) ? pst * 0.97 : pst * 0.5;
            else break;
            if (pst < 1e-05) {
                retcode = HDSDP_RETCODE_FAILED;
                goto exit_cleanup;
            }
        }
        for (int i = 0; i < h->nRows; ++i) h->aux1[i] = -pst * h->d1[i] / h->mu;
        CALL(cones_ratio(h, 0.0, h->aux1.data(), 0.0, BUFFER_DUALCHECK, &mx));
        st = h->bnd.ratio_test(0.0, h->aux1.data(), BUFFER_DUALCHECK);
        mx = std::min(mx, st);
        mx = std::min(mx * 0.97, 1e+05);
        h->mu = pst * h->mu / (1.0 + mx) + (1.0 - pst) * (h->pObjInternal - h->dObjInternal) / h->allConeDims;
    }
    h->mu = std::max(h->mu, lower);
    h->mu = std::min(h->mu, upper);
exit_cleanup:
    return retcode;
}

void feasible_build_step(hdsdp *h) {
    for (int depth = 0; depth < 64; ++depth) {
        for (int i = 0; i < h->nRows; ++i) h->dy[i] = h->d1[i] / h->mu - h->d2[i];
        double prox = 0.0;
        for (int i = 0; i < h->nRows; ++i) {
            h->aux1[i] = h->rowRHS[i] / h->mu - h->kkt.asinv[i];
            prox += h->aux1[i] * h->dy[i];
        }
        if (prox < 0.0) {
            h->proxNorm = 1e+02;
            return;
        }
        prox = std::sqrt(prox);
        h->proxNorm = prox;
        if (prox < 0.1) {
            h->mu = 0.1 * h->mu;
            continue;
        }
        return;
    }
}

double get_potential(hdsdp *h, double rho, const double *y, int which) {
    double pot = 0.0, obj = 0.0, ld = 0.0;
    cones_barrier(h, 0.0, nullptr, which, &ld);
    pot -= ld;
    h->bnd.get_barrier(0.0, nullptr, which, &ld);
    pot -= ld;
    for (int i = 0; i < h->nRows; ++i) obj += h->rowRHS[i] * y[i];
    pot += rho * std::log(h->pObjInternal - obj);
    return pot;
}

hdsdp_retcode reduce_potential(hdsdp *h) {
    hdsdp_retcode retcode = HDSDP_RETCODE_OK;
    double mx = 0.0, step = 0.0, now = 0.0, nw = 0.0, req = 0.0, minTol = 0.0;
    const double rho = (h->pObjVal - h->dObjVal) / h->mu;
    int interior = 0;
    if (h->nSmallStep >= 2) minTol = 0.5;
    if (h->proxNorm < 0.5) req = 0.05;
    CALL(ratio_test_all(h, 0.0, &mx));
    step = std::min(mx * 0.95, 1.0);
    now = get_potential(h, rho, h->y.data(), BUFFER_DUALVAR);
    for (int iTry = 0;; ++iTry) {
        for (int i = 0; i < h->nRows; ++i) h->aux1[i] = h->y[i] + step * h->dy[i];
        interior = is_interior(h, h->aux1.data());
        if (!interior) {
            step *= 0.33;
            if (iTry > 10000) {
                retcode = HDSDP_RETCODE_FAILED;
                goto exit_cleanup;
            }
            continue;
        }
        nw = get_potential(h, rho, h->aux1.data(), BUFFER_DUALVAR);
        if (nw <= now - req || step * h->proxNorm <= 0.001 || step < minTol) {
            h->y = h->aux1;
            break;
        }
        if (step < 1e-04) {
            interior = is_interior(h, h->y.data());
            if (!interior) retcode = HDSDP_RETCODE_FAILED;
            break;
        }
        step *= 0.3;
    }
    h->dStep = step;
    h->potentialVal = nw;
exit_cleanup:
    return retcode;
}

double get_barrier_val(hdsdp *h, const double *y, int which) {
    double bv = 0.0, obj = 0.0, ld = 0.0;
    cones_barrier(h, 0.0, nullptr, which, &ld);
    bv += ld;
    h->bnd.get_barrier(0.0, nullptr, which, &ld);
    bv += ld;
    for (int i = 0; i < h->nRows; ++i) obj += h->rowRHS[i] * y[i];
    bv = obj + h->mu * bv;
    return -bv;
}

hdsdp_retcode feasible_corrector(hdsdp *h) {
    hdsdp_retcode retcode = HDSDP_RETCODE_OK;
    const double shrink = h->allConeDims / (h->allConeDims + std::sqrt(h->allConeDims));
    int nMaxCorr = ip(h, INT_PARAM_CORRECTORB);
    if (nMaxCorr == 0) return retcode;
    if (h->proxNorm < 0.1) nMaxCorr = 0;
    if (h->dStep < 1e-02) nMaxCorr = 0;
    if (h->dStep < 0.1 && h->mu < 1e-05) {
        nMaxCorr = 0;
        ip(h, INT_PARAM_CORRECTORB) = 0;
    }
    if (h->dStep < 1e-03) {
        nMaxCorr = 0;
        ip(h, INT_PARAM_CORRECTORB) = 0;
    }
    if (h->mu < 1e-06) {
        nMaxCorr = 0;
        ip(h, INT_PARAM_CORRECTORB) = 0;
    }
    double bNow = 0, bNew = 0, bDotD1 = 0, bDotD2 = 0, bDotCorr = 0;
    for (int i = 0; i < h->nRows; ++i) bDotD1 += h->d1[i] * h->rowRHS[i];
    for (int nCorr = 0; nCorr < nMaxCorr; ++nCorr) {
        if (h->mu < 1e-05) break;
        CALL(build_kkt(h, KKT_TYPE_CORRECTOR));
        h->kkt.add_bound(h->bnd, KKT_TYPE_CORRECTOR);
        h->d2 = h->kkt.asinv;
        CALL(kkt_solve(h, h->d2, nullptr));
        bDotD2 = 0.0;
        for (int i = 0; i < h->nRows; ++i) bDotD2 += h->rowRHS[i] * h->d2[i];
        if (bDotD2 > 0 && bDotD1 > 0) h->mu = bDotD1 / bDotD2;
        h->mu *= shrink;
        for (int i = 0; i < h->nRows; ++i) {
            h->aux1[i] = h->d1[i] / h->mu - h->d2[i];
            bDotCorr += h->rowRHS[i] * h->aux1[i];
        }
        double mx = HDSDP_INFINITY, st = 0.0;
        bNow = get_barrier_val(h, h->y.data(), BUFFER_DUALVAR);
        CALL(cones_ratio(h, 0.0, h->aux1.data(), 0.0, BUFFER_DUALVAR, &mx));
        st = h->bnd.ratio_test(0.0, h->aux1.data(), BUFFER_DUALVAR);
        mx = std::min(mx, st);
        mx = std::min(mx * 0.95, mx);
        mx = std::min(mx, dp(h, DBL_PARAM_POTRHOVAL) / h->proxNorm);
        for (int iTry = 0;; ++iTry) {
            for (int i = 0; i < h->nRows; ++i) h->aux2[i] = h->y[i] + mx * h->aux1[i];
            int interior = is_interior(h, h->aux2.data());
            if (!interior) {
                mx *= 0.5;
                if (iTry > 10000) {
                    retcode = HDSDP_RETCODE_FAILED;
                    goto exit_cleanup;
                }
                continue;
            }
            bNew = get_barrier_val(h, h->aux2.data(), BUFFER_DUALVAR);
            if (mx < 1e-04 || bNew <= bNow - std::fabs(0.05 * bDotCorr * mx)) break;
            const double t = 2 * (bNew - bNow + bDotCorr * mx) / (mx * mx);
            if ((bDotCorr / t < mx) && (bDotCorr / t > 0)) mx = bDotCorr / t;
            else mx *= 0.5;
        }
        if (mx < 1e-04) {
            is_interior(h, h->y.data());
            break;
        }
        h->y = h->aux2;
    }
exit_cleanup:
    return retcode;
}

int phaseB_ray_check(hdsdp *h, int force) {
    int ray = 0, interior = 0;
    if (h->pInfeas >= fd(h, D_RHSFRONORM) || force ||
        (h->pInfeas > 0.01 * fd(h, D_RHSONENORM) && h->mu < 1e-03)) {
        if (h->dObjVal < 0.0) return 0;
        double nrm = 0.0;
        for (int i = 0; i < h->nRows; ++i) nrm += h->y[i] * h->y[i];
        nrm = std::sqrt(nrm);
        for (int i = 0; i < h->nRows; ++i) h->aux1[i] = h->y[i] / nrm;
        cones_interior_expert(h, 0.0, -1.0, h->aux1.data(), 1e-08, BUFFER_DUALCHECK, &interior);
        if (interior) ray = 1;
    }
    return ray;
}

hdsdp_retcode run_psdp(hdsdp *h);

hdsdp_retcode phaseB_potential(hdsdp *h) {
    hdsdp_retcode retcode = HDSDP_RETCODE_OK;
    h->whichMethod = METHOD_POTENTIAL;
    const int maxIter = ip(h, INT_PARAM_MAXITER);
    const int primalMethod = ip(h, INT_PARAM_PSDP);
    const double absFeas = dp(h, DBL_PARAM_ABSFEASTOL), absOpt = dp(h, DBL_PARAM_ABSOPTTOL);
    const double relFeas = dp(h, DBL_PARAM_RELFEASTOL), relOpt = dp(h, DBL_PARAM_RELOPTTOL);
    const double timeLimit = dp(h, DBL_PARAM_TIMELIMIT);
    const double objOne = fd(h, D_OBJONENORM), objScal = fd(h, D_OBJSCALING), rhsScal = fd(h, D_RHSSCALING);
    const double nSum = (double) fi(h, N_SUMCONEDIMS);
    const double pdScal = objScal * rhsScal;
    int nIterInternal = 0;
    double feasTol = std::min(absFeas, relFeas * (1.0 + objOne)) * objScal / std::sqrt(nSum);
    int pObjType = 0, pObjFound = 0, noPObj = 0, ray = 0, force = 1;
    double pObjStart = 0.0;
    // HDSDP_PhaseB_Initialize
    if (h->tau != 1.0 || h->HStatus != HDSDP_DUAL_FEASIBLE) {
        h->resi = h->resi / h->tau;
        for (int i = 0; i < h->nRows; ++i) h->y[i] /= h->tau;
        if (!is_interior(h, h->y.data()) && h->verbose) printf("Incumbent dual solution is infeasible \n");
        h->HStatus = HDSDP_INTERNAL_ERROR;
        retcode = HDSDP_RETCODE_FAILED;
        goto exit_cleanup;
    }
    if (std::fabs(h->resi) > feasTol && h->verbose)
        printf("Dual infeasibility from previous algorithm exceeds user-specified tolerance \n");
    h->perturb = -10.0 * h->resi;
    h->resi = 0.0;
    set_residual(h, 0.0);
    for (ConeSlot &k : h->cones) {
        if (k.sdp) k.sdp->set_perturb(h->perturb);
        else k.lp->set_perturb(h->perturb);
    }
    if (h->perturb != 0.0) is_interior(h, h->y.data());
    pObjStart = h->pObjInternal;
    if (h->verbose) printf("HDSDP re-starts. Using feasible dual method \n\n");
    while (true) {
        nIterInternal += 1;
        if (nIterInternal > 10) force = 0;
        schur_precision(h);
        CALL(build_kkt(h, KKT_TYPE_INFEASIBLE));
        h->kkt.add_bound(h->bnd, KKT_TYPE_INFEASIBLE);
        if (h->mu > 1.0) h->kkt.regularize(1e-06);
        h->d2 = h->kkt.asinv;
        h->d3 = h->kkt.asinvrd;
        CALL(h->kkt.factorize());
        CALL(kkt_solve(h, h->rowRHS, &h->d1));
        CALL(kkt_solve(h, h->d2, nullptr));
        pObjType = prox_measure(h);
        if (pObjType < 0) {
            h->HStatus = HDSDP_SUSPECT_INFEAS_OR_UNBOUNDED;
        } else {
            pObjFound += pObjType;
            if (pObjType) noPObj = 0;
            else noPObj += 1;
        }
        CALL(phaseB_choose_barrier(h, pObjType));
        feasible_build_step(h);
        ray = phaseB_ray_check(h, force);
        if (ray) {
            if (h->verbose) printf("HDSDP detects a dual improving ray \n");
            h->HStatus = HDSDP_INFEAS_OR_UNBOUNDED;
            break;
        }
        CALL(reduce_potential(h));
        if (h->dStep < 1e-03) h->nSmallStep += 1;
        CALL(feasible_corrector(h));
        print_log(h, METHOD_POTENTIAL);
        if (h->comp < (std::fabs(h->pObjVal) + std::fabs(h->dObjVal) + 1.0) * relOpt && h->comp < absOpt / pdScal) {
            h->HStatus = HDSDP_PRIMAL_DUAL_OPTIMAL;
            break;
        }
        if (h->comp < (std::fabs(h->pObjVal) + std::fabs(h->dObjVal) + 1.0) * 0.1 && primalMethod) {
            retcode = run_psdp(h);
            break;
        }
        if (h->nSmallStep > 3) {
            h->HStatus = HDSDP_NUMERICAL;
            break;
        }
        if (h->HStatus == HDSDP_SUSPECT_INFEAS_OR_UNBOUNDED) break;
        if (wall() - h->timeBegin >= timeLimit) {
            h->HStatus = HDSDP_TIMELIMIT;
            break;
        }
        h->nIterCount += 1;
        if (h->nIterCount >= maxIter) {
            h->HStatus = HDSDP_MAXITER;
            break;
        }
        if (noPObj >= 10 && h->pObjInternal != pObjStart) {
            h->HStatus = HDSDP_NUMERICAL;
            break;
        }
    }
exit_cleanup:
    return retcode;
}

// ---------------------------------------------------------------- primal values
// The primal marker (mu, y, dy) of HDSDPGetConeValues (interface/hdsdp.c:711-745): the
// accurate one when it exists, else the inaccurate one.
void primal_marker(hdsdp *h, double &mu, const std::vector<double> *&y, const std::vector<double> *&dy) {
    mu = h->accMu;
    y = &h->accY;
    dy = &h->accDy;
    if (mu <= 0.0) {
        mu = h->inaccMu;
        y = &h->inaccY;
        dy = &h->inaccDy;
    }
}

// X and S of an SDP cone (device, leading dimension c.ld)
void sdp_values(hdsdp *h, SdpCone &c, double *X, double *S) {
    double mu;
    const std::vector<double> *y, *dy;
    primal_marker(h, mu, y, dy);
    if (X) c.get_primal(mu, y->data(), dy->data(), X);
    if (S) c.get_dual(S);
}

// x and s of an LP cone (host vectors of its dimension)
void lp_values(hdsdp *h, LpCone &lp, double *x, double *sl) {
    double mu;
    const std::vector<double> *y, *dy;
    primal_marker(h, mu, y, dy);
    if (x) lp.get_primal(mu, y->data(), dy->data(), x);
    if (sl) lp.get_dual(sl);
}

// ---------------------------------------------------------------- primal refinement
hdsdp_retcode run_psdp(hdsdp *h) {
    hdsdp_retcode retcode = HDSDP_RETCODE_OK;
    SdpCone &c = *h->cone;
    const int n = c.n, m = h->nRows;
    const long ld = c.ld;
    cudaStream_t s = c.s;
    double *X = nullptr, *X0 = nullptr, *S = nullptr, *XStep = nullptr, *Buf = nullptr;
    DenseFactor XF;
    Lanczos lzp;
    std::vector<double> pinf(m), rhs(m);
    double mu = h->mu;
    const double relOpt = dp(h, DBL_PARAM_RELOPTTOL), absOpt = dp(h, DBL_PARAM_ABSOPTTOL);
    const double pdScal = fd(h, D_OBJSCALING) * fd(h, D_RHSSCALING);
    // HPSDPInit (interface/hdsdp_psdp.c:81-90): one dense SDP cone, dual feasible
    if (h->nCones > 1 || h->dInfeas > 0.0 || h->cones[0].type != HDSDP_CONETYPE_DENSE_SDP) return HDSDP_RETCODE_FAILED;
    for (double **p : {&X, &X0, &S, &XStep, &Buf}) HB_CUDA(hb::cmalloc(p, sizeof(double) * ld * n));
    XF.alloc(n);
    lzp.init(n, s);
    sdp_values(h, c, X, nullptr);
    HB_CUDA(cudaMemcpyAsync(X0, X, sizeof(double) * ld * n, cudaMemcpyDeviceToDevice, s));
    h->kkt.primalX = X;
    if (h->verbose) printf("Primal solver is initialized. \n");
    CALL(h->kkt.build(c, KKT_TYPE_PRIMAL));
    CALL(h->kkt.factorize());
    for (int it = 0; it < 5; ++it) {
        std::fill(pinf.begin(), pinf.end(), 0.0);
        c.atimesx(X, pinf.data());
        double pinfNorm = 0.0;
        for (int i = 0; i < m; ++i) {
            const double t = h->rowRHS[i] - pinf[i];
            pinfNorm += t * t;
        }
        pinfNorm = std::sqrt(pinfNorm);
        c.get_dual(S);
        // Buf = X S X
        gemm(s, n, n, n, 1.0, S, ld, 0, X, ld, 0, 0.0, XStep, ld, 0);
        gemm(s, n, n, n, 1.0, X, ld, 0, XStep, ld, 0, 0.0, Buf, ld, 0);
        symmetrize_avg(s, n, Buf, ld);
        std::fill(rhs.begin(), rhs.end(), 0.0);
        c.atimesx(Buf, rhs.data());
        for (int i = 0; i < m; ++i) rhs[i] -= mu * pinf[i];
        CALL(h->kkt.solve(rhs.data(), h->dy.data()));
        double dualStep = 0.0;
        CALL(c.ratio_test(0.0, h->dy.data(), 1.0, BUFFER_DUALVAR, &dualStep));
        // Buf += X0 dS X0
        gemm(s, n, n, n, 1.0, c.dS, ld, 0, X0, ld, 0, 0.0, XStep, ld, 0);
        gemm(s, n, n, n, 1.0, X0, ld, 0, XStep, ld, 0, 1.0, Buf, ld, 0);
        // XStep = X - Buf / mu
        copy_matrix(s, n, n, X, ld, XStep, ld);
        axpy(s, (int) (ld * n), -1.0 / mu, Buf, XStep);
        if (it == 0) {
            if (!factorize(s, XF, X, ld)) {
                retcode = HDSDP_RETCODE_FAILED;
                goto exit_cleanup;
            }
        }
        double primalStep = 0.0;
        CALL(lzp.solve(XF, XStep, ld, &primalStep, &h->timers));
        primalStep = std::min(0.95 * primalStep, 1.0);
        dualStep = std::min(0.95 * dualStep, 1.0);
        axpy(s, (int) (ld * n), primalStep, XStep, X);
        for (int i = 0; i < m; ++i) h->y[i] += dualStep * h->dy[i];
        c.update(1.0, h->y.data());
        int interior = 0;
        CALL(c.interior_check(1.0, h->y.data(), &interior));
        if (!interior) {
            retcode = HDSDP_RETCODE_FAILED;
            goto exit_cleanup;
        }
        if (!factorize(s, XF, X, ld)) {
            retcode = HDSDP_RETCODE_FAILED;
            goto exit_cleanup;
        }
        double dualObj = 0.0;
        for (int i = 0; i < m; ++i) dualObj += h->rowRHS[i] * h->y[i];
        const double primalObj = c.trace_cx(X);
        frob_dot(s, n, X, ld, S, ld, c.d_scal);
        HB_CUDA(cudaMemcpyAsync(c.h_scal, c.d_scal, sizeof(double), cudaMemcpyDeviceToHost, s));
        HB_CUDA(cudaStreamSynchronize(s));
        const double compl_ = c.h_scal[0] / n;
        mu = std::min(mu, compl_ / (5.0 * n));
        h->pObjVal = primalObj;
        h->dObjVal = dualObj;
        h->pInfeas = pinfNorm;
        h->mu = mu;
        h->dStep = dualStep;
        const double elapsed = wall() - h->timeBegin;
        h->nIterCount += 1;
        h->log.push_back({elapsed, primalObj, dualObj, mu,
                          (primalObj - dualObj) / (std::fabs(primalObj) + std::fabs(dualObj) + 1.0), 3});
        if (h->verbose)
            printf("    %5d  %+15.8e  %+15.8e  %8.2e  %8.2e  %5.2f %5.2f     %4.1f \n", h->nIterCount + 1, primalObj,
                   dualObj, pinfNorm, mu, primalStep, dualStep, elapsed);
        if (h->comp < (std::fabs(h->pObjVal) + std::fabs(h->dObjVal) + 1.0) * relOpt && h->comp < absOpt / pdScal)
            break;
    }
exit_cleanup:
    h->kkt.primalX = nullptr;
    for (double *p : {X, X0, S, XStep, Buf})
        if (p) hb::cache_free(p);
    XF.release();
    lzp.release();
    return retcode;
}

hdsdp_retcode conic_solve(hdsdp *h, int dOnly) {
    hdsdp_retcode retcode = HDSDP_RETCODE_OK;
    CALL(phaseA_infeasible(h, dOnly));
    if (h->HStatus == HDSDP_SUSPECT_INFEAS_OR_UNBOUNDED) {
        if (h->verbose) printf("\nInfeasible method stops due to suspected infeasibility \n");
        CALL(phaseA_hsd(h, dOnly));
    } else if (h->HStatus == HDSDP_DUAL_FEASIBLE) {
        if (h->verbose) printf("\nInfeasible method finds a dual feasible solution \n");
        CALL(phaseB_potential(h));
    }
exit_cleanup:
    return retcode;
}

// Smallest eigenvalue sign test of X: Cholesky succeeds -> lambda_min > 0; otherwise the
// most negative eigenvalue is bracketed by bisection on X + sigma I.
// lambda_min(X) for the DIMACS check (the reference calls dsyevr, interface/hdsdp.c:833): 1 if
// X is positive definite, else -t for the smallest shift t with X + t I positive definite,
// found by Cholesky attempts: a geometric search up from 1e-14 max|X_ii| by factors of 16,
// then a geometric bisection to 1e-3 relative (at most about 25 factorisations; a
// shift below 1e-14 max|X_ii| is reported as that bound).
double min_eig_estimate(SdpCone &c, double *X) {
    DenseFactor &F = c.Fcheck;
    c.invalidate_check_factor();
    if (factorize(c.s, F, X, c.ld)) return 1.0;
    const int n = c.n;
    double *T = c.dev.T1;
    double *dgd = c.dev.T2;   // n x ld scratch, free during the check
    copy_matrix(c.s, 1, n, X, c.ld + 1, dgd, 1);
    std::vector<double> dg(n);
    HB_CUDA(cudaMemcpyAsync(dg.data(), dgd, sizeof(double) * n, cudaMemcpyDeviceToHost, c.s));
    HB_CUDA(cudaStreamSynchronize(c.s));
    double scale = 1.0;
    for (double v : dg) scale = std::max(scale, std::fabs(v));
    auto pd_at = [&](double t) {
        copy_matrix(c.s, n, n, X, c.ld, T, c.ld);
        add_diag(c.s, n, T, c.ld, t);
        return factorize(c.s, F, T, c.ld);
    };
    double lo = 0.0, hi = 1e-14 * scale;
    for (int it = 0; it < 40 && !pd_at(hi); ++it) {
        lo = hi;
        hi *= 16.0;
    }
    for (int it = 0; it < 40 && lo > 0.0 && hi > lo * (1.0 + 1e-3); ++it) {
        const double mid = std::sqrt(lo * hi);
        if (pd_at(mid)) hi = mid;
        else lo = mid;
    }
    return (lo > 0.0) ? -0.5 * (lo + hi) : -hi;
}

void release_cones(hdsdp *h) {
    if (h->d_yall) hb::cache_free(h->d_yall);
    if (h->h_yall) hb::cache_free_host(h->h_yall);
    h->d_yall = h->h_yall = nullptr;
    for (ConeSlot &k : h->cones) {
        if (k.sdp) {
            k.sdp->release();
            delete k.sdp;
            k.sdp = nullptr;
        }
        if (k.lp) {
            k.lp->release();
            delete k.lp;
            k.lp = nullptr;
        }
    }
    h->cone = nullptr;
}

}  // namespace

// =====================================================================================
// Public C API
// =====================================================================================
extern "C" {

hdsdp_retcode HUserDataCreate(user_data **pHdata) {
    if (!pHdata) return HDSDP_RETCODE_FAILED;
    user_data *u = (user_data *) calloc(1, sizeof(user_data));
    if (!u) return HDSDP_RETCODE_MEMORY;
    *pHdata = u;
    return HDSDP_RETCODE_OK;
}

void HUserDataSetConeData(user_data *Hdata, cone_type cone, int nRow, int nCol, int *coneMatBeg, int *coneMatIdx,
                          double *coneMatElem) {
    Hdata->cone = cone;
    Hdata->nConicRow = nRow;
    Hdata->nConicCol = nCol;
    Hdata->coneMatBeg = coneMatBeg;
    Hdata->coneMatIdx = coneMatIdx;
    Hdata->coneMatElem = coneMatElem;
}

cone_type HUserDataChooseCone(user_data *Hdata) {
    if (Hdata->cone == HDSDP_CONETYPE_SOCP || Hdata->cone == HDSDP_CONETYPE_BOUND || Hdata->cone == HDSDP_CONETYPE_LP ||
        Hdata->cone == HDSDP_CONETYPE_SPARSE_SDP || Hdata->cone == HDSDP_CONETYPE_SCALAR_BOUND)
        return Hdata->cone;
    if (Hdata->cone == HDSDP_CONETYPE_DENSE_SDP) {
        int nz = 0;
        for (int i = 0; i < Hdata->nConicRow; ++i)
            if (Hdata->coneMatBeg[i + 2] - Hdata->coneMatBeg[i + 1] > 0) nz += 1;
        return (nz > HDSDP_SPARSE_CONE_THRESHOLD * Hdata->nConicRow) ? HDSDP_CONETYPE_DENSE_SDP
                                                                     : HDSDP_CONETYPE_SPARSE_SDP;
    }
    return HDSDP_CONETYPE_UNKNOWN;
}

void HUserDataClear(user_data *Hdata) {
    if (Hdata) memset(Hdata, 0, sizeof(user_data));
}

void HUserDataDestroy(user_data **pHdata) {
    if (!pHdata) return;
    HUserDataClear(*pHdata);
    free(*pHdata);
    *pHdata = nullptr;
}

hdsdp_retcode HDSDPCreate(hdsdp **pHSolver) {
    if (!pHSolver) return HDSDP_RETCODE_FAILED;
    hdsdp *h = new (std::nothrow) hdsdp();
    if (!h) return HDSDP_RETCODE_MEMORY;
    int dev = 0;
    if (cudaGetDeviceCount(&dev) != cudaSuccess || dev == 0) {
        fprintf(stderr, "[hdsdp_b200] no CUDA device available: this library has no CPU path\n");
        delete h;
        return HDSDP_RETCODE_FAILED;
    }
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete h;
        return HDSDP_RETCODE_FAILED;
    }
    const char *v = getenv("HDSDP_B200_VERBOSE");
    h->verbose = v ? atoi(v) : 0;
    *pHSolver = h;
    return HDSDP_RETCODE_OK;
}

hdsdp_retcode HDSDPInit(hdsdp *h, int nRows, int nCones) {
    if (nRows < 1 || nCones < 1) return HDSDP_RETCODE_FAILED;
    release_cones(h);
    h->nRows = nRows;
    h->nCones = nCones;
    h->cones.assign(nCones, ConeSlot());
    default_params(h);
    h->rowRHS.assign(nRows, 0.0);
    for (auto *v : {&h->y, &h->dy, &h->d1, &h->d2, &h->d3, &h->d4, &h->aux1, &h->aux2, &h->pInfUp, &h->pInfLow,
                    &h->accY, &h->accDy, &h->inaccY, &h->inaccDy})
        v->assign(nRows, 0.0);
    h->mu = 1e+10;
    h->comp = HDSDP_INFINITY;
    h->accMu = -1.0;
    h->inaccMu = -1.0;
    h->HStatus = HDSDP_UNKNOWN;
    return HDSDP_RETCODE_OK;
}

hdsdp_retcode HDSDPSetCone(hdsdp *h, int iCone, void *userCone) {
    user_data *u = (user_data *) userCone;
    if (!u || iCone < 0 || iCone >= h->nCones || (int) h->cones.size() != h->nCones) return HDSDP_RETCODE_FAILED;
    // HConeSetData (interface/hdsdp_conic.c:50-60) takes the type HUserDataChooseCone picks
    const cone_type t = HUserDataChooseCone(u);
    if (t != HDSDP_CONETYPE_DENSE_SDP && t != HDSDP_CONETYPE_SPARSE_SDP && t != HDSDP_CONETYPE_LP) {
        fprintf(stderr, "[hdsdp_b200] cone %d: type %d is not supported (SDP blocks and LP cones are)\n", iCone,
                (int) t);
        return HDSDP_RETCODE_FAILED;
    }
    h->cones[iCone].usr = u;
    h->cones[iCone].type = t;
    return HDSDP_RETCODE_OK;
}

void HDSDPSetDualObjective(hdsdp *h, double *dObj) {
    std::copy(dObj, dObj + h->nRows, h->rowRHS.begin());
}

void HDSDPSetIntParam(hdsdp *h, int p, int v) {
    if (p >= 3 || p < 0) return;
    h->HIntParams[p] = v;
}

void HDSDPSetDblParam(hdsdp *h, int p, double v) {
    if (p >= 13 || p < 0) return;
    h->HDblParams[p] = v;
}

hdsdp_retcode HDSDPCheckSolution(hdsdp *h, double dErrs[6]) {
    for (int i = 0; i < 6; ++i) dErrs[i] = 1.0;
    if (h->inaccMu < 0.0 && h->accMu < 0.0) {
        h->HStatus = HDSDP_NUMERICAL;
        return HDSDP_RETCODE_OK;
    }
    const int m = h->nRows;
    double dualInfeas = h->perturb * std::sqrt((double) fi(h, N_SUMCONEDIMS));
    double primalObj = 0.0, dualObj = 0.0, compl_ = 0.0, minEig = HDSDP_INFINITY;
    const double pScal = fd(h, D_RHSSCALING), dScal = fd(h, D_OBJSCALING);
    for (int i = 0; i < m; ++i) dualObj += h->rowRHS[i] * h->y[i];
    std::vector<double> ax(m, 0.0);
    // per cone: A X into the residual, <X, S>, <C, X>, and lambda_min(X) (min x for an LP cone)
    for (ConeSlot &k : h->cones) {
        if (k.sdp) {
            SdpCone &c = *k.sdp;
            const int n = c.n;
            const long ld = c.ld;
            double *X = nullptr, *S = nullptr;
            HB_CUDA(hb::cmalloc(&X, sizeof(double) * ld * n));
            HB_CUDA(hb::cmalloc(&S, sizeof(double) * ld * n));
            HB_CUDA(cudaMemsetAsync(X, 0, sizeof(double) * ld * n, c.s));
            sdp_values(h, c, X, S);
            c.atimesx(X, ax.data());
            frob_dot(c.s, n, X, ld, S, ld, c.d_scal);
            HB_CUDA(cudaMemcpyAsync(c.h_scal, c.d_scal, sizeof(double), cudaMemcpyDeviceToHost, c.s));
            HB_CUDA(cudaStreamSynchronize(c.s));
            compl_ += c.h_scal[0];
            primalObj += c.trace_cx(X);
            minEig = std::min(minEig, min_eig_estimate(c, X));
            hb::cache_free(X);
            hb::cache_free(S);
        } else {
            LpCone &lp = *k.lp;
            std::vector<double> xl(lp.nCol, 0.0), sl(lp.nCol, 0.0);
            lp_values(h, lp, xl.data(), sl.data());
            lp.atimesx(xl.data(), ax.data());
            double d = 0.0;
            for (int q = 0; q < lp.nCol; ++q) d += xl[q] * sl[q];
            compl_ += d;
            primalObj += lp.trace_cx(xl.data());
            double mn = HDSDP_INFINITY;
            for (double v : xl) mn = std::min(mn, v);
            minEig = std::min(minEig, mn);
        }
    }
    dualObj /= (pScal * dScal);
    primalObj /= (pScal * dScal);
    double pinf = 0.0;
    for (int i = 0; i < m; ++i) {
        ax[i] -= h->rowRHS[i];
        pinf += ax[i] * ax[i];
    }
    pinf = std::sqrt(pinf) / fd(h, D_RHSSCALING);
    dualInfeas = dualInfeas / fd(h, D_OBJSCALING);
    dErrs[0] = pinf / (1.0 + fd(h, D_RHSONENORM));
    dErrs[1] = (minEig < 0.0) ? -minEig / (1.0 + fd(h, D_RHSONENORM)) : 0.0;
    dErrs[2] = dualInfeas / (1.0 + fd(h, D_OBJONENORM));
    dErrs[3] = 0.0;
    dErrs[4] = (primalObj - dualObj) / (std::fabs(primalObj) + std::fabs(dualObj) + 1.0);
    dErrs[5] = compl_ / (std::fabs(primalObj) + std::fabs(dualObj) + 1.0);
    double mx = 0.0;
    for (int i = 0; i < 6; ++i) mx = std::max(mx, std::fabs(dErrs[i]));
    h->pObjVal = primalObj;
    h->dObjVal = dualObj;
    if (mx > 1e-02) {
        if (h->accMu < 0.0) h->HStatus = HDSDP_NUMERICAL;
        else {
            if (h->verbose) printf("\nDealing with primal solution\n");
            h->accMu = -1.0;
            return HDSDPCheckSolution(h, dErrs);
        }
    } else {
        h->HStatus = HDSDP_PRIMAL_DUAL_OPTIMAL;
    }
    return device_error_flag() ? HDSDP_RETCODE_FAILED : HDSDP_RETCODE_OK;
}

hdsdp_retcode HDSDPOptimize(hdsdp *h, int dOptOnly) {
    hdsdp_retcode retcode = HDSDP_RETCODE_OK;
    double tp0 = 0.0, tp1 = 0.0, tp2 = 0.0;
    h->timeBegin = wall();
    h->timers = Timers();
    h->log.clear();
    adjoint_release(h->adj);
    {
        // every cone set, at least one of them an SDP block
        int nSdp = 0;
        if ((int) h->cones.size() != h->nCones) return HDSDP_RETCODE_FAILED;
        for (ConeSlot &k : h->cones) {
            if (!k.usr) return HDSDP_RETCODE_FAILED;
            if (k.type != HDSDP_CONETYPE_LP) nSdp += 1;
        }
        if (nSdp == 0) {
            fprintf(stderr, "[hdsdp_b200] the problem has no SDP cone\n");
            return HDSDP_RETCODE_FAILED;
        }
    }
    release_cones(h);
    h->kkt.release();
    tp0 = wall();
    // HConeProcData + HConePresolveData per cone in order (interface/hdsdp.c:630-633)
    for (ConeSlot &k : h->cones) {
        const user_data *u = k.usr;
        if (u->nConicRow != h->nRows) {
            retcode = HDSDP_RETCODE_FAILED;
            goto exit_cleanup;
        }
        if (k.type == HDSDP_CONETYPE_LP) {
            k.lp = new LpCone();
            CALL(k.lp->proc_data(u->nConicRow, u->nConicCol, u->coneMatBeg, u->coneMatIdx, u->coneMatElem, h->stream));
        } else {
            k.sdp = new SdpCone();
            k.sdp->precision = h->precision;
            k.sdp->sparseMode = h->sparseSlack;
            CALL(k.sdp->proc_data(u->nConicRow, u->nConicCol, u->coneMatBeg, u->coneMatIdx, u->coneMatElem,
                                  k.type == HDSDP_CONETYPE_SPARSE_SDP));
            if (k.sdp->m == 0) {
                fprintf(stderr, "[hdsdp_b200] an SDP block has no constraint\n");
                retcode = HDSDP_RETCODE_FAILED;
                goto exit_cleanup;
            }
            tp1 = wall();
            CALL(k.sdp->presolve());
            tp2 += wall() - tp1;
            if (!h->cone) h->cone = k.sdp;
        }
    }
    tp1 = wall();
    get_statistics(h);
    adjust_params(h);
    h->bnd.proc(h->nRows, dp(h, DBL_PARAM_DUALBOX_LOW), dp(h, DBL_PARAM_DUALBOX_UP));
    for (ConeSlot &k : h->cones)
        if (k.sdp) CALL(k.sdp->setup_device(h->stream, &h->timers));
    if (h->verbose) {
        double up = 0.0, upMap = 0.0;
        for (ConeSlot &k : h->cones)
            if (k.sdp) {
                up += k.sdp->dev.t_upload_total;
                upMap += k.sdp->dev.t_upload_map;
            }
        printf("  set-up: data %.3f s (rank-one detection %.3f s), device upload %.3f s (coefficients %.3f s, "
               "of which gather map %.3f s)\n",
               tp1 - tp0, tp2, wall() - tp1, up, upMap);
    }
    {
        // the block-arrow Schur complement when every cone is a sparse SDP cone (the
        // reference's sparse KKT, interface/hdsdp_schur.c:224-246)
        std::vector<SdpCone *> sp;
        bool allSparse = true;
        for (ConeSlot &k : h->cones) {
            if (k.sdp && k.sdp->sparse) sp.push_back(k.sdp);
            else allSparse = false;
        }
        // the vector of the batched cone updates (several SDP cones)
        if (batched_cones(h)) {
            HB_CUDA(hb::cmalloc(&h->d_yall, sizeof(double) * std::max(h->nRows, 1)));
            HB_CUDA(hb::cmalloc_host(&h->h_yall, sizeof(double) * std::max(h->nRows, 1)));
        }
        // (an LDL^T factorisation asked for applies to the dense M)
        const bool useArrow = allSparse && h->schurLdl != 1 && arrow_chosen(h->sparseSchur, h->nRows, sp);
        h->kkt.init(h->nRows, h->stream, &h->timers, !useArrow);
        h->kkt.ldlMode = h->schurLdl;
        if (useArrow && !h->kkt.setup_arrow(sp)) {
            retcode = HDSDP_RETCODE_MEMORY;
            goto exit_cleanup;
        }
        if (h->verbose && useArrow) {
            double info[6];
            h->kkt.arrow_info(info);
            printf("  Schur complement: block arrow, %d cones (largest local block %d), %d coupling rows\n",
                   (int) info[2], (int) info[3], (int) info[1]);
        }
    }
    if (device_error_flag()) {
        retcode = HDSDP_RETCODE_MEMORY;
        goto exit_cleanup;
    }
    if (h->verbose) {
        printf("  Correctors A %d B %d  dual box [%g, %g]  %s", ip(h, INT_PARAM_CORRECTORA),
               ip(h, INT_PARAM_CORRECTORB), h->bnd.lo, h->bnd.up, h->modelFeatures.c_str());
        printf("\n");
    }
    {
        // Iterations run on the solver stream with the data resident: time them with events there.
        cudaEvent_t ev0, ev1;
        HB_CUDA(cudaEventCreate(&ev0));
        HB_CUDA(cudaEventCreate(&ev1));
        h->timers.setup = wall() - h->timeBegin;
        HB_CUDA(cudaEventRecord(ev0, h->stream));
        retcode = conic_solve(h, dOptOnly);
        if (h->HStatus != HDSDP_INFEAS_OR_UNBOUNDED && h->HStatus != HDSDP_SUSPECT_INFEAS_OR_UNBOUNDED)
            retcode = HDSDPCheckSolution(h, h->dErrs);
        HB_CUDA(cudaEventRecord(ev1, h->stream));
        HB_CUDA(cudaEventSynchronize(ev1));
        float ms = 0.f;
        HB_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
        h->timers.ipm_device = 1e-3 * ms;
        cudaEventDestroy(ev0);
        cudaEventDestroy(ev1);
    }
    h->optimized = true;
    if (h->verbose)
        printf("DIMACS error metric:\n    %5.2e %5.2e %5.2e %5.2e %5.2e %5.2e \n", h->dErrs[0], h->dErrs[1],
               h->dErrs[2], h->dErrs[3], h->dErrs[4], h->dErrs[5]);
exit_cleanup:
    h->timers.total = wall() - h->timeBegin;
    return retcode;
}

hdsdp_retcode HDSDPGetRowDual(hdsdp *h, double *pObjVal, double *dObjVal, double *dualVal) {
    if (pObjVal) *pObjVal = h->pObjVal;
    if (dObjVal) *dObjVal = h->dObjVal;
    if (dualVal) std::copy(h->y.begin(), h->y.end(), dualVal);
    return HDSDP_RETCODE_OK;
}

void HDSDPGetConeValues(hdsdp *h, int iCone, double *conePrimal, double *coneDual, double *coneAuxi) {
    (void) coneAuxi;
    if (!h || iCone < 0 || iCone >= (int) h->cones.size()) return;
    ConeSlot &k = h->cones[iCone];
    if (k.lp) {
        lp_values(h, *k.lp, conePrimal, coneDual);  // x and s of the LP cone
        return;
    }
    if (!k.sdp) return;
    SdpCone &c = *k.sdp;
    const int n = c.n;
    const long ld = c.ld;
    double *X = nullptr, *S = nullptr;
    if (conePrimal) HB_CUDA(hb::cmalloc(&X, sizeof(double) * ld * n));
    if (coneDual) HB_CUDA(hb::cmalloc(&S, sizeof(double) * ld * n));
    if (X) {
        HB_CUDA(cudaMemcpy2DAsync(X, sizeof(double) * ld, conePrimal, sizeof(double) * n, sizeof(double) * n, n,
                                  cudaMemcpyHostToDevice, c.s));
    }
    sdp_values(h, c, X, S);
    if (X)
        HB_CUDA(cudaMemcpy2DAsync(conePrimal, sizeof(double) * n, X, sizeof(double) * ld, sizeof(double) * n, n,
                                  cudaMemcpyDeviceToHost, c.s));
    if (S)
        HB_CUDA(cudaMemcpy2DAsync(coneDual, sizeof(double) * n, S, sizeof(double) * ld, sizeof(double) * n, n,
                                  cudaMemcpyDeviceToHost, c.s));
    HB_CUDA(cudaStreamSynchronize(c.s));
    if (X) hb::cache_free(X);
    if (S) hb::cache_free(S);
}

void HDSDPClear(hdsdp *h) {
    if (!h) return;
    adjoint_release(h->adj);
    release_cones(h);
    h->kkt.release();
}

void HDSDPDestroy(hdsdp **pHSolver) {
    if (!pHSolver || !*pHSolver) return;
    hdsdp *h = *pHSolver;
    HDSDPClear(h);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    *pHSolver = nullptr;
}

}  // extern "C"

// ---- accessors used by the extension API (ext.cu) ----
namespace hb {
int solver_status(hdsdp *h) { return (int) h->HStatus; }
int solver_iters(hdsdp *h) { return h->nIterCount; }
void solver_set_psdp(hdsdp *h, int on) { h->HIntParams[INT_PARAM_PSDP] = on; }
void solver_cone_values(hdsdp *h, double *X, double *S) {
    if (h->cone) sdp_values(h, *h->cone, X, S);
}
double solver_obj_scal(hdsdp *h) { return fd(h, D_OBJSCALING); }
double solver_rhs_scal(hdsdp *h) { return fd(h, D_RHSSCALING); }
}  // namespace hb
