/*
 * Probes into the reference HDSDP solver, compiled together with the
 * unmodified reference sources into oracle/_ref/libhdsdp_ref.so.
 *
 * TEST INFRASTRUCTURE ONLY: used by tests/ (golden-vector generation and
 * parity checks) and by bench.py's reference/CPU-baseline arm.
 *
 * The reference API has no getter for the solver status or the iteration
 * count (interface/hdsdp.h:105-116), so these read the internal solver
 * struct (interface/def_hdsdp.h:57-136). The Schur / ratio-test probes drive
 * the reference's own cone and KKT layers the way tests/test_file_io.c:21-170
 * does, and copy out the assembled Schur complement
 * (interface/def_hdsdp_schur.h:32-68).
 */
#include <string.h>
#include "def_hdsdp.h"
#include "hdsdp_conic.h"
#include "hdsdp_schur.h"
#include "def_hdsdp_schur.h"
#include "def_hdsdp_user_data.h"

int oracle_status(hdsdp *h) { return (int) h->HStatus; }
int oracle_iters(hdsdp *h) { return h->nIterCount; }
double oracle_perturb(hdsdp *h) { return h->dPerturb; }
double oracle_mu(hdsdp *h) { return h->dBarrierMu; }
int oracle_int_param(hdsdp *h, int i) { return h->HIntParams[i]; }
/* Parameters the public setter refuses (index >= 3, interface/hdsdp.c:596-604),
   e.g. INT_PARAM_PSDP = 4 to run dual potential reduction without refinement. */
void oracle_set_int_param(hdsdp *h, int i, int v) { h->HIntParams[i] = v; }
double oracle_dbl_param(hdsdp *h, int i) { return h->HDblParams[i]; }
int oracle_int_feature(hdsdp *h, int i) { return h->HIntFeatures[i]; }
double oracle_dbl_feature(hdsdp *h, int i) { return h->HDblFeatures[i]; }

/*
 * Assemble the Schur complement of one SDP block at dual point (y, resi):
 * S = C - sum_i y_i A_i - resi * I, then M_ij = <A_i, S^-1 A_j S^-1>,
 * ASinv_i = <A_i, S^-1>, ASinvRdSinv_i = resi * <A_i, S^-2>, trace(S^-1).
 * typeKKT follows interface/hdsdp_conic.h:16-19 (0 = INFEASIBLE).
 * M is returned as the full lower triangle, column-major m x m.
 * Returns 0 on success, 1 if S is not positive definite, -1 on error.
 */
int oracle_schur_probe(int m, int n, int *Ap, int *Ai, double *Ax, double *y, double resi,
                       int typeKKT, double *Mout, double *asinv, double *asinvrd, double *asinvcs,
                       double *scal3) {
    hdsdp_retcode retcode = HDSDP_RETCODE_OK;
    hdsdp_cone *cone = NULL;
    hdsdp_kkt *kkt = NULL;
    user_data ud;
    int isInterior = 0;
    int ret = -1;

    ud.cone = HDSDP_CONETYPE_DENSE_SDP;
    ud.nConicRow = m;
    ud.nConicCol = n;
    ud.coneMatBeg = Ap;
    ud.coneMatIdx = Ai;
    ud.coneMatElem = Ax;

    HDSDP_CALL(HConeCreate(&cone));
    HDSDP_CALL(HConeSetData(cone, &ud));
    HDSDP_CALL(HConeProcData(cone));
    HDSDP_CALL(HConePresolveData(cone));
    HConeSetStart(cone, resi);
    HDSDP_CALL(HConeCheckIsInterior(cone, 1.0, y, &isInterior));
    if (!isInterior) { ret = 1; goto exit_cleanup; }

    HDSDP_CALL(HKKTCreate(&kkt));
    HDSDP_CALL(HKKTInit(kkt, m, 1, &cone));
    HDSDP_CALL(HKKTBuildUp(kkt, typeKKT));
    if (Mout && kkt->kktMatElem && !kkt->isKKTSparse) {
        for (int j = 0; j < m; ++j)
            for (int i = j; i < m; ++i)
                Mout[(size_t) j * m + i] = kkt->kktMatElem[(size_t) j * m + i];
    }
    memcpy(asinv, kkt->dASinvVec, sizeof(double) * m);
    memcpy(asinvrd, kkt->dASinvRdSinvVec, sizeof(double) * m);
    if (asinvcs) memcpy(asinvcs, kkt->dASinvCSinvVec, sizeof(double) * m);
    if (scal3) {
        scal3[0] = kkt->dCSinv;
        scal3[1] = kkt->dCSinvCSinv;
        scal3[2] = kkt->dCSinvRdSinv;
        scal3[3] = kkt->dTraceSinv;
    }
    ret = 0;

exit_cleanup:
    if (kkt) HKKTDestroy(&kkt);
    if (cone) HConeDestroy(&cone);
    (void) retcode;
    return ret;
}

/*
 * First ratio test of a fresh SDP block (interface/hdsdp_conic_sdp.c:1638-1682):
 * S = C - A^T y - resi I, dS = -A^T dy + ada * resi * I, returns the step
 * bound from the reference Lanczos (linalg/hdsdp_lanczos.c:161-292) and the
 * log-determinant of S. Returns 0 on success, 1 if S is not interior.
 */
int oracle_ratio_probe(int m, int n, int *Ap, int *Ai, double *Ax, double *y, double resi,
                       double *dy, double ada, double *step, double *logdet) {
    hdsdp_retcode retcode = HDSDP_RETCODE_OK;
    hdsdp_cone *cone = NULL;
    user_data ud;
    int isInterior = 0;
    int ret = -1;

    ud.cone = HDSDP_CONETYPE_DENSE_SDP;
    ud.nConicRow = m;
    ud.nConicCol = n;
    ud.coneMatBeg = Ap;
    ud.coneMatIdx = Ai;
    ud.coneMatElem = Ax;

    HDSDP_CALL(HConeCreate(&cone));
    HDSDP_CALL(HConeSetData(cone, &ud));
    HDSDP_CALL(HConeProcData(cone));
    HDSDP_CALL(HConePresolveData(cone));
    HConeSetStart(cone, resi);
    HDSDP_CALL(HConeCheckIsInterior(cone, 1.0, y, &isInterior));
    if (!isInterior) { ret = 1; goto exit_cleanup; }
    HDSDP_CALL(HConeGetLogBarrier(cone, 0.0, NULL, BUFFER_DUALVAR, logdet));
    HDSDP_CALL(HConeRatioTest(cone, 0.0, dy, ada, BUFFER_DUALVAR, step));
    ret = 0;

exit_cleanup:
    if (cone) HConeDestroy(&cone);
    (void) retcode;
    return ret;
}

/*
 * The dense Schur complement a KKT object holds after HKKTBuildUp (the lower
 * triangle of kktMatElem, interface/def_hdsdp_schur.h:42-80), copied into the
 * column-major m x m array Mout. Returns 0, or -1 for a sparse Schur complement.
 */
int oracle_kkt_matrix(hdsdp_kkt *kkt, int m, double *Mout) {
    if (!kkt || kkt->isKKTSparse || !kkt->kktMatElem) return -1;
    for (int j = 0; j < m; ++j)
        for (int i = j; i < m; ++i)
            Mout[(size_t) j * m + i] = kkt->kktMatElem[(size_t) j * m + i];
    return 0;
}
