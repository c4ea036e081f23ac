/*
 * hdsdp_conic.h -- the conic callback interface and the KKT (Schur complement)
 * manager, drop-in for the reference's interface/def_hdsdp_conic.h:56-104 (the
 * hdsdp_cone function table), interface/hdsdp_conic.h (HCone* dispatch) and
 * interface/hdsdp_schur.h:10-21 (HKKT*).
 *
 * A host that drives the interior-point iteration itself calls the cones through
 * this table exactly as the reference's algorithm does (interface/hdsdp_algo.c):
 * HConeSetData binds the implementation chosen by HUserDataChooseCone, and every
 * hook keeps the reference's argument meaning and buffer semantics
 * (BUFFER_DUALVAR: S and its factor; BUFFER_DUALCHECK: a trial S and its factor;
 * BUFFER_DUALSTEP: dS). In this library the SDP cones' matrices (S, dS, S^-1, the
 * factors) and the Schur matrix M stay in GPU memory: the hooks take and return
 * host scalars and m-vectors, and n x n host arrays only where the reference's
 * hooks do (primal and dual recovery, A X, <C, X>).
 *
 * The Schur matrix is built by coneBuildSchur into an hdsdp_kkt made by HKKTCreate
 * and HKKTInit; its right-hand-side vectors and scalars are read with HKKTExport
 * (the reference's callers read the same fields from the struct). HKKTGetMatrix
 * copies M to the host (no reference counterpart: the reference's M is host memory).
 *
 * All cones and KKT objects made through this interface on one device share one
 * CUDA stream of the library; like the reference's, the interface is not reentrant.
 */
#ifndef HDSDP_B200_CONIC_H
#define HDSDP_B200_CONIC_H

#include <stdint.h>
#include "hdsdp.h"
#include "hdsdp_user_data.h"

/* interface/hdsdp_conic.h:16-30 */
#define KKT_TYPE_INFEASIBLE  (0)
#define KKT_TYPE_CORRECTOR   (1)
#define KKT_TYPE_HOMOGENEOUS (2)
#define KKT_TYPE_PRIMAL      (3)

#define ABS_NORM    (1)
#define FRO_NORM    (2)

#define BUFFER_DUALVAR   (0)
#define BUFFER_DUALCHECK (1)
#define BUFFER_DUALSTEP  (2)

/* interface/def_hdsdp_conic.h:56-104: the same members in the same order. */
typedef struct {

    cone_type cone;

    void  *usrData;
    void  *coneData;

    hdsdp_retcode (*coneCreate)    ( void ** );
    hdsdp_retcode (*coneProcData)    ( void *, int, int, int *, int *, double * );
    hdsdp_retcode (*conePresolveData) ( void * );
    void          (*coneDestroyData) ( void ** );

    void   (*coneSetStart)    ( void *, double );
    void   (*coneUpdate)      ( void *, double, double * );
    hdsdp_retcode (*coneRatioTest)   ( void *, double, double *, double, int, double * );

    int64_t (*coneGetSymNnz)   ( void * );
    int     (*coneGetDim)      ( void * );
    void    (*coneAddSymNz)    ( void *, int, int * );
    void    (*coneGetKKTMap)   ( void *, int, int * );
    hdsdp_retcode (*coneBuildSchur)  ( void *, void *, int );
    hdsdp_retcode (*coneBuildSchurFixed) ( void *, void *, int, int );

    hdsdp_retcode (*coneInteriorCheck) ( void *, double, double *, int * );
    hdsdp_retcode (*coneInteriorCheckExpert) ( void *, double, double, double *, double, int, int *);
    hdsdp_retcode (*coneGetBarrier)  ( void *, double, double *, int, double * );
    hdsdp_retcode (*coneAxpyBufferAndCheck) ( void *, double, int, int * );
    void    (*coneReduceResi)  ( void *, double );
    void    (*coneSetPerturb)  ( void *, double );
    void    (*conePRecover)    ( void *, double, double *, double *, double *, double *);
    void    (*coneDRecover)    ( void *, double *, double * );
    void    (*coneATimesX)     ( void *, double *, double * );
    double  (*coneTraceCX)     ( void *, double * );

    double  (*coneGetCoeffNorm) ( void *, int );
    double  (*coneGetObjNorm)  ( void *, int );
    void    (*coneScal)        ( void *, double );

    void    (*coneView)        ( void * );

    void    (*getstat)         ( void *, double *, int [20], double [20] );

} hdsdp_cone;

/* The Schur complement system (interface/def_hdsdp_schur.h:42-80); opaque here. */
typedef struct hdsdp_kkt_internal hdsdp_kkt;

#ifdef __cplusplus
extern "C" {
#endif

/* interface/hdsdp_conic.c:23  HConeCreate */
extern hdsdp_retcode HConeCreate( hdsdp_cone **pHCone );
/* interface/hdsdp_conic.c:38  HConeGetVarBufferDim */
extern int HConeGetVarBufferDim( hdsdp_cone *HCone );
/* interface/hdsdp_conic.c:50  HConeSetData: binds the dense SDP, sparse SDP, LP or
   scalar bound implementation (HUserDataChooseCone) */
extern hdsdp_retcode HConeSetData( hdsdp_cone *HCone, user_data *usrData );
/* interface/hdsdp_conic.c:221  HConeProcData */
extern hdsdp_retcode HConeProcData( hdsdp_cone *HCone );
/* interface/hdsdp_conic.c:235  HConePresolveData */
extern hdsdp_retcode HConePresolveData( hdsdp_cone *HCone );
/* interface/hdsdp_conic.c:190  HConeClear */
extern void HConeClear( hdsdp_cone *HCone );
/* interface/hdsdp_conic.c:202  HConeDestroy */
extern void HConeDestroy( hdsdp_cone **pHCone );
/* interface/hdsdp_conic.c:214  HConeView */
extern void HConeView( hdsdp_cone *HCone );
/* interface/hdsdp_conic.c:402  HConeDetectFeature */
extern void HConeDetectFeature( hdsdp_cone *HCone, double *rowRHS, int coneIntFeatures[20], double coneDblFeatures[20] );
/* interface/hdsdp_conic.c:246  HConeSetStart */
extern void HConeSetStart( hdsdp_cone *HCone, double dConeStartVal );
/* interface/hdsdp_conic.c:252  HConeUpdate */
extern void HConeUpdate( hdsdp_cone *HCone, double barHsdTau, double *rowDual );
/* interface/hdsdp_conic.c:258  HConeRatioTest */
extern hdsdp_retcode HConeRatioTest( hdsdp_cone *HCone, double barHsdTauStep, double *rowDualStep, double dAdaRatio,
                                     int whichBuffer, double *maxStep );
/* interface/hdsdp_conic.c:264  HConeGetSymNnz */
extern int64_t HConeGetSymNnz( hdsdp_cone *HCone );
/* interface/hdsdp_conic.c:269  HConeAddSymNz */
extern void HConeAddSymNz( hdsdp_cone *HCone, int iCol, int *schurMatCol );
/* interface/hdsdp_conic.c:275  HConeGetSymMapping */
extern void HConeGetSymMapping( hdsdp_cone *HCone, int iCol, int *schurMatCol );
/* interface/hdsdp_conic.c:281  HConeGetDim */
extern int HConeGetDim( hdsdp_cone *HCone );
/* interface/hdsdp_conic.c:286  HConeGetCoeffNorm */
extern double HConeGetCoeffNorm( hdsdp_cone *HCone, int whichNorm );
/* interface/hdsdp_conic.c:291  HConeGetObjNorm */
extern double HConeGetObjNorm( hdsdp_cone *HCone, int whichNorm );
/* interface/hdsdp_conic.c:296  HConeBuildSchurComplement (schurMat is an hdsdp_kkt *) */
extern hdsdp_retcode HConeBuildSchurComplement( hdsdp_cone *HCone, void *schurMat, int typeKKT );
/* interface/hdsdp_conic.c:318  HConeBuildSchurComplementFixed */
extern hdsdp_retcode HConeBuildSchurComplementFixed( hdsdp_cone *HCone, void *schurMat, int typeKKT, int kktStrategy );
/* interface/hdsdp_conic.c:324  HConeGetLogBarrier */
extern hdsdp_retcode HConeGetLogBarrier( hdsdp_cone *HCone, double barHsdTau, double *rowDual, int whichBuffer,
                                         double *logdet );
/* interface/hdsdp_conic.c:333  HConeAddStepToBufferAndCheck */
extern hdsdp_retcode HConeAddStepToBufferAndCheck( hdsdp_cone *HCone, double dStep, int whichBuffer, int *isInterior );
/* interface/hdsdp_conic.c:342  HConeCheckIsInterior */
extern hdsdp_retcode HConeCheckIsInterior( hdsdp_cone *HCone, double barHsdTau, double *rowDual, int *isInterior );
/* interface/hdsdp_conic.c:351  HConeCheckIsInteriorExpert */
extern hdsdp_retcode HConeCheckIsInteriorExpert( hdsdp_cone *HCone, double dCCoef, double dACoefScal, double *dACoef,
                                                 double dEyeCoef, int whichBuffer, int *isInterior );
/* interface/hdsdp_conic.c:360  HConeReduceResi */
extern void HConeReduceResi( hdsdp_cone *HCone, double resiReduction );
/* interface/hdsdp_conic.c:366  HConeSetPerturb */
extern void HConeSetPerturb( hdsdp_cone *HCone, double dPerturb );
/* interface/hdsdp_conic.c:372  HConeGetPrimal */
extern void HConeGetPrimal( hdsdp_cone *HCone, double dBarrierMu, double *dRowDual, double *dRowDualStep,
                            double *dConePrimal, double *dConePrimal2 );
/* interface/hdsdp_conic.c:378  HConeGetDual */
extern void HConeGetDual( hdsdp_cone *HCone, double *dConeDual, double *dConeDual2 );
/* interface/hdsdp_conic.c:384  HConeComputeATimesX (accumulates into dATimesX) */
extern void HConeComputeATimesX( hdsdp_cone *HCone, double *dConePrimal, double *dATimesX );
/* interface/hdsdp_conic.c:390  HConeComputeTraceCX */
extern double HConeComputeTraceCX( hdsdp_cone *HCone, double *dConePrimal );
/* interface/hdsdp_conic.c:395  HConeScalByConstant */
extern void HConeScalByConstant( hdsdp_cone *HCone, double dScal );

/* interface/hdsdp_schur.c:167  HKKTCreate */
extern hdsdp_retcode HKKTCreate( hdsdp_kkt **pHKKT );
/* interface/hdsdp_schur.c:181  HKKTInit: M is kept dense on the device */
extern hdsdp_retcode HKKTInit( hdsdp_kkt *HKKT, int nRow, int nCones, hdsdp_cone **cones );
/* interface/hdsdp_schur.c:256  HKKTBuildUp: clean, then every cone's coneBuildSchur in order */
extern hdsdp_retcode HKKTBuildUp( hdsdp_kkt *HKKT, int typeKKT );
/* interface/hdsdp_schur.c:270  HKKTBuildUpExtraCone: add one more cone's terms (the bound cone) */
extern hdsdp_retcode HKKTBuildUpExtraCone( hdsdp_kkt *HKKT, hdsdp_cone *cone, int typeKKT );
/* interface/hdsdp_schur.c:279  HKKTBuildUpFixed */
extern hdsdp_retcode HKKTBuildUpFixed( hdsdp_kkt *HKKT, int typeKKT, int kktStrategy );
/* interface/hdsdp_schur.c:293  HKKTExport (any output may be NULL) */
extern void HKKTExport( hdsdp_kkt *HKKT, double *dKKTASinvVec, double *dKKTASinvRdSinvVec, double *dKKTASinvCSinvVec,
                        double *dCSinvCSinv, double *dCSinv, double *dCSinvRdCSinv, double *dTraceSinv );
/* interface/hdsdp_schur.c:328  HKKTFactorize */
extern hdsdp_retcode HKKTFactorize( hdsdp_kkt *HKKT );
/* interface/hdsdp_schur.c:338  HKKTSolve (dLhsVec NULL: in place) */
extern hdsdp_retcode HKKTSolve( hdsdp_kkt *HKKT, double *dRhsVec, double *dLhsVec );
/* interface/hdsdp_schur.c:348  HKKTRegularize */
extern void HKKTRegularize( hdsdp_kkt *HKKT, double dKKTReg );
/* interface/hdsdp_schur.c:375  HKKTClear */
extern void HKKTClear( hdsdp_kkt *HKKT );
/* interface/hdsdp_schur.c:400  HKKTDestroy */
extern void HKKTDestroy( hdsdp_kkt **pHKKT );
/* No reference counterpart: copy the lower triangle of M (nRow x nRow, column-major)
   from the device into a host array (the upper triangle is left as it is). */
extern hdsdp_retcode HKKTGetMatrix( hdsdp_kkt *HKKT, double *dKKTMat );

#ifdef __cplusplus
}
#endif

#endif /* HDSDP_B200_CONIC_H */
