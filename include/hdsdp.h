/*
 * hdsdp.h -- public C API of the B200 HDSDP library (libhdsdp_b200.so).
 *
 * Drop-in for the reference solver's public header, interface/hdsdp.h:40-116:
 * the same return codes, status values, parameter indices and function
 * signatures, so C code written against the reference links against this
 * library unchanged. Each entry point below names the reference function it
 * replaces.
 *
 * Threading: every solver object owns its own CUDA stream and device
 * buffers, so distinct solver objects may be used from distinct host
 * threads. One solver object must not be used from two threads at once.
 */
#ifndef HDSDP_B200_HDSDP_H
#define HDSDP_B200_HDSDP_H

#define KKT_ACCURACY (1e-12)
#define HDSDP_SPARSE_CONE_THRESHOLD  (0.3)
#define HDSDP_SPARSE_SCHUR_THRESHOLD (0.3)

typedef enum {
    HDSDP_RETCODE_OK,
    HDSDP_RETCODE_FAILED,
    HDSDP_RETCODE_MEMORY,
} hdsdp_retcode;

typedef enum {
    HDSDP_UNKNOWN,
    HDSDP_DUAL_FEASIBLE,
    HDSDP_DUAL_OPTIMAL,
    HDSDP_PRIMAL_DUAL_OPTIMAL,
    HDSDP_MAXITER,
    HDSDP_SUSPECT_INFEAS_OR_UNBOUNDED,
    HDSDP_INFEAS_OR_UNBOUNDED,
    HDSDP_TIMELIMIT,
    HDSDP_USER_INTERRUPT,
    HDSDP_INTERNAL_ERROR,
    HDSDP_NUMERICAL
} hdsdp_status;

typedef struct hdsdp_solver_internal hdsdp;

#define HDSDP_INFINITY          1e+30

/* Integer parameters (interface/hdsdp.h:68-72) */
#define INT_PARAM_MAXITER       0
#define INT_PARAM_CORRECTORA    1
#define INT_PARAM_CORRECTORB    2
#define INT_PARAM_THREADS       3
#define INT_PARAM_PSDP          4

/* Double parameters (interface/hdsdp.h:74-88) */
#define DBL_PARAM_RELFEASTOL    0
#define DBL_PARAM_RELOPTTOL     1
#define DBL_PARAM_ABSFEASTOL    2
#define DBL_PARAM_ABSOPTTOL     3
#define DBL_PARAM_TIMELIMIT     4
#define DBL_PARAM_POTRHOVAL     5
#define DBL_PARAM_HSDGAMMA      6
#define DBL_PARAM_DUALBOX_LOW   7
#define DBL_PARAM_DUALBOX_UP    8
#define DBL_PARAM_BARMUSTART    9
#define DBL_PARAM_DUALSTART    10
#define DBL_PARAM_POBJSTART    11
#define DBL_PARAM_TRXESTIMATE  12
#define DBL_PARAM_PRECORDACC   13

#ifdef __cplusplus
extern "C" {
#endif

/* interface/hdsdp.c:472  HDSDPCreate */
extern hdsdp_retcode HDSDPCreate( hdsdp **pHSolver );
/* interface/hdsdp.c:493  HDSDPInit */
extern hdsdp_retcode HDSDPInit( hdsdp *HSolver, int nRows, int nCones );
/* interface/hdsdp.c:570  HDSDPSetCone (userCone is a user_data *) */
extern hdsdp_retcode HDSDPSetCone( hdsdp *HSolver, int iCone, void *userCone );
/* interface/hdsdp.c:580  HDSDPSetDualObjective (copies b) */
extern void HDSDPSetDualObjective( hdsdp *HSolver, double *dObj );
/* interface/hdsdp.c:617  HDSDPOptimize */
extern hdsdp_retcode HDSDPOptimize( hdsdp *HSolver, int dOptOnly );
/* interface/hdsdp.c:596  HDSDPSetIntParam (indices 0-2, others ignored) */
extern void HDSDPSetIntParam( hdsdp *HSolver, int intParam, int intParamVal );
/* interface/hdsdp.c:607  HDSDPSetDblParam (indices 0-12, others ignored) */
extern void HDSDPSetDblParam( hdsdp *HSolver, int intParam, double dblParamVal );
/* interface/hdsdp.c:691  HDSDPGetRowDual */
extern hdsdp_retcode HDSDPGetRowDual( hdsdp *HSolver, double *pObjVal, double *dObjVal, double *dualVal );
/* interface/hdsdp.c:711  HDSDPGetConeValues: X, S and an n x n scratch, column-major full */
extern void HDSDPGetConeValues( hdsdp *HSolver, int iCone, double *conePrimal, double *coneDual, double *coneAuxi );
/* interface/hdsdp.c:753  HDSDPCheckSolution: six DIMACS errors */
extern hdsdp_retcode HDSDPCheckSolution( hdsdp *HSolver, double diErrors[6] );
/* interface/hdsdp.c:908  HDSDPClear */
extern void HDSDPClear( hdsdp *HSolver );
/* interface/hdsdp.c:945  HDSDPDestroy */
extern void HDSDPDestroy( hdsdp **pHSolver );

#ifdef __cplusplus
}
#endif

#endif /* HDSDP_B200_HDSDP_H */
