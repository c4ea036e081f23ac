/*
 * hdsdp_user_data.h -- conic user data, drop-in for the reference's
 * interface/hdsdp_user_data.h:18-23 and interface/def_hdsdp_conic.h:22-32.
 *
 * An SDP block is a CSC matrix with n(n+1)/2 rows and m+1 columns: column 0
 * is the objective C, column i is A_i; the row index of lower-triangle entry
 * (i, j), i >= j, is (2n - j - 1) j / 2 + i (interface/hdsdp_utils.h:49).
 * The arrays are held by pointer (not copied) until HDSDPOptimize has run,
 * as in the reference (interface/hdsdp_user_data.c:60-71).
 */
#ifndef HDSDP_B200_USER_DATA_H
#define HDSDP_B200_USER_DATA_H

#include "hdsdp.h"

typedef enum {
    HDSDP_CONETYPE_UNKNOWN,
    HDSDP_CONETYPE_LP,
    HDSDP_CONETYPE_BOUND,
    HDSDP_CONETYPE_SCALAR_BOUND,
    HDSDP_CONETYPE_DENSE_SDP,
    HDSDP_CONETYPE_SPARSE_SDP,
    HDSDP_CONETYPE_SOCP
} cone_type;

typedef struct hdsdp_user_data user_data;

#ifdef __cplusplus
extern "C" {
#endif

/* interface/hdsdp_user_data.c:38  HUserDataCreate */
extern hdsdp_retcode HUserDataCreate( user_data **pHdata );
/* interface/hdsdp_user_data.c:60  HUserDataSetConeData */
extern void HUserDataSetConeData( user_data *Hdata, cone_type cone, int nRow, int nCol,
                                  int *coneMatBeg, int *coneMatIdx, double *coneMatElem );
/* interface/hdsdp_user_data.c:73  HUserDataChooseCone */
extern cone_type HUserDataChooseCone( user_data *Hdata );
/* interface/hdsdp_user_data.c:102  HUserDataClear */
extern void HUserDataClear( user_data *Hdata );
/* interface/hdsdp_user_data.c:113  HUserDataDestroy */
extern void HUserDataDestroy( user_data **pHdata );

#ifdef __cplusplus
}
#endif

#endif /* HDSDP_B200_USER_DATA_H */
