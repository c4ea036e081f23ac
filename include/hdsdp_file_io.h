/*
 * hdsdp_file_io.h -- SDPA sparse-format reader with the reference's interface
 * (interface/hdsdp_file_io.h:7). The caller owns every array it returns and frees
 * each with free(): blkDims, rowRHS, coneMatBeg[k] / coneMatIdx[k] / coneMatElem[k]
 * for k < nBlks and the three pointer arrays, and the LP arrays when nLPCols > 0.
 *
 * nBlks counts the SDP blocks; a negative last block size in the file is a diagonal LP
 * block, returned as a CSC matrix with nLPCols rows and nConstrs + 1 columns. Each SDP
 * block is a CSC matrix with PACK_NNZ(n) rows (packed lower triangle) and nConstrs + 1
 * columns, column 0 being the objective matrix with its sign flipped, the form that
 * HUserDataSetConeData takes: each SDP block becomes one cone (HDSDP_CONETYPE_DENSE_SDP
 * user data) and the LP block one LP cone (HDSDP_CONETYPE_LP user data).
 */
#ifndef HDSDP_FILE_IO_H
#define HDSDP_FILE_IO_H

#include "hdsdp.h"

#ifdef __cplusplus
extern "C" {
#endif

extern hdsdp_retcode HReadSDPA( char *fname, int *pnConstrs, int *pnBlks, int **pblkDims, double **prowRHS,
                                int ***pconeMatBeg, int ***pconeMatIdx, double ***pconeMatElem, int *pnCols,
                                int *pnLPCols, int **pLpMatBeg, int **pLpMatIdx, double **pLpMatElem, int *pnElems );

#ifdef __cplusplus
}
#endif

#endif /* HDSDP_FILE_IO_H */
