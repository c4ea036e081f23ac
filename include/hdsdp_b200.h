/*
 * hdsdp_b200.h -- entry points that the B200 library adds next to the
 * reference API of hdsdp.h. None of these has a counterpart in the reference
 * interface; each comment names the reference code whose behaviour it
 * exposes.
 */
#ifndef HDSDP_B200_EXT_H
#define HDSDP_B200_EXT_H

#include "hdsdp.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Solver status and iteration count: the reference keeps these in its private
   solver struct (interface/def_hdsdp.h:111, :122) and has no getter. */
extern int HDSDPGetStatus( hdsdp *HSolver );
extern int HDSDPGetIterCount( hdsdp *HSolver );

/* Enable / disable the five-step primal refinement run when Phase B reaches a
   10% gap (interface/hdsdp_algo.c:1803-1810). The reference's setter refuses
   index INT_PARAM_PSDP (interface/hdsdp.c:598). With it off, Phase B runs to
   its own convergence test (interface/hdsdp_algo.c:1797-1801). */
extern void HDSDPSetPrimalRefinement( hdsdp *HSolver, int on );

/* Schur-assembly arithmetic: 0 = FP64 throughout (default); 1 = split
   precision (dense rank-one Schur block as BF16x3 products with FP32
   accumulation on the tcgen05 tensor cores, FP64 everywhere else);
   2 = split precision while the relative gap is above 1e-3, FP64 after. */
extern void HDSDPSetPrecision( hdsdp *HSolver, int mode );

/* Factorisation of the dual slack S for positive-definiteness checks, log det and the
   Lanczos step bound: -1 = automatic (default): a sparse factorisation (minimum-degree
   rounds on the device and a dense front) for the trial points of blocks of order
   >= 1500 whose front is at most 70% of the order, the dense Cholesky for the accepted
   point, whose S^-1 the Schur build uses; 0 = always the dense cooperative Cholesky;
   1 = sparse for every check whenever the pattern allows it. S^-1 and primal recovery
   refactor densely when their buffer was factored sparsely. This is where the reference uses Pardiso for sparse dual
   matrices (interface/hdsdp_conic_sdp.c:153-275). Takes effect at the next
   HDSDPOptimize. */
extern void HDSDPSetSparseSlack( hdsdp *HSolver, int mode );

/* out[0] = SDP cones factored sparsely, out[1] = dense-front order of the first of
   them, out[2] = its minimum-degree rounds, out[3] = sparse factorisations in the
   last solve (all cones), out[4] = vertices eliminated before the front, out[5] = the
   sparse factorisations of trial points, out[6] / out[7] = dense factorisations that
   followed a sparse one because a consumer needed L (accepted point / trial point). */
extern void HDSDPGetSparseSlackInfo( hdsdp *HSolver, double out[8] );

/* Form of the Schur complement M when every cone of the problem is a sparse SDP cone (no
   dense SDP cone, no LP cone; where the reference takes its sparse KKT,
   interface/hdsdp_schur.c:224-246, factored through Pardiso): a block arrow. Rows held by
   one cone only form that cone's diagonal block; rows held by several cones (or by none)
   form the coupling block, factored after the Schur complement of the cones' blocks.
   -1 = automatic (default): the block arrow for m >= 4096 when it needs at most a quarter
   of the dense factorisation's flops; 0 = always the dense M; 1 = the block arrow whenever
   the cones allow it. Takes effect at the next HDSDPOptimize. */
extern void HDSDPSetSparseSchur( hdsdp *HSolver, int mode );

/* out[0] = 1 if the last solve used the block arrow, out[1] = coupling rows, out[2] =
   cones, out[3] = the largest cone's local rows, out[4] = device bytes the block arrow
   holds (blocks, factors, coupling block, scratch), out[5] = device bytes the dense M and
   its factor would take. */
extern void HDSDPGetSparseSchurInfo( hdsdp *HSolver, double out[6] );

/* Factorisation of the dense Schur complement M. 0 (default) = Cholesky; when it fails,
   retried with diagonal shifts up to 1e-6 of the largest diagonal entry, and when every
   shift fails, the LDL^T factorisation with Bunch-Kaufman pivoting of the unshifted M (the
   indefinite solver the reference switches to, linalg/hdsdp_linsolver.c:1367-1380). 1 =
   LDL^T for every factorisation of M (the block-arrow form is then not used). Takes effect
   at the next HDSDPOptimize. */
extern void HDSDPSetSchurLDL( hdsdp *HSolver, int mode );

/* Per-iteration record of the last solve: elapsed seconds, primal and dual
   objective, barrier parameter, relative gap (p - d) / (1 + |p| + |d|) and
   phase (0 infeasible, 1 embedding, 2 potential reduction, 3 refinement),
   as printed by the reference's iteration log (interface/hdsdp_algo.c:151-193).
   Returns the number of records (arrays may be NULL to query it). */
extern int HDSDPGetIterLog( hdsdp *HSolver, int maxLen, double *t, double *pObj, double *dObj,
                            double *mu, double *gap, int *phase );

/* Wall-clock split of the last solve in seconds:
   [0] Schur assembly  [1] Schur factorisation  [2] Schur solves  [3] S factorisations
   [4] S inverse       [5] Lanczos              [6] S assembly    [7] primal recovery
   [8] total           [9] #Schur builds       [10] #S factorisations
   [11] #Lanczos runs  [12] #Lanczos matvecs    [13] #Schur solves
   [14] Lanczos: L^-1 (host time to enqueue it)  [15] Lanczos: host eigen [16] Lanczos: device wait
   [17] Schur: matrix  [18] Schur: <A_i, W>     [19] Schur: <A_i, W^2>
   [20] presolve + upload of the data (host wall clock)
   [21] iterations + final DIMACS check, CUDA events on the solver stream
   [22] #S factorisations reused (the same dual slack factored before) */
extern void HDSDPGetTimers( hdsdp *HSolver, double out[23] );

/* The library keeps freed device and pinned host buffers for reuse by later
   solvers of the same sizes (no reference counterpart). This hands the cached
   buffers back to the driver; call it when the library will not be used for a
   while. */
extern void hdsdpb_release_cached_memory( void );

/* Number of kernel launches this library has issued in the process so far
   (all solvers and entry points). No reference counterpart. */
extern long long hdsdpb_launch_count( void );

/* Number of device and pinned-host buffer requests this library has made in the
   process so far, whether served from its cache or by the driver (all solvers and
   entry points). No reference counterpart; lets a caller confirm that a call path
   allocates nothing. */
extern long long hdsdpb_alloc_calls( void );

/* Live kernel timing by family (no reference counterpart): bit f of `mask`
   enables family f = 0 FP64 GEMM, 1 Cholesky of the dual slack (cooperative potrf,
   order n), 2 triangular inverse, 3 Schur gather pair kernels, 4 BF16x3 split GEMM,
   5 Cholesky of the Schur matrix (the same kernel, order m). While enabled, each
   launch of the family is bracketed by CUDA events on its own stream; enabling
   resets the totals. hdsdpb_kstat_read returns the launches, the summed event time
   in ms and the summed algorithmic work (flops for 0-2, 4, 5; compulsory bytes for 3). */
extern int hdsdpb_kstat_enable( int mask );
extern int hdsdpb_kstat_read( int family, long long *launches, double *ms, double *work );

/* Vector-Jacobian product of the solution map of the last HDSDPOptimize
   (no reference counterpart). gy (m) and GX (n x n, column-major,
   symmetric) are the gradients of a loss with respect to y* and X*; either
   may be NULL (zero). Writes the gradient with respect to b into gb (m),
   with respect to C as a full symmetric n x n matrix into gC, and with
   respect to every stored value of the cone's CSC data (columns 0..m, the
   user's Ap[m+1] entries) into gAx; outputs may be NULL. Computed by
   implicit differentiation of the optimality conditions at the final
   iterate in the Nesterov-Todd scaling; the first call after a solve builds
   and factors the scaled Schur matrix, later calls reuse it. The user's CSC
   arrays must still be alive. Returns HDSDP_RETCODE_OK or HDSDP_RETCODE_FAILED. */
extern hdsdp_retcode HDSDPAdjoint( hdsdp *HSolver, const double *gy, const double *GX, double *gb,
                                   double *gC, double *gAx );

/* ---- Kernel-level entry points (host buffers in, host buffers out) ---------------- */

/* Schur complement of one SDP block given in the user-data CSC layout, at
   S = C - sum_i y_i A_i - resi * I: the GPU counterpart of the reference's
   HKKTBuildUp(KKT_TYPE_INFEASIBLE) (interface/hdsdp_schur.c:256-268).
   Writes M (m x m, lower triangle, column-major), ASinv_i = <A_i, S^-1>,
   ASinvRdSinv_i = resi <A_i, S^-2> and trace(S^-1).
   Returns 0 on success, 1 if S is not positive definite, -1 on error. */
extern int hdsdpb_schur_probe( int m, int n, const int *Ap, const int *Ai, const double *Ax,
                               const double *y, double resi, int precision, double *M,
                               double *asinv, double *asinvrd, double *traceSinv );

/* First Lanczos ratio test on S = C - A^T y - resi I along dS = -A^T dy + ada * resi * I
   (interface/hdsdp_conic_sdp.c:1638-1682), plus log det S.
   Returns 0 on success, 1 if S is not positive definite, -1 on error. */
extern int hdsdpb_ratio_probe( int m, int n, const int *Ap, const int *Ai, const double *Ax,
                               const double *y, double resi, const double *dy, double ada,
                               double *step, double *logdet );

/* Cholesky factorisation of a symmetric n x n matrix (lower triangle read),
   with the positive-definiteness test of the reference's dual checks
   (linalg/hdsdp_linsolver.c:521-553). Writes L (lower, full n x n storage,
   upper part zero) and sum(log L_ii). Returns 0 if positive definite, 1 if not. */
extern int hdsdpb_cholesky( int n, const double *S, double *L, double *logdiag );

/* count factorisations of order n <= 1024 (S: count column-major n x n matrices): mode 0 one
   CTA per matrix in shared launches (the multi-cone path), mode 1 each on the whole GPU (the
   cooperative kernel). L and K = L^-1 (lower), logdiag = sum log L_ii and status (0 positive
   definite, 1 not) per matrix; any output may be NULL. Returns 0, or -1 on bad arguments or a
   CUDA error. */
extern int hdsdpb_cholesky_batch( int count, int n, int mode, const double *S, double *L, double *K,
                                  double *logdiag, int *status );

/* Solution of S x = b through the Cholesky factor of S by blocked forward and backward
   substitution with L (the reference's dpotrs use, linalg/hdsdp_linsolver.c:607-633; the
   solver uses it for Schur systems of order >= 6000). Returns 0 on success, 1 if S is
   not positive definite, -1 on error. */
extern int hdsdpb_cholesky_solve( int n, const double *S, const double *b, double *x );

/* Solution of S x = b for a symmetric, possibly indefinite S (n x n, column-major, only
   its lower triangle read) through P S P^T = L D L^T with Bunch-Kaufman pivoting (the
   reference's dsytrf / dsytrs use, linalg/hdsdp_linsolver.c:1118-1190). out (may be NULL):
   {2 x 2 pivots, negative eigenvalues, positive eigenvalues} of D, the inertia of S.
   Returns 0 on success, k > 0 if the pivot column of step k is zero (S singular) or not
   finite, -1 on error. */
extern int hdsdpb_ldl_solve( int n, const double *S, const double *b, double *x, int out[3] );

/* Allocation-free variant of hdsdpb_cholesky (no reference counterpart), for callers
   that cannot call cudaMalloc on their call path (a host framework whose allocator
   owns the device memory, a plugin barred from allocating, a latency-critical loop
   that cannot take the synchronisation of cudaMalloc/cudaFree). Same arguments and
   return values, but all device scratch is one static device array sized for
   n <= HDSDPB_NOALLOC_MAX_N (about 1.2 MB per GPU, held until exit); nothing is
   allocated or freed per call. Returns -2 (with a message on stderr) when n exceeds
   the limit. The first call on a device looks up the array's address and should come
   before any stream capture; calls that overlap on the GPU share the scratch and race.
   The work runs on the legacy default stream (so it also waits for the caller's
   blocking streams), and the call returns after synchronising that stream. */
#define HDSDPB_NOALLOC_MAX_N 256
extern int hdsdpb_cholesky_noalloc( int n, const double *S, double *L, double *logdiag );

/* Inverse of a symmetric positive definite n x n matrix through its Cholesky
   factor (the reference's dpotri use, linalg/hdsdp_linsolver.c:647-669).
   Returns 0 on success, 1 if not positive definite. */
extern int hdsdpb_inverse( int n, const double *S, double *Sinv );

/* The Cholesky factor L of a symmetric positive definite n x n matrix together with its
   inverse K = L^-1, as the solver forms them for its Schur matrix below 6000 rows (K in the
   factorisation's own launch; above order 3840 the recursive blocked form). Column-major
   host buffers; L and K are written with zeros above the diagonal. Returns 0 on success, 1
   if not positive definite, -1 on error. */
extern int hdsdpb_cholesky_inverse_factor( int n, const double *S, double *L, double *K );

/* FP64 GEMM on the tensor-core path: C = alpha op(A) op(B) + beta C with
   column-major host buffers (op = transpose when trans != 0). */
extern int hdsdpb_gemm( int M, int N, int K, double alpha, const double *A, int lda, int transA,
                        const double *B, int ldb, int transB, double beta, double *C, int ldc );

/* Split-precision product on the tcgen05 tensor cores: C = op(A) op(B) with
   every FP64 operand split into BF16 hi + lo parts and the three products
   hi*hi + hi*lo + lo*hi accumulated in FP32 (relative error about 2^-16 of
   sum |a||b|). Column-major host buffers. Returns 0 on success, 2 if the
   tensor-core path could not be set up, -1 on error. */
extern int hdsdpb_split_gemm( int M, int N, int K, const double *A, int lda, int transA,
                              const double *B, int ldb, int transB, double *C, int ldc );

/* Device-resident timing of one kernel family on an n x n problem (CUDA events
   on the launching stream, 2 warm-up calls): 0 GEMM NN, 1 GEMM TN lower,
   2 Cholesky, 3 triangular inverse L^-1, 4 matrix-vector product,
   5 Lanczos step bound, 6 rank-64 SYRK update, 7 Cholesky that also forms L^-1,
   8 Cholesky without it, 9 solve with the factor (forward and backward substitution),
   10 as 7 on the one-launch kernel at every order (7 takes the recursive blocked form
   above order 3840), 11 as 8 on the one-launch kernel at every order (8 takes the
   recursive form above order 8192). Writes milliseconds per call. */
extern int hdsdpb_kernel_timing( int which, int n, int reps, double *ms );

/* Host only (no device work): the ordering of the sparse factorisation of S for the
   pattern of nedge off-diagonal pairs (ei[k], ej[k]) with degree cap `cap`.
   out = {rounds, front order, eliminated vertices, slots, Schur contributions};
   front (length n, may be NULL) receives the front's vertices in increasing order.
   Returns 0, or -1 for invalid input. */
extern int hdsdpb_sparse_analyse( int n, int nedge, const int *ei, const int *ej, int cap, double out[5],
                                  int *front );

/* The sparse factorisation of S (column-major n x n, host; pattern = the nedge
   off-diagonal pairs) with degree cap `cap`, timed over `reps` calls after a warm-up,
   beside the dense factorisation of the same S. out = {positive definite (1/0),
   log det S, ms per sparse factorisation, ms per dense factorisation, front order}.
   Returns 0, or -1 for invalid input. */
extern int hdsdpb_sparse_cholesky( int n, int nedge, const int *ei, const int *ej, const double *S, int cap,
                                   int reps, double out[5] );

/* With the sparse factor S = L L^T (pattern as above, cap 64): t = L^-T x and
   y = L^-1 (D t) for a host n x n D and n-vector x (t may be NULL). The operator the
   Lanczos step bound uses with D = -dS. Returns 0, 1 if S is not positive definite,
   -1 for invalid input. */
extern int hdsdpb_sparse_congruence( int n, int nedge, const int *ei, const int *ej, const double *S,
                                     const double *D, const double *x, double *y, double *t );

/* Milliseconds taken by `reps` grid-wide barriers in one cooperative launch of
   `blocks` blocks of 256 threads (cost model of the persistent factorisation). */
extern int hdsdpb_gridsync_probe( int blocks, int reps, double *ms );

#ifdef __cplusplus
}
#endif

#endif /* HDSDP_B200_EXT_H */
