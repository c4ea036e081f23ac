// Dense FP64 linear algebra on the B200: GEMM on the DMMA (FP64 tensor-core)
// path, blocked Cholesky with a positive-definiteness flag, triangular
// inverse, column-dot matrix-vector products and small reductions.
//
// All matrices are column-major FP64 with an explicit leading dimension.
// Symmetric matrices are stored full (both triangles) unless a routine says
// it reads only the lower triangle.
#pragma once
#include <cuda_runtime.h>
#include "dev.cuh"

namespace hb {

enum GemmFlags : int {
    GEMM_C_LOWER = 1,      // compute / write only entries with row >= col
    GEMM_A_LOWER = 2,      // op(A)(i,k) == 0 for k > i  (read as zero)
    GEMM_A_UPPER = 4,      // op(A)(i,k) == 0 for k < i
    GEMM_B_LOWER = 8,      // op(B)(k,j) == 0 for k < j
    GEMM_B_UPPER = 16,     // op(B)(k,j) == 0 for k > j
};

// C = alpha * op(A) * op(B) + beta * C   (op = transpose when trans != 0).
// If abort_flag is non-null and *abort_flag != 0 when a tile starts, the tile is skipped.
void gemm(cudaStream_t s, int M, int N, int K, double alpha, const double *A, long lda, int transA,
          const double *B, long ldb, int transB, double beta, double *C, long ldc, int flags = 0,
          const int *abort_flag = nullptr);

// One GEMM of a group: C = alpha * op(A) * op(B) + beta * C with the flags above.
struct GemmDesc {
    int M, N, K;
    double alpha, beta;
    const double *A;
    long lda;
    int ta;
    const double *B;
    long ldb;
    int tb;
    double *C;
    long ldc;
    int flags;
    const int *abort_flag;
};
// A group of independent GEMMs (device array of descriptors, none larger than maxM x maxN)
// in one launch on the 64 x 64 DMMA tiles.
void gemm_grouped(cudaStream_t s, const GemmDesc *d_desc, int count, int maxM, int maxN);

// Column-dot matrix-vector product:
//   out[i] = alpha * sum_{k in R(i)} A[k + i*lda] * x[k] + beta * out[i],  i < ncols
// with R(i) = [0, nrows) (mode 0), [i, nrows) (mode 1), [0, i] (mode 2).
void coldot(cudaStream_t s, int nrows, int ncols, const double *A, long lda, const double *x,
            double *out, double alpha, double beta, int mode);

// Symmetric indefinite factorisation P S P^T = L D L^T (Bunch-Kaufman pivoting, ldl.cu).
// A holds D's 1 x 1 and 2 x 2 blocks on and below the diagonal and L^T strictly above it;
// perm the symmetric permutation, piv the pivot size at the first index of each block
// (1 or 2; -1 at the second index of a 2 x 2 block).
constexpr int kMaxLdlGrid = 1024;
struct LdlFactor {
    int n = 0;
    long ld = 0;
    double *A = nullptr;
    int *perm = nullptr, *piv = nullptr, *d_info = nullptr;
    double *cm = nullptr, *part = nullptr, *w = nullptr;
    double *h_info = nullptr;   // pinned: the info word (0, or the step whose pivot column is zero or NaN)
    bool ok = false;
    void release();
};
// Factor the full symmetric n x n matrix S (leading dimension ldS; only its lower triangle
// is read); waits for the stream. False for an exactly singular or non-finite pivot.
bool ldl_factorize(cudaStream_t s, LdlFactor &F, const double *S, long ldS, int n);
// x = S^-1 b (device vectors; x may alias b), enqueued on s.
void ldl_solve(cudaStream_t s, LdlFactor &F, const double *b, double *x);

// Factor object for an n x n symmetric positive definite matrix.
// L holds the lower Cholesky factor, Dinv the inverses of its 64 x 64
// diagonal blocks, K = L^-1 and KT = L^-T (computed on demand).
constexpr int kFuseInverseMax = 2048;
// Above kRecMinN a factorisation that also forms K = L^-1 (the Schur matrix below 6000 rows)
// takes the recursive blocked form: the two diagonal halves (recursively, down to blocks of
// at most kRecLeafMaxN rows) on the cooperative kernel with their own K, the off-diagonal
// work as FP64 GEMMs. Measured on B200 (factor and K, ms): order 3595 3.13 one launch
// against 3.22 recursive, 4096 4.25 / 3.79, 5120 7.48 / 6.36, 5999 11.6 / 9.98.
constexpr int kRecMinN = 3840;
constexpr int kRecLeafMaxN = 2560;
// Above kRecNoKMinN a factorisation without K takes the recursive form too: L21 = A21 L11^-T
// by a recursive triangular solve whose leaves are GEMMs with the diagonal blocks' own K
// (kept in an n x kRecLeafMaxN strip). Measured on B200 (factor only, ms, one launch against
// recursive): order 6016 5.62 / 6.67, 8000 11.8 / 11.7, 12000 36.8 / 31.2, 16000 83.9 / 64.4.
constexpr int kRecNoKMinN = 8192;

struct DenseFactor {
    int n = 0;
    long ld = 0;
    double *L = nullptr;
    double *Dinv = nullptr;   // n x 64 (block b at rows [64b, 64b+64))
    double *K = nullptr;
    double *KT = nullptr;
    int *d_info = nullptr;    // device: 0 = success, k > 0 = pivot k failed
    int *h_info = nullptr;    // pinned host mirror
    // With stat_logdet set (the default; alloc() makes d_info and h_info 16 bytes each), a
    // factorisation also writes sum log L_ii next to the info word and both come back in one
    // copy; factor_status() then holds log det = 2 sum log L_ii in `logdet`.
    bool stat_logdet = true;
    bool logdet_valid = false;
    double logdet = 0.0;
    bool factored = false;
    bool ok = false;
    bool k_valid = false;
    // n <= kFuseInverseMax: the factorisation kernel also forms K and KT (allocated with
    // the factor, zero outside their triangles)
    bool fuse_k = false;
    bool k_pending = false;   // the last factorisation was enqueued with the fused inverse
    // fuse_inverse: the factorisation kernel also forms K = L^-1 and K^T (worth it for a
    // factor whose inverse is always used, and for small n where the K work hides behind
    // the panel chain); -1 picks n <= kFuseInverseMax.
    // scratch of chol_solve (allocated on first use): per-block ready flags of the forward
    // and backward sweeps, the intermediate vector, and the epoch tag of the last solve
    unsigned *d_flags = nullptr;
    double *d_tmp = nullptr;
    unsigned epoch = 0;
    // scratch of the recursive form for orders above kRecLeafMaxN with the inverse factor
    // (allocated on first use): the diagonal blocks' status words and an n x n/2 product
    int *d_rec_info = nullptr;
    double *d_rec_w = nullptr;
    double *d_rec_ks = nullptr, *d_rec_kts = nullptr;   // the diagonal blocks' K and K^T (no-K form)
    bool no_rec = false;      // keep the one-launch factorisation at every order (timing)
    int kfamily = KF_POTRF;   // kernel-timing family of this factor's factorisations
    void alloc(int n_, int fuse_inverse = -1);
    void release();
};

// x = (L L^T)^-1 b with the factor's L and diagonal-block inverses (no K needed): a
// forward and a backward blocked substitution in one cooperative launch. b and x are
// device vectors of length n and may alias. Returns false if the launch failed or a
// bounded wait inside it gave up.
bool chol_solve(cudaStream_t s, DenseFactor &F, const double *b, double *x);
// Reads and clears the flag raised when a wait inside chol_solve gave up (synchronising).
int chol_solve_error();

// Copy the lower triangle of S (n x n, ldS) into F.L and factorise it.
// Returns true if S is positive definite (dpotrf semantics: fails on a
// non-positive or NaN pivot). Synchronises the stream.
bool factorize(cudaStream_t s, DenseFactor &F, const double *S, long ldS);
// Enqueue the factorisation without synchronising; call factor_status() later.
void factorize_async(cudaStream_t s, DenseFactor &F, const double *S, long ldS);
bool factor_status(cudaStream_t s, DenseFactor &F);
// Enqueue the factorisations of F[q] (order <= kSmallFactorMaxN) of S[q] (ldS[q]) for
// q < count, one CTA each, in launches of up to 36 of them: the arithmetic of
// factorize_async on a grid of one block, which gives the same factor on any grid. Call
// factor_status() (or factor_status_ready() after a wait) on each afterwards, and wait for
// the stream before the same host thread enqueues another batch. Worth it for several
// matrices of moderate order: one CTA takes about as long for order 256 as the whole-GPU
// kernel, and many run at once.
constexpr int kSmallFactorMaxN = 1024;
// the order up to which factor_buffers batches the cones' dense factorisations
constexpr int kBatchFactorMaxN = 256;
void factorize_small_batch(cudaStream_t s, DenseFactor *const *F, const double *const *S, const long *ldS, int count);
// factor_status() without its wait, for a caller that has synchronised the stream since
// the factorisation was enqueued
bool factor_status_ready(DenseFactor &F);
// K = L^-1 and KT = K^T (lower / upper triangular). Requires a successful factor.
void compute_inverse_factor(cudaStream_t s, DenseFactor &F);
// W = S^-1 = K^T K, full symmetric, into W (ldW).
void compute_inverse(cudaStream_t s, DenseFactor &F, double *W, long ldW);
// sum_i log L_ii (device scalar out).
void log_diag_sum(cudaStream_t s, const DenseFactor &F, double *d_out);
// Copy the diagonal of L into out (n).
void copy_diag(cudaStream_t s, const DenseFactor &F, double *d_out);

// Small vector / matrix helpers
void fill(cudaStream_t s, double *x, double v, size_t n);
void axpy(cudaStream_t s, int n, double a, const double *x, double *y);
void symmetrize_lower(cudaStream_t s, int n, double *A, long lda);   // A(j,i) = A(i,j), i > j
void symmetrize_avg(cudaStream_t s, int n, double *A, long lda);     // A = (A + A^T)/2
void add_diag(cudaStream_t s, int n, double *A, long lda, double v);
void add_diag_vec(cudaStream_t s, int n, double *A, long lda, const double *d);
void copy_matrix(cudaStream_t s, int rows, int cols, const double *A, long lda, double *B, long ldb);
void transpose(cudaStream_t s, int n, const double *A, long lda, double *B, long ldb);
void scale_matrix(cudaStream_t s, int rows, int cols, double *A, long lda, double a);
// d_out[0] = sum_ij A_ij * B_ij over the full n x n matrices
void frob_dot(cudaStream_t s, int n, const double *A, long lda, const double *B, long ldb, double *d_out);
// d_out[0] = trace(A)
void trace(cudaStream_t s, int n, const double *A, long lda, double *d_out);
// d_out = x . y
void dot(cudaStream_t s, int n, const double *x, const double *y, double *d_out);
// Column j of A scaled by d[j]
void scale_columns(cudaStream_t s, int rows, int cols, const double *A, long lda, const double *d,
                   double *B, long ldb);

}  // namespace hb
