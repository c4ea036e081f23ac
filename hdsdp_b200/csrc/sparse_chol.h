// Sparse Cholesky of the dual slack S for sparse dual patterns (the role Pardiso plays for
// the reference's sparse dual matrices, interface/hdsdp_conic_sdp.c:153-275 and
// linalg/hdsdp_linsolver.c:47-450).
//
// Ordering (host, once per cone, from the fixed pattern of S): multiple minimum degree
// in rounds. Each round eliminates an independent set of vertices whose degree is at
// most the round's minimum degree plus a quarter of it; rounds stop once the minimum
// degree exceeds a cap. The vertices left form the dense front. On a MaxCut pattern
// with n = 8000 and 40,000 edges, a cap of 64 ends after 13 rounds with a front of
// 4,409: the front's dense factorisation is 17% of the dense flops, and the sparse
// part is 49k entries of L.
//
// Numeric factorisation (device, every call): the entries the rounds read or update are
// gathered from S into a slot array; per round one kernel scales the eliminated columns
// (l_jj = sqrt(s_jj), l_aj = s_aj / l_jj; the set is independent, so the columns do not
// interact) and one kernel applies their Schur updates, each target entry summing its
// contributions in a fixed order (deterministic, no atomics). The front is then
// gathered from S, overwritten at the updated slots, and factored by the dense
// cooperative Cholesky. S is positive definite iff every pivot of the rounds and the
// front factorisation is positive; log det S = 2 (sum log l_jj + sum log diag L_front).
//
// The factor answers positive-definiteness checks and log det, and applies L^-1 and L^-T
// for the Lanczos step bound (the rounds as triangular solves, the front through its
// inverse factor). Consumers that need S^-1 or L as a matrix (the Schur build, primal
// recovery) run the dense factorisation of the same S.
#pragma once
#include <vector>
#include <cuda_runtime.h>
#include "la.h"

namespace hb {

struct HybridFactor {
    int n = 0, nslot = 0, nelim = 0, nfront = 0, nrounds = 0, nfix = 0;
    long nnbr = 0, ncontrib = 0;
    std::vector<int> roundElim, roundTgt;  // per round: [begin, end) of its eliminated vertices / targets
    // device symbolic data
    int *d_srow = nullptr, *d_scol = nullptr;              // slot -> (row >= col)
    int *d_dslot = nullptr, *d_nptr = nullptr, *d_nslot = nullptr;
    int *d_tslot = nullptr, *d_cptr = nullptr, *d_ca = nullptr, *d_cb = nullptr;
    int *d_front = nullptr, *d_fixslot = nullptr;
    long *d_fixpos = nullptr;
    // triangular solves: per entry its row and column vertex, per eliminated index its
    // vertex, and the entries of each eliminated row / front row (row structure of L)
    int *d_nbrv = nullptr, *d_colv = nullptr, *d_elimv = nullptr;
    int *d_inptr = nullptr, *d_inent = nullptr, *d_finptr = nullptr, *d_finent = nullptr;
    double *fa = nullptr, *fb = nullptr;  // front-length work vectors
    long seq = 0;                         // numeric factorisations done (identifies the held factor)
    // host symbolic data, held from analyse() to upload()
    std::vector<int> hSrow, hScol, hDslot, hNptr, hNslot, hTslot, hCptr, hCa, hCb, hFront, hFixslot;
    std::vector<int> hNbrV, hColV, hElimV, hInptr, hInent, hFinptr, hFinent;
    std::vector<long> hFixpos;
    // numeric workspace
    double *wv = nullptr, *lval = nullptr, *ldiag = nullptr, *Sf = nullptr;
    long ldf = 0;
    DenseFactor Ff;
    int *d_info = nullptr, *h_info = nullptr;
    double *d_logdet = nullptr, *h_logdet = nullptr;

    // Ordering and symbolic analysis of the pattern adj (sorted neighbour lists, no
    // diagonal). Returns false when the front is not small enough to pay off
    // (front > maxFrontFrac * n) unless force is set.
    bool analyse(int n_, const std::vector<std::vector<int>> &adj, int cap, double maxFrontFrac, bool force);
    void upload(cudaStream_t s);
    // Enqueue the factorisation of the lower triangle of S (leading dimension ld).
    void factor_async(cudaStream_t s, const double *S, long ld);
    // Wait for it: true iff S is positive definite; logdet = log det S when it is.
    bool finish(cudaStream_t s, double *logdet);
    // y = L^-1 (alpha D) L^-T x for the held factor (D dense n x n, vectors of length n in
    // the original order; t is an n-vector of scratch). The front's inverse factor must
    // have been formed (compute_inverse_factor(s, Ff)).
    void apply_congruence(cudaStream_t s, const double *D, long ldD, double alpha, const double *x, double *t,
                          double *u, double *y);
    void release();
};

}  // namespace hb
