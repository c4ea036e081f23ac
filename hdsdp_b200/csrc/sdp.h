// Device representation of one dense SDP block and the kernels that touch
// its coefficient matrices: dual-slack assembly S = dC*C + dA*sum_j w_j A_j +
// dEye*I, Schur-complement assembly M_ij = <A_i, W A_j W> for a symmetric
// W (S^-1 in the dual method, X in primal refinement), and the inner-product
// vectors <A_j, Z> and <A_j, W^2>.
//
// Constraint classes (chosen at presolve, every class pair is covered):
//   SP   sparse triplets, at most kSpMax lower-triangle entries  -> gathers from W
//   R1S  rank one s*a*a^T with at most kR1SmallMax nonzeros      -> gathers from W
//   R1D  rank one with a denser factor                            -> GEMMs V = W*A1, G = A1^T*V
//   DR   dense or heavily populated coefficient                   -> B = W*A*W by GEMM, then gathers
//   ZERO no contribution
// Reference: interface/hdsdp_conic_sdp.c:683-981 (strategies M2-M5, which all
// compute the same M, cross-checked by HUtilKKTCheck at interface/hdsdp_utils.c:293-464).
#pragma once
#include <vector>
#include <cuda_runtime.h>
#include "la.h"
#include "split.h"

namespace hb {

constexpr int kSpMax = 16;
constexpr int kR1SmallMax = 8;

enum CoeffClass { CLS_ZERO = 0, CLS_SP = 1, CLS_R1S = 2, CLS_R1D = 3, CLS_DR = 4 };

// Host-side description of one coefficient matrix after presolve.
struct HostCoeff {
    int cls = CLS_ZERO;
    // SP / DR sparse source: lower-triangle triplets (row >= col)
    std::vector<int> r, c;
    std::vector<double> v;
    // rank one: sign * a a^T, a stored sparse (idx ascending)
    double sign = 0.0;
    std::vector<int> aidx;
    std::vector<double> aval;
    // DR from a dense packed column: full lower packed values (n(n+1)/2) or triplets above
    bool dense_packed = false;
    std::vector<double> packed;
};

struct SdpDevice {
    int n = 0, m = 0;
    long ld = 0;
    cudaStream_t stream = nullptr;

    // Objective, full symmetric n x n
    double *Cfull = nullptr;

    // SP class
    int nsp = 0;
    int *sp_id = nullptr, *sp_ptr = nullptr, *sp_r = nullptr, *sp_c = nullptr;
    double *sp_v = nullptr;
    // R1S class
    int nr1s = 0;
    int *r1s_id = nullptr, *r1s_ptr = nullptr, *r1s_p = nullptr;
    double *r1s_a = nullptr, *r1s_sign = nullptr;
    // R1D class: A1 is n x nr1d dense
    int nr1d = 0;
    int *r1d_id = nullptr;
    double *r1d_sign = nullptr;
    double *A1 = nullptr;
    // DR class: full n x n matrices
    int ndr = 0;
    std::vector<int> dr_id;
    std::vector<double *> dr_mat;
    // S assembly gather map over SP and R1S lower entries
    int npos = 0;
    int *pos_r = nullptr, *pos_c = nullptr, *pos_ptr = nullptr, *ent_j = nullptr;
    double *ent_v = nullptr;
    // Gather map of the dense rank-one class over its supports (used instead of the
    // rank-nr1d GEMM when the supports are sparse): per lower position the list of
    // (constraint, s_i a_ip a_iq), in constraint order
    bool r1d_gather = false;
    double t_upload_map = 0.0, t_upload_total = 0.0;  // host seconds spent in upload()
    // sliced layout: positions in slices of 32; entry e of the slice's lane l sits at
    // slice_ptr[slice] + 32 e + l (slices padded to their longest list, pos2_cnt per position)
    int npos2 = 0;
    int *pos2_r = nullptr, *pos2_c = nullptr, *pos2_cnt = nullptr;
    // positions whose lists are longer than kLongList (the diagonal ones: one entry per
    // constraint whose support holds the row) are kept out of the slices, whose padding
    // and slowest lane they would set, in a contiguous layout summed by a warp each:
    // entries of long position q at posL_ptr[q] .. posL_ptr[q + 1]
    int nposL = 0;
    int *posL_r = nullptr, *posL_c = nullptr;
    long long *posL_ptr = nullptr;
    int *entL_j = nullptr;
    double *entL_v = nullptr;
    long long *pos2_ptr = nullptr;
    int *ent2_j = nullptr;
    double *ent2_v = nullptr;

    // scratch
    double *V = nullptr;       // n x max(nr1d, nr1s) (W * A_r1)
    double *Vt = nullptr;      // n x nr1d scratch for inner products
    double *Vs = nullptr;      // n x nr1s scratch for rank-one x sparse cross terms
    double *G = nullptr;       // nr1d x nr1d
    double *T1 = nullptr;      // n x n
    double *T2 = nullptr;      // n x n
    double *vecbuf = nullptr;  // m
    double *d_w = nullptr;     // m + 1 weights
    double *d_scal = nullptr;  // small scalars
    double *h_scal = nullptr;  // pinned mirror

    // Split precision (BF16x3 on tcgen05) for the dense rank-one Schur block:
    // 0 FP64; 1 split for every build (set per build by the solver's policy)
    int precision = 0;
    SplitOperand opA1;        // rows: the nr1d factors a_i, K: n
    SplitOperand opK, opKT;   // L^-1 and L^-T of the dual slack (rows n, K n)
    SplitOperand opB;         // B = L^-1 A1 as rows b_i (rows nr1d, K n)
    bool split_ready = false; // G and opB hold the last split Schur build
    double *colsq = nullptr;  // nr1d

    void upload(int n_, int m_, const HostCoeff &C, const std::vector<HostCoeff> &A, cudaStream_t s);
    void release();

    // S = dC*C + dA*sum_j w_j A_j + dEye*I (full symmetric), w on device (length m)
    void assemble(double dC, double dA, const double *d_wvec, double dEye, double *S, long ldS);

    // Schur complement M (m x m, lower triangle written) from symmetric W.
    // With precision 1 and Kinv = L^-1 (W = Kinv^T Kinv) the dense rank-one
    // block is formed as (B^T B) o (B^T B), B = Kinv A1, in split precision.
    void schur_matrix(const double *W, long ldW, double *M, long ldM, const double *Kinv = nullptr);
    // out[j] = <A_j, Z> for all j (Z full symmetric). With reuse_v the dense
    // rank-one part reads V = Z * A1 left by the last schur_matrix(Z) call;
    // otherwise it forms Vt = Z * A1 and leaves it for inner_all_sq.
    void inner_all(const double *Z, long ldZ, double *out, bool reuse_v = false);
    // out[j] = <A_j, W^2> for all j: reuse_v as above; reuse_vt reads the Vt =
    // W * A1 left by inner_all(W) just before.
    void inner_all_sq(const double *W, long ldW, double *out, bool reuse_v = false, bool reuse_vt = false);
    // <C, Z>
    double c_inner(const double *Z, long ldZ);
    // W = S^-1 = Kinv^T Kinv (Kinv = L^-1, lower) as the lower part of a BF16x3 split
    // product on the tensor cores, then mirrored to the full matrix. Used in split
    // precision for the blocks that read W (sparse, sparse rank-one and dense
    // coefficients). False if the tensor-core path is unavailable.
    bool split_inverse(const double *Kinv, double *W, long ldW);
    // the Schur build of this cone can run in schur_build_batch (coefficients of the sparse
    // and sparse rank-one classes only)
    bool batchable() const { return nr1d == 0 && ndr == 0; }
};

// One cone's share of a batched Schur build: from W (lower triangle as the GEMM writes it;
// mirrored here as symmetrize_lower does) the Schur block M (ldM x m, zeroed first; null:
// none, as in a corrector build), <A_i, W> into inner, <A_i, W^2> into innersq and tr W into
// trace (null: skipped). Output addresses may be mapped pinned host memory.
struct SchurBuildJob {
    double *W;
    long ldW;
    int n, m;
    double *M;
    long ldM;
    int nsp;
    const int *sp_id, *sp_ptr, *sp_r, *sp_c;
    const double *sp_v;
    int nr1s;
    const int *r1s_id, *r1s_ptr, *r1s_p;
    const double *r1s_a, *r1s_sign;
    double *Vs;
    long ldv;
    double *inner, *innersq, *trace;
    int reuse_vt;   // inner_all_sq's reuse_vt (no effect on these classes; kept for the record)
};
// The builds of jobs[0 .. count) (device array), one CTA each: the operations of
// symmetrize_lower, trace, schur_matrix, inner_all and inner_all_sq for these classes, each
// output entry formed by the same arithmetic as those kernels form it.
void schur_build_batch(cudaStream_t s, const SchurBuildJob *d_jobs, int count);
SchurBuildJob schur_build_job(const SdpDevice &d, double *W, long ldW, double *M, long ldM);

}  // namespace hb
