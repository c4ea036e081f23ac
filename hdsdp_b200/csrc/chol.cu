// Persistent cooperative Cholesky factorisation and triangular inverse.
//
// One cooperative launch covers the whole factorisation: for every 64-column
// panel, block 0 factors the diagonal block (and inverts it), the grid
// synchronises, all blocks solve the panel rows, synchronise, then update the
// trailing lower triangle tile by tile on the DMMA path, and synchronise
// again. A failed pivot (non-positive or NaN, the dpotrf test used by the
// reference's positive-definiteness checks, linalg/hdsdp_linsolver.c:521-553)
// is published in *info and every block leaves at the next grid barrier.
//
// The triangular inverse K = L^-1 uses the same structure on block rows:
// X_i <- Dinv_i X_i, then X_below -= L_below,i X_i.
#include "la.h"
#include <cooperative_groups.h>
#include <mutex>
#include <algorithm>
#include <vector>
#include <utility>

namespace cg = cooperative_groups;

namespace hb {

#ifdef HB_CHOL_STAMPS
// Diagnostic build only (never defined in the library build): per-phase %globaltimer
// stamps of the cooperative factorisation, written by thread 0 of a block.
__device__ unsigned long long *g_chol_stamps = nullptr;
void chol_set_stamps(unsigned long long *p) { cudaMemcpyToSymbol(g_chol_stamps, &p, sizeof(p)); }
#define CHOL_STAMP(slot)                                                  \
    do {                                                                  \
        if (threadIdx.x == 0 && g_chol_stamps && (slot) < 8192) {         \
            unsigned long long t_;                                        \
            asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t_));        \
            g_chol_stamps[(slot)] = t_;                                   \
        }                                                                 \
    } while (0)
#else
#define CHOL_STAMP(slot) \
    do {                 \
    } while (0)
#endif

namespace {
constexpr int NB = 64;

constexpr int TP = 68;                         // tile pitch (conflict-free DMMA fragment reads)
constexpr int SM_DOUBLES = 4 * 64 * TP;        // four 64 x 68 tiles
constexpr int COOP_THREADS = 256;

__device__ __forceinline__ void cpa8(double *sdst, const double *gsrc, bool pred) {
    const unsigned saddr = (unsigned) __cvta_generic_to_shared(sdst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(saddr), "l"(gsrc), "r"(pred ? 8 : 0));
}
__device__ __forceinline__ void cpa_wait_all() {
    asm volatile("cp.async.commit_group;\n" ::);
    asm volatile("cp.async.wait_group 0;\n" ::);
}

// 16-byte copy of which the first `bytes` (0, 8 or 16) come from global memory and the
// rest is zero filled; both addresses 16-byte aligned.
__device__ __forceinline__ void cpa16(double *sdst, const double *gsrc, int bytes) {
    const unsigned saddr = (unsigned) __cvta_generic_to_shared(sdst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(saddr), "l"(gsrc), "r"(bytes));
}

// Stage columns 0..ncols-1 of the 64-row tile G (column-major, pitch ldg) into S (pitch
// TP): entries with row < nr and column < nc are copied, the rest of those columns is
// zero. Two rows move per copy when G and ldg keep every pair 16-byte aligned. The
// caller waits with cpa_wait_all().
__device__ __forceinline__ void stage_tile(double *S, const double *G, long ldg, int nr, int nc, int ncols) {
    if (((((size_t) G) & 15) == 0) && ((ldg & 1) == 0)) {
        for (int idx = threadIdx.x; idx < 32 * ncols; idx += blockDim.x) {
            const int r = (idx & 31) * 2, c = idx >> 5;
            const int cnt = (c < nc) ? min(2, max(0, nr - r)) : 0;
            cpa16(&S[r + c * TP], cnt ? G + (size_t) r + (size_t) c * ldg : G, 8 * cnt);
        }
    } else {
        for (int idx = threadIdx.x; idx < 64 * ncols; idx += blockDim.x) {
            const int r = idx & 63, c = idx >> 6;
            const bool ok = r < nr && c < nc;
            cpa8(&S[r + c * TP], ok ? G + (size_t) r + (size_t) c * ldg : G, ok);
        }
    }
}

__device__ __forceinline__ void dmma_c(double &d0, double &d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}


// ---------------------------------------------------------------------------------
// Diagonal-block factorisation: four 16-column sub-panels. Warp 0 factors and inverts
// each 16 x 16 pivot block in registers; the panel below, the trailing update and the
// off-diagonal blocks of the 64 x 64 inverse are DMMA products in shared memory with
// the other warps.
// ---------------------------------------------------------------------------------
constexpr unsigned FULL = 0xffffffffu;

// Factor T[off.., off..] (16 x 16, lower, pitch TP) in place and write its inverse to
// X[off.., off..]. Executed by one whole warp with two lane roles: lane r < 16 holds row
// r of the block, lane 16 + k holds column k of the inverse (starting as e_k). For each
// column c one set of broadcasts of L(q, c), q > c, drives both the trailing update
// A(r, q) -= L(r, c) L(q, c) and the forward elimination X(q, k) -= L(q, c) X(c, k):
// the two are the same instruction, v[q] -= v[c] L(q, c), on every lane (a lane of the
// second role is never masked by the row test). The broadcasts of a column are issued
// before their uses so that their latencies overlap.
__device__ __forceinline__ bool warp_chol_inv16(double *T, double *X, int off, int lane) {
    const bool row_role = lane < 16;
    double v[16];
#pragma unroll
    for (int q = 0; q < 16; ++q)
        v[q] = row_role ? ((q <= lane) ? T[(off + lane) + (off + q) * TP] : 0.0) : ((q == lane - 16) ? 1.0 : 0.0);
    // one reciprocal square root per column: L_cc = p rsqrt(p), the column below scales
    // by rsqrt(p), and so does row c of the inverse. The pivot of column c + 1 only
    // needs L(c + 1, c), so it is formed first and its reciprocal square root runs
    // while the rest of column c is applied.
    double p = __shfl_sync(FULL, v[0], 0);
    bool bad = !(p > 0.0);
    double rs = rsqrt(p);
    // fixed trip counts keep v[] and lq[] in registers (the loops unroll completely)
#pragma unroll
    for (int c = 0; c < 16; ++c) {
        v[c] = (lane == c) ? p * rs : v[c] * rs;
        double pn = 1.0, rn = 1.0;
        if (c + 1 < 16) {
            // lane c + 1 holds L(c + 1, c) itself: it forms the next pivot without waiting
            // for the broadcast that the other lanes' update of column c + 1 needs (the same
            // fused multiply-add, so the same value as that update gives)
            const double own = v[c + 1] - v[c] * v[c];
            pn = __shfl_sync(FULL, own, c + 1);
            const double l1 = __shfl_sync(FULL, v[c], c + 1);
            if (lane >= c + 1) v[c + 1] -= v[c] * l1;
            if (!(pn > 0.0)) bad = true;
            rn = rsqrt(pn);
        }
        double lq[16];
#pragma unroll
        for (int q = c + 2; q < 16; ++q) lq[q] = __shfl_sync(FULL, v[c], q);
#pragma unroll
        for (int q = c + 2; q < 16; ++q)
            if (lane >= q) v[q] -= v[c] * lq[q];
        p = pn;
        rs = rn;
    }
    if (row_role) {
#pragma unroll
        for (int q = 0; q < 16; ++q)
            if (q <= lane) T[(off + lane) + (off + q) * TP] = v[q];
    } else {
        const int k = lane - 16;
#pragma unroll
        for (int q = 0; q < 16; ++q)
            if (q >= k) X[(off + q) + (off + k) * TP] = v[q];
    }
    return !bad;
}

// C (rows x cols, multiples of 8) = / += alpha * A (rows x K) * op(B), K a multiple of 4,
// in shared memory (pitch TP) on the DMMA path; 8 x 8 tiles dealt to the warps starting
// at warp `w0`. A(r, k) = Ab[r + k*TP]; op(B)(k, c) = bt ? Bb[c + k*TP] : Bb[k + c*TP].
// With lower set, tiles strictly above the diagonal are skipped.
// With nwarp set, only warps w0 .. w0 + nwarp - 1 take part (and all of them must call).
__device__ __forceinline__ void smem_mma(double *Cb, const double *Ab, const double *Bb, int bt, int rows, int cols,
                                         int K, double alpha, bool accumulate, bool lower, int w0 = 0,
                                         int nwarp = 0) {
    const int lane = threadIdx.x & 31, w = (threadIdx.x >> 5) - w0;
    const int nw = nwarp ? nwarp : (int) (blockDim.x >> 5);
    const int tr = rows >> 3, ntile = tr * (cols >> 3);
    for (int t = w; t < ntile; t += nw) {
        const int ti = t % tr, tj = t / tr;
        if (lower && ti < tj) continue;
        double c0 = 0.0, c1 = 0.0;
        for (int k0 = 0; k0 < K; k0 += 4) {
            const int kk = k0 + (lane & 3);
            const double av = Ab[(ti * 8 + (lane >> 2)) + kk * TP];
            const int cc = tj * 8 + (lane >> 2);
            const double bv = bt ? Bb[cc + kk * TP] : Bb[kk + cc * TP];
            dmma_c(c0, c1, av, bv);
        }
        const int r = ti * 8 + (lane >> 2), c = tj * 8 + (lane & 3) * 2;
        if (accumulate) {
            Cb[r + c * TP] += alpha * c0;
            Cb[r + (c + 1) * TP] += alpha * c1;
        } else {
            Cb[r + c * TP] = alpha * c0;
            Cb[r + (c + 1) * TP] = alpha * c1;
        }
    }
}

// Shared-memory regions of the factorisation kernel (64 x TP doubles each): tile
// products use regions 0 and 1; the diagonal-block factorisation keeps its block in
// region 3, the previous panel's rows in region 2 and the inverse in region 1.
constexpr int R_X = 1, R_P = 2, R_T = 3;
__device__ __forceinline__ double *region(double *sm, int r) { return sm + (size_t) r * 64 * TP; }

// Block row i of the inverse of the 64 x 64 diagonal block, off the diagonal:
// X_ij = -X_ii sum_{k=j}^{i-1} L_ik X_kj for j < i (16 x 16 blocks), by warps
// w0 .. w0 + nwarp - 1 (nwarp 0: all warps); `bar` synchronises exactly those warps
// between the two products. Scratch: rows 0-15, columns 16-63 of P.
template <typename Bar>
__device__ __forceinline__ void inverse_block_row(const double *T, double *X, double *P, int i, int w0, int nwarp,
                                                  Bar bar) {
    for (int j = 0; j < i; ++j)
        smem_mma(P + 16 * (j + 1) * TP, T + 16 * i + 16 * j * TP, X + 16 * j + 16 * j * TP, 0, 16, 16, 16 * (i - j),
                 1.0, false, false, w0, nwarp);
    bar();
    for (int j = 0; j < i; ++j)
        smem_mma(X + 16 * i + 16 * j * TP, X + 16 * i + 16 * i * TP, P + 16 * (j + 1) * TP, 0, 16, 16, 16, -1.0,
                 false, false, w0, nwarp);
}

// Factor the nb x nb diagonal block at (j0, j0) and write its inverse to Dinv (64
// columns, zero padded). The block is first updated in shared memory by the previous
// panel's rows, A_jj -= P P^T, when they are given: `staged` (block and rows already in
// regions 3 and 2, copies possibly still in flight) or Pp (nb x 64 rows, pitch ldp,
// staged here). Executed by one block. Returns false (and sets *info) on a failed
// pivot. The strictly upper part of the diagonal block in L holds zeros (copy_lower_k
// and every later write keep it so), which lets whole column segments be staged.
__device__ bool potf2_dev(double *L, long ld, int j0, int nb, double *Dinv, long ldd, int *info, double *sm,
                          const double *Pp = nullptr, long ldp = 0, bool staged = false) {
    double *T = region(sm, R_T), *X = region(sm, R_X), *P = region(sm, R_P);
    __shared__ int fail;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    double *Ljj = L + (size_t) j0 + (size_t) j0 * ld;
    if (!staged) {
        stage_tile(T, Ljj, ld, nb, nb, 64);
        if (Pp) stage_tile(P, Pp, ldp, nb, 64, 64);
    }
    for (int idx = tid; idx < 64 * 64; idx += blockDim.x) X[(idx & 63) + (idx >> 6) * TP] = 0.0;
    cpa_wait_all();
    if (tid == 0) fail = 0;
    for (int r = nb + tid; r < 64; r += blockDim.x) T[r + r * TP] = 1.0;  // pad with the identity
    __syncthreads();
    const int sb = 4096 + (j0 / 64) * 32;
    (void) sb;
    CHOL_STAMP(sb);
    const int nwork = (int) (blockDim.x >> 5) - 1;
    auto bar_workers = [nwork]() { asm volatile("bar.sync 1, %0;\n" ::"r"(32 * nwork) : "memory"); };
    // The update A_jj -= P P^T by the previous panel's rows: warp 0 updates the first 16 x 16
    // diagonal block and starts factoring it while the other warps update the rest (the
    // padded rows of P are zero, so the identity padding survives).
    if (staged || Pp) {
        if (warp == 0) {
            smem_mma(T, P, P, 1, 16, 16, 64, -1.0, true, true, 0, 1);
            __syncwarp();
        } else {
            smem_mma(T + 16, P + 16, P, 1, 48, 16, 64, -1.0, true, false, 1, nwork);
            smem_mma(T + 16 + 16 * TP, P + 16, P + 16, 1, 48, 48, 64, -1.0, true, true, 1, nwork);
        }
    }
    // Four 16-column sweeps with a one-block look-ahead: after sweep s and the panel below
    // it, warp 0 updates only the next diagonal block and goes on to factor it, while the
    // other warps apply the rest of the trailing update (and a block row of the inverse);
    // sweep s + 1 touches only the next diagonal block of T and of X.
    for (int s0 = 0; s0 < 64; s0 += 16) {
        if (warp == 0) {
            const bool ok = warp_chol_inv16(T, X, s0, lane);
            if (lane == 0 && !ok) fail = s0 + 1;
        } else if (s0 >= 32) {
            // block row s0/16 - 1 of the inverse while warp 0 factors block s0/16
            inverse_block_row(T, X, P, s0 / 16 - 1, 1, nwork, bar_workers);
        }
        __syncthreads();
        CHOL_STAMP(sb + 1 + (s0 >> 4) * 2);
        if (fail) break;
        const int rem = 64 - s0 - 16;
        if (rem > 0) {
            // panel below: P = T_below X_ss^T (all warps)
            smem_mma(P + s0 + 16, T + (s0 + 16) + s0 * TP, X + s0 + s0 * TP, 1, rem, 16, 16, 1.0, false, false);
            __syncthreads();
            if (warp == 0) {
                // the next diagonal block and its rows of the panel
                const int r0 = s0 + 16;
                smem_mma(T + r0 + r0 * TP, P + r0, P + r0, 1, 16, 16, 16, -1.0, true, true, 0, 1);
                for (int idx = lane; idx < 256; idx += 32) {
                    const int r = r0 + (idx & 15), c = idx >> 4;
                    T[r + (s0 + c) * TP] = P[r + c * TP];
                }
                __syncwarp();
            } else if (rem > 16) {
                // rows below the next diagonal block: T[r1.., r0..] -= P_rest [P_next; P_rest]^T
                const int r0 = s0 + 16, r1 = s0 + 32, rr = rem - 16;
                smem_mma(T + r1 + r0 * TP, P + r1, P + r0, 1, rr, 16, 16, -1.0, true, false, 1, nwork);
                smem_mma(T + r1 + r1 * TP, P + r1, P + r1, 1, rr, rr, 16, -1.0, true, true, 1, nwork);
                for (int idx = tid - 32; idx < rr * 16; idx += 32 * nwork) {
                    const int r = r1 + (idx & 15) + 16 * (idx >> 8), c = (idx >> 4) & 15;
                    T[r + (s0 + c) * TP] = P[r + c * TP];
                }
            }
        }
        CHOL_STAMP(sb + 2 + (s0 >> 4) * 2);
    }
    if (fail) {
        if (tid == 0) *info = j0 + fail;
        return false;
    }
    // the last block row of the inverse, with all warps
    inverse_block_row(T, X, P, 3, 0, 0, []() { __syncthreads(); });
    __syncthreads();
    CHOL_STAMP(sb + 10);
    // write L (lower part only) and Dinv (zero beyond column nb), two rows per store
    const bool vl = ((((size_t) Ljj) & 15) == 0) && ((ld & 1) == 0);
    const bool vd = ((((size_t) (Dinv + j0)) & 15) == 0) && ((ldd & 1) == 0);
    for (int idx = tid; idx < 32 * 64; idx += blockDim.x) {
        const int r = (idx & 31) * 2, cc = idx >> 5;
        if (r >= nb) continue;
        const bool two = r + 1 < nb;
        if (cc < nb && r + 1 >= cc) {
            double *dst = Ljj + (size_t) r + (size_t) cc * ld;
            if (two && r >= cc && vl) {
                *reinterpret_cast<double2 *>(dst) = make_double2(T[r + cc * TP], T[r + 1 + cc * TP]);
            } else {
                if (r >= cc) dst[0] = T[r + cc * TP];
                if (two) dst[1] = T[r + 1 + cc * TP];
            }
        }
        const double d0 = (cc < nb) ? X[r + cc * TP] : 0.0;
        const double d1 = (cc < nb) ? X[r + 1 + cc * TP] : 0.0;
        double *dd = Dinv + (size_t) (j0 + r) + (size_t) cc * ldd;
        if (two && vd) {
            *reinterpret_cast<double2 *>(dd) = make_double2(d0, d1);
        } else {
            dd[0] = d0;
            if (two) dd[1] = d1;
        }
    }
    __syncthreads();
    CHOL_STAMP(sb + 11);
    return true;
}

// Tile product on the DMMA path over K = nb <= 64:
//   mode 0:  C -= A * op(B)      mode 1:  C = A * op(B)      mode 2:  C = -A * op(B)
// A(r, k) = A[r + k*lda]; op(B)(k, c) = bt ? B[c + k*ldb] : B[k + c*ldb].
// C is the 64 x 64 tile at C (pitch ldc) clipped to mr x nc; with diag set only
// row >= col entries are written.
struct TileJob {
    double *C;
    long ldc;
    int mr, nc;
    const double *A;
    long lda;
    int ar;
    const double *B;
    long ldb;
    int bt, bc, nb;
    bool diag;
    int mode;
};

// Issue the copies of a job's operands into As / Bs (pitch TP, zero padded).
__device__ __forceinline__ void stage_job(const TileJob &J, double *As, double *Bs) {
    const int kp = (J.nb + 3) & ~3;
    stage_tile(As, J.A, J.lda, J.ar, J.nb, kp);
    if (J.bt) {
        stage_tile(Bs, J.B, J.ldb, J.bc, J.nb, kp);
    } else {
        for (int idx = threadIdx.x; idx < 64 * kp; idx += blockDim.x) {
            const int r = idx & 63, k = idx >> 6;
            const bool okb = r < J.bc && k < J.nb;
            cpa8(&Bs[r + k * TP], okb ? J.B + (size_t) k + (size_t) r * J.ldb : J.B, okb);
        }
    }
}

// This thread's C entries of a mode-0 job (zero otherwise), in fragment order.
__device__ __forceinline__ void load_c(const TileJob &J, double (&cv)[4][2][2]) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int wm = (w & 1) * 32, wn = (w >> 1) * 16;
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j)
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const int r = wm + i * 8 + (lane >> 2), c = wn + j * 8 + (lane & 3) * 2 + e;
                cv[i][j][e] = (J.mode == 0 && r < J.mr && c < J.nc && !(J.diag && r < c))
                                  ? J.C[(size_t) r + (size_t) c * J.ldc]
                                  : 0.0;
            }
}

// acc = As * Bs^T over k < kp (8 warps: a 32 x 16 block of 8 x 8 DMMA tiles each).
__device__ __forceinline__ void dmma_tile(const double *As, const double *Bs, int kp, double (&acc)[4][2][2]) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int wm = (w & 1) * 32, wn = (w >> 1) * 16;
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
    for (int k = 0; k < kp; k += 4) {
        const int kk = k + (lane & 3);
        double a[4], b[2];
#pragma unroll
        for (int i = 0; i < 4; ++i) a[i] = As[(wm + i * 8 + (lane >> 2)) + kk * TP];
#pragma unroll
        for (int j = 0; j < 2; ++j) b[j] = Bs[(wn + j * 8 + (lane >> 2)) + kk * TP];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 2; ++j) dmma_c(acc[i][j][0], acc[i][j][1], a[i], b[j]);
    }
}

// Write the job's result; with Ct also transposed to Ct (pitch ldct), with Csm also
// into shared memory (pitch TP, zeros outside the written entries).
__device__ __forceinline__ void store_tile(const TileJob &J, const double (&cv)[4][2][2],
                                           const double (&acc)[4][2][2], double *Ct, long ldct, double *Csm) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int wm = (w & 1) * 32, wn = (w >> 1) * 16;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int r = wm + i * 8 + (lane >> 2);
#pragma unroll
        for (int j = 0; j < 2; ++j)
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const int c = wn + j * 8 + (lane & 3) * 2 + e;
                const bool valid = r < J.mr && c < J.nc && !(J.diag && r < c);
                const double val =
                    (J.mode == 0) ? cv[i][j][e] - acc[i][j][e] : (J.mode == 2) ? -acc[i][j][e] : acc[i][j][e];
                if (valid) {
                    J.C[(size_t) r + (size_t) c * J.ldc] = val;
                    if (Ct) Ct[(size_t) c + (size_t) r * ldct] = val;
                }
                if (Csm) Csm[r + c * TP] = valid ? val : 0.0;
            }
    }
}

// One tile product with its operands staged in regions 0 and 1. Operands are staged
// first, so C may alias A or B (in-place panel solves).
__device__ void tile_mma_dev(double *Cb, long ldc, int mr, int nc, const double *Ab, long lda, int ar,
                             const double *Bb, long ldb, int bt, int bc, int nb, bool diag, int mode, double *sm,
                             double *Ct = nullptr, long ldct = 0, double *Csm = nullptr) {
    const TileJob J{Cb, ldc, mr, nc, Ab, lda, ar, Bb, ldb, bt, bc, nb, diag, mode};
    double *As = sm, *Bs = sm + 64 * TP;
    stage_job(J, As, Bs);
    double cv[4][2][2];
    load_c(J, cv);  // while the operand copies are in flight
    cpa_wait_all();
    __syncthreads();
    double acc[4][2][2];
    dmma_tile(As, Bs, (nb + 3) & ~3, acc);
    store_tile(J, cv, acc, Ct, ldct, Csm);
    __syncthreads();
}

// Mode-0 jobs t0, t0 + step, ... (< t1) of one block, double buffered: the operands
// of the next job are copied into the other pair of regions (0/1 and 2/3) and its C
// entries loaded into registers while the current job's products run. The jobs'
// C tiles must be disjoint from each other and from every operand.
template <typename JobOf>
__device__ void tile_stream(JobOf job_of, long t0, long t1, long step, double *sm) {
    if (t0 >= t1) return;
    TileJob cur, nxt;
    job_of(t0, cur);
    int b = 0;
    stage_job(cur, sm + (size_t) (2 * b) * 64 * TP, sm + (size_t) (2 * b + 1) * 64 * TP);
    asm volatile("cp.async.commit_group;\n" ::);
    double cv[4][2][2], cvn[4][2][2];
    load_c(cur, cv);
    for (long t = t0;; t += step) {
        const bool more = t + step < t1;
        if (more) {
            job_of(t + step, nxt);
            stage_job(nxt, sm + (size_t) (2 * (b ^ 1)) * 64 * TP, sm + (size_t) (2 * (b ^ 1) + 1) * 64 * TP);
            asm volatile("cp.async.commit_group;\n" ::);
            load_c(nxt, cvn);
            asm volatile("cp.async.wait_group 1;\n" ::);
        } else {
            asm volatile("cp.async.wait_group 0;\n" ::);
        }
        __syncthreads();
        double acc[4][2][2];
        dmma_tile(sm + (size_t) (2 * b) * 64 * TP, sm + (size_t) (2 * b + 1) * 64 * TP, (cur.nb + 3) & ~3, acc);
        store_tile(cur, cv, acc, nullptr, 0, nullptr);
        __syncthreads();  // the buffer just read may be refilled
        if (!more) break;
        cur = nxt;
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                cv[i][j][0] = cvn[i][j][0];
                cv[i][j][1] = cvn[i][j][1];
            }
        b ^= 1;
    }
}

__device__ __forceinline__ void tri_index(long t, int &ti, int &tj) {
    ti = (int) ((sqrt(8.0 * (double) t + 1.0) - 1.0) * 0.5);
    while ((long) ti * (ti + 1) / 2 > t) --ti;
    while ((long) (ti + 1) * (ti + 2) / 2 <= t) ++ti;
    tj = (int) (t - (long) ti * (ti + 1) / 2);
}

// Right-looking blocked Cholesky with one-panel look-ahead: in the update phase of
// panel j, block 0 first updates the diagonal tile of panel j+1 and factors it while
// the other blocks update the rest of the trailing matrix.
//
// With K set, the inverse factor K = L^-1 (and KT = K^T) is formed alongside, right
// looking by 64-row blocks, on the blocks that would otherwise wait for block 0:
// while panel j is solved, the rows below block j-1 of K receive
// X(r, c) -= L(r, j-1) K(j-1, c) (the first update of a tile assigns -L K); while the
// trailing matrix is updated, block row j is finalised as K(j, c) = Dinv_j X(j, c) and
// K(j, j) = Dinv_j. The strictly upper blocks of K and the strictly lower blocks of KT
// are never written (they must hold zeros).
__device__ __forceinline__ void k_update_tile(const double *L, long ld, double *K, int n, int r, int c, int k,
                                              double *sm) {
    const int mr = min(64, n - 64 * r);
    tile_mma_dev(K + (size_t) 64 * r + (size_t) 64 * c * ld, ld, mr, 64, L + (size_t) 64 * r + (size_t) 64 * k * ld,
                 ld, mr, K + (size_t) 64 * k + (size_t) 64 * c * ld, ld, 0, 64, 64, false, (k == c) ? 2 : 0, sm);
}

__device__ __forceinline__ void k_final_tile(const double *Dinv, long ldd, double *K, double *KT, long ld, int n,
                                             int bj, int c, double *sm) {
    const int mr = min(64, n - 64 * bj);
    if (c < bj) {
        double *X = K + (size_t) 64 * bj + (size_t) 64 * c * ld;
        tile_mma_dev(X, ld, mr, 64, Dinv + (size_t) 64 * bj, ldd, mr, X, ld, 0, 64, mr, false, 1, sm,
                     KT + (size_t) 64 * c + (size_t) 64 * bj * ld, ld);
    } else {
        for (int idx = threadIdx.x; idx < 64 * 64; idx += blockDim.x) {
            const int r = idx & 63, cc = idx >> 6;
            if (r < mr && cc < mr) {
                const double v = Dinv[(size_t) (64 * bj + r) + (size_t) cc * ldd];
                K[(size_t) (64 * bj + r) + (size_t) (64 * bj + cc) * ld] = v;
                KT[(size_t) (64 * bj + cc) + (size_t) (64 * bj + r) * ld] = v;
            }
        }
        __syncthreads();
    }
}

// The factorisation on a grid of ngrid blocks, this one being block bid; gsync() is the
// grid-wide barrier, garrive() / gwait(token) its two halves. The cooperative kernel runs it
// on its grid; a batched launch runs it with one block per matrix (bid 0, ngrid 1, gsync a
// block barrier). Every tile is computed by the same operations whatever the grid, so the
// result does not depend on it.
template <class GSync, class GArrive, class GWait>
__device__ void potrf_body(double *L, long ld, int n, double *Dinv, long ldd, int *info, double *K, double *KT,
                           int bid, int ngrid, GSync gsync, GArrive garrive, GWait gwait, double *sm) {
    const int nblk = (n + 63) / 64;
    if (bid == 0) potf2_dev(L, ld, 0, min(NB, n), Dinv, ldd, info, sm);
    gsync();
    for (int j0 = 0; j0 < n; j0 += NB) {
        if (*(volatile int *) info) return;
        const int nb = min(NB, n - j0);
        const int rows = n - j0 - nb;
        if (rows <= 0) break;
        const int bj = j0 / 64;
        double *P = L + (size_t) (j0 + nb) + (size_t) j0 * ld;
        const int nchunk = (rows + 63) / 64;
        const int pb = (j0 / 64) * 16 + (bid == 1 ? 8 : 0);
        (void) pb;
        if (bid <= 1) CHOL_STAMP(pb + 0);
        // panel solve; with K, the update of K's rows r >= bj by block row bj - 1
        const long nx = (K && bj >= 1) ? (long) (nblk - bj) * bj : 0;
        // block 0 stages the next diagonal block now (its updates by earlier panels are
        // complete) and keeps its own solved chunk 0, the rows that update that block
        const int nbn = min(NB, rows);
        if (bid == 0)
            stage_tile(region(sm, R_T), L + (size_t) (j0 + nb) + (size_t) (j0 + nb) * ld, ld, nbn, nbn, 64);
        for (long t = bid; t < nchunk + nx; t += ngrid) {
            if (t < nchunk) {
                const int ch = (int) t;
                const int mr = min(64, rows - ch * 64);
                tile_mma_dev(P + ch * 64, ld, mr, nb, P + ch * 64, ld, mr, Dinv + j0, ldd, 1, nb, nb, false, 1, sm,
                             nullptr, 0, (t == 0) ? region(sm, R_P) : nullptr);
            } else {
                const long u = t - nchunk;
                k_update_tile(L, ld, K, n, bj + (int) (u / bj), (int) (u % bj), bj - 1, sm);
            }
        }
        if (bid <= 1) CHOL_STAMP(pb + 1);
        // block 0 goes on to the next diagonal block, which needs only what it holds itself
        // (its solved chunk 0 and the staged block): it arrives at the barrier without waiting,
        // and waits for it only after that factorisation
        const bool early = (bid == 0 && ngrid > 1);
        unsigned int tok = 0;
        if (early) tok = garrive();
        else gsync();
        if (bid <= 1) CHOL_STAMP(pb + 2);
        const long ntile = (long) nchunk * (nchunk + 1) / 2;
        const long nk = K ? bj + 1 : 0;
        double *A22 = L + (size_t) (j0 + nb) + (size_t) (j0 + nb) * ld;
        if (bid == 0) {
            // tile (0, 0) is the next diagonal block: update it in shared memory and factor it
            CHOL_STAMP(pb + 3);
            potf2_dev(L, ld, j0 + nb, nbn, Dinv, ldd, info, sm, nullptr, 0, true);
            CHOL_STAMP(pb + 4);
        }
        if (early) gwait(tok);
        // remaining tiles (and K's block row bj), spread over the other blocks
        // (block 0 joins when the grid has one block)
        const int nworker = (ngrid > 1) ? (int) ngrid - 1 : 1;
        const int wid = (ngrid > 1) ? (int) bid - 1 : 0;
        if (wid >= 0) {
            auto trailing = [&](long t, TileJob &J) {
                int ti, tj;
                tri_index(t, ti, tj);
                const int mr = min(64, rows - ti * 64), nc = min(64, rows - tj * 64);
                J = TileJob{A22 + (size_t) ti * 64 + (size_t) tj * 64 * ld, ld, mr, nc, P + ti * 64, ld, mr,
                            P + tj * 64, ld, 1, nc, nb, ti == tj, 0};
            };
            tile_stream(trailing, 1 + wid, ntile, nworker, sm);
            for (long t = 1 + wid; t < ntile + nk; t += nworker)
                if (t >= ntile) k_final_tile(Dinv, ldd, K, KT, ld, n, bj, (int) (t - ntile), sm);
        }
        if (bid == 1) CHOL_STAMP(pb + 3);
        gsync();
        if (bid <= 1) CHOL_STAMP(pb + 5);
    }
    if (!K || *(volatile int *) info) return;
    // the last block row of K: its update by block row nblk - 2, then its final form
    const int bj = nblk - 1;
    if (bj >= 1) {
        for (int c = bid; c < bj; c += ngrid) k_update_tile(L, ld, K, n, bj, c, bj - 1, sm);
        gsync();
    }
    for (int c = bid; c <= bj; c += ngrid) k_final_tile(Dinv, ldd, K, KT, ld, n, bj, c, sm);
}

__global__ void __launch_bounds__(COOP_THREADS, 1) potrf_coop_kernel(double *L, long ld, int n, double *Dinv,
                                                                  long ldd, int *info, double *K, double *KT) {
    cg::grid_group grid = cg::this_grid();
    extern __shared__ double sm[];
    potrf_body(
        L, ld, n, Dinv, ldd, info, K, KT, (int) blockIdx.x, (int) gridDim.x, [&]() { grid.sync(); },
        [&]() { return grid.barrier_arrive(); }, [&](unsigned int t) { grid.barrier_wait(std::move(t)); }, sm);
}

// Several factorisations in one launch, one CTA each: the copy of the lower triangle, the
// factorisation of the cooperative kernel on a grid of one block (with K = L^-1 and K^T for
// a fused factor), and sum log L_ii next to the info word as the log-diagonal kernel forms
// it; the results are those of the cooperative kernel on any grid.
struct SmallFactorJob {
    const double *S;
    double *L, *Dinv, *K, *KT;
    long lds, ld;
    int *info;
    double *hinfo;   // device address of the factor's pinned status words (written directly)
    int n, logdet;
};
constexpr int kSmallBatch = 36;
struct SmallFactorBatch {
    SmallFactorJob job[kSmallBatch];
};

// sum_i log L_ii (n <= 1024) summed as the log-diagonal kernel sums it with its 1024
// threads (one term per thread, a shuffle tree per warp, then one over the 32 warp sums),
// by COOP_THREADS threads each standing in for four: the same additions in the same order.
__device__ double logdiag_1024(int n, const double *L, long ld) {
    __shared__ double red[32];
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    constexpr int kV = 1024 / COOP_THREADS;
#pragma unroll
    for (int q = 0; q < kV; ++q) {
        const int v = t + COOP_THREADS * q;
        double x = (v < n) ? log(L[(size_t) v + (size_t) v * ld]) : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if (lane == 0) red[w + (COOP_THREADS / 32) * q] = x;
    }
    __syncthreads();
    double x = 0.0;
    if (w == 0) {
        x = red[lane];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    }
    __syncthreads();
    return x;
}

__device__ void small_factor_job(const SmallFactorJob &J, double *sm) {
    const int n = J.n;
    for (int idx = threadIdx.x; idx < n * n; idx += blockDim.x) {
        const int r = idx % n, c = idx / n;
        J.L[(size_t) r + (size_t) c * J.ld] = (r >= c) ? J.S[(size_t) r + (size_t) c * J.lds] : 0.0;
    }
    if (threadIdx.x == 0) *J.info = 0;
    __threadfence_block();
    __syncthreads();
    potrf_body(
        J.L, J.ld, n, J.Dinv, J.ld, J.info, J.K, J.KT, 0, 1, []() { __syncthreads(); },
        []() {
            __syncthreads();
            return 0u;
        },
        [](unsigned int) {}, sm);
    __syncthreads();
    double acc = 0.0;
    if (J.logdet) {
        __threadfence_block();
        __syncthreads();
        acc = logdiag_1024(n, J.L, J.ld);
        if (threadIdx.x == 0) reinterpret_cast<double *>(J.info)[1] = acc;
    }
    if (threadIdx.x == 0) {
        // the status words straight into the host's pinned mirror
        const int v = *(volatile int *) J.info;
        reinterpret_cast<volatile int *>(J.hinfo)[0] = v;
        if (J.logdet) J.hinfo[1] = acc;
    }
}

__global__ void __launch_bounds__(COOP_THREADS, 1) potrf_small_batch_kernel(const SmallFactorBatch B) {
    extern __shared__ double sm[];
    small_factor_job(B.job[blockIdx.x], sm);
}

// the same, the jobs in global memory (more than fit the parameters)
__global__ void __launch_bounds__(COOP_THREADS, 1) potrf_batch_array_kernel(const SmallFactorJob *__restrict__ jobs) {
    extern __shared__ double sm[];
    const SmallFactorJob J = jobs[blockIdx.x];
    small_factor_job(J, sm);
}

__global__ void __launch_bounds__(COOP_THREADS, 1) trtri_coop_kernel(const double *L, double *K, long ld, int n,
                                                                  const double *Dinv, long ldd) {
    cg::grid_group grid = cg::this_grid();
    extern __shared__ double sm[];
    for (int i0 = 0; i0 < n; i0 += NB) {
        const int nb = min(NB, n - i0);
        const int cend = i0 + nb;
        const int nchunk = (cend + 63) / 64;
        for (int ch = blockIdx.x; ch < nchunk; ch += gridDim.x) {
            // X_i chunk <- Dinv_i * X_i chunk  (in place)
            const int nc = min(64, cend - ch * 64);
            double *Xc = K + i0 + (size_t) ch * 64 * ld;
            tile_mma_dev(Xc, ld, nb, nc, Dinv + i0, ldd, nb, Xc, ld, 0, nc, nb, false, 1, sm);
        }
        grid.sync();
        const int rows = n - cend;
        if (rows <= 0) break;
        const int rt = (rows + 63) / 64;
        const long ntile = (long) rt * nchunk;
        // C = K[cend + 64 ti.., 64 tj..] -= L[cend + 64 ti.., i0..i0+nb) * K[i0..i0+nb, 64 tj..]
        auto update = [&](long t, TileJob &J) {
            const int ti = (int) (t % rt), tj = (int) (t / rt);
            const int mr = min(64, rows - ti * 64), nc = min(64, cend - tj * 64);
            J = TileJob{K + (size_t) (cend + ti * 64) + (size_t) tj * 64 * ld, ld, mr, nc,
                        L + (size_t) (cend + ti * 64) + (size_t) i0 * ld, ld, mr, K + i0 + (size_t) tj * 64 * ld, ld,
                        0, nc, nb, false, 0};
        };
        tile_stream(update, blockIdx.x, ntile, gridDim.x, sm);
        grid.sync();
    }
}

// Blocked substitution for L L^T x = b, one cooperative launch. The 64-row blocks of
// the vector are dealt to the CTAs (block k to CTA k mod grid); a CTA keeps, in shared
// memory, the accumulated products of its unfinished blocks with the solved ones.
// Forward sweep: the owner of block j forms t_j = Dinv_j (b_j - acc_j) and publishes it
// with flag_f[j] = epoch; every CTA then adds L_kj t_j to its unfinished blocks. The
// chain from block to block is kept short: each CTA prefetches into shared memory the
// tile L_{k,k-1} and Dinv_k of its next block k while it works on older ones, and when
// t_{k-1} appears it finishes and publishes block k before any other update. The other
// updates of a step are one pass over all of the CTA's unfinished blocks (many loads in
// flight). After a grid barrier the backward sweep does the same from the last block up
// with L^T and Dinv^T. Every wait on a flag is bounded; on giving up the CTA raises
// g_tri_err and the others skip their work (every CTA still reaches the grid barrier).
__device__ int g_tri_err = 0;
constexpr long TRI_WAIT_LIMIT = 1L << 22;

__device__ __forceinline__ bool tri_wait(const unsigned *flag, unsigned epoch) {
    for (long it = 0; it < TRI_WAIT_LIMIT; ++it) {
        if ((int) (*(volatile const unsigned *) flag - epoch) >= 0) return true;
        if ((it & 1023) == 1023 && *(volatile int *) &g_tri_err) return false;
    }
    atomicExch(&g_tri_err, 1);
    return false;
}

__global__ void __launch_bounds__(COOP_THREADS, 1)
    tri_solve_coop_kernel(const double *__restrict__ L, long ld, int n, const double *__restrict__ Dinv, long ldd,
                          const double *b, double *t, double *x, unsigned *flag_f, unsigned *flag_b,
                          unsigned epoch) {
    cg::grid_group grid = cg::this_grid();
    extern __shared__ double sm[];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int G = gridDim.x, me = blockIdx.x;
    const int nblk = (n + 63) / 64;
    const int nown = (me < nblk) ? (nblk - 1 - me) / G + 1 : 0;
    double *Lt = sm;                       // 64 x TP: the tile that feeds the next block
    double *Dt = sm + 64 * TP;             // 64 x TP: that block's Dinv
    double *acc = sm + 2 * 64 * TP;        // nown x 64
    double *xs = acc + (size_t) nown * 64; // the solved block being applied
    double *xn = xs + 64;                  // the block this CTA just published
    double *red = xn + 64;                 // 4 x 64 partial sums
    __shared__ int abort_;
    if (tid == 0) abort_ = 0;
    auto kof = [&](int c) { return me + c * G; };
    auto nbof = [&](int j) { return min(64, n - 64 * j); };
    auto fetch = [&](const double *v, int j, const unsigned *flag) {
        if (tid == 0 && !tri_wait(flag + j, epoch)) abort_ = 1;
        __threadfence();
        __syncthreads();
        if (tid < 64) xs[tid] = (!abort_ && tid < nbof(j)) ? __ldcg(v + 64 * j + tid) : 0.0;
        __syncthreads();
    };
    auto take_next = [&]() {
        if (tid < 64) xs[tid] = xn[tid];
        __syncthreads();
    };
    // v = rhs_k - acc_c; out_k = Dt v (transpose: Dt^T v) into xn and out, then publish
    auto finish = [&](int c, const double *rhs, double *out, bool transpose, unsigned *flag) {
        const int k = kof(c), nb = nbof(k);
        double *a = acc + (size_t) c * 64;
        if (tid < 64) red[tid] = (tid < nb) ? rhs[64 * k + tid] - a[tid] : 0.0;
        __syncthreads();
        for (int o = warp; o < 64; o += 8) {
            double sum = 0.0;
            for (int q = lane; q < 64; q += 32) sum += (transpose ? Dt[q + o * TP] : Dt[o + q * TP]) * red[q];
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, off);
            if (lane == 0) xn[o] = (o < nb) ? sum : 0.0;
        }
        __syncthreads();
        if (tid < nb) out[64 * k + tid] = xn[tid];
        __threadfence();
        __syncthreads();
        if (tid == 0) atomicExch(flag + k, epoch);
    };
    auto wait_tiles = [&]() {
        asm volatile("cp.async.wait_all;\n" ::);
        __syncthreads();
    };

    // ---- forward sweep: t = L^-1 b
    for (int i = tid; i < nown * 64; i += blockDim.x) acc[i] = 0.0;
    __syncthreads();
    if (nown > 0 && !*(volatile int *) &g_tri_err) {
        // next block k: L_{k,k-1} (rows of k, columns of k-1) and Dinv_k
        auto prefetch_f = [&](int k) {
            if (k > 0) stage_tile(Lt, L + (size_t) (64 * k) + (size_t) (64 * (k - 1)) * ld, ld, nbof(k), 64, 64);
            stage_tile(Dt, Dinv + (size_t) (64 * k), ldd, nbof(k), nbof(k), 64);
            asm volatile("cp.async.commit_group;\n" ::);
        };
        int c = 0;
        bool have = false;
        prefetch_f(kof(0));
        if (me == 0) {
            wait_tiles();
            finish(0, b, t, false, flag_f);
            have = true;
            c = 1;
            if (c < nown) prefetch_f(kof(c));
        }
        const int last = kof(nown - 1);
        for (int j = 0; j < last && !abort_; ++j) {
            if (have) {
                take_next();
                have = false;
            } else {
                fetch(t, j, flag_f);
                if (abort_) break;
            }
            if (c < nown && kof(c) == j + 1) {
                // the next block: acc += L_{j+1,j} t_j from the prefetched tile, then finish it
                wait_tiles();
                {
                    const int r = tid & 63, q = tid >> 6;
                    double sum = 0.0;
#pragma unroll
                    for (int cc = 16 * q; cc < 16 * q + 16; ++cc) sum += Lt[r + cc * TP] * xs[cc];
                    red[q * 64 + r] = sum;
                }
                __syncthreads();
                if (tid < 64) acc[(size_t) c * 64 + tid] += red[tid] + red[64 + tid] + red[128 + tid] + red[192 + tid];
                __syncthreads();
                finish(c, b, t, false, flag_f);
                have = true;
                ++c;
                if (c < nown) prefetch_f(kof(c));
            }
            // every other unfinished block (all beyond block j + 1): acc_k += L_kj t_j
            for (int item = tid; item < (nown - c) * 64; item += blockDim.x) {
                const int cc = c + (item >> 6), r = item & 63, k = kof(cc);
                if (r >= nbof(k)) continue;
                const double *row = L + (size_t) (64 * k + r) + (size_t) (64 * j) * ld;
                double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
#pragma unroll 4
                for (int q = 0; q < 64; q += 4) {
                    s0 += row[(size_t) q * ld] * xs[q];
                    s1 += row[(size_t) (q + 1) * ld] * xs[q + 1];
                    s2 += row[(size_t) (q + 2) * ld] * xs[q + 2];
                    s3 += row[(size_t) (q + 3) * ld] * xs[q + 3];
                }
                acc[(size_t) cc * 64 + r] += (s0 + s1) + (s2 + s3);
            }
            __syncthreads();
        }
    }
    asm volatile("cp.async.wait_all;\n" ::);
    grid.sync();
    // ---- backward sweep: x = L^-T t
    for (int i = tid; i < nown * 64; i += blockDim.x) acc[i] = 0.0;
    __syncthreads();
    if (nown > 0 && !*(volatile int *) &g_tri_err) {
        // next block k (downwards): L_{k+1,k} (rows of k+1, columns of k) and Dinv_k
        auto prefetch_b = [&](int k) {
            if (k < nblk - 1) stage_tile(Lt, L + (size_t) (64 * (k + 1)) + (size_t) (64 * k) * ld, ld, nbof(k + 1), 64, 64);
            stage_tile(Dt, Dinv + (size_t) (64 * k), ldd, nbof(k), nbof(k), 64);
            asm volatile("cp.async.commit_group;\n" ::);
        };
        int c = nown - 1;
        bool have = false;
        prefetch_b(kof(c));
        if (kof(c) == nblk - 1) {
            wait_tiles();
            finish(c, t, x, true, flag_b);
            have = true;
            --c;
            if (c >= 0) prefetch_b(kof(c));
        }
        for (int j = nblk - 1; j > me && !abort_; --j) {
            if (have) {
                take_next();
                have = false;
            } else {
                fetch(x, j, flag_b);
                if (abort_) break;
            }
            if (c >= 0 && kof(c) == j - 1) {
                // the next block: acc += L_{j,j-1}^T x_j from the prefetched tile, then finish it
                wait_tiles();
                for (int o = warp; o < 64; o += 8) {
                    double sum = 0.0;
                    for (int q = lane; q < 64; q += 32) sum += Lt[q + o * TP] * xs[q];
#pragma unroll
                    for (int off = 16; off > 0; off >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, off);
                    if (lane == 0) acc[(size_t) c * 64 + o] += sum;
                }
                __syncthreads();
                finish(c, t, x, true, flag_b);
                have = true;
                --c;
                if (c >= 0) prefetch_b(kof(c));
            }
            // every other unfinished block (all below block j - 1): acc_k += L_jk^T x_j,
            // a warp per output column, four columns at a time
            const int nbj = nbof(j);
            for (int item = warp * 4; item < (c + 1) * 64; item += 32) {
                double s4[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int cc = (item + u) >> 6, o = (item + u) & 63, k = kof(cc);
                    const double *col = L + (size_t) (64 * j) + (size_t) (64 * k + o) * ld;
                    for (int q = lane; q < nbj; q += 32) s4[u] += col[q] * xs[q];
                }
#pragma unroll
                for (int u = 0; u < 4; ++u) {
#pragma unroll
                    for (int off = 16; off > 0; off >>= 1) s4[u] += __shfl_xor_sync(0xffffffffu, s4[u], off);
                }
                if (lane == 0) {
#pragma unroll
                    for (int u = 0; u < 4; ++u) acc[(size_t) ((item + u) >> 6) * 64 + ((item + u) & 63)] += s4[u];
                }
            }
            __syncthreads();
        }
    }
    asm volatile("cp.async.wait_all;\n" ::);
}

__global__ void copy_lower_k(int n, const double *S, long lds, double *L, long ldl) {
    const long total = (long) n * n;
    for (long idx = blockIdx.x * (long) blockDim.x + threadIdx.x; idx < total; idx += (long) gridDim.x * blockDim.x) {
        const int r = (int) (idx % n), c = (int) (idx / n);
        L[(size_t) r + (size_t) c * ldl] = (r >= c) ? S[(size_t) r + (size_t) c * lds] : 0.0;
    }
}

__global__ void identity_k(int n, double *A, long lda) {
    const long total = (long) n * n;
    for (long idx = blockIdx.x * (long) blockDim.x + threadIdx.x; idx < total; idx += (long) gridDim.x * blockDim.x) {
        const int r = (int) (idx % n), c = (int) (idx / n);
        A[(size_t) r + (size_t) c * lda] = (r == c) ? 1.0 : 0.0;
    }
}

__global__ void zero_info_k(int *p) { *p = 0; }

int sm_count() { return device_sm_count(); }

int coop_grid(const void *fn) {
    // resident cooperative CTAs, per device and kernel (two kernels use this)
    static std::atomic<int> cached[kMaxDevices][2];
    const int slot = (fn == (const void *) potrf_coop_kernel) ? 0 : 1;
    const int dev = current_device();
    int v = cached[dev][slot].load(std::memory_order_acquire);
    if (v) return v;
    static std::atomic<unsigned long long> init[2];
    once_per_device(init[slot], [&] {
        const int smem = SM_DOUBLES * (int) sizeof(double);
        HB_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        int per = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, COOP_THREADS, smem);
        cached[dev][slot].store(std::max(1, device_sm_count() * std::max(per, 1)), std::memory_order_release);
    });
    return cached[dev][slot].load(std::memory_order_acquire);
}

int grid_for_n(long total) {
    long b = (total + 255) / 256;
    return (int) std::min<long>(std::max<long>(b, 1), 148L * 16);
}
}  // namespace

bool coop_factorize_enqueue(cudaStream_t s, DenseFactor &F, const double *S, long ldS) {
    const int n = F.n;
    zero_info_k<<<hb::counted(1), 1, 0, s>>>(F.d_info);
    copy_lower_k<<<hb::counted(grid_for_n((long) n * n)), 256, 0, s>>>(n, S, ldS, F.L, F.ld);
    const void *fn = (const void *) potrf_coop_kernel;
    const long t0 = (long) ((n - 1) / 64 + 1);
    // with the fused inverse, the update of K's rows needs up to t0^2 / 4 tiles per phase
    // at most one block per SM, so that the block factoring the diagonal never shares an SM
    const long want = F.fuse_k ? t0 * (t0 + 1) / 2 + t0 * t0 / 4 : t0 * (t0 + 1) / 2;
    const int grid = (int) std::max(1L, std::min<long>(std::min(coop_grid(fn), sm_count()), want));
    double *Lp = F.L;
    long ld = F.ld;
    int nn = n;
    double *Dp = F.Dinv;
    long ldd = F.ld;
    int *ip = F.d_info;
    double *Kp = F.fuse_k ? F.K : nullptr;
    double *KTp = F.fuse_k ? F.KT : nullptr;
    void *args[] = {&Lp, &ld, &nn, &Dp, &ldd, &ip, &Kp, &KTp};
    const bool timed = kstat_on(F.kfamily);
    if (timed) kstat_begin(F.kfamily, s, (double) n * n * n / 3.0);
    cudaError_t e = cudaLaunchCooperativeKernel(fn, hb::counted(grid), COOP_THREADS, args, SM_DOUBLES * sizeof(double), s);
    if (timed) kstat_end(s);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return true;
}

// ---- recursive blocked form (orders above kRecLeafMaxN, with K = L^-1) ----------------
//   L11 L11^T = A11 (recursively; a block of at most kRecLeafMaxN rows on the cooperative
//   kernel, which also forms its K and K^T), L21 = A21 K11^T, A22 -= L21 L21^T,
//   L22 L22^T = A22 (recursively), K21 = -K22 (L21 K11), KT12 = K21^T.
// The split falls on a 64-row boundary, so every diagonal block's 64 x 64 inverses land in
// Dinv where the one-launch factorisation puts them. Each diagonal block reports its status
// in a word of its own; the first failure (with its global pivot index) becomes the
// factor's status.
namespace {
constexpr int kRecMaxLeaves = 128;
struct RecLeaves {
    int off[kRecMaxLeaves];
    int count;
};

__global__ void rec_info_kernel(const RecLeaves R, const int *leaf_info, int *info) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    int v = 0;
    for (int q = 0; q < R.count && v == 0; ++q)
        if (leaf_info[q] != 0) v = leaf_info[q] + R.off[q];
    *info = v;
}

// B (cols x rows) = A^T for A rows x cols
__global__ void transpose_rect_kernel(int rows, int cols, const double *A, long lda, double *B, long ldb) {
    __shared__ double tile[32][33];
    const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        const int r = bx + threadIdx.x, c = by + j;
        if (r < rows && c < cols) tile[j][threadIdx.x] = A[(size_t) r + (size_t) c * lda];
    }
    __syncthreads();
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        const int r = by + threadIdx.x, c = bx + j;   // B(r, c) = A(c, r)
        if (r < cols && c < rows) B[(size_t) r + (size_t) c * ldb] = tile[threadIdx.x][j];
    }
}

int rec_split(int n) { return ((n / 2) / 64) * 64; }

// the diagonal block [off, off + n) of F on the cooperative kernel, its K and K^T into Kp / KTp
// (leading dimension F.ld)
bool rec_leaf(cudaStream_t s, DenseFactor &F, int off, int n, double *Kp, double *KTp, RecLeaves &R) {
    if (R.count >= kRecMaxLeaves) return false;
    DenseFactor V;   // a view of the diagonal block in F's buffers (never released)
    V.n = n;
    V.ld = F.ld;
    V.L = F.L + off + (size_t) off * F.ld;
    V.Dinv = F.Dinv + off;
    V.K = Kp;
    V.KT = KTp;
    V.d_info = F.d_rec_info + R.count;
    V.fuse_k = true;
    V.kfamily = F.kfamily;
    R.off[R.count++] = off;
    return coop_factorize_enqueue(s, V, V.L, F.ld);
}

bool rec_factor(cudaStream_t s, DenseFactor &F, int off, int n, RecLeaves &R) {
    const long ld = F.ld;
    if (n <= kRecLeafMaxN)
        return rec_leaf(s, F, off, n, F.K + off + (size_t) off * ld, F.KT + off + (size_t) off * ld, R);
    const int n1 = rec_split(n), n2 = n - n1;
    if (!rec_factor(s, F, off, n1, R)) return false;
    double *L21 = F.L + (off + n1) + (size_t) off * ld;
    double *A22 = F.L + (off + n1) + (size_t) (off + n1) * ld;
    const double *K11 = F.K + off + (size_t) off * ld, *KT11 = F.KT + off + (size_t) off * ld;
    const double *K22 = F.K + (off + n1) + (size_t) (off + n1) * ld;
    double *K21 = F.K + (off + n1) + (size_t) off * ld, *KT12 = F.KT + off + (size_t) (off + n1) * ld;
    double *W = F.d_rec_w;   // n2 x n1, leading dimension ld
    gemm(s, n2, n1, n1, 1.0, L21, ld, 0, KT11, ld, 0, 0.0, W, ld, GEMM_B_UPPER);      // A21 K11^T
    copy_matrix(s, n2, n1, W, ld, L21, ld);
    gemm(s, n2, n2, n1, -1.0, L21, ld, 0, L21, ld, 1, 1.0, A22, ld, GEMM_C_LOWER);    // A22 -= L21 L21^T
    if (!rec_factor(s, F, off + n1, n2, R)) return false;
    gemm(s, n2, n1, n1, 1.0, L21, ld, 0, K11, ld, 0, 0.0, W, ld, GEMM_B_LOWER);       // L21 K11
    gemm(s, n2, n1, n2, -1.0, K22, ld, 0, W, ld, 0, 0.0, K21, ld, GEMM_A_LOWER);      // -K22 (L21 K11)
    dim3 grid((n2 + 31) / 32, (n1 + 31) / 32), block(32, 8);
    transpose_rect_kernel<<<hb::counted(grid), block, 0, s>>>(n2, n1, K21, ld, KT12, ld);
    return cudaGetLastError() == cudaSuccess;
}

// X (rows x nL, leading dimension ldx) <- X L^-T for the diagonal block L of F at [Loff, Loff +
// nL), split as the factorisation split it: a leaf is one GEMM with that block's K^T (kept in
// the strip), otherwise Xa <- Xa La^-T, Xc -= Xa Lb^T, Xc <- Xc Lc^-T
bool rec_trsm(cudaStream_t s, DenseFactor &F, double *X, long ldx, int rows, int Loff, int nL) {
    const long ld = F.ld;
    if (nL <= kRecLeafMaxN) {
        gemm(s, rows, nL, nL, 1.0, X, ldx, 0, F.d_rec_kts + Loff, ld, 0, 0.0, F.d_rec_w, ld, GEMM_B_UPPER);
        copy_matrix(s, rows, nL, F.d_rec_w, ld, X, ldx);
        return true;
    }
    const int n1 = rec_split(nL), nc = nL - n1;
    if (!rec_trsm(s, F, X, ldx, rows, Loff, n1)) return false;
    gemm(s, rows, nc, n1, -1.0, X, ldx, 0, F.L + (Loff + n1) + (size_t) Loff * ld, ld, 1, 1.0, X + (size_t) n1 * ldx,
         ldx, 0);
    return rec_trsm(s, F, X + (size_t) n1 * ldx, ldx, rows, Loff + n1, nc);
}

// the recursive form without K: the diagonal blocks' K (and K^T) go to the strips
bool rec_factor_nok(cudaStream_t s, DenseFactor &F, int off, int n, RecLeaves &R) {
    const long ld = F.ld;
    if (n <= kRecLeafMaxN) return rec_leaf(s, F, off, n, F.d_rec_ks + off, F.d_rec_kts + off, R);
    const int n1 = rec_split(n), n2 = n - n1;
    if (!rec_factor_nok(s, F, off, n1, R)) return false;
    double *L21 = F.L + (off + n1) + (size_t) off * ld;
    double *A22 = F.L + (off + n1) + (size_t) (off + n1) * ld;
    if (!rec_trsm(s, F, L21, ld, n2, off, n1)) return false;                            // A21 L11^-T
    gemm(s, n2, n2, n1, -1.0, L21, ld, 0, L21, ld, 1, 1.0, A22, ld, GEMM_C_LOWER);    // A22 -= L21 L21^T
    return rec_factor_nok(s, F, off + n1, n2, R);
}
}  // namespace

bool rec_factorize_enqueue(cudaStream_t s, DenseFactor &F, const double *S, long ldS) {
    const int n = F.n;
    if (!F.d_rec_info && hb::cmalloc(&F.d_rec_info, sizeof(int) * kRecMaxLeaves) != cudaSuccess) {
        F.d_rec_info = nullptr;
        return false;
    }
    if (!F.d_rec_w && hb::cmalloc(&F.d_rec_w, sizeof(double) * F.ld * ((n + 1) / 2)) != cudaSuccess) {
        F.d_rec_w = nullptr;
        return false;
    }
    HB_CUDA(cudaMemsetAsync(F.d_rec_info, 0, sizeof(int) * kRecMaxLeaves, s));
    copy_lower_k<<<hb::counted(grid_for_n((long) n * n)), 256, 0, s>>>(n, S, ldS, F.L, F.ld);
    RecLeaves R;
    R.count = 0;
    const bool ok = rec_factor(s, F, 0, n, R);
    rec_info_kernel<<<hb::counted(1), 32, 0, s>>>(R, F.d_rec_info, F.d_info);
    if (!ok) device_error_flag() = 1;
    return ok && cudaGetLastError() == cudaSuccess;
}

bool rec_factorize_nok_enqueue(cudaStream_t s, DenseFactor &F, const double *S, long ldS) {
    const int n = F.n;
    const size_t strip = (size_t) F.ld * kRecLeafMaxN;
    if (!F.d_rec_info && hb::cmalloc(&F.d_rec_info, sizeof(int) * kRecMaxLeaves) != cudaSuccess) {
        F.d_rec_info = nullptr;
        return false;
    }
    if (!F.d_rec_w && hb::cmalloc(&F.d_rec_w, sizeof(double) * F.ld * std::max((n + 1) / 2, kRecLeafMaxN)) !=
                          cudaSuccess) {
        F.d_rec_w = nullptr;
        return false;
    }
    if (!F.d_rec_ks) {
        // zero outside the blocks' triangles, which the cooperative kernel never writes
        if (hb::cmalloc(&F.d_rec_ks, sizeof(double) * strip) != cudaSuccess ||
            hb::cmalloc(&F.d_rec_kts, sizeof(double) * strip) != cudaSuccess) {
            if (F.d_rec_ks) hb::cache_free(F.d_rec_ks);
            F.d_rec_ks = F.d_rec_kts = nullptr;
            return false;
        }
        HB_CUDA(cudaMemsetAsync(F.d_rec_ks, 0, sizeof(double) * strip, s));
        HB_CUDA(cudaMemsetAsync(F.d_rec_kts, 0, sizeof(double) * strip, s));
    }
    HB_CUDA(cudaMemsetAsync(F.d_rec_info, 0, sizeof(int) * kRecMaxLeaves, s));
    copy_lower_k<<<hb::counted(grid_for_n((long) n * n)), 256, 0, s>>>(n, S, ldS, F.L, F.ld);
    RecLeaves R;
    R.count = 0;
    const bool ok = rec_factor_nok(s, F, 0, n, R);
    rec_info_kernel<<<hb::counted(1), 32, 0, s>>>(R, F.d_rec_info, F.d_info);
    if (!ok) device_error_flag() = 1;
    return ok && cudaGetLastError() == cudaSuccess;
}

// The factorisations of F[0..count) (each n <= kSmallFactorMaxN) of S[i] (ldS[i]) in launches of up to
// kSmallBatch CTAs, the status words written into each factor's pinned host mirror by the
// kernel; returns false (nothing enqueued) if a mirror has no device address, or false
// after a failed launch.
bool small_factor_batch_enqueue(cudaStream_t s, DenseFactor *const *F, const double *const *S, const long *ldS,
                                int count) {
    static std::atomic<unsigned long long> attr{0};
    once_per_device(attr, [] {
        HB_CUDA(cudaFuncSetAttribute((const void *) potrf_small_batch_kernel,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, SM_DOUBLES * (int) sizeof(double)));
        HB_CUDA(cudaFuncSetAttribute((const void *) potrf_batch_array_kernel,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, SM_DOUBLES * (int) sizeof(double)));
    });
    std::vector<SmallFactorJob> jobs(count);
    for (int q = 0; q < count; ++q) {
        DenseFactor &G = *F[q];
        double *hd = nullptr;
        if (cudaHostGetDevicePointer((void **) &hd, G.h_info, 0) != cudaSuccess || !hd) {
            cudaGetLastError();
            return false;
        }
        jobs[q] = SmallFactorJob{S[q], G.L, G.Dinv, G.fuse_k ? G.K : nullptr, G.fuse_k ? G.KT : nullptr, ldS[q], G.ld,
                                 G.d_info, hd, G.n, G.stat_logdet ? 1 : 0};
    }
    if (count <= kSmallBatch) {
        SmallFactorBatch B;
        for (int q = 0; q < count; ++q) B.job[q] = jobs[q];
        potrf_small_batch_kernel<<<hb::counted(count), COOP_THREADS, SM_DOUBLES * sizeof(double), s>>>(B);
        return cudaGetLastError() == cudaSuccess;
    }
    // more jobs than fit the parameters: one launch over a device copy of them, in a buffer kept
    // per host thread and device (every caller waits for the launch before its thread enqueues
    // another batch, so the buffer is free again by then)
    struct JobBuf {
        SmallFactorJob *p = nullptr;
        size_t cap = 0;
    };
    thread_local JobBuf buf[kMaxDevices];
    JobBuf &b = buf[current_device()];
    if (b.cap < (size_t) count) {
        if (b.p) hb::cache_free(b.p);
        b.cap = (size_t) count;
        if (hb::cmalloc(&b.p, sizeof(SmallFactorJob) * b.cap) != cudaSuccess) {
            b.p = nullptr;
            b.cap = 0;
            return false;
        }
    }
    HB_CUDA(cudaMemcpyAsync(b.p, jobs.data(), sizeof(SmallFactorJob) * count, cudaMemcpyHostToDevice, s));
    potrf_batch_array_kernel<<<hb::counted(count), COOP_THREADS, SM_DOUBLES * sizeof(double), s>>>(b.p);
    return cudaGetLastError() == cudaSuccess;
}

bool chol_solve(cudaStream_t s, DenseFactor &F, const double *b, double *x) {
    const int n = F.n;
    if (n <= 0) return true;
    const int nblk = (n + 63) / 64;
    if (!F.d_flags) {
        HB_CUDA(hb::cmalloc(&F.d_flags, sizeof(unsigned) * 2 * nblk));
        HB_CUDA(cudaMemsetAsync(F.d_flags, 0, sizeof(unsigned) * 2 * nblk, s));
        F.epoch = 0;
    }
    if (!F.d_tmp) HB_CUDA(hb::cmalloc(&F.d_tmp, sizeof(double) * n));
    if (!F.d_flags || !F.d_tmp) return false;
    F.epoch += 1;
    const void *fn = (const void *) tri_solve_coop_kernel;
    const int G = std::min(nblk, sm_count());
    const int nown = (nblk + G - 1) / G;
    const int smem = (2 * 64 * TP + nown * 64 + 2 * 64 + 4 * 64) * (int) sizeof(double);
    {
        // the largest dynamic shared memory requested so far, per device
        static std::mutex mu;
        static int smem_set[kMaxDevices] = {0};
        std::lock_guard<std::mutex> g(mu);
        int &cur = smem_set[current_device()];
        if (smem > cur) {
            if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess)
                return false;
            cur = smem;
        }
    }
    const double *Lp = F.L;
    long ld = F.ld;
    int nn = n;
    const double *Dp = F.Dinv;
    long ldd = F.ld;
    const double *bp = b;
    double *tp = F.d_tmp, *xp = x;
    unsigned *ff = F.d_flags, *fb = F.d_flags + nblk;
    unsigned ep = F.epoch;
    void *args[] = {&Lp, &ld, &nn, &Dp, &ldd, &bp, &tp, &xp, &ff, &fb, &ep};
    cudaError_t e = cudaLaunchCooperativeKernel(fn, hb::counted(G), COOP_THREADS, args, smem, s);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return true;
}

int chol_solve_error() {
    int h = 0;
    cudaMemcpyFromSymbol(&h, g_tri_err, sizeof(int));
    if (h) {
        const int z = 0;
        cudaMemcpyToSymbol(g_tri_err, &z, sizeof(int));
    }
    return h;
}

bool coop_inverse_enqueue(cudaStream_t s, DenseFactor &F) {
    const int n = F.n;
    identity_k<<<hb::counted(grid_for_n((long) n * n)), 256, 0, s>>>(n, F.K, F.ld);
    const void *fn = (const void *) trtri_coop_kernel;
    const long t0 = (long) ((n - 1) / 64 + 1);
    const int grid = (int) std::max(1L, std::min<long>(coop_grid(fn), t0 * t0 / 4 + 1));
    const double *Lp = F.L;
    double *Kp = F.K;
    long ld = F.ld;
    int nn = n;
    const double *Dp = F.Dinv;
    long ldd = F.ld;
    void *args[] = {&Lp, &Kp, &ld, &nn, &Dp, &ldd};
    const bool timed = kstat_on(KF_TRTRI);
    if (timed) kstat_begin(KF_TRTRI, s, (double) n * n * n / 3.0);
    cudaError_t e = cudaLaunchCooperativeKernel(fn, hb::counted(grid), COOP_THREADS, args, SM_DOUBLES * sizeof(double), s);
    if (timed) kstat_end(s);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return true;
}

}  // namespace hb
