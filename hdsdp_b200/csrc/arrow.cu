// Sparse Schur complement for problems made of sparse SDP cones (the reference's sparse
// KKT, interface/hdsdp_schur.c:46-139, chosen at :181-254 when no cone's pattern reaches
// HDSDP_SPARSE_SCHUR_THRESHOLD = 30 % of m^2), as a block-arrow factorisation on the GPU.
//
// A sparse cone touches only its own rows, so M_ij != 0 only when rows i and j share a
// cone. Rows held by exactly one cone are that cone's local rows; rows held by two or more
// cones (or by none: they get only the bound cone's diagonal) are coupling rows. With the
// local rows of each cone first and the coupling rows last, M is a block arrow:
//
//     M = [ M_11          B_1^T ]        L_kk = chol(M_kk),  W_k = B_k L_kk^-T,
//         [      ...      ...   ]        L_cc = chol(M_cc - sum_k W_k W_k^T),
//         [           M_KK B_K^T ]
//         [ B_1  ...  B_K  M_cc ]
//
// and a solve runs z_k = L_kk^-1 b_k, x_c = L_cc^-T L_cc^-1 (b_c - sum_k W_k z_k),
// x_k = L_kk^-T (z_k - W_k^T x_c), followed by one step of iterative refinement on the
// FP64 residual, as the dense Schur solve does. Memory is sum_k l_k^2 + n_c (n_c + 2 sum_k
// l_k) doubles instead of m^2. Each cone's Schur block (built over its own rows by the
// cone's kernels) is scattered into M_kk, B_k and M_cc by one kernel.
#include "solver.h"
#include <algorithm>
#include <cmath>
#include <cstdio>

namespace hb {

// One block's operand in a batched matrix-vector product: A is rows x cols, column-major;
// x and y are offsets into the vectors the launch is given.
struct BlkOp {
    const double *A;
    long lda;
    int rows, cols, xoff, yoff, mode;
};

// One square block of the arrow (a local block, or the coupling block last) for the batched
// diagonal and mirror operations: order l, its rows at packed offset off.
struct BlkDiag {
    double *A;
    long ld;
    int l, off;
};

struct ArrowSchur {
    int m = 0, nc = 0, ncone = 0;
    std::vector<int> lk;              // local rows per cone
    std::vector<int> off;             // packed offset of cone k's local rows; coupling at off[ncone]
    std::vector<int> perm;            // packed index -> problem row
    std::vector<const SdpCone *> cone;
    std::vector<int *> d_code;        // per cone, per row of its list: local index, or -(coupling index + 1)
    std::vector<double *> Mkk, Bk, Wk;   // Mkk: blocks of Mall; Bk / Wk: column blocks of Ball / Wall
    double *Mall = nullptr;           // every local block, one after the other
    size_t mallSize = 0;
    BlkDiag *dblk = nullptr;          // the local blocks and the coupling block, for the batched
    int ndblk = 0, maxdl = 0;         // diagonal and mirror operations
    double *Ball = nullptr, *Wall = nullptr;   // n_c x sum l_k: [B_1 ... B_K], [W_1 ... W_K]
    GemmDesc *wdesc = nullptr;        // W_k = B_k K_k^T for the blocks with local rows
    int nw = 0;
    // the coupling update Wall Wall^T split along its inner dimension when M_cc is too small to
    // keep the GPU busy: nsplit partial products (column chunks of Wall) into P
    GemmDesc *sdesc = nullptr;
    double *P = nullptr;
    int nsplit = 0;
    std::vector<long> ldk;
    std::vector<DenseFactor> Fk;
    double *Mcc = nullptr, *Mcf = nullptr;
    long ldc = 0, ldb = 0;
    DenseFactor Fc;
    double *b = nullptr, *x = nullptr, *r = nullptr, *z = nullptr, *t = nullptr;   // packed m-vectors
    double *d_diag = nullptr;
    double *hb_ = nullptr;            // pinned host packed scratch (m)
    double shift = 0.0;
    // the per-block matrix-vector products of a solve, each one batched launch over the
    // blocks (device descriptor arrays, built once the blocks are allocated)
    BlkOp *opsK = nullptr, *opsKT = nullptr, *opsWt = nullptr, *opsMkk = nullptr, *opsBt = nullptr;
    BlkOp *opsW = nullptr, *opsB = nullptr;
    int nops = 0, nopsB = 0;          // blocks with local rows; nopsB = nops + 1 (M_cc)
    int maxl = 0, gsplit = 1;         // largest local block; column splits of the gemv
    double *U = nullptr;              // nc x (nopsB * gsplit) partial sums of the gemv
    long ldu = 0;
    double bytes = 0.0;               // device memory of the blocks, their factors and scratch
};

namespace {

__global__ void arrow_scatter_kernel(int mk, const double *__restrict__ Msub, long lds, const int *__restrict__ code,
                                     double *Mkk, long ldk, double *Bk, long ldb, double *Mcc, long ldc) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    for (int j = blockIdx.y * blockDim.y + threadIdx.y; j < mk; j += gridDim.y * blockDim.y) {
        if (i < j || i >= mk) continue;
        const double v = Msub[(size_t) i + (size_t) j * lds];
        const int ci = code[i], cj = code[j];
        if (ci >= 0 && cj >= 0) {
            Mkk[(size_t) ci + (size_t) cj * ldk] += v;          // ci >= cj: local order follows row order
        } else if (ci < 0 && cj >= 0) {
            Bk[(size_t) (-ci - 1) + (size_t) cj * ldb] += v;
        } else if (ci >= 0 && cj < 0) {
            Bk[(size_t) (-cj - 1) + (size_t) ci * ldb] += v;
        } else {
            const int a = -ci - 1, c = -cj - 1;
            Mcc[(size_t) max(a, c) + (size_t) min(a, c) * ldc] += v;
        }
    }
}

void zero_blocks(cudaStream_t s, ArrowSchur &A) {
    if (A.mallSize > 0) HB_CUDA(cudaMemsetAsync(A.Mall, 0, sizeof(double) * A.mallSize, s));
    if (A.nc > 0 && A.off[A.ncone] > 0)
        HB_CUDA(cudaMemsetAsync(A.Ball, 0, sizeof(double) * A.ldb * A.off[A.ncone], s));
    if (A.nc > 0) HB_CUDA(cudaMemsetAsync(A.Mcc, 0, sizeof(double) * A.ldc * A.nc, s));
}

// on the diagonal of every block (blockIdx.y): op 0 reads it into out[off + i], op 1 adds v,
// op 2 adds d[off + i]
__global__ void arrow_diag_kernel(const BlkDiag *__restrict__ b, int op, double v, const double *__restrict__ d,
                                  double *out) {
    const BlkDiag B = b[blockIdx.y];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < B.l; i += gridDim.x * blockDim.x) {
        double *p = B.A + (size_t) i * (B.ld + 1);
        if (op == 0) out[B.off + i] = *p;
        else if (op == 1) *p += v;
        else *p += d[B.off + i];
    }
}

// A(j, i) = A(i, j), i > j, in every block (blockIdx.z), 32 x 32 tiles
__global__ void arrow_mirror_kernel(const BlkDiag *__restrict__ b) {
    const BlkDiag B = b[blockIdx.z];
    const int i0 = blockIdx.x * 32, j0 = blockIdx.y * 32;
    if (i0 >= B.l || j0 >= B.l || i0 + 31 < j0) return;
    for (int e = threadIdx.x; e < 32 * 32; e += blockDim.x) {
        const int i = i0 + (e & 31), j = j0 + (e >> 5);
        if (i < B.l && j < B.l && i > j) B.A[(size_t) j + (size_t) i * B.ld] = B.A[(size_t) i + (size_t) j * B.ld];
    }
}

void arrow_diag(cudaStream_t s, ArrowSchur &A, int op, double v, const double *d, double *out) {
    if (A.ndblk == 0) return;
    dim3 grd((A.maxdl + 255) / 256, A.ndblk);
    arrow_diag_kernel<<<counted(grd), 256, 0, s>>>(A.dblk, op, v, d, out);
    HB_CUDA(cudaGetLastError());
}

// diag (packed order) added to the diagonals of the blocks
void add_diag_packed(cudaStream_t s, ArrowSchur &A, const double *d) { arrow_diag(s, A, 2, 0.0, d, nullptr); }

void add_diag_all(cudaStream_t s, ArrowSchur &A, double v) { arrow_diag(s, A, 1, v, nullptr, nullptr); }

// every block's lower triangle mirrored into its upper one
void mirror_blocks(cudaStream_t s, ArrowSchur &A) {
    if (A.ndblk == 0) return;
    const int t = (A.maxdl + 31) / 32;
    dim3 grd(t, t, A.ndblk);
    arrow_mirror_kernel<<<counted(grd), 256, 0, s>>>(A.dblk);
    HB_CUDA(cudaGetLastError());
}

// the diagonals of all blocks, packed, on the host
void diag_to_host(cudaStream_t s, ArrowSchur &A, double *h_buf) {
    arrow_diag(s, A, 0, 0.0, nullptr, A.t);
    HB_CUDA(cudaMemcpyAsync(h_buf, A.t, sizeof(double) * A.m, cudaMemcpyDeviceToHost, s));
    HB_CUDA(cudaStreamSynchronize(s));
}

// y = K x (K lower) and y = K^T x with K = L^-1 of a factor
void apply_k(cudaStream_t s, DenseFactor &F, const double *x, double *y) {
    coldot(s, F.n, F.n, F.KT, F.ld, x, y, 1.0, 0.0, 2);
}
void apply_kt(cudaStream_t s, DenseFactor &F, const double *x, double *y) {
    coldot(s, F.n, F.n, F.K, F.ld, x, y, 1.0, 0.0, 1);
}

constexpr int kArrowBatchMaxN = 512;   // local blocks factored one CTA each up to this order
constexpr int kColWarps = 8;      // columns per block of the batched column-dot kernel
constexpr int kGemvRows = 128;    // rows per block of the batched gemv
constexpr int kGemvCols = 256;    // columns per split of the batched gemv

// y[yoff + i] = alpha * sum_{r in R(i)} A(r, i) x[xoff + r] + beta * y[yoff + i] for every
// column i of every op (blockIdx.y), R as in coldot: one warp per column.
__global__ void bcoldot_kernel(const BlkOp *__restrict__ ops, const double *__restrict__ x, double *y,
                               double alpha, double beta) {
    const BlkOp op = ops[blockIdx.y];
    const int lane = threadIdx.x & 31;
    const int i = blockIdx.x * kColWarps + (threadIdx.x >> 5);
    if (i >= op.cols) return;
    const int r0 = (op.mode == 1) ? i : 0;
    const int r1 = (op.mode == 2) ? i + 1 : op.rows;
    const double *a = op.A + (size_t) i * op.lda;
    const double *xv = x + op.xoff;
    double acc = 0.0;
    for (int r = r0 + lane; r < r1; r += 32) acc = fma(a[r], xv[r], acc);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) {
        double *yp = y + op.yoff + i;
        *yp = (beta == 0.0) ? alpha * acc : alpha * acc + beta * *yp;
    }
}

// U(i, op * gridDim.z + split) = sum over the split's columns j of A(i, j) x[xoff + j]: one
// thread per row (coalesced down a column), every entry of U written.
__global__ void bgemv_kernel(const BlkOp *__restrict__ ops, const double *__restrict__ x, double *U, long ldu,
                             int nrowsU) {
    const BlkOp op = ops[blockIdx.y];
    const int i = blockIdx.x * kGemvRows + threadIdx.x;
    if (i >= nrowsU) return;
    const int j0 = blockIdx.z * kGemvCols, j1 = min(op.cols, j0 + kGemvCols);
    double acc = 0.0;
    if (i < op.rows) {
        const double *xv = x + op.xoff;
        for (int j = j0; j < j1; ++j) acc = fma(op.A[(size_t) i + (size_t) j * op.lda], xv[j], acc);
    }
    U[(size_t) i + (size_t) (blockIdx.y * gridDim.z + blockIdx.z) * ldu] = acc;
}

// y[i] = (b ? b[i] : 0) + alpha * sum_p U(i, p), i < n
__global__ void rowsum_kernel(int n, int np, const double *__restrict__ U, long ldu, const double *b, double alpha,
                              double *y) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double acc = 0.0;
    for (int p = 0; p < np; ++p) acc += U[(size_t) i + (size_t) p * ldu];
    y[i] = (b ? b[i] : 0.0) + alpha * acc;
}

// r = b - y + shift * x
__global__ void residual_kernel(int n, const double *b, const double *y, const double *x, double shift, double *r) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) r[i] = (b[i] - y[i]) + shift * x[i];
}

void bcoldot(cudaStream_t s, const ArrowSchur &A, const BlkOp *ops, const double *x, double *y, double alpha,
             double beta) {
    if (A.nops == 0) return;
    dim3 grd((A.maxl + kColWarps - 1) / kColWarps, A.nops);
    bcoldot_kernel<<<counted(grd), 32 * kColWarps, 0, s>>>(ops, x, y, alpha, beta);
    HB_CUDA(cudaGetLastError());
}

// out_c = base_c + alpha * sum over the ops of A_k x_k (n_c rows)
void bgemv_sum(cudaStream_t s, const ArrowSchur &A, const BlkOp *ops, int nops, const double *x, const double *base,
               double alpha, double *out) {
    dim3 grd((A.nc + kGemvRows - 1) / kGemvRows, nops, A.gsplit);
    bgemv_kernel<<<counted(grd), kGemvRows, 0, s>>>(ops, x, A.U, A.ldu, A.nc);
    HB_CUDA(cudaGetLastError());
    rowsum_kernel<<<counted((A.nc + 127) / 128), 128, 0, s>>>(A.nc, nops * A.gsplit, A.U, A.ldu, base, alpha, out);
    HB_CUDA(cudaGetLastError());
}

// x = M^-1 b with the factors (packed vectors, which may alias; z and t scratch)
bool arrow_apply_inverse(cudaStream_t s, ArrowSchur &A, const double *b, double *x) {
    const int nc = A.nc, K = A.ncone;
    bcoldot(s, A, A.opsK, b, A.z, 1.0, 0.0);                                       // z_k = L_kk^-1 b_k
    if (nc > 0) {
        double *tc = A.t + A.off[K], *zc = A.z + A.off[K], *xc = x + A.off[K];
        if (A.nops > 0) bgemv_sum(s, A, A.opsW, A.nops, A.z, b + A.off[K], -1.0, tc);   // t_c = b_c - sum W_k z_k
        else copy_matrix(s, nc, 1, b + A.off[K], nc, tc, nc);
        if (A.Fc.fuse_k) {
            apply_k(s, A.Fc, tc, zc);
            apply_kt(s, A.Fc, zc, xc);
        } else if (!chol_solve(s, A.Fc, tc, xc)) {
            return false;
        }
        bcoldot(s, A, A.opsWt, x, A.z, -1.0, 1.0);                                 // z_k -= W_k^T x_c
    }
    bcoldot(s, A, A.opsKT, A.z, x, 1.0, 0.0);                                      // x_k = L_kk^-T z_k
    return true;
}

// y = M x (packed; the blocks hold full symmetric storage after factorize)
void arrow_matvec(cudaStream_t s, ArrowSchur &A, const double *x, double *y) {
    bcoldot(s, A, A.opsMkk, x, y, 1.0, 0.0);                                       // y_k = M_kk x_k
    if (A.nc > 0) {
        bcoldot(s, A, A.opsBt, x, y, 1.0, 1.0);                                    // y_k += B_k^T x_c
        bgemv_sum(s, A, A.opsB, A.nopsB, x, nullptr, 1.0, y + A.off[A.ncone]);     // y_c = M_cc x_c + sum B_k x_k
    }
}

// Mcf = Mcc - sum_s P_s over the lower triangle (P_s: nc x nc partial products, pitch ld,
// one after the other), the partials subtracted in order
__global__ void arrow_split_sum_kernel(int nc, int ns, const double *__restrict__ P, long ld,
                                       const double *__restrict__ Mcc, double *Mcf, long ldc) {
    const long total = (long) nc * nc;
    for (long idx = blockIdx.x * (long) blockDim.x + threadIdx.x; idx < total; idx += (long) gridDim.x * blockDim.x) {
        const int i = (int) (idx % nc), j = (int) (idx / nc);
        if (i < j) continue;
        double v = Mcc[(size_t) i + (size_t) j * ldc];
        for (int q = 0; q < ns; ++q) v -= P[(size_t) q * ld * nc + (size_t) i + (size_t) j * ld];
        Mcf[(size_t) i + (size_t) j * ldc] = v;
    }
}

// the factors of the current blocks (W_k and the coupling block's Schur complement)
bool arrow_factor_once(cudaStream_t s, ArrowSchur &A) {
    const int nc = A.nc, K = A.ncone;
    // every block's factorisation enqueued (blocks of order <= kArrowBatchMaxN one CTA each,
    // in shared launches; larger ones on the whole GPU), then their statuses read together
    std::vector<DenseFactor *> bF;
    std::vector<const double *> bS;
    std::vector<long> bld;
    for (int k = 0; k < K; ++k) {
        if (A.lk[k] == 0) continue;
        if (K > 1 && A.lk[k] <= kArrowBatchMaxN) {
            bF.push_back(&A.Fk[k]);
            bS.push_back(A.Mkk[k]);
            bld.push_back(A.ldk[k]);
        } else {
            factorize_async(s, A.Fk[k], A.Mkk[k], A.ldk[k]);
        }
    }
    if (!bF.empty()) factorize_small_batch(s, bF.data(), bS.data(), bld.data(), (int) bF.size());
    HB_CUDA(cudaStreamSynchronize(s));
    bool ok = true;
    for (int k = 0; k < K; ++k)
        if (A.lk[k] > 0 && !factor_status_ready(A.Fk[k])) ok = false;
    if (!ok) return false;
    for (int k = 0; k < K; ++k)
        if (A.lk[k] > 0) compute_inverse_factor(s, A.Fk[k]);   // formed by the factorisation kernel already
    if (nc == 0) return true;
    // W_k = B_k L_kk^-T = B_k K_k^T for every block in one launch, then
    // M_cc - sum_k W_k W_k^T = M_cc - Wall Wall^T as one product
    gemm_grouped(s, A.wdesc, A.nw, nc, A.maxl);
    if (A.nsplit > 0) {
        // few coupling rows and many local ones: the product split along its inner dimension
        // (one grouped launch, a partial product per column chunk), the partials subtracted from
        // M_cc in chunk order
        gemm_grouped(s, A.sdesc, A.nsplit, nc, nc);
        const long total = (long) nc * nc;
        arrow_split_sum_kernel<<<counted((int) std::min<long>((total + 255) / 256, 4096)), 256, 0, s>>>(
            nc, A.nsplit, A.P, A.ldc, A.Mcc, A.Mcf, A.ldc);
        HB_CUDA(cudaGetLastError());
    } else {
        copy_matrix(s, nc, nc, A.Mcc, A.ldc, A.Mcf, A.ldc);
        if (A.off[K] > 0)
            gemm(s, nc, nc, A.off[K], -1.0, A.Wall, A.ldb, 0, A.Wall, A.ldb, 1, 1.0, A.Mcf, A.ldc, GEMM_C_LOWER);
    }
    if (!hb::factorize(s, A.Fc, A.Mcf, A.ldc)) return false;
    if (A.Fc.fuse_k) compute_inverse_factor(s, A.Fc);
    return true;
}

}  // namespace

// Automatic choice: the block arrow is taken from this order on when its factorisation
// needs at most a quarter of the dense one's flops (below it the dense Cholesky of M takes
// about as long as the per-block launches and synchronisations of the arrow).
constexpr int kArrowMinM = 4096;
constexpr double kArrowMaxFlopRatio = 0.25;

bool arrow_chosen(int mode, int m, const std::vector<SdpCone *> &cones) {
    if (mode == 0 || cones.empty() || m <= 0) return false;
    if (mode == 1) return true;
    if (m < kArrowMinM) return false;
    std::vector<int> holders(m, 0), owner(m, -1);
    for (size_t k = 0; k < cones.size(); ++k)
        for (int r : cones[k]->rows) {
            holders[r] += 1;
            owner[r] = (int) k;
        }
    std::vector<double> l(cones.size(), 0.0);
    double nc = 0.0;
    for (int r = 0; r < m; ++r) {
        if (holders[r] == 1) l[owner[r]] += 1.0;
        else nc += 1.0;
    }
    double flops = nc * nc * nc / 3.0;
    for (double lk : l) flops += lk * lk * lk / 3.0 + nc * lk * lk + nc * nc * lk;
    return flops <= kArrowMaxFlopRatio * (double) m * m * m / 3.0;
}

bool KKT::setup_arrow(const std::vector<SdpCone *> &cones) {
    release_arrow();
    ArrowSchur *A = new ArrowSchur();
    A->m = m;
    A->ncone = (int) cones.size();
    std::vector<int> holders(m, 0), owner(m, -1);
    for (int k = 0; k < A->ncone; ++k)
        for (int r : cones[k]->rows) {
            holders[r] += 1;
            owner[r] = k;
        }
    std::vector<int> cidx(m, -1);   // coupling index of a row
    A->lk.assign(A->ncone, 0);
    for (int r = 0; r < m; ++r) {
        if (holders[r] == 1) A->lk[owner[r]] += 1;
        else cidx[r] = A->nc++;
    }
    A->off.assign(A->ncone + 1, 0);
    for (int k = 0; k < A->ncone; ++k) A->off[k + 1] = A->off[k] + A->lk[k];
    A->perm.assign(m, 0);
    std::vector<int> lidx(m, -1), fill(A->off.begin(), A->off.end() - 1);
    for (int r = 0; r < m; ++r) {
        if (holders[r] == 1) {
            const int k = owner[r];
            lidx[r] = fill[k] - A->off[k];
            A->perm[fill[k]++] = r;
        } else {
            A->perm[A->off[A->ncone] + cidx[r]] = r;
        }
    }
    A->ldc = pad_ld(std::max(A->nc, 1));
    A->ldb = A->ldc;
    A->Mkk.assign(A->ncone, nullptr);
    A->Bk.assign(A->ncone, nullptr);
    A->Wk.assign(A->ncone, nullptr);
    A->ldk.assign(A->ncone, 0);
    A->d_code.assign(A->ncone, nullptr);
    A->Fk.resize(A->ncone);
    A->cone.assign(cones.begin(), cones.end());
    for (int k = 0; k < A->ncone; ++k) {
        std::vector<int> code;
        code.reserve(cones[k]->rows.size());
        for (int r : cones[k]->rows) code.push_back(holders[r] == 1 ? lidx[r] : -(cidx[r] + 1));
        HB_CUDA(cmalloc(&A->d_code[k], sizeof(int) * std::max<size_t>(code.size(), 1)));
        if (!code.empty())
            HB_CUDA(cudaMemcpyAsync(A->d_code[k], code.data(), sizeof(int) * code.size(), cudaMemcpyHostToDevice, s));
        const int l = A->lk[k];
        if (l == 0) continue;
        A->ldk[k] = pad_ld(l);
        A->mallSize += (size_t) A->ldk[k] * l;
        A->Fk[k].alloc(l, 1);
        A->Fk[k].kfamily = KF_POTRF_SCHUR;
    }
    if (A->mallSize > 0) {
        HB_CUDA(cmalloc(&A->Mall, sizeof(double) * A->mallSize));
        size_t at = 0;
        for (int k = 0; k < A->ncone; ++k) {
            if (A->lk[k] == 0) continue;
            A->Mkk[k] = A->Mall + at;
            at += (size_t) A->ldk[k] * A->lk[k];
        }
    }
    if (A->nc > 0 && A->off[A->ncone] > 0) {
        const size_t cols = (size_t) A->off[A->ncone];
        HB_CUDA(cmalloc(&A->Ball, sizeof(double) * A->ldb * cols));
        HB_CUDA(cmalloc(&A->Wall, sizeof(double) * A->ldb * cols));
        std::vector<GemmDesc> wd;
        for (int k = 0; k < A->ncone; ++k) {
            const int l = A->lk[k];
            if (l == 0) continue;
            A->Bk[k] = A->Ball + (size_t) A->off[k] * A->ldb;
            A->Wk[k] = A->Wall + (size_t) A->off[k] * A->ldb;
            wd.push_back(GemmDesc{A->nc, l, l, 1.0, 0.0, A->Bk[k], A->ldb, 0, A->Fk[k].K, A->Fk[k].ld, 1, A->Wk[k],
                                  A->ldb, GEMM_B_UPPER, nullptr});
        }
        A->nw = (int) wd.size();
        HB_CUDA(cmalloc(&A->wdesc, sizeof(GemmDesc) * wd.size()));
        HB_CUDA(cudaMemcpyAsync(A->wdesc, wd.data(), sizeof(GemmDesc) * wd.size(), cudaMemcpyHostToDevice, s));
        // split the coupling update when its 64 x 64 output tiles are few against the SMs and its
        // inner dimension long: chunks of at least 512 columns, the partials within 256 MB
        const long tiles = (long) ((A->nc + 63) / 64) * ((A->nc + 63) / 64);
        const long kk = (long) cols;
        if (tiles < 4L * device_sm_count() && kk >= 4096) {
            long ns = std::min<long>(4L * device_sm_count() / std::max(tiles, 1L), kk / 512);
            const long cap = (256L << 20) / (8L * A->ldc * A->nc);
            ns = std::max(1L, std::min(ns, cap));
            if (ns > 1) {
                A->nsplit = (int) ns;
                HB_CUDA(cmalloc(&A->P, sizeof(double) * A->ldc * A->nc * ns));
                std::vector<GemmDesc> sd;
                const long chunk = (kk + ns - 1) / ns;
                for (long q = 0; q < ns; ++q) {
                    const long c0 = q * chunk, c1 = std::min(kk, c0 + chunk);
                    double *Pq = A->P + (size_t) q * A->ldc * A->nc;
                    const double *Wq = A->Wall + (size_t) c0 * A->ldb;
                    sd.push_back(GemmDesc{A->nc, A->nc, (int) (c1 - c0), 1.0, 0.0, Wq, A->ldb, 0, Wq, A->ldb, 1, Pq,
                                          A->ldc, GEMM_C_LOWER, nullptr});
                }
                HB_CUDA(cmalloc(&A->sdesc, sizeof(GemmDesc) * sd.size()));
                HB_CUDA(cudaMemcpyAsync(A->sdesc, sd.data(), sizeof(GemmDesc) * sd.size(), cudaMemcpyHostToDevice, s));
            }
        }
    }
    if (A->nc > 0) {
        HB_CUDA(cmalloc(&A->Mcc, sizeof(double) * A->ldc * A->nc));
        HB_CUDA(cmalloc(&A->Mcf, sizeof(double) * A->ldc * A->nc));
        A->Fc.alloc(A->nc, A->nc < kTriSolveMinM ? 1 : 0);
        A->Fc.kfamily = KF_POTRF_SCHUR;
    }
    {
        std::vector<BlkDiag> bd;
        for (int k = 0; k < A->ncone; ++k)
            if (A->lk[k] > 0) bd.push_back(BlkDiag{A->Mkk[k], A->ldk[k], A->lk[k], A->off[k]});
        if (A->nc > 0) bd.push_back(BlkDiag{A->Mcc, A->ldc, A->nc, A->off[A->ncone]});
        A->ndblk = (int) bd.size();
        for (const BlkDiag &b : bd) A->maxdl = std::max(A->maxdl, b.l);
        if (!bd.empty()) {
            HB_CUDA(cmalloc(&A->dblk, sizeof(BlkDiag) * bd.size()));
            HB_CUDA(cudaMemcpyAsync(A->dblk, bd.data(), sizeof(BlkDiag) * bd.size(), cudaMemcpyHostToDevice, s));
        }
    }
    for (double **p : {&A->b, &A->x, &A->r, &A->z, &A->t, &A->d_diag}) HB_CUDA(cmalloc(p, sizeof(double) * m));
    HB_CUDA(cmalloc_host(&A->hb_, sizeof(double) * m));
    // descriptors of the batched block products
    {
        const int K = A->ncone, nc = A->nc, offc = A->off[K];
        std::vector<BlkOp> oK, oKT, oWt, oMkk, oBt, oW, oB;
        for (int k = 0; k < K; ++k) {
            const int l = A->lk[k];
            if (l == 0) continue;
            const int o = A->off[k];
            const DenseFactor &F = A->Fk[k];
            A->maxl = std::max(A->maxl, l);
            oK.push_back({F.KT, F.ld, l, l, o, o, 2});
            oKT.push_back({F.K, F.ld, l, l, o, o, 1});
            oMkk.push_back({A->Mkk[k], A->ldk[k], l, l, o, o, 0});
            if (nc > 0) {
                oWt.push_back({A->Wk[k], A->ldb, nc, l, offc, o, 0});
                oBt.push_back({A->Bk[k], A->ldb, nc, l, offc, o, 0});
                oW.push_back({A->Wk[k], A->ldb, nc, l, o, 0, 0});
                oB.push_back({A->Bk[k], A->ldb, nc, l, o, 0, 0});
            }
        }
        if (nc > 0) oB.push_back({A->Mcc, A->ldc, nc, nc, offc, 0, 0});
        A->nops = (int) oK.size();
        A->nopsB = (int) oB.size();
        auto up = [&](BlkOp **d, const std::vector<BlkOp> &h) {
            if (h.empty()) return;
            HB_CUDA(cmalloc(d, sizeof(BlkOp) * h.size()));
            HB_CUDA(cudaMemcpyAsync(*d, h.data(), sizeof(BlkOp) * h.size(), cudaMemcpyHostToDevice, s));
        };
        up(&A->opsK, oK);
        up(&A->opsKT, oKT);
        up(&A->opsMkk, oMkk);
        up(&A->opsWt, oWt);
        up(&A->opsBt, oBt);
        up(&A->opsW, oW);
        up(&A->opsB, oB);
        if (nc > 0) {
            A->gsplit = (std::max(A->maxl, nc) + kGemvCols - 1) / kGemvCols;
            A->ldu = pad_ld(nc);
            HB_CUDA(cmalloc(&A->U, sizeof(double) * A->ldu * A->nopsB * A->gsplit));
        }
    }
    HB_CUDA(cudaStreamSynchronize(s));
    {
        // device memory held: local blocks, their factors (L, K, K^T, diagonal-block inverses),
        // B_k and W_k, the coupling block, its copy and factor, the solve's vectors and scratch
        double b = 0.0;
        for (int k = 0; k < A->ncone; ++k) {
            const double l = A->lk[k], ldk = A->ldk[k];
            if (l == 0) continue;
            b += ldk * l * 4 + ldk * 64 + 2.0 * A->ldb * l;
        }
        if (A->nc > 0) b += 4.0 * A->ldc * A->nc + A->ldc * 64;
        b += 6.0 * m + A->ldu * (double) A->nopsB * A->gsplit;
        A->bytes = 8.0 * b;
    }
    arrow = A;
    mOpen = false;
    return !device_error_flag();
}

void KKT::release_arrow() {
    if (!arrow) return;
    ArrowSchur &A = *arrow;
    auto f = [](void *p) { if (p) cache_free(p); };
    for (int k = 0; k < A.ncone; ++k) {
        f(A.d_code[k]);
        A.Fk[k].release();
    }
    f(A.Mall);
    f(A.dblk);
    f(A.sdesc);
    f(A.P);
    f(A.Ball);
    f(A.Wall);
    f(A.wdesc);
    f(A.Mcc);
    f(A.Mcf);
    A.Fc.release();
    for (double *p : {A.b, A.x, A.r, A.z, A.t, A.d_diag, A.U}) f(p);
    for (BlkOp *p : {A.opsK, A.opsKT, A.opsWt, A.opsMkk, A.opsBt, A.opsW, A.opsB}) f(p);
    if (A.hb_) cache_free_host(A.hb_);
    delete arrow;
    arrow = nullptr;
}

void KKT::arrow_open() {
    if (mOpen) return;
    zero_blocks(s, *arrow);
    mOpen = true;
}

// a sparse cone's Schur block (Msub over its rows, leading dimension ldsub) into the blocks
void KKT::arrow_add(const SdpCone &cone, const double *Msub, long ldsub) {
    arrow_open();
    ArrowSchur &A = *arrow;
    const int k = (int) (std::find(A.cone.begin(), A.cone.end(), &cone) - A.cone.begin());
    if (k == A.ncone) {
        device_error_flag() = 1;
        return;
    }
    const int mk = cone.m;
    dim3 blk(32, 8), grd((mk + 31) / 32, std::min((mk + 7) / 8, 4096));
    arrow_scatter_kernel<<<counted(grd), blk, 0, s>>>(mk, Msub, ldsub, A.d_code[k], A.Mkk[k], A.ldk[k], A.Bk[k],
                                                      A.ldb, A.Mcc, A.ldc);
    HB_CUDA(cudaGetLastError());
}

// the bound cone's diagonal (problem order, host) onto the blocks
void KKT::arrow_add_diag(const double *h_diag) {
    arrow_open();
    ArrowSchur &A = *arrow;
    for (int p = 0; p < m; ++p) A.hb_[p] = h_diag[A.perm[p]];
    HB_CUDA(cudaMemcpyAsync(A.d_diag, A.hb_, sizeof(double) * m, cudaMemcpyHostToDevice, s));
    add_diag_packed(s, A, A.d_diag);
    HB_CUDA(cudaStreamSynchronize(s));
}

void KKT::arrow_regularize(double reg) {
    ArrowSchur &A = *arrow;
    diag_to_host(s, A, A.hb_);
    double mn = HDSDP_INFINITY;
    for (int p = 0; p < m; ++p) mn = std::min(mn, A.hb_[p]);
    reg = reg * mn;
    reg = std::min(reg, 1e-05);
    if (reg < 1e-14) reg = 0.0;
    if (reg != 0.0) add_diag_all(s, A, reg);
}

bool KKT::arrow_factorize() {
    ArrowSchur &A = *arrow;
    mirror_blocks(s, A);
    A.shift = 0.0;
    bool ok = arrow_factor_once(s, A);
    if (!ok) {
        // as the dense Schur factorisation: retry with growing diagonal shifts
        diag_to_host(s, A, A.hb_);
        double mx = 0.0;
        for (int p = 0; p < m; ++p) mx = std::max(mx, std::fabs(A.hb_[p]));
        for (double eps = 1e-14; eps <= 1e-6 && !ok; eps *= 100.0) {
            add_diag_all(s, A, eps * std::max(mx, 1.0));
            A.shift += eps * std::max(mx, 1.0);
            ok = arrow_factor_once(s, A);
        }
        if (ok) printf("KKT system is almost indefinite. Using a shifted Cholesky factor. \n");
    }
    HB_CUDA(cudaStreamSynchronize(s));
    return ok;
}

bool KKT::arrow_solve(const double *rhs, double *lhs) {
    ArrowSchur &A = *arrow;
    for (int p = 0; p < m; ++p) A.hb_[p] = rhs[A.perm[p]];
    HB_CUDA(cudaMemcpyAsync(A.b, A.hb_, sizeof(double) * m, cudaMemcpyHostToDevice, s));
    bool ok = arrow_apply_inverse(s, A, A.b, A.x);
    // one step of iterative refinement on the residual of the unshifted system
    arrow_matvec(s, A, A.x, A.r);
    residual_kernel<<<counted((m + 255) / 256), 256, 0, s>>>(m, A.b, A.r, A.x, A.shift, A.r);
    HB_CUDA(cudaGetLastError());
    ok = arrow_apply_inverse(s, A, A.r, A.r) && ok;   // b and x may alias
    axpy(s, m, 1.0, A.r, A.x);
    HB_CUDA(cudaMemcpyAsync(A.hb_, A.x, sizeof(double) * m, cudaMemcpyDeviceToHost, s));
    HB_CUDA(cudaStreamSynchronize(s));
    if (!A.Fc.fuse_k && A.nc > 0 && chol_solve_error()) ok = false;
    for (int p = 0; p < m; ++p) lhs[A.perm[p]] = A.hb_[p];
    return ok;
}

void KKT::arrow_info(double out[6]) const {
    // the dense M and its factor (L and the diagonal-block inverses; K and K^T below
    // kTriSolveMinM) for comparison
    const double ld = (double) pad_ld(m);
    out[5] = 8.0 * (ld * m * (m < kTriSolveMinM ? 4.0 : 2.0) + ld * 64);
    if (!arrow) {
        out[0] = out[1] = out[2] = out[3] = out[4] = 0.0;
        return;
    }
    out[0] = 1.0;
    out[1] = arrow->nc;
    out[2] = arrow->ncone;
    int mx = 0;
    for (int l : arrow->lk) mx = std::max(mx, l);
    out[3] = mx;
    out[4] = arrow->bytes;
}

}  // namespace hb
