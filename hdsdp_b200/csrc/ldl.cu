// Symmetric indefinite factorisation P A P^T = L D L^T with Bunch-Kaufman partial pivoting
// (1 x 1 and 2 x 2 pivots, alpha = (1 + sqrt 17) / 8) and its solve, on the device. This is
// the indefinite solver the reference switches its Schur system to when the Cholesky fails
// (linalg/hdsdp_linsolver.c:1367-1380 and :1407-1420 switch; :1118-1190 factor with LAPACK
// dsytrf and solve with dsytrs).
//
// Factorisation: one launch, right-looking and unblocked, on a grid of resident blocks
// (cooperative launch; one block for small orders). The trailing matrix is the lower
// triangle; column j belongs to block j mod grid for the whole factorisation. Each step:
//   - the pivot choice, taken by every thread from the pivot column's largest magnitude
//     below the diagonal (found by the column's owner at the end of the previous step) and,
//     when the diagonal is small, the largest magnitude in row / column imax (one
//     grid-wide reduction);
//   - the symmetric interchange, if any (one grid barrier);
//   - the rank-1 or rank-2 update of the trailing lower triangle, the multipliers written
//     transposed into the rows above it (U = L^T in the strictly upper triangle) (one grid
//     barrier).
// Every entry is formed by the same operations on any grid, so the factor does not depend
// on the grid. A zero pivot column (exactly singular) or a NaN pivot stops the
// factorisation with *info = step + 1.
//
// Solve (one block): y = P b; L z = y by 32-row blocks (dot products down the columns of
// U for the rows of the block, then one warp for the block's triangle); D w = z; L^T v = w
// by 32-row blocks from the bottom (one warp for the block's triangle, then axpys down the
// columns of U); x = P^T v.
#include "la.h"
#include <cooperative_groups.h>
#include <algorithm>
#include <cmath>

namespace cg = cooperative_groups;

namespace hb {
namespace {
constexpr int kLdlThreads = 512;
constexpr double kBkAlpha = 0.64038820320220756873;  // (1 + sqrt(17)) / 8
constexpr int kLdlBatch = 8;                          // owned columns whose loads are issued together
constexpr int kLdlSingleBlockMax = 384;               // orders factored by one block

struct LdlArgs {
    double *A;
    long ld;
    int n;
    int *perm, *piv, *info;
    // two slots of {largest magnitude below the diagonal of the pivot column, its row, the
    // pivot column's diagonal entry}: step t reads slot t & 1 while the owner of the next
    // pivot column fills slot (t + 1) & 1, so no block overwrites what a slower one has
    // still to read
    double *cm;
    double *part;   // per-block partial maxima of the row / column search
    int smemCols;   // 1: the pivot columns are staged in shared memory
};

__device__ __forceinline__ double ldcg(const double *p) { return __ldcg(p); }

// largest value (ties: smallest index) over the block; every thread gets the result
__device__ void block_argmax(double &v, int &idx) {
    __shared__ double rv[32];
    __shared__ int ri[32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    auto better = [](double a, int ia, double b, int ib) { return a > b || (a == b && ib < ia); };
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, v, o);
        const int oi = __shfl_xor_sync(0xffffffffu, idx, o);
        if (better(ov, oi, v, idx)) {
            v = ov;
            idx = oi;
        }
    }
    __syncthreads();
    if (lane == 0) {
        rv[w] = v;
        ri[w] = idx;
    }
    __syncthreads();
    v = rv[0];
    idx = ri[0];
    for (int q = 1; q < nw; ++q)
        if (better(rv[q], ri[q], v, idx)) {
            v = rv[q];
            idx = ri[q];
        }
}

// cm = {max_{i > j} |A(i, j)|, its row (j when the column has no entries below the
// diagonal), A(j, j)} over the lower triangle; called by one whole block
__device__ void column_argmax(const double *A, long ld, int n, int j, double *cm) {
    double v = -1.0;
    int idx = n;
    for (int i = j + 1 + threadIdx.x; i < n; i += blockDim.x) {
        const double a = fabs(ldcg(&A[i + (long) j * ld]));
        if (a > v) {
            v = a;
            idx = i;
        }
    }
    block_argmax(v, idx);
    if (threadIdx.x == 0) {
        cm[0] = (v < 0.0) ? 0.0 : v;
        cm[1] = (v < 0.0) ? (double) j : (double) idx;
        cm[2] = ldcg(&A[j + (long) j * ld]);
    }
}

template <class GSync>
__device__ void ldl_body(const LdlArgs P, int bid, int ngrid, GSync gsync, double *sm) {
    double *A = P.A;
    const long ld = P.ld;
    const int n = P.n, tid = threadIdx.x, nt = blockDim.x;
    const long gtid = (long) bid * nt + tid, gstride = (long) ngrid * nt;
    __shared__ double red[32];
    __shared__ double sdiag;   // the next pivot column's diagonal entry, as its owner updated it
    for (long i = gtid; i < n; i += gstride) {
        P.perm[i] = (int) i;
        P.piv[i] = 0;
    }
    if (bid == 0) column_argmax(A, ld, n, 0, P.cm);
    gsync();
    int k = 0;
    for (int step = 0; k < n; ++step) {
        // the decision's inputs: written before the last grid barrier and not written again
        // until every block has passed the next one
        const double *cmr = P.cm + 3 * (step & 1);
        double *cmw = P.cm + 3 * ((step + 1) & 1);
        const double colmax = ldcg(&cmr[0]);
        const int imax = (int) ldcg(&cmr[1]);
        const double akk = ldcg(&cmr[2]);
        const double absakk = fabs(akk);
        if (isnan(akk) || isnan(colmax) || !(fmax(absakk, colmax) > 0.0)) {
            if (gtid == 0) *P.info = k + 1;
            return;   // every block reads the same values and leaves here
        }
        int kp = k, kstep = 1;
        if (absakk < kBkAlpha * colmax) {
            // A(imax, imax) is read before the barrier below: after it, a faster block may
            // already be interchanging it
            const double aimax = fabs(ldcg(&A[imax + (long) imax * ld]));
            // the largest off-diagonal magnitude in row / column imax of the trailing matrix
            double mx = 0.0;
            for (long j = k + gtid; j < n; j += gstride) {
                if (j == imax) continue;
                const double v = (j < imax) ? ldcg(&A[imax + j * ld]) : ldcg(&A[j + (long) imax * ld]);
                mx = fmax(mx, fabs(v));
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
            if ((tid & 31) == 0) red[tid >> 5] = mx;
            __syncthreads();
            if (tid == 0) {
                double b = 0.0;
                for (int q = 0; q < (nt + 31) / 32; ++q) b = fmax(b, red[q]);
                P.part[bid] = b;
            }
            gsync();
            double rowmax = 0.0;
            for (int c = 0; c < ngrid; ++c) rowmax = fmax(rowmax, ldcg(&P.part[c]));
            if (absakk >= kBkAlpha * colmax * (colmax / rowmax)) {
                kp = k;
            } else if (aimax >= kBkAlpha * rowmax) {
                kp = imax;
            } else {
                kp = imax;
                kstep = 2;
            }
        }
        const int kk = k + kstep - 1;
        if (kp != kk) {
            // the symmetric interchange of kk and kp: (a) rows below kp of columns kk and kp,
            // (b) rows between of column kk with the columns between of row kp, (c) rows above
            // k of columns kk and kp (the multipliers of the earlier steps), (d) the two
            // diagonal entries, (e) for a 2 x 2 pivot, rows kk and kp of column k
            const long na = n - kp - 1, nb = kp - kk - 1, nc = k;
            const long total = na + nb + nc + 1 + (kstep == 2 ? 1 : 0);
            for (long t = gtid; t < total; t += gstride) {
                double *x, *y;
                if (t < na) {
                    const long i = kp + 1 + t;
                    x = &A[i + (long) kk * ld];
                    y = &A[i + (long) kp * ld];
                } else if (t < na + nb) {
                    const long i = kk + 1 + (t - na);
                    x = &A[i + (long) kk * ld];
                    y = &A[kp + i * ld];
                } else if (t < na + nb + nc) {
                    const long r = t - na - nb;
                    x = &A[r + (long) kk * ld];
                    y = &A[r + (long) kp * ld];
                } else if (t == na + nb + nc) {
                    x = &A[kk + (long) kk * ld];
                    y = &A[kp + (long) kp * ld];
                } else {
                    x = &A[kk + (long) k * ld];
                    y = &A[kp + (long) k * ld];
                }
                const double a = ldcg(x), b = ldcg(y);
                *x = b;
                *y = a;
            }
            if (gtid == 0) {
                const int tp = P.perm[kk];
                P.perm[kk] = P.perm[kp];
                P.perm[kp] = tp;
            }
            gsync();
        }
        if (gtid == 0) {
            P.piv[k] = kstep;
            if (kstep == 2) {
                P.piv[k + 1] = -1;
                A[k + (long) (k + 1) * ld] = 0.0;   // no multiplier inside the pivot block
            }
        }
        const int j0 = kk + 1, nr = n - j0;
        if (nr > 0) {
            // the pivot block: 1 / d, or the scaled inverse s [[d11, -1], [-1, d22]] of
            // [[a, b], [b, c]] with d11 = c / b, d22 = a / b, s = 1 / (b (d11 d22 - 1))
            const double a = ldcg(&A[k + (long) k * ld]);
            double dinv = 0.0, d11 = 0.0, d22 = 0.0, sc = 0.0;
            if (kstep == 1) {
                dinv = 1.0 / a;
            } else {
                const double b = ldcg(&A[k + 1 + (long) k * ld]), c = ldcg(&A[k + 1 + (long) (k + 1) * ld]);
                d11 = c / b;
                d22 = a / b;
                sc = (1.0 / (d11 * d22 - 1.0)) / b;
            }
            const double *g0 = A + j0 + (long) k * ld, *g1 = A + j0 + (long) (k + 1) * ld;
            double *s0 = sm, *s1 = sm + nr;
            const int first = j0 + (int) (((long) bid - j0 % ngrid + ngrid) % ngrid);   // first owned column
            const int nown = (first < n) ? (n - 1 - first) / ngrid + 1 : 0;
            double *mul0 = sm + (P.smemCols ? 2 * (size_t) nr : 0), *mul1 = mul0 + nown;
            if (nown > 0) {
                if (P.smemCols) {
                    for (int i = tid; i < nr; i += nt) {
                        s0[i] = ldcg(&g0[i]);
                        if (kstep == 2) s1[i] = ldcg(&g1[i]);
                    }
                }
                // multipliers of the owned columns' rows, also stored transposed above the diagonal
                for (int q = tid; q < nown; q += nt) {
                    const int j = first + q * ngrid;
                    const double x0 = ldcg(&g0[j - j0]);
                    if (kstep == 1) {
                        const double l = x0 * dinv;
                        mul0[q] = l;
                        A[k + (long) j * ld] = l;
                    } else {
                        const double x1 = ldcg(&g1[j - j0]);
                        const double w0 = sc * (d11 * x0 - x1), w1 = sc * (d22 * x1 - x0);
                        mul0[q] = w0;
                        mul1[q] = w1;
                        A[k + (long) j * ld] = w0;
                        A[k + 1 + (long) j * ld] = w1;
                    }
                }
                __syncthreads();
                const double *c0 = P.smemCols ? s0 : g0, *c1 = P.smemCols ? s1 : g1;
                const bool pivcol = (first == j0);   // this block owns the next pivot column
                double best = -1.0;
                int bidx = n;
                // rows i of this thread, owned columns j <= i in groups whose loads go out together
                for (int i = j0 + tid; i < n; i += nt) {
                    const double a0 = P.smemCols ? c0[i - j0] : ldcg(&c0[i - j0]);
                    const double a1 = (kstep == 2) ? (P.smemCols ? c1[i - j0] : ldcg(&c1[i - j0])) : 0.0;
                    const int qend = (i < first) ? 0 : min(nown, (i - first) / ngrid + 1);   // owned j <= i
                    for (int q0 = 0; q0 < qend; q0 += kLdlBatch) {
                        double v[kLdlBatch];
#pragma unroll
                        for (int u = 0; u < kLdlBatch; ++u) {
                            const int q = q0 + u;
                            v[u] = (q < qend) ? ldcg(&A[i + (long) (first + q * ngrid) * ld]) : 0.0;
                        }
#pragma unroll
                        for (int u = 0; u < kLdlBatch; ++u) {
                            const int q = q0 + u;
                            if (q < qend) {
                                const double nv = (kstep == 1) ? v[u] - a0 * mul0[q]
                                                               : v[u] - (a0 * mul0[q] + a1 * mul1[q]);
                                A[i + (long) (first + q * ngrid) * ld] = nv;
                                if (pivcol && q == 0) {
                                    const double m = fabs(nv);
                                    if (i == j0) {
                                        sdiag = nv;
                                    } else if (m > best) {
                                        best = m;
                                        bidx = i;
                                    }
                                }
                            }
                        }
                    }
                }
                if (pivcol) {
                    block_argmax(best, bidx);   // (its barriers also order this block's writes)
                    if (tid == 0) {
                        cmw[0] = (best < 0.0) ? 0.0 : best;
                        cmw[1] = (best < 0.0) ? (double) j0 : (double) bidx;
                        cmw[2] = sdiag;
                    }
                }
            }
        }
        gsync();
        k += kstep;
    }
}

__global__ void __launch_bounds__(kLdlThreads, 1) ldl_coop_kernel(const LdlArgs P) {
    extern __shared__ double sm[];
    cg::grid_group grid = cg::this_grid();
    ldl_body(P, (int) blockIdx.x, (int) gridDim.x, [&]() { grid.sync(); }, sm);
}

__global__ void __launch_bounds__(kLdlThreads, 1) ldl_block_kernel(const LdlArgs P) {
    extern __shared__ double sm[];
    ldl_body(P, 0, 1, []() {
        __threadfence_block();
        __syncthreads();
    }, sm);
}

// [w_k, w_k+1] = D_k^-1 [z_k, z_k+1] for the 2 x 2 pivot block at k (the factorisation's
// scaled form)
__device__ __forceinline__ void solve2(double a, double b, double c, double &z0, double &z1) {
    const double d11 = c / b, d22 = a / b, sc = (1.0 / (d11 * d22 - 1.0)) / b;
    const double w0 = sc * (d11 * z0 - z1), w1 = sc * (d22 * z1 - z0);
    z0 = w0;
    z1 = w1;
}

// x = A^-1 b from the factor; w is n doubles of scratch. One block of kLdlThreads threads.
__global__ void __launch_bounds__(kLdlThreads, 1) ldl_solve_kernel(const double *__restrict__ A, long ld, int n,
                                                             const int *__restrict__ perm,
                                                             const int *__restrict__ piv, const double *b,
                                                             double *x, double *w) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nt = blockDim.x, nwarp = nt >> 5;
    for (int i = tid; i < n; i += nt) w[i] = b[perm[i]];
    __syncthreads();
    // L z = y; L(i, r) = A(r, i) for r < i
    for (int i0 = 0; i0 < n; i0 += 32) {
        const int nbk = min(32, n - i0);
        for (int rr = warp; rr < nbk; rr += nwarp) {
            const int i = i0 + rr;
            double s = 0.0;
            for (int r = lane; r < i0; r += 32) s += A[r + (long) i * ld] * w[r];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            if (lane == 0) w[i] -= s;
        }
        __syncthreads();
        if (warp == 0) {
            double u[32];
#pragma unroll
            for (int r = 0; r < 32; ++r) u[r] = (r < lane && lane < nbk) ? A[(i0 + r) + (long) (i0 + lane) * ld] : 0.0;
            double y = (lane < nbk) ? w[i0 + lane] : 0.0;
#pragma unroll
            for (int r = 0; r < 32; ++r) {
                const double zr = __shfl_sync(0xffffffffu, y, r);
                y -= u[r] * zr;
            }
            if (lane < nbk) w[i0 + lane] = y;
        }
        __syncthreads();
    }
    // D w = z
    for (int i = tid; i < n; i += nt) {
        if (piv[i] == 1) {
            w[i] = w[i] / A[i + (long) i * ld];
        } else if (piv[i] == 2) {
            double z0 = w[i], z1 = w[i + 1];
            solve2(A[i + (long) i * ld], A[i + 1 + (long) i * ld], A[i + 1 + (long) (i + 1) * ld], z0, z1);
            w[i] = z0;
            w[i + 1] = z1;
        }
    }
    __syncthreads();
    // L^T v = w, blocks from the bottom; v(i) = w(i) - sum_{r > i} A(i, r) v(r)
    for (int r0 = ((n - 1) / 32) * 32; r0 >= 0; r0 -= 32) {
        const int nbk = min(32, n - r0);
        if (warp == 0) {
            double u[32];
#pragma unroll
            for (int r = 0; r < 32; ++r) u[r] = (lane < r && r < nbk) ? A[(r0 + lane) + (long) (r0 + r) * ld] : 0.0;
            double y = (lane < nbk) ? w[r0 + lane] : 0.0;
#pragma unroll
            for (int r = 31; r >= 0; --r) {
                const double vr = __shfl_sync(0xffffffffu, y, r);
                y -= u[r] * vr;
            }
            if (lane < nbk) w[r0 + lane] = y;
        }
        __syncthreads();
        for (int i = tid; i < r0; i += nt) {
            double s = 0.0;
            for (int q = 0; q < nbk; ++q) s += A[i + (long) (r0 + q) * ld] * w[r0 + q];
            w[i] -= s;
        }
        __syncthreads();
    }
    for (int i = tid; i < n; i += nt) x[perm[i]] = w[i];
}

__global__ void ldl_copy_kernel(int n, const double *S, long lds, double *A, long ld, int *info) {
    const long total = (long) n * n;
    for (long e = blockIdx.x * (long) blockDim.x + threadIdx.x; e < total; e += (long) gridDim.x * blockDim.x) {
        const long i = e % n, j = e / n;
        A[i + j * ld] = S[i + j * lds];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) *info = 0;
}

size_t ldl_smem(int n, int grid, bool cols) {
    const size_t nown = (size_t) n / grid + 2;
    return sizeof(double) * ((cols ? 2 * (size_t) n : 0) + 2 * nown);
}
constexpr size_t kLdlSmemMax = 200 * 1024;
}  // namespace

void LdlFactor::release() {
    for (double *p : {A, cm, part, w})
        if (p) hb::cache_free(p);
    for (int *p : {perm, piv, d_info})
        if (p) hb::cache_free(p);
    if (h_info) hb::cache_free_host(h_info);
    A = cm = part = w = h_info = nullptr;
    perm = piv = d_info = nullptr;
    n = 0;
    ok = false;
}

bool ldl_factorize(cudaStream_t s, LdlFactor &F, const double *S, long ldS, int n) {
    if (n <= 0) return false;
    if (F.n != n) {
        F.release();
        F.n = n;
        F.ld = (n + 1) & ~1L;
        HB_CUDA(hb::cmalloc(&F.A, sizeof(double) * F.ld * n));
        HB_CUDA(hb::cmalloc(&F.perm, sizeof(int) * n));
        HB_CUDA(hb::cmalloc(&F.piv, sizeof(int) * n));
        HB_CUDA(hb::cmalloc(&F.d_info, sizeof(int) * 4));
        HB_CUDA(hb::cmalloc(&F.cm, sizeof(double) * 6));
        HB_CUDA(hb::cmalloc(&F.part, sizeof(double) * kMaxLdlGrid));
        HB_CUDA(hb::cmalloc(&F.w, sizeof(double) * n));
        HB_CUDA(hb::cmalloc_host(&F.h_info, sizeof(double) * 2));
        if (!F.A || !F.perm || !F.piv || !F.d_info || !F.cm || !F.part || !F.w || !F.h_info) {
            F.release();
            return false;
        }
    }
    const long total = (long) n * n;
    const int cgrid = (int) std::min<long>(std::max<long>((total + 255) / 256, 1), 148L * 16);
    ldl_copy_kernel<<<hb::counted(cgrid), 256, 0, s>>>(n, S, ldS, F.A, F.ld, F.d_info);
    HB_CUDA(cudaGetLastError());
    LdlArgs P{F.A, F.ld, n, F.perm, F.piv, F.d_info, F.cm, F.part, 0};
    if (n <= kLdlSingleBlockMax) {
        P.smemCols = ldl_smem(n, 1, true) <= kLdlSmemMax ? 1 : 0;
        const size_t smem = ldl_smem(n, 1, P.smemCols);
        static std::atomic<unsigned long long> attr{0};
        once_per_device(attr, [] {
            HB_CUDA(cudaFuncSetAttribute((const void *) ldl_block_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int) kLdlSmemMax));
        });
        ldl_block_kernel<<<hb::counted(1), kLdlThreads, smem, s>>>(P);
        HB_CUDA(cudaGetLastError());
    } else {
        static std::atomic<int> resident[kMaxDevices];
        static std::atomic<unsigned long long> attr{0};
        const int dev = current_device();
        once_per_device(attr, [&] {
            HB_CUDA(cudaFuncSetAttribute((const void *) ldl_coop_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int) kLdlSmemMax));
            int per = 0;
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, ldl_coop_kernel, kLdlThreads, kLdlSmemMax);
            resident[dev].store(std::max(1, std::min(per, 1)) * device_sm_count());
        });
        const int grid = std::max(1, std::min({resident[dev].load(), kMaxLdlGrid, n}));
        P.smemCols = ldl_smem(n, grid, true) <= kLdlSmemMax ? 1 : 0;
        const size_t smem = ldl_smem(n, grid, P.smemCols);
        void *args[] = {&P};
        HB_CUDA(cudaLaunchCooperativeKernel((const void *) ldl_coop_kernel, hb::counted(grid), kLdlThreads, args, smem,
                                            s));
    }
    HB_CUDA(cudaMemcpyAsync(F.h_info, F.d_info, sizeof(int), cudaMemcpyDeviceToHost, s));
    HB_CUDA(cudaStreamSynchronize(s));
    F.ok = (reinterpret_cast<int *>(F.h_info)[0] == 0) && !device_error_flag();
    return F.ok;
}

void ldl_solve(cudaStream_t s, LdlFactor &F, const double *b, double *x) {
    ldl_solve_kernel<<<hb::counted(1), kLdlThreads, 0, s>>>(F.A, F.ld, F.n, F.perm, F.piv, b, x, F.w);
    HB_CUDA(cudaGetLastError());
}

}  // namespace hb
