// Kernels on the coefficient matrices of one dense SDP block.
//
// Reference formulas (interface/hdsdp_conic_sdp.c, linalg/hdsdp_sdpdata.c):
//   dual slack        S = dC*C + dA*sum_j w_j A_j + dEye*I   (sdpDenseConeIUpdateBuffer :343-402)
//   Schur matrix      M_ij = <A_i, W A_j W>                    (KKT2-KKT5 :683-981)
//   vectors           <A_j, W>, <A_j, W^2>                     (ASinv, ASinvRdSinv)
// For a symmetric sparse A = sum_e v_e (E_rc + E_cr) (diagonal entries once):
//   <A, Z>        = sum_e v_e * (r != c ? 2 Z_rc : Z_rr)
//   <A, W B W>    = sum_e sum_f v_e u_f * pair(e, f)       (pair below)
#include "sdp.h"
#include <cub/device/device_scan.cuh>
#include <cub/device/device_radix_sort.cuh>
#include <chrono>
#include <unordered_map>
#include <algorithm>
#include <cstring>

namespace hb {

namespace {

template <typename T>
T *upload_vec(const std::vector<T> &h, cudaStream_t s) {
    if (h.empty()) return nullptr;
    T *d = nullptr;
    HB_CUDA(hb::cmalloc(&d, sizeof(T) * h.size()));
    HB_CUDA(cudaMemcpyAsync(d, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice, s));
    return d;
}

// ---- rank-one gather map, built on the device. Row q of the coefficient factors lists
// the constraints whose support holds q, ascending, with a_jq (rptr / rj / ra). The
// entries of lower position (r, c) (packed index (2n - c - 1) c / 2 + r) are the merge
// of rows r and c. Launched on a grid of (row blocks, columns c); rows below c return.
__device__ __forceinline__ long long r1map_pos(int n, int r, int c) { return (long long) (2LL * n - c - 1) * c / 2 + r; }

// Lists longer than this leave the sliced layout for the warp-per-position one.
constexpr int kLongList = 64;

__global__ void r1map_count_kernel(int n, const int *__restrict__ rptr, const int *__restrict__ rj, int *cnt,
                                   int *used, int *longf) {
    const int c = blockIdx.y, r = c + blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    int x = rptr[r], xe = rptr[r + 1], y = rptr[c], ye = rptr[c + 1], k = 0;
    while (x < xe && y < ye) {
        const int a = rj[x], b = rj[y];
        if (a < b) ++x;
        else if (a > b) ++y;
        else { ++k; ++x; ++y; }
    }
    const long long q = r1map_pos(n, r, c);
    cnt[q] = k;
    used[q] = k > 0 && k <= kLongList;
    longf[q] = k > kLongList;
}

// used positions in packed order: row, column and entry count at their slot
// (short and long positions each in packed order: slot / lslot are their ranks)
__global__ void r1map_place_kernel(int n, const int *__restrict__ cnt, const int *__restrict__ slot, int *pr, int *pc,
                                   int *pcnt, const int *__restrict__ lslot, int *lr, int *lc, long long *llen) {
    const int c = blockIdx.y, r = c + blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    const long long q = r1map_pos(n, r, c);
    const int k = cnt[q];
    if (k == 0) return;
    if (k > kLongList) {
        const int sl = lslot[q];
        lr[sl] = r;
        lc[sl] = c;
        llen[sl] = k;
        return;
    }
    const int sl = slot[q];
    pr[sl] = r;
    pc[sl] = c;
    pcnt[sl] = k;
}

// positions reordered by list length (perm[i] = the packed rank of the i-th): row, column and
// count gathered to the new order, inv[perm[i]] = i
__global__ void r1map_permute_kernel(int npos, const int *__restrict__ perm, const int *__restrict__ pr,
                                     const int *__restrict__ pc, int *pr2, int *pc2, int *inv) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npos) return;
    const int p = perm[i];
    pr2[i] = pr[p];
    pc2[i] = pc[p];
    inv[p] = i;
}

__global__ void iota_kernel(int n, int *x) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[i] = i;
}

// slices of 32 positions padded to their longest list: 32 * max count per slice
__global__ void r1map_slice_kernel(int npos, int nslice, const int *__restrict__ pcnt, long long *len) {
    const int sl = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (sl > nslice) return;
    int k = 0;
    if (sl < nslice && sl * 32 + lane < npos) k = pcnt[sl * 32 + lane];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) k = max(k, __shfl_xor_sync(0xffffffffu, k, off));
    if (lane == 0) len[sl] = (sl < nslice) ? 32LL * k : 0LL;
}

// entry e of the short position at slot p lands at sptr[p / 32] + 32 e + p % 32, that of
// the long position at lslot p at lptr[p] + e; in constraint order, with value s_j a_jr a_jc
__global__ void r1map_fill_kernel(int n, const int *__restrict__ rptr, const int *__restrict__ rj,
                                  const double *__restrict__ ra, const double *__restrict__ sgn,
                                  const int *__restrict__ cnt, const int *__restrict__ slot,
                                  const int *__restrict__ inv, const long long *__restrict__ sptr, int *ej,
                                  double *ev, const int *__restrict__ lslot, const long long *__restrict__ lptr,
                                  int *lj, double *lv) {
    const int c = blockIdx.y, r = c + blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    const long long q = r1map_pos(n, r, c);
    const int k = cnt[q];
    if (k == 0) return;
    int *dj = ej;
    double *dv = ev;
    long long at, step;
    if (k > kLongList) {
        at = lptr[lslot[q]];
        step = 1;
        dj = lj;
        dv = lv;
    } else {
        const int sl = inv[slot[q]];
        at = sptr[sl >> 5] + (sl & 31);
        step = 32;
    }
    int x = rptr[r], xe = rptr[r + 1], y = rptr[c], ye = rptr[c + 1];
    while (x < xe && y < ye) {
        const int a = rj[x], b = rj[y];
        if (a < b) ++x;
        else if (a > b) ++y;
        else {
            dj[at] = a;
            dv[at] = sgn[a] * ra[x] * ra[y];
            at += step;
            ++x;
            ++y;
        }
    }
}

template <typename T>
void exclusive_sum(cudaStream_t s, const T *in, T *out, long long count) {
    size_t bytes = 0;
    HB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, (int64_t) count, s));
    void *tmp = nullptr;
    HB_CUDA(hb::cmalloc(&tmp, bytes));
    HB_CUDA(cub::DeviceScan::ExclusiveSum(tmp, bytes, in, out, (int64_t) count, s));
    hb::cache_free(tmp);
}

int grid1(long total, int threads = 256) {
    long b = (total + threads - 1) / threads;
    return (int) std::min<long>(std::max<long>(b, 1), 148L * 16);
}

// tr(E_ab' W E_cd' W) summed over the symmetric expansions of (a,b) and (c,d).
__device__ __forceinline__ double pair_term(const double *W, long ld, int a, int b, int c, int d) {
    auto w = [&](int i, int j) { return W[(size_t) i + (size_t) j * ld]; };
    if (a != b && c != d) return 2.0 * (w(b, c) * w(a, d) + w(b, d) * w(a, c));
    if (a == b && c != d) return 2.0 * w(a, c) * w(a, d);
    if (a != b && c == d) return 2.0 * w(a, c) * w(b, c);
    double x = w(a, c);
    return x * x;
}

__global__ void scatter_sym_kernel(int nnz, const int *r, const int *c, const double *v, double *A, long lda) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nnz; e += gridDim.x * blockDim.x) {
        A[(size_t) r[e] + (size_t) c[e] * lda] = v[e];
        A[(size_t) c[e] + (size_t) r[e] * lda] = v[e];
    }
}

__global__ void s_init_kernel(int n, const double *C, long ldc, double dC, double dEye, double *S, long lds) {
    const long total = (long) n * n;
    for (long idx = blockIdx.x * (long) blockDim.x + threadIdx.x; idx < total; idx += (long) gridDim.x * blockDim.x) {
        int r = (int) (idx % n), c = (int) (idx / n);
        double v = (dC != 0.0) ? dC * C[(size_t) r + (size_t) c * ldc] : 0.0;
        if (r == c) v += dEye;
        S[(size_t) r + (size_t) c * lds] = v;
    }
}

__global__ void s_gather_kernel(int npos, const int *pr, const int *pc, const int *ptr, const int *ej,
                                const double *ev, const double *w, double dA, double *S, long lds) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < npos; p += gridDim.x * blockDim.x) {
        double acc = 0.0;
        for (int e = ptr[p]; e < ptr[p + 1]; ++e) acc += ev[e] * w[ej[e]];
        acc *= dA;
        const int r = pr[p], c = pc[p];
        S[(size_t) r + (size_t) c * lds] += acc;
        if (r != c) S[(size_t) c + (size_t) r * lds] += acc;
    }
}

// Same as s_gather_kernel over the sliced rank-one gather map: a warp reads its slice's
// entries e for all 32 lanes at once (coalesced); each position sums in entry order.
__global__ void s_gather2_kernel(int npos, const int *pr, const int *pc, const long long *sptr, const int *cnt,
                                 const int *ej, const double *ev, const double *w, double dA, double *S, long lds) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < npos; p += gridDim.x * blockDim.x) {
        const long long base = sptr[p >> 5] + (p & 31);
        const int ne = cnt[p];
        double acc = 0.0;
        for (int e = 0; e < ne; ++e) acc += ev[base + 32LL * e] * w[ej[base + 32LL * e]];
        acc *= dA;
        const int r = pr[p], c = pc[p];
        S[(size_t) r + (size_t) c * lds] += acc;
        if (r != c) S[(size_t) c + (size_t) r * lds] += acc;
    }
}

// The long lists, one warp per position in the contiguous layout: lane l sums entries
// l, l + 32, ..., then the warp adds its lanes (a fixed order).
__global__ void s_gather2_long_kernel(int npos, const int *pr, const int *pc, const long long *ptr, const int *ej,
                                      const double *ev, const double *w, double dA, double *S, long lds) {
    const int lane = threadIdx.x & 31;
    for (int p = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; p < npos; p += (gridDim.x * blockDim.x) >> 5) {
        const long long b = ptr[p], e1 = ptr[p + 1];
        double acc = 0.0;
        for (long long e = b + lane; e < e1; e += 32) acc += ev[e] * w[ej[e]];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) {
            acc *= dA;
            const int r = pr[p], c = pc[p];
            S[(size_t) r + (size_t) c * lds] += acc;
            if (r != c) S[(size_t) c + (size_t) r * lds] += acc;
        }
    }
}

__global__ void r1d_weights_kernel(int k, const int *id, const double *sign, const double *w, double dA, double *d) {
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < k; a += gridDim.x * blockDim.x) d[a] = dA * sign[a] * w[id[a]];
}

__global__ void axpy_mat_devscale_kernel(int n, const double *A, long lda, const double *w, int j, double dA,
                                         double *S, long lds) {
    const double a = dA * w[j];
    if (a == 0.0) return;
    const long total = (long) n * n;
    for (long idx = blockIdx.x * (long) blockDim.x + threadIdx.x; idx < total; idx += (long) gridDim.x * blockDim.x) {
        int r = (int) (idx % n), c = (int) (idx / n);
        S[(size_t) r + (size_t) c * lds] += a * A[(size_t) r + (size_t) c * lda];
    }
}

// ---- Schur pair kernels -------------------------------------------------------------
__global__ void schur_spsp_kernel(int nsp, const int *id, const int *ptr, const int *rr, const int *cc,
                                  const double *vv, const double *W, long ldw, double *M, long ldm) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    const int b = blockIdx.y * blockDim.y + threadIdx.y;
    if (a >= nsp || b > a) return;
    double acc = 0.0;
    for (int e = ptr[a]; e < ptr[a + 1]; ++e)
        for (int f = ptr[b]; f < ptr[b + 1]; ++f) acc += vv[e] * vv[f] * pair_term(W, ldw, rr[e], cc[e], rr[f], cc[f]);
    M[(size_t) id[a] + (size_t) id[b] * ldm] = acc;
}

__global__ void schur_r1s_kernel(int k, const int *id, const int *ptr, const int *pp, const double *aa,
                                 const double *sg, const double *W, long ldw, double *M, long ldm) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    const int b = blockIdx.y * blockDim.y + threadIdx.y;
    if (a >= k || b > a) return;
    double g = 0.0;
    for (int t = ptr[a]; t < ptr[a + 1]; ++t) {
        double gt = 0.0;
        for (int u = ptr[b]; u < ptr[b + 1]; ++u) gt += aa[u] * W[(size_t) pp[t] + (size_t) pp[u] * ldw];
        g += aa[t] * gt;
    }
    M[(size_t) id[a] + (size_t) id[b] * ldm] = sg[a] * sg[b] * g * g;
}

__global__ void schur_hadamard_kernel(int k, const int *id, const double *sg, const double *G, long ldg,
                                      double *M, long ldm) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    const int b = blockIdx.y * blockDim.y + threadIdx.y;
    if (a >= k || b > a) return;
    const double g = G[(size_t) a + (size_t) b * ldg];
    M[(size_t) id[a] + (size_t) id[b] * ldm] = sg[a] * sg[b] * g * g;
}

// (a in R1D with column V[:,a]) x (b in R1S): (a_b^T v_a)^2 s_a s_b
__global__ void schur_r1d_r1s_kernel(int kd, const int *idd, const double *sgd, const double *V, long ldv,
                                     int ks, const int *ids, const int *ptr, const int *pp, const double *aa,
                                     const double *sgs, double *M, long ldm) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    const int a = blockIdx.y * blockDim.y + threadIdx.y;
    if (a >= kd || b >= ks) return;
    double g = 0.0;
    for (int u = ptr[b]; u < ptr[b + 1]; ++u) g += aa[u] * V[(size_t) pp[u] + (size_t) a * ldv];
    const int i = idd[a], j = ids[b];
    const int hi = max(i, j), lo = min(i, j);
    M[(size_t) hi + (size_t) lo * ldm] = sgd[a] * sgs[b] * g * g;
}

// V[:, b] = sum_t a_t W[:, p_t] for R1S constraints
__global__ void r1s_build_v_kernel(int n, int ks, const int *ptr, const int *pp, const double *aa,
                                   const double *W, long ldw, double *V, long ldv) {
    const int b = blockIdx.y;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        double acc = 0.0;
        for (int t = ptr[b]; t < ptr[b + 1]; ++t) acc += aa[t] * W[(size_t) k + (size_t) pp[t] * ldw];
        V[(size_t) k + (size_t) b * ldv] = acc;
    }
}

// (a: rank one with column V[:,a], sign sg) x (b in SP): s_a * v^T A_b v
__global__ void schur_r1_sp_kernel(int kr, const int *idr, const double *sgr, const double *V, long ldv,
                                   int nsp, const int *ids, const int *ptr, const int *rr, const int *cc,
                                   const double *vv, double *M, long ldm) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    const int a = blockIdx.y * blockDim.y + threadIdx.y;
    if (a >= kr || b >= nsp) return;
    const double *v = V + (size_t) a * ldv;
    double acc = 0.0;
    for (int f = ptr[b]; f < ptr[b + 1]; ++f) {
        const int r = rr[f], c = cc[f];
        acc += vv[f] * ((r != c) ? 2.0 * v[r] * v[c] : v[r] * v[r]);
    }
    const int i = idr[a], j = ids[b];
    const int hi = max(i, j), lo = min(i, j);
    M[(size_t) hi + (size_t) lo * ldm] = sgr[a] * acc;
}

__global__ void scatter_row_kernel(int m, int i, const double *t, double *M, long ldm) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < m; j += gridDim.x * blockDim.x) {
        const int hi = max(i, j), lo = min(i, j);
        M[(size_t) hi + (size_t) lo * ldm] = t[j];
    }
}

// ---- inner products -------------------------------------------------------------------
__global__ void inner_sp_kernel(int nsp, const int *id, const int *ptr, const int *rr, const int *cc,
                                const double *vv, const double *Z, long ldz, double *out) {
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < nsp; a += gridDim.x * blockDim.x) {
        double acc = 0.0;
        for (int e = ptr[a]; e < ptr[a + 1]; ++e) {
            const int r = rr[e], c = cc[e];
            const double z = Z[(size_t) r + (size_t) c * ldz];
            acc += vv[e] * ((r != c) ? 2.0 * z : z);
        }
        out[id[a]] = acc;
    }
}

__global__ void inner_r1s_kernel(int k, const int *id, const int *ptr, const int *pp, const double *aa,
                                 const double *sg, const double *Z, long ldz, double *out) {
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < k; a += gridDim.x * blockDim.x) {
        double acc = 0.0;
        for (int t = ptr[a]; t < ptr[a + 1]; ++t) {
            double at = 0.0;
            for (int u = ptr[a]; u < ptr[a + 1]; ++u) at += aa[u] * Z[(size_t) pp[t] + (size_t) pp[u] * ldz];
            acc += aa[t] * at;
        }
        out[id[a]] = sg[a] * acc;
    }
}

// out[id[a]] = sg[a] * sum_k X[k,a] * Y[k,a]   (warp per column)
__global__ void coldot_pair_kernel(int n, int k, const int *id, const double *sg, const double *X, long ldx,
                                   const double *Y, long ldy, double *out) {
    const int a = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (a >= k) return;
    const double *x = X + (size_t) a * ldx;
    const double *y = Y + (size_t) a * ldy;
    double acc = 0.0;
    for (int r = lane; r < n; r += 32) acc += x[r] * y[r];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) out[id[a]] = sg[a] * acc;
}

// out[id_a] = s_a G_aa
__global__ void r1d_diag_kernel(int k, const int *id, const double *sg, const double *G, long ldg, double *out) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a < k) out[id[a]] = sg[a] * G[(size_t) a * (ldg + 1)];
}

// out[id_a] = s_a v_a
__global__ void r1d_scatter_kernel(int k, const int *id, const double *sg, const double *v, double *out) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a < k) out[id[a]] = sg[a] * v[a];
}

// <A_a, W^2> for SP: sum_e v_e (r != c ? 2 : 1) * W[:,r].W[:,c]   (warp per constraint)
__global__ void innersq_sp_kernel(int n, int nsp, const int *id, const int *ptr, const int *rr, const int *cc,
                                  const double *vv, const double *W, long ldw, double *out) {
    const int a = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (a >= nsp) return;
    double acc = 0.0;
    for (int e = ptr[a]; e < ptr[a + 1]; ++e) {
        const int r = rr[e], c = cc[e];
        const double *wr = W + (size_t) r * ldw;
        const double *wc = W + (size_t) c * ldw;
        double d = 0.0;
        for (int k = lane; k < n; k += 32) d += wr[k] * wc[k];
        acc += vv[e] * ((r != c) ? 2.0 : 1.0) * d;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) out[id[a]] = acc;
}

// <A_a, W^2> for R1S: s * || sum_t a_t W[:, p_t] ||^2   (warp per constraint)
__global__ void innersq_r1s_kernel(int n, int k, const int *id, const int *ptr, const int *pp, const double *aa,
                                   const double *sg, const double *W, long ldw, double *out) {
    const int a = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (a >= k) return;
    double acc = 0.0;
    for (int r = lane; r < n; r += 32) {
        double v = 0.0;
        for (int t = ptr[a]; t < ptr[a + 1]; ++t) v += aa[t] * W[(size_t) r + (size_t) pp[t] * ldw];
        acc += v * v;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) out[id[a]] = sg[a] * acc;
}

// sum over i < n of f(i) as a 1024-thread block forms it (one term per thread, a shuffle tree
// per warp, then one over the 32 warp sums; n <= 1024), by a block of 256 threads
template <class F>
__device__ double sum_as_1024(int n, F f) {
    __shared__ double red[32];
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int v = t + 256 * q;
        double x = (v < n) ? f(v) : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if (lane == 0) red[w + 8 * q] = x;
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

__global__ void __launch_bounds__(256) schur_build_batch_kernel(const SchurBuildJob *__restrict__ jobs) {
    const SchurBuildJob J = jobs[blockIdx.x];
    const int n = J.n, tid = threadIdx.x, nt = blockDim.x;
    double *W = J.W;
    const long ldw = J.ldW;
    // W(j, i) = W(i, j), i > j
    for (long idx = tid; idx < (long) n * n; idx += nt) {
        const int i = (int) (idx % n), j = (int) (idx / n);
        if (i > j) W[(size_t) j + (size_t) i * ldw] = W[(size_t) i + (size_t) j * ldw];
    }
    __syncthreads();
    if (J.trace) {
        const double tr = sum_as_1024(n, [&](int i) { return W[(size_t) i + (size_t) i * ldw]; });
        if (tid == 0) *J.trace = tr;
    }
    const int nsp = J.nsp, nr1s = J.nr1s;
    if (J.M) {
        double *M = J.M;
        const long ldm = J.ldM;
        for (long idx = tid; idx < ldm * J.m; idx += nt) M[idx] = 0.0;
        __syncthreads();
        for (long t = tid; t < (long) nsp * nsp; t += nt) {   // schur_spsp_kernel
            const int a = (int) (t % nsp), b = (int) (t / nsp);
            if (b > a) continue;
            const int *ptr = J.sp_ptr, *rr = J.sp_r, *cc = J.sp_c;
            const double *vv = J.sp_v;
            double acc = 0.0;
            for (int e = ptr[a]; e < ptr[a + 1]; ++e)
                for (int f = ptr[b]; f < ptr[b + 1]; ++f)
                    acc += vv[e] * vv[f] * pair_term(W, ldw, rr[e], cc[e], rr[f], cc[f]);
            M[(size_t) J.sp_id[a] + (size_t) J.sp_id[b] * ldm] = acc;
        }
        for (long t = tid; t < (long) nr1s * nr1s; t += nt) {   // schur_r1s_kernel
            const int a = (int) (t % nr1s), b = (int) (t / nr1s);
            if (b > a) continue;
            const int *ptr = J.r1s_ptr, *pp = J.r1s_p;
            const double *aa = J.r1s_a;
            double g = 0.0;
            for (int u0 = ptr[a]; u0 < ptr[a + 1]; ++u0) {
                double gt = 0.0;
                for (int u = ptr[b]; u < ptr[b + 1]; ++u) gt += aa[u] * W[(size_t) pp[u0] + (size_t) pp[u] * ldw];
                g += aa[u0] * gt;
            }
            M[(size_t) J.r1s_id[a] + (size_t) J.r1s_id[b] * ldm] = J.r1s_sign[a] * J.r1s_sign[b] * g * g;
        }
        if (nr1s > 0 && nsp > 0) {
            for (long t = tid; t < (long) n * nr1s; t += nt) {   // r1s_build_v_kernel
                const int k = (int) (t % n), b = (int) (t / n);
                double acc = 0.0;
                for (int u = J.r1s_ptr[b]; u < J.r1s_ptr[b + 1]; ++u)
                    acc += J.r1s_a[u] * W[(size_t) k + (size_t) J.r1s_p[u] * ldw];
                J.Vs[(size_t) k + (size_t) b * J.ldv] = acc;
            }
            __syncthreads();
            for (long t = tid; t < (long) nsp * nr1s; t += nt) {   // schur_r1_sp_kernel
                const int b = (int) (t % nsp), a = (int) (t / nsp);
                const double *v = J.Vs + (size_t) a * J.ldv;
                double acc = 0.0;
                for (int f = J.sp_ptr[b]; f < J.sp_ptr[b + 1]; ++f) {
                    const int r = J.sp_r[f], c = J.sp_c[f];
                    acc += J.sp_v[f] * ((r != c) ? 2.0 * v[r] * v[c] : v[r] * v[r]);
                }
                const int i = J.r1s_id[a], j = J.sp_id[b];
                const int hi = max(i, j), lo = min(i, j);
                M[(size_t) hi + (size_t) lo * ldm] = J.r1s_sign[a] * acc;
            }
        }
    }
    // inner_all
    if (nsp + nr1s < J.m)
        for (int i = tid; i < J.m; i += nt) J.inner[i] = 0.0;
    __syncthreads();
    for (int a = tid; a < nsp; a += nt) {   // inner_sp_kernel
        double acc = 0.0;
        for (int e = J.sp_ptr[a]; e < J.sp_ptr[a + 1]; ++e) {
            const int r = J.sp_r[e], c = J.sp_c[e];
            const double z = W[(size_t) r + (size_t) c * ldw];
            acc += J.sp_v[e] * ((r != c) ? 2.0 * z : z);
        }
        J.inner[J.sp_id[a]] = acc;
    }
    for (int a = tid; a < nr1s; a += nt) {   // inner_r1s_kernel
        double acc = 0.0;
        for (int u0 = J.r1s_ptr[a]; u0 < J.r1s_ptr[a + 1]; ++u0) {
            double at = 0.0;
            for (int u = J.r1s_ptr[a]; u < J.r1s_ptr[a + 1]; ++u)
                at += J.r1s_a[u] * W[(size_t) J.r1s_p[u0] + (size_t) J.r1s_p[u] * ldw];
            acc += J.r1s_a[u0] * at;
        }
        J.inner[J.r1s_id[a]] = J.r1s_sign[a] * acc;
    }
    if (!J.innersq) return;
    // inner_all_sq: one warp per constraint, as innersq_sp_kernel / innersq_r1s_kernel
    __syncthreads();
    if (nsp + nr1s < J.m)
        for (int i = tid; i < J.m; i += nt) J.innersq[i] = 0.0;
    __syncthreads();
    const int lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
    for (int a = warp; a < nsp; a += nw) {
        double acc = 0.0;
        for (int e = J.sp_ptr[a]; e < J.sp_ptr[a + 1]; ++e) {
            const int r = J.sp_r[e], c = J.sp_c[e];
            const double *wr = W + (size_t) r * ldw;
            const double *wc = W + (size_t) c * ldw;
            double d = 0.0;
            for (int k = lane; k < n; k += 32) d += wr[k] * wc[k];
            acc += J.sp_v[e] * ((r != c) ? 2.0 : 1.0) * d;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) J.innersq[J.sp_id[a]] = acc;
    }
    for (int a = warp; a < nr1s; a += nw) {
        double acc = 0.0;
        for (int r = lane; r < n; r += 32) {
            double v = 0.0;
            for (int u = J.r1s_ptr[a]; u < J.r1s_ptr[a + 1]; ++u) v += J.r1s_a[u] * W[(size_t) r + (size_t) J.r1s_p[u] * ldw];
            acc += v * v;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) J.innersq[J.r1s_id[a]] = J.r1s_sign[a] * acc;
    }
}

}  // namespace

void schur_build_batch(cudaStream_t s, const SchurBuildJob *d_jobs, int count) {
    for (int b0 = 0; b0 < count; b0 += 65535) {
        schur_build_batch_kernel<<<hb::counted(std::min(65535, count - b0)), 256, 0, s>>>(d_jobs + b0);
        HB_CUDA(cudaGetLastError());
    }
}

SchurBuildJob schur_build_job(const SdpDevice &d, double *W, long ldW, double *M, long ldM) {
    SchurBuildJob J{};
    J.W = W;
    J.ldW = ldW;
    J.n = d.n;
    J.m = d.m;
    J.M = M;
    J.ldM = ldM;
    J.nsp = d.nsp;
    J.sp_id = d.sp_id;
    J.sp_ptr = d.sp_ptr;
    J.sp_r = d.sp_r;
    J.sp_c = d.sp_c;
    J.sp_v = d.sp_v;
    J.nr1s = d.nr1s;
    J.r1s_id = d.r1s_id;
    J.r1s_ptr = d.r1s_ptr;
    J.r1s_p = d.r1s_p;
    J.r1s_a = d.r1s_a;
    J.r1s_sign = d.r1s_sign;
    J.Vs = d.Vs;
    J.ldv = d.ld;
    return J;
}

static double host_seconds() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

void SdpDevice::upload(int n_, int m_, const HostCoeff &C, const std::vector<HostCoeff> &A, cudaStream_t s) {
    const double tu0 = host_seconds();
    n = n_;
    m = m_;
    ld = pad_ld(n);
    stream = s;
    HB_CUDA(hb::cmalloc(&Cfull, sizeof(double) * ld * n));
    HB_CUDA(cudaMemsetAsync(Cfull, 0, sizeof(double) * ld * n, s));
    if (!C.r.empty()) {
        int *dr = upload_vec(C.r, s), *dc = upload_vec(C.c, s);
        double *dv = upload_vec(C.v, s);
        scatter_sym_kernel<<<hb::counted(grid1((long) C.r.size())), 256, 0, s>>>((int) C.r.size(), dr, dc, dv, Cfull, ld);
        HB_CUDA(cudaStreamSynchronize(s));
        hb::cache_free(dr);
        hb::cache_free(dc);
        hb::cache_free(dv);
    }

    std::vector<int> spid, spptr{0}, spr, spc;
    std::vector<double> spv;
    std::vector<int> r1sid, r1sptr{0}, r1sp;
    std::vector<double> r1sa, r1ssg;
    std::vector<int> r1did;
    std::vector<double> r1dsg;
    std::vector<std::pair<int, int>> r1d_src;  // (constraint, unused)
    // gather map: key = r * n + c
    std::unordered_map<long long, std::vector<std::pair<int, double>>> posmap;
    std::vector<long long> posorder;
    auto addpos = [&](int r, int c, int j, double v) {
        long long key = (long long) r * n + c;
        auto it = posmap.find(key);
        if (it == posmap.end()) {
            posorder.push_back(key);
            posmap[key].push_back({j, v});
        } else {
            it->second.push_back({j, v});
        }
    };

    for (int j = 0; j < m; ++j) {
        const HostCoeff &a = A[j];
        if (a.cls == CLS_SP) {
            spid.push_back(j);
            for (size_t e = 0; e < a.r.size(); ++e) {
                spr.push_back(a.r[e]);
                spc.push_back(a.c[e]);
                spv.push_back(a.v[e]);
                addpos(a.r[e], a.c[e], j, a.v[e]);
            }
            spptr.push_back((int) spr.size());
        } else if (a.cls == CLS_R1S) {
            r1sid.push_back(j);
            r1ssg.push_back(a.sign);
            for (size_t t = 0; t < a.aidx.size(); ++t) {
                r1sp.push_back(a.aidx[t]);
                r1sa.push_back(a.aval[t]);
            }
            r1sptr.push_back((int) r1sp.size());
            for (size_t t = 0; t < a.aidx.size(); ++t)
                for (size_t u = 0; u <= t; ++u)
                    addpos(a.aidx[t], a.aidx[u], j, a.sign * a.aval[t] * a.aval[u]);
        } else if (a.cls == CLS_R1D) {
            r1did.push_back(j);
            r1dsg.push_back(a.sign);
        } else if (a.cls == CLS_DR) {
            dr_id.push_back(j);
        }
    }

    nsp = (int) spid.size();
    sp_id = upload_vec(spid, s);
    sp_ptr = upload_vec(spptr, s);
    sp_r = upload_vec(spr, s);
    sp_c = upload_vec(spc, s);
    sp_v = upload_vec(spv, s);

    nr1s = (int) r1sid.size();
    r1s_id = upload_vec(r1sid, s);
    r1s_ptr = upload_vec(r1sptr, s);
    r1s_p = upload_vec(r1sp, s);
    r1s_a = upload_vec(r1sa, s);
    r1s_sign = upload_vec(r1ssg, s);

    nr1d = (int) r1did.size();
    r1d_id = upload_vec(r1did, s);
    r1d_sign = upload_vec(r1dsg, s);
    if (nr1d > 0) {
        std::vector<double> hA1((size_t) ld * nr1d, 0.0);
        for (int a = 0; a < nr1d; ++a) {
            const HostCoeff &c = A[r1did[a]];
            for (size_t t = 0; t < c.aidx.size(); ++t) hA1[(size_t) a * ld + c.aidx[t]] = c.aval[t];
        }
        A1 = upload_vec(hA1, s);
        HB_CUDA(hb::cmalloc(&G, sizeof(double) * pad_ld(nr1d) * nr1d));
        if (precision >= 1) {
            // the factors a_i are fixed: split them once
            bool ok = opA1.alloc(nr1d, n) && opK.alloc(n, n) && opKT.alloc(n, n) && opB.alloc(nr1d, n);
            HB_CUDA(hb::cmalloc(&colsq, sizeof(double) * nr1d));
            if (ok) split_from_f64(s, opA1, A1, ld, true);
            else opA1.release();
        }
    }
    const int vcols = std::max(std::max(nr1d, nr1s), 1);
    HB_CUDA(hb::cmalloc(&V, sizeof(double) * ld * vcols));
    if (nr1d > 0) HB_CUDA(hb::cmalloc(&Vt, sizeof(double) * ld * nr1d));
    if (nr1s > 0 && nsp > 0) HB_CUDA(hb::cmalloc(&Vs, sizeof(double) * ld * nr1s));

    ndr = (int) dr_id.size();
    for (int i = 0; i < ndr; ++i) {
        const HostCoeff &c = A[dr_id[i]];
        double *mat = nullptr;
        HB_CUDA(hb::cmalloc(&mat, sizeof(double) * ld * n));
        HB_CUDA(cudaMemsetAsync(mat, 0, sizeof(double) * ld * n, s));
        int *dr = upload_vec(c.r, s), *dc = upload_vec(c.c, s);
        double *dv = upload_vec(c.v, s);
        if (!c.r.empty())
            scatter_sym_kernel<<<hb::counted(grid1((long) c.r.size())), 256, 0, s>>>((int) c.r.size(), dr, dc, dv, mat, ld);
        HB_CUDA(cudaStreamSynchronize(s));
        hb::cache_free(dr);
        hb::cache_free(dc);
        hb::cache_free(dv);
        dr_mat.push_back(mat);
    }

    // S-assembly gather map
    std::vector<int> pr, pc, pptr{0}, ej;
    std::vector<double> ev;
    pr.reserve(posorder.size());
    for (long long key : posorder) {
        pr.push_back((int) (key / n));
        pc.push_back((int) (key % n));
        for (auto &e : posmap[key]) {
            ej.push_back(e.first);
            ev.push_back(e.second);
        }
        pptr.push_back((int) ej.size());
    }
    npos = (int) pr.size();
    pos_r = upload_vec(pr, s);
    pos_c = upload_vec(pc, s);
    pos_ptr = upload_vec(pptr, s);
    ent_j = upload_vec(ej, s);
    ent_v = upload_vec(ev, s);

    // Rank-one gather map: cheaper than the rank-nr1d GEMM when its bytes (12 per entry)
    // stay under a quarter of the GEMM's flops (DMMA ~20 TFLOP/s against ~5 TB/s HBM).
    r1d_gather = false;
    const double tm0 = host_seconds();
    if (nr1d > 0) {
        long long entries = 0;
        for (int j : r1did) {
            const long long k = (long long) A[j].aidx.size();
            entries += k * (k + 1) / 2;
        }
        const double gemm_flops = 2.0 * n * (double) n * nr1d;
        if (12.0 * (double) entries < 0.25 * gemm_flops && (long long) n * (n + 1) / 2 < (1LL << 31)) {
            // Per row q, the constraints whose support holds q, ascending, with a_jq (host).
            // The entries of lower position (r, c) are the merge of rows r and c, in
            // constraint order, with values s_j a_jr a_jc; the merges, the compaction of
            // the used positions and the sliced layout run on the device (r1map_*).
            std::vector<int> rptr(n + 1, 0);
            for (int j : r1did)
                for (int q : A[j].aidx) rptr[q + 1] += 1;
            for (int q = 0; q < n; ++q) rptr[q + 1] += rptr[q];
            std::vector<int> rj(rptr[n]);
            std::vector<double> ra(rptr[n]);
            {
                std::vector<int> fill(rptr.begin(), rptr.end() - 1);
                for (int j : r1did) {  // r1did ascending: each row list ends up sorted by j
                    const HostCoeff &a = A[j];
                    for (size_t t = 0; t < a.aidx.size(); ++t) {
                        const int at = fill[a.aidx[t]]++;
                        rj[at] = j;
                        ra[at] = a.aval[t];
                    }
                }
            }
            std::vector<double> sgn(m, 0.0);
            for (int j : r1did) sgn[j] = A[j].sign;
            // the map itself is built on the device from the row lists
            const long long npack = (long long) n * (n + 1) / 2;
            int *d_rptr = upload_vec(rptr, s), *d_rj = upload_vec(rj, s);
            double *d_ra = upload_vec(ra, s), *d_sgn = upload_vec(sgn, s);
            int *d_cnt = nullptr, *d_used = nullptr, *d_slot = nullptr, *d_long = nullptr, *d_lslot = nullptr;
            HB_CUDA(hb::cmalloc(&d_cnt, sizeof(int) * npack));
            HB_CUDA(hb::cmalloc(&d_used, sizeof(int) * npack));
            HB_CUDA(hb::cmalloc(&d_slot, sizeof(int) * npack));
            HB_CUDA(hb::cmalloc(&d_long, sizeof(int) * npack));
            HB_CUDA(hb::cmalloc(&d_lslot, sizeof(int) * npack));
            const dim3 pgrid((n + 255) / 256, n);
            r1map_count_kernel<<<hb::counted(pgrid), 256, 0, s>>>(n, d_rptr, d_rj, d_cnt, d_used, d_long);
            exclusive_sum(s, d_used, d_slot, npack);
            exclusive_sum(s, d_long, d_lslot, npack);
            int tail[4] = {0, 0, 0, 0};
            HB_CUDA(cudaMemcpyAsync(&tail[0], d_slot + npack - 1, sizeof(int), cudaMemcpyDeviceToHost, s));
            HB_CUDA(cudaMemcpyAsync(&tail[1], d_used + npack - 1, sizeof(int), cudaMemcpyDeviceToHost, s));
            HB_CUDA(cudaMemcpyAsync(&tail[2], d_lslot + npack - 1, sizeof(int), cudaMemcpyDeviceToHost, s));
            HB_CUDA(cudaMemcpyAsync(&tail[3], d_long + npack - 1, sizeof(int), cudaMemcpyDeviceToHost, s));
            HB_CUDA(cudaStreamSynchronize(s));
            npos2 = tail[0] + tail[1];
            nposL = tail[2] + tail[3];
            HB_CUDA(hb::cmalloc(&posL_r, sizeof(int) * std::max(nposL, 1)));
            HB_CUDA(hb::cmalloc(&posL_c, sizeof(int) * std::max(nposL, 1)));
            HB_CUDA(hb::cmalloc(&posL_ptr, sizeof(long long) * (nposL + 1)));
            long long *d_llen = nullptr;
            HB_CUDA(hb::cmalloc(&d_llen, sizeof(long long) * (nposL + 1)));
            HB_CUDA(cudaMemsetAsync(d_llen, 0, sizeof(long long) * (nposL + 1), s));
            const int nslice = (npos2 + 31) / 32;
            HB_CUDA(hb::cmalloc(&pos2_r, sizeof(int) * std::max(npos2, 1)));
            HB_CUDA(hb::cmalloc(&pos2_c, sizeof(int) * std::max(npos2, 1)));
            HB_CUDA(hb::cmalloc(&pos2_cnt, sizeof(int) * std::max(npos2, 1)));
            HB_CUDA(hb::cmalloc(&pos2_ptr, sizeof(long long) * (nslice + 1)));
            long long *d_len = nullptr;
            HB_CUDA(hb::cmalloc(&d_len, sizeof(long long) * (nslice + 1)));
            r1map_place_kernel<<<hb::counted(pgrid), 256, 0, s>>>(n, d_cnt, d_slot, pos2_r, pos2_c, pos2_cnt, d_lslot,
                                                                  posL_r, posL_c, d_llen);
            exclusive_sum(s, d_llen, posL_ptr, (long long) nposL + 1);
            long long totalL = 0;
            HB_CUDA(cudaMemcpyAsync(&totalL, posL_ptr + nposL, sizeof(long long), cudaMemcpyDeviceToHost, s));
            // the short positions ordered by list length (a stable sort: packed order within a
            // length), so that the 32 positions of a slice have lists of about the same length
            // and the slices carry little padding; each position's sum is unchanged
            int *d_inv = nullptr;
            HB_CUDA(hb::cmalloc(&d_inv, sizeof(int) * std::max(npos2, 1)));
            if (npos2 > 0) {
                int *d_iota = nullptr, *d_perm = nullptr, *d_cnt2 = nullptr, *d_r2 = nullptr, *d_c2 = nullptr;
                for (int **p : {&d_iota, &d_perm, &d_cnt2, &d_r2, &d_c2}) HB_CUDA(hb::cmalloc(p, sizeof(int) * npos2));
                iota_kernel<<<hb::counted((npos2 + 255) / 256), 256, 0, s>>>(npos2, d_iota);
                size_t bytes = 0;
                HB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, bytes, pos2_cnt, d_cnt2, d_iota, d_perm, npos2, 0,
                                                        8, s));
                void *tmp = nullptr;
                HB_CUDA(hb::cmalloc(&tmp, bytes));
                HB_CUDA(cub::DeviceRadixSort::SortPairs(tmp, bytes, pos2_cnt, d_cnt2, d_iota, d_perm, npos2, 0, 8, s));
                r1map_permute_kernel<<<hb::counted((npos2 + 255) / 256), 256, 0, s>>>(npos2, d_perm, pos2_r, pos2_c,
                                                                                     d_r2, d_c2, d_inv);
                HB_CUDA(cudaMemcpyAsync(pos2_r, d_r2, sizeof(int) * npos2, cudaMemcpyDeviceToDevice, s));
                HB_CUDA(cudaMemcpyAsync(pos2_c, d_c2, sizeof(int) * npos2, cudaMemcpyDeviceToDevice, s));
                HB_CUDA(cudaMemcpyAsync(pos2_cnt, d_cnt2, sizeof(int) * npos2, cudaMemcpyDeviceToDevice, s));
                HB_CUDA(cudaStreamSynchronize(s));
                hb::cache_free(tmp);
                for (int *p : {d_iota, d_perm, d_cnt2, d_r2, d_c2}) hb::cache_free(p);
            }
            r1map_slice_kernel<<<hb::counted((int) ((32LL * (nslice + 1) + 255) / 256)), 256, 0, s>>>(
                npos2, nslice, pos2_cnt, d_len);
            exclusive_sum(s, d_len, pos2_ptr, (long long) nslice + 1);
            long long total = 0;
            HB_CUDA(cudaMemcpyAsync(&total, pos2_ptr + nslice, sizeof(long long), cudaMemcpyDeviceToHost, s));
            HB_CUDA(cudaStreamSynchronize(s));
            HB_CUDA(hb::cmalloc(&ent2_j, sizeof(int) * std::max(total, 1LL)));
            HB_CUDA(hb::cmalloc(&ent2_v, sizeof(double) * std::max(total, 1LL)));
            HB_CUDA(cudaMemsetAsync(ent2_j, 0, sizeof(int) * std::max(total, 1LL), s));
            HB_CUDA(cudaMemsetAsync(ent2_v, 0, sizeof(double) * std::max(total, 1LL), s));
            HB_CUDA(hb::cmalloc(&entL_j, sizeof(int) * std::max(totalL, 1LL)));
            HB_CUDA(hb::cmalloc(&entL_v, sizeof(double) * std::max(totalL, 1LL)));
            r1map_fill_kernel<<<hb::counted(pgrid), 256, 0, s>>>(n, d_rptr, d_rj, d_ra, d_sgn, d_cnt, d_slot, d_inv,
                                                                 pos2_ptr, ent2_j, ent2_v, d_lslot, posL_ptr, entL_j,
                                                                 entL_v);
            HB_CUDA(cudaGetLastError());
            HB_CUDA(cudaStreamSynchronize(s));
            hb::cache_free(d_inv);
            for (int *p : {d_rptr, d_rj, d_cnt, d_used, d_slot, d_long, d_lslot}) hb::cache_free(p);
            hb::cache_free(d_llen);
            hb::cache_free(d_ra);
            hb::cache_free(d_sgn);
            hb::cache_free(d_len);
            r1d_gather = true;
        }
    }

    t_upload_map = host_seconds() - tm0;
    HB_CUDA(hb::cmalloc(&T1, sizeof(double) * ld * n));
    HB_CUDA(hb::cmalloc(&T2, sizeof(double) * ld * n));
    HB_CUDA(hb::cmalloc(&vecbuf, sizeof(double) * std::max(m, 1)));
    HB_CUDA(hb::cmalloc(&d_w, sizeof(double) * (std::max(m, nr1d) + 1)));
    HB_CUDA(hb::cmalloc(&d_scal, sizeof(double) * 16));
    HB_CUDA(hb::cmalloc_host(&h_scal, sizeof(double) * 16));
    HB_CUDA(cudaStreamSynchronize(s));
    t_upload_total = host_seconds() - tu0;
}

void SdpDevice::release() {
    auto f = [](void *p) { if (p) hb::cache_free(p); };
    f(Cfull);
    f(sp_id); f(sp_ptr); f(sp_r); f(sp_c); f(sp_v);
    f(r1s_id); f(r1s_ptr); f(r1s_p); f(r1s_a); f(r1s_sign);
    f(r1d_id); f(r1d_sign); f(A1); f(G); f(V); f(Vt); f(Vs);
    for (double *p : dr_mat) f(p);
    dr_mat.clear();
    f(pos_r); f(pos_c); f(pos_ptr); f(ent_j); f(ent_v);
    f(pos2_r); f(pos2_c); f(pos2_cnt); f(pos2_ptr); f(ent2_j); f(ent2_v);
    pos2_r = pos2_c = pos2_cnt = ent2_j = nullptr;
    f(posL_r); f(posL_c); f(posL_ptr); f(entL_j); f(entL_v);
    posL_r = posL_c = entL_j = nullptr;
    posL_ptr = nullptr;
    entL_v = nullptr;
    nposL = 0;
    pos2_ptr = nullptr;
    ent2_v = nullptr;
    npos2 = 0;
    r1d_gather = false;
    f(T1); f(T2); f(vecbuf); f(d_w); f(d_scal); f(colsq);
    colsq = nullptr;
    opA1.release();
    opK.release();
    opKT.release();
    opB.release();
    split_ready = false;
    if (h_scal) hb::cache_free_host(h_scal);
    h_scal = nullptr;
}

void SdpDevice::assemble(double dC, double dA, const double *d_wvec, double dEye, double *S, long ldS) {
    cudaStream_t s = stream;
    s_init_kernel<<<hb::counted(grid1((long) n * n)), 256, 0, s>>>(n, Cfull, ld, dC, dEye, S, ldS);
    if (dA != 0.0) {
        if (npos > 0)
            s_gather_kernel<<<hb::counted(grid1(npos)), 256, 0, s>>>(npos, pos_r, pos_c, pos_ptr, ent_j, ent_v, d_wvec, dA, S, ldS);
        if (nr1d > 0 && r1d_gather) {
            if (npos2 > 0)
                s_gather2_kernel<<<hb::counted(grid1(npos2)), 256, 0, s>>>(npos2, pos2_r, pos2_c, pos2_ptr, pos2_cnt,
                                                                           ent2_j, ent2_v, d_wvec, dA, S, ldS);
            if (nposL > 0)
                s_gather2_long_kernel<<<hb::counted(grid1(32L * nposL)), 256, 0, s>>>(
                    nposL, posL_r, posL_c, posL_ptr, entL_j, entL_v, d_wvec, dA, S, ldS);
        } else if (nr1d > 0) {
            r1d_weights_kernel<<<hb::counted(grid1(nr1d)), 256, 0, s>>>(nr1d, r1d_id, r1d_sign, d_wvec, dA, d_w);
            scale_columns(s, n, nr1d, A1, ld, d_w, V, ld);
            gemm(s, n, n, nr1d, 1.0, V, ld, 0, A1, ld, 1, 1.0, S, ldS, 0);
        }
        for (int i = 0; i < ndr; ++i)
            axpy_mat_devscale_kernel<<<hb::counted(grid1((long) n * n)), 256, 0, s>>>(n, dr_mat[i], ld, d_wvec, dr_id[i], dA, S, ldS);
    }
    HB_CUDA(cudaGetLastError());
}

void SdpDevice::schur_matrix(const double *W, long ldW, double *M, long ldM, const double *Kinv) {
    cudaStream_t s = stream;
    split_ready = false;
    HB_CUDA(cudaMemsetAsync(M, 0, sizeof(double) * ldM * m, s));
    dim3 blk(32, 8);
    // compulsory traffic of a gather pair kernel: the lower triangles of W (read) and of its M block (written)
    const double wbytes = 8.0 * n * (n + 1) / 2;
    if (nsp > 0) {
        dim3 grd((nsp + 31) / 32, (nsp + 7) / 8);
        const bool timed = kstat_on(KF_SCHUR_PAIR);
        if (timed) kstat_begin(KF_SCHUR_PAIR, s, wbytes + 8.0 * nsp * (nsp + 1) / 2);
        schur_spsp_kernel<<<hb::counted(grd), blk, 0, s>>>(nsp, sp_id, sp_ptr, sp_r, sp_c, sp_v, W, ldW, M, ldM);
        if (timed) kstat_end(s);
    }
    if (nr1s > 0) {
        dim3 grd((nr1s + 31) / 32, (nr1s + 7) / 8);
        const bool timed = kstat_on(KF_SCHUR_PAIR);
        if (timed) kstat_begin(KF_SCHUR_PAIR, s, wbytes + 8.0 * nr1s * (nr1s + 1) / 2);
        schur_r1s_kernel<<<hb::counted(grd), blk, 0, s>>>(nr1s, r1s_id, r1s_ptr, r1s_p, r1s_a, r1s_sign, W, ldW, M, ldM);
        if (timed) kstat_end(s);
    }
    if (nr1d > 0) {
        const long ldg = pad_ld(nr1d);
        bool split = false;
        if (precision == 1 && Kinv && opA1.hi) {
            // B = L^-1 A1 (split operand), G = B^T B (lower) in BF16x3 with FP32 accumulation
            split_from_f64(s, opK, Kinv, ld, false);
            split_from_f64(s, opKT, Kinv, ld, true);
            SplitGemm g1;
            g1.M = n;
            g1.N = nr1d;
            g1.K = n;
            g1.a_lower = true;
            g1.epi = SPLIT_EPI_SPLIT;
            g1.out = &opB;
            SplitGemm g2;
            g2.M = g2.N = nr1d;
            g2.K = n;
            g2.lower_tiles = true;
            g2.C = G;
            g2.ldc = ldg;
            split = split_gemm(s, opK, opA1, g1) && split_gemm(s, opB, opB, g2);
            split_ready = split;
        }
        // V = W * A1 (FP64): the whole product when not split, else only for the cross terms
        if (!split || nr1s > 0 || nsp > 0) gemm(s, n, nr1d, n, 1.0, W, ldW, 0, A1, ld, 0, 0.0, V, ld, 0);
        // G = A1^T V (lower),  M = (s s^T) o G o G
        if (!split) gemm(s, nr1d, nr1d, n, 1.0, A1, ld, 1, V, ld, 0, 0.0, G, ldg, GEMM_C_LOWER);
        dim3 grd((nr1d + 31) / 32, (nr1d + 7) / 8);
        schur_hadamard_kernel<<<hb::counted(grd), blk, 0, s>>>(nr1d, r1d_id, r1d_sign, G, ldg, M, ldM);
        if (nr1s > 0) {
            dim3 g2((nr1s + 31) / 32, (nr1d + 7) / 8);
            schur_r1d_r1s_kernel<<<hb::counted(g2), blk, 0, s>>>(nr1d, r1d_id, r1d_sign, V, ld, nr1s, r1s_id, r1s_ptr, r1s_p,
                                                    r1s_a, r1s_sign, M, ldM);
        }
        if (nsp > 0) {
            dim3 g3((nsp + 31) / 32, (nr1d + 7) / 8);
            schur_r1_sp_kernel<<<hb::counted(g3), blk, 0, s>>>(nr1d, r1d_id, r1d_sign, V, ld, nsp, sp_id, sp_ptr, sp_r, sp_c,
                                                  sp_v, M, ldM);
        }
    }
    if (nr1s > 0 && nsp > 0) {
        dim3 gv(grid1(n) > 64 ? 64 : grid1(n), nr1s);
        r1s_build_v_kernel<<<hb::counted(gv), 256, 0, s>>>(n, nr1s, r1s_ptr, r1s_p, r1s_a, W, ldW, Vs, ld);
        dim3 g3((nsp + 31) / 32, (nr1s + 7) / 8);
        schur_r1_sp_kernel<<<hb::counted(g3), blk, 0, s>>>(nr1s, r1s_id, r1s_sign, Vs, ld, nsp, sp_id, sp_ptr, sp_r, sp_c, sp_v,
                                              M, ldM);
    }
    for (int i = 0; i < ndr; ++i) {
        // B_i = W A_i W, then M_ij = <A_j, B_i>
        gemm(s, n, n, n, 1.0, dr_mat[i], ld, 0, W, ldW, 0, 0.0, T1, ld, 0);
        gemm(s, n, n, n, 1.0, W, ldW, 0, T1, ld, 0, 0.0, T2, ld, 0);
        symmetrize_avg(s, n, T2, ld);
        inner_all(T2, ld, vecbuf);
        scatter_row_kernel<<<hb::counted(grid1(m)), 256, 0, s>>>(m, dr_id[i], vecbuf, M, ldM);
    }
    HB_CUDA(cudaGetLastError());
}

bool SdpDevice::split_inverse(const double *Kinv, double *W, long ldW) {
    if (!opKT.hi || opKT.rows != n || opKT.k != n) {
        if (!opKT.alloc(n, n)) return false;
    }
    split_from_f64(stream, opKT, Kinv, ld, true);  // the rows of the operand are the columns of Kinv
    SplitGemm g;
    g.M = g.N = g.K = n;
    g.lower_tiles = true;
    g.a_upper = true;  // column i of Kinv vanishes above row i
    g.C = W;
    g.ldc = ldW;
    if (!split_gemm(stream, opKT, opKT, g)) return false;
    symmetrize_lower(stream, n, W, ldW);
    return true;
}

void SdpDevice::inner_all(const double *Z, long ldZ, double *out, bool reuse_v) {
    cudaStream_t s = stream;
    // rows with a zero coefficient (another cone's constraints) are written by no kernel
    if (nsp + nr1s + nr1d + ndr < m) HB_CUDA(cudaMemsetAsync(out, 0, sizeof(double) * m, s));
    if (nsp > 0) inner_sp_kernel<<<hb::counted(grid1(nsp)), 256, 0, s>>>(nsp, sp_id, sp_ptr, sp_r, sp_c, sp_v, Z, ldZ, out);
    if (nr1s > 0)
        inner_r1s_kernel<<<hb::counted(grid1(nr1s)), 256, 0, s>>>(nr1s, r1s_id, r1s_ptr, r1s_p, r1s_a, r1s_sign, Z, ldZ, out);
    if (nr1d > 0 && reuse_v && split_ready) {
        // <A_i, W> = s_i a_i^T W a_i = s_i G_ii
        r1d_diag_kernel<<<hb::counted(grid1(nr1d)), 256, 0, s>>>(nr1d, r1d_id, r1d_sign, G, pad_ld(nr1d), out);
    } else if (nr1d > 0) {
        if (!reuse_v) gemm(s, n, nr1d, n, 1.0, Z, ldZ, 0, A1, ld, 0, 0.0, Vt, ld, 0);
        const double *Vz = reuse_v ? V : Vt;
        coldot_pair_kernel<<<hb::counted((nr1d * 32 + 255) / 256), 256, 0, s>>>(n, nr1d, r1d_id, r1d_sign, A1, ld, Vz, ld, out);
    }
    for (int i = 0; i < ndr; ++i) frob_dot(s, n, dr_mat[i], ld, Z, ldZ, out + dr_id[i]);
    HB_CUDA(cudaGetLastError());
}

void SdpDevice::inner_all_sq(const double *W, long ldW, double *out, bool reuse_v, bool reuse_vt) {
    cudaStream_t s = stream;
    if (nsp + nr1s + nr1d + ndr < m) HB_CUDA(cudaMemsetAsync(out, 0, sizeof(double) * m, s));
    if (nsp > 0)
        innersq_sp_kernel<<<hb::counted((nsp * 32 + 255) / 256), 256, 0, s>>>(n, nsp, sp_id, sp_ptr, sp_r, sp_c, sp_v, W, ldW, out);
    if (nr1s > 0)
        innersq_r1s_kernel<<<hb::counted((nr1s * 32 + 255) / 256), 256, 0, s>>>(n, nr1s, r1s_id, r1s_ptr, r1s_p, r1s_a, r1s_sign,
                                                                   W, ldW, out);
    if (nr1d > 0 && reuse_v && split_ready) {
        // <A_i, W^2> = s_i |W a_i|^2 = s_i |L^-T b_i|^2: column sums of squares of L^-T B
        HB_CUDA(cudaMemsetAsync(colsq, 0, sizeof(double) * nr1d, s));
        SplitGemm g;
        g.M = n;
        g.N = nr1d;
        g.K = n;
        g.epi = SPLIT_EPI_COLSQ;
        g.colsq = colsq;
        if (split_gemm(s, opKT, opB, g)) {
            r1d_scatter_kernel<<<hb::counted(grid1(nr1d)), 256, 0, s>>>(nr1d, r1d_id, r1d_sign, colsq, out);
        } else {
            gemm(s, n, nr1d, n, 1.0, W, ldW, 0, A1, ld, 0, 0.0, Vt, ld, 0);
            coldot_pair_kernel<<<hb::counted((nr1d * 32 + 255) / 256), 256, 0, s>>>(n, nr1d, r1d_id, r1d_sign, Vt, ld,
                                                                                    Vt, ld, out);
        }
    } else if (nr1d > 0) {
        if (!reuse_v && !reuse_vt) gemm(s, n, nr1d, n, 1.0, W, ldW, 0, A1, ld, 0, 0.0, Vt, ld, 0);
        const double *Vw = reuse_v ? V : Vt;
        coldot_pair_kernel<<<hb::counted((nr1d * 32 + 255) / 256), 256, 0, s>>>(n, nr1d, r1d_id, r1d_sign, Vw, ld, Vw, ld, out);
    }
    for (int i = 0; i < ndr; ++i) {
        gemm(s, n, n, n, 1.0, dr_mat[i], ld, 0, W, ldW, 0, 0.0, T1, ld, 0);
        frob_dot(s, n, T1, ld, W, ldW, out + dr_id[i]);
    }
    HB_CUDA(cudaGetLastError());
}

double SdpDevice::c_inner(const double *Z, long ldZ) {
    frob_dot(stream, n, Cfull, ld, Z, ldZ, d_scal);
    HB_CUDA(cudaMemcpyAsync(h_scal, d_scal, sizeof(double), cudaMemcpyDeviceToHost, stream));
    HB_CUDA(cudaStreamSynchronize(stream));
    return h_scal[0];
}

}  // namespace hb
