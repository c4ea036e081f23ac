// Sparse Cholesky of the dual slack S: multiple-minimum-degree rounds on the device and
// a dense front factored by the cooperative Cholesky (see sparse_chol.h).
#include "sparse_chol.h"
#include "dev.cuh"
#include <algorithm>
#include <iterator>
#include <cmath>
#include <utility>

namespace hb {

namespace {

// slot values <- lower-triangle entries of S
__global__ void hy_gather_kernel(int ns, const int *__restrict__ row, const int *__restrict__ col,
                                 const double *__restrict__ S, long ld, double *__restrict__ wv) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < ns; e += gridDim.x * blockDim.x)
        wv[e] = S[(size_t) row[e] + (size_t) col[e] * ld];
}

// One warp per eliminated vertex j of a round: l_jj = sqrt(s_jj), l_aj = s_aj / l_jj. A
// pivot that is not positive marks S as not positive definite (the factor continues with
// l_jj = 1 so that no NaN spreads).
__global__ void hy_scale_kernel(int e0, int e1, const int *__restrict__ dslot, const int *__restrict__ nptr,
                                const int *__restrict__ nslot, const double *__restrict__ wv,
                                double *__restrict__ lval, double *__restrict__ ldiag, int *__restrict__ info) {
    const int j = e0 + (int) ((blockIdx.x * (size_t) blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (j >= e1) return;
    const double d = wv[dslot[j]];
    double l = 1.0;
    if (d > 0.0) l = sqrt(d);
    else if (lane == 0) atomicExch(info, 1);
    if (lane == 0) ldiag[j] = l;
    const double inv = 1.0 / l;
    for (int k = nptr[j] + lane; k < nptr[j + 1]; k += 32) lval[k] = wv[nslot[k]] * inv;
}

// One thread per target entry of a round: s_ab -= sum over its contributions l_aj l_bj,
// in the order the analysis listed them.
__global__ void hy_update_kernel(int t0, int t1, const int *__restrict__ tslot, const int *__restrict__ cptr,
                                 const int *__restrict__ ca, const int *__restrict__ cb,
                                 const double *__restrict__ lval, double *__restrict__ wv) {
    for (int t = t0 + blockIdx.x * blockDim.x + threadIdx.x; t < t1; t += gridDim.x * blockDim.x) {
        double acc = wv[tslot[t]];
        for (int c = cptr[t]; c < cptr[t + 1]; ++c) acc = fma(-lval[ca[c]], lval[cb[c]], acc);
        wv[tslot[t]] = acc;
    }
}

// Sf = S[front, front], lower triangle (front increasing, so row >= col carries over)
__global__ void hy_front_kernel(int f, const int *__restrict__ front, const double *__restrict__ S, long ld,
                                double *__restrict__ Sf, long ldf) {
    for (int q = blockIdx.y * blockDim.y + threadIdx.y; q < f; q += gridDim.y * blockDim.y) {
        const size_t cq = (size_t) front[q] * ld;
        for (int p = q + blockIdx.x * blockDim.x + threadIdx.x; p < f; p += gridDim.x * blockDim.x)
            Sf[(size_t) p + (size_t) q * ldf] = S[(size_t) front[p] + cq];
    }
}

// front entries the rounds updated
__global__ void hy_fix_kernel(int nfix, const int *__restrict__ fixslot, const long *__restrict__ fixpos,
                              const double *__restrict__ wv, double *__restrict__ Sf) {
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < nfix; x += gridDim.x * blockDim.x)
        Sf[fixpos[x]] = wv[fixslot[x]];
}

// out = sum log l_jj (one block)
__global__ void hy_logsum_kernel(int ne, const double *__restrict__ ldiag, double *__restrict__ out) {
    __shared__ double red[32];
    double acc = 0.0;
    for (int j = threadIdx.x; j < ne; j += blockDim.x) acc += log(ldiag[j]);
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        acc = (threadIdx.x < (blockDim.x >> 5)) ? red[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
        if (threadIdx.x == 0) *out = acc;
    }
}

// Backward substitution through round r (rounds taken last to first):
// u_v = (x_v - sum_a l_av u_a) / l_vv over the entries of column v.
__global__ void hy_bwd_round_kernel(int e0, int e1, const int *__restrict__ elimv, const int *__restrict__ nptr,
                                    const int *__restrict__ nbrv, const double *__restrict__ lval,
                                    const double *__restrict__ ldiag, const double *__restrict__ x,
                                    double *__restrict__ u) {
    for (int j = e0 + blockIdx.x * blockDim.x + threadIdx.x; j < e1; j += gridDim.x * blockDim.x) {
        const int v = elimv[j];
        double acc = x[v];
        for (int k = nptr[j]; k < nptr[j + 1]; ++k) acc = fma(-lval[k], u[nbrv[k]], acc);
        u[v] = acc / ldiag[j];
    }
}

// Forward substitution through round r: y_v = (w_v - sum over row v's entries l_vu y_u) / l_vv.
__global__ void hy_fwd_round_kernel(int e0, int e1, const int *__restrict__ elimv, const int *__restrict__ inptr,
                                    const int *__restrict__ inent, const int *__restrict__ colv,
                                    const double *__restrict__ lval, const double *__restrict__ ldiag,
                                    const double *__restrict__ w, double *__restrict__ y) {
    for (int j = e0 + blockIdx.x * blockDim.x + threadIdx.x; j < e1; j += gridDim.x * blockDim.x) {
        const int v = elimv[j];
        double acc = w[v];
        for (int q = inptr[j]; q < inptr[j + 1]; ++q) {
            const int k = inent[q];
            acc = fma(-lval[k], y[colv[k]], acc);
        }
        y[v] = acc / ldiag[j];
    }
}

// The front's right-hand side after the rounds: z_p = w_F[p] - sum l_F[p],u y_u.
__global__ void hy_fwd_front_kernel(int f, const int *__restrict__ front, const int *__restrict__ finptr,
                                    const int *__restrict__ finent, const int *__restrict__ colv,
                                    const double *__restrict__ lval, const double *__restrict__ w,
                                    const double *__restrict__ y, double *__restrict__ z) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < f; p += gridDim.x * blockDim.x) {
        double acc = w[front[p]];
        for (int q = finptr[p]; q < finptr[p + 1]; ++q) {
            const int k = finent[q];
            acc = fma(-lval[k], y[colv[k]], acc);
        }
        z[p] = acc;
    }
}

__global__ void hy_gather_vec_kernel(int f, const int *__restrict__ front, const double *__restrict__ x,
                                     double *__restrict__ xf) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < f; p += gridDim.x * blockDim.x) xf[p] = x[front[p]];
}

__global__ void hy_scatter_vec_kernel(int f, const int *__restrict__ front, const double *__restrict__ xf,
                                      double *__restrict__ x) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < f; p += gridDim.x * blockDim.x) x[front[p]] = xf[p];
}

template <class T>
void to_device(T **d, const std::vector<T> &h) {
    HB_CUDA(hb::cmalloc(d, sizeof(T) * std::max<size_t>(h.size(), 1)));
    if (!h.empty()) HB_CUDA(cudaMemcpy(*d, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice));
}

int blocks_for(long work, int per) { return (int) std::max<long>(1, std::min<long>((work + per - 1) / per, 148L * 16)); }

}  // namespace

bool HybridFactor::analyse(int n_, const std::vector<std::vector<int>> &adj0, int cap, double maxFrontFrac,
                           bool force) {
    n = n_;
    for (auto *v : {&hSrow, &hScol, &hDslot, &hNptr, &hNslot, &hTslot, &hCptr, &hCa, &hCb, &hFront, &hFixslot,
                    &hNbrV, &hColV, &hElimV, &hInptr, &hInent, &hFinptr, &hFinent})
        v->clear();
    hFixpos.clear();
    // adjacency as sorted vectors; eliminating v turns its neighbours into a clique
    std::vector<std::vector<int>> A(adj0);
    std::vector<char> alive(n, 1), mark(n, 0);
    // slot of the entry (a, b), a >= b: open addressing on the key a * n + b
    std::vector<long long> hkey((size_t) 1 << 16, -1);
    std::vector<int> hval(hkey.size());
    size_t hmask = hkey.size() - 1;
    auto hpos = [&](long long key) {
        size_t h = (size_t) ((unsigned long long) key * 0x9E3779B97F4A7C15ull >> 20) & hmask;
        while (hkey[h] != -1 && hkey[h] != key) h = (h + 1) & hmask;
        return h;
    };
    auto slot = [&](int a, int b) {
        if (a < b) std::swap(a, b);
        const long long key = (long long) a * n + b;
        size_t h = hpos(key);
        if (hkey[h] == key) return hval[h];
        const int s = (int) hSrow.size();
        hSrow.push_back(a);
        hScol.push_back(b);
        hkey[h] = key;
        hval[h] = s;
        if (2 * hSrow.size() > hkey.size()) {  // keep the load below one half
            std::vector<long long> ok;
            std::vector<int> ov;
            ok.swap(hkey);
            ov.swap(hval);
            hkey.assign(ok.size() * 2, -1);
            hval.assign(hkey.size(), 0);
            hmask = hkey.size() - 1;
            for (size_t i = 0; i < ok.size(); ++i)
                if (ok[i] != -1) {
                    const size_t g = hpos(ok[i]);
                    hkey[g] = ok[i];
                    hval[g] = ov[i];
                }
        }
        return s;
    };
    hNptr.push_back(0);
    hCptr.push_back(0);
    roundElim.assign(1, 0);
    roundTgt.assign(1, 0);
    const long maxContrib = 64L << 20;
    std::vector<std::pair<int, int>> order;
    std::vector<int> tmp, N;
    std::vector<int> tgtStamp, tgtLocal;  // per slot: round that made it a target, its index there
    std::vector<int> tgtSlot, tri;        // tri: (local target, entry a, entry b) per contribution
    while (true) {
        order.clear();
        for (int v = 0; v < n; ++v)
            if (alive[v]) order.push_back({(int) A[v].size(), v});
        if (order.empty()) break;
        std::sort(order.begin(), order.end());
        const int mind = order[0].first;
        if (mind > cap) break;
        const int thr = std::min(cap, mind + std::max(1, mind / 4));
        std::fill(mark.begin(), mark.end(), 0);
        std::vector<int> picked;
        for (const auto &p : order) {
            if (p.first > thr) break;
            const int v = p.second;
            if (mark[v]) continue;
            picked.push_back(v);
            mark[v] = 1;
            for (int u : A[v]) mark[u] = 1;
        }
        // the round's columns and Schur updates; the picked set is independent, so one
        // column's elimination does not change another's neighbours
        const int round = (int) roundElim.size();
        tgtSlot.clear();
        tri.clear();
        for (int v : picked) {
            N = A[v];  // sorted
            hDslot.push_back(slot(v, v));
            hElimV.push_back(v);
            const int base = (int) hNslot.size();
            for (int a : N) {
                hNslot.push_back(slot(a, v));
                hNbrV.push_back(a);
                hColV.push_back(v);
            }
            hNptr.push_back((int) hNslot.size());
            for (size_t p = 0; p < N.size(); ++p)
                for (size_t q = 0; q <= p; ++q) {
                    const int sl = slot(N[p], N[q]);
                    if ((size_t) sl >= tgtStamp.size()) {
                        tgtStamp.resize(2 * (size_t) sl + 16, 0);
                        tgtLocal.resize(tgtStamp.size(), 0);
                    }
                    if (tgtStamp[sl] != round) {
                        tgtStamp[sl] = round;
                        tgtLocal[sl] = (int) tgtSlot.size();
                        tgtSlot.push_back(sl);
                    }
                    const int t = tgtLocal[sl];
                    tri.push_back(t);
                    tri.push_back(base + (int) p);
                    tri.push_back(base + (int) q);
                }
            for (int u : N) {
                tmp.clear();
                std::set_union(A[u].begin(), A[u].end(), N.begin(), N.end(), std::back_inserter(tmp));
                tmp.erase(std::remove_if(tmp.begin(), tmp.end(), [&](int w) { return w == u || w == v; }),
                          tmp.end());
                A[u].swap(tmp);
            }
            std::vector<int>().swap(A[v]);
            alive[v] = 0;
        }
        // contributions grouped by target (counting sort, insertion order kept)
        const int nt = (int) tgtSlot.size();
        std::vector<int> cnt(nt + 1, 0);
        for (size_t c = 0; c < tri.size(); c += 3) cnt[tri[c] + 1] += 1;
        for (int t = 0; t < nt; ++t) cnt[t + 1] += cnt[t];
        const size_t c0 = hCa.size();
        hCa.resize(c0 + tri.size() / 3);
        hCb.resize(c0 + tri.size() / 3);
        std::vector<int> cur(cnt.begin(), cnt.end() - 1);
        for (size_t c = 0; c < tri.size(); c += 3) {
            const int at = cur[tri[c]]++;
            hCa[c0 + at] = tri[c + 1];
            hCb[c0 + at] = tri[c + 2];
        }
        for (int t = 0; t < nt; ++t) {
            hTslot.push_back(tgtSlot[t]);
            hCptr.push_back((int) (c0 + cnt[t + 1]));
        }
        roundElim.push_back(roundElim.back() + (int) picked.size());
        roundTgt.push_back((int) hTslot.size());
        if ((long) hCa.size() > maxContrib) return false;
    }
    nrounds = (int) roundElim.size() - 1;
    nelim = roundElim.back();
    for (int v = 0; v < n; ++v)
        if (alive[v]) hFront.push_back(v);
    nfront = (int) hFront.size();
    if (!force && (nrounds == 0 || nfront > maxFrontFrac * n)) return false;
    ldf = pad_ld(std::max(nfront, 1));
    std::vector<int> fidx(n, -1);
    for (int p = 0; p < nfront; ++p) fidx[hFront[p]] = p;
    for (int s = 0; s < (int) hSrow.size(); ++s) {
        const int p = fidx[hSrow[s]], q = fidx[hScol[s]];
        if (p >= 0 && q >= 0) {
            hFixslot.push_back(s);
            hFixpos.push_back((long) p + (long) q * ldf);
        }
    }
    // row structure of L: the entries of each eliminated row and of each front row, in
    // entry order
    std::vector<int> elimIdx(n, -1);
    for (int j = 0; j < (int) hElimV.size(); ++j) elimIdx[hElimV[j]] = j;
    std::vector<int> cntE(hElimV.size() + 1, 0), cntF(nfront + 1, 0);
    for (size_t k = 0; k < hNbrV.size(); ++k) {
        const int a = hNbrV[k];
        if (elimIdx[a] >= 0) cntE[elimIdx[a] + 1] += 1;
        else cntF[fidx[a] + 1] += 1;
    }
    for (size_t j = 0; j < hElimV.size(); ++j) cntE[j + 1] += cntE[j];
    for (int p = 0; p < nfront; ++p) cntF[p + 1] += cntF[p];
    hInptr = cntE;
    hFinptr = cntF;
    hInent.assign(cntE.back(), 0);
    hFinent.assign(cntF.back(), 0);
    for (size_t k = 0; k < hNbrV.size(); ++k) {
        const int a = hNbrV[k];
        if (elimIdx[a] >= 0) hInent[cntE[elimIdx[a]]++] = (int) k;
        else hFinent[cntF[fidx[a]]++] = (int) k;
    }
    nslot = (int) hSrow.size();
    nnbr = (long) hNslot.size();
    ncontrib = (long) hCa.size();
    nfix = (int) hFixslot.size();
    return true;
}

void HybridFactor::upload(cudaStream_t s) {
    (void) s;
    to_device(&d_srow, hSrow);
    to_device(&d_scol, hScol);
    to_device(&d_dslot, hDslot);
    to_device(&d_nptr, hNptr);
    to_device(&d_nslot, hNslot);
    to_device(&d_tslot, hTslot);
    to_device(&d_cptr, hCptr);
    to_device(&d_ca, hCa);
    to_device(&d_cb, hCb);
    to_device(&d_front, hFront);
    to_device(&d_fixslot, hFixslot);
    to_device(&d_fixpos, hFixpos);
    to_device(&d_nbrv, hNbrV);
    to_device(&d_colv, hColV);
    to_device(&d_elimv, hElimV);
    to_device(&d_inptr, hInptr);
    to_device(&d_inent, hInent);
    to_device(&d_finptr, hFinptr);
    to_device(&d_finent, hFinent);
    for (auto *v : {&hSrow, &hScol, &hDslot, &hNptr, &hNslot, &hTslot, &hCptr, &hCa, &hCb, &hFront, &hFixslot,
                    &hNbrV, &hColV, &hElimV, &hInptr, &hInent, &hFinptr, &hFinent})
        std::vector<int>().swap(*v);
    std::vector<long>().swap(hFixpos);
    HB_CUDA(hb::cmalloc(&wv, sizeof(double) * std::max(nslot, 1)));
    HB_CUDA(hb::cmalloc(&lval, sizeof(double) * std::max<long>(nnbr, 1)));
    HB_CUDA(hb::cmalloc(&ldiag, sizeof(double) * std::max(nelim, 1)));
    if (nfront > 0) {
        HB_CUDA(hb::cmalloc(&Sf, sizeof(double) * ldf * nfront));
        HB_CUDA(cudaMemset(Sf, 0, sizeof(double) * ldf * nfront));
        Ff.alloc(nfront, 0);
        HB_CUDA(hb::cmalloc(&fa, sizeof(double) * nfront));
        HB_CUDA(hb::cmalloc(&fb, sizeof(double) * nfront));
    }
    HB_CUDA(hb::cmalloc(&d_info, sizeof(int)));
    HB_CUDA(hb::cmalloc_host(&h_info, sizeof(int)));
    HB_CUDA(hb::cmalloc(&d_logdet, sizeof(double) * 2));
    HB_CUDA(hb::cmalloc_host(&h_logdet, sizeof(double) * 2));
    legacy_fence();
}

void HybridFactor::factor_async(cudaStream_t s, const double *S, long ld) {
    ++seq;
    HB_CUDA(cudaMemsetAsync(d_info, 0, sizeof(int), s));
    HB_CUDA(cudaMemsetAsync(d_logdet, 0, sizeof(double) * 2, s));
    hy_gather_kernel<<<hb::counted(blocks_for(nslot, 256)), 256, 0, s>>>(nslot, d_srow, d_scol, S, ld, wv);
    for (int r = 0; r < nrounds; ++r) {
        const int e0 = roundElim[r], e1 = roundElim[r + 1];
        if (e1 > e0)
            hy_scale_kernel<<<hb::counted((int) ((32L * (e1 - e0) + 255) / 256)), 256, 0, s>>>(
                e0, e1, d_dslot, d_nptr, d_nslot, wv, lval, ldiag, d_info);
        const int t0 = roundTgt[r], t1 = roundTgt[r + 1];
        if (t1 > t0)
            hy_update_kernel<<<hb::counted(blocks_for(t1 - t0, 256)), 256, 0, s>>>(t0, t1, d_tslot, d_cptr, d_ca, d_cb,
                                                                                  lval, wv);
    }
    if (nelim > 0) hy_logsum_kernel<<<hb::counted(1), 1024, 0, s>>>(nelim, ldiag, d_logdet);
    if (nfront > 0) {
        dim3 blk(32, 8), grd((unsigned) std::min((nfront + 31) / 32, 64), (unsigned) std::min((nfront + 7) / 8, 1024));
        hy_front_kernel<<<hb::counted(grd), blk, 0, s>>>(nfront, d_front, S, ld, Sf, ldf);
        if (nfix > 0)
            hy_fix_kernel<<<hb::counted(blocks_for(nfix, 256)), 256, 0, s>>>(nfix, d_fixslot, d_fixpos, wv, Sf);
        factorize_async(s, Ff, Sf, ldf);
        log_diag_sum(s, Ff, d_logdet + 1);
    }
    HB_CUDA(cudaMemcpyAsync(h_logdet, d_logdet, sizeof(double) * 2, cudaMemcpyDeviceToHost, s));
    HB_CUDA(cudaMemcpyAsync(h_info, d_info, sizeof(int), cudaMemcpyDeviceToHost, s));
    HB_CUDA(cudaGetLastError());
}

bool HybridFactor::finish(cudaStream_t s, double *logdet) {
    bool ok = true;
    if (nfront > 0) ok = factor_status(s, Ff);  // synchronises the stream
    else HB_CUDA(cudaStreamSynchronize(s));
    ok = ok && (*h_info == 0);
    if (logdet) *logdet = 2.0 * (h_logdet[0] + (nfront > 0 ? h_logdet[1] : 0.0));
    return ok;
}

void HybridFactor::apply_congruence(cudaStream_t s, const double *D, long ldD, double alpha, const double *x,
                                    double *t, double *u, double *y) {
    const int fb1 = blocks_for(nfront, 256);
    // t = L^-T x: the front first (its block of L^-T is Kf^T), then the rounds last to first
    if (nfront > 0) {
        hy_gather_vec_kernel<<<hb::counted(fb1), 256, 0, s>>>(nfront, d_front, x, fa);
        coldot(s, nfront, nfront, Ff.K, Ff.ld, fa, fb, 1.0, 0.0, 1);
        hy_scatter_vec_kernel<<<hb::counted(fb1), 256, 0, s>>>(nfront, d_front, fb, t);
    }
    for (int r = nrounds - 1; r >= 0; --r) {
        const int e0 = roundElim[r], e1 = roundElim[r + 1];
        if (e1 > e0)
            hy_bwd_round_kernel<<<hb::counted(blocks_for(e1 - e0, 128)), 128, 0, s>>>(e0, e1, d_elimv, d_nptr, d_nbrv,
                                                                                    lval, ldiag, x, t);
    }
    // u = alpha D t
    coldot(s, n, n, D, ldD, t, u, alpha, 0.0, 0);
    // y = L^-1 u: the rounds first to last, then the front (its block of L^-1 is Kf)
    for (int r = 0; r < nrounds; ++r) {
        const int e0 = roundElim[r], e1 = roundElim[r + 1];
        if (e1 > e0)
            hy_fwd_round_kernel<<<hb::counted(blocks_for(e1 - e0, 128)), 128, 0, s>>>(e0, e1, d_elimv, d_inptr, d_inent,
                                                                                    d_colv, lval, ldiag, u, y);
    }
    if (nfront > 0) {
        hy_fwd_front_kernel<<<hb::counted(fb1), 256, 0, s>>>(nfront, d_front, d_finptr, d_finent, d_colv, lval, u, y, fa);
        coldot(s, nfront, nfront, Ff.KT, Ff.ld, fa, fb, 1.0, 0.0, 2);
        hy_scatter_vec_kernel<<<hb::counted(fb1), 256, 0, s>>>(nfront, d_front, fb, y);
    }
    HB_CUDA(cudaGetLastError());
}

void HybridFactor::release() {
    auto f = [](void *p) {
        if (p) hb::cache_free(p);
    };
    f(d_srow); f(d_scol); f(d_dslot); f(d_nptr); f(d_nslot); f(d_tslot); f(d_cptr); f(d_ca); f(d_cb);
    f(d_front); f(d_fixslot); f(d_fixpos); f(wv); f(lval); f(ldiag); f(Sf); f(d_info); f(d_logdet);
    f(d_nbrv); f(d_colv); f(d_elimv); f(d_inptr); f(d_inent); f(d_finptr); f(d_finent); f(fa); f(fb);
    d_nbrv = d_colv = d_elimv = d_inptr = d_inent = d_finptr = d_finent = nullptr;
    fa = fb = nullptr;
    if (h_info) hb::cache_free_host(h_info);
    if (h_logdet) hb::cache_free_host(h_logdet);
    d_srow = d_scol = d_dslot = d_nptr = d_nslot = d_tslot = d_cptr = d_ca = d_cb = d_front = d_fixslot = nullptr;
    d_fixpos = nullptr;
    wv = lval = ldiag = Sf = d_logdet = h_logdet = nullptr;
    d_info = h_info = nullptr;
    Ff.release();
}

}  // namespace hb
