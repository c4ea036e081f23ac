// Extension entry points of the B200 HDSDP library (include/hdsdp_b200.h).
#include "solver.h"
#include "split.h"
#include "../../include/hdsdp_b200.h"
#include <algorithm>
#include <cstring>
#include <cmath>
#include <vector>
#include <cooperative_groups.h>

using namespace hb;

extern "C" {

int HDSDPGetStatus(hdsdp *h) { return (int) h->HStatus; }
int HDSDPGetIterCount(hdsdp *h) { return h->nIterCount; }
void HDSDPSetPrimalRefinement(hdsdp *h, int on) { h->HIntParams[INT_PARAM_PSDP] = on ? 1 : 0; }
void HDSDPSetPrecision(hdsdp *h, int mode) { h->precision = mode; }
void HDSDPSetSparseSlack(hdsdp *h, int mode) { h->sparseSlack = mode; }
void HDSDPSetSparseSchur(hdsdp *h, int mode) { h->sparseSchur = mode; }
void HDSDPGetSparseSchurInfo(hdsdp *h, double out[6]) { h->kkt.arrow_info(out); }
void HDSDPSetSchurLDL(hdsdp *h, int mode) { h->schurLdl = (mode == 1) ? 1 : 0; }

// Host only (no device work): the ordering of the sparse factorisation of S for the
// pattern of nedge off-diagonal pairs (ei[k], ej[k]) with degree cap `cap`.
// out = {rounds, front order, eliminated vertices, slots, Schur contributions}; front
// (length n, may be null) receives the front's vertices in increasing order.
int hdsdpb_sparse_analyse(int n, int nedge, const int *ei, const int *ej, int cap, double out[5], int *front) {
    if (n <= 0 || nedge < 0 || !out) return -1;
    std::vector<std::vector<int>> adj(n);
    for (int k = 0; k < nedge; ++k) {
        if (ei[k] < 0 || ei[k] >= n || ej[k] < 0 || ej[k] >= n) return -1;
        if (ei[k] == ej[k]) continue;
        adj[ei[k]].push_back(ej[k]);
        adj[ej[k]].push_back(ei[k]);
    }
    for (auto &l : adj) {
        std::sort(l.begin(), l.end());
        l.erase(std::unique(l.begin(), l.end()), l.end());
    }
    hb::HybridFactor f;
    if (!f.analyse(n, adj, cap, 1.0, true)) return -1;
    out[0] = f.nrounds;
    out[1] = f.nfront;
    out[2] = f.nelim;
    out[3] = f.nslot;
    out[4] = (double) f.ncontrib;
    if (front)
        for (int p = 0; p < f.nfront; ++p) front[p] = f.hFront[p];
    return 0;
}

void HDSDPGetSparseSlackInfo(hdsdp *h, double out[8]) {
    for (int i = 0; i < 8; ++i) out[i] = 0.0;
    for (const hb::ConeSlot &k : h->cones) {
        if (!k.sdp || !k.sdp->hy) continue;
        if (out[0] == 0.0) {
            out[1] = k.sdp->hy->nfront;
            out[2] = k.sdp->hy->nrounds;
            out[4] = k.sdp->hy->nelim;
        }
        out[0] += 1.0;
        out[3] += (double) k.sdp->nHybrid;
        out[5] += (double) k.sdp->nHybridCheck;
        out[6] += (double) k.sdp->nDenseAfter[0];
        out[7] += (double) k.sdp->nDenseAfter[1];
    }
}

int HDSDPGetIterLog(hdsdp *h, int maxLen, double *t, double *pObj, double *dObj, double *mu, double *gap,
                    int *phase) {
    const int n = (int) h->log.size();
    for (int i = 0; i < n && i < maxLen; ++i) {
        const IterRecord &r = h->log[i];
        if (t) t[i] = r.t;
        if (pObj) pObj[i] = r.pobj;
        if (dObj) dObj[i] = r.dobj;
        if (mu) mu[i] = r.mu;
        if (gap) gap[i] = r.gap;
        if (phase) phase[i] = r.phase;
    }
    return n;
}

void HDSDPGetTimers(hdsdp *h, double out[23]) {
    const Timers &t = h->timers;
    long reuse = 0;
    for (const hb::ConeSlot &k : h->cones)
        if (k.sdp) reuse += k.sdp->nFactorReuse;
    const double v[23] = {t.schur, t.schur_factor, t.schur_solve, t.s_factor, t.s_inverse, t.lanczos, t.assemble,
                          t.primal, t.total, (double) t.n_schur, (double) t.n_sfactor, (double) t.n_lanczos,
                          (double) t.n_lanczos_mv, (double) t.n_schur_solve, t.lz_inverse, t.lz_host, t.lz_wait,
                          t.sch_matrix, t.sch_inner, t.sch_innersq, t.setup, t.ipm_device,
                          (double) reuse};
    std::memcpy(out, v, sizeof(v));
}

long long hdsdpb_launch_count(void) { return hb::launch_counter(); }

long long hdsdpb_alloc_calls(void) { return hb::alloc_counter(); }

void hdsdpb_release_cached_memory(void) {
    cudaDeviceSynchronize();
    hb::cache_release();
}

int hdsdpb_kstat_enable(int mask) {
    hb::kstat_enable(mask);
    return 0;
}

int hdsdpb_kstat_read(int family, long long *launches, double *ms, double *work) {
    return hb::kstat_read(family, launches, ms, work);
}

static int probe_setup(SdpCone &c, cudaStream_t s, int m, int n, const int *Ap, const int *Ai, const double *Ax,
                       int precision) {
    if (c.proc_data(m, n, Ap, Ai, Ax) != HDSDP_RETCODE_OK) return -1;
    if (c.presolve() != HDSDP_RETCODE_OK) return -1;
    c.precision = precision;
    if (c.setup_device(s, nullptr) != HDSDP_RETCODE_OK) return -1;
    return 0;
}

int hdsdpb_schur_probe(int m, int n, const int *Ap, const int *Ai, const double *Ax, const double *y, double resi,
                       int precision, double *M, double *asinv, double *asinvrd, double *traceSinv) {
    cudaStream_t s;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return -1;
    SdpCone c;
    KKT k;
    int ret = probe_setup(c, s, m, n, Ap, Ai, Ax, precision);
    if (ret == 0) {
        c.set_start(resi);
        int interior = 0;
        c.interior_check(1.0, y, &interior);
        if (!interior) ret = 1;
    }
    if (ret == 0) {
        k.init(m, s, nullptr);
        if (k.build(c, KKT_TYPE_INFEASIBLE) != HDSDP_RETCODE_OK) ret = -1;
        if (ret == 0) {
            if (M) {
                std::vector<double> h((size_t) k.ldm * m);
                cudaMemcpy(h.data(), k.M, sizeof(double) * k.ldm * m, cudaMemcpyDeviceToHost);
                for (int j = 0; j < m; ++j)
                    for (int i = 0; i < m; ++i) M[(size_t) j * m + i] = (i >= j) ? h[(size_t) j * k.ldm + i] : 0.0;
            }
            std::memcpy(asinv, k.asinv.data(), sizeof(double) * m);
            std::memcpy(asinvrd, k.asinvrd.data(), sizeof(double) * m);
            if (traceSinv) *traceSinv = k.dTraceSinv;
        }
        k.release();
    }
    c.release();
    cudaStreamDestroy(s);
    return device_error_flag() ? -1 : ret;
}

int hdsdpb_ratio_probe(int m, int n, const int *Ap, const int *Ai, const double *Ax, const double *y, double resi,
                       const double *dy, double ada, double *step, double *logdet) {
    cudaStream_t s;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return -1;
    SdpCone c;
    int ret = probe_setup(c, s, m, n, Ap, Ai, Ax, 0);
    if (ret == 0) {
        c.set_start(resi);
        int interior = 0;
        c.interior_check(1.0, y, &interior);
        if (!interior) ret = 1;
    }
    if (ret == 0) {
        if (c.get_barrier(0.0, nullptr, BUFFER_DUALVAR, logdet) != HDSDP_RETCODE_OK) ret = -1;
        if (ret == 0 && c.ratio_test(0.0, dy, ada, BUFFER_DUALVAR, step) != HDSDP_RETCODE_OK) ret = -1;
    }
    c.release();
    cudaStreamDestroy(s);
    return device_error_flag() ? -1 : ret;
}

int hdsdpb_cholesky(int n, const double *S, double *L, double *logdiag) {
    if (n < 0 || (n > 0 && !S)) return -1;
    if (n == 0) {
        if (logdiag) *logdiag = 0.0;
        return 0;
    }
    cudaStream_t s;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return -1;
    const long ld = pad_ld(n);
    double *dS = nullptr, *dl = nullptr;
    hb::cmalloc(&dS, sizeof(double) * ld * n);
    hb::cmalloc(&dl, sizeof(double));
    cudaMemcpy2D(dS, sizeof(double) * ld, S, sizeof(double) * n, sizeof(double) * n, n, cudaMemcpyHostToDevice);
    legacy_fence();
    DenseFactor F;
    F.alloc(n);
    const bool ok = factorize(s, F, dS, ld);
    if (ok) {
        log_diag_sum(s, F, dl);
        if (logdiag) cudaMemcpyAsync(logdiag, dl, sizeof(double), cudaMemcpyDeviceToHost, s);
        if (L) {
            std::vector<double> h((size_t) ld * n);
            cudaMemcpyAsync(h.data(), F.L, sizeof(double) * ld * n, cudaMemcpyDeviceToHost, s);
            cudaStreamSynchronize(s);
            for (int j = 0; j < n; ++j)
                for (int i = 0; i < n; ++i) L[(size_t) j * n + i] = (i >= j) ? h[(size_t) j * ld + i] : 0.0;
        }
    }
    cudaStreamSynchronize(s);
    F.release();
    hb::cache_free(dS);
    hb::cache_free(dl);
    cudaStreamDestroy(s);
    if (device_error_flag()) return -1;
    return ok ? 0 : 1;
}

// count factorisations of order n (S: count column-major n x n matrices, host), either one
// CTA per matrix in shared launches (mode 0, factorize_small_batch) or each on the whole
// GPU (mode 1, the cooperative kernel). Out (each may be null): L and K = L^-1 (lower,
// count x n x n), logdiag = sum log L_ii, status (0 positive definite, 1 not).
int hdsdpb_cholesky_batch(int count, int n, int mode, const double *S, double *L, double *K, double *logdiag,
                          int *status) {
    if (count < 0 || n <= 0 || n > kSmallFactorMaxN || !S || (mode != 0 && mode != 1)) return -1;
    if (count == 0) return 0;
    cudaStream_t s;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return -1;
    const long ld = pad_ld(n);
    std::vector<DenseFactor> F(count);
    std::vector<DenseFactor *> Fp(count);
    std::vector<const double *> Sp(count);
    std::vector<long> lds(count, ld);
    double *dS = nullptr;
    hb::cmalloc(&dS, sizeof(double) * ld * n * count);
    for (int q = 0; q < count; ++q) {
        cudaMemcpy2D(dS + (size_t) q * ld * n, sizeof(double) * ld, S + (size_t) q * n * n, sizeof(double) * n,
                     sizeof(double) * n, n, cudaMemcpyHostToDevice);
        F[q].alloc(n, 1);
        Fp[q] = &F[q];
        Sp[q] = dS + (size_t) q * ld * n;
    }
    legacy_fence();
    if (mode == 0) {
        factorize_small_batch(s, Fp.data(), Sp.data(), lds.data(), count);
    } else {
        for (int q = 0; q < count; ++q) factorize_async(s, F[q], Sp[q], ld);
    }
    HB_CUDA(cudaStreamSynchronize(s));
    std::vector<double> h((size_t) ld * n);
    for (int q = 0; q < count; ++q) {
        const bool ok = factor_status_ready(F[q]);
        if (status) status[q] = ok ? 0 : 1;
        if (logdiag) logdiag[q] = ok ? 0.5 * F[q].logdet : 0.0;
        for (int which = 0; which < 2; ++which) {
            double *out = which ? K : L;
            if (!out) continue;
            cudaMemcpy(h.data(), which ? F[q].K : F[q].L, sizeof(double) * ld * n, cudaMemcpyDeviceToHost);
            double *o = out + (size_t) q * n * n;
            for (int j = 0; j < n; ++j)
                for (int i = 0; i < n; ++i) o[(size_t) j * n + i] = (ok && i >= j) ? h[(size_t) j * ld + i] : 0.0;
        }
        F[q].release();
    }
    hb::cache_free(dS);
    cudaStreamDestroy(s);
    return device_error_flag() ? -1 : 0;
}

// The sparse factorisation of S (column-major n x n, host; its pattern given by the
// nedge off-diagonal pairs) with degree cap `cap`, timed over `reps` calls after one
// warm-up call, and the dense cooperative factorisation of the same S timed the same
// way. out = {positive definite (1/0), log det, ms per sparse factorisation, ms per
// dense factorisation, dense-front order}. Returns 0, or -1 on invalid input.
int hdsdpb_sparse_cholesky(int n, int nedge, const int *ei, const int *ej, const double *S, int cap, int reps,
                           double out[5]) {
    if (n <= 0 || nedge < 0 || !S || !out || reps < 1) return -1;
    std::vector<std::vector<int>> adj(n);
    for (int k = 0; k < nedge; ++k) {
        if (ei[k] < 0 || ei[k] >= n || ej[k] < 0 || ej[k] >= n) return -1;
        if (ei[k] == ej[k]) continue;
        adj[ei[k]].push_back(ej[k]);
        adj[ej[k]].push_back(ei[k]);
    }
    for (auto &l : adj) {
        std::sort(l.begin(), l.end());
        l.erase(std::unique(l.begin(), l.end()), l.end());
    }
    hb::HybridFactor f;
    if (!f.analyse(n, adj, cap, 1.0, true)) return -1;
    cudaStream_t s;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return -1;
    f.upload(s);
    const long ld = pad_ld(n);
    double *dS = nullptr;
    hb::cmalloc(&dS, sizeof(double) * ld * n);
    cudaMemcpy2D(dS, sizeof(double) * ld, S, sizeof(double) * n, sizeof(double) * n, n, cudaMemcpyHostToDevice);
    legacy_fence();
    double logdet = 0.0;
    f.factor_async(s, dS, ld);
    bool ok = f.finish(s, &logdet);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, s);
    for (int r = 0; r < reps; ++r) {
        f.factor_async(s, dS, ld);
        ok = f.finish(s, &logdet) && ok;
    }
    cudaEventRecord(e1, s);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    out[0] = ok ? 1.0 : 0.0;
    out[1] = logdet;
    out[2] = ms / reps;
    out[4] = f.nfront;
    DenseFactor F;
    F.alloc(n, 0);
    factorize(s, F, dS, ld);
    cudaEventRecord(e0, s);
    for (int r = 0; r < reps; ++r) factorize(s, F, dS, ld);
    cudaEventRecord(e1, s);
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(&ms, e0, e1);
    out[3] = ms / reps;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    F.release();
    f.release();
    hb::cache_free(dS);
    cudaStreamDestroy(s);
    return device_error_flag() ? -1 : 0;
}

// With the sparse factor S = L L^T (pattern as above, cap 64): t = L^-T x and
// y = L^-1 (D t) for host n x n D and n-vector x. Returns 0, 1 if S is not positive
// definite, -1 on invalid input.
int hdsdpb_sparse_congruence(int n, int nedge, const int *ei, const int *ej, const double *S, const double *D,
                             const double *x, double *y, double *t) {
    if (n <= 0 || nedge < 0 || !S || !D || !x || !y) return -1;
    std::vector<std::vector<int>> adj(n);
    for (int k = 0; k < nedge; ++k) {
        if (ei[k] < 0 || ei[k] >= n || ej[k] < 0 || ej[k] >= n) return -1;
        if (ei[k] == ej[k]) continue;
        adj[ei[k]].push_back(ej[k]);
        adj[ej[k]].push_back(ei[k]);
    }
    for (auto &l : adj) {
        std::sort(l.begin(), l.end());
        l.erase(std::unique(l.begin(), l.end()), l.end());
    }
    hb::HybridFactor f;
    if (!f.analyse(n, adj, 64, 1.0, true)) return -1;
    cudaStream_t s;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return -1;
    f.upload(s);
    const long ld = pad_ld(n);
    double *dS = nullptr, *dD = nullptr, *dv = nullptr;
    hb::cmalloc(&dS, sizeof(double) * ld * n);
    hb::cmalloc(&dD, sizeof(double) * ld * n);
    hb::cmalloc(&dv, sizeof(double) * 4 * ld);
    cudaMemcpy2D(dS, sizeof(double) * ld, S, sizeof(double) * n, sizeof(double) * n, n, cudaMemcpyHostToDevice);
    cudaMemcpy2D(dD, sizeof(double) * ld, D, sizeof(double) * n, sizeof(double) * n, n, cudaMemcpyHostToDevice);
    cudaMemcpy(dv, x, sizeof(double) * n, cudaMemcpyHostToDevice);
    legacy_fence();
    f.factor_async(s, dS, ld);
    const bool ok = f.finish(s, nullptr);
    if (ok) {
        if (f.nfront > 0) compute_inverse_factor(s, f.Ff);
        f.apply_congruence(s, dD, ld, 1.0, dv, dv + ld, dv + 2 * ld, dv + 3 * ld);
        cudaMemcpyAsync(y, dv + 3 * ld, sizeof(double) * n, cudaMemcpyDeviceToHost, s);
        if (t) cudaMemcpyAsync(t, dv + ld, sizeof(double) * n, cudaMemcpyDeviceToHost, s);
    }
    cudaStreamSynchronize(s);
    f.release();
    hb::cache_free(dS);
    hb::cache_free(dD);
    hb::cache_free(dv);
    cudaStreamDestroy(s);
    if (device_error_flag()) return -1;
    return ok ? 0 : 1;
}

int hdsdpb_ldl_solve(int n, const double *S, const double *b, double *x, int out[3]) {
    if (n < 0 || (n > 0 && (!S || !b || !x))) return -1;
    if (out) out[0] = out[1] = out[2] = 0;
    if (n == 0) return 0;
    cudaStream_t s;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return -1;
    const long ld = pad_ld(n);
    double *dS = nullptr, *dx = nullptr;
    hb::cmalloc(&dS, sizeof(double) * ld * n);
    hb::cmalloc(&dx, sizeof(double) * n);
    cudaMemcpy2D(dS, sizeof(double) * ld, S, sizeof(double) * n, sizeof(double) * n, n, cudaMemcpyHostToDevice);
    cudaMemcpy(dx, b, sizeof(double) * n, cudaMemcpyHostToDevice);
    legacy_fence();
    LdlFactor F;
    const bool ok = ldl_factorize(s, F, dS, ld, n);
    int ret = ok ? 0 : (F.h_info ? reinterpret_cast<int *>(F.h_info)[0] : -1);
    if (!ok && ret <= 0) ret = -1;
    if (ok) {
        ldl_solve(s, F, dx, dx);
        cudaMemcpyAsync(x, dx, sizeof(double) * n, cudaMemcpyDeviceToHost, s);
        if (out) {
            // the inertia of S from the blocks of D
            std::vector<int> piv(n);
            std::vector<double> dg(n), sub(n, 0.0);
            cudaMemcpyAsync(piv.data(), F.piv, sizeof(int) * n, cudaMemcpyDeviceToHost, s);
            cudaMemcpy2DAsync(dg.data(), sizeof(double), F.A, sizeof(double) * (F.ld + 1), sizeof(double), n,
                              cudaMemcpyDeviceToHost, s);
            if (n > 1)
                cudaMemcpy2DAsync(sub.data(), sizeof(double), F.A + 1, sizeof(double) * (F.ld + 1), sizeof(double),
                                  n - 1, cudaMemcpyDeviceToHost, s);
            cudaStreamSynchronize(s);
            for (int i = 0; i < n; ++i) {
                if (piv[i] == 1) {
                    (dg[i] < 0.0 ? out[1] : out[2]) += 1;
                } else if (piv[i] == 2 && i + 1 < n) {
                    out[0] += 1;
                    const double det = dg[i] * dg[i + 1] - sub[i] * sub[i];
                    if (det < 0.0) {
                        out[1] += 1;
                        out[2] += 1;
                    } else {
                        (dg[i] + dg[i + 1] < 0.0 ? out[1] : out[2]) += 2;
                    }
                }
            }
        }
    }
    cudaStreamSynchronize(s);
    F.release();
    hb::cache_free(dS);
    hb::cache_free(dx);
    cudaStreamDestroy(s);
    if (device_error_flag()) return -1;
    return ret;
}

int hdsdpb_cholesky_solve(int n, const double *S, const double *b, double *x) {
    if (n < 0 || (n > 0 && (!S || !b || !x))) return -1;
    if (n == 0) return 0;
    cudaStream_t s;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return -1;
    const long ld = pad_ld(n);
    double *dS = nullptr, *dx = nullptr;
    hb::cmalloc(&dS, sizeof(double) * ld * n);
    hb::cmalloc(&dx, sizeof(double) * n);
    cudaMemcpy2D(dS, sizeof(double) * ld, S, sizeof(double) * n, sizeof(double) * n, n, cudaMemcpyHostToDevice);
    cudaMemcpy(dx, b, sizeof(double) * n, cudaMemcpyHostToDevice);
    legacy_fence();
    DenseFactor F;
    F.alloc(n, 0);
    bool ok = factorize(s, F, dS, ld);
    int ret = ok ? 0 : 1;
    if (ok) {
        if (!chol_solve(s, F, dx, dx)) ret = -1;
        cudaMemcpyAsync(x, dx, sizeof(double) * n, cudaMemcpyDeviceToHost, s);
    }
    cudaStreamSynchronize(s);
    if (ok && chol_solve_error()) ret = -1;
    F.release();
    hb::cache_free(dS);
    hb::cache_free(dx);
    cudaStreamDestroy(s);
    if (device_error_flag()) return -1;
    return ret;
}

int hdsdpb_inverse(int n, const double *S, double *Sinv) {
    if (n < 0 || (n > 0 && (!S || !Sinv))) return -1;
    if (n == 0) return 0;
    cudaStream_t s;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return -1;
    const long ld = pad_ld(n);
    double *dS = nullptr, *dW = nullptr;
    hb::cmalloc(&dS, sizeof(double) * ld * n);
    hb::cmalloc(&dW, sizeof(double) * ld * n);
    cudaMemcpy2D(dS, sizeof(double) * ld, S, sizeof(double) * n, sizeof(double) * n, n, cudaMemcpyHostToDevice);
    legacy_fence();
    DenseFactor F;
    F.alloc(n);
    const bool ok = factorize(s, F, dS, ld);
    if (ok) {
        compute_inverse(s, F, dW, ld);
        cudaMemcpy2DAsync(Sinv, sizeof(double) * n, dW, sizeof(double) * ld, sizeof(double) * n, n,
                          cudaMemcpyDeviceToHost, s);
    }
    cudaStreamSynchronize(s);
    F.release();
    hb::cache_free(dS);
    hb::cache_free(dW);
    cudaStreamDestroy(s);
    if (device_error_flag()) return -1;
    return ok ? 0 : 1;
}

int hdsdpb_cholesky_inverse_factor(int n, const double *S, double *L, double *K) {
    if (n < 0 || (n > 0 && (!S || !L || !K))) return -1;
    if (n == 0) return 0;
    cudaStream_t s;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return -1;
    const long ld = pad_ld(n);
    double *dS = nullptr;
    hb::cmalloc(&dS, sizeof(double) * ld * n);
    cudaMemcpy2D(dS, sizeof(double) * ld, S, sizeof(double) * n, sizeof(double) * n, n, cudaMemcpyHostToDevice);
    legacy_fence();
    DenseFactor F;
    F.alloc(n, 1);
    const bool ok = factorize(s, F, dS, ld);
    if (ok) {
        compute_inverse_factor(s, F);   // no work when the factorisation formed K
        std::vector<double> h((size_t) ld * n);
        cudaMemcpyAsync(h.data(), F.L, sizeof(double) * ld * n, cudaMemcpyDeviceToHost, s);
        cudaStreamSynchronize(s);
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) L[(size_t) j * n + i] = (i >= j) ? h[(size_t) j * ld + i] : 0.0;
        cudaMemcpyAsync(h.data(), F.K, sizeof(double) * ld * n, cudaMemcpyDeviceToHost, s);
        cudaStreamSynchronize(s);
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) K[(size_t) j * n + i] = (i >= j) ? h[(size_t) j * ld + i] : 0.0;
    }
    cudaStreamSynchronize(s);
    F.release();
    hb::cache_free(dS);
    cudaStreamDestroy(s);
    if (device_error_flag()) return -1;
    return ok ? 0 : 1;
}

int hdsdpb_gemm(int M, int N, int K, double alpha, const double *A, int lda, int transA, const double *B, int ldb,
                int transB, double beta, double *C, int ldc) {
    const int ar = transA ? K : M, ac = transA ? M : K;
    const int br = transB ? N : K, bc = transB ? K : N;
    if (M < 0 || N < 0 || K < 0 || lda < (ar > 1 ? ar : 1) || ldb < (br > 1 ? br : 1) || ldc < (M > 1 ? M : 1))
        return -1;
    if (M == 0 || N == 0) return 0;
    cudaStream_t s;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return -1;
    double *dA = nullptr, *dB = nullptr, *dC = nullptr;
    hb::cmalloc(&dA, sizeof(double) * (size_t) lda * ac);
    hb::cmalloc(&dB, sizeof(double) * (size_t) ldb * bc);
    hb::cmalloc(&dC, sizeof(double) * (size_t) ldc * N);
    cudaMemcpy(dA, A, sizeof(double) * (size_t) lda * ac, cudaMemcpyHostToDevice);
    cudaMemcpy(dB, B, sizeof(double) * (size_t) ldb * bc, cudaMemcpyHostToDevice);
    cudaMemcpy(dC, C, sizeof(double) * (size_t) ldc * N, cudaMemcpyHostToDevice);
    legacy_fence();
    gemm(s, M, N, K, alpha, dA, lda, transA, dB, ldb, transB, beta, dC, ldc, 0);
    cudaMemcpyAsync(C, dC, sizeof(double) * (size_t) ldc * N, cudaMemcpyDeviceToHost, s);
    cudaStreamSynchronize(s);
    hb::cache_free(dA);
    hb::cache_free(dB);
    hb::cache_free(dC);
    cudaStreamDestroy(s);
    return device_error_flag() ? -1 : 0;
}

int hdsdpb_split_gemm(int M, int N, int K, const double *A, int lda, int transA, const double *B, int ldb,
                      int transB, double *C, int ldc) {
    const int ar = transA ? K : M, ac = transA ? M : K;
    const int br = transB ? N : K, bc = transB ? K : N;
    if (M < 0 || N < 0 || K < 0 || lda < (ar > 1 ? ar : 1) || ldb < (br > 1 ? br : 1) || ldc < (M > 1 ? M : 1))
        return -1;
    if (M == 0 || N == 0) return 0;
    cudaStream_t s;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return -1;
    double *dA = nullptr, *dB = nullptr, *dC = nullptr;
    HB_CUDA(hb::cmalloc(&dA, sizeof(double) * (size_t) lda * (ac > 0 ? ac : 1)));
    HB_CUDA(hb::cmalloc(&dB, sizeof(double) * (size_t) ldb * (bc > 0 ? bc : 1)));
    HB_CUDA(hb::cmalloc(&dC, sizeof(double) * (size_t) ldc * N));
    HB_CUDA(cudaMemcpy(dA, A, sizeof(double) * (size_t) lda * ac, cudaMemcpyHostToDevice));
    HB_CUDA(cudaMemcpy(dB, B, sizeof(double) * (size_t) ldb * bc, cudaMemcpyHostToDevice));
    HB_CUDA(cudaMemset(dC, 0, sizeof(double) * (size_t) ldc * N));
    legacy_fence();
    SplitOperand opA, opB;
    int ret = 0;
    if (!opA.alloc(M, K) || !opB.alloc(N, K)) ret = 2;
    if (ret == 0) {
        // operand rows: op(A)(r, k) and op(B)(k, c) read as rows c
        split_from_f64(s, opA, dA, lda, transA != 0);
        split_from_f64(s, opB, dB, ldb, transB == 0);
        SplitGemm g;
        g.M = M;
        g.N = N;
        g.K = K;
        g.C = dC;
        g.ldc = ldc;
        if (!split_gemm(s, opA, opB, g)) ret = 2;
    }
    HB_CUDA(cudaStreamSynchronize(s));
    if (ret == 0 && split_error(s)) ret = -1;
    if (ret == 0) HB_CUDA(cudaMemcpy(C, dC, sizeof(double) * (size_t) ldc * N, cudaMemcpyDeviceToHost));
    opA.release();
    opB.release();
    hb::cache_free(dA);
    hb::cache_free(dB);
    hb::cache_free(dC);
    cudaStreamDestroy(s);
    if (device_error_flag()) return -1;
    return ret;
}

}  // extern "C"

// ---- device-resident kernel timing (CUDA events on the launching stream) ----
namespace {
__global__ void fill_spd_kernel(int n, double *A, long ld, unsigned seed) {
    const long total = (long) n * n;
    for (long idx = blockIdx.x * (long) blockDim.x + threadIdx.x; idx < total; idx += (long) gridDim.x * blockDim.x) {
        const int r = (int) (idx % n), c = (int) (idx / n);
        const int lo = min(r, c), hi = max(r, c);
        unsigned h = (unsigned) (lo * 2654435761u) ^ (unsigned) (hi * 40503u) ^ seed;
        h ^= h >> 13; h *= 0x5bd1e995u; h ^= h >> 15;
        double v = ((double) (h & 0xffffff) / 16777216.0 - 0.5) / n;
        if (r == c) v += 1.0;
        A[(size_t) r + (size_t) c * ld] = v;
    }
}
}  // namespace

extern "C" int hdsdpb_kernel_timing(int which, int n, int reps, double *ms) {
    cudaStream_t s;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return -1;
    const long ld = pad_ld(n);
    double *A = nullptr, *B = nullptr, *Cm = nullptr, *x = nullptr, *y = nullptr;
    hb::cmalloc(&A, sizeof(double) * ld * n);
    hb::cmalloc(&B, sizeof(double) * ld * n);
    hb::cmalloc(&Cm, sizeof(double) * ld * n);
    hb::cmalloc(&x, sizeof(double) * ld);
    hb::cmalloc(&y, sizeof(double) * ld);
    fill_spd_kernel<<<hb::counted(1024), 256, 0, s>>>(n, A, ld, 1u);
    fill_spd_kernel<<<hb::counted(1024), 256, 0, s>>>(n, B, ld, 7u);
    fill(s, x, 1.0, n);
    DenseFactor F;
    F.alloc(n, (which == 7 || which == 10) ? 1 : ((which == 8 || which == 9 || which == 11) ? 0 : -1));
    F.no_rec = (which == 10 || which == 11);
    Lanczos lz;
    if (which == 5) lz.init(n, s);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    auto once = [&]() {
        switch (which) {
            case 0: gemm(s, n, n, n, 1.0, A, ld, 0, B, ld, 0, 0.0, Cm, ld, 0); break;
            case 1: gemm(s, n, n, n, 1.0, A, ld, 1, B, ld, 0, 0.0, Cm, ld, GEMM_C_LOWER); break;
            case 2: factorize_async(s, F, A, ld); break;
            case 3: F.k_valid = false; compute_inverse_factor(s, F); break;
            case 4: coldot(s, n, n, A, ld, x, y, 1.0, 0.0, 0); break;
            case 5: { double st; lz.solve(F, B, ld, &st, nullptr); } break;
            case 6: gemm(s, n, n, 64, -1.0, A, ld, 0, B, ld, 1, 1.0, Cm, ld, GEMM_C_LOWER); break;
            case 7:
            case 8:
            case 10:
            case 11: factorize_async(s, F, A, ld); break;
            case 9: chol_solve(s, F, x, y); break;
        }
    };
    if (which == 3 || which == 5 || which == 9) factorize(s, F, A, ld);
    for (int i = 0; i < 2; ++i) once();
    cudaStreamSynchronize(s);
    cudaEventRecord(e0, s);
    for (int i = 0; i < reps; ++i) once();
    cudaEventRecord(e1, s);
    cudaEventSynchronize(e1);
    float t = 0.f;
    cudaEventElapsedTime(&t, e0, e1);
    *ms = t / reps;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (which == 5) lz.release();
    const bool solve_failed = (which == 9) && chol_solve_error();
    F.release();
    for (double *p : {A, B, Cm, x, y}) hb::cache_free(p);
    cudaStreamDestroy(s);
    return (device_error_flag() || solve_failed) ? -1 : 0;
}

namespace {
__global__ void gridsync_probe_kernel(int reps, int *sink) {
    cooperative_groups::grid_group g = cooperative_groups::this_grid();
    for (int i = 0; i < reps; ++i) g.sync();
    if (blockIdx.x == 0 && threadIdx.x == 0) *sink = reps;
}
}  // namespace

// Milliseconds for `reps` grid-wide barriers of a cooperative launch of `blocks` x 256 threads.
extern "C" int hdsdpb_gridsync_probe(int blocks, int reps, double *ms) {
    int *sink = nullptr;
    hb::cmalloc(&sink, sizeof(int));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    void *args[] = {&reps, &sink};
    cudaEventRecord(e0, 0);
    cudaError_t e = cudaLaunchCooperativeKernel((const void *) gridsync_probe_kernel, hb::counted(blocks), 256, args, 0, 0);
    cudaEventRecord(e1, 0);
    cudaEventSynchronize(e1);
    float t = 0.f;
    cudaEventElapsedTime(&t, e0, e1);
    *ms = t;
    hb::cache_free(sink);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return e == cudaSuccess ? 0 : -1;
}

