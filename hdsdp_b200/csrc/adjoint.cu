// Adjoint of the SDP solution map at the final iterate (no reference counterpart).
//
// The solve returns (y*, X*, S* = C - A^T y*). The iterate is first purified
// into an exactly complementary pair: with X* - S* = Q diag(lambda) Q^T,
// Xbar = Q diag(lambda+) Q^T and Sbar = Q diag(lambda-) Q^T, computed without
// an eigensolver from the spectral projector P+ = (I + sign(X* - S*)) / 2
// (Newton-Schulz sign iteration, FP64 GEMMs). The derivative is that of the
// central-path point at a small mu, Xhat = Xbar + mu Sbar^+, Shat = Sbar +
// mu Xbar^+ (Xhat Shat = mu I exactly), whose Nesterov-Todd scaling is
// N = Xbar / sqrt(mu) + sqrt(mu) Sbar^+ (N Shat N = Xhat). Linearising
//   A(X) = b,  A^T(y) + S = C,  X = N S N
// there gives, with E = dC - sum_i y_i dA_i,
//     M dy = db - dA(X) + A(N E N),   dX = N (A^T dy - E) N,
//     M_ij = <A_i, N A_j N>,
// and for a loss L = <G_X, X*> + g_y^T y* the vector-Jacobian product
//     u = g_y + A(N G_X N),   v = M^-1 u,   Z = N (A^T(v) - G_X) N,
//     dL/db = v,   dL/dC = Z,   dL/dA_i = -v_i Xhat - y_i Z.
// For strictly complementary solutions the result does not depend on mu to
// first order; mu is <X*, S*>/n clipped to [1e-8, 1e-6]: the condition number of M
// grows like 1/mu^2, and below 1e-8 it passes what FP64 resolves (about 1e16), so a
// smaller mu only adds rounding noise to the gradient. M is assembled by
// the solver's Schur kernels with N in place of S^-1. N, M and its factor are
// cached after the first call for a solve, so further calls cost two n x n
// products, one Schur solve and the A(.)/A^T(.) maps.
#include "solver.h"
#include "../../include/hdsdp_b200.h"
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

namespace hb {
void solver_cone_values(hdsdp *h, double *X, double *S);
double solver_obj_scal(hdsdp *h);
double solver_rhs_scal(hdsdp *h);

namespace {

__global__ void grad_values_kernel(long nnz, const int *__restrict__ col, const int *__restrict__ ri,
                                   const int *__restrict__ ci, const double *__restrict__ X,
                                   const double *__restrict__ Z, long ld, const double *__restrict__ v,
                                   const double *__restrict__ y, double *out) {
    for (long e = blockIdx.x * (long) blockDim.x + threadIdx.x; e < nnz; e += (long) gridDim.x * blockDim.x) {
        const int c = col[e], i = ri[e], j = ci[e];
        const double f = (i == j) ? 1.0 : 2.0;  // an off-diagonal packed entry stands for (i, j) and (j, i)
        const size_t o = (size_t) i + (size_t) j * ld;
        out[e] = (c == 0) ? f * Z[o] : f * (-v[c - 1] * X[o] - y[c - 1] * Z[o]);
    }
}

__global__ void ns_step_kernel(int n, const double *P, long ld, double *T) {
    // T = 1.5 I - 0.5 P
    const long total = (long) n * n;
    for (long t = blockIdx.x * (long) blockDim.x + threadIdx.x; t < total; t += (long) gridDim.x * blockDim.x) {
        const int i = (int) (t % n), j = (int) (t / n);
        const size_t o = (size_t) i + (size_t) j * ld;
        T[o] = (i == j ? 1.5 : 0.0) - 0.5 * P[o];
    }
}

int grid_for(long n) { return (int) std::min<long>((n + 255) / 256, 148L * 8); }

}  // namespace

struct AdjointState {
    int n = 0, m = 0;
    long ld = 0, ldm = 0;
    double *X = nullptr, *S = nullptr, *N = nullptr, *T1 = nullptr, *T2 = nullptr, *Y = nullptr, *Z = nullptr,
           *P = nullptr, *D = nullptr, *M = nullptr;
    double *d_u = nullptr, *d_v = nullptr, *d_t = nullptr, *d_r = nullptr, *d_y = nullptr, *d_scal = nullptr;
    double *h_scal = nullptr;
    int *d_col = nullptr, *d_ri = nullptr, *d_ci = nullptr;
    double *d_gax = nullptr;
    long nnz = 0;
    DenseFactor FS, FM;
    std::vector<double> yuser;
    bool ready = false;

    void release() {
        for (double *p : {X, S, N, T1, T2, Y, Z, P, D, M, d_u, d_v, d_t, d_r, d_y, d_scal, d_gax})
            if (p) hb::cache_free(p);
        for (int *p : {d_col, d_ri, d_ci})
            if (p) hb::cache_free(p);
        if (h_scal) hb::cache_free_host(h_scal);
        X = S = N = T1 = T2 = Y = Z = P = D = M = d_u = d_v = d_t = d_r = d_y = d_scal = d_gax = nullptr;
        d_col = d_ri = d_ci = nullptr;
        h_scal = nullptr;
        FS.release();
        FM.release();
        ready = false;
    }
};

void adjoint_release(AdjointState *&a) {
    if (!a) return;
    a->release();
    delete a;
    a = nullptr;
}

namespace {

double host_scalar(cudaStream_t s, const double *d, double *h) {
    HB_CUDA(cudaMemcpyAsync(h, d, sizeof(double), cudaMemcpyDeviceToHost, s));
    HB_CUDA(cudaStreamSynchronize(s));
    return *h;
}

// Schur systems of at least this order are solved with L (triangular solves) instead
// of through the explicit inverse factor, which would cost a second factorisation.
constexpr int kAdjTriSolveMinM = 6000;

// x = M^-1 y with the factor: through K = L^-1 (M = L L^T) for small m, by triangular
// solves with L for large m.
bool factor_apply(cudaStream_t s, AdjointState &a, const double *y, double *x) {
    if (a.FM.fuse_k) {
        coldot(s, a.m, a.m, a.FM.KT, a.ldm, y, a.d_t, 1.0, 0.0, 2);  // t = K y
        coldot(s, a.m, a.m, a.FM.K, a.ldm, a.d_t, x, 1.0, 0.0, 1);   // x = K^T t
        return true;
    }
    return chol_solve(s, a.FM, y, x);
}

// v = M^-1 u with two steps of iterative refinement (M is ill-conditioned in the
// directions of the optimal face).
bool schur_solve(cudaStream_t s, AdjointState &a, const double *u, double *v) {
    const int m = a.m;
    bool ok = factor_apply(s, a, u, v);
    for (int it = 0; it < 2; ++it) {
        coldot(s, m, m, a.M, a.ldm, v, a.d_r, -1.0, 0.0, 0);  // r = -M v
        axpy(s, m, 1.0, u, a.d_r);                           // r = u - M v
        ok = ok && factor_apply(s, a, a.d_r, a.d_r);
        axpy(s, m, 1.0, a.d_r, v);
    }
    return ok;
}

hdsdp_retcode prepare(hdsdp *h, AdjointState &a) {
    SdpCone &c = *h->cone;
    cudaStream_t s = c.s;
    const int n = c.n, m = h->nRows;
    const long ld = c.ld, ldm = pad_ld(m);
    a.n = n;
    a.m = m;
    a.ld = ld;
    a.ldm = ldm;
    for (double **p : {&a.X, &a.S, &a.N, &a.T1, &a.T2, &a.Y, &a.Z, &a.P, &a.D})
        HB_CUDA(hb::cmalloc(p, sizeof(double) * ld * n));
    HB_CUDA(hb::cmalloc(&a.M, sizeof(double) * ldm * m));
    for (double **p : {&a.d_u, &a.d_v, &a.d_t, &a.d_r, &a.d_y}) HB_CUDA(hb::cmalloc(p, sizeof(double) * (m + 1)));
    HB_CUDA(hb::cmalloc(&a.d_scal, sizeof(double) * 4));
    HB_CUDA(hb::cmalloc_host(&a.h_scal, sizeof(double) * 4));
    a.FS.alloc(n);
    a.FM.alloc(m, m < kAdjTriSolveMinM ? 1 : 0);
    if (device_error_flag()) return HDSDP_RETCODE_MEMORY;

    // the solution in the user's units
    const double objScal = solver_obj_scal(h), rhsScal = solver_rhs_scal(h);
    HB_CUDA(cudaMemsetAsync(a.X, 0, sizeof(double) * ld * n, s));
    solver_cone_values(h, a.X, nullptr);
    if (rhsScal != 1.0) scale_matrix(s, n, n, a.X, ld, 1.0 / rhsScal);
    a.yuser.assign(m, 0.0);
    for (int i = 0; i < m; ++i) a.yuser[i] = h->y[i] / objScal;
    HB_CUDA(cudaMemcpyAsync(a.d_y, a.yuser.data(), sizeof(double) * m, cudaMemcpyHostToDevice, s));
    c.dev.assemble(1.0 / objScal, -1.0, a.d_y, 0.0, a.S, ld);  // S = C - A^T y
    HB_CUDA(cudaStreamSynchronize(s));

    // mu of the final iterate, then the purified complementary pair: with
    // Z = X - S = Q diag(lambda) Q^T, Xbar = Q diag(lambda+) Q^T and
    // Sbar = Q diag(lambda-) Q^T, from the spectral projector P+ = (I + sign Z)/2
    // (sign Z by the Newton-Schulz iteration Y <- Y (3I - Y^2)/2, GEMMs only).
    frob_dot(s, n, a.X, ld, a.S, ld, a.d_scal);
    const double xs = host_scalar(s, a.d_scal, a.h_scal) / n;
    const double mu = std::min(1e-6, std::max(1e-8, xs));
    copy_matrix(s, n, n, a.X, ld, a.Z, ld);
    axpy(s, (int) (ld * n), -1.0, a.S, a.Z);
    frob_dot(s, n, a.Z, ld, a.Z, ld, a.d_scal);
    const double cnorm = std::sqrt(host_scalar(s, a.d_scal, a.h_scal));
    if (!(cnorm > 0.0) || !std::isfinite(cnorm)) return HDSDP_RETCODE_FAILED;
    copy_matrix(s, n, n, a.Z, ld, a.Y, ld);
    scale_matrix(s, n, n, a.Y, ld, 1.0 / cnorm);
    double *Yk = a.Y, *Yn = a.T1;
    bool converged = false;
    int polish = 2;  // quadratic convergence: two more steps reach the rounding level
    for (int it = 0; it < 100 && polish > 0; ++it) {
        if (converged) --polish;
        gemm(s, n, n, n, 1.0, Yk, ld, 0, Yk, ld, 0, 0.0, a.P, ld, 0);                 // P = Y^2
        ns_step_kernel<<<hb::counted(grid_for((long) n * n)), 256, 0, s>>>(n, a.P, ld, a.N);  // T = 1.5 I - 0.5 P
        gemm(s, n, n, n, 1.0, Yk, ld, 0, a.N, ld, 0, 0.0, Yn, ld, 0);                 // Y <- Y T
        std::swap(Yk, Yn);
        if (!converged && it % 4 == 3) {
            add_diag(s, n, a.P, ld, -1.0);
            frob_dot(s, n, a.P, ld, a.P, ld, a.d_scal);
            converged = std::sqrt(host_scalar(s, a.d_scal, a.h_scal)) < 1e-12 * std::sqrt((double) n);
        }
    }
    if (!converged) return HDSDP_RETCODE_FAILED;
    copy_matrix(s, n, n, Yk, ld, a.D, ld);                       // D = P+ = (I + sign Z) / 2
    scale_matrix(s, n, n, a.D, ld, 0.5);
    add_diag(s, n, a.D, ld, 0.5);
    symmetrize_avg(s, n, a.D, ld);
    gemm(s, n, n, n, 1.0, a.Z, ld, 0, a.D, ld, 0, 0.0, a.T2, ld, 0);  // T2 = Xbar = Z P+
    symmetrize_avg(s, n, a.T2, ld);
    copy_matrix(s, n, n, a.T2, ld, a.S, ld);                     // S = Sbar = Xbar - Z
    axpy(s, (int) (ld * n), -1.0, a.Z, a.S);
    // Sbar^+ = (Sbar + P+)^-1 - P+ (Sbar + P+ is positive definite)
    copy_matrix(s, n, n, a.S, ld, a.P, ld);
    axpy(s, (int) (ld * n), 1.0, a.D, a.P);
    if (!factorize(s, a.FS, a.P, ld)) return HDSDP_RETCODE_FAILED;
    compute_inverse(s, a.FS, a.N, ld);
    axpy(s, (int) (ld * n), -1.0, a.D, a.N);                      // N (scratch) = Sbar^+
    // central point at mu: Xhat = Xbar + mu Sbar^+, NT scaling Nt = Xbar / sqrt(mu) + sqrt(mu) Sbar^+
    copy_matrix(s, n, n, a.T2, ld, a.Y, ld);
    scale_matrix(s, n, n, a.Y, ld, 1.0 / std::sqrt(mu));
    axpy(s, (int) (ld * n), std::sqrt(mu), a.N, a.Y);
    copy_matrix(s, n, n, a.T2, ld, a.X, ld);
    axpy(s, (int) (ld * n), mu, a.N, a.X);
    std::swap(a.N, a.Y);                                          // a.N holds the scaling from here on

    // Schur matrix in the NT scaling and its factor
    c.dev.schur_matrix(a.N, ld, a.M, ldm);
    symmetrize_lower(s, m, a.M, ldm);
    if (!factorize(s, a.FM, a.M, ldm)) return HDSDP_RETCODE_FAILED;
    if (a.FM.fuse_k) compute_inverse_factor(s, a.FM);

    // (column, row, col) of every stored value of the user's CSC data
    const user_data *u = h->cones[0].usr;
    a.nnz = u->coneMatBeg[m + 1];
    std::vector<int> col(a.nnz), ri(a.nnz), ci(a.nnz);
    std::vector<long> start(n);
    for (int j = 0; j < n; ++j) start[j] = (long) (2L * n - j - 1) * j / 2 + j;
    for (int k = 0; k <= m; ++k)
        for (int e = u->coneMatBeg[k]; e < u->coneMatBeg[k + 1]; ++e) {
            const long p = u->coneMatIdx[e];
            int j = (int) (std::upper_bound(start.begin(), start.end(), p) - start.begin()) - 1;
            col[e] = k;
            ci[e] = j;
            ri[e] = (int) (p - start[j] + j);
        }
    if (a.nnz > 0) {
        HB_CUDA(hb::cmalloc(&a.d_col, sizeof(int) * a.nnz));
        HB_CUDA(hb::cmalloc(&a.d_ri, sizeof(int) * a.nnz));
        HB_CUDA(hb::cmalloc(&a.d_ci, sizeof(int) * a.nnz));
        HB_CUDA(hb::cmalloc(&a.d_gax, sizeof(double) * a.nnz));
        HB_CUDA(cudaMemcpyAsync(a.d_col, col.data(), sizeof(int) * a.nnz, cudaMemcpyHostToDevice, s));
        HB_CUDA(cudaMemcpyAsync(a.d_ri, ri.data(), sizeof(int) * a.nnz, cudaMemcpyHostToDevice, s));
        HB_CUDA(cudaMemcpyAsync(a.d_ci, ci.data(), sizeof(int) * a.nnz, cudaMemcpyHostToDevice, s));
    }
    HB_CUDA(cudaStreamSynchronize(s));
    if (device_error_flag()) return HDSDP_RETCODE_FAILED;
    a.ready = true;
    return HDSDP_RETCODE_OK;
}

}  // namespace

hdsdp_retcode adjoint_vjp(hdsdp *h, AdjointState *&state, const double *gy, const double *GX, double *gb,
                          double *gC, double *gAx) {
    // defined for a problem of one dense SDP cone
    if (!h || !h->optimized || !h->cone || h->nCones != 1 || h->cone->sparse) return HDSDP_RETCODE_FAILED;
    if (!state) state = new AdjointState();
    AdjointState &a = *state;
    if (!a.ready) {
        a.release();
        hdsdp_retcode r = prepare(h, a);
        if (r != HDSDP_RETCODE_OK) {
            a.release();
            return r;
        }
    }
    SdpCone &c = *h->cone;
    cudaStream_t s = c.s;
    const int n = a.n, m = a.m;
    const long ld = a.ld;
    // u = g_y + A(N G_X N)
    if (GX) {
        HB_CUDA(cudaMemcpy2DAsync(a.D, sizeof(double) * ld, GX, sizeof(double) * n, sizeof(double) * n, n,
                                  cudaMemcpyHostToDevice, s));
        gemm(s, n, n, n, 1.0, a.N, ld, 0, a.D, ld, 0, 0.0, a.T1, ld, 0);
        gemm(s, n, n, n, 1.0, a.T1, ld, 0, a.N, ld, 0, 0.0, a.T2, ld, 0);
        symmetrize_avg(s, n, a.T2, ld);
        HB_CUDA(cudaMemsetAsync(a.d_u, 0, sizeof(double) * m, s));
        c.dev.inner_all(a.T2, ld, a.d_u);
    } else {
        HB_CUDA(cudaMemsetAsync(a.D, 0, sizeof(double) * ld * n, s));
        HB_CUDA(cudaMemsetAsync(a.d_u, 0, sizeof(double) * m, s));
    }
    if (gy) {
        HB_CUDA(cudaMemcpyAsync(a.d_r, gy, sizeof(double) * m, cudaMemcpyHostToDevice, s));
        axpy(s, m, 1.0, a.d_r, a.d_u);
    }
    // v = M^-1 u
    if (!schur_solve(s, a, a.d_u, a.d_v)) return HDSDP_RETCODE_FAILED;
    // Z = N (A^T v - G_X) N
    c.dev.assemble(0.0, 1.0, a.d_v, 0.0, a.T2, ld);
    axpy(s, (int) (ld * n), -1.0, a.D, a.T2);
    gemm(s, n, n, n, 1.0, a.N, ld, 0, a.T2, ld, 0, 0.0, a.T1, ld, 0);
    gemm(s, n, n, n, 1.0, a.T1, ld, 0, a.N, ld, 0, 0.0, a.Z, ld, 0);
    symmetrize_avg(s, n, a.Z, ld);
    if (gb) HB_CUDA(cudaMemcpyAsync(gb, a.d_v, sizeof(double) * m, cudaMemcpyDeviceToHost, s));
    if (gC)
        HB_CUDA(cudaMemcpy2DAsync(gC, sizeof(double) * n, a.Z, sizeof(double) * ld, sizeof(double) * n, n,
                                  cudaMemcpyDeviceToHost, s));
    if (gAx && a.nnz > 0) {
        grad_values_kernel<<<hb::counted(grid_for(a.nnz)), 256, 0, s>>>(a.nnz, a.d_col, a.d_ri, a.d_ci, a.X, a.Z,
                                                                         ld, a.d_v, a.d_y, a.d_gax);
        HB_CUDA(cudaMemcpyAsync(gAx, a.d_gax, sizeof(double) * a.nnz, cudaMemcpyDeviceToHost, s));
    }
    HB_CUDA(cudaStreamSynchronize(s));
    if (!a.FM.fuse_k && chol_solve_error()) return HDSDP_RETCODE_FAILED;
    return device_error_flag() ? HDSDP_RETCODE_FAILED : HDSDP_RETCODE_OK;
}

}  // namespace hb

extern "C" hdsdp_retcode HDSDPAdjoint(hdsdp *h, const double *gy, const double *GX, double *gb, double *gC,
                                      double *gAx) {
    return hb::adjoint_vjp(h, h->adj, gy, GX, gb, gC, gAx);
}
