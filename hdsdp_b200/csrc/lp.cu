// LP cone s = c - A^T y - r >= 0 next to the SDP block (interface/hdsdp_conic_lp.c).
//
// The slack vectors are host-side O(nnz) work, like the scalar bound cone. The cone's
// Schur block, M_ij += sum_k A_ki A_kj / s_k^2, touches only the constraint pairs that
// share an LP column; those pairs are found once and each build adds their values to
// the device Schur matrix after the SDP block's terms, in the order of the reference's
// dense loop (interface/hdsdp_conic_lp.c:284-300).
#include "solver.h"
#include <algorithm>
#include <cmath>

namespace hb {

namespace {
__global__ void add_pairs_kernel(int np, const int *__restrict__ pi, const int *__restrict__ pj,
                                 const double *__restrict__ v, double *M, long ldm) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < np; t += gridDim.x * blockDim.x)
        M[(size_t) pi[t] + (size_t) pj[t] * ldm] += v[t];
}
}  // namespace

// LPConeProcDataImpl (interface/hdsdp_conic_lp.c:99-158): column 0 of the user's CSC is
// c, columns 1..m the constraints.
hdsdp_retcode LpCone::proc_data(int nRow, int nCol_, const int *Ap, const int *Ai, const double *Ax,
                                cudaStream_t stream) {
    m = nRow;
    nCol = nCol_;
    st = stream;
    obj.assign(nCol, 0.0);
    for (int e = Ap[0]; e < Ap[1]; ++e) obj[Ai[e]] = Ax[e];
    const int off = Ap[1];
    beg.assign(m + 1, 0);
    for (int i = 0; i <= m; ++i) beg[i] = Ap[i + 1] - off;
    idx.assign(Ai + off, Ai + Ap[m + 1]);
    val.assign(Ax + off, Ax + Ap[m + 1]);
    for (int k : idx)
        if (k < 0 || k >= nCol) return HDSDP_RETCODE_FAILED;
    s.assign(nCol, 0.0);
    sChk.assign(nCol, 0.0);
    sStep.assign(nCol, 0.0);
    sInv.assign(nCol, 0.0);
    buf.assign(nCol, 0.0);
    // constraint pairs (i >= j) sharing an LP column
    std::vector<std::vector<int>> rowsOf(nCol);
    for (int i = 0; i < m; ++i)
        for (int e = beg[i]; e < beg[i + 1]; ++e) rowsOf[idx[e]].push_back(i);
    std::vector<int> mark(m, -1);
    pairI.clear();
    pairJ.clear();
    for (int i = 0; i < m; ++i) {
        for (int e = beg[i]; e < beg[i + 1]; ++e)
            for (int j : rowsOf[idx[e]])
                if (j <= i && mark[j] != i) {
                    mark[j] = i;
                    pairI.push_back(i);
                    pairJ.push_back(j);
                }
    }
    pairVal.assign(pairI.size(), 0.0);
    if (!pairI.empty()) {
        const size_t np = pairI.size();
        HB_CUDA(hb::cmalloc(&d_pi, sizeof(int) * np));
        HB_CUDA(hb::cmalloc(&d_pj, sizeof(int) * np));
        HB_CUDA(hb::cmalloc(&d_pv, sizeof(double) * np));
        HB_CUDA(cudaMemcpyAsync(d_pi, pairI.data(), sizeof(int) * np, cudaMemcpyHostToDevice, st));
        HB_CUDA(cudaMemcpyAsync(d_pj, pairJ.data(), sizeof(int) * np, cudaMemcpyHostToDevice, st));
        HB_CUDA(cudaStreamSynchronize(st));
    }
    return HDSDP_RETCODE_OK;
}

void LpCone::release() {
    if (d_pi) hb::cache_free(d_pi);
    if (d_pj) hb::cache_free(d_pj);
    if (d_pv) hb::cache_free(d_pv);
    d_pi = d_pj = nullptr;
    d_pv = nullptr;
}

// LPConeGetObjNorm / LPConeGetCoeffNorm (interface/hdsdp_conic_lp.c:171-198); the
// coefficient norms count an entry whose LP column equals its constraint index at half
// weight, as csp_sum_abs / csp_fro_norm do (linalg/sparse_opts.c:54-76).
double LpCone::obj_norm(int type) const {
    double d = 0.0;
    if (type == ABS_NORM) {
        for (double v : obj) d += std::fabs(v);
        return d;
    }
    for (double v : obj) d += v * v;
    return std::sqrt(d);
}

double LpCone::coeff_norm(int type) const {
    double d = 0.0;
    for (int i = 0; i < m; ++i)
        for (int e = beg[i]; e < beg[i + 1]; ++e) {
            const double a = val[e];
            if (type == ABS_NORM) d += (idx[e] == i) ? 0.5 * std::fabs(a) : std::fabs(a);
            else d += (idx[e] == i) ? 0.5 * a * a : a * a;
        }
    return type == ABS_NORM ? d : std::sqrt(d);
}

void LpCone::scal(double a) {
    for (double &v : obj) v /= a;
}

// LPConeGetStatsImpl (interface/hdsdp_conic_lp.c:507-634): implied dual bounds from
// constraints with at most two LP entries, and free-variable pairs (no dual interior).
void LpCone::detect_feature(int intF[20], double dblF[20]) const {
    if (nCol % 2 != 0 || nCol < 100) return;
    std::vector<double> up(m, 0.0), lo(m, 0.0);
    bool implied = true, isUp = false, isLo = false;
    for (int i = 0; i < m && implied; ++i) {
        for (int e = beg[i]; e < beg[i + 1]; ++e) {
            if (beg[i + 1] - beg[i] > 2) {
                implied = false;
                break;
            }
            if (val[e] > 0.0) {
                if (up[i]) {
                    implied = false;
                    break;
                }
                isUp = true;
                up[i] = std::max(up[i], obj[idx[e]] / val[e]);
            } else {
                if (lo[i]) {
                    implied = false;
                    break;
                }
                isLo = true;
                lo[i] = std::min(lo[i], obj[idx[e]] / val[e]);
            }
        }
    }
    if (implied) {
        intF[6] = 1;  // implied dual bound
        if (isUp) {
            double b = 1.0;
            for (int i = 0; i < m; ++i) b = std::max(b, up[i]);
            if (b <= 0.0) b = 1.0;
            dblF[9] = b;  // upper
        }
        if (isLo) {
            double b = -1.0;
            for (int i = 0; i < m; ++i) b = std::min(b, lo[i]);
            if (b >= 0.0) b = -1.0;
            dblF[10] = b;  // lower
        }
    }
    const int half = nCol / 2;
    for (int k = 0; k < half; ++k)
        if (obj[k] + obj[k + half] != 0.0) return;
    for (int i = 0; i < m; ++i) {
        const int cnt = beg[i + 1] - beg[i], h = cnt / 2;
        if (cnt % 2 != 0) return;
        for (int r = 0; r < h; ++r)
            if (val[beg[i] + r] + val[beg[i] + r + h] != 0.0) return;
    }
    intF[3] = 1;  // no dual interior
}

// LPConeIUpdateBuffer (interface/hdsdp_conic_lp.c:44-81):
// target = dC c + dAs A^T y + (dEye [+ perturbation outside the step buffer]) e
void LpCone::update_buffer(double dC, double dAs, const double *y, double dEye, int which) {
    std::vector<double> &t = (which == BUFFER_DUALVAR) ? s : (which == BUFFER_DUALCHECK) ? sChk : sStep;
    std::fill(t.begin(), t.end(), 0.0);
    if (dAs != 0.0)
        for (int i = 0; i < m; ++i)
            for (int e = beg[i]; e < beg[i + 1]; ++e) t[idx[e]] += dAs * y[i] * val[e];
    for (int k = 0; k < nCol; ++k) t[k] += dC * obj[k];
    if (which != BUFFER_DUALSTEP) dEye += dualPerturb;
    if (dEye != 0.0)
        for (int k = 0; k < nCol; ++k) t[k] += dEye;
}

static int all_positive(const std::vector<double> &v) {
    for (double x : v)
        if (x <= 0.0) return 0;
    return 1;
}

// LPConeRatioTestImpl (interface/hdsdp_conic_lp.c:213-245): the running minimum starts
// at 0, so a direction that never decreases a slack gives the cap 100.
double LpCone::ratio_test(double dtau, const double *dy, double ada, int which) {
    update_buffer(dtau, -1.0, dy, ada * dualResidual, BUFFER_DUALSTEP);
    const std::vector<double> &t = (which == BUFFER_DUALVAR) ? s : sChk;
    double mx = 0.0;
    for (int k = 0; k < nCol; ++k) mx = std::min(mx, sStep[k] / t[k]);
    mx = 1.0 / mx;
    return (mx > 0.0) ? 100.0 : -mx;
}

int LpCone::interior_check(double tau, const double *y) {
    update(tau, y);
    return all_positive(s);
}

int LpCone::interior_check_expert(double dC, double dAs, const double *y, double dEye, int which) {
    update_buffer(dC, dAs, y, dEye, which);
    return all_positive(which == BUFFER_DUALVAR ? s : sChk);
}

// LPConeGetBarrier (interface/hdsdp_conic_lp.c:379-400)
double LpCone::get_barrier(double tau, const double *y, int which) {
    if (y) update(tau, y);
    const std::vector<double> &t = (which == BUFFER_DUALVAR) ? s : sChk;
    double ld = 0.0;
    for (double v : t) ld += std::log(v);
    return ld;
}

// LPConeAddStepToBufferAndCheck (interface/hdsdp_conic_lp.c:402-417)
int LpCone::add_step_and_check(double step, int which) {
    std::vector<double> &t = (which == BUFFER_DUALVAR) ? s : sChk;
    if (which != BUFFER_DUALVAR) sChk = s;
    for (int k = 0; k < nCol; ++k) t[k] += step * sStep[k];
    return all_positive(t);
}

// LPConeGetPrimal (interface/hdsdp_conic_lp.c:419-439): x = mu (s + A^T dy) / s^2 at
// s = c - A^T y; left untouched when that slack is not interior.
void LpCone::get_primal(double mu, const double *y, const double *dy, double *x) {
    if (!interior_check_expert(1.0, -1.0, y, 0.0, BUFFER_DUALCHECK)) {
        printf("Recovery step is infeasible\n");
        return;
    }
    update_buffer(0.0, 1.0, dy, 0.0, BUFFER_DUALSTEP);
    for (int k = 0; k < nCol; ++k) x[k] = mu * (sChk[k] + sStep[k]) / (sChk[k] * sChk[k]);
}

void LpCone::get_dual(double *out) const { std::copy(s.begin(), s.end(), out); }

void LpCone::atimesx(const double *x, double *out) const {
    for (int i = 0; i < m; ++i) {
        double a = 0.0;
        for (int e = beg[i]; e < beg[i + 1]; ++e) a += x[idx[e]] * val[e];
        out[i] += a;
    }
}

double LpCone::trace_cx(const double *x) const {
    double d = 0.0;
    for (int k = 0; k < nCol; ++k) d += obj[k] * x[k];
    return d;
}

// LPConeGetKKT (interface/hdsdp_conic_lp.c:252-319), after the SDP block's build.
void KKT::add_lp(LpCone &lp, int type) {
    const int nc = lp.nCol;
    for (int k = 0; k < nc; ++k) lp.sInv[k] = 1.0 / lp.s[k];
    auto atx = [&](const std::vector<double> &x, std::vector<double> &y) {
        for (int i = 0; i < m; ++i) {
            double a = 0.0;
            for (int e = lp.beg[i]; e < lp.beg[i + 1]; ++e) a += x[lp.idx[e]] * lp.val[e];
            y[i] += a;
        }
    };
    atx(lp.sInv, asinv);
    if (lp.dualResidual) {
        for (int k = 0; k < nc; ++k) dTraceSinv += lp.sInv[k];
        for (int k = 0; k < nc; ++k) lp.buf[k] = lp.dualResidual * lp.sInv[k] * lp.sInv[k];
        atx(lp.buf, asinvrd);
    }
    if (type == KKT_TYPE_CORRECTOR) return;
    open_m();
    // M_ij += sum over column j of A_kj (A_ki / s_k^2), the value for column i kept per LP
    // column (the last of a repeated index wins, as in the reference's buffer)
    if (!lp.pairI.empty()) {
        std::fill(lp.buf.begin(), lp.buf.end(), 0.0);
        size_t p = 0;
        const size_t np = lp.pairI.size();
        while (p < np) {
            const int i = lp.pairI[p];
            for (int e = lp.beg[i]; e < lp.beg[i + 1]; ++e) {
                const int k = lp.idx[e];
                lp.buf[k] = lp.val[e] * (lp.sInv[k] * lp.sInv[k]);
            }
            for (; p < np && lp.pairI[p] == i; ++p) {
                const int j = lp.pairJ[p];
                double v = 0.0;
                for (int e = lp.beg[j]; e < lp.beg[j + 1]; ++e) v += lp.val[e] * lp.buf[lp.idx[e]];
                lp.pairVal[p] = v;
            }
            for (int e = lp.beg[i]; e < lp.beg[i + 1]; ++e) lp.buf[lp.idx[e]] = 0.0;
        }
        HB_CUDA(cudaMemcpyAsync(lp.d_pv, lp.pairVal.data(), sizeof(double) * np, cudaMemcpyHostToDevice, s));
        add_pairs_kernel<<<hb::counted((int) std::min<size_t>((np + 255) / 256, 148 * 8)), 256, 0, s>>>(
            (int) np, lp.d_pi, lp.d_pj, lp.d_pv, M, ldm);
        HB_CUDA(cudaGetLastError());
        HB_CUDA(cudaStreamSynchronize(s));
    }
    if (type == KKT_TYPE_HOMOGENEOUS) {
        for (int k = 0; k < nc; ++k) {
            const double d = lp.obj[k] * lp.sInv[k];
            dCSinv += d;
            dCSinvCSinv += d * d;
        }
        for (int k = 0; k < nc; ++k) lp.buf[k] = lp.obj[k] * lp.sInv[k] * lp.sInv[k];
        atx(lp.buf, asinvcs);
    }
}

}  // namespace hb
