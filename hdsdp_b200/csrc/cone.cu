// Dense SDP cone, scalar bound cone, Schur (KKT) system and Lanczos step
// estimator of the B200 HDSDP solver.
#include "solver.h"
#include <cooperative_groups.h>
#include <cmath>
#include <cstring>
#include <cstdlib>
#include <algorithm>
#include <chrono>

namespace hb {

// Schur systems of at least this order are solved by triangular solves with L rather
// than through K = L^-1: forming K costs as much as the factorisation, while a solve
// with L reads L once.

// Hybrid sparse factorisation of S: automatic from this order on, minimum-degree rounds
// up to this degree, and used only when the dense front is at most this fraction of n
// (front flops at most a third of the dense factorisation's).
constexpr int kHybridMinN = 1500;
constexpr int kHybridCap = 64;
constexpr double kHybridMaxFront = 0.7;


static double wall() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

// ======================================================================================
// Presolve: coefficient types and rank-one extraction
// ======================================================================================
namespace {

// Packed lower-triangle index -> (row, col) (interface/hdsdp_utils.h:49).
inline void unpack(int n, long p, int &i, int &j) {
    // column j starts at j*(2n - j + 1)/2
    long lo = 0, hi = n - 1;
    while (lo < hi) {
        long mid = (lo + hi + 1) / 2;
        long start = mid * (2L * n - mid + 1) / 2;
        if (start <= p) lo = mid;
        else hi = mid - 1;
    }
    j = (int) lo;
    i = (int) (p - ((2L * n - lo - 1) * lo) / 2);
}

// Rank-one test of a sparse lower triplet matrix, following the acceptance rules of
// tsp_r1_extract (linalg/sparse_opts.c:151-214): the first stored entry must be
// diagonal, its column defines a, the entry count must be that of a's outer product,
// and the reconstruction error in the 1-norm must not exceed 1e-10.
bool sparse_rank_one(int n, const std::vector<int> &r, const std::vector<int> &c, const std::vector<double> &v,
                     double &sgn, std::vector<double> &a) {
    const int nnz = (int) v.size();
    if (nnz == 0) return false;
    a.assign(n, 0.0);
    const int i0 = r[0];
    if (r[0] != c[0]) return false;
    if (nnz == 1) {
        sgn = v[0];
        a[i0] = 1.0;
        return true;
    }
    const double s = (v[0] > 0) ? 1.0 : -1.0;
    const double root = std::sqrt(std::fabs(v[0]));
    int k = 0, anz = 0;
    for (k = 0; k < nnz; ++k) {
        if (c[k] > i0) break;
        a[r[k]] = v[k] / root;
        anz += 1;
    }
    if (nnz != anz * (anz + 1) / 2) return false;
    if (k == n) return false;
    double eps = 0.0;
    for (int e = 0; e < nnz; ++e) eps += std::fabs(v[e] - s * a[r[e]] * a[c[e]]);
    if (eps > 1e-10) return false;
    sgn = s;
    return true;
}

// Rank-one test of a dense packed matrix (pds_r1_extract, linalg/dense_opts.c:174-230):
// a is read from the column of the first nonzero diagonal entry.
bool dense_rank_one(int n, const std::vector<double> &P, double &sgn, std::vector<double> &a) {
    long k = 0;
    int i;
    for (i = 0; i < n; ++i) {
        if (P[k] != 0) break;
        k += n - i;
    }
    if (i == n) return false;
    const double s = (P[k] > 0) ? 1.0 : -1.0;
    const double root = std::sqrt(std::fabs(P[k]));
    a.assign(n, 0.0);
    const long colStart = ((2L * n - i - 1) * i) / 2;
    for (int q = 0; q < n; ++q) a[q] = P[colStart + q] / root;
    double eps = 0.0;
    long id = 0;
    for (int col = 0; col < n; ++col) {
        for (int j = 0; j < n - col; ++j) eps += std::fabs(P[id + j] - s * a[col] * a[col + j]);
        id += n - col;
        if (eps > 1e-10) return false;
    }
    sgn = s;
    return true;
}

// Normalise a = a / ||a||, sign *= ||a||^2 (linalg/hdsdp_sdpdata.c:880-899).
void normalize_r1(HostCoeff &h) {
    double nrm = 0.0;
    for (double x : h.aval) nrm += x * x;
    nrm = std::sqrt(nrm);
    h.sign *= nrm * nrm;
    for (double &x : h.aval) x /= nrm;
}

}  // namespace

// sdpDenseConeProcDataImpl / sdpSparseConeProcDataImpl (interface/hdsdp_conic_sdp.c:1407-1484):
// a sparse cone keeps the constraints with a nonzero column, counting the others as zero
// coefficients.
hdsdp_retcode SdpCone::proc_data(int nRow, int nCol, const int *Ap, const int *Ai, const double *Ax,
                                 bool sparseCone) {
    n = nCol;
    mAll = nRow;
    sparse = sparseCone;
    rows.clear();
    if (sparse) {
        for (int i = 0; i < nRow; ++i)
            if (Ap[i + 2] - Ap[i + 1] > 0) rows.push_back(i);
    }
    m = sparse ? (int) rows.size() : nRow;
    A.assign(m, HostCoeff());
    refType.assign(m, REF_ZERO);
    for (int k = 0; k < 5; ++k) stats[k] = 0;
    if (sparse) stats[REF_ZERO] = nRow - m;
    const long npack = (long) n * (n + 1) / 2;
    auto load = [&](int col, HostCoeff &h, int &type) -> hdsdp_retcode {
        const int s0 = Ap[col], s1 = Ap[col + 1];
        std::vector<std::pair<long, double>> ent;
        ent.reserve(s1 - s0);
        for (int e = s0; e < s1; ++e) {
            if (Ai[e] < 0 || Ai[e] >= npack) return HDSDP_RETCODE_FAILED;
            ent.push_back({(long) Ai[e], Ax[e]});
        }
        auto less = [](const std::pair<long, double> &x, const std::pair<long, double> &y) {
            return x.first < y.first;
        };
        if (!std::is_sorted(ent.begin(), ent.end(), less)) std::stable_sort(ent.begin(), ent.end(), less);
        const int nnz = (int) ent.size();
        h.r.resize(nnz);
        h.c.resize(nnz);
        h.v.resize(nnz);
        // sorted packed indices: walk the columns instead of searching for each entry
        int jc = 0;
        long colStart = 0, nextStart = n;
        for (int e = 0; e < nnz; ++e) {
            const long q = ent[e].first;
            if (q >= nextStart) {
                unpack(n, q, h.r[e], h.c[e]);
                jc = h.c[e];
                colStart = ((2L * n - jc - 1) * jc) / 2;  // packed index of (i, jc) is colStart + i
                nextStart = colStart + n;                 // first index of column jc + 1
            } else {
                h.c[e] = jc;
                h.r[e] = (int) (q - colStart);
            }
            h.v[e] = ent[e].second;
        }
        // sdpDataMatSetData (linalg/hdsdp_sdpdata.c:2262-2286)
        if (nnz == 0) type = REF_ZERO;
        else if (nnz > 0.3 * npack) {
            type = REF_DENSE;
            h.dense_packed = true;
            h.packed.assign(npack, 0.0);
            for (auto &p : ent) h.packed[p.first] = p.second;
        } else type = REF_SPARSE;
        return HDSDP_RETCODE_OK;
    };
    if (load(0, C, refTypeC) != HDSDP_RETCODE_OK) return HDSDP_RETCODE_FAILED;
    stats[refTypeC] += 1;
    int bad = 0;
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : bad)
    for (int i = 0; i < m; ++i)
        if (load((sparse ? rows[i] : i) + 1, A[i], refType[i]) != HDSDP_RETCODE_OK) bad += 1;
    if (bad) return HDSDP_RETCODE_FAILED;
    for (int i = 0; i < m; ++i) stats[refType[i]] += 1;
    return HDSDP_RETCODE_OK;
}

const double *SdpCone::local(const double *v) {
    if (!sparse || !v) return v;
    ybuf.resize(m);
    for (int i = 0; i < m; ++i) ybuf[i] = v[rows[i]];
    return ybuf.data();
}

// sdpDenseConePresolveImpl (interface/hdsdp_conic_sdp.c:1486-1514): rank-one detection.
hdsdp_retcode SdpCone::presolve() {
    auto eig = [&](HostCoeff &h, int &type) {
        double sgn = 0.0;
        std::vector<double> a;
        bool r1 = false;
        if (type == REF_SPARSE) r1 = sparse_rank_one(n, h.r, h.c, h.v, sgn, a);
        else if (type == REF_DENSE) r1 = dense_rank_one(n, h.packed, sgn, a);
        if (!r1) return;
        int nz = 0;
        for (int q = 0; q < n; ++q)
            if (std::fabs(a[q]) > 1e-10) nz += 1;
        h.sign = sgn;
        h.aidx.clear();
        h.aval.clear();
        if (nz > 0.5 * n) {
            type = REF_DSR1;
            for (int q = 0; q < n; ++q) {
                h.aidx.push_back(q);
                h.aval.push_back(a[q]);
            }
        } else {
            type = REF_SPR1;
            for (int q = 0; q < n; ++q)
                if (std::fabs(a[q]) > 1e-10) {
                    h.aidx.push_back(q);
                    h.aval.push_back(a[q]);
                }
        }
        normalize_r1(h);
    };
    eig(C, refTypeC);
    for (int i = 0; i < m; ++i) stats[refType[i]] -= 1;
#pragma omp parallel for schedule(dynamic, 16)
    for (int i = 0; i < m; ++i) eig(A[i], refType[i]);
    for (int i = 0; i < m; ++i) stats[refType[i]] += 1;
    // device class per row
    for (int i = 0; i < m; ++i) {
        HostCoeff &h = A[i];
        switch (refType[i]) {
            case REF_ZERO: h.cls = CLS_ZERO; break;
            case REF_SPARSE: h.cls = ((int) h.r.size() <= kSpMax) ? CLS_SP : CLS_DR; break;
            case REF_DENSE: h.cls = CLS_DR; break;
            case REF_SPR1: h.cls = ((int) h.aidx.size() <= kR1SmallMax) ? CLS_R1S : CLS_R1D; break;
            case REF_DSR1: h.cls = CLS_R1D; break;
        }
    }
    return HDSDP_RETCODE_OK;
}

static double coeff_norm_of(const HostCoeff &h, int type, int which) {
    double nrm = 0.0;
    if (type == REF_ZERO) return 0.0;
    if (type == REF_SPARSE || type == REF_DENSE) {
        for (size_t e = 0; e < h.v.size(); ++e) {
            const bool diag = h.r[e] == h.c[e];
            if (which == FRO_NORM) nrm += diag ? h.v[e] * h.v[e] : 2.0 * h.v[e] * h.v[e];
            else nrm += diag ? std::fabs(h.v[e]) : 2.0 * std::fabs(h.v[e]);
        }
        return which == FRO_NORM ? std::sqrt(nrm) : nrm;
    }
    // rank one: |sign| * ||a||_2^2 or |sign| * ||a||_1^2 (hdsdp_sdpdata.c:272-309)
    double s2 = 0.0, s1 = 0.0;
    for (double x : h.aval) {
        s2 += x * x;
        s1 += std::fabs(x);
    }
    return which == FRO_NORM ? s2 * std::fabs(h.sign) : s1 * s1 * std::fabs(h.sign);
}

double SdpCone::obj_norm(int type) const { return coeff_norm_of(C, refTypeC, type); }

double SdpCone::coeff_norm(int type) const {
    double nrm = 0.0;
    for (int i = 0; i < m; ++i) {
        double t = coeff_norm_of(A[i], refType[i], type);
        nrm += (type == ABS_NORM) ? t : t * t;
    }
    return (type == ABS_NORM) ? nrm : std::sqrt(nrm);
}

void SdpCone::scal(double a) {
    objScal *= a;
    if (refTypeC == REF_SPR1 || refTypeC == REF_DSR1) C.sign *= a;
}

// sdpDenseConeFeatureDetectImpl (interface/hdsdp_conic_sdp.c:2560-2654)
void SdpCone::detect_feature(const double *rowRHS, int intF[20], double dblF[20]) const {
    intF[15] = stats[REF_ZERO];
    intF[17] = stats[REF_DENSE];
    intF[16] = stats[REF_SPARSE];
    intF[18] = stats[REF_SPR1];
    intF[19] = stats[REF_DSR1];
    auto rank = [&](int i) {
        if (refType[i] == REF_ZERO) return 0;
        if (refType[i] == REF_SPR1 || refType[i] == REF_DSR1) return 1;
        return n;
    };
    bool noPrimalInterior = false;
    for (int i = 0; i < m; ++i)
        if (rank(i) == 1 && std::fabs(rowRHS[i]) < 1e-03 * coeff_norm_of(A[i], refType[i], FRO_NORM))
            noPrimalInterior = true;
    if (noPrimalInterior) intF[2] = 1;

    bool impliedTrace = false;
    double traceX = 0.0;
    for (int i = 0; i < m; ++i) {
        if (refType[i] != REF_SPARSE) continue;
        const HostCoeff &h = A[i];
        if ((int) h.v.size() != n) continue;
        bool eye = true;
        const double d = h.v[0];
        for (size_t e = 0; e < h.v.size(); ++e)
            if (h.r[e] != h.c[e] || h.v[e] != d) { eye = false; break; }
        if (eye && rowRHS[i] / d > 0.0) {
            impliedTrace = true;
            traceX = rowRHS[i] / d;
            break;
        }
    }
    // The reference resets the estimate here before storing it (conic_sdp.c:2622).
    traceX = 0.0;
    std::vector<int> unitCol(std::max(m, n), 0);
    if (!impliedTrace) {
        for (int i = 0; i < m; ++i) {
            const HostCoeff &h = A[i];
            if (refType[i] == REF_SPR1 && h.aidx.size() == 1 && h.aval[0] == 1.0 && h.sign == 1.0 &&
                !unitCol[h.aidx[0]]) {
                unitCol[h.aidx[0]] = 1;
                traceX += rowRHS[i];
            }
        }
    }
    int nSumUnit = 0;
    for (int i = 0; i < m; ++i) nSumUnit += unitCol[i];
    if (nSumUnit == n) impliedTrace = true;
    if (impliedTrace) {
        intF[5] = 1;
        dblF[11] = traceX;
    }
    if (stats[REF_DENSE] >= 0.7 * m) intF[4] = 1;
}

// Pattern of S = C - sum y_i A_i (+ diagonal): neighbour lists from the stored lower
// entries of C and of every A_i. False when it is too dense for a sparse factorisation
// to pay (more than n^2 / 8 off-diagonal entries listed).
static bool slack_pattern(int n, const HostCoeff &C, const std::vector<HostCoeff> &A,
                          std::vector<std::vector<int>> &adj) {
    long total = (long) C.r.size();
    for (const HostCoeff &h : A) total += (long) h.r.size();
    if (total > (long) n * n / 8) return false;
    std::vector<long long> keys;
    keys.reserve(total);
    auto add = [&](const HostCoeff &h) {
        for (size_t e = 0; e < h.r.size(); ++e)
            if (h.r[e] != h.c[e]) keys.push_back((long long) h.r[e] * n + h.c[e]);
    };
    add(C);
    for (const HostCoeff &h : A) add(h);
    std::sort(keys.begin(), keys.end());
    keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
    if ((long) keys.size() > (long) n * n / 8) return false;
    adj.assign(n, {});
    for (long long k : keys) {
        const int a = (int) (k / n), b = (int) (k % n);
        adj[a].push_back(b);
        adj[b].push_back(a);
    }
    for (auto &l : adj) std::sort(l.begin(), l.end());
    return true;
}

hdsdp_retcode SdpCone::setup_device(cudaStream_t stream, Timers *t) {
    s = stream;
    tm = t;
    ld = pad_ld(n);
    // device copy of the (scaled) objective from its lower triplets
    HostCoeff Cdev = C;
    for (double &v : Cdev.v) v *= objScal;
    dev.precision = precision;
    dev.upload(n, m, Cdev, A, s);
    HB_CUDA(hb::cmalloc(&Svar, sizeof(double) * ld * n));
    HB_CUDA(hb::cmalloc(&Scheck, sizeof(double) * ld * n));
    HB_CUDA(hb::cmalloc(&dS, sizeof(double) * ld * n));
    HB_CUDA(hb::cmalloc(&W, sizeof(double) * ld * n));
    HB_CUDA(cudaMemsetAsync(Svar, 0, sizeof(double) * ld * n, s));
    HB_CUDA(cudaMemsetAsync(Scheck, 0, sizeof(double) * ld * n, s));
    HB_CUDA(cudaMemsetAsync(dS, 0, sizeof(double) * ld * n, s));
    Fvar.alloc(n);
    Fcheck.alloc(n);
    facKeepOk = pinVar = false;
    lz.init(n, s);
    hyVar = hyCheck = false;
    if (sparseMode != 0 && (sparseMode == 1 || n >= kHybridMinN)) {
        std::vector<std::vector<int>> adj;
        if (slack_pattern(n, C, A, adj)) {
            hy = new HybridFactor();
            if (hy->analyse(n, adj, kHybridCap, kHybridMaxFront, sparseMode == 1)) {
                hy->upload(s);
            } else {
                hy->release();
                delete hy;
                hy = nullptr;
            }
        }
    }
    if (!hy) Fkeep.alloc(n);   // the kept factor of the accepted point (dense factors only)
    HB_CUDA(hb::cmalloc(&d_y, sizeof(double) * std::max(m, 1)));
    HB_CUDA(hb::cmalloc(&d_vec, sizeof(double) * std::max(m, 1)));
    HB_CUDA(hb::cmalloc(&d_vec2, sizeof(double) * std::max(m, 1)));
    HB_CUDA(hb::cmalloc_host(&h_vec2, sizeof(double) * std::max(m, 1)));
    if (sparse && m > 0) {
        HB_CUDA(hb::cmalloc(&d_rows, sizeof(int) * m));
        HB_CUDA(cudaMemcpyAsync(d_rows, rows.data(), sizeof(int) * m, cudaMemcpyHostToDevice, s));
    }
    HB_CUDA(hb::cmalloc_host(&h_vec, sizeof(double) * std::max(m, 1)));
    HB_CUDA(hb::cmalloc(&d_scal, sizeof(double) * 8));
    HB_CUDA(hb::cmalloc_host(&h_scal, sizeof(double) * 8));
    HB_CUDA(cudaStreamSynchronize(s));
    return device_error_flag() ? HDSDP_RETCODE_MEMORY : HDSDP_RETCODE_OK;
}

void SdpCone::release() {
    dev.release();
    auto f = [](void *p) { if (p) hb::cache_free(p); };
    f(Svar); f(Scheck); f(dS); f(W); f(d_y); f(d_vec); f(d_vec2); f(d_scal); f(d_rows); f(Mown);
    Mown = nullptr;
    if (h_vec) hb::cache_free_host(h_vec);
    if (h_vec2) hb::cache_free_host(h_vec2);
    d_vec2 = h_vec2 = nullptr;
    if (h_scal) hb::cache_free_host(h_scal);
    Svar = Scheck = dS = W = d_y = d_vec = d_scal = h_vec = h_scal = nullptr;
    d_rows = nullptr;
    Fvar.release();
    Fcheck.release();
    Fkeep.release();
    facKeepOk = pinVar = false;
    lz.release();
    if (hy) {
        hy->release();
        delete hy;
        hy = nullptr;
    }
    hyVar = hyCheck = false;
}

// target = dC*C + dAs*sum_i y_i A_i + (dEye [+ perturbation])*I
// (sdpDenseConeIUpdateBuffer, interface/hdsdp_conic_sdp.c:343-402)
// The host part: the buffer `which` (*target) is to hold dC*C + dAs*sum y_i A_i + dEye*I,
// dEye with the cone's perturbation for the slack buffers; false when it holds that already.
// *ly: the cone's coefficient vector (y itself for a dense cone).
bool SdpCone::buffer_plan(double dC, double dAs, const double *y, double &dEye, int which, double **target,
                          const double **ly) {
    y = local(y);
    *ly = y;
    *target = (which == BUFFER_DUALVAR) ? Svar : (which == BUFFER_DUALCHECK) ? Scheck : dS;
    if (which == BUFFER_DUALSTEP) return true;
    dEye += dualPerturb;
    SlackSig &sig = (which == BUFFER_DUALVAR) ? sigVar : sigCheck;
    SlackSig next;
    next.valid = true;
    next.dC = dC;
    next.dAs = dAs;
    next.dEye = dEye;
    next.y.assign(y, y + m);
    if (sig.same(next)) return false;  // the buffer already holds exactly this matrix
    sig = std::move(next);
    return true;
}

void SdpCone::update_buffer(double dC, double dAs, const double *y, double dEye, int which) {
    double t0 = wall();
    double *target = nullptr;
    const double *ly = nullptr;
    if (buffer_plan(dC, dAs, y, dEye, which, &target, &ly)) {
        std::memcpy(h_vec, ly, sizeof(double) * m);
        HB_CUDA(cudaMemcpyAsync(d_y, h_vec, sizeof(double) * m, cudaMemcpyHostToDevice, s));
        dev.assemble(dC, dAs, d_y, dEye, target, ld);
    }
    if (tm) tm->assemble += wall() - t0;
}

namespace {
// S assembly of several small cones whose coefficients all sit in the gather map (no dense
// rank-one or dense class), one CTA each: s_init_kernel's and s_gather_kernel's arithmetic
// in one launch, the coefficients read from the problem's vector through the cone's rows.
struct AsmJob {
    const double *C;
    double *S;
    const int *pr, *pc, *ptr, *ej, *rows;
    const double *ev;
    long ldc, lds;
    double dEye;
    int n, npos;
};
constexpr int kAsmBatch = 32;
constexpr int kAsmBatchMaxN = 128;
struct AsmBatch {
    AsmJob job[kAsmBatch];
};

__global__ void s_assemble_batch_kernel(const AsmBatch B, const double *__restrict__ y, double dC, double dA) {
    const AsmJob &J = B.job[blockIdx.x];
    const int n = J.n;
    const long total = (long) n * n;
    for (long idx = threadIdx.x; idx < total; idx += blockDim.x) {
        const int r = (int) (idx % n), c = (int) (idx / n);
        double v = (dC != 0.0) ? dC * J.C[(size_t) r + (size_t) c * J.ldc] : 0.0;
        if (r == c) v += J.dEye;
        J.S[(size_t) r + (size_t) c * J.lds] = v;
    }
    if (dA == 0.0) return;
    __syncthreads();
    for (int p = threadIdx.x; p < J.npos; p += blockDim.x) {
        double acc = 0.0;
        for (int e = J.ptr[p]; e < J.ptr[p + 1]; ++e) {
            const int j = J.ej[e];
            acc += J.ev[e] * y[J.rows ? J.rows[j] : j];
        }
        acc *= dA;
        const int r = J.pr[p], c = J.pc[p];
        J.S[(size_t) r + (size_t) c * J.lds] += acc;
        if (r != c) J.S[(size_t) c + (size_t) r * J.lds] += acc;
    }
}
}  // namespace

// update_buffer for several cones (one stream): one upload of y (problem order, mAll) into
// d_yall (device, pinned staging h_yall), the small gather-map cones assembled in shared
// launches, the others one by one; every buffer gets the values update_buffer gives it.
void assemble_buffers(const std::vector<SdpCone *> &cones, double dC, double dAs, const double *y,
                      const std::vector<double> &dEye, int which, double *d_yall, double *h_yall) {
    if (cones.empty()) return;
    const double t0 = wall();
    cudaStream_t s = cones[0]->s;
    Timers *tm = cones[0]->tm;
    std::vector<AsmJob> jobs;
    bool uploaded = false;
    for (size_t q = 0; q < cones.size(); ++q) {
        SdpCone *c = cones[q];
        double e = dEye[q], *target = nullptr;
        const double *ly = nullptr;
        if (!c->buffer_plan(dC, dAs, y, e, which, &target, &ly)) continue;
        const SdpDevice &d = c->dev;
        if (c->n <= kAsmBatchMaxN && (dAs == 0.0 || (d.nr1d == 0 && d.ndr == 0))) {
            if (!uploaded) {
                std::memcpy(h_yall, y, sizeof(double) * c->mAll);
                HB_CUDA(cudaMemcpyAsync(d_yall, h_yall, sizeof(double) * c->mAll, cudaMemcpyHostToDevice, s));
                uploaded = true;
            }
            jobs.push_back(AsmJob{d.Cfull, target, d.pos_r, d.pos_c, d.pos_ptr, d.ent_j, c->sparse ? c->d_rows : nullptr,
                                  d.ent_v, d.ld, c->ld, e, c->n, d.npos});
        } else {
            std::memcpy(c->h_vec, ly, sizeof(double) * c->m);
            HB_CUDA(cudaMemcpyAsync(c->d_y, c->h_vec, sizeof(double) * c->m, cudaMemcpyHostToDevice, s));
            c->dev.assemble(dC, dAs, c->d_y, e, target, c->ld);
        }
    }
    for (size_t b0 = 0; b0 < jobs.size(); b0 += kAsmBatch) {
        const int nb = (int) std::min<size_t>(kAsmBatch, jobs.size() - b0);
        AsmBatch B;
        for (int q = 0; q < nb; ++q) B.job[q] = jobs[b0 + q];
        s_assemble_batch_kernel<<<counted(nb), 256, 0, s>>>(B, d_yall, dC, dAs);
        HB_CUDA(cudaGetLastError());
    }
    if (tm) tm->assemble += wall() - t0;
}

static void copy_factor(cudaStream_t s, DenseFactor &dst, const DenseFactor &src) {
    HB_CUDA(cudaMemcpyAsync(dst.L, src.L, sizeof(double) * src.ld * src.n, cudaMemcpyDeviceToDevice, s));
    HB_CUDA(cudaMemcpyAsync(dst.Dinv, src.Dinv, sizeof(double) * src.ld * 64, cudaMemcpyDeviceToDevice, s));
    dst.k_valid = false;
    if (src.k_valid && src.K && src.KT) {
        if (!dst.K) HB_CUDA(hb::cmalloc(&dst.K, sizeof(double) * dst.ld * dst.n));
        if (!dst.KT) HB_CUDA(hb::cmalloc(&dst.KT, sizeof(double) * dst.ld * dst.n));
        HB_CUDA(cudaMemcpyAsync(dst.K, src.K, sizeof(double) * src.ld * src.n, cudaMemcpyDeviceToDevice, s));
        HB_CUDA(cudaMemcpyAsync(dst.KT, src.KT, sizeof(double) * src.ld * src.n, cudaMemcpyDeviceToDevice, s));
        dst.k_valid = true;
    }
    dst.factored = true;
    dst.ok = src.ok;
    dst.logdet_valid = src.logdet_valid;
    dst.logdet = src.logdet;
}

hdsdp_retcode SdpCone::update(double tau, const double *y) {
    update_buffer(tau, -1.0, y, -dualResidual, BUFFER_DUALVAR);
    return HDSDP_RETCODE_OK;
}

static bool timed_factor(cudaStream_t s, DenseFactor &F, const double *S, long ld, Timers *tm) {
    double t0 = wall();
    bool ok = factorize(s, F, S, ld);
    if (tm) {
        tm->s_factor += wall() - t0;
        tm->n_sfactor += 1;
    }
    return ok;
}

void SdpCone::keep_var() {
    if (Fkeep.L && pinVar && facVarOk && facVar.valid) {
        std::swap(Fvar, Fkeep);
        facKeep = facVar;
        facKeepOk = true;
    }
    pinVar = false;
}

bool SdpCone::restore_var() {
    if (!Fkeep.L || !facKeepOk || !sigVar.same(facKeep)) return false;
    std::swap(Fvar, Fkeep);
    std::swap(facVar, facKeep);
    std::swap(facVarOk, facKeepOk);
    hyVar = false;
    pinVar = true;
    ++nFactorReuse;
    return true;
}

bool SdpCone::factor_buffer(int which) {
    const bool var = (which == BUFFER_DUALVAR);
    DenseFactor &F = var ? Fvar : Fcheck;
    const SlackSig &sig = var ? sigVar : sigCheck;
    SlackSig &fsig = var ? facVar : facCheck;
    bool &fok = var ? facVarOk : facCheckOk;
    const SlackSig &osig = var ? facCheck : facVar;
    const bool ook = var ? facCheckOk : facVarOk;
    if (sig.same(fsig)) {
        ++nFactorReuse;
        return fok;
    }
    if (var && restore_var()) return facVarOk;
    if (sig.same(osig) && ook) {
        if (var ? hyCheck : hyVar) {
            // the other object holds a hybrid result for the same matrix
            (var ? hyVar : hyCheck) = true;
            (var ? hyLogdetVar : hyLogdetCheck) = var ? hyLogdetCheck : hyLogdetVar;
            (var ? hySeqVar : hySeqCheck) = var ? hySeqCheck : hySeqVar;
            F.factored = F.ok = true;
            F.k_valid = false;
        } else {
            if (var) keep_var();
            copy_factor(s, F, var ? Fcheck : Fvar);
            (var ? hyVar : hyCheck) = false;
        }
        fsig = sig;
        fok = true;
        ++nFactorReuse;
        return true;
    }
    if (var) keep_var();
    const bool ok = use_hybrid(which) ? hybrid_factor(which) : timed_factor(s, F, var ? Svar : Scheck, ld, tm);
    if (!use_hybrid(which)) (var ? hyVar : hyCheck) = false;
    fsig = sig;
    fok = ok;
    return ok;
}

// factor_buffer in two phases, for several cones at once: factor_plan() settles what
// factor_buffer would do without waiting for the device. FP_DONE: the result is known
// (*ok); FP_SMALL: a dense factorisation of order <= kBatchFactorMaxN, to be enqueued by
// the caller with the other cones' (factorize_small_batch); FP_ASYNC: enqueued here.
// factor_finish() then reads the status of an FP_SMALL or FP_ASYNC factorisation.
int SdpCone::factor_plan(int which, bool *ok) {
    const bool var = (which == BUFFER_DUALVAR);
    const SlackSig &sig = var ? sigVar : sigCheck;
    const SlackSig &fsig = var ? facVar : facCheck;
    const SlackSig &osig = var ? facCheck : facVar;
    const bool ook = var ? facCheckOk : facVarOk;
    if (sig.same(fsig) || (var && Fkeep.L && facKeepOk && sig.same(facKeep)) || (sig.same(osig) && ook) ||
        use_hybrid(which)) {
        *ok = factor_buffer(which);   // reuse, the kept factor, copy or the hybrid factorisation
        return FP_DONE;
    }
    if (var) keep_var();
    if (n <= kBatchFactorMaxN) return FP_SMALL;
    factorize_async(s, var ? Fvar : Fcheck, var ? Svar : Scheck, ld);
    return FP_ASYNC;
}

bool SdpCone::factor_finish(int which, bool synced) {
    const bool var = (which == BUFFER_DUALVAR);
    DenseFactor &F = var ? Fvar : Fcheck;
    const bool ok = synced ? factor_status_ready(F) : factor_status(s, F);
    (var ? hyVar : hyCheck) = false;
    (var ? facVar : facCheck) = var ? sigVar : sigCheck;
    (var ? facVarOk : facCheckOk) = ok;
    if (tm) tm->n_sfactor += 1;
    return ok;
}

// The buffer `which` of every cone of `cones` factored as factor_buffer does, with the
// dense factorisations of small blocks in one batched launch and one wait for all.
void factor_buffers(const std::vector<SdpCone *> &cones, int which, std::vector<char> &ok) {
    const double t0 = wall();
    ok.assign(cones.size(), 0);
    std::vector<int> plan(cones.size(), 0);
    std::vector<DenseFactor *> F;
    std::vector<const double *> S;
    std::vector<long> ldS;
    const bool var = (which == BUFFER_DUALVAR);
    Timers *tm = nullptr;
    for (size_t q = 0; q < cones.size(); ++q) {
        SdpCone &c = *cones[q];
        bool r = false;
        plan[q] = c.factor_plan(which, &r);
        ok[q] = r ? 1 : 0;
        if (plan[q] == SdpCone::FP_SMALL) {
            F.push_back(var ? &c.Fvar : &c.Fcheck);
            S.push_back(var ? c.Svar : c.Scheck);
            ldS.push_back(c.ld);
        }
        if (c.tm) tm = c.tm;
    }
    if (!F.empty()) factorize_small_batch(cones[0]->s, F.data(), S.data(), ldS.data(), (int) F.size());
    HB_CUDA(cudaStreamSynchronize(cones[0]->s));
    for (size_t q = 0; q < cones.size(); ++q)
        if (plan[q] != SdpCone::FP_DONE) ok[q] = cones[q]->factor_finish(which, true) ? 1 : 0;
    if (tm) tm->s_factor += wall() - t0;
}

// Positive-definiteness and log det of the buffer `which` through the hybrid factor.
bool SdpCone::hybrid_factor(int which) {
    const bool var = (which == BUFFER_DUALVAR);
    const double t0 = wall();
    hy->factor_async(s, var ? Svar : Scheck, ld);
    double logdet = 0.0;
    const bool ok = hy->finish(s, &logdet);
    DenseFactor &F = var ? Fvar : Fcheck;
    F.factored = true;
    F.ok = ok;
    F.k_valid = false;
    (var ? hyVar : hyCheck) = true;
    (var ? hyLogdetVar : hyLogdetCheck) = logdet;
    (var ? hySeqVar : hySeqCheck) = hy->seq;
    ++nHybrid;
    if (!var) ++nHybridCheck;
    if (tm) {
        tm->s_factor += wall() - t0;
        tm->n_sfactor += 1;
    }
    return ok;
}

// The dense factor of the buffer `which` in Fvar / Fcheck, formed now if the last
// factorisation of it was a hybrid one.
bool SdpCone::ensure_dense(int which) {
    const bool var = (which == BUFFER_DUALVAR);
    bool &h = var ? hyVar : hyCheck;
    DenseFactor &F = var ? Fvar : Fcheck;
    if (!h) return F.ok;
    const bool ok = timed_factor(s, F, var ? Svar : Scheck, ld, tm);
    h = false;
    ++nDenseAfter[var ? 0 : 1];
    return ok;
}

hdsdp_retcode SdpCone::ratio_test(double dtau, const double *dy, double ada, int which, double *step) {
    update_buffer(dtau, -1.0, dy, ada * dualResidual, BUFFER_DUALSTEP);
    DenseFactor &F = (which == BUFFER_DUALVAR) ? Fvar : Fcheck;
    if (n == 1) {
        double vals[2];
        HB_CUDA(cudaMemcpyAsync(&vals[0], dS, sizeof(double), cudaMemcpyDeviceToHost, s));
        HB_CUDA(cudaMemcpyAsync(&vals[1], (which == BUFFER_DUALVAR) ? Svar : Scheck, sizeof(double),
                                cudaMemcpyDeviceToHost, s));
        HB_CUDA(cudaStreamSynchronize(s));
        *step = (vals[0] > 0.0) ? HDSDP_INFINITY : (-vals[1] / vals[0]);
        return HDSDP_RETCODE_OK;
    }
    const bool var = (which == BUFFER_DUALVAR);
    if (hy && (var ? hyVar : hyCheck) && (var ? hySeqVar : hySeqCheck) == hy->seq) {
        // the sparse factor of this buffer is the one held: the step bound runs on it
        lz.hyOp = hy;
        const hdsdp_retcode r = lz.solve(F, dS, ld, step, tm);
        lz.hyOp = nullptr;
        return r;
    }
    if (hy && !ensure_dense(var ? BUFFER_DUALVAR : BUFFER_DUALCHECK)) return HDSDP_RETCODE_FAILED;
    return lz.solve(F, dS, ld, step, tm);
}

hdsdp_retcode SdpCone::interior_check(double tau, const double *y, int *interior) {
    update(tau, y);
    *interior = factor_buffer(BUFFER_DUALVAR) ? 1 : 0;
    return device_error_flag() ? HDSDP_RETCODE_FAILED : HDSDP_RETCODE_OK;
}

hdsdp_retcode SdpCone::interior_check_expert(double dC, double dAs, const double *y, double dEye, int which,
                                             int *interior) {
    update_buffer(dC, dAs, y, dEye, which);
    *interior = factor_buffer(which == BUFFER_DUALVAR ? BUFFER_DUALVAR : BUFFER_DUALCHECK) ? 1 : 0;
    return device_error_flag() ? HDSDP_RETCODE_FAILED : HDSDP_RETCODE_OK;
}

hdsdp_retcode SdpCone::get_barrier(double tau, const double *y, int which, double *logdet) {
    DenseFactor &F = (which == BUFFER_DUALVAR) ? Fvar : Fcheck;
    if (y) {
        update(tau, y);
        if (!factor_buffer(BUFFER_DUALVAR)) return HDSDP_RETCODE_FAILED;
    }
    if (which == BUFFER_DUALVAR ? hyVar : hyCheck) {
        *logdet = (which == BUFFER_DUALVAR) ? hyLogdetVar : hyLogdetCheck;
        return HDSDP_RETCODE_OK;
    }
    if (F.logdet_valid) {   // read back with the factorisation's status
        *logdet = F.logdet;
        return HDSDP_RETCODE_OK;
    }
    log_diag_sum(s, F, d_scal);
    HB_CUDA(cudaMemcpyAsync(h_scal, d_scal, sizeof(double), cudaMemcpyDeviceToHost, s));
    HB_CUDA(cudaStreamSynchronize(s));
    *logdet = 2.0 * h_scal[0];
    return HDSDP_RETCODE_OK;
}

void SdpCone::add_step(double step, int which) {
    if (which == BUFFER_DUALVAR) {
        keep_var();
        axpy(s, (int) (ld * n), step, dS, Svar);
        sigVar.valid = false;
        facVar.valid = false;
    } else {
        HB_CUDA(cudaMemcpyAsync(Scheck, Svar, sizeof(double) * ld * n, cudaMemcpyDeviceToDevice, s));
        axpy(s, (int) (ld * n), step, dS, Scheck);
        sigCheck.valid = false;
        facCheck.valid = false;
    }
}

hdsdp_retcode SdpCone::add_step_and_check(double step, int which, int *interior) {
    if (which == BUFFER_DUALVAR) {
        keep_var();
        axpy(s, (int) (ld * n), step, dS, Svar);
        sigVar.valid = false;
        facVar.valid = false;
        facVarOk = use_hybrid(BUFFER_DUALVAR) ? hybrid_factor(BUFFER_DUALVAR) : timed_factor(s, Fvar, Svar, ld, tm);
        if (!use_hybrid(BUFFER_DUALVAR)) hyVar = false;
        *interior = facVarOk ? 1 : 0;
    } else {
        HB_CUDA(cudaMemcpyAsync(Scheck, Svar, sizeof(double) * ld * n, cudaMemcpyDeviceToDevice, s));
        axpy(s, (int) (ld * n), step, dS, Scheck);
        sigCheck.valid = false;
        facCheck.valid = false;
        facCheckOk = use_hybrid(BUFFER_DUALCHECK) ? hybrid_factor(BUFFER_DUALCHECK)
                                                  : timed_factor(s, Fcheck, Scheck, ld, tm);
        if (!use_hybrid(BUFFER_DUALCHECK)) hyCheck = false;
        *interior = facCheckOk ? 1 : 0;
    }
    return device_error_flag() ? HDSDP_RETCODE_FAILED : HDSDP_RETCODE_OK;
}

// X = mu * (S^-1 + S^-1 (A^* dy) S^-1) at S = C - A^T y (+ perturbation), computed as
// mu * K^T (K dS K^T + I) K with K = L^-1 (sdpDenseConeGetPrimal, conic_sdp.c:2328-2379).
void SdpCone::get_primal(double mu, const double *y, const double *dy, double *X) {
    double t0 = wall();
    int interior = 0;
    interior_check_expert(1.0, -1.0, y, 0.0, BUFFER_DUALCHECK, &interior);
    if (!interior) {
        printf("Recovery step is infeasible\n");
        return;
    }
    if (hy && !ensure_dense(BUFFER_DUALCHECK)) {
        printf("Recovery step is infeasible\n");
        return;
    }
    update_buffer(0.0, 1.0, dy, 0.0, BUFFER_DUALSTEP);
    compute_inverse_factor(s, Fcheck);
    double *T1 = dev.T1, *T2 = dev.T2;
    const double *K = Fcheck.K;
    gemm(s, n, n, n, 1.0, K, ld, 0, dS, ld, 0, 0.0, T1, ld, GEMM_A_LOWER);                    // K dS
    gemm(s, n, n, n, 1.0, T1, ld, 0, K, ld, 1, 0.0, T2, ld, GEMM_B_UPPER);                    // (K dS) K^T
    add_diag(s, n, T2, ld, 1.0);
    symmetrize_avg(s, n, T2, ld);
    gemm(s, n, n, n, 1.0, T2, ld, 0, K, ld, 0, 0.0, T1, ld, GEMM_B_LOWER);                    // T2 K
    gemm(s, n, n, n, mu, K, ld, 1, T1, ld, 0, 0.0, X, ld, GEMM_A_UPPER);                      // K^T T2 K
    symmetrize_avg(s, n, X, ld);
    HB_CUDA(cudaStreamSynchronize(s));
    if (tm) tm->primal += wall() - t0;
}

void SdpCone::get_dual(double *S) {
    HB_CUDA(cudaMemcpyAsync(S, Svar, sizeof(double) * ld * n, cudaMemcpyDeviceToDevice, s));
}

void SdpCone::atimesx(const double *X, double *out) {
    if (m == 0) return;
    dev.inner_all(X, ld, d_vec);
    HB_CUDA(cudaMemcpyAsync(h_vec, d_vec, sizeof(double) * m, cudaMemcpyDeviceToHost, s));
    HB_CUDA(cudaStreamSynchronize(s));
    for (int i = 0; i < m; ++i) out[sparse ? rows[i] : i] += h_vec[i];
}

double SdpCone::trace_cx(const double *X) { return dev.c_inner(X, ld); }

// ======================================================================================
// Scalar bound cone (interface/hdsdp_conic_bound.c)
// ======================================================================================
void BoundCone::proc(int m_, double l, double u) {
    m = m_;
    lo = l;
    up = u;
    for (auto *v : {&dl, &du, &dlInv, &duInv, &dlStep, &duStep, &dlChk, &duChk}) v->assign(m, 0.0);
}

void BoundCone::update_buffer(double dC, double dAs, const double *y, int which) {
    std::vector<double> &L = (which == BUFFER_DUALVAR) ? dl : (which == BUFFER_DUALCHECK) ? dlChk : dlStep;
    std::vector<double> &U = (which == BUFFER_DUALVAR) ? du : (which == BUFFER_DUALCHECK) ? duChk : duStep;
    for (int i = 0; i < m; ++i) {
        U[i] = dC * up + dAs * y[i];
        L[i] = -dC * lo - dAs * y[i];
    }
}

double BoundCone::ratio_test(double dtau, const double *dy, int which) {
    update_buffer(dtau, -1.0, dy, BUFFER_DUALSTEP);
    const std::vector<double> &L = (which == BUFFER_DUALVAR) ? dl : dlChk;
    const std::vector<double> &U = (which == BUFFER_DUALVAR) ? du : duChk;
    double mx = 0.0;
    for (int i = 0; i < m; ++i) {
        mx = std::min(mx, dlStep[i] / L[i]);
        mx = std::min(mx, duStep[i] / U[i]);
    }
    mx = 1.0 / mx;
    return (mx > 0.0) ? 100.0 : -mx;
}

int BoundCone::interior_check(double tau, const double *y) {
    update(tau, y);
    for (int i = 0; i < m; ++i)
        if (dl[i] <= 0.0) return 0;
    for (int i = 0; i < m; ++i)
        if (du[i] <= 0.0) return 0;
    return 1;
}

int BoundCone::interior_check_expert(double dC, double dAs, const double *y, int which) {
    update_buffer(dC, dAs, y, which);
    const std::vector<double> &L = (which == BUFFER_DUALVAR) ? dl : dlChk;
    const std::vector<double> &U = (which == BUFFER_DUALVAR) ? du : duChk;
    for (int i = 0; i < m; ++i)
        if (L[i] <= 0.0) return 0;
    for (int i = 0; i < m; ++i)
        if (U[i] <= 0.0) return 0;
    return 1;
}

hdsdp_retcode BoundCone::get_barrier(double tau, const double *y, int which, double *logdet) {
    const std::vector<double> &L = (which == BUFFER_DUALVAR) ? dl : dlChk;
    const std::vector<double> &U = (which == BUFFER_DUALVAR) ? du : duChk;
    if (y) update(tau, y);
    double ld = 0.0;
    for (int i = 0; i < m; ++i) ld += std::log(L[i]) + std::log(U[i]);
    if (ld != ld) {
        printf("Bound constraint is violated\n");
        return HDSDP_RETCODE_FAILED;
    }
    *logdet = ld;
    return HDSDP_RETCODE_OK;
}

int BoundCone::add_step_and_check(double step, int which) {
    std::vector<double> &L = (which == BUFFER_DUALVAR) ? dl : dlChk;
    std::vector<double> &U = (which == BUFFER_DUALVAR) ? du : duChk;
    if (which != BUFFER_DUALVAR) {
        dlChk = dl;
        duChk = du;
    }
    for (int i = 0; i < m; ++i) {
        L[i] += step * dlStep[i];
        U[i] += step * duStep[i];
        if (L[i] <= 0.0 || U[i] <= 0.0) return 0;
    }
    return 1;
}

void BoundCone::get_primal(double mu, const double *y, const double *dy, double *lower, double *upper) const {
    for (int i = 0; i < m; ++i) {
        const double st = -dy[i];
        const double su = up - y[i];
        const double sl = y[i] - lo;
        lower[i] = mu * (1.0 / sl - st / (sl * sl));
        upper[i] = mu * (1.0 / su + st / (su * su));
    }
}

// ======================================================================================
// Schur complement system
// ======================================================================================
void KKT::init(int m_, cudaStream_t stream, Timers *t, bool denseM) {
    m = m_;
    s = stream;
    tm = t;
    ldm = pad_ld(m);
    if (denseM) {
        HB_CUDA(hb::cmalloc(&M, sizeof(double) * ldm * m));
        HB_CUDA(cudaMemsetAsync(M, 0, sizeof(double) * ldm * m, s));
        F.alloc(m, m < kTriSolveMinM ? 1 : 0);
        F.kfamily = KF_POTRF_SCHUR;
    }
    asinv.assign(m, 0.0);
    asinvrd.assign(m, 0.0);
    asinvcs.assign(m, 0.0);
    diag_add.assign(m, 0.0);
    for (double **p : {&d_rhs, &d_x, &d_r, &d_t, &d_diag}) HB_CUDA(hb::cmalloc(p, sizeof(double) * m));
    HB_CUDA(hb::cmalloc_host(&h_buf, sizeof(double) * m));
}

void KKT::release() {
    release_arrow();
    if (d_wdesc) hb::cache_free(d_wdesc);
    if (d_jobs) hb::cache_free(d_jobs);
    d_wdesc = nullptr;
    d_jobs = nullptr;
    fusedCap = 0;
    if (M) hb::cache_free(M);
    M = nullptr;
    if (Msub) hb::cache_free(Msub);
    Msub = nullptr;
    msubCap = 0;
    F.release();
    ldl.release();
    ldlActive = false;
    for (double **p : {&d_rhs, &d_x, &d_r, &d_t, &d_diag}) {
        if (*p) hb::cache_free(*p);
        *p = nullptr;
    }
    if (h_buf) hb::cache_free_host(h_buf);
    h_buf = nullptr;
}

void KKT::clean(int type) {
    std::fill(asinv.begin(), asinv.end(), 0.0);
    std::fill(asinvrd.begin(), asinvrd.end(), 0.0);
    if (type == KKT_TYPE_HOMOGENEOUS) {
        std::fill(asinvcs.begin(), asinvcs.end(), 0.0);
        dCSinv = dCSinvCSinv = dCSinvRdSinv = 0.0;
    }
    dTraceSinv = 0.0;
    // HKKTClean (interface/hdsdp_schur.c:141-164): these builds form M anew
    if (type == KKT_TYPE_INFEASIBLE || type == KKT_TYPE_HOMOGENEOUS || type == KKT_TYPE_PRIMAL) mOpen = false;
}

void KKT::open_m() {
    if (arrow) return arrow_open();
    if (mOpen) return;
    HB_CUDA(cudaMemsetAsync(M, 0, sizeof(double) * ldm * m, s));
    mOpen = true;
}

// M[rows[i], rows[j]] += B[i, j] over the lower triangle i >= j of a cone's Schur block
// (rows == nullptr: the identity). rows increases, so the lower triangle of B lands in the
// lower triangle of M.
__global__ void scatter_lower_kernel(int mk, const double *__restrict__ B, long ldb, const int *__restrict__ rows,
                                     double *__restrict__ M, long ldm) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    for (int j = blockIdx.y * blockDim.y + threadIdx.y; j < mk; j += gridDim.y * blockDim.y) {
        if (i < j || i >= mk) continue;
        const long gi = rows ? rows[i] : i, gj = rows ? rows[j] : j;
        M[gi + gj * ldm] += B[i + (long) j * ldb];
    }
}

// dst[rows[i]] += scale * d_src[i] (rows == nullptr: the identity)
static void add_host(std::vector<double> &dst, const double *d_src, double *h_buf, int m, double scale,
                     cudaStream_t s, const std::vector<int> *rows = nullptr) {
    if (m == 0) return;
    HB_CUDA(cudaMemcpyAsync(h_buf, d_src, sizeof(double) * m, cudaMemcpyDeviceToHost, s));
    HB_CUDA(cudaStreamSynchronize(s));
    if (rows)
        for (int i = 0; i < m; ++i) dst[(*rows)[i]] += scale * h_buf[i];
    else
        for (int i = 0; i < m; ++i) dst[i] += scale * h_buf[i];
}

// Smallest block order for which split precision also forms S^-1 on the tensor cores
// (the n^3/3 product; below it the FP64 product takes tens of microseconds).
constexpr int kSplitInverseMinN = 1024;

// sdpDenseConeGetKKT / GetKKTByFixedStrategy (interface/hdsdp_conic_sdp.c:1722-1872)
// (interface/hdsdp_conic_sdp.c:1874-1938 for a sparse cone): adds the cone's terms to M and
// to the right-hand-side vectors of the build that clean() opened.
hdsdp_retcode KKT::add_sdp(SdpCone &cone, int type) {
    double t0 = wall();
    const int n = cone.n;
    const std::vector<int> *rows = cone.sparse ? &cone.rows : nullptr;
    const long ld = cone.ld;
    const double r = cone.dualResidual;
    const double *Wp = nullptr;
    if (type == KKT_TYPE_PRIMAL) {
        if (!primalX) return HDSDP_RETCODE_FAILED;
        Wp = primalX;
    } else {
        if (cone.hy && !cone.ensure_dense(BUFFER_DUALVAR)) return HDSDP_RETCODE_FAILED;
        double ti = wall();
        // split precision: W = K^T K on the tensor cores once n makes the product worth it
        bool done = false;
        if (cone.dev.precision == 1 && n >= kSplitInverseMinN) {
            compute_inverse_factor(s, cone.Fvar);
            done = cone.dev.split_inverse(cone.Fvar.K, cone.W, ld);
        }
        if (!done) compute_inverse(s, cone.Fvar, cone.W, ld);
        if (tm) {
            HB_CUDA(cudaStreamSynchronize(s));
            tm->s_inverse += wall() - ti;
        }
        Wp = cone.W;
        cone.pinVar = true;   // the accepted point's factor
    }
    SdpDevice &dev = cone.dev;
    if (type == KKT_TYPE_CORRECTOR) {
        dev.inner_all(Wp, ld, cone.d_vec);
        add_host(asinv, cone.d_vec, h_buf, cone.m, 1.0, s, rows);
        if (r != 0.0) {
            dev.inner_all_sq(Wp, ld, cone.d_vec, false, true);
            add_host(asinvrd, cone.d_vec, h_buf, cone.m, r, s, rows);
        }
        if (tm) tm->schur += wall() - t0;
        return device_error_flag() ? HDSDP_RETCODE_FAILED : HDSDP_RETCODE_OK;
    }
    if (r != 0.0) {
        trace(s, n, Wp, ld, cone.d_scal);
        HB_CUDA(cudaMemcpyAsync(cone.h_scal, cone.d_scal, sizeof(double), cudaMemcpyDeviceToHost, s));
        HB_CUDA(cudaStreamSynchronize(s));
        dTraceSinv += cone.h_scal[0];
    }
    double tq = wall();
    if (!rows && !mOpen) {
        // the first contribution, from a cone holding every constraint: written outright
        dev.schur_matrix(Wp, ld, M, ldm, (type == KKT_TYPE_PRIMAL) ? nullptr : cone.Fvar.K);
        mOpen = true;
    } else if (cone.m > 0) {
        open_m();
        const int mk = cone.m;
        const long ldk = pad_ld(mk);
        if (msubCap < (size_t) ldk * mk) {
            if (Msub) hb::cache_free(Msub);
            msubCap = (size_t) ldk * mk;
            HB_CUDA(hb::cmalloc(&Msub, sizeof(double) * msubCap));
        }
        dev.schur_matrix(Wp, ld, Msub, ldk, (type == KKT_TYPE_PRIMAL) ? nullptr : cone.Fvar.K);
        if (arrow) {
            arrow_add(cone, Msub, ldk);
        } else {
            dim3 blk(32, 8), grd((mk + 31) / 32, std::min((mk + 7) / 8, 4096));
            scatter_lower_kernel<<<hb::counted(grd), blk, 0, s>>>(mk, Msub, ldk, cone.d_rows, M, ldm);
            HB_CUDA(cudaGetLastError());
        }
    }
    if (tm) {
        HB_CUDA(cudaStreamSynchronize(s));
        tm->sch_matrix += wall() - tq;
        tq = wall();
    }
    dev.inner_all(Wp, ld, cone.d_vec, true);
    add_host(asinv, cone.d_vec, h_buf, cone.m, 1.0, s, rows);
    if (tm) {
        tm->sch_inner += wall() - tq;
        tq = wall();
    }
    if (r != 0.0) {
        dev.inner_all_sq(Wp, ld, cone.d_vec, true);
        add_host(asinvrd, cone.d_vec, h_buf, cone.m, r, s, rows);
    }
    if (tm) tm->sch_innersq += wall() - tq;
    if (type == KKT_TYPE_HOMOGENEOUS) {
        // B = W C W; <A_i, B>, <C, W>, <C, B>, r * tr(B)
        gemm(s, n, n, n, 1.0, dev.Cfull, dev.ld, 0, Wp, ld, 0, 0.0, dev.T1, dev.ld, 0);
        gemm(s, n, n, n, 1.0, Wp, ld, 0, dev.T1, dev.ld, 0, 0.0, dev.T2, dev.ld, 0);
        symmetrize_avg(s, n, dev.T2, dev.ld);
        dev.inner_all(dev.T2, dev.ld, cone.d_vec);
        add_host(asinvcs, cone.d_vec, h_buf, cone.m, 1.0, s, rows);
        dCSinv += dev.c_inner(Wp, ld);
        dCSinvCSinv += dev.c_inner(dev.T2, dev.ld);
        if (r != 0.0) {
            trace(s, n, dev.T2, dev.ld, cone.d_scal);
            HB_CUDA(cudaMemcpyAsync(cone.h_scal, cone.d_scal, sizeof(double), cudaMemcpyDeviceToHost, s));
            HB_CUDA(cudaStreamSynchronize(s));
            dCSinvRdSinv += r * cone.h_scal[0];
        }
    }
    HB_CUDA(cudaStreamSynchronize(s));
    if (tm) {
        tm->schur += wall() - t0;
        tm->n_schur += 1;
    }
    return device_error_flag() ? HDSDP_RETCODE_FAILED : HDSDP_RETCODE_OK;
}

// cones whose Schur build runs in the fused per-cone kernel
constexpr int kFusedBuildMaxN = 512;
constexpr int kFusedBuildMaxM = 1024;

// add_sdp for every cone of `cones` (a build of type KKT_TYPE_INFEASIBLE or
// KKT_TYPE_CORRECTOR, the cones in the user's order): all device work is enqueued first,
// each cone's vectors and trace come back into its own pinned buffers, and after one wait
// the host sums are formed in the cones' order, with the operations add_sdp uses, so the
// result is the same to the bit.
hdsdp_retcode KKT::add_sdp_batch(const std::vector<SdpCone *> &cones, int type) {
    const double t0 = wall();
    const bool corr = (type == KKT_TYPE_CORRECTOR);
    // Cones of the sparse and sparse rank-one classes only (FP64, no sparse slack factor,
    // moderate size) are built together: every W = K^T K in one grouped GEMM, then one CTA per
    // cone forms its Schur block (into its own scratch), <A_i, W>, <A_i, W^2> and tr W, the
    // vectors written straight into the cone's pinned host buffers.
    std::vector<char> fused(cones.size(), 0);
    {
        std::vector<GemmDesc> wd;
        std::vector<SchurBuildJob> jobs;
        int maxn = 0;
        auto mapped = [](void *h) {
            void *d = nullptr;
            if (cudaHostGetDevicePointer(&d, h, 0) != cudaSuccess) {
                cudaGetLastError();
                return (double *) nullptr;
            }
            return (double *) d;
        };
        for (size_t q = 0; q < cones.size(); ++q) {
            SdpCone &c = *cones[q];
            if (!c.dev.batchable() || c.hy || c.n > kFusedBuildMaxN || c.m > kFusedBuildMaxM || c.m == 0) continue;
            if (c.dev.precision == 1 && c.n >= kSplitInverseMinN) continue;
            double *hv = mapped(c.h_vec), *hv2 = mapped(c.h_vec2), *hs = mapped(c.h_scal);
            if (!hv || !hv2 || !hs) continue;
            const long ldk = pad_ld(c.m);
            if (!corr && !c.Mown) HB_CUDA(hb::cmalloc(&c.Mown, sizeof(double) * ldk * c.m));
            compute_inverse_factor(s, c.Fvar);   // formed by the factorisation kernel already
            wd.push_back(GemmDesc{c.n, c.n, c.n, 1.0, 0.0, c.Fvar.K, c.Fvar.ld, 1, c.Fvar.K, c.Fvar.ld, 0, c.W, c.ld,
                                  GEMM_C_LOWER | GEMM_A_UPPER | GEMM_B_LOWER, nullptr});
            c.pinVar = true;   // the accepted point's factor
            SchurBuildJob J = schur_build_job(c.dev, c.W, c.ld, corr ? nullptr : c.Mown, ldk);
            const double r = c.dualResidual;
            J.inner = hv;
            J.innersq = (r != 0.0) ? hv2 : nullptr;
            J.trace = (!corr && r != 0.0) ? hs : nullptr;
            J.reuse_vt = corr ? 1 : 0;
            jobs.push_back(J);
            maxn = std::max(maxn, c.n);
            fused[q] = 1;
        }
        if (!jobs.empty()) {
            if (fusedCap < jobs.size()) {
                HB_CUDA(cudaStreamSynchronize(s));
                if (d_wdesc) hb::cache_free(d_wdesc);
                if (d_jobs) hb::cache_free(d_jobs);
                fusedCap = jobs.size();
                HB_CUDA(hb::cmalloc(&d_wdesc, sizeof(GemmDesc) * fusedCap));
                HB_CUDA(hb::cmalloc(&d_jobs, sizeof(SchurBuildJob) * fusedCap));
            }
            HB_CUDA(cudaMemcpyAsync(d_wdesc, wd.data(), sizeof(GemmDesc) * wd.size(), cudaMemcpyHostToDevice, s));
            HB_CUDA(cudaMemcpyAsync(d_jobs, jobs.data(), sizeof(SchurBuildJob) * jobs.size(), cudaMemcpyHostToDevice, s));
            gemm_grouped(s, d_wdesc, (int) wd.size(), maxn, maxn);
            schur_build_batch(s, d_jobs, (int) jobs.size());
        }
    }
    for (size_t q = 0; q < cones.size(); ++q) {
        SdpCone &cone = *cones[q];
        if (fused[q]) {
            // the cone's Schur block into M, in the cones' order
            if (!corr) {
                const int mk = cone.m;
                const long ldk = pad_ld(mk);
                open_m();
                if (arrow) {
                    arrow_add(cone, cone.Mown, ldk);
                } else {
                    dim3 blk(32, 8), grd((mk + 31) / 32, std::min((mk + 7) / 8, 4096));
                    scatter_lower_kernel<<<hb::counted(grd), blk, 0, s>>>(mk, cone.Mown, ldk, cone.d_rows, M, ldm);
                    HB_CUDA(cudaGetLastError());
                }
            }
            continue;
        }
        const int n = cone.n;
        const long ld = cone.ld;
        const double r = cone.dualResidual;
        if (cone.hy && !cone.ensure_dense(BUFFER_DUALVAR)) return HDSDP_RETCODE_FAILED;
        bool done = false;
        if (cone.dev.precision == 1 && n >= kSplitInverseMinN) {
            compute_inverse_factor(s, cone.Fvar);
            done = cone.dev.split_inverse(cone.Fvar.K, cone.W, ld);
        }
        if (!done) compute_inverse(s, cone.Fvar, cone.W, ld);
        cone.pinVar = true;   // the accepted point's factor
        const double *Wp = cone.W;
        SdpDevice &dev = cone.dev;
        const int mk = cone.m;
        if (type == KKT_TYPE_CORRECTOR) {
            dev.inner_all(Wp, ld, cone.d_vec);
            if (mk > 0) HB_CUDA(cudaMemcpyAsync(cone.h_vec, cone.d_vec, sizeof(double) * mk, cudaMemcpyDeviceToHost, s));
            if (r != 0.0) {
                dev.inner_all_sq(Wp, ld, cone.d_vec2, false, true);
                if (mk > 0)
                    HB_CUDA(cudaMemcpyAsync(cone.h_vec2, cone.d_vec2, sizeof(double) * mk, cudaMemcpyDeviceToHost, s));
            }
            continue;
        }
        if (r != 0.0) {
            trace(s, n, Wp, ld, cone.d_scal);
            HB_CUDA(cudaMemcpyAsync(cone.h_scal, cone.d_scal, sizeof(double), cudaMemcpyDeviceToHost, s));
        }
        if (!cone.sparse && !mOpen) {
            dev.schur_matrix(Wp, ld, M, ldm, cone.Fvar.K);
            mOpen = true;
        } else if (mk > 0) {
            open_m();
            const long ldk = pad_ld(mk);
            if (msubCap < (size_t) ldk * mk) {
                // the scratch grows: the blocks enqueued so far must have read the old one
                HB_CUDA(cudaStreamSynchronize(s));
                if (Msub) hb::cache_free(Msub);
                msubCap = (size_t) ldk * mk;
                HB_CUDA(hb::cmalloc(&Msub, sizeof(double) * msubCap));
            }
            dev.schur_matrix(Wp, ld, Msub, ldk, cone.Fvar.K);
            if (arrow) {
                arrow_add(cone, Msub, ldk);
            } else {
                dim3 blk(32, 8), grd((mk + 31) / 32, std::min((mk + 7) / 8, 4096));
                scatter_lower_kernel<<<hb::counted(grd), blk, 0, s>>>(mk, Msub, ldk, cone.d_rows, M, ldm);
                HB_CUDA(cudaGetLastError());
            }
        }
        dev.inner_all(Wp, ld, cone.d_vec, true);
        if (mk > 0) HB_CUDA(cudaMemcpyAsync(cone.h_vec, cone.d_vec, sizeof(double) * mk, cudaMemcpyDeviceToHost, s));
        if (r != 0.0) {
            dev.inner_all_sq(Wp, ld, cone.d_vec2, true);
            if (mk > 0)
                HB_CUDA(cudaMemcpyAsync(cone.h_vec2, cone.d_vec2, sizeof(double) * mk, cudaMemcpyDeviceToHost, s));
        }
    }
    HB_CUDA(cudaStreamSynchronize(s));
    for (SdpCone *cp : cones) {
        SdpCone &cone = *cp;
        const double r = cone.dualResidual;
        const std::vector<int> *rows = cone.sparse ? &cone.rows : nullptr;
        auto acc = [&](std::vector<double> &dst, const double *h, double scale) {
            if (rows)
                for (int i = 0; i < cone.m; ++i) dst[(*rows)[i]] += scale * h[i];
            else
                for (int i = 0; i < cone.m; ++i) dst[i] += scale * h[i];
        };
        if (type != KKT_TYPE_CORRECTOR && r != 0.0) dTraceSinv += cone.h_scal[0];
        acc(asinv, cone.h_vec, 1.0);
        if (r != 0.0) acc(asinvrd, cone.h_vec2, r);
    }
    if (tm) {
        tm->schur += wall() - t0;
        if (type != KKT_TYPE_CORRECTOR) tm->n_schur += (long) cones.size();
    }
    return device_error_flag() ? HDSDP_RETCODE_FAILED : HDSDP_RETCODE_OK;
}

// sBoundConeGetKKT (interface/hdsdp_conic_bound.c:199-241)
void KKT::add_bound(BoundCone &b, int type) {
    for (int i = 0; i < b.m; ++i) {
        b.dlInv[i] = 1.0 / b.dl[i];
        b.duInv[i] = 1.0 / b.du[i];
    }
    for (int i = 0; i < m; ++i) {
        asinv[i] -= b.dlInv[i];
        asinv[i] += b.duInv[i];
    }
    if (type == KKT_TYPE_CORRECTOR) return;
    for (int i = 0; i < b.m; ++i) h_buf[i] = b.dlInv[i] * b.dlInv[i] + b.duInv[i] * b.duInv[i];
    if (arrow) {
        arrow_add_diag(h_buf);
    } else {
        open_m();
        HB_CUDA(cudaMemcpyAsync(d_diag, h_buf, sizeof(double) * m, cudaMemcpyHostToDevice, s));
        add_diag_vec(s, m, M, ldm, d_diag);
        HB_CUDA(cudaStreamSynchronize(s));
    }
    if (type == KKT_TYPE_HOMOGENEOUS) {
        for (int i = 0; i < b.m; ++i) {
            dCSinv += b.up * b.duInv[i];
            double sq = b.duInv[i] * b.duInv[i];
            asinvcs[i] += b.up * sq;
            dCSinvCSinv += b.up * b.up * sq;
            dCSinv -= b.lo * b.dlInv[i];
            sq = b.dlInv[i] * b.dlInv[i];
            asinvcs[i] += b.lo * sq;
            dCSinvCSinv += b.lo * b.lo * sq;
        }
    }
}

// HKKTRegularize (interface/hdsdp_schur.c:348-373)
void KKT::regularize(double reg) {
    if (arrow) return arrow_regularize(reg);
    copy_matrix(s, 1, m, M, ldm + 1, d_t, 1);
    HB_CUDA(cudaMemcpyAsync(h_buf, d_t, sizeof(double) * m, cudaMemcpyDeviceToHost, s));
    HB_CUDA(cudaStreamSynchronize(s));
    double mn = HDSDP_INFINITY;
    for (int i = 0; i < m; ++i) mn = std::min(mn, h_buf[i]);
    reg = reg * mn;
    reg = std::min(reg, 1e-05);
    if (reg < 1e-14) reg = 0.0;
    if (reg != 0.0) add_diag(s, m, M, ldm, reg);
}

hdsdp_retcode KKT::factorize() {
    double t0 = wall();
    if (arrow) {
        const bool ok = arrow_factorize();
        if (tm) tm->schur_factor += wall() - t0;
        return ok && !device_error_flag() ? HDSDP_RETCODE_OK : HDSDP_RETCODE_FAILED;
    }
    symmetrize_lower(s, m, M, ldm);
    shift = 0.0;
    ldlActive = false;
    if (ldlMode == 1) {
        const bool ok = ldl_factorize(s, ldl, M, ldm, m);
        ldlActive = ok;
        if (tm) tm->schur_factor += wall() - t0;
        return ok && !device_error_flag() ? HDSDP_RETCODE_OK : HDSDP_RETCODE_FAILED;
    }
    bool ok = hb::factorize(s, F, M, ldm);
    if (!ok) {
        // The reference switches to an LDL^T factorisation here (linsolver.c:1373-1377);
        // this library first retries the Cholesky with a small diagonal shift, and takes
        // the LDL^T factor of the unshifted M when every shift fails.
        copy_matrix(s, 1, m, M, ldm + 1, d_t, 1);
        HB_CUDA(cudaMemcpyAsync(h_buf, d_t, sizeof(double) * m, cudaMemcpyDeviceToHost, s));
        HB_CUDA(cudaStreamSynchronize(s));
        double mx = 0.0;
        for (int i = 0; i < m; ++i) mx = std::max(mx, std::fabs(h_buf[i]));
        for (double eps = 1e-14; eps <= 1e-6 && !ok; eps *= 100.0) {
            add_diag(s, m, M, ldm, eps * std::max(mx, 1.0));
            shift += eps * std::max(mx, 1.0);
            ok = hb::factorize(s, F, M, ldm);
        }
        if (ok) {
            printf("KKT system is almost indefinite. Using a shifted Cholesky factor. \n");
        } else {
            copy_matrix(s, 1, m, d_t, 1, M, ldm + 1);   // the unshifted diagonal back
            shift = 0.0;
            ok = ldl_factorize(s, ldl, M, ldm, m);
            ldlActive = ok;
            if (ok) printf("KKT system is almost indefinite. Switch to LDL. \n");
            if (tm) tm->schur_factor += wall() - t0;
            return ok && !device_error_flag() ? HDSDP_RETCODE_OK : HDSDP_RETCODE_FAILED;
        }
    }
    if (ok && F.fuse_k) compute_inverse_factor(s, F);
    HB_CUDA(cudaStreamSynchronize(s));
    if (tm) tm->schur_factor += wall() - t0;
    return ok && !device_error_flag() ? HDSDP_RETCODE_OK : HDSDP_RETCODE_FAILED;
}

// x = M^-1 b with one step of iterative refinement on the FP64 residual.
hdsdp_retcode KKT::solve(const double *rhs, double *lhs) {
    double t0 = wall();
    if (arrow) {
        if (!arrow_solve(rhs, lhs)) device_error_flag() = 1;
        if (tm) {
            tm->schur_solve += wall() - t0;
            tm->n_schur_solve += 1;
        }
        return device_error_flag() ? HDSDP_RETCODE_FAILED : HDSDP_RETCODE_OK;
    }
    std::memcpy(h_buf, rhs, sizeof(double) * m);
    HB_CUDA(cudaMemcpyAsync(d_rhs, h_buf, sizeof(double) * m, cudaMemcpyHostToDevice, s));
    if (ldlActive) {
        ldl_solve(s, ldl, d_rhs, d_x);
        HB_CUDA(cudaMemcpyAsync(d_r, d_rhs, sizeof(double) * m, cudaMemcpyDeviceToDevice, s));
        coldot(s, m, m, M, ldm, d_x, d_r, -1.0, 1.0, 0);   // r = b - M x
        ldl_solve(s, ldl, d_r, d_r);
        axpy(s, m, 1.0, d_r, d_x);
        HB_CUDA(cudaMemcpyAsync(h_buf, d_x, sizeof(double) * m, cudaMemcpyDeviceToHost, s));
        HB_CUDA(cudaStreamSynchronize(s));
        std::memcpy(lhs, h_buf, sizeof(double) * m);
        if (tm) {
            tm->schur_solve += wall() - t0;
            tm->n_schur_solve += 1;
        }
        return device_error_flag() ? HDSDP_RETCODE_FAILED : HDSDP_RETCODE_OK;
    }
    bool ok = true;
    if (F.fuse_k) {
        coldot(s, m, m, F.KT, F.ld, d_rhs, d_t, 1.0, 0.0, 2);   // t = K b
        coldot(s, m, m, F.K, F.ld, d_t, d_x, 1.0, 0.0, 1);      // x = K^T t
    } else {
        ok = chol_solve(s, F, d_rhs, d_x);
    }
    HB_CUDA(cudaMemcpyAsync(d_r, d_rhs, sizeof(double) * m, cudaMemcpyDeviceToDevice, s));
    coldot(s, m, m, M, ldm, d_x, d_r, -1.0, 1.0, 0);        // r = b - M x
    if (shift != 0.0) axpy(s, m, shift, d_x, d_r);          // residual of the unshifted system
    if (F.fuse_k) {
        coldot(s, m, m, F.KT, F.ld, d_r, d_t, 1.0, 0.0, 2);
        coldot(s, m, m, F.K, F.ld, d_t, d_r, 1.0, 0.0, 1);
    } else {
        ok = ok && chol_solve(s, F, d_r, d_r);
    }
    axpy(s, m, 1.0, d_r, d_x);
    HB_CUDA(cudaMemcpyAsync(h_buf, d_x, sizeof(double) * m, cudaMemcpyDeviceToHost, s));
    HB_CUDA(cudaStreamSynchronize(s));
    if (!F.fuse_k && chol_solve_error()) ok = false;
    if (!ok) device_error_flag() = 1;
    std::memcpy(lhs, h_buf, sizeof(double) * m);
    if (tm) {
        tm->schur_solve += wall() - t0;
        tm->n_schur_solve += 1;
    }
    return device_error_flag() ? HDSDP_RETCODE_FAILED : HDSDP_RETCODE_OK;
}

// ======================================================================================
// Lanczos (linalg/hdsdp_lanczos.c:161-292)
// ======================================================================================
namespace {
__device__ double bsum(double v) {
    __shared__ double red[32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) red[w] = v;
    __syncthreads();
    const int nw = (blockDim.x + 31) >> 5;
    v = (threadIdx.x < nw) ? red[threadIdx.x] : 0.0;
    if (w == 0) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (threadIdx.x == 0) red[0] = v;
    }
    __syncthreads();
    v = red[0];
    __syncthreads();
    return v;
}

// One Lanczos orthogonalisation step; single block.
__global__ void lanczos_orth_kernel(int n, double *V, long ldv, int k, double *w, double *ab, int maxdim) {
    const double *vk = V + (size_t) k * ldv;
    if (k > 0) {
        const double h = ab[maxdim + k - 1];
        const double *vp = V + (size_t) (k - 1) * ldv;
        for (int i = threadIdx.x; i < n; i += blockDim.x) w[i] -= h * vp[i];
        __syncthreads();
    }
    double acc = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) acc += w[i] * vk[i];
    const double alp = bsum(acc);
    acc = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double x = w[i] - alp * vk[i];
        w[i] = x;
        acc += x * x;
    }
    const double nrm = sqrt(bsum(acc));
    if (threadIdx.x == 0) ab[k] = alp;
    if (nrm > 0.0) {
        double *vn = V + (size_t) (k + 1) * ldv;
        for (int i = threadIdx.x; i < n; i += blockDim.x) vn[i] = w[i] / nrm;
        if (threadIdx.x == 0) ab[maxdim + k] = nrm;
    }
}

// v = (a ? a : 0) + b, then normalise into V[:,0]; single block.
__global__ void lanczos_start_kernel(int n, const double *a, const double *b, double *V) {
    double acc = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double x = (a ? a[i] : 0.0) + b[i];
        V[i] = x;
        acc += x * x;
    }
    const double nrm = sqrt(bsum(acc));
    for (int i = threadIdx.x; i < n; i += blockDim.x) V[i] = (nrm > 0.0) ? V[i] / nrm : 0.0;
}

// z = V[:, 0..k] * y
__global__ void lanczos_combine_kernel(int n, const double *V, long ldv, int kp1, const double *y, double *z) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double acc = 0.0;
        for (int j = 0; j < kp1; ++j) acc += V[(size_t) i + (size_t) j * ldv] * y[j];
        z[i] = acc;
    }
}

// z -= lam * x; out = ||z||; single block
__global__ void lanczos_resid_kernel(int n, double *z, const double *x, double lam, double *out) {
    double acc = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double t = z[i] - lam * x[i];
        z[i] = t;
        acc += t * t;
    }
    const double v = sqrt(bsum(acc));
    if (threadIdx.x == 0) *out = v;
}

// ---- Lanczos steps of larger blocks in one cooperative launch per check interval.
//
// Steps k0 .. k1-1 of the three-term recurrence for M = K (-D) K^T (K = L^-1 lower,
// KT = K^T), taken exactly as lanczos_orth_kernel takes them (w = M v_k - beta v_{k-1},
// alpha = w.v_k, w -= alpha v_k, beta = |w|, v_{k+1} = w / beta when beta > 0). Block b
// owns columns [b*cpb, (b+1)*cpb) of every product and reduces each column with
// kLzWpc warps; the dot products go through per-block partial sums that every block
// adds up in the same order, so all blocks hold the same alpha and beta. Four grid-wide
// barriers per step. Values written inside the launch are read with ld.global.cg.
constexpr int kLzThreads = 1024, kLzWpc = 4;
constexpr int kLzCols = kLzThreads / 32 / kLzWpc;   // columns per block and pass
constexpr int kLzSmemMax = 200 * 1024;              // dynamic shared memory of the cached variant
constexpr int kLzFusedMaxN = 2048;                  // K, K^T and D (3 x 8 n^2 bytes) still fit the L2

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// out[j] = scale * sum_i A(i, j) x[i] over the rows of column j that `mode` keeps
// (0 all, 1 i >= j, 2 i <= j), for the block's columns [j0, j1).
__device__ void lz_block_coldot(int n, const double *__restrict__ A, long lda, const double *x, double *out,
                                double scale, int mode, int j0, int j1, double *red) {
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int cslot = w / kLzWpc, seg = w % kLzWpc;
    for (int jb = j0; jb < j1; jb += kLzCols) {
        const int j = jb + cslot;
        double acc = 0.0;
        if (j < j1) {
            const int lo = (mode == 1) ? j : 0, hi = (mode == 2) ? j + 1 : n;
            const int len = hi - lo;
            const int chunk = (((len + kLzWpc - 1) / kLzWpc) + 31) & ~31;
            const int a0 = lo + seg * chunk, a1 = min(hi, a0 + chunk);
            const double *col = A + (size_t) j * lda;
            int k = a0 + lane;
            for (; k + 32 < a1; k += 64) acc += __ldg(col + k) * __ldcg(x + k) + __ldg(col + k + 32) * __ldcg(x + k + 32);
            for (; k < a1; k += 32) acc += __ldg(col + k) * __ldcg(x + k);
        }
        acc = warp_sum(acc);
        if (lane == 0) red[w] = acc;
        __syncthreads();
        if (threadIdx.x < kLzCols && jb + (int) threadIdx.x < j1) {
            double t = 0.0;
#pragma unroll
            for (int q = 0; q < kLzWpc; ++q) t += red[threadIdx.x * kLzWpc + q];
            out[jb + threadIdx.x] = scale * t;
        }
        __syncthreads();
    }
}

// sum of part[0 .. G) in a fixed order, the same in every block
__device__ double lz_grid_sum(const double *part, int G, double *red) {
    if (threadIdx.x < 32) {
        double v = 0.0;
        for (int q = threadIdx.x; q < G; q += 32) v += __ldcg(part + q);
        v = warp_sum(v);
        if (threadIdx.x == 0) red[0] = v;
    }
    __syncthreads();
    const double v = red[0];
    __syncthreads();
    return v;
}

// The block's columns held in shared memory for the whole launch: region K (column j,
// rows j..n-1), region KT (rows 0..j), region D (rows 0..n-1), packed column after column;
// a block with cpb columns holds cpb (2n + 1) doubles. Local column c starts at
// c (n - j0) - c (c - 1) / 2 in K, c (j0 + 1) + c (c - 1) / 2 in KT and c n in D.
__host__ __device__ inline long lz_cached_doubles(int n, int cpb) { return (long) cpb * (2L * n + 1); }

// w -= beta_{k-1} v_{k-1} and the block's partial w.v_k into part[blockIdx.x]
__device__ void lz_orth_partial(int j0, int j1, int k, const double *V, long ldv, const double *ab, int maxdim,
                                double *w, double *part, double *red) {
    const double *vk = V + (size_t) k * ldv;
    const double bprev = (k > 0) ? __ldcg(ab + maxdim + k - 1) : 0.0;
    double pa = 0.0;
    for (int j = j0 + threadIdx.x; j < j1; j += blockDim.x) {
        double x = w[j];
        if (k > 0) x -= bprev * __ldcg(V + (size_t) (k - 1) * ldv + j);
        w[j] = x;
        pa += x * __ldcg(vk + j);
    }
    pa = warp_sum(pa);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = pa;
    __syncthreads();
    if (threadIdx.x == 0) {
        double v = 0.0;
        for (int q = 0; q < kLzThreads / 32; ++q) v += red[q];
        part[blockIdx.x] = v;
    }
}

// w -= alpha v_k and the block's partial |w|^2 into part[G + blockIdx.x]
__device__ void lz_norm_partial(int j0, int j1, int k, double alp, const double *V, long ldv, double *w, double *part,
                                int G, double *red) {
    const double *vk = V + (size_t) k * ldv;
    double pn = 0.0;
    for (int j = j0 + threadIdx.x; j < j1; j += blockDim.x) {
        const double x = w[j] - alp * __ldcg(vk + j);
        w[j] = x;
        pn += x * x;
    }
    pn = warp_sum(pn);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = pn;
    __syncthreads();
    if (threadIdx.x == 0) {
        double v = 0.0;
        for (int q = 0; q < kLzThreads / 32; ++q) v += red[q];
        part[G + blockIdx.x] = v;
    }
}

// v_{k+1} = w / beta over the block's columns; alpha and beta recorded by block 0
__device__ void lz_next(int j0, int j1, int k, double alp, double nrm, double *V, long ldv, double *ab, int maxdim,
                        const double *w) {
    if (nrm > 0.0) {
        double *vn = V + (size_t) (k + 1) * ldv;
        for (int j = j0 + threadIdx.x; j < j1; j += blockDim.x) vn[j] = w[j] / nrm;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        ab[k] = alp;
        if (nrm > 0.0) ab[maxdim + k] = nrm;
    }
}

// Streaming variant: the block's columns of K, K^T and D are read from L2 in every step.
__global__ void __launch_bounds__(kLzThreads, 1)
    lanczos_steps_kernel(int n, const double *K, const double *KT, long ldk, const double *D, long ldD, double *V,
                         long ldv, double *ab, int maxdim, int k0, int k1, double *t, double *u, double *w,
                         double *part) {
    cooperative_groups::grid_group grid = cooperative_groups::this_grid();
    __shared__ double red[kLzThreads / 32];
    const int G = gridDim.x;
    const int cpb = (n + G - 1) / G;
    const int j0 = min(n, (int) blockIdx.x * cpb), j1 = min(n, j0 + cpb);
    for (int k = k0; k < k1; ++k) {
        const double *vk = V + (size_t) k * ldv;
        lz_block_coldot(n, K, ldk, vk, t, 1.0, 1, j0, j1, red);     // t = K^T v_k
        grid.sync();
        lz_block_coldot(n, D, ldD, t, u, -1.0, 0, j0, j1, red);     // u = -D t
        grid.sync();
        lz_block_coldot(n, KT, ldk, u, w, 1.0, 2, j0, j1, red);     // w = K u
        lz_orth_partial(j0, j1, k, V, ldv, ab, maxdim, w, part, red);
        grid.sync();
        const double alp = lz_grid_sum(part, G, red);
        lz_norm_partial(j0, j1, k, alp, V, ldv, w, part, G, red);
        grid.sync();
        const double nrm = sqrt(lz_grid_sum(part + G, G, red));
        lz_next(j0, j1, k, alp, nrm, V, ldv, ab, maxdim, w);
        grid.sync();
    }
}

// Shared-memory variant (n small enough for a block's share of columns to fit): the
// block's columns of K, K^T and D are loaded into shared memory once per launch
// (lz_cached_doubles(n, cpb) doubles) and each product's input vector is staged there (n
// more doubles); kLzWpc warps reduce each column. v_{k+1} = w / beta is read by the next
// step's first product straight from w (the last grid barrier of a step publishes w, and
// every block holds beta), so a step takes four grid-wide barriers.
__global__ void __launch_bounds__(kLzThreads, 1)
    lanczos_steps_smem_kernel(int n, const double *K, const double *KT, long ldk, const double *D, long ldD,
                              double *V, long ldv, double *ab, int maxdim, int k0, int k1, double *w, double *tg,
                              double *ug, double *part) {
    cooperative_groups::grid_group grid = cooperative_groups::this_grid();
    __shared__ double red[kLzThreads / 32];
    __shared__ double scal[2];
    extern __shared__ double dyn[];
    const int G = gridDim.x;
    const int cpb = (n + G - 1) / G;
    const int j0 = min(n, (int) blockIdx.x * cpb), j1 = min(n, j0 + cpb);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = kLzThreads / 32;
    const long nc = j1 - j0;
    double *sK = dyn;
    double *sKT = sK + (nc * (n - j0) - nc * (nc - 1) / 2);
    double *sD = sKT + (nc * (j0 + 1) + nc * (nc - 1) / 2);
    double *sx = dyn + lz_cached_doubles(n, cpb);
    for (long c = 0; c < nc; ++c) {
        const int j = j0 + (int) c;
        double *dk = sK + c * (n - j0) - c * (c - 1) / 2;
        double *dkt = sKT + c * (j0 + 1) + c * (c - 1) / 2;
        double *dd = sD + c * n;
        const double *gk = K + (size_t) j * ldk, *gkt = KT + (size_t) j * ldk, *gd = D + (size_t) j * ldD;
        for (int i = j + threadIdx.x; i < n; i += blockDim.x) dk[i - j] = __ldg(gk + i);
        for (int i = threadIdx.x; i <= j; i += blockDim.x) dkt[i] = __ldg(gkt + i);
        for (int i = threadIdx.x; i < n; i += blockDim.x) dd[i] = __ldg(gd + i);
    }
    // sx = x / div (div 0: zeros; the same division that forms v_{k+1})
    auto stage = [&](const double *x, double div) {
        for (int i = threadIdx.x; i < n; i += blockDim.x)
            sx[i] = (div == 1.0) ? __ldcg(x + i) : (div > 0.0) ? __ldcg(x + i) / div : 0.0;
        __syncthreads();
    };
    // out[j] = scale * sum over the rows `mode` keeps (0 all, 1 i >= j, 2 i <= j) of column j
    const int cslot = warp / kLzWpc, seg = warp % kLzWpc;
    auto coldot = [&](int mode, const double *reg, double *out, double scale) {
        for (int jb = j0; jb < j1; jb += kLzCols) {
            const int j = jb + cslot;
            double acc = 0.0;
            if (j < j1) {
                const long c = j - j0;
                const int lo = (mode == 1) ? j : 0, hi = (mode == 2) ? j + 1 : n;
                const double *col = (mode == 1)   ? reg + c * (n - j0) - c * (c - 1) / 2 - lo
                                    : (mode == 2) ? reg + c * (j0 + 1) + c * (c - 1) / 2
                                                  : reg + c * n;
                const int len = hi - lo;
                const int chunk = (((len + kLzWpc - 1) / kLzWpc) + 31) & ~31;
                const int a0 = lo + seg * chunk, a1 = min(hi, a0 + chunk);
                for (int k = a0 + lane; k < a1; k += 32) acc += col[k] * sx[k];
            }
            acc = warp_sum(acc);
            if (lane == 0) red[warp] = acc;
            __syncthreads();
            if (threadIdx.x < kLzCols && jb + (int) threadIdx.x < j1) {
                double t = 0.0;
#pragma unroll
                for (int q = 0; q < kLzWpc; ++q) t += red[threadIdx.x * kLzWpc + q];
                out[jb + threadIdx.x] = scale * t;
            }
            if (jb + kLzCols < j1) __syncthreads();   // red is reused by the next pass
        }
    };
    // block total of v (one value per thread) into *slot
    auto block_part = [&](double v, double *slot) {
        v = warp_sum(v);
        if (lane == 0) red[warp] = v;
        __syncthreads();
        if (threadIdx.x == 0) {
            double tot = 0.0;
            for (int q = 0; q < nwarp; ++q) tot += red[q];
            *slot = tot;
        }
    };
    // sum of p[0 .. G) in a fixed order, the same in every block
    auto grid_total = [&](const double *p, int which) {
        if (warp == 0) {
            double v = 0.0;
            for (int q = lane; q < G; q += 32) v += __ldcg(p + q);
            v = warp_sum(v);
            if (lane == 0) scal[which] = v;
        }
        __syncthreads();
        return scal[which];
    };
    double nrmPrev = 0.0;
    for (int k = k0; k < k1; ++k) {
        const double *vk = V + (size_t) k * ldv;
        if (k > k0) stage(w, nrmPrev);
        else stage(vk, 1.0);
        coldot(1, sK, tg, 1.0);     // t = K^T v_k
        grid.sync();
        stage(tg, 1.0);
        coldot(0, sD, ug, -1.0);    // u = -D t
        grid.sync();
        stage(ug, 1.0);
        coldot(2, sKT, w, 1.0);     // w = K u
        __syncthreads();
        // w -= beta_{k-1} v_{k-1}; partial w.v_k
        const double bprev = (k > 0) ? __ldcg(ab + maxdim + k - 1) : 0.0;
        double pa = 0.0;
        for (int j = j0 + threadIdx.x; j < j1; j += blockDim.x) {
            double x = w[j];
            if (k > 0) x -= bprev * __ldcg(V + (size_t) (k - 1) * ldv + j);
            w[j] = x;
            pa += x * __ldcg(vk + j);
        }
        block_part(pa, part + blockIdx.x);
        grid.sync();
        const double alp = grid_total(part, 0);
        double pn = 0.0;
        for (int j = j0 + threadIdx.x; j < j1; j += blockDim.x) {
            const double x = w[j] - alp * __ldcg(vk + j);
            w[j] = x;
            pn += x * x;
        }
        block_part(pn, part + G + blockIdx.x);
        grid.sync();
        const double nrm = sqrt(grid_total(part + G, 1));
        lz_next(j0, j1, k, alp, nrm, V, ldv, ab, maxdim, w);
        nrmPrev = nrm;
    }
}

// ---- Lanczos for blocks of order <= kSmallLanczosN: one CTA holds K = L^-1, D and the
// Lanczos basis in shared memory and runs every step in one launch (the stepwise path
// spends four launches per step, which dominates for small blocks).
constexpr int kSmallLanczosN = kSmallLanczosMaxN;

__host__ __device__ inline int small_ld(int n) { return n | 1; }  // odd stride: fewer bank conflicts

inline size_t small_lanczos_smem(int n, int maxdim) {
    return sizeof(double) * ((size_t) 2 * n * small_ld(n) + (size_t) (maxdim + 1) * n + 4 * (size_t) n);
}

// K (lower, leading dimension ldk) and D into shared memory (leading dimension small_ld(n))
__device__ void small_load(int n, const double *K, long ldk, const double *D, long ldD, double *sK, double *sD) {
    const int ls = small_ld(n);
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
        const int i = e % n, j = e / n;
        sK[i + j * ls] = (i >= j) ? K[(size_t) i + (size_t) j * ldk] : 0.0;
        sD[i + j * ls] = D[(size_t) i + (size_t) j * ldD];
    }
    __syncthreads();
}

// y = K (-D) (K^T x), one warp per output entry
__device__ void small_mv(int n, const double *sK, const double *sD, const double *x, double *t, double *u,
                         double *y) {
    const int ls = small_ld(n), lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int i = warp; i < n; i += nw) {  // t = K^T x
        double a = 0.0;
        for (int k = i + lane; k < n; k += 32) a += sK[k + i * ls] * x[k];
        for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
        if (lane == 0) t[i] = a;
    }
    __syncthreads();
    for (int i = warp; i < n; i += nw) {  // u = -D t
        double a = 0.0;
        for (int k = lane; k < n; k += 32) a += sD[k + i * ls] * t[k];
        for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
        if (lane == 0) u[i] = -a;
    }
    __syncthreads();
    for (int i = warp; i < n; i += nw) {  // y = K u
        double a = 0.0;
        for (int k = lane; k <= i; k += 32) a += sK[i + k * ls] * u[k];
        for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
        if (lane == 0) y[i] = a;
    }
    __syncthreads();
}

// Start vector v0 = normalise(a + b) (a may be null), then maxdim steps of the
// three-term recurrence exactly as lanczos_orth_kernel takes them; the basis V (all
// maxdim + 1 columns, zero past a breakdown) and alpha / beta go to global memory.
__device__ void lanczos_small_body(int n, const double *K, long ldk, const double *D, long ldD, const double *a,
                                   const double *b, double *V, long ldv, double *ab, int maxdim) {
    extern __shared__ double sm[];
    const int ls = small_ld(n);
    double *sK = sm, *sD = sK + (size_t) n * ls, *sV = sD + (size_t) n * ls, *w = sV + (size_t) (maxdim + 1) * n;
    double *t = w + n, *u = t + n, *sab = u + n;  // sab: 2 * maxdim + 2 <= 4n is not guaranteed: kept in ab
    (void) sab;
    small_load(n, K, ldk, D, ldD, sK, sD);
    for (int e = threadIdx.x; e < (maxdim + 1) * n; e += blockDim.x) sV[e] = 0.0;
    for (int e = threadIdx.x; e < 2 * maxdim + 2; e += blockDim.x) ab[e] = 0.0;
    __syncthreads();
    double acc = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double x = (a ? a[i] : 0.0) + b[i];
        sV[i] = x;
        acc += x * x;
    }
    double nrm = sqrt(bsum(acc));
    for (int i = threadIdx.x; i < n; i += blockDim.x) sV[i] = (nrm > 0.0) ? sV[i] / nrm : 0.0;
    __syncthreads();
    double betaPrev = 0.0;
    for (int k = 0; k < maxdim; ++k) {
        const double *vk = sV + (size_t) k * n;
        small_mv(n, sK, sD, vk, t, u, w);
        if (k > 0) {
            const double *vp = sV + (size_t) (k - 1) * n;
            for (int i = threadIdx.x; i < n; i += blockDim.x) w[i] -= betaPrev * vp[i];
            __syncthreads();
        }
        acc = 0.0;
        for (int i = threadIdx.x; i < n; i += blockDim.x) acc += w[i] * vk[i];
        const double alp = bsum(acc);
        acc = 0.0;
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            const double x = w[i] - alp * vk[i];
            w[i] = x;
            acc += x * x;
        }
        nrm = sqrt(bsum(acc));
        if (threadIdx.x == 0) ab[k] = alp;
        betaPrev = 0.0;
        if (nrm > 0.0) {
            double *vn = sV + (size_t) (k + 1) * n;
            for (int i = threadIdx.x; i < n; i += blockDim.x) vn[i] = w[i] / nrm;
            if (threadIdx.x == 0) ab[maxdim + k] = nrm;
            betaPrev = nrm;
        }
        __syncthreads();
    }
    for (int e = threadIdx.x; e < (maxdim + 1) * n; e += blockDim.x) {
        const int i = e % n, j = e / n;
        V[(size_t) i + (size_t) j * ldv] = sV[e];
    }
}

// The Ritz part of a converged check: z1 = V y1, z2 = M z1 (warm <- z2),
// out[0] = |z2 - lam z1|; z2 = V y2, z1 = M z2, out[1] = |z1 - lam z2|.
__device__ void lanczos_small_ritz_body(int n, const double *K, long ldk, const double *D, long ldD,
                                       const double *V, long ldv, int kp1, const double *y, double lam,
                                       double *warm, double *out) {
    extern __shared__ double sm[];
    const int ls = small_ld(n);
    double *sK = sm, *sD = sK + (size_t) n * ls, *z1 = sD + (size_t) n * ls, *z2 = z1 + n, *t = z2 + n, *u = t + n;
    small_load(n, K, ldk, D, ldD, sK, sD);
    for (int pass = 0; pass < 2; ++pass) {
        const double *yc = y + pass * kp1;
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            double a = 0.0;
            for (int j = 0; j < kp1; ++j) a += V[(size_t) i + (size_t) j * ldv] * yc[j];
            z1[i] = a;
        }
        __syncthreads();
        small_mv(n, sK, sD, z1, t, u, z2);
        double acc = 0.0;
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            if (pass == 0) warm[i] = z2[i];
            const double r = z2[i] - lam * z1[i];
            acc += r * r;
        }
        const double v = sqrt(bsum(acc));
        if (threadIdx.x == 0) out[pass] = v;
        __syncthreads();
    }
}

__global__ void lanczos_small_kernel(int n, const double *K, long ldk, const double *D, long ldD, const double *a,
                                     const double *b, double *V, long ldv, double *ab, int maxdim) {
    lanczos_small_body(n, K, ldk, D, ldD, a, b, V, ldv, ab, maxdim);
}

__global__ void lanczos_small_ritz_kernel(int n, const double *K, long ldk, const double *D, long ldD,
                                          const double *V, long ldv, int kp1, const double *y, double lam,
                                          double *warm, double *out) {
    lanczos_small_ritz_body(n, K, ldk, D, ldD, V, ldv, kp1, y, lam, warm, out);
}

// Several cones' small-block runs in one launch, one CTA each.
// hab / hout: device addresses of the host's pinned mirrors of ab / out, written directly
// when set
struct LzStepJob {
    const double *K, *D, *a, *b;
    double *V, *ab, *hab;
    long ldk, ldD, ldv;
    int n, maxdim;
};
struct LzRitzJob {
    const double *K, *D, *V, *y;
    double *warm, *out, *hout;
    long ldk, ldD, ldv;
    double lam;
    int n, kp1;
};
constexpr int kLzBatch = 32;
constexpr int kLzHostParallel = 8;   // cones from which the host replays run on several threads
// the two small-block kernels over a job array in device memory (any number of cones) or
// over at most kLzBatch jobs passed by value
template <class Job> struct LzPack {
    Job job[kLzBatch];
};
__device__ void lz_run(const LzStepJob &J) {
    lanczos_small_body(J.n, J.K, J.ldk, J.D, J.ldD, J.a, J.b, J.V, J.ldv, J.ab, J.maxdim);
    if (J.hab) {
        __threadfence_block();
        __syncthreads();
        for (int e = threadIdx.x; e < 2 * J.maxdim + 2; e += blockDim.x) J.hab[e] = J.ab[e];
    }
}
__device__ void lz_run(const LzRitzJob &J) {
    lanczos_small_ritz_body(J.n, J.K, J.ldk, J.D, J.ldD, J.V, J.ldv, J.kp1, J.y, J.lam, J.warm, J.out);
    if (J.hout) {
        __threadfence_block();
        __syncthreads();
        if (threadIdx.x < 2) J.hout[threadIdx.x] = J.out[threadIdx.x];
    }
}
template <class Job> __global__ void lz_pack_kernel(const LzPack<Job> B) { lz_run(B.job[blockIdx.x]); }
template <class Job> __global__ void lz_array_kernel(const Job *__restrict__ jobs) { lz_run(jobs[blockIdx.x]); }

// one launch over every job: by value when they fit the parameters, else from a device copy
// kept per host thread, device and job type (stream-ordered behind the launches before it)
template <class Job> void lz_launch(cudaStream_t s, const std::vector<Job> &jobs, size_t smem) {
    const int count = (int) jobs.size();
    if (count == 0) return;
    if (count <= kLzBatch) {
        LzPack<Job> B;
        for (int q = 0; q < count; ++q) B.job[q] = jobs[q];
        lz_pack_kernel<Job><<<hb::counted(count), 256, smem, s>>>(B);
        HB_CUDA(cudaGetLastError());
        return;
    }
    struct Buf {
        Job *p = nullptr;
        size_t cap = 0;
    };
    thread_local Buf buf[kMaxDevices];
    Buf &b = buf[current_device()];
    if (b.cap < jobs.size()) {
        if (b.p) hb::cache_free(b.p);
        b.p = nullptr;
        b.cap = 0;
        HB_CUDA(hb::cmalloc(&b.p, sizeof(Job) * jobs.size()));
        b.cap = jobs.size();
    }
    HB_CUDA(cudaMemcpyAsync(b.p, jobs.data(), sizeof(Job) * jobs.size(), cudaMemcpyHostToDevice, s));
    lz_array_kernel<Job><<<hb::counted(count), 256, smem, s>>>(b.p);
    HB_CUDA(cudaGetLastError());
}
template <class Job> void lz_allow_smem(int bytes) {
    HB_CUDA(cudaFuncSetAttribute((const void *) lz_pack_kernel<Job>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    HB_CUDA(cudaFuncSetAttribute((const void *) lz_array_kernel<Job>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
}

// All eigenpairs of the symmetric tridiagonal matrix with diagonal d[0..n) and
// off-diagonal e[0..n-1): QL iteration with implicit Wilkinson shifts, rotations
// accumulated into Z (column-major n x n, columns are eigenvectors).
void tridiag_eig(int n, std::vector<double> d, std::vector<double> e, std::vector<double> &evals,
                 std::vector<double> &Z) {
    Z.assign((size_t) n * n, 0.0);
    for (int i = 0; i < n; ++i) Z[(size_t) i * n + i] = 1.0;
    e.resize(n, 0.0);
    e[n - 1] = 0.0;
    for (int l = 0; l < n; ++l) {
        for (int iter = 0; iter < 60; ++iter) {
            int mm = l;
            for (; mm < n - 1; ++mm) {
                const double dd = std::fabs(d[mm]) + std::fabs(d[mm + 1]);
                if (std::fabs(e[mm]) <= 1e-15 * dd) break;
            }
            if (mm == l) break;
            double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
            double r = std::hypot(g, 1.0);
            g = d[mm] - d[l] + e[l] / (g + (g >= 0 ? r : -r));
            double sn = 1.0, c = 1.0, p = 0.0;
            int i = mm - 1;
            for (; i >= l; --i) {
                double f = sn * e[i], b = c * e[i];
                r = std::hypot(f, g);
                e[i + 1] = r;
                if (r == 0.0) {
                    d[i + 1] -= p;
                    e[mm] = 0.0;
                    break;
                }
                sn = f / r;
                c = g / r;
                g = d[i + 1] - p;
                r = (d[i] - g) * sn + 2.0 * c * b;
                p = sn * r;
                d[i + 1] = g + p;
                g = c * r - b;
                for (int k = 0; k < n; ++k) {
                    f = Z[(size_t) (i + 1) * n + k];
                    Z[(size_t) (i + 1) * n + k] = sn * Z[(size_t) i * n + k] + c * f;
                    Z[(size_t) i * n + k] = c * Z[(size_t) i * n + k] - sn * f;
                }
            }
            if (r == 0.0 && i >= l) continue;
            d[l] -= p;
            e[l] = g;
            e[mm] = 0.0;
        }
    }
    evals = d;
}
}  // namespace

void Lanczos::init(int n_, cudaStream_t s_) {
    n = n_;
    s = s_;
    ld = pad_ld(n);
    HB_CUDA(hb::cmalloc(&V, sizeof(double) * ld * (maxdim + 1)));
    for (double **p : {&w, &z1, &z2, &t1, &u, &warm, &init_vec, &pert_vec}) HB_CUDA(hb::cmalloc(p, sizeof(double) * ld));
    HB_CUDA(hb::cmalloc(&d_ab, sizeof(double) * (2 * maxdim + 2)));
    HB_CUDA(hb::cmalloc_host(&h_ab, sizeof(double) * (2 * maxdim + 2)));
    HB_CUDA(hb::cmalloc(&part, sizeof(double) * 2 * kLanczosMaxBlocks));
    HB_CUDA(hb::cmalloc(&d_y, sizeof(double) * 2 * (maxdim + 1)));
    HB_CUDA(hb::cmalloc(&d_scal, sizeof(double) * 4));
    HB_CUDA(hb::cmalloc_host(&h_scal, sizeof(double) * 4));
    HB_CUDA(hb::cmalloc_host(&h_yv, sizeof(double) * 2 * (maxdim + 1)));
    auto mapped = [](double *h) {
        double *d = nullptr;
        if (cudaHostGetDevicePointer((void **) &d, h, 0) != cudaSuccess) {
            cudaGetLastError();
            d = nullptr;
        }
        return d;
    };
    dm_ab = mapped(h_ab);
    dm_scal = mapped(h_scal);
    dm_yv = mapped(h_yv);
    // Deterministic start and perturbation vectors: srand(n) then, per entry,
    // srand(rand()) and sqrt(sqrt(rand() % 1627)) * (rand() % 2 - 0.5)
    // (HLanczosIPrepare / HLanczosIPerturb, linalg/hdsdp_lanczos.c:33-53).
    std::vector<double> h(n);
    srand(n);
    for (int i = 0; i < n; ++i) {
        srand(rand());
        const int r1 = rand() % 1627;
        const int r2 = rand() % 2;
        h[i] = std::sqrt(std::sqrt((double) r1)) * (r2 - 0.5);
    }
    HB_CUDA(cudaMemcpy(init_vec, h.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
    srand(n);
    for (int i = 0; i < n; ++i) {
        srand(rand());
        const int r1 = rand() % 1627;
        const int r2 = rand() % 2;
        h[i] = 1e-03 * std::sqrt(std::sqrt((double) r1)) * (r2 - 0.5);
    }
    HB_CUDA(cudaMemcpy(pert_vec, h.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
    legacy_fence();
    nComputed = 0;
}

void Lanczos::release() {
    for (double **p : {&V, &w, &z1, &z2, &t1, &u, &warm, &init_vec, &pert_vec, &d_ab, &d_y, &d_scal, &part}) {
        if (*p) hb::cache_free(*p);
        *p = nullptr;
    }
    if (h_ab) hb::cache_free_host(h_ab);
    if (h_scal) hb::cache_free_host(h_scal);
    h_ab = h_scal = nullptr;
    if (h_yv) hb::cache_free_host(h_yv);
    h_yv = dm_ab = dm_scal = dm_yv = nullptr;
}

hdsdp_retcode Lanczos::solve(DenseFactor &F, const double *D, long ldD, double *maxStep, Timers *tm) {
    double t0 = wall();
    if (hyOp) {
        if (hyOp->nfront > 0) compute_inverse_factor(s, hyOp->Ff);
    } else {
        compute_inverse_factor(s, F);
    }
    if (tm) tm->lz_inverse += wall() - t0;   // enqueue time: the steps' launch follows without a wait
    // buffers: V columns, w (Mv), t1 / z1 / z2 temporaries
    auto mv = [&](const double *x, double *y) {
        if (hyOp) {
            hyOp->apply_congruence(s, D, ldD, -1.0, x, t1, u, y);  // y = L^-1 (-D) L^-T x
        } else {
            coldot(s, n, n, F.K, F.ld, x, t1, 1.0, 0.0, 1);   // t1 = L^-T x
            coldot(s, n, n, D, ldD, t1, u, -1.0, 0.0, 0);     // u  = -D t1
            coldot(s, n, n, F.KT, F.ld, u, y, 1.0, 0.0, 2);   // y  = L^-1 u
        }
        if (tm) tm->n_lanczos_mv += 1;
    };
    // small blocks: every step in one launch, then the checks below replay the schedule on
    // the recorded alpha / beta (a step's values do not depend on later steps)
    const bool small = !hyOp && n <= kSmallLanczosN;
    if (small) {
        static std::atomic<unsigned long long> attr{0};
        once_per_device(attr, [] {
            const int bytes = (int) small_lanczos_smem(kSmallLanczosN, 30);
            HB_CUDA(cudaFuncSetAttribute((const void *) lanczos_small_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
            HB_CUDA(cudaFuncSetAttribute((const void *) lanczos_small_ritz_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
        });
        lanczos_small_kernel<<<hb::counted(1), 256, small_lanczos_smem(n, maxdim), s>>>(
            n, F.K, F.ld, D, ldD, nComputed == 0 ? nullptr : warm, nComputed == 0 ? init_vec : pert_vec, V, ld, d_ab,
            maxdim);
        HB_CUDA(cudaGetLastError());
        HB_CUDA(cudaMemcpyAsync(h_ab, d_ab, sizeof(double) * (2 * maxdim + 2), cudaMemcpyDeviceToHost, s));
        HB_CUDA(cudaStreamSynchronize(s));
        if (tm) tm->n_lanczos_mv += maxdim;
    } else {
        HB_CUDA(cudaMemsetAsync(V, 0, sizeof(double) * ld * (maxdim + 1), s));
        HB_CUDA(cudaMemsetAsync(d_ab, 0, sizeof(double) * (2 * maxdim + 2), s));
        if (nComputed == 0) lanczos_start_kernel<<<hb::counted(1), 1024, 0, s>>>(n, nullptr, init_vec, V);
        else lanczos_start_kernel<<<hb::counted(1), 1024, 0, s>>>(n, warm, pert_vec, V);
    }
    // dense factor: the steps up to each check run in one cooperative launch; with the
    // columns of K, K^T and D held in shared memory when one block's share fits. Above
    // kLzFusedMaxN the three matrices stream from DRAM, where the per-step launches keep
    // more loads in flight than the cooperative grid.
    const bool fused = !small && !hyOp && n <= kLzFusedMaxN;
    int lzGrid = 0;
    bool lzCached = false;
    size_t lzSmem = 0;
    if (fused) {
        static std::atomic<int> capacity[kMaxDevices][2];
        static std::atomic<unsigned long long> attr{0};
        once_per_device(attr, [] {
            HB_CUDA(cudaFuncSetAttribute((const void *) lanczos_steps_smem_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, kLzSmemMax));
        });
        const int sms = device_sm_count();
        const int cpbCached = (n + sms - 1) / sms;
        const size_t need = sizeof(double) * (size_t) (lz_cached_doubles(n, cpbCached) + n);
        lzCached = need <= (size_t) kLzSmemMax;
        const int slot = lzCached ? 1 : 0;
        int cap = capacity[current_device()][slot].load(std::memory_order_relaxed);
        if (!cap) {
            int per = 0;
            if (lzCached)
                cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, lanczos_steps_smem_kernel, kLzThreads, kLzSmemMax);
            else
                cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, lanczos_steps_kernel, kLzThreads, 0);
            cap = std::max(1, per) * sms;
            capacity[current_device()][slot].store(cap, std::memory_order_relaxed);
        }
        if (lzCached) {
            // one block per SM, so that every block's columns fit its shared memory
            lzGrid = std::min(std::min(cap, sms), kLanczosMaxBlocks);
            const int cpb = (n + lzGrid - 1) / lzGrid;
            lzSmem = sizeof(double) * (size_t) (lz_cached_doubles(n, cpb) + n);
            if (lzSmem > (size_t) kLzSmemMax) lzCached = false;
        }
        if (!lzCached) {
            lzSmem = 0;
            lzGrid = std::max(1, std::min(std::min(cap, kLanczosMaxBlocks), (n + kLzCols - 1) / kLzCols));
        }
    }
    int stepsDone = 0;

    hdsdp_retcode ret = HDSDP_RETCODE_OK;
    bool done = false;
    int lastChecked = -1;
    const int freq = std::min(maxdim / 5, 3);
    std::vector<double> T, ev, evec;
    auto scheduled = [&](int k) { return ((k + 1) % freq == 0) || k >= maxdim - 1; };
    for (int k = 0; k < maxdim && !done; ++k) {
        if (fused) {
            if (k >= stepsDone) {
                int k1 = k;
                while (!scheduled(k1)) ++k1;
                k1 += 1;  // through the next check
                const double *Kp = F.K, *KTp = F.KT, *Dp = D;
                long ldk = F.ld, ldd = ldD, ldv = ld;
                int nn = n, md = maxdim, ka = k, kb = k1;
                double *Vp = V, *abp = d_ab, *tp = t1, *up = u, *wp = w, *pp = part;
                if (lzCached) {
                    void *args[] = {&nn, &Kp, &KTp, &ldk, &Dp, &ldd, &Vp, &ldv, &abp, &md, &ka, &kb, &wp, &tp, &up, &pp};
                    HB_CUDA(cudaLaunchCooperativeKernel((const void *) lanczos_steps_smem_kernel, hb::counted(lzGrid),
                                                        kLzThreads, args, lzSmem, s));
                } else {
                    void *args[] = {&nn, &Kp, &KTp, &ldk, &Dp, &ldd, &Vp, &ldv, &abp, &md, &ka, &kb, &tp, &up, &wp, &pp};
                    HB_CUDA(cudaLaunchCooperativeKernel((const void *) lanczos_steps_kernel, hb::counted(lzGrid),
                                                        kLzThreads, args, 0, s));
                }
                if (tm) tm->n_lanczos_mv += k1 - k;
                stepsDone = k1;
            }
        } else if (!small) {
            mv(V + (size_t) k * ld, w);
            lanczos_orth_kernel<<<hb::counted(1), 1024, 0, s>>>(n, V, ld, k, w, d_ab, maxdim);
        }
        const bool sched = scheduled(k);
        if (!sched) continue;
        if (!small) {
            HB_CUDA(cudaMemcpyAsync(h_ab, d_ab, sizeof(double) * (2 * maxdim + 2), cudaMemcpyDeviceToHost, s));
            double tw = wall();
            HB_CUDA(cudaStreamSynchronize(s));
            if (tm) tm->lz_wait += wall() - tw;
        }
        double th = wall();
        // The reference also checks as soon as a step breaks down (zero norm).
        int kc = k;
        for (int q = lastChecked + 1; q <= k; ++q)
            if (h_ab[maxdim + q] == 0.0) { kc = q; break; }
        lastChecked = k;
        const int kp1 = kc + 1;
        if (kp1 < 2) {  // two eigenpairs cannot be extracted from a 1 x 1 problem
            ret = HDSDP_RETCODE_FAILED;
            break;
        }
        std::vector<double> dd(h_ab, h_ab + kp1), ee(h_ab + maxdim, h_ab + maxdim + kp1);
        ee[kp1 - 1] = 0.0;
        tridiag_eig(kp1, dd, ee, ev, evec);
        if (tm) tm->lz_host += wall() - th;
        int i1 = 0, i2 = 0;  // largest, second largest
        for (int i = 1; i < kp1; ++i)
            if (ev[i] > ev[i1]) i1 = i;
        i2 = (i1 == 0) ? 1 : 0;
        for (int i = 0; i < kp1; ++i)
            if (i != i1 && ev[i] > ev[i2]) i2 = i;
        const double betak = h_ab[maxdim + kc];
        const double resiVal = std::fabs(betak * evec[(size_t) kc + (size_t) i1 * kp1]);
        if (!(resiVal < 1e-04 || kc >= maxdim - 1)) {
            if (kc != k) { done = true; }  // unreachable for a breakdown (resiVal == 0)
            continue;
        }
        const double eigMin1 = ev[i1], eigMin2 = ev[i2];
        std::vector<double> yy(2 * kp1);
        for (int i = 0; i < kp1; ++i) {
            yy[i] = evec[(size_t) i + (size_t) i1 * kp1];
            yy[kp1 + i] = evec[(size_t) i + (size_t) i2 * kp1];
        }
        HB_CUDA(cudaMemcpyAsync(d_y, yy.data(), sizeof(double) * 2 * kp1, cudaMemcpyHostToDevice, s));
        if (small) {
            lanczos_small_ritz_kernel<<<hb::counted(1), 256, small_lanczos_smem(n, maxdim), s>>>(
                n, F.K, F.ld, D, ldD, V, ld, kp1, d_y, eigMin1, warm, d_scal);
            HB_CUDA(cudaGetLastError());
            if (tm) tm->n_lanczos_mv += 2;
        } else {
            lanczos_combine_kernel<<<hb::counted((n + 255) / 256), 256, 0, s>>>(n, V, ld, kp1, d_y, z1);
            mv(z1, z2);
            HB_CUDA(cudaMemcpyAsync(warm, z2, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
            lanczos_resid_kernel<<<hb::counted(1), 1024, 0, s>>>(n, z2, z1, eigMin1, d_scal);
            lanczos_combine_kernel<<<hb::counted((n + 255) / 256), 256, 0, s>>>(n, V, ld, kp1, d_y + kp1, z2);
            mv(z2, z1);
            lanczos_resid_kernel<<<hb::counted(1), 1024, 0, s>>>(n, z1, z2, eigMin1, d_scal + 1);
        }
        HB_CUDA(cudaMemcpyAsync(h_scal, d_scal, sizeof(double) * 2, cudaMemcpyDeviceToHost, s));
        HB_CUDA(cudaStreamSynchronize(s));
        const double resiVal1 = h_scal[0], resiVal2 = h_scal[1];
        const double resiDiff = eigMin1 - eigMin2 - resiVal2;
        double valGamma = (resiDiff > 0) ? resiDiff : 1e-16;
        const double sq = resiVal1 * resiVal1 / valGamma;
        valGamma = std::min(resiVal1, sq);
        if (valGamma < 1e-03 || valGamma + eigMin1 <= 0.5) {
            *maxStep = (valGamma + eigMin1 <= 0.0) ? HDSDP_INFINITY : 1.0 / (valGamma + eigMin1);
            done = true;
        } else {
            if (betak == 0.0) {
                ret = HDSDP_RETCODE_FAILED;
                break;
            }
            *maxStep = 1.0 / (valGamma + eigMin1);
            if (kc != k) done = true;
        }
    }
    HB_CUDA(cudaStreamSynchronize(s));
    if (ret == HDSDP_RETCODE_OK) nComputed += 1;
    if (tm) {
        tm->lanczos += wall() - t0;
        tm->n_lanczos += 1;
    }
    return ret;
}

// The small-block path of Lanczos::solve for several cones at once: their steps in one
// launch, then the host replays each cone's check schedule; the Ritz evaluations that the
// checks of one round ask for run in one launch and one wait. Per cone, every value and
// decision is the one Lanczos::solve computes.
namespace {
struct LzRun {
    LzTask *t;
    int k = 0, lastChecked = -1;
    bool done = false;
    double host_s = 0.0;   // seconds of host eigensolves (summed into the timers afterwards)
    // the Ritz evaluation asked for
    int kc = 0;
    double eigMin1 = 0, eigMin2 = 0, betak = 0;
    std::vector<double> ev, evec;
};

// runs the schedule from step k on; true when a Ritz evaluation is needed (its
// coefficients uploaded), false when the run has ended
bool lz_advance(LzRun &R) {
    Lanczos &L = *R.t->lz;
    const int maxdim = L.maxdim;
    const int freq = std::min(maxdim / 5, 3);
    auto scheduled = [&](int k) { return ((k + 1) % freq == 0) || k >= maxdim - 1; };
    for (; R.k < maxdim && !R.done; ++R.k) {
        const int k = R.k;
        if (!scheduled(k)) continue;
        const double th = wall();
        int kc = k;
        for (int q = R.lastChecked + 1; q <= k; ++q)
            if (L.h_ab[maxdim + q] == 0.0) { kc = q; break; }
        R.lastChecked = k;
        const int kp1 = kc + 1;
        if (kp1 < 2) {
            R.t->ret = HDSDP_RETCODE_FAILED;
            R.done = true;
            return false;
        }
        std::vector<double> dd(L.h_ab, L.h_ab + kp1), ee(L.h_ab + maxdim, L.h_ab + maxdim + kp1);
        ee[kp1 - 1] = 0.0;
        tridiag_eig(kp1, dd, ee, R.ev, R.evec);
        R.host_s += wall() - th;
        int i1 = 0, i2 = 0;
        for (int i = 1; i < kp1; ++i)
            if (R.ev[i] > R.ev[i1]) i1 = i;
        i2 = (i1 == 0) ? 1 : 0;
        for (int i = 0; i < kp1; ++i)
            if (i != i1 && R.ev[i] > R.ev[i2]) i2 = i;
        const double betak = L.h_ab[maxdim + kc];
        const double resiVal = std::fabs(betak * R.evec[(size_t) kc + (size_t) i1 * kp1]);
        if (!(resiVal < 1e-04 || kc >= maxdim - 1)) {
            if (kc != k) R.done = true;
            continue;
        }
        R.kc = kc;
        R.eigMin1 = R.ev[i1];
        R.eigMin2 = R.ev[i2];
        R.betak = betak;
        std::vector<double> yy(2 * kp1);
        for (int i = 0; i < kp1; ++i) {
            yy[i] = R.evec[(size_t) i + (size_t) i1 * kp1];
            yy[kp1 + i] = R.evec[(size_t) i + (size_t) i2 * kp1];
        }
        if (L.dm_yv) std::memcpy(L.h_yv, yy.data(), sizeof(double) * 2 * kp1);   // read by the kernel in place
        else HB_CUDA(cudaMemcpyAsync(L.d_y, yy.data(), sizeof(double) * 2 * kp1, cudaMemcpyHostToDevice, L.s));
        return true;
    }
    return false;
}

// the outcome of the Ritz evaluation in h_scal; the schedule then moves on past step k
void lz_ritz_done(LzRun &R) {
    Lanczos &L = *R.t->lz;
    const double resiVal1 = L.h_scal[0], resiVal2 = L.h_scal[1];
    const double resiDiff = R.eigMin1 - R.eigMin2 - resiVal2;
    double valGamma = (resiDiff > 0) ? resiDiff : 1e-16;
    const double sq = resiVal1 * resiVal1 / valGamma;
    valGamma = std::min(resiVal1, sq);
    if (valGamma < 1e-03 || valGamma + R.eigMin1 <= 0.5) {
        *R.t->maxStep = (valGamma + R.eigMin1 <= 0.0) ? HDSDP_INFINITY : 1.0 / (valGamma + R.eigMin1);
        R.done = true;
    } else {
        if (R.betak == 0.0) {
            R.t->ret = HDSDP_RETCODE_FAILED;
            R.done = true;
            return;
        }
        *R.t->maxStep = 1.0 / (valGamma + R.eigMin1);
        if (R.kc != R.k) R.done = true;
    }
    R.k += 1;
}
}  // namespace

void lanczos_small_batch(std::vector<LzTask> &tasks) {
    if (tasks.empty()) return;
    const double t0 = wall();
    cudaStream_t s = tasks[0].lz->s;
    Timers *tm = tasks[0].tm;
    static std::atomic<unsigned long long> attr{0};
    once_per_device(attr, [] {
        const int bytes = (int) small_lanczos_smem(kSmallLanczosN, 30);
        lz_allow_smem<LzStepJob>(bytes);
        lz_allow_smem<LzRitzJob>(bytes);
    });
    for (LzTask &t : tasks) {
        t.ret = HDSDP_RETCODE_OK;
        compute_inverse_factor(s, *t.F);
    }
    if (tm) tm->lz_inverse += wall() - t0;   // enqueue time: the steps' launch follows without a wait
    int maxn = 0, maxdim = 0;
    for (LzTask &t : tasks) {
        maxn = std::max(maxn, t.lz->n);
        maxdim = std::max(maxdim, t.lz->maxdim);
    }
    const size_t smem = small_lanczos_smem(maxn, maxdim);
    // device addresses of the pinned mirrors (alpha / beta and the Ritz residuals), which
    // the kernels write directly; a task without one gets copies
    std::vector<double *> hab(tasks.size()), hsc(tasks.size());
    std::vector<LzStepJob> steps(tasks.size());
    for (size_t q = 0; q < tasks.size(); ++q) {
        LzTask &t = tasks[q];
        Lanczos &L = *t.lz;
        hab[q] = L.dm_ab;
        hsc[q] = L.dm_scal;
        steps[q] = LzStepJob{t.F->K, t.D, L.nComputed == 0 ? nullptr : L.warm,
                             L.nComputed == 0 ? L.init_vec : L.pert_vec, L.V, L.d_ab, hab[q], t.F->ld, t.ldD,
                             L.ld, L.n, L.maxdim};
    }
    lz_launch(s, steps, smem);
    for (size_t q = 0; q < tasks.size(); ++q) {
        Lanczos &L = *tasks[q].lz;
        if (!hab[q])
            HB_CUDA(cudaMemcpyAsync(L.h_ab, L.d_ab, sizeof(double) * (2 * L.maxdim + 2), cudaMemcpyDeviceToHost, s));
        if (tm) tm->n_lanczos_mv += L.maxdim;
    }
    HB_CUDA(cudaStreamSynchronize(s));
    // the host replays of the cones are independent: with many cones they run on several
    // host threads (each cone's own steps stay in order, so every value is the same)
    std::vector<LzRun> runs(tasks.size());
    std::vector<LzRun *> want;
    const int nrun = (int) runs.size();
    std::vector<char> ask(nrun, 0);
    for (int q = 0; q < nrun; ++q) runs[q].t = &tasks[q];
    const bool par0 = nrun >= kLzHostParallel;
    (void) par0;
#pragma omp parallel for schedule(dynamic, 1) if (par0)
    for (int q = 0; q < nrun; ++q) ask[q] = lz_advance(runs[q]) ? 1 : 0;
    for (int q = 0; q < nrun; ++q)
        if (ask[q]) want.push_back(&runs[q]);
    while (!want.empty()) {
        std::vector<LzRitzJob> ritz(want.size());
        for (size_t q = 0; q < want.size(); ++q) {
            LzRun &R = *want[q];
            Lanczos &L = *R.t->lz;
            ritz[q] = LzRitzJob{R.t->F->K, R.t->D, L.V, L.dm_yv ? L.dm_yv : L.d_y, L.warm, L.d_scal,
                                hsc[R.t - tasks.data()], R.t->F->ld, R.t->ldD, L.ld, R.eigMin1, L.n, R.kc + 1};
        }
        lz_launch(s, ritz, smem);
        for (LzRun *R : want) {
            Lanczos &L = *R->t->lz;
            if (!hsc[R->t - tasks.data()])
                HB_CUDA(cudaMemcpyAsync(L.h_scal, L.d_scal, sizeof(double) * 2, cudaMemcpyDeviceToHost, s));
            if (tm) tm->n_lanczos_mv += 2;
        }
        HB_CUDA(cudaStreamSynchronize(s));
        const int nw = (int) want.size();
        std::vector<char> again(nw, 0);
        const bool par = nw >= kLzHostParallel;
        (void) par;
#pragma omp parallel for schedule(dynamic, 1) if (par)
        for (int q = 0; q < nw; ++q) {
            lz_ritz_done(*want[q]);
            again[q] = lz_advance(*want[q]) ? 1 : 0;
        }
        std::vector<LzRun *> next;
        for (int q = 0; q < nw; ++q)
            if (again[q]) next.push_back(want[q]);
        want.swap(next);
    }
    if (tm)
        for (const LzRun &R : runs) tm->lz_host += R.host_s;
    for (LzTask &t : tasks)
        if (t.ret == HDSDP_RETCODE_OK) t.lz->nComputed += 1;
    if (tm) {
        tm->lanczos += wall() - t0;
        tm->n_lanczos += (long) tasks.size();
    }
}

}  // namespace hb
