// Dense FP64 linear algebra kernels for sm_100a.
//
// The GEMM issues FP64 tensor-core MMAs (mma.sync m8n8k4 .f64, the DMMA
// path); Blackwell's tcgen05 has no f64 kind, so this is the FP64 tensor
// instruction on B200. Every factorisation routine below reduces to this
// GEMM plus small 64 x 64 kernels.
#include "la.h"
#include <vector>
#include <mutex>
#include <unordered_map>
#include <cmath>
#include <algorithm>

namespace hb {

int &device_error_flag() {
    static int flag = 0;
    return flag;
}

int current_device() {
    int d = 0;
    if (cudaGetDevice(&d) != cudaSuccess || d < 0 || d >= kMaxDevices) d = 0;
    return d;
}

namespace {
std::mutex &init_mutex() {
    static std::mutex *mu = new std::mutex();  // never destroyed: set-up may run during exit
    return *mu;
}
}  // namespace

void once_per_device(std::atomic<unsigned long long> &mask, const std::function<void()> &fn) {
    const unsigned long long bit = 1ull << current_device();
    if (mask.load(std::memory_order_acquire) & bit) return;
    std::lock_guard<std::mutex> g(init_mutex());
    if (mask.load(std::memory_order_relaxed) & bit) return;
    fn();
    mask.fetch_or(bit, std::memory_order_release);
}

int device_sm_count() {
    static std::atomic<int> sms[kMaxDevices];
    const int d = current_device();
    int v = sms[d].load(std::memory_order_relaxed);
    if (v > 0) return v;
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, d);
    if (v <= 0) v = 1;
    sms[d].store(v, std::memory_order_relaxed);
    return v;
}

namespace {
struct BlockCache {
    std::mutex mu;
    std::unordered_map<size_t, std::vector<void *>> free_dev, free_host;
    std::unordered_map<void *, size_t> size_dev, size_host;
};
BlockCache &block_cache() {
    static BlockCache *c = new BlockCache();  // never destroyed: frees may run during exit
    return *c;
}
}  // namespace

long long &alloc_counter() {
    static long long count = 0;
    return count;
}

cudaError_t cache_malloc(void **p, size_t bytes) {
    __atomic_fetch_add(&alloc_counter(), 1LL, __ATOMIC_RELAXED);
    BlockCache &c = block_cache();
    if (bytes == 0) bytes = 1;
    {
        std::lock_guard<std::mutex> g(c.mu);
        auto it = c.free_dev.find(bytes);
        if (it != c.free_dev.end() && !it->second.empty()) {
            *p = it->second.back();
            it->second.pop_back();
            return cudaSuccess;
        }
    }
    cudaError_t e = cudaMalloc(p, bytes);
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        cache_release();
        e = cudaMalloc(p, bytes);
    }
    if (e == cudaSuccess) {
        std::lock_guard<std::mutex> g(c.mu);
        c.size_dev[*p] = bytes;
    } else {
        *p = nullptr;
    }
    return e;
}

void cache_free(void *p) {
    if (!p) return;
    BlockCache &c = block_cache();
    std::lock_guard<std::mutex> g(c.mu);
    auto it = c.size_dev.find(p);
    if (it == c.size_dev.end()) {
        cudaFree(p);  // not ours: hand it back directly
        return;
    }
    c.free_dev[it->second].push_back(p);
}

cudaError_t cache_malloc_host(void **p, size_t bytes) {
    __atomic_fetch_add(&alloc_counter(), 1LL, __ATOMIC_RELAXED);
    BlockCache &c = block_cache();
    if (bytes == 0) bytes = 1;
    {
        std::lock_guard<std::mutex> g(c.mu);
        auto it = c.free_host.find(bytes);
        if (it != c.free_host.end() && !it->second.empty()) {
            *p = it->second.back();
            it->second.pop_back();
            return cudaSuccess;
        }
    }
    cudaError_t e = cudaMallocHost(p, bytes);
    if (e == cudaSuccess) {
        std::lock_guard<std::mutex> g(c.mu);
        c.size_host[*p] = bytes;
    } else {
        *p = nullptr;
    }
    return e;
}

void cache_free_host(void *p) {
    if (!p) return;
    BlockCache &c = block_cache();
    std::lock_guard<std::mutex> g(c.mu);
    auto it = c.size_host.find(p);
    if (it == c.size_host.end()) {
        cudaFreeHost(p);
        return;
    }
    c.free_host[it->second].push_back(p);
}

void cache_release() {
    BlockCache &c = block_cache();
    std::lock_guard<std::mutex> g(c.mu);
    for (auto &kv : c.free_dev)
        for (void *q : kv.second) {
            cudaFree(q);
            c.size_dev.erase(q);
        }
    for (auto &kv : c.free_host)
        for (void *q : kv.second) {
            cudaFreeHost(q);
            c.size_host.erase(q);
        }
    c.free_dev.clear();
    c.free_host.clear();
}

long long &launch_counter() {
    static long long count = 0;
    return count;
}

namespace {
struct KStatRec {
    int family;
    cudaEvent_t e0, e1;
    double work;
};
struct KStatState {
    int mask = 0;
    std::vector<KStatRec> pending;
    std::vector<cudaEvent_t> pool;
    long long launches[KF_COUNT] = {};
    double ms[KF_COUNT] = {}, work[KF_COUNT] = {};
    cudaEvent_t take() {
        cudaEvent_t e;
        if (!pool.empty()) {
            e = pool.back();
            pool.pop_back();
        } else {
            HB_CUDA(cudaEventCreate(&e));
        }
        return e;
    }
    void resolve() {
        for (KStatRec &r : pending) {
            float t = 0.f;
            HB_CUDA(cudaEventSynchronize(r.e1));
            HB_CUDA(cudaEventElapsedTime(&t, r.e0, r.e1));
            launches[r.family] += 1;
            ms[r.family] += t;
            work[r.family] += r.work;
            pool.push_back(r.e0);
            pool.push_back(r.e1);
        }
        pending.clear();
    }
};
KStatState &kstat() {
    static KStatState st;
    return st;
}
}  // namespace

void kstat_enable(int mask) {
    KStatState &st = kstat();
    st.resolve();
    st.mask = mask;
    for (int f = 0; f < KF_COUNT; ++f) {
        st.launches[f] = 0;
        st.ms[f] = st.work[f] = 0.0;
    }
}

bool kstat_on(int family) { return (kstat().mask >> family) & 1; }

void kstat_begin(int family, cudaStream_t s, double work) {
    KStatState &st = kstat();
    KStatRec r{family, st.take(), st.take(), work};
    HB_CUDA(cudaEventRecord(r.e0, s));
    st.pending.push_back(r);
}

void kstat_end(cudaStream_t s) {
    KStatState &st = kstat();
    HB_CUDA(cudaEventRecord(st.pending.back().e1, s));
    if (st.pending.size() > 4096) st.resolve();
}

int kstat_read(int family, long long *launches, double *ms, double *work) {
    if (family < 0 || family >= KF_COUNT) return -1;
    KStatState &st = kstat();
    st.resolve();
    if (launches) *launches = st.launches[family];
    if (ms) *ms = st.ms[family];
    if (work) *work = st.work[family];
    return 0;
}

// ------------------------------------------------------------------------------------
// GEMM: 64 x 64 x 16 CTA tile, 4 warps (2 x 2), 32 x 32 warp tile of 8 x 8 DMMA tiles.
// ------------------------------------------------------------------------------------
namespace {
constexpr int BM = 64, BN = 64, BK = 16, GT = 128;

using GemmP = GemmDesc;

__device__ __forceinline__ void dmma(double &d0, double &d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

__device__ __forceinline__ double load_a(const GemmP &p, int m, int k) {
    if (m >= p.M || k >= p.K) return 0.0;
    if ((p.flags & GEMM_A_LOWER) && k > m) return 0.0;
    if ((p.flags & GEMM_A_UPPER) && k < m) return 0.0;
    return p.ta ? p.A[(size_t) k + (size_t) m * p.lda] : p.A[(size_t) m + (size_t) k * p.lda];
}

__device__ __forceinline__ double load_b(const GemmP &p, int k, int n) {
    if (n >= p.N || k >= p.K) return 0.0;
    if ((p.flags & GEMM_B_LOWER) && k < n) return 0.0;
    if ((p.flags & GEMM_B_UPPER) && k > n) return 0.0;
    return p.tb ? p.B[(size_t) n + (size_t) k * p.ldb] : p.B[(size_t) k + (size_t) n * p.ldb];
}

// one 64 x 64 tile (bx, by) of C
__device__ __forceinline__ void gemm_tile(const GemmP &p, int bx, int by) {
    const int m0 = bx * BM;
    const int n0 = by * BN;
    if ((p.flags & GEMM_C_LOWER) && m0 + BM - 1 < n0) return;
    if (p.abort_flag && *p.abort_flag) return;

    int kmin = 0, kmax = p.K;
    if (p.flags & GEMM_A_LOWER) kmax = min(kmax, m0 + BM);
    if (p.flags & GEMM_A_UPPER) kmin = max(kmin, m0);
    if (p.flags & GEMM_B_LOWER) kmin = max(kmin, n0);
    if (p.flags & GEMM_B_UPPER) kmax = min(kmax, n0 + BN);
    kmin = (kmin / BK) * BK;

    __shared__ double As[2][BK][BM + 4];
    __shared__ double Bs[2][BK][BN + 4];

    const int t = threadIdx.x;
    const int lane = t & 31;
    const int w = t >> 5;
    const int wm = (w & 1) * 32;
    const int wn = (w >> 1) * 32;

    double acc[4][4][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

    double ra[8], rb[8];
    auto gload = [&](int k0) {
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            int r, kk;
            if (!p.ta) { r = t & 63; kk = (t >> 6) + 2 * i; }
            else { kk = t & 15; r = (t >> 4) + 8 * i; }
            ra[i] = load_a(p, m0 + r, k0 + kk);
            int c, kb;
            if (!p.tb) { kb = t & 15; c = (t >> 4) + 8 * i; }
            else { c = t & 63; kb = (t >> 6) + 2 * i; }
            rb[i] = load_b(p, k0 + kb, n0 + c);
        }
    };
    auto sstore = [&](int buf) {
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            int r, kk;
            if (!p.ta) { r = t & 63; kk = (t >> 6) + 2 * i; }
            else { kk = t & 15; r = (t >> 4) + 8 * i; }
            As[buf][kk][r] = ra[i];
            int c, kb;
            if (!p.tb) { kb = t & 15; c = (t >> 4) + 8 * i; }
            else { c = t & 63; kb = (t >> 6) + 2 * i; }
            Bs[buf][kb][c] = rb[i];
        }
    };

    if (kmin < kmax) {
        gload(kmin);
        sstore(0);
        __syncthreads();
        int buf = 0;
        for (int k0 = kmin; k0 < kmax; k0 += BK) {
            const bool more = (k0 + BK) < kmax;
            if (more) gload(k0 + BK);
#pragma unroll
            for (int ks = 0; ks < BK; ks += 4) {
                double a[4], b[4];
#pragma unroll
                for (int i = 0; i < 4; ++i) a[i] = As[buf][ks + (lane & 3)][wm + i * 8 + (lane >> 2)];
#pragma unroll
                for (int j = 0; j < 4; ++j) b[j] = Bs[buf][ks + (lane & 3)][wn + j * 8 + (lane >> 2)];
#pragma unroll
                for (int i = 0; i < 4; ++i)
#pragma unroll
                    for (int j = 0; j < 4; ++j) dmma(acc[i][j][0], acc[i][j][1], a[i], b[j]);
            }
            if (more) sstore(buf ^ 1);
            __syncthreads();
            buf ^= 1;
        }
    }

#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int row = m0 + wm + i * 8 + (lane >> 2);
        if (row >= p.M) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const int col = n0 + wn + j * 8 + (lane & 3) * 2 + e;
                if (col >= p.N) continue;
                if ((p.flags & GEMM_C_LOWER) && row < col) continue;
                double *cp = p.C + (size_t) row + (size_t) col * p.ldc;
                double v = p.alpha * acc[i][j][e];
                if (p.beta != 0.0) v += p.beta * (*cp);
                *cp = v;
            }
        }
    }
}

__global__ void __launch_bounds__(GT) gemm_kernel(GemmP p) { gemm_tile(p, blockIdx.x, blockIdx.y); }

// one GEMM of a group per blockIdx.z (tiles beyond its own M x N exit)
__global__ void __launch_bounds__(GT) gemm_grouped_kernel(const GemmP *__restrict__ ps) {
    const GemmP p = ps[blockIdx.z];
    if ((int) blockIdx.x * BM >= p.M || (int) blockIdx.y * BN >= p.N) return;
    gemm_tile(p, blockIdx.x, blockIdx.y);
}
}  // namespace

void gemm_grouped(cudaStream_t s, const GemmDesc *d_desc, int count, int maxM, int maxN) {
    if (count <= 0 || maxM <= 0 || maxN <= 0) return;
    for (int z0 = 0; z0 < count; z0 += 65535) {
        dim3 grid((maxM + BM - 1) / BM, (maxN + BN - 1) / BN, std::min(65535, count - z0));
        gemm_grouped_kernel<<<hb::counted(grid), GT, 0, s>>>(d_desc + z0);
        HB_CUDA(cudaGetLastError());
    }
}

// ------------------------------------------------------------------------------------
// Large-tile GEMM: 128 x 128 x 16 CTA tile, 8 warps (4 along M x 2 along N), warp tile
// 32 x 64 = 4 x 8 DMMA fragments, 3-stage cp.async pipeline with zero-fill predicates.
// Shared-memory layout per operand follows its global contiguity so the loads stay
// coalesced; row pitches of 132 / 20 doubles make the fragment reads conflict-free.
// ------------------------------------------------------------------------------------
namespace {
constexpr int L_BM = 128, L_BN = 128, L_BK = 16, L_T = 256, L_ST = 3;
constexpr int L_PK = L_BM + 4;   // pitch of a k-major tile row (128 contiguous elements)
constexpr int L_PM = L_BK + 4;   // pitch of an m/n-major tile row (16 contiguous k)
constexpr int L_STAGE = 2560;    // doubles per operand per stage (max of 16*132, 128*20)

__device__ __forceinline__ void cp_async8(double *sdst, const double *gsrc, bool pred) {
    const unsigned saddr = (unsigned) __cvta_generic_to_shared(sdst);
    const int bytes = pred ? 8 : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(saddr), "l"(gsrc), "r"(bytes));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

template <int TA, int TB>
__global__ void __launch_bounds__(L_T) gemm_large_kernel(GemmP p) {
    const int m0 = blockIdx.x * L_BM;
    const int n0 = blockIdx.y * L_BN;
    if ((p.flags & GEMM_C_LOWER) && m0 + L_BM - 1 < n0) return;
    if (p.abort_flag && *p.abort_flag) return;
    int kmin = 0, kmax = p.K;
    if (p.flags & GEMM_A_LOWER) kmax = min(kmax, m0 + L_BM);
    if (p.flags & GEMM_A_UPPER) kmin = max(kmin, m0);
    if (p.flags & GEMM_B_LOWER) kmin = max(kmin, n0);
    if (p.flags & GEMM_B_UPPER) kmax = min(kmax, n0 + L_BN);
    kmin = (kmin / L_BK) * L_BK;
    const int nk = (kmax > kmin) ? (kmax - kmin + L_BK - 1) / L_BK : 0;

    extern __shared__ double smem[];
    double *As = smem;
    double *Bs = smem + L_ST * L_STAGE;
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    const int wm = (w & 3) * 32, wn = (w >> 2) * 64;

    auto issue = [&](int kt, int stage) {
        const int k0 = kmin + kt * L_BK;
        double *as = As + stage * L_STAGE;
        double *bs = Bs + stage * L_STAGE;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            int m, k;
            if (!TA) { m = t & 127; k = (t >> 7) + 2 * i; }
            else { k = t & 15; m = (t >> 4) + 16 * i; }
            const int gm = m0 + m, gk = k0 + k;
            bool ok = gm < p.M && gk < p.K;
            if ((p.flags & GEMM_A_LOWER) && gk > gm) ok = false;
            if ((p.flags & GEMM_A_UPPER) && gk < gm) ok = false;
            const double *src = ok ? (TA ? p.A + (size_t) gk + (size_t) gm * p.lda : p.A + (size_t) gm + (size_t) gk * p.lda) : p.A;
            double *dst = TA ? as + m * L_PM + k : as + k * L_PK + m;
            cp_async8(dst, src, ok);
        }
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            int n, k;
            if (!TB) { k = t & 15; n = (t >> 4) + 16 * i; }
            else { n = t & 127; k = (t >> 7) + 2 * i; }
            const int gn = n0 + n, gk = k0 + k;
            bool ok = gn < p.N && gk < p.K;
            if ((p.flags & GEMM_B_LOWER) && gk < gn) ok = false;
            if ((p.flags & GEMM_B_UPPER) && gk > gn) ok = false;
            const double *src = ok ? (TB ? p.B + (size_t) gn + (size_t) gk * p.ldb : p.B + (size_t) gk + (size_t) gn * p.ldb) : p.B;
            double *dst = TB ? bs + k * L_PK + n : bs + n * L_PM + k;
            cp_async8(dst, src, ok);
        }
    };

    double acc[4][8][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

#pragma unroll
    for (int st = 0; st < L_ST - 1; ++st) {
        if (st < nk) issue(st, st);
        cp_commit();
    }
    for (int kt = 0; kt < nk; ++kt) {
        cp_wait<L_ST - 2>();
        __syncthreads();
        const int nxt = kt + L_ST - 1;
        if (nxt < nk) issue(nxt, nxt % L_ST);
        cp_commit();
        const double *as = As + (kt % L_ST) * L_STAGE;
        const double *bs = Bs + (kt % L_ST) * L_STAGE;
#pragma unroll
        for (int ks = 0; ks < L_BK; ks += 4) {
            const int kk = ks + (lane & 3);
            double a[4], b[8];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int m = wm + i * 8 + (lane >> 2);
                a[i] = TA ? as[m * L_PM + kk] : as[kk * L_PK + m];
            }
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int n = wn + j * 8 + (lane >> 2);
                b[j] = TB ? bs[kk * L_PK + n] : bs[n * L_PM + kk];
            }
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 8; ++j) dmma(acc[i][j][0], acc[i][j][1], a[i], b[j]);
        }
    }
    cp_wait<0>();

#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int row = m0 + wm + i * 8 + (lane >> 2);
        if (row >= p.M) continue;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const int col = n0 + wn + j * 8 + (lane & 3) * 2 + e;
                if (col >= p.N) continue;
                if ((p.flags & GEMM_C_LOWER) && row < col) continue;
                double *cp = p.C + (size_t) row + (size_t) col * p.ldc;
                double v = p.alpha * acc[i][j][e];
                if (p.beta != 0.0) v += p.beta * (*cp);
                *cp = v;
            }
        }
    }
}

constexpr int L_SMEM = 2 * L_ST * L_STAGE * (int) sizeof(double);

template <int TA, int TB>
void launch_large(const GemmP &p, cudaStream_t s) {
    static std::atomic<unsigned long long> init{0};
    once_per_device(init, [] {
        HB_CUDA(cudaFuncSetAttribute(gemm_large_kernel<TA, TB>, cudaFuncAttributeMaxDynamicSharedMemorySize, L_SMEM));
    });
    dim3 grid((p.M + L_BM - 1) / L_BM, (p.N + L_BN - 1) / L_BN);
    gemm_large_kernel<TA, TB><<<hb::counted(grid), L_T, L_SMEM, s>>>(p);
}
}  // namespace

void gemm(cudaStream_t s, int M, int N, int K, double alpha, const double *A, long lda, int transA,
          const double *B, long ldb, int transB, double beta, double *C, long ldc, int flags,
          const int *abort_flag) {
    if (M <= 0 || N <= 0) return;
    GemmP p{M, N, K, alpha, beta, A, lda, transA, B, ldb, transB, C, ldc, flags, abort_flag};
    const bool timed = kstat_on(KF_GEMM);
    if (timed) {
        // algorithmic flops: halve for a triangular output or a triangular operand
        double f = 2.0 * M * N * (double) K;
        if (flags & GEMM_C_LOWER) f *= 0.5;
        if (flags & (GEMM_A_LOWER | GEMM_A_UPPER)) f *= 0.5;
        if (flags & (GEMM_B_LOWER | GEMM_B_UPPER)) f *= 0.5;
        kstat_begin(KF_GEMM, s, f);
    }
    // Large tiles once the 128 x 128 grid fills the machine; 64 x 64 tiles otherwise.
    const long tiles = (long) ((M + L_BM - 1) / L_BM) * ((N + L_BN - 1) / L_BN);
    if (tiles >= 96 && K >= 64) {
        if (!transA && !transB) launch_large<0, 0>(p, s);
        else if (transA && !transB) launch_large<1, 0>(p, s);
        else if (!transA && transB) launch_large<0, 1>(p, s);
        else launch_large<1, 1>(p, s);
    } else {
        dim3 grid((M + BM - 1) / BM, (N + BN - 1) / BN);
        gemm_kernel<<<hb::counted(grid), GT, 0, s>>>(p);
    }
    HB_CUDA(cudaGetLastError());
    if (timed) kstat_end(s);
}

// ------------------------------------------------------------------------------------
// Column-dot matrix-vector product (one warp per output entry).
// ------------------------------------------------------------------------------------
namespace {
__global__ void coldot_kernel(int nrows, int ncols, const double *__restrict__ A, long lda,
                              const double *__restrict__ x, double *out, double alpha, double beta,
                              int mode) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= ncols) return;
    const int i = warp;
    int lo = 0, hi = nrows;
    if (mode == 1) lo = i;
    else if (mode == 2) hi = min(nrows, i + 1);
    const double *col = A + (size_t) i * lda;
    double acc = 0.0;
    int k = lo + lane;
    for (; k + 96 < hi; k += 128) {
        acc += col[k] * x[k] + col[k + 32] * x[k + 32] + col[k + 64] * x[k + 64] + col[k + 96] * x[k + 96];
    }
    for (; k < hi; k += 32) acc += col[k] * x[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) {
        double v = alpha * acc;
        if (beta != 0.0) v += beta * out[i];
        out[i] = v;
    }
}
}  // namespace

// One block of S warps per column: the column's row range is cut into S segments of a
// multiple of 32 rows, each warp reduces its segment, and warp 0 combines them. Used when
// one warp per column would leave the SMs with too few loads in flight.
template <int S>
__global__ void __launch_bounds__(32 * S) coldot_seg_kernel(int nrows, const double *__restrict__ A, long lda,
                                                          const double *__restrict__ x, double *out, double alpha,
                                                          double beta, int mode) {
    __shared__ double part[S];
    const int i = blockIdx.x, w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int lo = 0, hi = nrows;
    if (mode == 1) lo = i;
    else if (mode == 2) hi = min(nrows, i + 1);
    const int len = max(hi - lo, 0);
    const int chunk = (((len + S - 1) / S) + 31) & ~31;
    const int k0 = lo + w * chunk, k1 = min(hi, k0 + chunk);
    const double *col = A + (size_t) i * lda;
    double acc = 0.0;
    int k = k0 + lane;
    for (; k + 96 < k1; k += 128) {
        acc += col[k] * x[k] + col[k + 32] * x[k + 32] + col[k + 64] * x[k + 64] + col[k + 96] * x[k + 96];
    }
    for (; k < k1; k += 32) acc += col[k] * x[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) part[w] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
#pragma unroll
        for (int q = 0; q < S; ++q) t += part[q];
        double v = alpha * t;
        if (beta != 0.0) v += beta * out[i];
        out[i] = v;
    }
}

void coldot(cudaStream_t s, int nrows, int ncols, const double *A, long lda, const double *x,
            double *out, double alpha, double beta, int mode) {
    if (ncols <= 0) return;
    if (ncols < 4096 && nrows >= 256) {
        // few columns: several warps per column keep enough loads in flight
        if (ncols < 1024)
            coldot_seg_kernel<8><<<hb::counted(ncols), 256, 0, s>>>(nrows, A, lda, x, out, alpha, beta, mode);
        else
            coldot_seg_kernel<4><<<hb::counted(ncols), 128, 0, s>>>(nrows, A, lda, x, out, alpha, beta, mode);
    } else {
        const int threads = 256;
        const long warps = ncols;
        const int blocks = (int) ((warps * 32 + threads - 1) / threads);
        coldot_kernel<<<hb::counted(blocks), threads, 0, s>>>(nrows, ncols, A, lda, x, out, alpha, beta, mode);
    }
    HB_CUDA(cudaGetLastError());
}

// ------------------------------------------------------------------------------------
// Cholesky: 64 x 64 diagonal-block factorisation + inverse, panel solve, SYRK update.
// ------------------------------------------------------------------------------------
namespace {
constexpr int NB = 64;

// Factorise the nb x nb diagonal block at (j0, j0) in shared memory, write it back,
// and store its triangular inverse in Dinv rows [j0, j0 + nb), columns [0, nb).
__global__ void __launch_bounds__(256) potf2_kernel(double *A, long lda, int nb, int j0, double *Dinv,
                                                    long ldd, int *info) {
    if (*info) return;
    extern __shared__ double sm[];
    double *T = sm;                 // T[r + c * 65]
    double *Ti = sm + 65 * 64;      // inverse
    __shared__ int fail;
    const int tid = threadIdx.x;
    for (int idx = tid; idx < nb * nb; idx += blockDim.x) {
        int r = idx % nb, c = idx / nb;
        T[r + c * 65] = (r >= c) ? A[(size_t) (j0 + r) + (size_t) (j0 + c) * lda] : 0.0;
    }
    if (tid == 0) fail = 0;
    __syncthreads();
    for (int c = 0; c < nb; ++c) {
        if (tid == 0) {
            double d = T[c + c * 65];
            if (!(d > 0.0)) fail = c + 1;
            else T[c + c * 65] = sqrt(d);
        }
        __syncthreads();
        if (fail) break;
        const double piv = T[c + c * 65];
        for (int r = c + 1 + tid; r < nb; r += blockDim.x) T[r + c * 65] /= piv;
        __syncthreads();
        const int rem = nb - c - 1;
        for (int idx = tid; idx < rem * rem; idx += blockDim.x) {
            int r = c + 1 + idx % rem, q = c + 1 + idx / rem;
            if (r >= q) T[r + q * 65] -= T[r + c * 65] * T[q + c * 65];
        }
        __syncthreads();
    }
    if (fail) {
        if (tid == 0) *info = j0 + fail;
        return;
    }
    for (int idx = tid; idx < nb * nb; idx += blockDim.x) {
        int r = idx % nb, c = idx / nb;
        if (r >= c) A[(size_t) (j0 + r) + (size_t) (j0 + c) * lda] = T[r + c * 65];
    }
    // Triangular inverse, one column per thread (forward substitution on e_c).
    if (tid < nb) {
        const int c = tid;
        for (int r = 0; r < c; ++r) Ti[r + c * 65] = 0.0;
        Ti[c + c * 65] = 1.0 / T[c + c * 65];
        for (int r = c + 1; r < nb; ++r) {
            double acc = 0.0;
            for (int k = c; k < r; ++k) acc += T[r + k * 65] * Ti[k + c * 65];
            Ti[r + c * 65] = -acc / T[r + r * 65];
        }
    }
    __syncthreads();
    for (int idx = tid; idx < NB * NB; idx += blockDim.x) {
        int r = idx % NB, c = idx / NB;
        double v = (r < nb && c < nb) ? Ti[r + c * 65] : 0.0;
        if (r < nb) Dinv[(size_t) (j0 + r) + (size_t) c * ldd] = v;
    }
}

// P (rows x nb, in place) <- P * Tinv^T for the panel below a diagonal block.
__global__ void __launch_bounds__(256) trsm_panel_kernel(double *P, long ldp, int rows, int nb,
                                                         const double *Tinv, long ldt, const int *info) {
    if (*info) return;
    extern __shared__ double sm[];
    double *X = sm;             // 64 x nb, X[r + c*65]
    double *T = sm + 65 * 64;   // nb x nb, T[r + c*65]
    const int r0 = blockIdx.x * 64;
    const int tid = threadIdx.x;
    const int nr = min(64, rows - r0);
    for (int idx = tid; idx < 64 * nb; idx += blockDim.x) {
        int r = idx % 64, c = idx / 64;
        X[r + c * 65] = (r < nr) ? P[(size_t) (r0 + r) + (size_t) c * ldp] : 0.0;
    }
    for (int idx = tid; idx < nb * nb; idx += blockDim.x) {
        int r = idx % nb, c = idx / nb;
        T[r + c * 65] = Tinv[(size_t) r + (size_t) c * ldt];
    }
    __syncthreads();
    // out(r, c) = sum_{k <= c} X(r, k) * T(c, k)
    for (int idx = tid; idx < 64 * nb; idx += blockDim.x) {
        int r = idx % 64, c = idx / 64;
        if (r >= nr) continue;
        double acc = 0.0;
        for (int k = 0; k <= c; ++k) acc += X[r + k * 65] * T[c + k * 65];
        P[(size_t) (r0 + r) + (size_t) c * ldp] = acc;
    }
}

// X row block (nb x cols, in place) <- Tinv * X, Tinv lower nb x nb.
__global__ void __launch_bounds__(256) tri_left_kernel(double *X, long ldx, int nb, int cols,
                                                       const double *Tinv, long ldt) {
    extern __shared__ double sm[];
    double *Xs = sm;             // nb x 64
    double *T = sm + 65 * 64;
    const int c0 = blockIdx.x * 64;
    const int nc = min(64, cols - c0);
    const int tid = threadIdx.x;
    for (int idx = tid; idx < nb * 64; idx += blockDim.x) {
        int r = idx % nb, c = idx / nb;
        Xs[r + c * 65] = (c < nc) ? X[(size_t) r + (size_t) (c0 + c) * ldx] : 0.0;
    }
    for (int idx = tid; idx < nb * nb; idx += blockDim.x) {
        int r = idx % nb, c = idx / nb;
        T[r + c * 65] = Tinv[(size_t) r + (size_t) c * ldt];
    }
    __syncthreads();
    for (int idx = tid; idx < nb * 64; idx += blockDim.x) {
        int r = idx % nb, c = idx / nb;
        if (c >= nc) continue;
        double acc = 0.0;
        for (int k = 0; k <= r; ++k) acc += T[r + k * 65] * Xs[k + c * 65];
        X[(size_t) r + (size_t) (c0 + c) * ldx] = acc;
    }
}

__global__ void copy_lower_kernel(int n, const double *S, long lds, double *L, long ldl) {
    const long total = (long) n * n;
    for (long idx = blockIdx.x * (long) blockDim.x + threadIdx.x; idx < total; idx += (long) gridDim.x * blockDim.x) {
        int r = (int) (idx % n), c = (int) (idx / n);
        L[(size_t) r + (size_t) c * ldl] = (r >= c) ? S[(size_t) r + (size_t) c * lds] : 0.0;
    }
}

__global__ void set_identity_kernel(int n, double *A, long lda) {
    const long total = (long) n * n;
    for (long idx = blockIdx.x * (long) blockDim.x + threadIdx.x; idx < total; idx += (long) gridDim.x * blockDim.x) {
        int r = (int) (idx % n), c = (int) (idx / n);
        A[(size_t) r + (size_t) c * lda] = (r == c) ? 1.0 : 0.0;
    }
}

__global__ void zero_int_kernel(int *p) { *p = 0; }

int grid_for(long total, int threads = 256) {
    long b = (total + threads - 1) / threads;
    return (int) std::min<long>(std::max<long>(b, 1), 148L * 16);
}
}  // namespace

void DenseFactor::alloc(int n_, int fuse_inverse) {
    // the solve scratch is sized for n: drop any from an earlier size
    if (d_flags) hb::cache_free(d_flags);
    if (d_tmp) hb::cache_free(d_tmp);
    if (d_rec_w) hb::cache_free(d_rec_w);
    if (d_rec_ks) hb::cache_free(d_rec_ks);
    if (d_rec_kts) hb::cache_free(d_rec_kts);
    d_flags = nullptr;
    d_tmp = nullptr;
    d_rec_w = nullptr;
    d_rec_ks = d_rec_kts = nullptr;
    epoch = 0;
    n = n_;
    ld = pad_ld(n);
    HB_CUDA(hb::cmalloc(&L, sizeof(double) * ld * n));
    HB_CUDA(hb::cmalloc(&Dinv, sizeof(double) * ld * NB));
    // the info word and, 8 bytes on, sum log L_ii of the last factorisation
    HB_CUDA(hb::cmalloc(&d_info, 2 * sizeof(double)));
    HB_CUDA(hb::cmalloc_host(&h_info, 2 * sizeof(double)));
    *h_info = 0;
    stat_logdet = true;
    logdet_valid = false;
    HB_CUDA(cudaMemset(L, 0, sizeof(double) * ld * n));
    HB_CUDA(cudaMemset(Dinv, 0, sizeof(double) * ld * NB));
    fuse_k = (fuse_inverse < 0) ? (n <= kFuseInverseMax) : (fuse_inverse != 0);
    if (fuse_k) {
        HB_CUDA(hb::cmalloc(&K, sizeof(double) * ld * n));
        HB_CUDA(hb::cmalloc(&KT, sizeof(double) * ld * n));
        HB_CUDA(cudaMemset(K, 0, sizeof(double) * ld * n));
        HB_CUDA(cudaMemset(KT, 0, sizeof(double) * ld * n));
    }
    legacy_fence();
}

void DenseFactor::release() {
    if (L) hb::cache_free(L);
    if (Dinv) hb::cache_free(Dinv);
    if (K) hb::cache_free(K);
    if (KT) hb::cache_free(KT);
    if (d_info) hb::cache_free(d_info);
    if (d_flags) hb::cache_free(d_flags);
    if (d_tmp) hb::cache_free(d_tmp);
    if (d_rec_info) hb::cache_free(d_rec_info);
    if (d_rec_w) hb::cache_free(d_rec_w);
    if (d_rec_ks) hb::cache_free(d_rec_ks);
    if (d_rec_kts) hb::cache_free(d_rec_kts);
    d_flags = nullptr;
    d_tmp = nullptr;
    d_rec_info = nullptr;
    d_rec_w = nullptr;
    d_rec_ks = d_rec_kts = nullptr;
    epoch = 0;
    if (h_info) hb::cache_free_host(h_info);
    L = Dinv = K = KT = nullptr;
    d_info = nullptr;
    h_info = nullptr;
    factored = ok = k_valid = fuse_k = k_pending = false;
}

static void set_smem(const void *fn, int bytes) {
    HB_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
}

static int smem_bytes() { return 2 * 65 * 64 * (int) sizeof(double); }

static void ensure_attrs() {
    static std::atomic<unsigned long long> init{0};
    once_per_device(init, [] {
        set_smem((const void *) potf2_kernel, smem_bytes());
        set_smem((const void *) trsm_panel_kernel, smem_bytes());
        set_smem((const void *) tri_left_kernel, smem_bytes());
    });
}

bool coop_factorize_enqueue(cudaStream_t s, DenseFactor &F, const double *S, long ldS);
bool rec_factorize_enqueue(cudaStream_t s, DenseFactor &F, const double *S, long ldS);
bool rec_factorize_nok_enqueue(cudaStream_t s, DenseFactor &F, const double *S, long ldS);
bool coop_inverse_enqueue(cudaStream_t s, DenseFactor &F);

void factorize_async(cudaStream_t s, DenseFactor &F, const double *S, long ldS) {
    ensure_attrs();
    const int n = F.n;
    F.k_valid = false;
    F.k_pending = false;
    F.factored = true;
    F.logdet_valid = false;
    // info word (and sum log L_ii) back to the host in one copy
    auto status_copy = [&]() {
        if (F.stat_logdet) {
            log_diag_sum(s, F, reinterpret_cast<double *>(F.d_info) + 1);
            HB_CUDA(cudaMemcpyAsync(F.h_info, F.d_info, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
        } else {
            HB_CUDA(cudaMemcpyAsync(F.h_info, F.d_info, sizeof(int), cudaMemcpyDeviceToHost, s));
        }
    };
    if (F.fuse_k && F.K && F.KT && !F.no_rec && n > kRecMinN && rec_factorize_enqueue(s, F, S, ldS)) {
        F.k_pending = true;
        status_copy();
        return;
    }
    if (!F.fuse_k && !F.no_rec && n > kRecNoKMinN && rec_factorize_nok_enqueue(s, F, S, ldS)) {
        F.k_pending = false;
        status_copy();
        return;
    }
    if (coop_factorize_enqueue(s, F, S, ldS)) {
        F.k_pending = F.fuse_k && F.K && F.KT;
        status_copy();
        return;
    }
    zero_int_kernel<<<hb::counted(1), 1, 0, s>>>(F.d_info);
    copy_lower_kernel<<<hb::counted(grid_for((long) n * n)), 256, 0, s>>>(n, S, ldS, F.L, F.ld);
    for (int j0 = 0; j0 < n; j0 += NB) {
        const int nb = std::min(NB, n - j0);
        potf2_kernel<<<hb::counted(1), 256, smem_bytes(), s>>>(F.L, F.ld, nb, j0, F.Dinv, F.ld, F.d_info);
        const int rows = n - j0 - nb;
        if (rows > 0) {
            double *P = F.L + (size_t) (j0 + nb) + (size_t) j0 * F.ld;
            trsm_panel_kernel<<<hb::counted((rows + 63) / 64), 256, smem_bytes(), s>>>(P, F.ld, rows, nb,
                                                                         F.Dinv + j0, F.ld, F.d_info);
            double *A22 = F.L + (size_t) (j0 + nb) + (size_t) (j0 + nb) * F.ld;
            gemm(s, rows, rows, nb, -1.0, P, F.ld, 0, P, F.ld, 1, 1.0, A22, F.ld, GEMM_C_LOWER, F.d_info);
        }
    }
    status_copy();
    HB_CUDA(cudaGetLastError());
}

bool small_factor_batch_enqueue(cudaStream_t s, DenseFactor *const *F, const double *const *S, const long *ldS,
                                int count);

void factorize_small_batch(cudaStream_t s, DenseFactor *const *F, const double *const *S, const long *ldS, int count) {
    if (count <= 0) return;
    ensure_attrs();
    if (!small_factor_batch_enqueue(s, F, S, ldS, count)) {
        for (int q = 0; q < count; ++q) factorize_async(s, *F[q], S[q], ldS[q]);
        return;
    }
    for (int q = 0; q < count; ++q) {
        DenseFactor &G = *F[q];
        G.k_valid = false;
        G.k_pending = G.fuse_k && G.K && G.KT;
        G.factored = true;
        G.logdet_valid = false;
    }
}

bool factor_status_ready(DenseFactor &F) {
    F.ok = (*(volatile int *) F.h_info == 0);
    F.k_valid = F.ok && F.k_pending;
    F.k_pending = false;
    F.logdet_valid = F.ok && F.stat_logdet;
    if (F.logdet_valid) F.logdet = 2.0 * reinterpret_cast<const volatile double *>(F.h_info)[1];
    return F.ok;
}

bool factor_status(cudaStream_t s, DenseFactor &F) {
    HB_CUDA(cudaStreamSynchronize(s));
    F.ok = (*F.h_info == 0);
    F.k_valid = F.ok && F.k_pending;  // K and KT were formed by the factorisation kernel
    F.k_pending = false;
    F.logdet_valid = F.ok && F.stat_logdet;
    if (F.logdet_valid) F.logdet = 2.0 * reinterpret_cast<const double *>(F.h_info)[1];
    return F.ok;
}

bool factorize(cudaStream_t s, DenseFactor &F, const double *S, long ldS) {
    factorize_async(s, F, S, ldS);
    return factor_status(s, F);
}

void compute_inverse_factor(cudaStream_t s, DenseFactor &F) {
    ensure_attrs();
    if (F.k_valid) return;
    const int n = F.n;
    if (!F.K) HB_CUDA(hb::cmalloc(&F.K, sizeof(double) * F.ld * n));
    if (!F.KT) HB_CUDA(hb::cmalloc(&F.KT, sizeof(double) * F.ld * n));
    if (coop_inverse_enqueue(s, F)) {
        transpose(s, n, F.K, F.ld, F.KT, F.ld);
        F.k_valid = true;
        return;
    }
    set_identity_kernel<<<hb::counted(grid_for((long) n * n)), 256, 0, s>>>(n, F.K, F.ld);
    for (int i0 = 0; i0 < n; i0 += NB) {
        const int nb = std::min(NB, n - i0);
        const int cend = i0 + nb;
        tri_left_kernel<<<hb::counted((cend + 63) / 64), 256, smem_bytes(), s>>>(F.K + i0, F.ld, nb, cend, F.Dinv + i0, F.ld);
        const int rows = n - cend;
        if (rows > 0) {
            gemm(s, rows, cend, nb, -1.0, F.L + (size_t) cend + (size_t) i0 * F.ld, F.ld, 0, F.K + i0, F.ld, 0,
                 1.0, F.K + cend, F.ld, 0);
        }
    }
    transpose(s, n, F.K, F.ld, F.KT, F.ld);
    F.k_valid = true;
}

void compute_inverse(cudaStream_t s, DenseFactor &F, double *W, long ldW) {
    compute_inverse_factor(s, F);
    const int n = F.n;
    gemm(s, n, n, n, 1.0, F.K, F.ld, 1, F.K, F.ld, 0, 0.0, W, ldW, GEMM_C_LOWER | GEMM_A_UPPER | GEMM_B_LOWER);
    symmetrize_lower(s, n, W, ldW);
}

// ------------------------------------------------------------------------------------
// Small reductions and elementwise helpers.
// ------------------------------------------------------------------------------------
namespace {
__device__ double block_sum(double v) {
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
    }
    __syncthreads();
    return v;
}

__global__ void logdiag_kernel(int n, const double *L, long ld, double *out) {
    double acc = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) acc += log(L[(size_t) i + (size_t) i * ld]);
    acc = block_sum(acc);
    if (threadIdx.x == 0) *out = acc;
}

__global__ void copydiag_kernel(int n, const double *L, long ld, double *out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        out[i] = L[(size_t) i + (size_t) i * ld];
}

__global__ void fill_kernel(double *x, double v, size_t n) {
    for (size_t i = blockIdx.x * (size_t) blockDim.x + threadIdx.x; i < n; i += (size_t) gridDim.x * blockDim.x) x[i] = v;
}

__global__ void axpy_kernel(int n, double a, const double *x, double *y) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] += a * x[i];
}

// Upper triangle := lower triangle, by 32 x 32 tiles: the block of tile (bi, bj), bi <= bj,
// reads lower tile (bj, bi) along its columns into shared memory and writes upper tile
// (bi, bj) along its columns, so both sides are coalesced.
__global__ void symlower_kernel(int n, double *A, long lda) {
    __shared__ double tile[32][33];
    const int bi = blockIdx.x, bj = blockIdx.y;
    if (bi > bj) return;
    const int tx = threadIdx.x, ty = threadIdx.y;   // 32 x 8 threads
    for (int k = ty; k < 32; k += 8) {
        const int r = bj * 32 + tx, c = bi * 32 + k;   // lower tile (bj, bi): row r, column c
        if (r < n && c < n && r >= c) tile[k][tx] = A[(size_t) r + (size_t) c * lda];
    }
    __syncthreads();
    for (int k = ty; k < 32; k += 8) {
        const int r = bi * 32 + tx, c = bj * 32 + k;   // upper tile (bi, bj): row r, column c = element (c, r)
        if (r < n && c < n && r < c) A[(size_t) r + (size_t) c * lda] = tile[tx][k];
    }
}

__global__ void symavg_kernel(int n, double *A, long lda) {
    const long total = (long) n * n;
    for (long idx = blockIdx.x * (long) blockDim.x + threadIdx.x; idx < total; idx += (long) gridDim.x * blockDim.x) {
        int r = (int) (idx % n), c = (int) (idx / n);
        if (r > c) {
            double a = A[(size_t) r + (size_t) c * lda], b = A[(size_t) c + (size_t) r * lda];
            double v = 0.5 * (a + b);
            A[(size_t) r + (size_t) c * lda] = v;
            A[(size_t) c + (size_t) r * lda] = v;
        }
    }
}

__global__ void adddiag_kernel(int n, double *A, long lda, double v) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        A[(size_t) i + (size_t) i * lda] += v;
}

__global__ void adddiagvec_kernel(int n, double *A, long lda, const double *d) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        A[(size_t) i + (size_t) i * lda] += d[i];
}

__global__ void copymat_kernel(int rows, int cols, const double *A, long lda, double *B, long ldb) {
    const long total = (long) rows * cols;
    for (long idx = blockIdx.x * (long) blockDim.x + threadIdx.x; idx < total; idx += (long) gridDim.x * blockDim.x) {
        int r = (int) (idx % rows), c = (int) (idx / rows);
        B[(size_t) r + (size_t) c * ldb] = A[(size_t) r + (size_t) c * lda];
    }
}

__global__ void transpose_kernel(int n, const double *A, long lda, double *B, long ldb) {
    __shared__ double tile[32][33];
    const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        int r = bx + threadIdx.x, c = by + j;
        if (r < n && c < n) tile[j][threadIdx.x] = A[(size_t) r + (size_t) c * lda];
    }
    __syncthreads();
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        int r = by + threadIdx.x, c = bx + j;
        if (r < n && c < n) B[(size_t) r + (size_t) c * ldb] = tile[threadIdx.x][j];
    }
}

__global__ void scalemat_kernel(int rows, int cols, double *A, long lda, double a) {
    const long total = (long) rows * cols;
    for (long idx = blockIdx.x * (long) blockDim.x + threadIdx.x; idx < total; idx += (long) gridDim.x * blockDim.x) {
        int r = (int) (idx % rows), c = (int) (idx / rows);
        A[(size_t) r + (size_t) c * lda] *= a;
    }
}

__global__ void scalecols_kernel(int rows, int cols, const double *A, long lda, const double *d, double *B, long ldb) {
    const long total = (long) rows * cols;
    for (long idx = blockIdx.x * (long) blockDim.x + threadIdx.x; idx < total; idx += (long) gridDim.x * blockDim.x) {
        int r = (int) (idx % rows), c = (int) (idx / rows);
        B[(size_t) r + (size_t) c * ldb] = A[(size_t) r + (size_t) c * lda] * d[c];
    }
}

// Deterministic two-level reduction: each block reduces a fixed slice, then block 0
// of a second launch sums the partials.
__global__ void frob_partial_kernel(int n, const double *A, long lda, const double *B, long ldb, double *part) {
    double acc = 0.0;
    const long total = (long) n * n;
    for (long idx = blockIdx.x * (long) blockDim.x + threadIdx.x; idx < total; idx += (long) gridDim.x * blockDim.x) {
        int r = (int) (idx % n), c = (int) (idx / n);
        acc += A[(size_t) r + (size_t) c * lda] * B[(size_t) r + (size_t) c * ldb];
    }
    acc = block_sum(acc);
    if (threadIdx.x == 0) part[blockIdx.x] = acc;
}

__global__ void sum_partials_kernel(int np, const double *part, double *out) {
    double acc = 0.0;
    for (int i = threadIdx.x; i < np; i += blockDim.x) acc += part[i];
    acc = block_sum(acc);
    if (threadIdx.x == 0) *out = acc;
}

__global__ void trace_kernel(int n, const double *A, long lda, double *out) {
    double acc = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) acc += A[(size_t) i + (size_t) i * lda];
    acc = block_sum(acc);
    if (threadIdx.x == 0) *out = acc;
}

__global__ void dot_kernel(int n, const double *x, const double *y, double *out) {
    double acc = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) acc += x[i] * y[i];
    acc = block_sum(acc);
    if (threadIdx.x == 0) *out = acc;
}
}  // namespace

void log_diag_sum(cudaStream_t s, const DenseFactor &F, double *d_out) {
    logdiag_kernel<<<hb::counted(1), 1024, 0, s>>>(F.n, F.L, F.ld, d_out);
    HB_CUDA(cudaGetLastError());
}

void copy_diag(cudaStream_t s, const DenseFactor &F, double *d_out) {
    copydiag_kernel<<<hb::counted(grid_for(F.n)), 256, 0, s>>>(F.n, F.L, F.ld, d_out);
}

void fill(cudaStream_t s, double *x, double v, size_t n) {
    if (!n) return;
    fill_kernel<<<hb::counted(grid_for((long) n)), 256, 0, s>>>(x, v, n);
}

void axpy(cudaStream_t s, int n, double a, const double *x, double *y) {
    if (n <= 0) return;
    axpy_kernel<<<hb::counted(grid_for(n)), 256, 0, s>>>(n, a, x, y);
}

void symmetrize_lower(cudaStream_t s, int n, double *A, long lda) {
    if (n <= 0) return;
    const int nt = (n + 31) / 32;
    symlower_kernel<<<hb::counted(dim3(nt, nt)), dim3(32, 8), 0, s>>>(n, A, lda);
}

void symmetrize_avg(cudaStream_t s, int n, double *A, long lda) {
    symavg_kernel<<<hb::counted(grid_for((long) n * n)), 256, 0, s>>>(n, A, lda);
}

void add_diag(cudaStream_t s, int n, double *A, long lda, double v) {
    adddiag_kernel<<<hb::counted(grid_for(n)), 256, 0, s>>>(n, A, lda, v);
}

void add_diag_vec(cudaStream_t s, int n, double *A, long lda, const double *d) {
    adddiagvec_kernel<<<hb::counted(grid_for(n)), 256, 0, s>>>(n, A, lda, d);
}

void copy_matrix(cudaStream_t s, int rows, int cols, const double *A, long lda, double *B, long ldb) {
    if (rows <= 0 || cols <= 0) return;
    copymat_kernel<<<hb::counted(grid_for((long) rows * cols)), 256, 0, s>>>(rows, cols, A, lda, B, ldb);
}

void transpose(cudaStream_t s, int n, const double *A, long lda, double *B, long ldb) {
    dim3 grid((n + 31) / 32, (n + 31) / 32), block(32, 8);
    transpose_kernel<<<hb::counted(grid), block, 0, s>>>(n, A, lda, B, ldb);
}

void scale_matrix(cudaStream_t s, int rows, int cols, double *A, long lda, double a) {
    scalemat_kernel<<<hb::counted(grid_for((long) rows * cols)), 256, 0, s>>>(rows, cols, A, lda, a);
}

void scale_columns(cudaStream_t s, int rows, int cols, const double *A, long lda, const double *d,
                   double *B, long ldb) {
    scalecols_kernel<<<hb::counted(grid_for((long) rows * cols)), 256, 0, s>>>(rows, cols, A, lda, d, B, ldb);
}

void frob_dot(cudaStream_t s, int n, const double *A, long lda, const double *B, long ldb, double *d_out) {
    // partial sums in a buffer of the stream's own: solver objects on different streams
    // (one per host thread) must not share it
    static std::mutex mu;
    static std::unordered_map<cudaStream_t, double *> parts;
    const int np = 296;
    double *part = nullptr;
    {
        std::lock_guard<std::mutex> g(mu);
        double *&p = parts[s];
        if (!p) HB_CUDA(hb::cmalloc(&p, sizeof(double) * np));
        part = p;
    }
    if (!part) return;
    frob_partial_kernel<<<hb::counted(np), 256, 0, s>>>(n, A, lda, B, ldb, part);
    sum_partials_kernel<<<hb::counted(1), 512, 0, s>>>(np, part, d_out);
}

void trace(cudaStream_t s, int n, const double *A, long lda, double *d_out) {
    trace_kernel<<<hb::counted(1), 1024, 0, s>>>(n, A, lda, d_out);
}

void dot(cudaStream_t s, int n, const double *x, const double *y, double *d_out) {
    dot_kernel<<<hb::counted(1), 1024, 0, s>>>(n, x, y, d_out);
}

}  // namespace hb
