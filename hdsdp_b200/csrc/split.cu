// BF16x3 split-precision GEMM on tcgen05 with TMA-fed shared-memory stages
// and FP32 accumulators in tensor memory (see split.h).
#include "split.h"
#include <cudaTypedefs.h>
#include <algorithm>
#include <cstdio>

namespace hb {

namespace {

constexpr int BM = 128, BN = 128, BK = 64;  // BK = 64 BF16 = one 128-byte swizzle row
constexpr int STAGES = 3;
constexpr int TILE_BYTES = BM * BK * 2;     // 16 KB per operand tile
constexpr int STAGE_BYTES = 4 * TILE_BYTES; // A hi, A lo, B hi, B lo of one K block: all three products
constexpr int THREADS = 192;                // warp 0 TMA, warp 1 MMA + TMEM owner, warps 2-5 epilogue
constexpr int TMEM_COLS = 2 * BN;           // two FP32 accumulators: one tile drains while the next accumulates
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024 /* alignment */ + 256 /* barriers */;
constexpr long WAIT_LIMIT = 1L << 24;       // bounded mbarrier polls (about a second)

__device__ int g_split_err = 0;

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t) __cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count));
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    return done != 0;
}

// Bounded wait: gives up (raising the error flag) after WAIT_LIMIT polls or
// once another thread of the grid has raised it.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    for (long it = 0; it < WAIT_LIMIT; ++it) {
        if (mbar_try(bar, parity)) return true;
        if ((it & 1023) == 1023 && *(volatile int *) &g_split_err) return false;
    }
    atomicExch(&g_split_err, 1);
    return false;
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap *map, int x, int y, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            dst),
        "l"(map), "r"(x), "r"(y), "r"(bar)
        : "memory");
}

// Shared-memory matrix descriptor of a K-major tile with 128-byte rows,
// 128-byte swizzle, 8-row groups 1024 bytes apart (tcgen05 descriptor version 1).
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr) {
    uint64_t d = (uint64_t) ((saddr & 0x3FFFF) >> 4);
    d |= (uint64_t) 1 << 16;             // leading byte offset (unused for swizzled K-major)
    d |= (uint64_t) (1024 >> 4) << 32;   // stride byte offset: next 8-row group
    d |= (uint64_t) 1 << 46;             // descriptor version
    d |= (uint64_t) 2 << 61;             // 128-byte swizzle
    return d;
}

// Instruction descriptor: BF16 x BF16 -> FP32, both operands K-major, M = BM, N = BN.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t) (BN >> 3) << 17) |
                            ((uint32_t) (BM >> 4) << 24);

__device__ __forceinline__ void mma_bf16(uint32_t tmem, uint64_t a, uint64_t b, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
        "l"(a), "l"(b), "r"(kIdesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float *v) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int j = 0; j < 32; ++j) v[j] = __uint_as_float(r[j]);
}

struct KernelArgs {
    int M, N, nkb;             // nkb: K blocks per product (K padded to 64)
    int tiles_m, tiles_n;
    int lower_tiles, a_lower, a_upper;
    int epi;
    double alpha, beta;
    double *C;
    long ldc;
    __nv_bfloat16 *out_hi, *out_lo;
    long out_ld;
    int out_rows;              // rows of the output operand (N extent) that exist
    double *colsq;
};

__device__ __forceinline__ void tile_of(const KernelArgs &p, int b, int &tm, int &tn) {
    if (p.lower_tiles) {
        // b -> (tm, tn) with tn <= tm, row by row
        int t = (int) ((sqrt(8.0 * b + 1.0) - 1.0) * 0.5);
        while ((t + 1) * (t + 2) / 2 <= b) ++t;
        while (t * (t + 1) / 2 > b) --t;
        tm = t;
        tn = b - t * (t + 1) / 2;
    } else {
        tm = b % p.tiles_m;
        tn = b / p.tiles_m;
    }
}

// Persistent: each CTA takes one tile per round of gridDim.x tiles (see tile_seq). The
// producer warp streams K blocks of
// all its tiles through a ring of stages, each holding the four operand tiles of one
// K block (A hi, A lo, B hi, B lo), from which the MMA thread issues the three
// products hi*hi, hi*lo, lo*hi into one FP32 accumulator. Tiles alternate between two
// accumulators in tensor memory, so the epilogue warps drain one tile while the next
// one accumulates.
__global__ void __launch_bounds__(THREADS, 1)
    split_gemm_kernel(const __grid_constant__ CUtensorMap a_hi, const __grid_constant__ CUtensorMap a_lo,
                      const __grid_constant__ CUtensorMap b_hi, const __grid_constant__ CUtensorMap b_lo,
                      KernelArgs p) {
    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;
    uint8_t *gbase = smem_raw + (base - raw);
    // barriers: full[STAGES], empty[STAGES], acc_full[2], acc_empty[2], then the TMEM slot
    const uint32_t bar0 = base + STAGES * STAGE_BYTES;
    auto full = [&](int st) { return bar0 + 8u * st; };
    auto empty = [&](int st) { return bar0 + 8u * (STAGES + st); };
    auto acc_full = [&](int b) { return bar0 + 8u * (2 * STAGES + b); };
    auto acc_empty = [&](int b) { return bar0 + 8u * (2 * STAGES + 2 + b); };
    volatile uint32_t *tmem_slot = (volatile uint32_t *) (gbase + STAGES * STAGE_BYTES + 8 * (2 * STAGES + 4));

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ntiles = p.lower_tiles ? p.tiles_m * (p.tiles_m + 1) / 2 : p.tiles_m * p.tiles_n;
    // Tile i of this CTA (i = 0, 1, ...): rounds of gridDim.x tiles, dealt left to right
    // in even rounds and right to left in odd ones, which evens out the work when the
    // tiles' K ranges shrink along the tile order (triangular operands). Increasing in i.
    auto tile_seq = [&](int i) {
        const int pos = (i & 1) ? (int) gridDim.x - 1 - (int) blockIdx.x : (int) blockIdx.x;
        return i * (int) gridDim.x + pos;
    };
    // the K blocks a tile needs: [kfirst, klast)
    auto klast = [&](int m0) { return p.a_lower ? min(p.nkb, (m0 + BM + BK - 1) / BK) : p.nkb; };
    auto kfirst = [&](int m0) { return p.a_upper ? min(m0 / BK, p.nkb - 1) : 0; };

    if (threadIdx.x == 0) {
        for (int st = 0; st < STAGES; ++st) {
            mbar_init(full(st), 1);
            mbar_init(empty(st), 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(acc_full(b), 1);
            mbar_init(acc_empty(b), 4);  // one arrival per epilogue warp
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32((const void *) tmem_slot)),
                     "r"(TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0 && lane == 0) {
        // producer
        int it = 0;
        bool ok = true;
        for (int i = 0, tile; ok && (tile = tile_seq(i)) < ntiles; ++i) {
            int tm, tn;
            tile_of(p, tile, tm, tn);
            const int m0 = tm * BM, n0 = tn * BN, kb0 = kfirst(m0), kb1 = klast(m0);
            for (int kb = kb0; kb < kb1; ++kb, ++it) {
                const int st = it % STAGES;
                const uint32_t ph = (uint32_t) (it / STAGES) & 1u;
                if (!mbar_wait(empty(st), ph ^ 1u)) {
                    ok = false;
                    break;
                }
                mbar_expect_tx(full(st), STAGE_BYTES);
                const uint32_t sa = base + st * STAGE_BYTES;
                tma_load_2d(sa, &a_hi, kb * BK, m0, full(st));
                tma_load_2d(sa + TILE_BYTES, &a_lo, kb * BK, m0, full(st));
                tma_load_2d(sa + 2 * TILE_BYTES, &b_hi, kb * BK, n0, full(st));
                tma_load_2d(sa + 3 * TILE_BYTES, &b_lo, kb * BK, n0, full(st));
            }
        }
    } else if (warp == 1 && lane == 0) {
        // MMA issuer: per stage, four K=16 steps of each of the three products
        int it = 0;
        bool ok = true;
        for (int tc = 0, tile; ok && (tile = tile_seq(tc)) < ntiles; ++tc) {
            int tm, tn;
            tile_of(p, tile, tm, tn);
            const int kb0 = kfirst(tm * BM), kb1 = klast(tm * BM);
            const int b = tc & 1;
            if (!mbar_wait(acc_empty(b), ((uint32_t) (tc >> 1) & 1u) ^ 1u)) break;
            fence_after();
            const uint32_t d = tmem + (uint32_t) (b * BN);
            for (int kb = kb0; kb < kb1; ++kb, ++it) {
                const int st = it % STAGES;
                const uint32_t ph = (uint32_t) (it / STAGES) & 1u;
                if (!mbar_wait(full(st), ph)) {
                    ok = false;
                    break;
                }
                fence_after();
                const uint32_t sa = base + st * STAGE_BYTES;
                const uint64_t dah = smem_desc(sa), dal = smem_desc(sa + TILE_BYTES);
                const uint64_t dbh = smem_desc(sa + 2 * TILE_BYTES), dbl = smem_desc(sa + 3 * TILE_BYTES);
#pragma unroll
                for (int k = 0; k < BK / 16; ++k)
                    mma_bf16(d, dah + (uint64_t) (2 * k), dbh + (uint64_t) (2 * k), (kb != kb0 || k != 0) ? 1u : 0u);
#pragma unroll
                for (int k = 0; k < BK / 16; ++k) mma_bf16(d, dah + (uint64_t) (2 * k), dbl + (uint64_t) (2 * k), 1u);
#pragma unroll
                for (int k = 0; k < BK / 16; ++k) mma_bf16(d, dal + (uint64_t) (2 * k), dbh + (uint64_t) (2 * k), 1u);
                mma_commit(empty(st));
            }
            if (ok) mma_commit(acc_full(b));
        }
    } else if (warp >= 2) {
        // epilogue: warp w reads accumulator lanes 32 * (w % 4) ...
        const int q = warp & 3;
        for (int tc = 0, tile; (tile = tile_seq(tc)) < ntiles; ++tc) {
            int tm, tn;
            tile_of(p, tile, tm, tn);
            const int m0 = tm * BM, n0 = tn * BN;
            const int r = m0 + q * 32 + lane;
            const int b = tc & 1;
            if (!mbar_wait(acc_full(b), (uint32_t) (tc >> 1) & 1u)) break;
            fence_after();
            for (int c0 = 0; c0 < BN; c0 += 32) {
                float v[32];
                tmem_ld32(tmem + ((uint32_t) (q * 32) << 16) + (uint32_t) (b * BN + c0), v);
                if (p.epi == SPLIT_EPI_F64) {
                    if (r < p.M) {
#pragma unroll
                        for (int j = 0; j < 32; ++j) {
                            const int c = n0 + c0 + j;
                            if (c >= p.N || (p.lower_tiles && c > r)) continue;
                            double *dst = p.C + (size_t) r + (size_t) c * p.ldc;
                            double val = p.alpha * (double) v[j];
                            if (p.beta != 0.0) val += p.beta * *dst;
                            *dst = val;
                        }
                    }
                } else if (p.epi == SPLIT_EPI_SPLIT) {
                    if (r < p.out_ld) {
#pragma unroll
                        for (int j = 0; j < 32; ++j) {
                            const int c = n0 + c0 + j;
                            if (c >= p.out_rows) continue;
                            const float x = (float) p.alpha * v[j];
                            const __nv_bfloat16 h = __float2bfloat16_rn(x);
                            const __nv_bfloat16 l = __float2bfloat16_rn(x - __bfloat162float(h));
                            p.out_hi[(size_t) c * p.out_ld + r] = h;
                            p.out_lo[(size_t) c * p.out_ld + r] = l;
                        }
                    }
                } else {
#pragma unroll
                    for (int j = 0; j < 32; ++j) {
                        double sq = (r < p.M) ? (double) v[j] * (double) v[j] : 0.0;
#pragma unroll
                        for (int o = 16; o > 0; o >>= 1) sq += __shfl_xor_sync(0xffffffffu, sq, o);
                        const int c = n0 + c0 + j;
                        if (lane == 0 && c < p.N) atomicAdd(p.colsq + c, p.alpha * sq);
                    }
                }
            }
            // the accumulator may be overwritten once all four warps have read it
            fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(acc_empty(b));
        }
    }
    fence_before();
    __syncthreads();
    if (warp == 1) {
        fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS));
    }
}

// FP64 -> (hi, lo) BF16, K-major rows; X read with k contiguous (direct) or r contiguous (tiled transpose).
__global__ void split_direct_kernel(const double *__restrict__ X, long ld, int rows, int k, __nv_bfloat16 *hi,
                                    __nv_bfloat16 *lo, int rows_alloc, int kpad) {
    const long total = (long) rows_alloc * kpad;
    for (long t = blockIdx.x * (long) blockDim.x + threadIdx.x; t < total; t += (long) gridDim.x * blockDim.x) {
        const int r = (int) (t / kpad), kk = (int) (t - (long) r * kpad);
        const double x = (r < rows && kk < k) ? X[(size_t) kk + (size_t) r * ld] : 0.0;
        const __nv_bfloat16 h = __double2bfloat16(x);
        hi[t] = h;
        lo[t] = __double2bfloat16(x - (double) __bfloat162float(h));
    }
}

__global__ void split_transpose_kernel(const double *__restrict__ X, long ld, int rows, int k, __nv_bfloat16 *hi,
                                       __nv_bfloat16 *lo, int kpad) {
    __shared__ double tile[32][33];
    const int r0 = blockIdx.y * 32, k0 = blockIdx.x * 32;
    // read X(r, k) = X[r + k*ld] with r fastest
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        const int r = r0 + threadIdx.x, kk = k0 + j;
        tile[j][threadIdx.x] = (r < rows && kk < k) ? X[(size_t) r + (size_t) kk * ld] : 0.0;
    }
    __syncthreads();
    // write op(r, k) with k fastest
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        const int r = r0 + j, kk = k0 + threadIdx.x;
        const double x = tile[threadIdx.x][j];
        const __nv_bfloat16 h = __double2bfloat16(x);
        const size_t o = (size_t) r * kpad + kk;
        hi[o] = h;
        lo[o] = __double2bfloat16(x - (double) __bfloat162float(h));
    }
}

__global__ void read_err_kernel(int *out) {
    *out = g_split_err;
    g_split_err = 0;
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    // a driver entry point is process-wide: looked up once (thread-safe static init)
    static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            return (PFN_cuTensorMapEncodeTiled_v12000) p;
        return (PFN_cuTensorMapEncodeTiled_v12000) nullptr;
    }();
    return fn;
}

bool encode_map(CUtensorMap *map, __nv_bfloat16 *ptr, int rows_alloc, int kpad) {
    PFN_cuTensorMapEncodeTiled_v12000 fn = encode_fn();
    if (!fn) return false;
    cuuint64_t dims[2] = {(cuuint64_t) kpad, (cuuint64_t) rows_alloc};
    cuuint64_t strides[1] = {(cuuint64_t) kpad * 2};
    cuuint32_t box[2] = {BK, BM};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, ptr, dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

}  // namespace

bool SplitOperand::alloc(int rows_, int k_) {
    const int ra = ((rows_ + BM - 1) / BM) * BM, kp = ((k_ + BK - 1) / BK) * BK;
    if (hi && ra == rows_alloc && kp == kpad) {
        rows = rows_;
        k = k_;
        return true;
    }
    release();
    rows = rows_;
    k = k_;
    rows_alloc = ra;
    kpad = kp;
    const size_t bytes = (size_t) ra * kp * sizeof(__nv_bfloat16);
    HB_CUDA(hb::cmalloc(&hi, bytes));
    HB_CUDA(hb::cmalloc(&lo, bytes));
    HB_CUDA(cudaMemset(hi, 0, bytes));
    HB_CUDA(cudaMemset(lo, 0, bytes));
    legacy_fence();
    if (!hi || !lo) return false;
    return encode_map(&map_hi, hi, ra, kp) && encode_map(&map_lo, lo, ra, kp);
}

void SplitOperand::release() {
    if (hi) hb::cache_free(hi);
    if (lo) hb::cache_free(lo);
    hi = lo = nullptr;
    rows = k = rows_alloc = kpad = 0;
}

void split_from_f64(cudaStream_t s, SplitOperand &op, const double *X, long ld, bool k_contiguous) {
    if (k_contiguous) {
        const long total = (long) op.rows_alloc * op.kpad;
        const int blocks = (int) std::min<long>((total + 255) / 256, 148L * 16);
        split_direct_kernel<<<hb::counted(blocks), 256, 0, s>>>(X, ld, op.rows, op.k, op.hi, op.lo, op.rows_alloc,
                                                                op.kpad);
    } else {
        dim3 grid(op.kpad / 32, op.rows_alloc / 32);
        split_transpose_kernel<<<hb::counted(grid), dim3(32, 8), 0, s>>>(X, ld, op.rows, op.k, op.hi, op.lo, op.kpad);
    }
    HB_CUDA(cudaGetLastError());
}

bool split_gemm(cudaStream_t s, const SplitOperand &A, const SplitOperand &B, const SplitGemm &g) {
    if (g.M <= 0 || g.N <= 0) return true;
    if (!A.hi || !B.hi || A.kpad != B.kpad || g.M > A.rows_alloc || g.N > B.rows_alloc) return false;
    static std::atomic<unsigned long long> attr{0};
    bool attr_ok = true;
    once_per_device(attr, [&] {
        attr_ok = cudaFuncSetAttribute(split_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       SMEM_BYTES) == cudaSuccess;
    });
    if (!attr_ok) return false;
    KernelArgs p{};
    p.M = g.M;
    p.N = g.N;
    p.nkb = (std::min(g.K, A.kpad) + BK - 1) / BK;
    p.tiles_m = (g.M + BM - 1) / BM;
    p.tiles_n = (g.N + BN - 1) / BN;
    p.lower_tiles = g.lower_tiles ? 1 : 0;
    p.a_lower = g.a_lower ? 1 : 0;
    p.a_upper = g.a_upper ? 1 : 0;
    p.epi = g.epi;
    p.alpha = g.alpha;
    p.beta = g.beta;
    p.C = g.C;
    p.ldc = g.ldc;
    if (g.epi == SPLIT_EPI_SPLIT) {
        // the product's rows are the output operand's K entries, its columns the operand's rows
        if (!g.out || g.out->k != g.M || g.out->rows < g.N) return false;
        p.out_hi = g.out->hi;
        p.out_lo = g.out->lo;
        p.out_ld = g.out->kpad;
        p.out_rows = g.out->rows_alloc;
    }
    p.colsq = g.colsq;
    if (p.nkb <= 0) return false;
    const long tiles = g.lower_tiles ? (long) p.tiles_m * (p.tiles_m + 1) / 2 : (long) p.tiles_m * p.tiles_n;
    const long blocks = std::min<long>(tiles, device_sm_count());  // persistent: one CTA per SM at most
    const bool timed = kstat_on(KF_SPLIT_GEMM);
    if (timed) {
        double f = 3.0 * 2.0 * g.M * (double) g.N * g.K;
        if (g.lower_tiles) f *= 0.5;
        if (g.a_lower) f *= 0.5;
        if (g.a_upper) f *= (g.lower_tiles ? 1.0 / 3.0 : 0.5);  // lower part of a product of triangles: n^3/3 per product
        kstat_begin(KF_SPLIT_GEMM, s, f);
    }
    split_gemm_kernel<<<hb::counted((int) blocks), THREADS, SMEM_BYTES, s>>>(A.map_hi, A.map_lo, B.map_hi, B.map_lo,
                                                                             p);
    if (timed) kstat_end(s);
    HB_CUDA(cudaGetLastError());
    return true;
}

int split_error(cudaStream_t s) {
    int *d = nullptr, h = 0;
    HB_CUDA(cudaMallocAsync(&d, sizeof(int), s));
    read_err_kernel<<<hb::counted(1), 1, 0, s>>>(d);
    HB_CUDA(cudaMemcpyAsync(&h, d, sizeof(int), cudaMemcpyDeviceToHost, s));
    HB_CUDA(cudaFreeAsync(d, s));
    HB_CUDA(cudaStreamSynchronize(s));
    return h;
}

}  // namespace hb
