// Allocation-free variant of the Cholesky entry point (no reference counterpart).
//
// Some callers cannot call cudaMalloc on their call path: a host framework whose
// caching allocator already owns the device memory budget, a plugin that is not
// allowed to touch the allocator, or a latency-critical loop that cannot afford the
// device-wide synchronisation cudaMalloc/cudaFree may imply. For them,
// hdsdpb_cholesky_noalloc factors an n x n matrix (n <= HDSDPB_NOALLOC_MAX_N) exactly
// like hdsdpb_cholesky, but every device buffer it touches lives in one file-scope
// static __device__ array (about 1.2 MB, held by every GPU that loads the library until
// the process exits): nothing is allocated or freed per call, on the device or the
// host, and no stream is created (work runs on the legacy default stream). The caller
// passes its input matrix and output buffers on the host, as for hdsdpb_cholesky.
//
// Scratch layout (doubles, ld = 256): S copy [ld * 256] | L [ld * 256] |
// diagonal-block inverses [ld * 64] | log-det slot [1] | info word [1 int].
// The array keeps the previous call's contents. Only the info word must start at zero,
// and the factorisation clears it itself on every call; only the lower triangle of L
// (rows < n) is ever read back, so stale entries elsewhere are harmless.
//
// Host code cannot use the array's name as a device address. The first call on a
// device looks the address up with cudaGetSymbolAddress (with that device current),
// checks the result and caches it per device under a lock; that first call should
// therefore come before any stream capture. All calls share the one array: calls that
// overlap on the GPU (from several host threads, or interleaved on several streams) race.
//
// The work runs on the legacy default stream, so a call also waits for, and holds back,
// the caller's other blocking streams (not its non-blocking ones); the call returns after
// synchronising that stream alone. The return code reflects this call's CUDA errors
// only: the library's sticky error flag is compared with its value on entry.
#include "la.h"
#include "../../include/hdsdp_b200.h"
#include <cstdio>
#include <mutex>

namespace hb {
namespace {

constexpr int kMaxN = HDSDPB_NOALLOC_MAX_N;
constexpr long kLd = kMaxN;  // pad_ld(256) = 256
constexpr size_t kMatDoubles = (size_t) kLd * kMaxN;
constexpr size_t kScratchDoubles = 2 * kMatDoubles + (size_t) kLd * 64 + 2;

static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

std::atomic<double *> g_scratch_ptr[kMaxDevices];

double *scratch_for_current_device() {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return nullptr;
    double *p = g_scratch_ptr[dev].load(std::memory_order_acquire);
    if (p) return p;
    static std::mutex mu;
    std::lock_guard<std::mutex> g(mu);
    p = g_scratch_ptr[dev].load(std::memory_order_relaxed);
    if (!p) {
        void *q = nullptr;
        if (cudaGetSymbolAddress(&q, g_noalloc_scratch) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        p = (double *) q;
        g_scratch_ptr[dev].store(p, std::memory_order_release);
    }
    return p;
}

}  // namespace
}  // namespace hb

using namespace hb;

extern "C" int hdsdpb_cholesky_noalloc(int n, const double *S, double *L, double *logdiag) {
    if (n < 0 || (n > 0 && !S)) return -1;
    if (n > kMaxN) {
        fprintf(stderr, "[hdsdp_b200] hdsdpb_cholesky_noalloc: n = %d exceeds the static scratch limit %d\n", n,
                kMaxN);
        return -2;
    }
    if (n == 0) {
        if (logdiag) *logdiag = 0.0;
        return 0;
    }
    double *base = scratch_for_current_device();
    if (!base) return -1;
    const int err_on_entry = device_error_flag();
    const long ld = pad_ld(n);
    DenseFactor F;  // views into the scratch array (never alloc()/release()d)
    int h_info = 0;
    F.n = n;
    F.ld = ld;
    F.L = base + kMatDoubles;
    F.Dinv = base + 2 * kMatDoubles;
    F.d_info = (int *) (base + 2 * kMatDoubles + (size_t) kLd * 64 + 1);
    F.h_info = &h_info;
    F.stat_logdet = false;   // the info word alone: the scratch keeps one slot for it
    double *dS = base, *dl = base + 2 * kMatDoubles + (size_t) kLd * 64;
    cudaStream_t s = 0;
    if (cudaMemcpy2D(dS, sizeof(double) * ld, S, sizeof(double) * n, sizeof(double) * n, n,
                     cudaMemcpyHostToDevice) != cudaSuccess)
        return -1;
    const bool ok = factorize(s, F, dS, ld);
    if (ok) {
        log_diag_sum(s, F, dl);
        if (logdiag && cudaMemcpy(logdiag, dl, sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
        if (L) {
            if (cudaMemcpy2D(L, sizeof(double) * n, F.L, sizeof(double) * ld, sizeof(double) * n, n,
                             cudaMemcpyDeviceToHost) != cudaSuccess)
                return -1;
            for (int j = 0; j < n; ++j)
                for (int i = 0; i < j; ++i) L[(size_t) j * n + i] = 0.0;
        }
    }
    if (cudaStreamSynchronize(cudaStreamLegacy) != cudaSuccess || cudaGetLastError() != cudaSuccess) return -1;
    if (device_error_flag() != err_on_entry) return -1;
    return ok ? 0 : 1;
}
