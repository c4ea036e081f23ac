// Common device-side definitions for the B200 HDSDP library.
#pragma once
#include <cuda_runtime.h>
#include <atomic>
#include <cstdint>
#include <cstdio>
#include <functional>

namespace hb {

// Column-major indexing with a 64-bit leading dimension.
__host__ __device__ __forceinline__ size_t cm(long i, long j, long ld) { return (size_t) (i + j * ld); }

// Error reporting: device failures are reported through the solver's return code.
#define HB_CUDA(expr)                                                                     \
    do {                                                                                  \
        cudaError_t _e = (expr);                                                          \
        if (_e != cudaSuccess) {                                                          \
            fprintf(stderr, "[hdsdp_b200] CUDA error %s at %s:%d\n", cudaGetErrorString(_e), \
                    __FILE__, __LINE__);                                                  \
            hb::device_error_flag() = 1;                                                  \
        }                                                                                 \
    } while (0)

int &device_error_flag();

// Per-device one-time set-up. Function attributes and device properties belong to a
// device, and first calls may come from several host threads at once (on one device or
// several): fn() runs under a library-wide lock, once for each device, and the device's
// bit in `mask` is published after it has run. Devices 0..63.
constexpr int kMaxDevices = 64;
int current_device();
void once_per_device(std::atomic<unsigned long long> &mask, const std::function<void()> &fn);
// The current device's SM count, cached per device.
int device_sm_count();

// Plain cudaMemset / cudaMemcpy run on the legacy default stream, which the library's
// non-blocking streams do not wait for (a pageable host-to-device copy may still be in
// flight when cudaMemcpy returns). Call this after such set-up copies and before the
// first launch that reads their destination on another stream.
inline void legacy_fence() { HB_CUDA(cudaStreamSynchronize(cudaStreamLegacy)); }

// Host-side count of kernel launches issued by this library (all threads).
long long &launch_counter();
// Every launch site passes its grid through counted(), which bumps the counter.
template <class G>
inline G counted(G grid) {
    __atomic_fetch_add(&launch_counter(), 1LL, __ATOMIC_RELAXED);
    return grid;
}

// Live per-family kernel timing: while a family is enabled, every launch of it
// is bracketed by CUDA events on its own stream and its algorithmic work
// (flops or bytes) is recorded; kstat_read() resolves the events.
// KF_POTRF counts the dual-slack factorisations (order n), KF_POTRF_SCHUR those of the
// Schur matrix (order m): the same kernel, two workloads.
enum KFamily {
    KF_GEMM = 0, KF_POTRF = 1, KF_TRTRI = 2, KF_SCHUR_PAIR = 3, KF_SPLIT_GEMM = 4, KF_POTRF_SCHUR = 5,
    KF_COUNT = 6
};
void kstat_enable(int mask);
bool kstat_on(int family);
void kstat_begin(int family, cudaStream_t s, double work);
void kstat_end(cudaStream_t s);
int kstat_read(int family, long long *launches, double *ms, double *work);

// Caching allocator for the library's device and pinned host buffers: a freed block
// goes to a free list keyed by its exact size and is handed out again to the next
// request of that size, so consecutive solvers (and per-call scratch) do not go back to
// the driver. hdsdpb_release_cached_memory() returns the cached blocks. A block is only
// freed here after the stream work that uses it has been synchronised, so a block handed
// out again is never still in use.
cudaError_t cache_malloc(void **p, size_t bytes);
void cache_free(void *p);
cudaError_t cache_malloc_host(void **p, size_t bytes);
void cache_free_host(void *p);
void cache_release();
// Host-side count of cache_malloc / cache_malloc_host calls (all threads), whether the
// block came from a free list or from the driver.
long long &alloc_counter();
template <class T>
inline cudaError_t cmalloc(T **p, size_t bytes) {
    return cache_malloc((void **) p, bytes);
}
template <class T>
inline cudaError_t cmalloc_host(T **p, size_t bytes) {
    return cache_malloc_host((void **) p, bytes);
}

// Leading dimensions are padded to a multiple of 32 doubles (256 bytes) so that
// every column starts on a 256-byte boundary.
inline long pad_ld(long n) { return ((n + 31) / 32) * 32; }

}  // namespace hb
