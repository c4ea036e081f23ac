// Common device-side definitions for the B200 HDSDP library.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>

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

// Leading dimensions are padded to a multiple of 32 doubles (256 bytes) so that
// every column starts on a 256-byte boundary.
inline long pad_ld(long n) { return ((n + 31) / 32) * 32; }

}  // namespace hb
