// Split-precision products on the 5th-generation tensor cores (tcgen05).
//
// An FP64 operand x is carried as two BF16 parts, hi = bf16(x) and
// lo = bf16(x - hi), so that x = hi + lo up to 2^-16 |x|. A product
// sum_k A(r,k) B(c,k) is formed as the three BF16 products
// Ahi*Bhi + Ahi*Blo + Alo*Bhi, accumulated in FP32 in tensor memory
// (relative error about 2^-16 per term; the lo*lo term is dropped).
//
// Operands are stored K-major: row r of an operand holds its K entries
// contiguously (BF16, rows padded to 128, K padded to 64), the layout the
// TMA engine copies into 128-byte-swizzled shared-memory tiles for
// tcgen05.mma. Persistent CTAs take 128 x 128 output tiles in turn: a
// producer warp streams the four operand tiles of each K block (A hi, A lo,
// B hi, B lo) into a 3-stage ring by TMA, one thread issues the three
// products and commits each stage back to the producer, and four warps read
// the accumulator out of tensor memory for the epilogue, from one of two
// accumulators while the next tile fills the other.
#pragma once
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include "dev.cuh"

namespace hb {

struct SplitOperand {
    int rows = 0, k = 0;          // logical extent
    int rows_alloc = 0, kpad = 0; // rows padded to 128, k to 64
    __nv_bfloat16 *hi = nullptr, *lo = nullptr;
    CUtensorMap map_hi, map_lo;
    bool alloc(int rows_, int k_);
    void release();
};

// op(r, k) = X[k + r*ld] when k_contiguous (the columns of X are the rows of
// op), else X[r + k*ld]; entries outside rows x k are written as zero.
void split_from_f64(cudaStream_t s, SplitOperand &op, const double *X, long ld, bool k_contiguous);

enum SplitEpilogue {
    SPLIT_EPI_F64 = 0,    // C[r + c*ldc] = alpha * acc + beta * C[r + c*ldc]
    SPLIT_EPI_SPLIT = 1,  // out(c, r) = acc as a split operand (the result's columns become rows)
    SPLIT_EPI_COLSQ = 2,  // colsq[c] += alpha * sum_r acc(r, c)^2
};

struct SplitGemm {
    int M = 0, N = 0, K = 0;
    bool lower_tiles = false;  // compute only tiles meeting r >= c (write only r >= c)
    bool a_lower = false;      // A(r, k) = 0 for k > r: stop the K loop at the tile's last row
    bool a_upper = false;      // A(r, k) = 0 for k < r: start the K loop at the tile's first row
    int epi = SPLIT_EPI_F64;
    double alpha = 1.0, beta = 0.0;
    double *C = nullptr;
    long ldc = 0;
    SplitOperand *out = nullptr;
    double *colsq = nullptr;
};

// Runs one split-precision product; false if the tensor-core path is unavailable.
bool split_gemm(cudaStream_t s, const SplitOperand &A, const SplitOperand &B, const SplitGemm &g);

// Device flag raised when a bounded wait inside a split kernel gave up.
int split_error(cudaStream_t s);

}  // namespace hb
