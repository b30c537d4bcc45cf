// gemm.cuh — the tensor-core GEMM of the document encoder (gemm.cu).
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace culda {

enum : int {
    kEpiF32 = 0,       // out_f32 = alpha * acc (+ bias[col])
    kEpiBiasGelu = 1,  // out_f32 = acc + bias (pre-activation); out_bf16 / out_bf16_t = GELU of it
    kEpiGeluBwd = 2    // g = acc * GELU'(pre); out_bf16 / out_bf16_t = g; colsum[col] += sum over rows of g
};

// Outputs of one GEMM.  Row-major [M x N] arrays use row stride ldo; the
// transposed BF16 copy is [N x M] with row stride ld_t.
struct GemmEpilogue {
    float *out_f32 = nullptr;
    int ldo = 0;
    __nv_bfloat16 *out_bf16 = nullptr;
    __nv_bfloat16 *out_bf16_t = nullptr;
    int ld_t = 0;
    const float *bias = nullptr;
    const float *pre = nullptr;
    float *colsum = nullptr;
    float alpha = 1.0f;
    // split-K (kEpiF32 only): the K range is cut into k_splits CTAs per tile,
    // each adding its partial product into out_f32 with atomics (out_f32 must
    // hold zeros, or the value to add to, before the launch; bias is added once)
    int k_splits = 1;
};

// nullptr when the shapes, strides and pointers are acceptable, else why not.
const char *gemm_check(int M, int N, int K, const void *A, int lda, const void *B, int ldb, int epi,
                       const GemmEpilogue &ep);

// C = A[M x K] * B[N x K]^T with BF16 operands (row strides lda, ldb) and the
// given epilogue; M, N multiples of 128, K of 64.
cudaError_t gemm_bf16_nt(int M, int N, int K, const void *A, int lda, const void *B, int ldb, int epi,
                         const GemmEpilogue &ep, int32_t *error, cudaStream_t s);

}  // namespace culda
