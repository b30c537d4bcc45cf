/*
 * ref_compat.h — TEST INFRASTRUCTURE.  Force-included (nvcc -include) when
 * the reference's own sources are compiled for sm_100a by oracle/build_oracle.py;
 * no reference file is edited.
 *
 * 1. The reference uses the pre-Volta warp intrinsics __shfl, __shfl_up,
 *    __shfl_down and __ballot, which nvcc rejects for sm_70 and newer.  They
 *    are mapped to their *_sync forms with a full-warp mask; every call site in
 *    the reference is reached by all 32 lanes of a warp.
 * 2. DocChunk::allocGPU sizes wordPerplexity for numWords*32 doubles while
 *    LDAKernelTrain writes numSlots*32 of them (src_culda/model/doc_chunk.cpp:299,
 *    src_culda/kernel/lda_train_kernel.cu:261-262); numSlots exceeds numWords by
 *    at most 56, so up to 14 KB land past the allocation.  Every cudaMalloc of
 *    the reference is padded by 64 KB so that write stays inside memory the
 *    program owns.
 */
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>

#if defined(__CUDACC__)
#include <cuda_fp16.h>
#include <curand_kernel.h>
#define __shfl(v, ...) __shfl_sync(0xffffffffu, v, __VA_ARGS__)
#define __shfl_up(v, ...) __shfl_up_sync(0xffffffffu, v, __VA_ARGS__)
#define __shfl_down(v, ...) __shfl_down_sync(0xffffffffu, v, __VA_ARGS__)
#define __shfl_xor(v, ...) __shfl_xor_sync(0xffffffffu, v, __VA_ARGS__)
#define __ballot(p) __ballot_sync(0xffffffffu, (p))
#endif

static inline cudaError_t ref_compat_padded_malloc(void **p, size_t n) { return cudaMalloc(p, n + (size_t)65536); }
#define cudaMalloc(p, n) ref_compat_padded_malloc((void **)(p), (n))
