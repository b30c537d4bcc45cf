// encoder.cu — C entry points of the tensor-core GEMM and the document
// encoder of the learned Metropolis-Hastings proposal.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "gemm.cuh"
#include "internal.h"

using namespace culda;

extern "C" int culda_gemm_bf16(const culda_gemm_args *a, void *stream) {
    if (!a) {
        set_global_error("culda_gemm_bf16: null arguments");
        return CULDA_ERR_INVALID_ARG;
    }
    GemmEpilogue ep;
    ep.out_f32 = a->out_f32;
    ep.ldo = a->ldo;
    ep.out_bf16 = reinterpret_cast<__nv_bfloat16 *>(a->out_bf16);
    ep.out_bf16_t = reinterpret_cast<__nv_bfloat16 *>(a->out_bf16_t);
    ep.ld_t = a->ld_t;
    ep.bias = a->bias;
    ep.pre = a->pre;
    ep.colsum = a->colsum;
    ep.alpha = a->alpha;
    if (const char *why = gemm_check(a->m, a->n, a->k, a->a, a->lda, a->b, a->ldb, a->epilogue, ep)) {
        set_global_error("culda_gemm_bf16: %s", why);
        return CULDA_ERR_INVALID_ARG;
    }
    const cudaError_t e = gemm_bf16_nt(a->m, a->n, a->k, a->a, a->lda, a->b, a->ldb, a->epilogue, ep, a->error,
                                       static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) {
        set_global_error("culda_gemm_bf16: %s", cudaGetErrorString(e));
        return e == cudaErrorNotSupported ? CULDA_ERR_UNSUPPORTED : CULDA_ERR_CUDA;
    }
    return CULDA_OK;
}
