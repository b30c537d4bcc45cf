// chunked.cu — the per-rank half of doc-chunk data parallelism: a context
// that holds one chunk of the corpus's documents samples against word-topic
// counts shared by every chunk, and hands its own chunk's counts to the
// exchange that sums them.
//
// The reference runs -g N -c N as one host process driving N GPUs
// (src_culda/train/MultiChunkMultiGPUequal.h:88-172): every GPU samples its
// chunk against the same phi replica, then phi is copied to GPU 0, summed
// there and copied back (MasterGPUCollect / MasterGPUReduce /
// MasterGPUDistribute, src_culda/model/model_phi.cpp:105-144), and phiHead is
// rebuilt on every GPU.  Here each rank is one process with one context;
// culda_count_phi writes the chunk's counts into caller-owned device buffers,
// the caller sums those over ranks (an NCCL all-reduce of V*K + K int32) in
// place, and culda_set_shared_phi points the samplers at the summed buffers,
// which they read at every later iteration without a copy.
#include <cuda_runtime.h>

#include "../../include/culda_b200.h"
#include "context.h"
#include "internal.h"
#include "kernels.cuh"

using namespace culda;

extern "C" int culda_count_phi(culda_ctx *ctx, int32_t *d_phi, int32_t *d_nk) {
    if (!ctx || !d_phi || !d_nk) return fail(ctx, CULDA_ERR_INVALID_ARG, "culda_count_phi: invalid argument");
    CK(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    CK(cudaMemsetAsync(d_nk, 0, sizeof(int32_t) * (size_t)ctx->K, s));
    // stored tokens are word-major (reordered only inside each word), so the
    // input word ranges count the stored topics
    CK(launch_update_phi(ctx->K, ctx->V, ctx->d_word_ptr, ctx->d_z[ctx->cur], d_phi, d_nk, ctx->d_error, s));
    CK(cudaStreamSynchronize(s));
    int32_t e = 0;
    CK(cudaMemcpy(&e, ctx->d_error, sizeof(int32_t), cudaMemcpyDeviceToHost));
    if (e) return fail(ctx, CULDA_ERR_DEVICE_STATE, "culda_count_phi: device error 0x%x", e);
    return CULDA_OK;
}

extern "C" int culda_set_shared_phi(culda_ctx *ctx, int32_t *d_phi, int32_t *d_nk) {
    if (!ctx) return fail(ctx, CULDA_ERR_INVALID_ARG, "culda_set_shared_phi: null context");
    if ((d_phi == nullptr) != (d_nk == nullptr))
        return fail(ctx, CULDA_ERR_INVALID_ARG, "culda_set_shared_phi: give both buffers or neither");
    CK(cudaSetDevice(ctx->device));
    CK(cudaStreamSynchronize(ctx->stream));
    // drop the counts used so far: buffers of a fold-in model are the
    // context's own, shared buffers are the caller's
    if (!ctx->frozen_borrowed) {
        if (ctx->d_frozen_phi) cudaFree(ctx->d_frozen_phi);
        if (ctx->d_frozen_nk) cudaFree(ctx->d_frozen_nk);
    }
    ctx->d_frozen_phi = d_phi;
    ctx->d_frozen_nk = d_nk;
    ctx->frozen_borrowed = d_phi != nullptr;
    return build_graphs(ctx);
}
