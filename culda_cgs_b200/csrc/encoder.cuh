// encoder.cuh — internal interface of the document encoder (encoder.cu) for
// the context-level training and proposal code.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/culda_b200.h"

namespace culda {

// Where the cross-entropy target of batch row b comes from: a dense
// [batch x K] array, or the doc's accumulated topic counts acc[d*K + k]
// (summed over n snapshots) as (acc * inv_n + alpha) / (L_d + K alpha).
struct EncoderTarget {
    const float *dense = nullptr;
    const float *acc = nullptr;
    float inv_n = 1.0f;
    float alpha = 0.0f;
};

// One forward (+ backward, + Adam step) pass; probs (optional) receives q.
// batch_tokens is the batch's token count when the caller knows it, else -1
// (the backward pass then counts it on the device and reads it back).
// Returns a CULDA status; the loss is summed on the device into *d_loss.
int encoder_pass(culda_encoder *e, int batch, const int32_t *docs, const int64_t *doc_ptr, const int32_t *words,
                 const EncoderTarget *target, bool update, float *probs, cudaStream_t s, int64_t batch_tokens = -1);

// Mean cross-entropy of the passes since the last call (synchronises s).
int encoder_take_loss(culda_encoder *e, int batch_rows, double *loss, cudaStream_t s);

// FP32 master copy of tensor t (CULDA_ENC_*) and the BF16 refresh after a
// direct write to it.
float *encoder_tensor(culda_encoder *e, int t);
int encoder_refresh(culda_encoder *e, cudaStream_t s);
int encoder_num_words(const culda_encoder *e);

int encoder_k(const culda_encoder *e);
int encoder_max_batch(const culda_encoder *e);
int32_t *encoder_error_word(culda_encoder *e);

}  // namespace culda
