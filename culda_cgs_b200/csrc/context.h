// context.h — the context object behind the opaque culda_ctx handle, shared
// by the translation units that implement context-level entry points
// (context.cu: plain CGS; learned.cu: encoder training data, the learned
// Metropolis-Hastings proposal and fold-in).
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <vector>

#include "kernels.cuh"

struct culda_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    culda_params params{};
    int32_t D = 0, V = 0, K = 0;
    int64_t N = 0;
    int group_lanes = 8;
    int sample_blocks = culda::kSampleBlocksDefault;
    int tuned = 0;
    bool tune_pending = false;  // time the variants before iteration kTuneIteration
    float tune_ms = 0.f;
    int item_tokens = 0;

    int64_t *d_word_ptr = nullptr, *d_doc_ptr = nullptr;
    // Tokens are stored word by word as in the input, but inside each word
    // ordered by their doc's length; d_tok_index[i] is the input (word-major)
    // index of stored token i, the key of its Philox stream and of copy-out.
    int32_t *d_doc_ids = nullptr, *d_doc_tok = nullptr, *d_doc_order = nullptr, *d_tok_index = nullptr;
    uint16_t *d_z[2] = {nullptr, nullptr};
    uint16_t *d_zx = nullptr;  // topics in input order for copy-in / copy-out
    float *d_u = nullptr;      // the tokens' uniforms of the current iteration
    int cur = 0;
    culda::ThetaEntry *d_theta = nullptr;
    int64_t theta_cap = 0;
    int2 *d_rows = nullptr;
    int32_t *d_nk = nullptr;
    culda_item *d_items = nullptr, *d_hot_items = nullptr;
    int32_t num_items = 0, num_hot_items = 0, num_hot = 0;
    int32_t *d_seg_start = nullptr;  // first stored token of every segment
    int32_t num_segs = 0;
    int32_t *d_hot_phi = nullptr;
    double *d_item_ll = nullptr;
    int32_t *d_counter = nullptr;
    uint32_t *d_iter = nullptr;
    culda::DevStats *d_stats = nullptr;
    int32_t *d_error = nullptr;
    culda::DevStats *h_stats = nullptr;  // pinned (a slot of the process-wide pool)
    char *d_block = nullptr;             // every buffer above that culda_create allocates, in one allocation
    size_t block_bytes = 0;
    bool block_pooled = false;           // d_block came from the device's block pool (freed back to it)

    int sample_grid = 1, theta_grid = 1;
    // theta rebuild bins: docs of at least theta_min_len tokens (the first
    // theta_long of d_doc_order) are rebuilt a CTA each, the rest a warp each
    int theta_min_len = 0, theta_long = 0;
    float theta_tune_ms = 0.f;  // the chosen threshold's rebuild time when it was timed
    double doc_term = 0;  // sum_d L_d * log(L_d + K alpha)
    std::vector<int64_t> h_doc_ptr;
    std::vector<int32_t> h_max_ia;
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // recorded inside the iteration graph around the sampling and rebuild kernels
    cudaEvent_t ev_s0 = nullptr, ev_s1 = nullptr, ev_t0 = nullptr, ev_t1 = nullptr;
    uint32_t next_iteration = 1;
    std::string err;

    // Learned-proposal state (learned.cu), allocated on first use.
    int32_t *d_doc_words = nullptr;  // word id of every token in doc order (the doc_ptr CSR)
    float *d_acc = nullptr;          // [D x K] topic counts summed over the accumulated states
    int32_t n_acc = 0;               // states accumulated into d_acc
    uint16_t *d_ndk = nullptr;       // [D x K] dense doc-topic counts of the current state
    float *d_cdf = nullptr;          // [D x K] inclusive prefix sums of each doc's encoder proposal
    float *d_cdf_blk = nullptr;      // [D x K/32] the prefix at the end of every 32 topics
    float *d_probs = nullptr;        // [batch x K] encoder output scratch
    unsigned long long *d_mh_stats = nullptr;  // accepted moves, proposals of the last MH iteration
    bool has_proposal = false;

    // Fold-in: word-topic counts and topic totals held fixed (from a trained
    // model), used by the samplers instead of the counts of this corpus.
    int32_t *d_frozen_phi = nullptr;  // [V x K]
    int32_t *d_frozen_nk = nullptr;   // [K]
    // the two above are the caller's (culda_set_shared_phi), not freed here
    bool frozen_borrowed = false;
};

// Records the message of a failed call on the context (and thread-locally) and
// returns code.
int fail(culda_ctx *c, int code, const char *fmt, ...);

// CUDA errors as a failed call on the context `ctx` in scope.
#define CK(call)                                                                                           \
    do {                                                                                                   \
        cudaError_t e_ = (call);                                                                           \
        if (e_ != cudaSuccess)                                                                             \
            return fail(ctx, e_ == cudaErrorMemoryAllocation ? CULDA_ERR_OOM : CULDA_ERR_CUDA, "%s: %s (%s:%d)", \
                        #call, cudaGetErrorString(e_), __FILE__, __LINE__);                                \
    } while (0)

template <class T>
cudaError_t dalloc(T **p, size_t n) {
    return cudaMalloc((void **)p, std::max<size_t>(n, 1) * sizeof(T));
}

// Sampler parameters for topics d_z[cur] -> d_z[1-cur]; the Philox iteration
// comes from the device counter when iteration_ptr is set (graph launches).
culda::SampleParams sample_params(const culda_ctx *ctx, int cur, uint32_t iteration, const uint32_t *iteration_ptr);

// Event record that becomes an event node when the stream is being captured.
cudaError_t record_event(cudaEvent_t ev, cudaStream_t s);

// Theta rows and n_k from the current topics d_z[cur].
int rebuild_counts(culda_ctx *ctx);

// (Re)captures the two iteration graphs after a change of the sampler variant
// or of the counts it reads.
int build_graphs(culda_ctx *ctx);

// Topics of stored order d_src to host in input (word-major) order.
int topics_to_host(culda_ctx *ctx, const uint16_t *d_src, uint16_t *host);

// Frees the learned-proposal and fold-in buffers (learned.cu).
void free_learned_state(culda_ctx *ctx);
