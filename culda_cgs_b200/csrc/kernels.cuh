// kernels.cuh — launch interface of the sm_100a kernels (host side).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/culda_b200.h"
#include "internal.h"

namespace culda {

// One theta CSR entry: the count (at most 65535, the longest doc) in the low
// 16 bits and 4 * topic (the byte offset of the topic's phihat in the
// sampler's shared memory; K <= 4096) in the high 16 bits.  Four bytes per
// entry, like the reference's two int16 arrays, but read with one load.
using ThetaEntry = uint32_t;

__host__ __device__ inline uint32_t theta_entry(uint32_t topic, uint32_t count) { return (topic << 18) | count; }

// Everything the sampler reads, passed by value.
struct SampleParams {
    int32_t k;
    int32_t kmask;               // next power of two >= K, minus one (bounds every topic index)
    float alpha;
    float beta;
    float vbeta;                 // (float)V * beta, the reference's denominator term (lda_phi_kernel.cu:26)
    int32_t num_docs;
    int32_t num_items;
    int32_t num_hot;             // rows in hot_phi
    int64_t num_tokens;          // N: items must lie inside [0, N)
    int64_t theta_cap;           // entries in the theta array
    const int32_t *doc_ids;      // [N]
    const int32_t *tok_index;    // [N] word-major index of each stored token (Philox counter), or null
    const float *uniforms;       // [N] the tokens' uniforms for this iteration, or null (computed inline)
    const uint16_t *topics_in;   // [N]
    uint16_t *topics_out;        // [N]
    const ThetaEntry *theta;     // CSR rows
    const int2 *rows;            // [D] {start, end}
    const int32_t *nk;           // [K]
    const culda_item *items;     // [num_items]
    const int32_t *seg_start;    // [num_segs] first token of every segment
    int32_t num_segs;
    const int32_t *hot_phi;      // [num_hot * K]
    const int32_t *frozen_phi;   // [V * K] word-topic counts held fixed (fold-in), or null; then nk
                                 // holds the matching topic totals
    int32_t *item_counter;       // work queue head, zeroed before the launch
    double *item_ll;             // [num_items] sum of log(S+Q) per item
    uint64_t seed;
    uint32_t iteration;          // used when iteration_ptr is null
    const uint32_t *iteration_ptr;
    int32_t *error;
};

struct DevStats {
    double ll_sum;        // sum over tokens of log(S_t + Q_t)
    int64_t row_entries;  // sum_d L_d * rowlen_d after the theta rebuild   (stats slot 0)
    int64_t nnz;          // theta non-zeros after the rebuild              (stats slot 1)
    int64_t token_nnz;    // sum_d L_d * nnz_d after the rebuild            (stats slot 2)
    int32_t error;
    uint32_t iteration;   // Philox iteration the sampler used
};

inline int pow2_ceil(int k) {
    int p = 1;
    while (p < k) p <<= 1;
    return p;
}

// Sampler variants: lanes per token G and the register budget, given as the
// resident CTAs per SM the kernel is compiled for (kSampleBlocksDefault for
// every G; kSampleBlocksHigh for G = 4, 8, 16).  G = kFlatLanes is the
// warp-flattened walk, built for kSampleBlocksDefault and kFlatBlocks (56
// registers: its two-buffer walk spills at 48).
constexpr int kSampleBlocksDefault = 8;
constexpr int kSampleBlocksHigh = 10;
constexpr int kFlatBlocks = 9;
constexpr int kFlatLanes = -1;
size_t sample_smem_bytes(int k, int group_lanes);
bool sample_variant_exists(int group_lanes, int blocks_per_sm);
int sample_blocks_per_sm(int k, int group_lanes, int blocks_per_sm);
cudaError_t launch_sample(const SampleParams &p, int group_lanes, int blocks_per_sm, int grid, cudaStream_t s);

size_t theta_smem_bytes(int k);
int theta_blocks_per_sm(int k);
// The first num_long docs of doc_order (which must then be given) are taken
// a whole CTA each from the queue counter long_queue (cleared by the launch);
// the rest one warp each.
cudaError_t launch_theta_rebuild(int k, int num_docs, const int64_t *doc_ptr, const int32_t *doc_tok,
                                 const uint16_t *topics, const int32_t *doc_order, int2 *rows, ThetaEntry *theta,
                                 int32_t *nk, int64_t *stats, int32_t *error, int grid, cudaStream_t s,
                                 int num_long = 0, int32_t *long_queue = nullptr);

cudaError_t launch_hot_rows(int k, const culda_item *hot_items, int num_hot_items, const uint16_t *topics,
                            int32_t *hot_phi, int32_t *error, cudaStream_t s);

cudaError_t launch_finalize_ll(const double *item_ll, int num_items, DevStats *st, uint32_t *iteration_dev,
                               cudaStream_t s);

// Flags theta rows outside the array or misaligned, and entries whose topic
// is not below K (the kernel-level sampler checks a caller's theta with it).
cudaError_t launch_check_theta(int num_docs, int k, const int2 *rows, const ThetaEntry *theta, int64_t cap,
                               int32_t *error, cudaStream_t s);

cudaError_t launch_init_topics(int64_t n, int k, uint64_t seed, const int32_t *tok_index, uint16_t *z,
                               cudaStream_t s);

// u[i] = uniform of Philox(seed, {t_i, iteration, 0}), t_i = tok_index[i] (or i)
cudaError_t launch_uniforms(int64_t n, uint64_t seed, const uint32_t *iteration_dev, uint32_t iteration,
                            const int32_t *tok_index, float *u, cudaStream_t s);

cudaError_t launch_update_phi(int k, int num_words, const int64_t *word_ptr, const uint16_t *topics, int32_t *phi,
                              int32_t *nk, int32_t *error, cudaStream_t s);

cudaError_t launch_phi_head(int k, float beta, int num_words, const int32_t *phi, const int32_t *nk, float *out,
                            cudaStream_t s);

cudaError_t launch_doc_check(int64_t n, int num_docs, const int32_t *doc_ids, int32_t *doc_count, int32_t *error,
                             cudaStream_t s);

cudaError_t launch_loglik_joint(int k, int num_words, int num_docs, float alpha, float beta, const int64_t *word_ptr,
                                const uint16_t *topics, const int2 *rows, const ThetaEntry *theta,
                                const int64_t *doc_ptr, double *partials, int num_partials, int32_t *error,
                                cudaStream_t s);

// Internal token order: within each word, tokens sorted by their doc's length
// (longest first, doc id breaking ties).  keys[t] = (word << 16) | (65535 - L).
cudaError_t launch_order_keys(int num_words, int64_t num_tokens, const int64_t *word_ptr, const int32_t *doc_ids,
                              const int64_t *doc_ptr, uint64_t *keys, cudaStream_t s);
// The same order with 32-bit keys (num_words <= 2^24): keys[t] = (word << 8) |
// (255 - length class), 16 classes per doubling of L.
cudaError_t launch_order_keys32(int num_words, int64_t num_tokens, const int64_t *word_ptr, const int32_t *doc_ids,
                                const int64_t *doc_ptr, uint32_t *keys, cudaStream_t s);
template <class T>
cudaError_t launch_gather(int64_t n, const int32_t *index, const T *src, T *dst, cudaStream_t s);
template <class T>
cudaError_t launch_scatter(int64_t n, const int32_t *index, const T *src, T *dst, cudaStream_t s);
cudaError_t launch_iota(int64_t n, int32_t *v, cudaStream_t s);
cudaError_t launch_check_topics(int64_t n, int k, const uint16_t *z, int32_t *error, cudaStream_t s);

int num_sms(int device);

}  // namespace culda
