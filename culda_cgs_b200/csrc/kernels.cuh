// kernels.cuh — launch interface of the sm_100a kernels (host side).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/culda_b200.h"
#include "internal.h"

namespace culda {

// Everything the sampler reads, passed by value.
struct SampleParams {
    int32_t k;
    float alpha;
    float beta;
    float vbeta;                 // (float)V * beta, the reference's denominator term (lda_phi_kernel.cu:26)
    int32_t num_docs;
    int32_t num_items;
    int32_t num_hot;             // rows in hot_phi
    int64_t num_tokens;          // N: items must lie inside [0, N)
    int64_t theta_cap;           // entries in the theta array
    const int32_t *doc_ids;      // [N]
    const uint16_t *topics_in;   // [N]
    uint16_t *topics_out;        // [N]
    const uint32_t *theta;       // packed CSR
    const int2 *rows;            // [D] {start, end}
    const int32_t *nk;           // [K]
    const culda_item *items;     // [num_items]
    const int32_t *hot_phi;      // [num_hot * K]
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

size_t sample_smem_bytes(int k);
int sample_blocks_per_sm(int k, int group_lanes);
cudaError_t launch_sample(const SampleParams &p, int group_lanes, int grid, cudaStream_t s);

size_t theta_smem_bytes(int k);
int theta_blocks_per_sm(int k);
cudaError_t launch_theta_rebuild(int k, int num_docs, const int64_t *doc_ptr, const int32_t *doc_tok,
                                 const uint16_t *topics, const int32_t *doc_order, int2 *rows, uint32_t *theta,
                                 int32_t *nk, int64_t *stats, int32_t *error, int grid, cudaStream_t s);

cudaError_t launch_hot_rows(int k, const culda_item *hot_items, int num_hot_items, const uint16_t *topics,
                            int32_t *hot_phi, int32_t *error, cudaStream_t s);

cudaError_t launch_finalize_ll(const double *item_ll, int num_items, DevStats *st, uint32_t *iteration_dev,
                               cudaStream_t s);

cudaError_t launch_init_topics(int64_t n, int k, uint64_t seed, uint16_t *z, cudaStream_t s);

cudaError_t launch_update_phi(int k, int num_words, const int64_t *word_ptr, const uint16_t *topics, int32_t *phi,
                              int32_t *nk, int32_t *error, cudaStream_t s);

cudaError_t launch_phi_head(int k, float beta, int num_words, const int32_t *phi, const int32_t *nk, float *out,
                            cudaStream_t s);

cudaError_t launch_doc_check(int64_t n, int num_docs, const int32_t *doc_ids, int32_t *doc_count, int32_t *error,
                             cudaStream_t s);

cudaError_t launch_loglik_joint(int k, int num_words, int num_docs, float alpha, float beta, const int64_t *word_ptr,
                                const uint16_t *topics, const int2 *rows, const uint32_t *theta,
                                const int64_t *doc_ptr, const int32_t *nk, double *partials, int num_partials,
                                int32_t *error, cudaStream_t s);

int num_sms(int device);

}  // namespace culda
