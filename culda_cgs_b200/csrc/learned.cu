// learned.cu — the learned Metropolis-Hastings proposal and fold-in on a
// context: training pairs (document bag, accumulated topic distribution),
// encoder training over the context's documents, per-doc proposal tables, the
// MH iteration whose stationary target is the plain sampler's conditional on
// the frozen snapshot, p(k) ~ (n_dk + alpha) * phihat_wk, a frozen-model mode
// for new documents, and the encoder warm start of their topics.
//
// MH iteration (one launch per kernel, not graph-captured):
//   memset(work counter, hot rows) -> hot_rows -> dense n_dk table from the
//   theta CSR -> mh_kernel(z[c] -> z[1-c]) -> theta rebuild (as plain CGS).
// mh_kernel reuses the sampler's work items: per item the word's phihat row is
// built in shared memory from a histogram of the snapshot topics (or the hot
// row, or the frozen counts), then one thread per token runs `steps` steps:
//   doc step     k' ~ (n_dk + alpha): with probability L_d / (L_d + K alpha)
//                the topic of a uniformly chosen token of the doc, else a
//                uniform topic; accept with min(1, phihat_wk' / phihat_ws).
//   encoder step k' ~ q_d (two-level search of the doc's prefix table);
//                accept with min(1, (n_dk' + alpha) phihat_wk' q_d(s) /
//                ((n_ds + alpha) phihat_ws q_d(k'))).
// Steps alternate doc, encoder, doc, ... when a proposal is set; otherwise all
// are doc steps.  Each step leaves p invariant, so their sequence does too.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <numeric>
#include <vector>

#include "context.h"
#include "device_util.cuh"
#include "encoder.cuh"
#include "gemm.cuh"
#include "kernels.cuh"
#include "philox.h"

using namespace culda;

namespace {

// ------------------------------------------------------------------ kernels
// Word id of every token in doc order: doc_tok[i] is a stored (word-major)
// token index, whose word is the last w with word_ptr[w] <= doc_tok[i].
__global__ void doc_words_kernel(int64_t n, int num_words, const int64_t *__restrict__ word_ptr,
                                 const int32_t *__restrict__ doc_tok, int32_t *out) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t t = doc_tok[i];
        int lo = 0, hi = num_words - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (__ldg(word_ptr + mid) <= t)
                lo = mid;
            else
                hi = mid - 1;
        }
        out[i] = lo;
    }
}

// Warp per doc: the row's entries into a dense [D x K] table (set or added).
// A topic occurs at most once per row, so no two lanes touch one element.
template <class T>
__global__ void theta_to_dense_kernel(int D, int K, const int2 *__restrict__ rows,
                                      const ThetaEntry *__restrict__ theta, T *dense, bool add) {
    const int lane = threadIdx.x & 31;
    for (int d = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; d < D; d += (gridDim.x * blockDim.x) >> 5) {
        const int2 r = rows[d];
        for (int i = r.x + lane; i < r.y; i += 32) {
            const ThetaEntry e = theta[i];
            const uint32_t c = e & 0xFFFFu;
            if (!c) continue;
            T *p = dense + (size_t)d * K + (e >> 18);
            *p = add ? (T)(*p + (T)c) : (T)c;
        }
    }
}

// Warp per batch row: proposal (1 - mix) q + mix / K, inclusive prefix over
// the row (lane l sums topics [l*K/32, (l+1)*K/32), then a warp scan) and the
// prefix at the end of every 32 topics.
__global__ void proposal_table_kernel(int rows, int d0, int K, float mix, const float *__restrict__ probs,
                                      float *cdf, float *blk) {
    const int lane = threadIdx.x & 31;
    const int per = K >> 5, nb = K >> 5;
    const float u = mix / (float)K, a = 1.0f - mix;
    for (int b = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; b < rows; b += (gridDim.x * blockDim.x) >> 5) {
        const float *q = probs + (size_t)b * K + lane * per;
        float *c = cdf + (size_t)(d0 + b) * K + lane * per;
        float s = 0.f;
        for (int i = 0; i < per; ++i) {
            s += a * q[i] + u;
            c[i] = s;
        }
        float incl = s;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const float t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        const float base = incl - s;
        for (int i = 0; i < per; ++i) c[i] += base;
        __syncwarp();
        const float *row = cdf + (size_t)(d0 + b) * K;
        for (int j = lane; j < nb; j += 32) blk[(size_t)(d0 + b) * nb + j] = row[32 * j + 31];
    }
}

struct MHParams {
    int k;
    float alpha, beta, vbeta;
    int num_docs, num_items, num_hot;
    int64_t num_tokens;
    const int32_t *doc_ids;    // stored order
    const int32_t *tok_index;  // stored -> input index (Philox key), or null
    const uint16_t *topics_in;
    uint16_t *topics_out;
    const int64_t *doc_ptr;
    const int32_t *doc_tok;
    const int32_t *nk;
    const culda_item *items;
    const int32_t *hot_phi;
    const int32_t *frozen_phi;  // [V x K] fixed counts (fold-in) or null
    int32_t *item_counter;
    const uint16_t *ndk;  // [D x K]
    const float *cdf;     // [D x K] or null
    const float *blk;     // [D x K/32]
    uint64_t seed;
    uint32_t iteration;
    int steps;
    int32_t *error;
    unsigned long long *stats;  // {accepted, proposed}
};

constexpr int kMHThreads = 256;

// First index in [lo, lo + n) whose value exceeds t (lo + n - 1 when none does).
__device__ __forceinline__ int first_above(const float *__restrict__ v, int lo, int n, float t) {
    int l = lo, h = lo + n - 1;
    while (l < h) {
        const int mid = (l + h) >> 1;
        if (__ldg(v + mid) > t)
            h = mid;
        else
            l = mid + 1;
    }
    return l;
}

// The phihat row of the item's word into ph[] (inv[] holds 1 / (n_k + V beta)):
// frozen counts, the hot row, or a histogram of the item's snapshot topics.
// Ends with a barrier.
__device__ __forceinline__ void item_phi_row(const MHParams &p, const culda_item &item, float *ph, const float *inv,
                                             int *hist) {
    const int K = p.k, tid = threadIdx.x;
    const int *src;
    if (p.frozen_phi) {
        src = p.frozen_phi + (size_t)item.word * K;
    } else if (item.hot < 0) {
        for (int j = tid; j < K; j += blockDim.x) hist[j] = 0;
        __syncthreads();
        for (int64_t t = item.begin + tid; t < item.begin + item.count; t += blockDim.x) {
            const uint32_t z = p.topics_in[t];
            if (z < (uint32_t)K)
                atomicAdd(&hist[z], 1);
            else
                atomicOr(p.error, kErrTopicRange);
        }
        __syncthreads();
        src = hist;
    } else {
        src = p.hot_phi + (size_t)item.hot * K;
    }
    for (int j = tid; j < K; j += blockDim.x) ph[j] = ((float)src[j] + p.beta) * inv[j];
    __syncthreads();
}

__device__ __forceinline__ bool item_ok(const MHParams &p, const culda_item &item) {
    return item.begin >= 0 && item.count >= 0 && item.begin + item.count <= p.num_tokens && item.hot < p.num_hot &&
           item.word >= 0;
}

__global__ void __launch_bounds__(kMHThreads) mh_kernel(const MHParams p) {
    extern __shared__ float sm_mh[];
    const int K = p.k;
    float *ph = sm_mh;                                   // [K]
    float *inv = sm_mh + K;                              // [K]
    int *hist = reinterpret_cast<int *>(sm_mh + 2 * K);  // [K]
    __shared__ int s_item;
    const int tid = threadIdx.x;
    const float ka = (float)K * p.alpha;
    const int nb = K >> 5;
    unsigned long long acc_n = 0, prop_n = 0;

    for (int j = tid; j < K; j += blockDim.x) inv[j] = 1.0f / ((float)p.nk[j] + p.vbeta);
    for (;;) {
        if (tid == 0) s_item = atomicAdd(p.item_counter, 1);
        __syncthreads();
        const int it = s_item;
        if (it >= p.num_items) break;
        const culda_item item = p.items[it];
        if (!item_ok(p, item)) {
            if (tid == 0) atomicOr(p.error, kErrRowRange);
            __syncthreads();
            continue;
        }
        item_phi_row(p, item, ph, inv, hist);
        const int64_t iend = item.begin + item.count;
        for (int64_t t = item.begin + tid; t < iend; t += blockDim.x) {
            int s = p.topics_in[t];
            const int d = p.doc_ids[t];
            if ((unsigned)d >= (unsigned)p.num_docs || (unsigned)s >= (unsigned)K) {
                atomicOr(p.error, kErrDocRange);
                p.topics_out[t] = (uint16_t)min(max(s, 0), K - 1);
                continue;
            }
            const uint64_t key = p.tok_index ? (uint64_t)__ldg(p.tok_index + t) : (uint64_t)t;
            const int64_t d0 = p.doc_ptr[d];
            const int L = (int)(p.doc_ptr[d + 1] - d0);
            const uint16_t *nd = p.ndk + (size_t)d * K;
            for (int step = 0; step < p.steps; ++step) {
                const u32x4 x = philox_token4(p.seed, key, p.iteration, kPurposeMH + (uint32_t)step);
                int kp;
                float ratio;
                if (!(p.cdf && (step & 1))) {  // doc proposal
                    if (uniform_from_bits(x.x) * ((float)L + ka) < (float)L) {
                        const int i = (int)bounded_from_bits(x.y, (uint32_t)L);
                        kp = p.topics_in[p.doc_tok[d0 + i]];
                        if ((unsigned)kp >= (unsigned)K) kp = s;
                    } else {
                        kp = (int)bounded_from_bits(x.y, (uint32_t)K);
                    }
                    ratio = ph[kp] / ph[s];
                } else {  // encoder proposal
                    const float *row = p.cdf + (size_t)d * K;
                    const float total = __ldg(p.blk + (size_t)d * nb + nb - 1);
                    const float T = uniform_from_bits(x.y) * total;
                    const int b = first_above(p.blk + (size_t)d * nb, 0, nb, T);
                    kp = first_above(row, 32 * b, 32, T);
                    const float qk = __ldg(row + kp) - (kp > 0 ? __ldg(row + kp - 1) : 0.f);
                    const float qs = __ldg(row + s) - (s > 0 ? __ldg(row + s - 1) : 0.f);
                    const float pk = ((float)nd[kp] + p.alpha) * ph[kp];
                    const float ps = ((float)nd[s] + p.alpha) * ph[s];
                    ratio = (pk * qs) / (ps * qk);
                }
                ++prop_n;
                if (kp != s && uniform_from_bits(x.z) < ratio) {
                    s = kp;
                    ++acc_n;
                }
            }
            p.topics_out[t] = (uint16_t)s;
        }
        __syncthreads();  // ph / hist are rebuilt for the next item
    }
    if (p.stats) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            acc_n += __shfl_xor_sync(0xffffffffu, acc_n, o);
            prop_n += __shfl_xor_sync(0xffffffffu, prop_n, o);
        }
        if ((tid & 31) == 0 && prop_n) {
            atomicAdd(&p.stats[0], acc_n);
            atomicAdd(&p.stats[1], prop_n);
        }
    }
}

// Warm start: warp per token; the token's topic is drawn from
// q_d(k) * phihat_wk (q_d from the differences of the doc's proposal prefix
// table) by inverse CDF in ascending topic.  Lanes take consecutive topics,
// 32 at a time, so every table load is one coalesced line: a first pass sums
// the weights, a second runs a warp scan chunk by chunk until the running sum
// passes u * total (the last topic if rounding leaves it short).
__device__ __forceinline__ float warm_weight(const float *__restrict__ row, const float *ph, int c, int lane,
                                             float &carry) {
    const float cur = __ldg(row + c + lane);
    float prev = __shfl_up_sync(0xffffffffu, cur, 1);
    if (lane == 0) prev = carry;
    carry = __shfl_sync(0xffffffffu, cur, 31);
    return (cur - prev) * ph[c + lane];
}

__global__ void __launch_bounds__(kMHThreads) warm_start_kernel(const MHParams p) {
    extern __shared__ float sm_ws[];
    const int K = p.k;
    float *ph = sm_ws;
    float *inv = sm_ws + K;
    int *hist = reinterpret_cast<int *>(sm_ws + 2 * K);
    __shared__ int s_item;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
    for (int j = tid; j < K; j += blockDim.x) inv[j] = 1.0f / ((float)p.nk[j] + p.vbeta);
    for (;;) {
        if (tid == 0) s_item = atomicAdd(p.item_counter, 1);
        __syncthreads();
        const int it = s_item;
        if (it >= p.num_items) break;
        const culda_item item = p.items[it];
        if (!item_ok(p, item)) {
            if (tid == 0) atomicOr(p.error, kErrRowRange);
            __syncthreads();
            continue;
        }
        item_phi_row(p, item, ph, inv, hist);
        const int64_t iend = item.begin + item.count;
        for (int64_t t = item.begin + warp; t < iend; t += nwarps) {
            const int d = p.doc_ids[t];
            if ((unsigned)d >= (unsigned)p.num_docs) {
                if (lane == 0) atomicOr(p.error, kErrDocRange);
                continue;
            }
            const float *row = p.cdf + (size_t)d * K;
            float carry = 0.f, part = 0.f;
            for (int c = 0; c < K; c += 32) part += warm_weight(row, ph, c, lane, carry);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
            const uint64_t key = p.tok_index ? (uint64_t)__ldg(p.tok_index + t) : (uint64_t)t;
            const float T = uniform_from_bits(philox_token(p.seed, key, 0u, kPurposeWarm)) * part;
            int pick = K - 1;
            float base = 0.f;
            carry = 0.f;
            for (int c = 0; c < K; c += 32) {
                float incl = warm_weight(row, ph, c, lane, carry);
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const float v = __shfl_up_sync(0xffffffffu, incl, o);
                    if (lane >= o) incl += v;
                }
                incl += base;
                const unsigned hit = __ballot_sync(0xffffffffu, incl > T);
                if (hit) {
                    pick = c + __ffs(hit) - 1;
                    break;
                }
                base = __shfl_sync(0xffffffffu, incl, 31);
            }
            if (lane == 0) p.topics_out[t] = (uint16_t)pick;
        }
        __syncthreads();
    }
}

__global__ void bump_iteration_kernel(uint32_t *iteration) { *iteration += 1u; }

// Block per word (rows past V are zero): the word's topic profile
// (n_wk + beta) / (n_w + K beta) in BF16, from a histogram of its tokens.
__global__ void phi_profile_kernel(int V, int rows, int K, float beta, const int64_t *__restrict__ word_ptr,
                                   const uint16_t *__restrict__ topics, __nv_bfloat16 *out) {
    extern __shared__ int hist_p[];
    for (int w = blockIdx.x; w < rows; w += gridDim.x) {
        for (int j = threadIdx.x; j < K; j += blockDim.x) hist_p[j] = 0;
        __syncthreads();
        int64_t n = 0;
        if (w < V) {
            n = word_ptr[w + 1] - word_ptr[w];
            for (int64_t t = word_ptr[w] + threadIdx.x; t < word_ptr[w + 1]; t += blockDim.x) {
                const uint32_t z = topics[t];
                if (z < (uint32_t)K) atomicAdd(&hist_p[z], 1);
            }
        }
        __syncthreads();
        const float inv = 1.0f / ((float)n + (float)K * beta);
        for (int j = threadIdx.x; j < K; j += blockDim.x)
            out[(size_t)w * K + j] = __float2bfloat16_rn(w < V ? ((float)hist_p[j] + beta) * inv : 0.f);
        __syncthreads();
    }
}

// Random projection matrix R [256 x K], entries uniform with unit variance.
__global__ void projection_kernel(int n, uint64_t seed, __nv_bfloat16 *R) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        R[i] = __float2bfloat16_rn(
            1.7320508f * (2.0f * uniform_from_bits(philox_token(seed, (uint64_t)i, 0u, kPurposeWeights)) - 1.0f));
}

// Warp per word: E[w] = P[w] scaled to root-mean-square `rms`.
__global__ void rms_rows_kernel(int V, int cols, float rms, const float *__restrict__ P, float *E) {
    const int lane = threadIdx.x & 31;
    for (int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < V; w += (gridDim.x * blockDim.x) >> 5) {
        float ss = 0.f;
        for (int j = lane; j < cols; j += 32) ss += P[(size_t)w * cols + j] * P[(size_t)w * cols + j];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) ss += __shfl_xor_sync(0xffffffffu, ss, o);
        const float sc = ss > 0.f ? rms * rsqrtf(ss / (float)cols) : 0.f;
        for (int j = lane; j < cols; j += 32) E[(size_t)w * cols + j] = P[(size_t)w * cols + j] * sc;
    }
}

// ------------------------------------------------------------- host helpers
int ensure_doc_words(culda_ctx *ctx) {
    if (ctx->d_doc_words) return CULDA_OK;
    CK(dalloc(&ctx->d_doc_words, (size_t)ctx->N));
    doc_words_kernel<<<grid_for(ctx->N), 256, 0, ctx->stream>>>(ctx->N, ctx->V, ctx->d_word_ptr, ctx->d_doc_tok,
                                                                ctx->d_doc_words);
    CK(cudaGetLastError());
    return CULDA_OK;
}

int build_dense_theta(culda_ctx *ctx) {
    cudaStream_t s = ctx->stream;
    if (!ctx->d_ndk) CK(dalloc(&ctx->d_ndk, (size_t)ctx->D * ctx->K));
    CK(cudaMemsetAsync(ctx->d_ndk, 0, sizeof(uint16_t) * (size_t)ctx->D * ctx->K, s));
    theta_to_dense_kernel<uint16_t><<<grid_for((int64_t)ctx->D * 32), 256, 0, s>>>(
        ctx->D, ctx->K, ctx->d_rows, ctx->d_theta, ctx->d_ndk, false);
    CK(cudaGetLastError());
    return CULDA_OK;
}

MHParams mh_params(culda_ctx *ctx, int cur, uint32_t iteration, int steps) {
    MHParams p{};
    p.k = ctx->K;
    p.alpha = ctx->params.alpha;
    p.beta = ctx->params.beta;
    p.vbeta = ctx->params.beta * (float)ctx->V;
    p.num_docs = ctx->D;
    p.num_items = ctx->num_items;
    p.num_hot = ctx->num_hot;
    p.num_tokens = ctx->N;
    p.doc_ids = ctx->d_doc_ids;
    p.tok_index = ctx->d_tok_index;
    p.topics_in = ctx->d_z[cur];
    p.topics_out = ctx->d_z[1 - cur];
    p.doc_ptr = ctx->d_doc_ptr;
    p.doc_tok = ctx->d_doc_tok;
    p.nk = ctx->d_frozen_phi ? ctx->d_frozen_nk : ctx->d_nk;
    p.items = ctx->d_items;
    p.hot_phi = ctx->d_hot_phi;
    p.frozen_phi = ctx->d_frozen_phi;
    p.item_counter = ctx->d_counter;
    p.ndk = ctx->d_ndk;
    p.cdf = ctx->has_proposal ? ctx->d_cdf : nullptr;
    p.blk = ctx->d_cdf_blk;
    p.seed = ctx->params.seed;
    p.iteration = iteration;
    p.steps = steps;
    p.error = ctx->d_error;
    p.stats = ctx->d_mh_stats;
    return p;
}

int hot_rows_if_needed(culda_ctx *ctx, int cur) {
    cudaStream_t s = ctx->stream;
    if (ctx->num_hot > 0 && !ctx->d_frozen_phi) {
        CK(cudaMemsetAsync(ctx->d_hot_phi, 0, sizeof(int32_t) * (size_t)ctx->num_hot * ctx->K, s));
        CK(launch_hot_rows(ctx->K, ctx->d_hot_items, ctx->num_hot_items, ctx->d_z[cur], ctx->d_hot_phi, ctx->d_error,
                           s));
    }
    return CULDA_OK;
}

template <class Kernel>
int persistent_grid(culda_ctx *ctx, Kernel kernel, size_t smem, int *grid) {
    CK(allow_smem(reinterpret_cast<const void *>(kernel), smem, ctx->stream));
    int bps = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, kernel, kMHThreads, smem));
    *grid = std::max(1, std::min(ctx->num_items, num_sms(ctx->device) * std::max(bps, 1)));
    return CULDA_OK;
}

// Hot rows, the dense n_dk table and the MH kernel: topics d_z[cur] -> d_z[1-cur].
int launch_mh_pass(culda_ctx *ctx, int cur, uint32_t iteration, int steps) {
    cudaStream_t s = ctx->stream;
    if (!ctx->d_mh_stats) CK(dalloc(&ctx->d_mh_stats, 2));
    CK(cudaMemsetAsync(ctx->d_mh_stats, 0, 2 * sizeof(unsigned long long), s));
    CK(cudaMemsetAsync(ctx->d_counter, 0, sizeof(int32_t), s));
    int rc = hot_rows_if_needed(ctx, cur);
    if (rc) return rc;
    rc = build_dense_theta(ctx);
    if (rc) return rc;
    const size_t smem = 3 * (size_t)ctx->K * sizeof(float);
    int grid = 1;
    rc = persistent_grid(ctx, mh_kernel, smem, &grid);
    if (rc) return rc;
    CK(record_event(ctx->ev_s0, s));
    mh_kernel<<<grid, kMHThreads, smem, s>>>(mh_params(ctx, cur, iteration, steps));
    CK(cudaGetLastError());
    CK(record_event(ctx->ev_s1, s));
    return CULDA_OK;
}

int check_device_error(culda_ctx *ctx, const char *what) {
    int32_t e = 0;
    CK(cudaMemcpyAsync(&e, ctx->d_error, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (e) return fail(ctx, CULDA_ERR_DEVICE_STATE, "%s: device error 0x%x", what, e);
    return CULDA_OK;
}

}  // namespace

void free_learned_state(culda_ctx *ctx) {
    void *bufs[] = {ctx->d_doc_words, ctx->d_acc,    ctx->d_ndk,        ctx->d_cdf,        ctx->d_cdf_blk,
                    ctx->d_probs,     ctx->d_mh_stats, ctx->frozen_borrowed ? nullptr : ctx->d_frozen_phi,
                    ctx->frozen_borrowed ? nullptr : ctx->d_frozen_nk};
    for (void *b : bufs)
        if (b) cudaFree(b);
    ctx->frozen_borrowed = false;
    ctx->d_doc_words = nullptr;
    ctx->d_acc = nullptr;
    ctx->d_ndk = nullptr;
    ctx->d_cdf = nullptr;
    ctx->d_cdf_blk = nullptr;
    ctx->d_probs = nullptr;
    ctx->d_mh_stats = nullptr;
    ctx->d_frozen_phi = nullptr;
    ctx->d_frozen_nk = nullptr;
    ctx->has_proposal = false;
}

// ============================================================ C entry points
extern "C" int culda_accumulate_theta(culda_ctx *ctx) {
    if (!ctx) return fail(ctx, CULDA_ERR_INVALID_ARG, "culda_accumulate_theta: null context");
    CK(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    if (!ctx->d_acc) {
        CK(dalloc(&ctx->d_acc, (size_t)ctx->D * ctx->K));
        CK(cudaMemsetAsync(ctx->d_acc, 0, sizeof(float) * (size_t)ctx->D * ctx->K, s));
        ctx->n_acc = 0;
    }
    theta_to_dense_kernel<float><<<grid_for((int64_t)ctx->D * 32), 256, 0, s>>>(ctx->D, ctx->K, ctx->d_rows,
                                                                               ctx->d_theta, ctx->d_acc, true);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(s));
    ctx->n_acc += 1;
    return CULDA_OK;
}

extern "C" int culda_train_encoder(culda_ctx *ctx, culda_encoder *enc, int32_t epochs, uint64_t seed,
                                   double *loss) {
    if (!ctx || !enc || epochs <= 0) return fail(ctx, CULDA_ERR_INVALID_ARG, "culda_train_encoder: invalid argument");
    if (!ctx->d_acc || ctx->n_acc <= 0)
        return fail(ctx, CULDA_ERR_INVALID_ARG, "culda_train_encoder: no accumulated states (culda_accumulate_theta)");
    if (encoder_k(enc) != ctx->K || encoder_num_words(enc) != ctx->V)
        return fail(ctx, CULDA_ERR_INVALID_ARG, "culda_train_encoder: encoder shape does not match the context");
    CK(cudaSetDevice(ctx->device));
    int rc = ensure_doc_words(ctx);
    if (rc) return rc;
    cudaStream_t s = ctx->stream;
    const int B = std::min(encoder_max_batch(enc), ctx->D);
    int32_t *d_order = nullptr;
    CK(dalloc(&d_order, (size_t)ctx->D));
    std::vector<int32_t> order((size_t)ctx->D);
    EncoderTarget tg;
    tg.acc = ctx->d_acc;
    tg.inv_n = 1.0f / (float)ctx->n_acc;
    tg.alpha = ctx->params.alpha;
    double last = 0.0;
    for (int ep = 0; ep < epochs && rc == CULDA_OK; ++ep) {
        // Fisher-Yates with Philox draws keyed on (seed, position, epoch)
        std::iota(order.begin(), order.end(), 0);
        for (int32_t i = ctx->D - 1; i > 0; --i) {
            const uint32_t j = bounded_from_bits(philox_token(seed, (uint64_t)i, (uint32_t)ep, kPurposeShuffle),
                                                 (uint32_t)i + 1u);
            std::swap(order[(size_t)i], order[j]);
        }
        if (cudaMemcpyAsync(d_order, order.data(), sizeof(int32_t) * order.size(), cudaMemcpyHostToDevice, s) !=
            cudaSuccess) {
            rc = fail(ctx, CULDA_ERR_CUDA, "culda_train_encoder: order upload failed");
            break;
        }
        // batches of B docs; the last one holds the remainder
        const int steps = (ctx->D + B - 1) / B;
        for (int st = 0; st < steps && rc == CULDA_OK; ++st) {
            const int b0 = st * B, nb = std::min(B, ctx->D - b0);
            int64_t tokens = 0;  // the batch's tokens, known here from the host doc index
            for (int i = b0; i < b0 + nb; ++i)
                tokens += ctx->h_doc_ptr[(size_t)order[(size_t)i] + 1] - ctx->h_doc_ptr[(size_t)order[(size_t)i]];
            rc = encoder_pass(enc, nb, d_order + b0, ctx->d_doc_ptr, ctx->d_doc_words, &tg, true, nullptr, s,
                              tokens);
        }
        if (rc == CULDA_OK) rc = encoder_take_loss(enc, ctx->D, &last, s);
        if (rc) fail(ctx, rc, "culda_train_encoder: %s", global_error());
        // the host order buffer is rewritten by the next epoch
        if (cudaStreamSynchronize(s) != cudaSuccess && rc == CULDA_OK)
            rc = fail(ctx, CULDA_ERR_CUDA, "culda_train_encoder: sync failed");
    }
    cudaStreamSynchronize(s);
    cudaFree(d_order);
    if (rc == CULDA_OK && loss) *loss = last;
    return rc;
}

extern "C" int culda_encoder_init_from_phi(culda_ctx *ctx, culda_encoder *enc, uint64_t seed) {
    if (!ctx || !enc) return fail(ctx, CULDA_ERR_INVALID_ARG, "culda_encoder_init_from_phi: null argument");
    if (encoder_num_words(enc) != ctx->V || encoder_k(enc) != ctx->K)
        return fail(ctx, CULDA_ERR_INVALID_ARG, "culda_encoder_init_from_phi: encoder shape does not match the context");
    CK(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    const int K = ctx->K, V = ctx->V, Vp = (V + 127) & ~127, E = CULDA_ENC_EMBED;
    __nv_bfloat16 *prof = nullptr, *R = nullptr;
    float *P = nullptr;
    int rc = CULDA_OK;
    if (dalloc(&prof, (size_t)Vp * K) != cudaSuccess || dalloc(&R, (size_t)E * K) != cudaSuccess ||
        dalloc(&P, (size_t)Vp * E) != cudaSuccess) {
        rc = fail(ctx, CULDA_ERR_OOM, "culda_encoder_init_from_phi: out of device memory");
    } else {
        const size_t smem = (size_t)K * sizeof(int);
        cudaError_t e = allow_smem(reinterpret_cast<const void *>(&phi_profile_kernel), smem, s);
        if (e == cudaSuccess) {
            phi_profile_kernel<<<std::min(Vp, num_sms(ctx->device) * 8), 256, smem, s>>>(
                V, Vp, K, ctx->params.beta, ctx->d_word_ptr, ctx->d_z[ctx->cur], prof);
            projection_kernel<<<grid_for((int64_t)E * K), 256, 0, s>>>(E * K, seed, R);
            e = cudaGetLastError();
        }
        GemmEpilogue ep;
        ep.out_f32 = P;
        ep.ldo = E;
        if (e == cudaSuccess) e = gemm_bf16_nt(Vp, E, K, prof, K, R, K, kEpiF32, ep, ctx->d_error, s);
        if (e == cudaSuccess) {
            rms_rows_kernel<<<grid_for((int64_t)V * 32), 256, 0, s>>>(V, E, 0.3f, P,
                                                                      encoder_tensor(enc, CULDA_ENC_E));
            e = cudaGetLastError();
        }
        if (e != cudaSuccess) rc = fail(ctx, CULDA_ERR_CUDA, "culda_encoder_init_from_phi: %s", cudaGetErrorString(e));
        if (rc == CULDA_OK && encoder_refresh(enc, s) != CULDA_OK)
            rc = fail(ctx, CULDA_ERR_CUDA, "culda_encoder_init_from_phi: %s", global_error());
        if (rc == CULDA_OK) rc = check_device_error(ctx, "culda_encoder_init_from_phi");
    }
    cudaStreamSynchronize(s);
    if (prof) cudaFree(prof);
    if (R) cudaFree(R);
    if (P) cudaFree(P);
    return rc;
}

extern "C" int culda_set_proposal(culda_ctx *ctx, culda_encoder *enc, float mix) {
    if (!ctx) return fail(ctx, CULDA_ERR_INVALID_ARG, "culda_set_proposal: null context");
    if (!enc) {
        ctx->has_proposal = false;
        return CULDA_OK;
    }
    if (!(mix >= 0.f && mix < 1.f)) return fail(ctx, CULDA_ERR_INVALID_ARG, "culda_set_proposal: mix outside [0, 1)");
    if (encoder_k(enc) != ctx->K || encoder_num_words(enc) != ctx->V)
        return fail(ctx, CULDA_ERR_INVALID_ARG, "culda_set_proposal: encoder shape does not match the context");
    CK(cudaSetDevice(ctx->device));
    int rc = ensure_doc_words(ctx);
    if (rc) return rc;
    cudaStream_t s = ctx->stream;
    const int B = encoder_max_batch(enc), K = ctx->K;
    if (!ctx->d_cdf) CK(dalloc(&ctx->d_cdf, (size_t)ctx->D * K));
    if (!ctx->d_cdf_blk) CK(dalloc(&ctx->d_cdf_blk, (size_t)ctx->D * (K / 32)));
    if (ctx->d_probs) cudaFree(ctx->d_probs);
    ctx->d_probs = nullptr;
    CK(dalloc(&ctx->d_probs, (size_t)B * K));
    int32_t *d_docs = nullptr;
    CK(dalloc(&d_docs, (size_t)B));
    std::vector<int32_t> ids((size_t)B);
    for (int32_t d0 = 0; d0 < ctx->D && rc == CULDA_OK; d0 += B) {
        const int n = std::min(B, ctx->D - d0);
        std::iota(ids.begin(), ids.begin() + n, d0);
        if (cudaMemcpyAsync(d_docs, ids.data(), sizeof(int32_t) * (size_t)n, cudaMemcpyHostToDevice, s) !=
            cudaSuccess) {
            rc = fail(ctx, CULDA_ERR_CUDA, "culda_set_proposal: upload failed");
            break;
        }
        rc = encoder_pass(enc, n, d_docs, ctx->d_doc_ptr, ctx->d_doc_words, nullptr, false, ctx->d_probs, s);
        if (rc) {
            fail(ctx, rc, "culda_set_proposal: %s", global_error());
            break;
        }
        proposal_table_kernel<<<grid_for((int64_t)n * 32), 256, 0, s>>>(n, d0, K, mix, ctx->d_probs, ctx->d_cdf,
                                                                       ctx->d_cdf_blk);
        if (cudaGetLastError() != cudaSuccess) rc = fail(ctx, CULDA_ERR_CUDA, "culda_set_proposal: launch failed");
        // the host ids buffer is rewritten for the next batch
        if (cudaStreamSynchronize(s) != cudaSuccess) rc = fail(ctx, CULDA_ERR_CUDA, "culda_set_proposal: sync failed");
    }
    cudaFree(d_docs);
    if (rc) return rc;
    rc = encoder_take_loss(enc, 0, nullptr, s);
    if (rc) return fail(ctx, rc, "culda_set_proposal: %s", global_error());
    ctx->has_proposal = true;
    return CULDA_OK;
}

extern "C" int culda_get_proposal(culda_ctx *ctx, float *cdf) {
    if (!ctx || !cdf) return fail(ctx, CULDA_ERR_INVALID_ARG, "culda_get_proposal: null argument");
    if (!ctx->has_proposal) return fail(ctx, CULDA_ERR_INVALID_ARG, "culda_get_proposal: no proposal set");
    CK(cudaSetDevice(ctx->device));
    CK(cudaStreamSynchronize(ctx->stream));
    CK(cudaMemcpy(cdf, ctx->d_cdf, sizeof(float) * (size_t)ctx->D * ctx->K, cudaMemcpyDeviceToHost));
    return CULDA_OK;
}

extern "C" int culda_iterate_mh(culda_ctx *ctx, int32_t n, int32_t steps, culda_iter_stats *stats) {
    if (!ctx || n < 0 || steps < 1 || steps > 64)
        return fail(ctx, CULDA_ERR_INVALID_ARG, "culda_iterate_mh: invalid argument");
    CK(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    for (int i = 0; i < n; ++i) {
        const int cur = ctx->cur, nxt = 1 - cur;
        const uint32_t iteration = ctx->next_iteration;
        CK(cudaEventRecord(ctx->ev0, s));
        int rc = launch_mh_pass(ctx, cur, iteration, steps);
        if (rc) return rc;
        CK(cudaMemsetAsync(ctx->d_nk, 0, sizeof(int32_t) * (size_t)ctx->K, s));
        CK(cudaMemsetAsync(&ctx->d_stats->row_entries, 0, 3 * sizeof(int64_t), s));
        CK(record_event(ctx->ev_t0, s));
        CK(launch_theta_rebuild(ctx->K, ctx->D, ctx->d_doc_ptr, ctx->d_doc_tok, ctx->d_z[nxt], ctx->d_doc_order,
                                ctx->d_rows, ctx->d_theta, ctx->d_nk, &ctx->d_stats->row_entries, ctx->d_error,
                                ctx->theta_grid, s));
        CK(record_event(ctx->ev_t1, s));
        bump_iteration_kernel<<<1, 1, 0, s>>>(ctx->d_iter);
        CK(cudaGetLastError());
        CK(cudaEventRecord(ctx->ev1, s));
        DevStats h{};
        unsigned long long mh[2] = {0, 0};
        int32_t err = 0;
        CK(cudaMemcpyAsync(&h, ctx->d_stats, sizeof(DevStats), cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(mh, ctx->d_mh_stats, sizeof(mh), cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(&err, ctx->d_error, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        float ms = 0.f, ms_s = 0.f, ms_t = 0.f;
        CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
        CK(cudaEventElapsedTime(&ms_s, ctx->ev_s0, ctx->ev_s1));
        CK(cudaEventElapsedTime(&ms_t, ctx->ev_t0, ctx->ev_t1));
        ctx->cur = nxt;
        ctx->next_iteration = iteration + 1;
        if (stats) {
            culda_iter_stats &o = stats[i];
            o = culda_iter_stats{};
            o.iteration = (int32_t)iteration;
            o.status = err;
            o.seconds = ms * 1e-3;
            o.loglik = NAN;
            o.tokens_per_sec = ms > 0 ? (double)ctx->N / (ms * 1e-3) : 0.0;
            o.row_entries = h.row_entries;
            o.theta_nnz = h.nnz;
            o.token_nnz = h.token_nnz;
            o.sample_seconds = ms_s * 1e-3;
            o.rebuild_seconds = ms_t * 1e-3;
            o.accept_rate = mh[1] ? (double)mh[0] / (double)mh[1] : 0.0;
        }
        if (err) return fail(ctx, CULDA_ERR_DEVICE_STATE, "culda_iterate_mh: device error 0x%x", err);
    }
    return CULDA_OK;
}

extern "C" int culda_mh_snapshot(culda_ctx *ctx, uint32_t iteration, int32_t steps, uint16_t *topics_out) {
    if (!ctx || steps < 1 || steps > 64) return fail(ctx, CULDA_ERR_INVALID_ARG, "culda_mh_snapshot: invalid argument");
    CK(cudaSetDevice(ctx->device));
    int rc = launch_mh_pass(ctx, ctx->cur, iteration, steps);
    if (rc) return rc;
    rc = check_device_error(ctx, "culda_mh_snapshot");
    if (rc) return rc;
    if (!topics_out) return CULDA_OK;
    return topics_to_host(ctx, ctx->d_z[1 - ctx->cur], topics_out);
}

extern "C" int culda_set_frozen_phi(culda_ctx *ctx, const int32_t *phi, const int32_t *nk) {
    if (!ctx) return fail(ctx, CULDA_ERR_INVALID_ARG, "culda_set_frozen_phi: null context");
    CK(cudaSetDevice(ctx->device));
    CK(cudaStreamSynchronize(ctx->stream));
    if (ctx->frozen_borrowed) {  // shared counts of a chunked run: the caller's buffers
        ctx->d_frozen_phi = nullptr;
        ctx->d_frozen_nk = nullptr;
        ctx->frozen_borrowed = false;
    }
    if (!phi) {
        if (ctx->d_frozen_phi) cudaFree(ctx->d_frozen_phi);
        if (ctx->d_frozen_nk) cudaFree(ctx->d_frozen_nk);
        ctx->d_frozen_phi = nullptr;
        ctx->d_frozen_nk = nullptr;
        return build_graphs(ctx);
    }
    if (!nk) return fail(ctx, CULDA_ERR_INVALID_ARG, "culda_set_frozen_phi: phi without nk");
    const size_t n = (size_t)ctx->V * ctx->K;
    // the counts must be consistent: non-negative, and the rows summing to nk
    std::vector<int64_t> sum((size_t)ctx->K, 0);
    for (size_t i = 0; i < n; ++i) {
        if (phi[i] < 0) return fail(ctx, CULDA_ERR_INVALID_ARG, "culda_set_frozen_phi: negative count");
        sum[i % ctx->K] += phi[i];
    }
    for (int32_t k = 0; k < ctx->K; ++k)
        if (sum[(size_t)k] != nk[k])
            return fail(ctx, CULDA_ERR_INVALID_ARG, "culda_set_frozen_phi: nk[%d] = %d but phi sums to %lld", k, nk[k],
                        (long long)sum[(size_t)k]);
    if (!ctx->d_frozen_phi) CK(dalloc(&ctx->d_frozen_phi, n));
    if (!ctx->d_frozen_nk) CK(dalloc(&ctx->d_frozen_nk, (size_t)ctx->K));
    CK(cudaMemcpy(ctx->d_frozen_phi, phi, sizeof(int32_t) * n, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(ctx->d_frozen_nk, nk, sizeof(int32_t) * (size_t)ctx->K, cudaMemcpyHostToDevice));
    return build_graphs(ctx);
}

extern "C" int culda_warm_start(culda_ctx *ctx) {
    if (!ctx) return fail(ctx, CULDA_ERR_INVALID_ARG, "culda_warm_start: null context");
    if (!ctx->has_proposal) return fail(ctx, CULDA_ERR_INVALID_ARG, "culda_warm_start: no proposal (culda_set_proposal)");
    CK(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    const int cur = ctx->cur;
    CK(cudaMemsetAsync(ctx->d_counter, 0, sizeof(int32_t), s));
    int rc = hot_rows_if_needed(ctx, cur);
    if (rc) return rc;
    const size_t smem = 3 * (size_t)ctx->K * sizeof(float);
    int grid = 1;
    rc = persistent_grid(ctx, warm_start_kernel, smem, &grid);
    if (rc) return rc;
    warm_start_kernel<<<grid, kMHThreads, smem, s>>>(mh_params(ctx, cur, 0u, 0));
    CK(cudaGetLastError());
    rc = check_device_error(ctx, "culda_warm_start");
    if (rc) return rc;
    ctx->cur = 1 - cur;
    return rebuild_counts(ctx);
}
