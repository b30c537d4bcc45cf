// context.cu — the context API: device state of one corpus on one GPU, its
// set-up, the iteration captured as CUDA graphs, and copy-out in the
// reference's layouts.
//
// Replaces SingleChunkSingleGPU (src_culda/train/SingleChunkSingleGPU.h:5-157)
// and the device-owning parts of DocChunk, ModelPhi/ModelPhiGPU and
// ModelTheta/ModelThetaChunk.  One iteration is one graph launch:
//   memset(work counter, hot rows) -> hot_rows -> sample(z[c] -> z[1-c])
//   -> finalize_ll -> memset(n_k, stats) -> theta_rebuild(z[1-c])
//   -> stats D2H (pinned)
// Two graphs alternate the topic buffers (z is double-buffered so hot words
// split over several CTAs read a stable snapshot while others write).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <fstream>
#include <map>
#include <mutex>
#include <numeric>
#include <sstream>
#include <string>
#include <vector>

#include "context.h"
#include "kernels.cuh"
#include "philox.h"

using namespace culda;


namespace {

// ------------------------------------------------------------ autotuner
// Sampler variants and theta-rebuild bin thresholds are timed on the
// context's state; the fastest of each is kept.  Results are remembered per
// (device name, N, D, V, K): in the process, and in the file named by
// CULDA_TUNE_CACHE (lines "key group_lanes sample_blocks ms theta_min_len")
// when that variable is set.  theta_min_len 0 means every doc is rebuilt by
// one warp.
struct TuneResult {
    int group_lanes = 0, sample_blocks = 0;
    float ms = 0.f;
    int theta_min_len = -1;  // -1: not tuned (a cache line written before the rebuild was tuned)
};

std::mutex g_tune_mu;
std::map<std::string, TuneResult> g_tune_cache;

std::string tune_key(const culda_ctx *ctx) {
    cudaDeviceProp prop{};
    if (cudaGetDeviceProperties(&prop, ctx->device) != cudaSuccess) prop.name[0] = 0;
    std::ostringstream k;
    std::string name(prop.name);
    std::replace(name.begin(), name.end(), ' ', '_');
    k << name << ":N" << ctx->N << ":D" << ctx->D << ":V" << ctx->V << ":K" << ctx->K;
    return k.str();
}

bool tune_lookup(const std::string &key, TuneResult &r) {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) {
        r = it->second;
        return true;
    }
    const char *path = std::getenv("CULDA_TUNE_CACHE");
    if (!path || !*path) return false;
    std::ifstream f(path);
    std::string line;
    bool found = false;
    while (std::getline(f, line)) {
        std::istringstream ls(line);
        std::string k;
        TuneResult t;
        if (ls >> k >> t.group_lanes >> t.sample_blocks >> t.ms && k == key &&
            sample_variant_exists(t.group_lanes, t.sample_blocks)) {
            if (!(ls >> t.theta_min_len) || t.theta_min_len < 0) t.theta_min_len = -1;
            r = t;
            found = true;  // the last line for a key wins
        }
    }
    if (found) g_tune_cache[key] = r;
    return found;
}

void tune_store(const std::string &key, const TuneResult &r) {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_tune_cache[key] = r;
    const char *path = std::getenv("CULDA_TUNE_CACHE");
    if (!path || !*path) return;
    std::ofstream f(path, std::ios::app);
    f << key << ' ' << r.group_lanes << ' ' << r.sample_blocks << ' ' << r.ms << ' ' << r.theta_min_len << '\n';
}

}  // namespace

int fail(culda_ctx *c, int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (c) c->err = buf;
    set_global_error("%s", buf);
    return code;
}


// Queue counter of the theta rebuild's block bin: its own 64-byte line of the
// counter array (slot 0 is the sampler's work queue).
static int32_t *theta_queue(culda_ctx *ctx) { return ctx->d_counter + 16; }

// Docs of at least min_len tokens (a prefix of the longest-first doc order).
static int count_long_docs(const culda_ctx *ctx, int min_len) {
    if (min_len <= 0) return 0;
    int n = 0;
    for (int d = 0; d < ctx->D; ++d) n += (ctx->h_doc_ptr[(size_t)d + 1] - ctx->h_doc_ptr[(size_t)d]) >= min_len;
    return n;
}

static void set_theta_bins(culda_ctx *ctx, int min_len) {
    ctx->theta_min_len = min_len > 0 ? min_len : 0;
    ctx->theta_long = count_long_docs(ctx, ctx->theta_min_len);
}

// Default bin threshold: a doc whose tokens outnumber a warp's average share
// of the corpus (N over the launch's warps) would hold its warp past the rest
// of the launch, so it gets a whole CTA; never below 1024 tokens.
static int default_theta_min_len(const culda_ctx *ctx) {
    const int64_t warps = (int64_t)ctx->theta_grid * kThetaWarps;
    return (int)std::min<int64_t>(65536, std::max<int64_t>(1024, ctx->N / std::max<int64_t>(1, warps)));
}

// Sampler parameters for topics d_z[cur] -> d_z[1-cur]; the Philox iteration
// comes from the device counter when iteration_ptr is set (graph launches).
SampleParams sample_params(const culda_ctx *ctx, int cur, uint32_t iteration, const uint32_t *iteration_ptr) {
    SampleParams p{};
    p.k = ctx->K;
    p.kmask = pow2_ceil(ctx->K) - 1;
    p.alpha = ctx->params.alpha;
    p.beta = ctx->params.beta;
    p.vbeta = ctx->params.beta * (float)ctx->V;
    p.num_docs = ctx->D;
    p.num_items = ctx->num_items;
    p.num_hot = ctx->num_hot;
    p.num_tokens = ctx->N;
    p.theta_cap = ctx->theta_cap;
    p.doc_ids = ctx->d_doc_ids;
    p.tok_index = ctx->d_tok_index;
    p.uniforms = ctx->d_u;
    p.topics_in = ctx->d_z[cur];
    p.topics_out = ctx->d_z[1 - cur];
    p.theta = ctx->d_theta;
    p.rows = ctx->d_rows;
    p.nk = ctx->d_nk;
    p.items = ctx->d_items;
    p.seg_start = ctx->d_seg_start;
    p.num_segs = ctx->num_segs;
    p.hot_phi = ctx->d_hot_phi;
    p.frozen_phi = ctx->d_frozen_phi;
    if (ctx->d_frozen_phi) p.nk = ctx->d_frozen_nk;
    p.item_counter = ctx->d_counter;
    p.item_ll = ctx->d_item_ll;
    p.seed = ctx->params.seed;
    p.iteration = iteration;
    p.iteration_ptr = iteration_ptr;
    p.error = ctx->d_error;
    return p;
}

namespace {

__global__ void copy_error_kernel(const int32_t *err, DevStats *st) { st->error = *err; }

}  // namespace

// Inside a stream capture a plain event record only orders the capture; the
// external flag turns it into an event-record node of the graph so the event
// can be timed after each launch.
cudaError_t record_event(cudaEvent_t ev, cudaStream_t s) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaError_t e = cudaStreamIsCapturing(s, &cs);
    if (e != cudaSuccess) return e;
    return cs == cudaStreamCaptureStatusActive ? cudaEventRecordWithFlags(ev, s, cudaEventRecordExternal)
                                               : cudaEventRecord(ev, s);
}

namespace {

int record_iteration(culda_ctx *ctx, cudaStream_t s, int cur) {
    const int nxt = 1 - cur;
    CK(cudaMemsetAsync(ctx->d_counter, 0, sizeof(int32_t), s));
    if (ctx->num_hot > 0 && !ctx->d_frozen_phi) {
        CK(cudaMemsetAsync(ctx->d_hot_phi, 0, sizeof(int32_t) * (size_t)ctx->num_hot * ctx->K, s));
        CK(launch_hot_rows(ctx->K, ctx->d_hot_items, ctx->num_hot_items, ctx->d_z[cur], ctx->d_hot_phi, ctx->d_error,
                           s));
    }
    CK(launch_uniforms(ctx->N, ctx->params.seed, ctx->d_iter, 0u, ctx->d_tok_index, ctx->d_u, s));
    CK(record_event(ctx->ev_s0, s));
    CK(launch_sample(sample_params(ctx, cur, 0u, ctx->d_iter), ctx->group_lanes, ctx->sample_blocks,
                     ctx->sample_grid, s));
    CK(record_event(ctx->ev_s1, s));
    CK(launch_finalize_ll(ctx->d_item_ll, ctx->num_items, ctx->d_stats, ctx->d_iter, s));
    CK(cudaMemsetAsync(ctx->d_nk, 0, sizeof(int32_t) * (size_t)ctx->K, s));
    CK(cudaMemsetAsync(&ctx->d_stats->row_entries, 0, 3 * sizeof(int64_t), s));
    CK(record_event(ctx->ev_t0, s));
    CK(launch_theta_rebuild(ctx->K, ctx->D, ctx->d_doc_ptr, ctx->d_doc_tok, ctx->d_z[nxt], ctx->d_doc_order,
                            ctx->d_rows, ctx->d_theta, ctx->d_nk, &ctx->d_stats->row_entries, ctx->d_error,
                            ctx->theta_grid, s, ctx->theta_long, theta_queue(ctx)));
    CK(record_event(ctx->ev_t1, s));
    copy_error_kernel<<<1, 1, 0, s>>>(ctx->d_error, ctx->d_stats);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(ctx->h_stats, ctx->d_stats, sizeof(DevStats), cudaMemcpyDeviceToHost, s));
    return CULDA_OK;
}

}  // namespace

// Rebuild theta rows and n_k from the current topics (set-up and set_topics).
int rebuild_counts(culda_ctx *ctx) {
    cudaStream_t s = ctx->stream;
    CK(cudaMemsetAsync(ctx->d_nk, 0, sizeof(int32_t) * (size_t)ctx->K, s));
    CK(cudaMemsetAsync(&ctx->d_stats->row_entries, 0, 3 * sizeof(int64_t), s));
    CK(launch_theta_rebuild(ctx->K, ctx->D, ctx->d_doc_ptr, ctx->d_doc_tok, ctx->d_z[ctx->cur], ctx->d_doc_order,
                            ctx->d_rows, ctx->d_theta, ctx->d_nk, &ctx->d_stats->row_entries, ctx->d_error,
                            ctx->theta_grid, s, ctx->theta_long, theta_queue(ctx)));
    CK(cudaStreamSynchronize(s));
    int32_t e = 0;
    CK(cudaMemcpy(&e, ctx->d_error, sizeof(int32_t), cudaMemcpyDeviceToHost));
    if (e) return fail(ctx, CULDA_ERR_DEVICE_STATE, "theta rebuild reported device error 0x%x", e);
    return CULDA_OK;
}

namespace {

constexpr uint32_t kTuneIteration = 3;

// Times the theta rebuild of the current topics at each candidate bin
// threshold (0 = warp per doc for every doc) and keeps the fastest.  The
// rebuild of the same topics writes the same rows and n_k, so the state does
// not change.
int autotune_rebuild(culda_ctx *ctx, TuneResult &best) {
    cudaStream_t s = ctx->stream;
    const int dflt = default_theta_min_len(ctx);
    const int cands[] = {0, dflt, 65535, 16384, 8192, 4096, 2048, 1024, 512, 256};
    std::vector<int> seen_long;
    float best_ms = 0.f;
    int best_len = 0;
    for (int len : cands) {
        const int nl = count_long_docs(ctx, len);
        if (len > 0 && nl == 0) continue;
        if (std::find(seen_long.begin(), seen_long.end(), nl) != seen_long.end()) continue;  // same bins
        seen_long.push_back(nl);
        float t = 0.f;
        for (int rep = 0; rep < 3; ++rep) {
            CK(cudaMemsetAsync(ctx->d_nk, 0, sizeof(int32_t) * (size_t)ctx->K, s));
            CK(cudaMemsetAsync(&ctx->d_stats->row_entries, 0, 3 * sizeof(int64_t), s));
            CK(cudaEventRecord(ctx->ev0, s));
            CK(launch_theta_rebuild(ctx->K, ctx->D, ctx->d_doc_ptr, ctx->d_doc_tok, ctx->d_z[ctx->cur],
                                    ctx->d_doc_order, ctx->d_rows, ctx->d_theta, ctx->d_nk,
                                    &ctx->d_stats->row_entries, ctx->d_error, ctx->theta_grid, s, nl,
                                    theta_queue(ctx)));
            CK(cudaEventRecord(ctx->ev1, s));
            CK(cudaEventSynchronize(ctx->ev1));
            float ms = 0.f;
            CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
            if (rep == 1 || (rep == 2 && ms < t)) t = ms;
        }
        if (ctx->params.flags & CULDA_FLAG_VERBOSE)
            fprintf(stderr, "culda: autotune theta_min_len=%d (%d docs by a CTA): %.3f ms\n", len, nl, t);
        if (best_ms == 0.f || t < best_ms) {
            best_ms = t;
            best_len = len;
        }
    }
    best.theta_min_len = best_len;
    set_theta_bins(ctx, best_len);
    ctx->theta_tune_ms = best_ms;
    return CULDA_OK;
}

// Times each sampler variant on the current state: hot rows and
// uniforms once, then per variant one warm-up and two timed launches that
// write the other topic buffer.  The context's state does not change.
int autotune_sampler(culda_ctx *ctx) {
    static const int kCands[][2] = {{kFlatLanes, kSampleBlocksDefault}, {kFlatLanes, kFlatBlocks},
                                    {4, kSampleBlocksHigh},
                                    {8, kSampleBlocksHigh},                {16, kSampleBlocksHigh},
                                    {2, kSampleBlocksDefault},             {4, kSampleBlocksDefault},
                                    {8, kSampleBlocksDefault}};
    const std::string key = tune_key(ctx);
    TuneResult best;
    if (tune_lookup(key, best)) {
        const int bps = sample_blocks_per_sm(ctx->K, best.group_lanes, best.sample_blocks);
        if (bps > 0) {
            ctx->group_lanes = best.group_lanes;
            ctx->sample_blocks = best.sample_blocks;
            ctx->sample_grid = std::max(1, std::min(ctx->num_items, num_sms(ctx->device) * bps));
            ctx->tuned = 2;
            ctx->tune_ms = best.ms;
            if (best.theta_min_len >= 0) set_theta_bins(ctx, best.theta_min_len);
            return CULDA_OK;
        }
    }
    cudaStream_t s = ctx->stream;
    const int cur = ctx->cur;
    if (ctx->num_hot > 0 && !ctx->d_frozen_phi) {
        CK(cudaMemsetAsync(ctx->d_hot_phi, 0, sizeof(int32_t) * (size_t)ctx->num_hot * ctx->K, s));
        CK(launch_hot_rows(ctx->K, ctx->d_hot_items, ctx->num_hot_items, ctx->d_z[cur], ctx->d_hot_phi, ctx->d_error,
                           s));
    }
    CK(launch_uniforms(ctx->N, ctx->params.seed, nullptr, 1u, ctx->d_tok_index, ctx->d_u, s));
    const SampleParams sp = sample_params(ctx, cur, 1u, nullptr);
    best.ms = 0.f;
    for (const auto &c : kCands) {
        const int bps = sample_blocks_per_sm(ctx->K, c[0], c[1]);
        if (bps <= 0) continue;
        const int grid = std::max(1, std::min(ctx->num_items, num_sms(ctx->device) * bps));
        float t = 0.f;
        for (int rep = 0; rep < 3; ++rep) {
            CK(cudaMemsetAsync(ctx->d_counter, 0, sizeof(int32_t), s));
            CK(cudaEventRecord(ctx->ev0, s));
            CK(launch_sample(sp, c[0], c[1], grid, s));
            CK(cudaEventRecord(ctx->ev1, s));
            CK(cudaEventSynchronize(ctx->ev1));
            float ms = 0.f;
            CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
            if (rep == 1 || (rep == 2 && ms < t)) t = ms;
        }
        if (best.ms == 0.f || t < best.ms) {
            best.group_lanes = c[0];
            best.sample_blocks = c[1];
            best.ms = t;
        }
        if (ctx->params.flags & CULDA_FLAG_VERBOSE)
            fprintf(stderr, "culda: autotune G=%d blocks=%d grid=%d: %.3f ms\n", c[0], c[1], grid, t);
    }
    int32_t e = 0;
    CK(cudaMemcpy(&e, ctx->d_error, sizeof(int32_t), cudaMemcpyDeviceToHost));
    if (e) return fail(ctx, CULDA_ERR_DEVICE_STATE, "autotune: sampler reported device error 0x%x", e);
    if (best.ms == 0.f) return fail(ctx, CULDA_ERR_CUDA, "autotune: no sampler variant fits the device");
    ctx->group_lanes = best.group_lanes;
    ctx->sample_blocks = best.sample_blocks;
    ctx->sample_grid = std::max(
        1, std::min(ctx->num_items, num_sms(ctx->device) * sample_blocks_per_sm(ctx->K, best.group_lanes,
                                                                                 best.sample_blocks)));
    ctx->tuned = 1;
    ctx->tune_ms = best.ms;
    const int rc = autotune_rebuild(ctx, best);
    if (rc) return rc;
    CK(cudaMemcpy(&e, ctx->d_error, sizeof(int32_t), cudaMemcpyDeviceToHost));
    if (e) return fail(ctx, CULDA_ERR_DEVICE_STATE, "autotune: theta rebuild reported device error 0x%x", e);
    tune_store(key, best);
    return CULDA_OK;
}

}  // namespace

int build_graphs(culda_ctx *ctx) {
    for (int c = 0; c < 2; ++c) {
        if (ctx->graph[c]) {
            cudaGraphExecDestroy(ctx->graph[c]);
            ctx->graph[c] = nullptr;
        }
        if (ctx->params.flags & CULDA_FLAG_NO_GRAPH) continue;
        cudaGraph_t g = nullptr;
        CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
        int rc = record_iteration(ctx, ctx->stream, c);
        cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
        if (rc != CULDA_OK) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        CK(e);
        e = cudaGraphInstantiate(&ctx->graph[c], g, 0);
        cudaGraphDestroy(g);
        CK(e);
    }
    return CULDA_OK;
}

namespace {

int pick_group_lanes(int requested, int k) {
    if (requested == kFlatLanes || requested == 1 || requested == 2 || requested == 4 || requested == 8 ||
        requested == 16 || requested == 32)
        return requested;
    // the warp-flattened walk is the fastest variant on every measured
    // workload (60M tokens at K = 1024; 118M uneven tokens at K = 256..4096)
    (void)k;
    return requested == 0 ? kFlatLanes : 0;  // 0: not a variant
}

// the flat walk's default is the 56-register build (9 CTAs per SM), the
// group samplers' the 64-register one
int pick_sample_blocks(int requested, int group_lanes) {
    if (requested != 0) return requested;
    return group_lanes == kFlatLanes ? kFlatBlocks : kSampleBlocksDefault;
}


}  // namespace

// ------------------------------------------------------------- work items
// Work items, largest first (a counting sort on the token count, which is at
// most item_tokens <= 65535; stable, so equal counts keep word order).  Two
// passes over the words: the first counts the items of every size, the
// second writes each item straight to its sorted place (no intermediate list
// to grow and copy: at 100k words that took most of the builder's 4-6 ms).
std::vector<culda_item> build_items_vec(int32_t num_words, const int64_t *word_ptr, int32_t item_tokens,
                                        int32_t *num_hot) {
    std::vector<int64_t> start((size_t)item_tokens + 2, 0);
    int32_t hot = 0;
    // the slices of a word of len > item_tokens tokens: ns slices of sz tokens,
    // the last one shorter (as the reference splits hot words into slots,
    // doc_chunk.cpp:167-185)
    auto slices = [item_tokens](int64_t len, int64_t &ns, int64_t &sz) {
        ns = (len + item_tokens - 1) / item_tokens;
        sz = (len + ns - 1) / ns;
    };
    for (int32_t w = 0; w < num_words; ++w) {
        const int64_t len = word_ptr[w + 1] - word_ptr[w];
        if (len <= 0) continue;
        if (len <= item_tokens) {
            start[(size_t)(item_tokens - len) + 1]++;
        } else {
            int64_t ns, sz;
            slices(len, ns, sz);
            for (int64_t i = 0; i < ns; ++i) {
                const int64_t e = std::min((i + 1) * sz, len) - i * sz;
                if (e > 0) start[(size_t)(item_tokens - e) + 1]++;
            }
        }
    }
    for (size_t k = 1; k < start.size(); ++k) start[k] += start[k - 1];
    std::vector<culda_item> out((size_t)start.back());
    for (int32_t w = 0; w < num_words; ++w) {
        const int64_t len = word_ptr[w + 1] - word_ptr[w];
        if (len <= 0) continue;
        if (len <= item_tokens) {
            out[(size_t)start[(size_t)(item_tokens - len)]++] = culda_item{word_ptr[w], (int32_t)len, w, -1, 1};
        } else {
            int64_t ns, sz;
            slices(len, ns, sz);
            for (int64_t i = 0; i < ns; ++i) {
                const int64_t b = word_ptr[w] + i * sz, e = std::min(b + sz, word_ptr[w + 1]);
                if (e > b)
                    out[(size_t)start[(size_t)(item_tokens - (e - b))]++] =
                        culda_item{b, (int32_t)(e - b), w, hot, i == 0 ? 1 : 0};
            }
            ++hot;
        }
    }
    if (num_hot) *num_hot = hot;
    return out;
}

extern "C" int64_t culda_build_items(int32_t num_words, const int64_t *word_ptr, int32_t item_tokens,
                                     culda_item *items, int64_t max_items, int32_t *num_hot) {
    if (num_words <= 0 || !word_ptr || item_tokens <= 0 || item_tokens > 65535) {
        set_global_error("culda_build_items: invalid argument");
        return CULDA_ERR_INVALID_ARG;
    }
    const std::vector<culda_item> v = build_items_vec(num_words, word_ptr, item_tokens, num_hot);
    if (items) {
        if ((int64_t)v.size() > max_items) {
            set_global_error("culda_build_items: %zu items do not fit in %lld", v.size(), (long long)max_items);
            return CULDA_ERR_INVALID_ARG;
        }
        std::copy(v.begin(), v.end(), items);
    }
    return (int64_t)v.size();
}

extern "C" int64_t culda_build_segments(int64_t num_tokens, const int32_t *doc_ids, culda_item *items,
                                        int32_t num_items, int32_t max_len, int32_t *seg_start, int64_t max_segs) {
    if (num_tokens <= 0 || !doc_ids || !items || num_items <= 0 || max_len <= 0) {
        set_global_error("culda_build_segments: invalid argument");
        return CULDA_ERR_INVALID_ARG;
    }
    int64_t n = 0;
    for (int32_t i = 0; i < num_items; ++i) {
        culda_item &it = items[i];
        if (it.begin < 0 || it.count <= 0 || it.begin + it.count > num_tokens) {
            set_global_error("culda_build_segments: item %d outside the token range", i);
            return CULDA_ERR_INVALID_ARG;
        }
        const int64_t first = n;
        int64_t len = 0;
        for (int64_t t = it.begin; t < it.begin + it.count; ++t) {
            if (t == it.begin || doc_ids[t] != doc_ids[t - 1] || len == max_len) {
                if (seg_start) {
                    if (n >= max_segs) {
                        set_global_error("culda_build_segments: more than %lld segments", (long long)max_segs);
                        return CULDA_ERR_INVALID_ARG;
                    }
                    seg_start[n] = (int32_t)t;
                }
                ++n;
                len = 0;
            }
            ++len;
        }
        if (n >= INT32_MAX) return CULDA_ERR_UNSUPPORTED;
        it.seg_begin = (int32_t)first;
        it.seg_count = (int32_t)(n - first);
    }
    return n;
}

namespace {

constexpr int kSegmentMax = 32;  // tokens per segment (bounds the work of one group on one row)

// key[t] = t where a run of one doc starts (doc change), else 0; item starts
// are added by item_keys_kernel
__global__ void run_key_kernel(int64_t n, const int32_t *__restrict__ doc_ids, int32_t *key) {
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
        key[t] = (t == 0 || doc_ids[t] != doc_ids[t - 1]) ? (int32_t)t : 0;
}

// every item starts a run
__global__ void item_keys_kernel(const culda_item *__restrict__ items, int num_items, int32_t *key) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < num_items; i += gridDim.x * blockDim.x)
        key[items[i].begin] = (int32_t)items[i].begin;
}

struct MaxOp {
    __device__ __forceinline__ int32_t operator()(int32_t a, int32_t b) const { return a > b ? a : b; }
};

// flag[t] = 1 where a segment starts: every max_len tokens from a run start
__global__ void seg_flag_kernel(int64_t n, const int32_t *__restrict__ run_start, int32_t *flag) {
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t <= n; t += (int64_t)gridDim.x * blockDim.x)
        flag[t] = t < n && ((t - run_start[t]) % kSegmentMax) == 0 ? 1 : 0;
}

__global__ void seg_scatter_kernel(int64_t n, const int32_t *__restrict__ flag, const int32_t *__restrict__ index,
                                   int32_t *seg_start) {
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
        if (flag[t]) seg_start[index[t]] = (int32_t)t;
}

__global__ void item_segments_kernel(culda_item *items, int num_items, const int32_t *__restrict__ index) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < num_items; i += gridDim.x * blockDim.x) {
        culda_item &it = items[i];
        it.seg_begin = index[it.begin];
        it.seg_count = index[it.begin + it.count] - it.seg_begin;
    }
}

// A process-wide pool of pinned DevStats slots: a cudaMallocHost costs
// milliseconds, so contexts take slots from shared pinned pages and give them
// back on destroy (the pages live as long as the process).
std::mutex g_pinned_mu;
std::vector<DevStats *> g_pinned_free;

DevStats *pinned_stats_get() {
    std::lock_guard<std::mutex> lock(g_pinned_mu);
    if (g_pinned_free.empty()) {
        constexpr int kSlots = 64;
        DevStats *page = nullptr;
        if (cudaMallocHost((void **)&page, sizeof(DevStats) * kSlots) != cudaSuccess) return nullptr;
        for (int i = kSlots - 1; i >= 0; --i) g_pinned_free.push_back(page + i);
    }
    DevStats *p = g_pinned_free.back();
    g_pinned_free.pop_back();
    return p;
}

void pinned_stats_put(DevStats *p) {
    std::lock_guard<std::mutex> lock(g_pinned_mu);
    g_pinned_free.push_back(p);
}

// A process-wide stream-ordered memory pool per device for the contexts'
// blocks.  Its release threshold is "never", so a destroyed context's block
// stays reserved and the next culda_create on the device takes it back
// without mapping fresh pages (a cudaMalloc of the 1.9 GB block of the
// 60M-token corpus took 5 to 25 ms, and the cudaFree before it up to 20 ms);
// culda_trim_memory() hands the unused reserve back to the device.
constexpr int kPoolDevices = 64;
std::mutex g_pool_mu;
cudaMemPool_t g_pools[kPoolDevices] = {};

cudaMemPool_t block_pool(int device) {
    if (device < 0 || device >= kPoolDevices) return nullptr;
    std::lock_guard<std::mutex> lock(g_pool_mu);
    if (!g_pools[device]) {
        cudaMemPoolProps props;
        std::memset(&props, 0, sizeof(props));
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        cudaMemPool_t pool = nullptr;
        if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        uint64_t keep = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        g_pools[device] = pool;
    }
    return g_pools[device];
}

// Device space for the set-up's temporaries (sort keys and values, scan
// arrays, CUB scratch), carved by a bump allocator.  It is either a region of
// the context's block whose buffers are not used until set-up ends (owned =
// false) or, when that region is too small, one allocation of its own.
struct SetupArena {
    char *base = nullptr;
    size_t size = 0, used = 0;
    bool owned = false;
    void use(char *b, size_t s) {
        base = b;
        size = s;
        used = 0;
    }
    template <class T>
    T *take(size_t n) {
        const size_t bytes = (std::max<size_t>(n, 1) * sizeof(T) + 255) & ~(size_t)255;
        if (used + bytes > size) return nullptr;
        T *p = reinterpret_cast<T *>(base + used);
        used += bytes;
        return p;
    }
    void reset() { used = 0; }
};


// Segments of the stored token order, on the device (see culda_build_segments).
int build_segments_device(culda_ctx *ctx, SetupArena &arena) {
    cudaStream_t s = ctx->stream;
    const int64_t N = ctx->N;
    size_t tmp_bytes = 0, b2 = 0;
    int rc = CULDA_OK;
    auto grid = [](int64_t n) { return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 32)); };
    do {
#define CKS(call)                                                                                          \
    {                                                                                                      \
        cudaError_t e_ = (call);                                                                           \
        if (e_ != cudaSuccess) {                                                                           \
            rc = fail(ctx, CULDA_ERR_CUDA, "segments: %s: %s", #call, cudaGetErrorString(e_));             \
            break;                                                                                         \
        }                                                                                                  \
    }
        // two arrays: A holds the run keys, then the segment flags; B the run
        // starts, then the flags' exclusive prefix (the segment index)
        int32_t *A = arena.take<int32_t>((size_t)N + 1), *B = arena.take<int32_t>((size_t)N + 1);
        CKS(cub::DeviceScan::InclusiveScan(nullptr, tmp_bytes, A, B, MaxOp(), (int)N, s));
        CKS(cub::DeviceScan::ExclusiveSum(nullptr, b2, A, B, (int)N + 1, s));
        void *tmp = arena.take<char>(std::max(tmp_bytes, b2));
        if (!A || !B || !tmp) {
            rc = fail(ctx, CULDA_ERR_OOM, "segments: set-up arena too small");
            break;
        }
        tmp_bytes = std::max(tmp_bytes, b2);
        run_key_kernel<<<grid(N), 256, 0, s>>>(N, ctx->d_doc_ids, A);
        item_keys_kernel<<<grid(ctx->num_items), 256, 0, s>>>(ctx->d_items, ctx->num_items, A);
        CKS(cudaGetLastError());
        CKS(cub::DeviceScan::InclusiveScan(tmp, tmp_bytes, A, B, MaxOp(), (int)N, s));
        seg_flag_kernel<<<grid(N + 1), 256, 0, s>>>(N, B, A);
        CKS(cudaGetLastError());
        CKS(cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, A, B, (int)N + 1, s));
        int32_t total = 0;
        CKS(cudaMemcpyAsync(&total, B + N, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
        CKS(cudaStreamSynchronize(s));
        ctx->num_segs = total;  // d_seg_start holds one entry per token, the most there can be
        seg_scatter_kernel<<<grid(N), 256, 0, s>>>(N, A, B, ctx->d_seg_start);
        item_segments_kernel<<<grid(ctx->num_items), 256, 0, s>>>(ctx->d_items, ctx->num_items, B);
        CKS(cudaGetLastError());
        CKS(cudaStreamSynchronize(s));
#undef CKS
    } while (0);
    return rc;
}

}  // namespace

// --------------------------------------------------------------- create
extern "C" int culda_create(const culda_corpus *c, const culda_params *p, culda_ctx **out) {
    culda_ctx *ctx = nullptr;
    if (!c || !p || !out) return fail(ctx, CULDA_ERR_INVALID_ARG, "culda_create: null argument");
    *out = nullptr;
    if (p->k < 32 || p->k > 4096 || p->k % 32 != 0)
        return fail(ctx, CULDA_ERR_INVALID_ARG, "culda_create: K=%d must be a multiple of 32 in [32, 4096]", p->k);
    if (!(p->alpha > 0.f) || !(p->beta > 0.f) || !std::isfinite(p->alpha) || !std::isfinite(p->beta))
        return fail(ctx, CULDA_ERR_INVALID_ARG, "culda_create: alpha and beta must be positive");
    if (p->item_tokens < 0 || p->item_tokens > 65535)
        return fail(ctx, CULDA_ERR_INVALID_ARG, "culda_create: item_tokens=%d outside 0..65535", p->item_tokens);
    if ((p->flags & CULDA_FLAG_AUTOTUNE) && (p->group_lanes != 0 || p->sample_blocks != 0 || p->theta_min_len != 0))
        return fail(ctx, CULDA_ERR_INVALID_ARG,
                    "culda_create: CULDA_FLAG_AUTOTUNE needs group_lanes = sample_blocks = theta_min_len = 0");
    const int gl = pick_group_lanes(p->group_lanes, p->k);
    if (gl == 0) return fail(ctx, CULDA_ERR_INVALID_ARG, "culda_create: group_lanes=%d", p->group_lanes);
    const int sb = pick_sample_blocks(p->sample_blocks, gl);
    if (!sample_variant_exists(gl, sb))
        return fail(ctx, CULDA_ERR_INVALID_ARG, "culda_create: no sampler for group_lanes=%d sample_blocks=%d", gl,
                    p->sample_blocks);
    if (c->num_docs <= 0 || c->num_words <= 0 || c->num_tokens <= 0 || !c->doc_ptr || !c->word_ptr || !c->doc_ids)
        return fail(ctx, CULDA_ERR_INVALID_ARG, "culda_create: empty corpus");
    if (c->num_tokens >= (int64_t)INT32_MAX)
        return fail(ctx, CULDA_ERR_UNSUPPORTED, "culda_create: %lld tokens exceed the int32 token index",
                    (long long)c->num_tokens);
    if (c->doc_ptr[0] != 0 || c->word_ptr[0] != 0 || c->doc_ptr[c->num_docs] != c->num_tokens ||
        c->word_ptr[c->num_words] != c->num_tokens)
        return fail(ctx, CULDA_ERR_FORMAT, "culda_create: doc/word index totals do not match the token count");
    for (int32_t d = 0; d < c->num_docs; ++d) {
        const int64_t len = c->doc_ptr[d + 1] - c->doc_ptr[d];
        if (len < 0) return fail(ctx, CULDA_ERR_FORMAT, "culda_create: doc index decreases at doc %d", d);
        if (len > 65535)
            return fail(ctx, CULDA_ERR_UNSUPPORTED, "culda_create: doc %d has %lld tokens (theta counts are 16-bit)", d,
                        (long long)len);
    }
    for (int32_t w = 0; w < c->num_words; ++w)
        if (c->word_ptr[w + 1] < c->word_ptr[w])
            return fail(ctx, CULDA_ERR_FORMAT, "culda_create: word index decreases at word %d", w);
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0)
        return fail(ctx, CULDA_ERR_NO_DEVICE, "culda_create: no CUDA device");
    if (p->device < 0 || p->device >= ndev)
        return fail(ctx, CULDA_ERR_INVALID_ARG, "culda_create: device %d of %d", p->device, ndev);

    ctx = new culda_ctx();
    ctx->params = *p;
    ctx->device = p->device;
    ctx->D = c->num_docs;
    ctx->V = c->num_words;
    ctx->K = p->k;
    ctx->N = c->num_tokens;
    ctx->group_lanes = gl;
    ctx->sample_blocks = sb;
    int rc = CULDA_OK;
    SetupArena arena;  // the set-up's temporaries (sorts, segment scans)
    auto bail = [&](int code) {
        if (arena.owned && arena.base) cudaFree(arena.base);
        culda_destroy(ctx);
        return code;
    };
#define CKB(call)                                                                                              \
    do {                                                                                                       \
        cudaError_t e_ = (call);                                                                               \
        if (e_ != cudaSuccess) {                                                                               \
            fail(ctx, e_ == cudaErrorMemoryAllocation ? CULDA_ERR_OOM : CULDA_ERR_CUDA, "%s: %s", #call,       \
                 cudaGetErrorString(e_));                                                                      \
            set_global_error("%s", ctx->err.c_str());                                                          \
            return bail(e_ == cudaErrorMemoryAllocation ? CULDA_ERR_OOM : CULDA_ERR_CUDA);                     \
        }                                                                                                      \
    } while (0)

    CKB(cudaSetDevice(ctx->device));
    CKB(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
    CKB(cudaEventCreate(&ctx->ev0));
    CKB(cudaEventCreate(&ctx->ev1));
    CKB(cudaEventCreate(&ctx->ev_s0));
    CKB(cudaEventCreate(&ctx->ev_s1));
    CKB(cudaEventCreate(&ctx->ev_t0));
    CKB(cudaEventCreate(&ctx->ev_t1));
    cudaStream_t s = ctx->stream;
    const int64_t N = ctx->N;
    const int32_t D = ctx->D, V = ctx->V, K = ctx->K;
    // with CULDA_FLAG_VERBOSE, the wall time of each set-up phase (the stream
    // is synchronised at every mark, so the marks slow set-up down a little)
    const bool verbose = (p->flags & CULDA_FLAG_VERBOSE) != 0;
    auto t_last = std::chrono::steady_clock::now();
    auto mark = [&](const char *phase) {
        if (!verbose) return;
        cudaStreamSynchronize(s);
        const auto now = std::chrono::steady_clock::now();
        fprintf(stderr, "culda: set-up %-22s %8.2f ms\n", phase,
                std::chrono::duration<double, std::milli>(now - t_last).count());
        t_last = now;
    };

    // ---- host-side layout first: every persistent buffer's size is known
    // before the device is touched, so they all come from one allocation
    // (each cudaMalloc / cudaFree costs about a millisecond)
    const bool reorder = !(p->flags & CULDA_FLAG_NO_REORDER);
    // theta layout: capacity roundup32(min(L_d, K)) per doc (model_theta.cpp:50-56)
    ctx->h_doc_ptr.assign(c->doc_ptr, c->doc_ptr + D + 1);
    ctx->h_max_ia.resize((size_t)D + 1);
    std::vector<int2> rows((size_t)D);
    {
        std::vector<int64_t> docs_of_len(65536, 0);  // doc lengths are below 65536 (checked above)
        int64_t off = 0;
        for (int32_t d = 0; d < D; ++d) {
            int64_t len = c->doc_ptr[d + 1] - c->doc_ptr[d];
            docs_of_len[(size_t)len]++;
            if (len > K) len = K;
            len = (len + 31) / 32 * 32;
            if (off + len >= (int64_t)INT32_MAX) {
                fail(ctx, CULDA_ERR_UNSUPPORTED, "culda_create: theta capacity exceeds int32 offsets");
                return bail(CULDA_ERR_UNSUPPORTED);
            }
            ctx->h_max_ia[d] = (int32_t)off;
            rows[d] = make_int2((int)off, (int)off);
            off += len;
        }
        ctx->h_max_ia[D] = (int32_t)off;
        ctx->theta_cap = off;
        // sum_d L_d log(L_d + K alpha), one logarithm per distinct length
        for (size_t len = 1; len < docs_of_len.size(); ++len)
            if (docs_of_len[len])
                ctx->doc_term +=
                    (double)docs_of_len[len] * (double)len * std::log((double)len + (double)K * (double)p->alpha);
    }
    // grids
    const int sms = num_sms(ctx->device);
    int sbps = sample_blocks_per_sm(K, gl, sb);
    if (sbps <= 0) {
        fail(ctx, CULDA_ERR_CUDA, "culda_create: sampler does not fit on the device for K=%d", K);
        return bail(CULDA_ERR_CUDA);
    }
    int tbps = theta_blocks_per_sm(K);
    if (tbps <= 0) tbps = 1;
    ctx->theta_grid = std::max(1, std::min(sms * tbps, (D + kThetaWarps - 1) / kThetaWarps));
    set_theta_bins(ctx, p->theta_min_len > 0 ? p->theta_min_len
                        : p->theta_min_len < 0 ? 0 : default_theta_min_len(ctx));
    // work items: words, hot words split so that no item exceeds two thirds of
    // a CTA's share of the tokens (the largest go first; at 60M tokens items
    // of up to 11.5k, 32k, 49k and 65k tokens gave 6.33, 6.28, 7.17 and
    // 8.33 ms per sampler launch: items past a CTA's share leave a tail)
    std::vector<culda_item> items, hot;
    {
        int64_t it = p->item_tokens;
        if (it <= 0) it = std::max<int64_t>(1024, std::min<int64_t>(65535, 2 * N / ((int64_t)sms * sbps * 3)));
        ctx->item_tokens = (int)it;
        int32_t nhot = 0;
        items = build_items_vec(V, c->word_ptr, ctx->item_tokens, &nhot);
        if (items.empty() || (int64_t)items.size() >= INT32_MAX) {
            fail(ctx, CULDA_ERR_FORMAT, "culda_create: no tokens to sample");
            return bail(CULDA_ERR_FORMAT);
        }
        for (const culda_item &x : items)
            if (x.hot >= 0) hot.push_back(x);
        ctx->num_items = (int32_t)items.size();
        ctx->num_hot = nhot;
        ctx->num_hot_items = (int32_t)hot.size();
    }
    ctx->sample_grid = std::max(1, std::min(ctx->num_items, sms * sbps));

    // ---- one device block for every persistent buffer.  The buffers that
    // set-up does not touch until its end (doc-reverse index, segment starts,
    // topics, uniforms, theta) come last: while the sorts and scans run, that
    // region holds their temporaries instead of an allocation of its own.
    auto rnd = [](size_t bytes) { return (std::max<size_t>(bytes, 1) + 255) & ~(size_t)255; };
    size_t t_order = 0, t_doc = 0, t_scan = 0, t_sum = 0;
    // token-order keys: 32-bit (word, 8-bit length class) up to 2^24 words, else
    // 64-bit (word, exact length); the 32-bit sort moves a third of the bytes
    const bool key32 = V <= (1 << 24);
    int order_bits = key32 ? 9 : 17, doc_bits = 1;
    while ((1ll << (order_bits - (key32 ? 8 : 16))) < (int64_t)V) ++order_bits;
    while ((1ll << doc_bits) < (int64_t)D) ++doc_bits;
    if (key32)
        CKB(cub::DeviceRadixSort::SortPairs(nullptr, t_order, (const uint32_t *)nullptr, (uint32_t *)nullptr,
                                            (const int32_t *)nullptr, (int32_t *)nullptr, (int)N, 0, order_bits, s));
    else
        CKB(cub::DeviceRadixSort::SortPairs(nullptr, t_order, (const uint64_t *)nullptr, (uint64_t *)nullptr,
                                            (const int32_t *)nullptr, (int32_t *)nullptr, (int)N, 0, order_bits, s));
    CKB(cub::DeviceRadixSort::SortPairs(nullptr, t_doc, (const int32_t *)nullptr, (int32_t *)nullptr,
                                        (const int32_t *)nullptr, (int32_t *)nullptr, (int)N, 0, doc_bits, s));
    CKB(cub::DeviceScan::InclusiveScan(nullptr, t_scan, (const int32_t *)nullptr, (int32_t *)nullptr, MaxOp(), (int)N,
                                       s));
    CKB(cub::DeviceScan::ExclusiveSum(nullptr, t_sum, (const int32_t *)nullptr, (int32_t *)nullptr, (int)N + 1, s));
    // what each set-up phase takes from the arena (SetupArena rounds like rnd)
    const size_t need_check = rnd(sizeof(int32_t) * (size_t)D);
    const size_t key_bytes = key32 ? sizeof(uint32_t) : sizeof(uint64_t);
    const size_t need_order = reorder ? 2 * rnd(key_bytes * (size_t)N) + rnd(sizeof(int32_t) * (size_t)N) +
                                            rnd(t_order)
                                      : 0;
    const size_t need_rev = 2 * rnd(sizeof(int32_t) * (size_t)N) + rnd(t_doc);
    const size_t need_seg = 2 * rnd(sizeof(int32_t) * ((size_t)N + 1)) + rnd(std::max(t_scan, t_sum));
    size_t o_late = 0, o_after_doc_tok = 0, o_after_seg = 0;
    {
        size_t size = 0;
        auto add = [&size, &rnd](size_t bytes) {
            const size_t off = size;
            size += rnd(bytes);
            return off;
        };
        const size_t o_word_ptr = add(sizeof(int64_t) * ((size_t)V + 1));
        const size_t o_doc_ptr = add(sizeof(int64_t) * ((size_t)D + 1));
        const size_t o_doc_ids = add(sizeof(int32_t) * (size_t)N);
        const size_t o_error = add(64 * sizeof(int32_t));
        const size_t o_tok_index = reorder ? add(sizeof(int32_t) * (size_t)N) : 0;
        const size_t o_rows = add(sizeof(int2) * (size_t)D);
        const size_t o_doc_order = add(sizeof(int32_t) * (size_t)D);
        const size_t o_items = add(sizeof(culda_item) * items.size());
        const size_t o_hot_items = add(sizeof(culda_item) * hot.size());
        const size_t o_hot_phi = add(sizeof(int32_t) * (size_t)ctx->num_hot * K);
        const size_t o_item_ll = add(sizeof(double) * items.size());
        const size_t o_counter = add(64 * sizeof(int32_t));
        const size_t o_iter = add(sizeof(uint32_t));
        const size_t o_stats = add(sizeof(DevStats));
        const size_t o_nk = add(sizeof(int32_t) * (size_t)K);
        // the region set-up borrows, in the order it gives the buffers back
        const size_t o_doc_tok = add(sizeof(int32_t) * (size_t)N);
        const size_t o_seg_start = add(sizeof(int32_t) * (size_t)N);  // at most one segment per token
        const size_t o_z0 = add(sizeof(uint16_t) * (size_t)N);
        const size_t o_z1 = add(sizeof(uint16_t) * (size_t)N);
        const size_t o_zx = add(sizeof(uint16_t) * (size_t)N);
        const size_t o_u = add(sizeof(float) * (size_t)N);
        const size_t o_theta = add(sizeof(ThetaEntry) * (size_t)ctx->theta_cap);
        o_late = o_doc_tok;
        o_after_doc_tok = o_seg_start;
        o_after_seg = o_z0;
        if (cudaMemPool_t pool = block_pool(ctx->device)) {
            CKB(cudaMallocFromPoolAsync((void **)&ctx->d_block, size, pool, s));
            ctx->block_pooled = true;
        } else {
            CKB(cudaMalloc((void **)&ctx->d_block, size));
        }
        char *b = ctx->d_block;
        ctx->d_word_ptr = reinterpret_cast<int64_t *>(b + o_word_ptr);
        ctx->d_doc_ptr = reinterpret_cast<int64_t *>(b + o_doc_ptr);
        ctx->d_doc_ids = reinterpret_cast<int32_t *>(b + o_doc_ids);
        ctx->d_error = reinterpret_cast<int32_t *>(b + o_error);
        ctx->d_tok_index = reorder ? reinterpret_cast<int32_t *>(b + o_tok_index) : nullptr;
        ctx->d_doc_tok = reinterpret_cast<int32_t *>(b + o_doc_tok);
        ctx->d_theta = reinterpret_cast<ThetaEntry *>(b + o_theta);
        ctx->d_rows = reinterpret_cast<int2 *>(b + o_rows);
        ctx->d_doc_order = reinterpret_cast<int32_t *>(b + o_doc_order);
        ctx->d_items = reinterpret_cast<culda_item *>(b + o_items);
        ctx->d_hot_items = reinterpret_cast<culda_item *>(b + o_hot_items);
        ctx->d_hot_phi = reinterpret_cast<int32_t *>(b + o_hot_phi);
        ctx->d_item_ll = reinterpret_cast<double *>(b + o_item_ll);
        ctx->d_seg_start = reinterpret_cast<int32_t *>(b + o_seg_start);
        ctx->d_counter = reinterpret_cast<int32_t *>(b + o_counter);
        ctx->d_iter = reinterpret_cast<uint32_t *>(b + o_iter);
        ctx->d_stats = reinterpret_cast<DevStats *>(b + o_stats);
        ctx->d_nk = reinterpret_cast<int32_t *>(b + o_nk);
        ctx->d_z[0] = reinterpret_cast<uint16_t *>(b + o_z0);
        ctx->d_z[1] = reinterpret_cast<uint16_t *>(b + o_z1);
        ctx->d_zx = reinterpret_cast<uint16_t *>(b + o_zx);
        ctx->d_u = reinterpret_cast<float *>(b + o_u);
        ctx->block_bytes = size;
    }
    // the borrowed region serves every phase when it is large enough (theta's
    // capacity is at least about half the token count); otherwise set-up
    // allocates an arena of its own
    const size_t size = ctx->block_bytes;
    const bool borrow = std::max(need_check, need_order) <= size - o_late && need_rev <= size - o_after_doc_tok &&
                        need_seg <= size - o_after_seg;
    if (!borrow) {
        arena.size = std::max(std::max(need_check, need_order), std::max(need_rev, need_seg));
        CKB((cudaError_t)device_malloc((void **)&arena.base, arena.size));
        arena.owned = true;
    }
    // the arena for a phase that may use the block from offset `from` on
    auto arena_at = [&](size_t from) {
        if (arena.owned)
            arena.reset();
        else
            arena.use(ctx->d_block + from, size - from);
    };

    mark("host layout, block");
    // corpus upload
    CKB(cudaMemcpyAsync(ctx->d_word_ptr, c->word_ptr, sizeof(int64_t) * ((size_t)V + 1), cudaMemcpyHostToDevice, s));
    CKB(cudaMemcpyAsync(ctx->d_doc_ptr, c->doc_ptr, sizeof(int64_t) * ((size_t)D + 1), cudaMemcpyHostToDevice, s));
    CKB(cudaMemcpyAsync(ctx->d_doc_ids, c->doc_ids, sizeof(int32_t) * (size_t)N, cudaMemcpyHostToDevice, s));
    CKB(cudaMemsetAsync(ctx->d_error, 0, 64 * sizeof(int32_t), s));
    // docs longest first for the theta rebuild's warps: a counting sort on
    // the length (below 65536), stable in doc id, on the host while the
    // corpus goes up
    std::vector<int32_t> doc_order((size_t)D);
    {
        std::vector<int32_t> start(65537, 0);
        for (int32_t d = 0; d < D; ++d) start[(size_t)(65535 - (c->doc_ptr[d + 1] - c->doc_ptr[d])) + 1]++;
        for (size_t i = 1; i < start.size(); ++i) start[i] += start[i - 1];
        for (int32_t d = 0; d < D; ++d)
            doc_order[(size_t)start[(size_t)(65535 - (c->doc_ptr[d + 1] - c->doc_ptr[d]))]++] = d;
    }
    // the rest of the host layout goes up behind the corpus
    CKB(cudaMemcpyAsync(ctx->d_rows, rows.data(), sizeof(int2) * (size_t)D, cudaMemcpyHostToDevice, s));
    CKB(cudaMemcpyAsync(ctx->d_doc_order, doc_order.data(), sizeof(int32_t) * (size_t)D, cudaMemcpyHostToDevice, s));
    CKB(cudaMemcpyAsync(ctx->d_items, items.data(), sizeof(culda_item) * items.size(), cudaMemcpyHostToDevice, s));
    if (!hot.empty())
        CKB(cudaMemcpyAsync(ctx->d_hot_items, hot.data(), sizeof(culda_item) * hot.size(), cudaMemcpyHostToDevice, s));

    auto arena_free = [&]() {
        if (arena.owned && arena.base) cudaFree(arena.base);
        arena.base = nullptr;
        arena.owned = false;
    };
#define CKA(call)                                                                                              \
    do {                                                                                                       \
        const cudaError_t ea_ = (call);                                                                        \
        if (ea_ != cudaSuccess) {                                                                              \
            arena_free();                                                                                      \
            CKB(ea_);                                                                                          \
        }                                                                                                      \
    } while (0)

    // doc ids in range and doc lengths consistent with the payload
    {
        arena_at(o_late);
        int32_t *d_cnt = arena.take<int32_t>((size_t)D);
        if (!d_cnt) CKA(cudaErrorMemoryAllocation);
        CKA(cudaMemsetAsync(d_cnt, 0, sizeof(int32_t) * (size_t)D, s));
        CKA(launch_doc_check(N, D, ctx->d_doc_ids, d_cnt, ctx->d_error, s));
        std::vector<int32_t> cnt((size_t)D);
        int32_t e = 0;
        CKA(cudaMemcpyAsync(cnt.data(), d_cnt, sizeof(int32_t) * (size_t)D, cudaMemcpyDeviceToHost, s));
        CKA(cudaMemcpyAsync(&e, ctx->d_error, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
        CKA(cudaStreamSynchronize(s));
        if (e) {
            arena_free();
            fail(ctx, CULDA_ERR_FORMAT, "culda_create: a doc id is outside [0, %d)", D);
            return bail(CULDA_ERR_FORMAT);
        }
        for (int32_t d = 0; d < D; ++d)
            if (cnt[d] != c->doc_ptr[d + 1] - c->doc_ptr[d]) {
                arena_free();
                fail(ctx, CULDA_ERR_FORMAT, "culda_create: doc %d has %d tokens in the payload but length %lld", d,
                     cnt[d], (long long)(c->doc_ptr[d + 1] - c->doc_ptr[d]));
                return bail(CULDA_ERR_FORMAT);
            }
    }
    mark("upload, doc check");

    // Stored token order: inside each word, tokens sorted by their doc's
    // length, longest first (a stable sort on (word, length class of L_d), or
    // on (word, 65535 - L_d) past 2^24 words, keeps doc order among equal
    // keys).  Neighbouring segments then walk theta rows
    // of similar length.  Sampling results do not depend on this order:
    // each token's Philox stream is keyed on its input index.
    if (reorder) {
        arena_at(o_late);
        char *keys = arena.take<char>(key_bytes * (size_t)N), *keys_out = arena.take<char>(key_bytes * (size_t)N);
        int32_t *vals = arena.take<int32_t>((size_t)N);
        const int end_bit = order_bits;
        size_t tmp_bytes = 0;
        if (key32)
            CKA(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, (uint32_t *)keys, (uint32_t *)keys_out, vals,
                                                ctx->d_tok_index, (int)N, 0, end_bit, s));
        else
            CKA(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, (uint64_t *)keys, (uint64_t *)keys_out, vals,
                                                ctx->d_tok_index, (int)N, 0, end_bit, s));
        void *tmp = arena.take<char>(tmp_bytes);
        if (!keys || !keys_out || !vals || !tmp) CKA(cudaErrorMemoryAllocation);
        if (key32)
            CKA(launch_order_keys32(V, N, ctx->d_word_ptr, ctx->d_doc_ids, ctx->d_doc_ptr, (uint32_t *)keys, s));
        else
            CKA(launch_order_keys(V, N, ctx->d_word_ptr, ctx->d_doc_ids, ctx->d_doc_ptr, (uint64_t *)keys, s));
        CKA(launch_iota(N, vals, s));
        if (key32)
            CKA(cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, (uint32_t *)keys, (uint32_t *)keys_out, vals,
                                                ctx->d_tok_index, (int)N, 0, end_bit, s));
        else
            CKA(cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, (uint64_t *)keys, (uint64_t *)keys_out, vals,
                                                ctx->d_tok_index, (int)N, 0, end_bit, s));
        // the doc ids in the stored order, through the (now free) key buffer
        int32_t *ids2 = reinterpret_cast<int32_t *>(keys);
        CKA(launch_gather<int32_t>(N, ctx->d_tok_index, ctx->d_doc_ids, ids2, s));
        CKA(cudaMemcpyAsync(ctx->d_doc_ids, ids2, sizeof(int32_t) * (size_t)N, cudaMemcpyDeviceToDevice, s));
    }

    mark("token order sort");
    // doc-reverse index: stable radix sort of stored token positions by doc id
    // (the reference builds it on the host, doc_chunk.cpp:225-255)
    {
        arena_at(o_after_doc_tok);
        int32_t *keys_out = arena.take<int32_t>((size_t)N), *vals_in = arena.take<int32_t>((size_t)N);
        const int end_bit = doc_bits;
        size_t tmp_bytes = 0;
        CKA(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, ctx->d_doc_ids, keys_out, vals_in, ctx->d_doc_tok,
                                            (int)N, 0, end_bit, s));
        void *tmp = arena.take<char>(tmp_bytes);
        if (!keys_out || !vals_in || !tmp) CKA(cudaErrorMemoryAllocation);
        CKA(launch_iota(N, vals_in, s));
        CKA(cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, ctx->d_doc_ids, keys_out, vals_in, ctx->d_doc_tok, (int)N,
                                            0, end_bit, s));
    }
    mark("doc-reverse sort");
    arena_at(o_after_seg);
    rc = build_segments_device(ctx, arena);
    arena_free();
#undef CKA
    if (rc) return bail(rc);
    // theta's storage held set-up temporaries until now
    CKB(cudaMemsetAsync(ctx->d_theta, 0, sizeof(ThetaEntry) * (size_t)std::max<int64_t>(ctx->theta_cap, 1), s));

    ctx->h_stats = pinned_stats_get();
    if (!ctx->h_stats) {
        fail(ctx, CULDA_ERR_OOM, "culda_create: pinned host memory for the iteration statistics");
        return bail(CULDA_ERR_OOM);
    }
    memset(ctx->h_stats, 0, sizeof(DevStats));
    CKB(cudaMemsetAsync(ctx->d_stats, 0, sizeof(DevStats), s));
    const uint32_t one = 1;
    CKB(cudaMemcpyAsync(ctx->d_iter, &one, sizeof(uint32_t), cudaMemcpyHostToDevice, s));

    mark("segments");
    // topics: Philox init, then the initial counts (SingleChunkSingleGPU.h:24-41)
    CKB(launch_init_topics(N, K, p->seed, ctx->d_tok_index, ctx->d_z[0], s));
    ctx->cur = 0;
    rc = rebuild_counts(ctx);
    if (rc) return bail(rc);
    if (p->flags & CULDA_FLAG_AUTOTUNE) {
        // a cached result applies now; otherwise the variants are timed on the
        // state after the first iterations, whose theta rows are shorter than
        // the random initial ones and closer to the rest of the chain
        TuneResult r;
        if (tune_lookup(tune_key(ctx), r)) {
            rc = autotune_sampler(ctx);
            if (rc) return bail(rc);
        } else {
            ctx->tune_pending = true;
        }
    }
    mark("init topics, counts");
    rc = build_graphs(ctx);
    if (rc) return bail(rc);
    mark("graph capture");
    if (p->flags & CULDA_FLAG_VERBOSE)
        fprintf(stderr,
                "culda: D=%d V=%d N=%lld K=%d items=%d hot_words=%d hot_items=%d item_tokens=%d theta_cap=%lld "
                "sample_grid=%d theta_grid=%d G=%d sample_blocks=%d\n",
                D, V, (long long)N, K, ctx->num_items, ctx->num_hot, ctx->num_hot_items, ctx->item_tokens,
                (long long)ctx->theta_cap, ctx->sample_grid, ctx->theta_grid, ctx->group_lanes, ctx->sample_blocks);
    *out = ctx;
    return CULDA_OK;
#undef CKB
}

// -------------------------------------------------------------- iterate
extern "C" int culda_iterate(culda_ctx *ctx, int n, culda_iter_stats *stats) {
    if (!ctx || n < 0) return fail(ctx, CULDA_ERR_INVALID_ARG, "culda_iterate: invalid argument");
    CK(cudaSetDevice(ctx->device));
    for (int i = 0; i < n; ++i) {
        if (ctx->tune_pending && ctx->next_iteration >= kTuneIteration) {
            ctx->tune_pending = false;
            int rc = autotune_sampler(ctx);
            if (rc) return rc;
            rc = build_graphs(ctx);
            if (rc) return rc;
        }
        CK(cudaEventRecord(ctx->ev0, ctx->stream));
        if (ctx->graph[ctx->cur]) {
            CK(cudaGraphLaunch(ctx->graph[ctx->cur], ctx->stream));
        } else {
            int rc = record_iteration(ctx, ctx->stream, ctx->cur);
            if (rc) return rc;
        }
        CK(cudaEventRecord(ctx->ev1, ctx->stream));
        CK(cudaEventSynchronize(ctx->ev1));
        float ms = 0.f, ms_s = 0.f, ms_t = 0.f;
        CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
        CK(cudaEventElapsedTime(&ms_s, ctx->ev_s0, ctx->ev_s1));
        CK(cudaEventElapsedTime(&ms_t, ctx->ev_t0, ctx->ev_t1));
        ctx->cur = 1 - ctx->cur;
        const DevStats h = *ctx->h_stats;
        ctx->next_iteration = h.iteration + 1;
        if (stats) {
            culda_iter_stats &o = stats[i];
            o.iteration = (int32_t)h.iteration;
            o.status = h.error;
            o.seconds = ms * 1e-3;
            o.loglik = (h.ll_sum - ctx->doc_term) / (double)ctx->N;
            o.tokens_per_sec = ms > 0 ? (double)ctx->N / (ms * 1e-3) : 0.0;
            o.row_entries = h.row_entries;
            o.theta_nnz = h.nnz;
            o.token_nnz = h.token_nnz;
            o.sample_seconds = ms_s * 1e-3;
            o.rebuild_seconds = ms_t * 1e-3;
        }
        if (h.error) return fail(ctx, CULDA_ERR_DEVICE_STATE, "iteration %u: device error word 0x%x", h.iteration, h.error);
    }
    return CULDA_OK;
}

// Device topics in stored order -> host array in input (word-major) order.
int topics_to_host(culda_ctx *ctx, const uint16_t *d_src, uint16_t *host) {
    cudaStream_t s = ctx->stream;
    if (ctx->d_tok_index) {
        CK(launch_scatter<uint16_t>(ctx->N, ctx->d_tok_index, d_src, ctx->d_zx, s));
        d_src = ctx->d_zx;
    }
    CK(cudaMemcpyAsync(host, d_src, sizeof(uint16_t) * (size_t)ctx->N, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return CULDA_OK;
}

extern "C" int culda_set_topics(culda_ctx *ctx, const uint16_t *topics) {
    if (!ctx || !topics) return fail(ctx, CULDA_ERR_INVALID_ARG, "culda_set_topics: null argument");
    CK(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    CK(cudaMemcpyAsync(ctx->d_zx, topics, sizeof(uint16_t) * (size_t)ctx->N, cudaMemcpyHostToDevice, s));
    int32_t *flag = ctx->d_error + 32;  // a spare word of the error buffer
    CK(cudaMemsetAsync(flag, 0, sizeof(int32_t), s));
    CK(launch_check_topics(ctx->N, ctx->K, ctx->d_zx, flag, s));
    int32_t bad = 0;
    CK(cudaMemcpyAsync(&bad, flag, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (bad) return fail(ctx, CULDA_ERR_INVALID_ARG, "culda_set_topics: a topic is >= K=%d; state unchanged", ctx->K);
    if (ctx->d_tok_index)
        CK(launch_gather<uint16_t>(ctx->N, ctx->d_tok_index, ctx->d_zx, ctx->d_z[ctx->cur], s));
    else
        CK(cudaMemcpyAsync(ctx->d_z[ctx->cur], ctx->d_zx, sizeof(uint16_t) * (size_t)ctx->N, cudaMemcpyDeviceToDevice,
                           s));
    return rebuild_counts(ctx);
}

extern "C" int culda_get_topics(culda_ctx *ctx, uint16_t *topics) {
    if (!ctx) return fail(ctx, CULDA_ERR_INVALID_ARG, "culda_get_topics: null context");
    CK(cudaSetDevice(ctx->device));
    return topics ? topics_to_host(ctx, ctx->d_z[ctx->cur], topics) : CULDA_OK;
}

extern "C" int culda_get_phi(culda_ctx *ctx, int32_t *phi, int32_t *nk) {
    if (!ctx) return fail(ctx, CULDA_ERR_INVALID_ARG, "culda_get_phi: null context");
    CK(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    if (phi) {
        int32_t *d_phi = nullptr, *d_nk2 = nullptr;
        CK(dalloc(&d_phi, (size_t)ctx->V * ctx->K));
        CK(dalloc(&d_nk2, (size_t)ctx->K));
        CK(cudaMemsetAsync(d_nk2, 0, sizeof(int32_t) * (size_t)ctx->K, s));
        CK(launch_update_phi(ctx->K, ctx->V, ctx->d_word_ptr, ctx->d_z[ctx->cur], d_phi, d_nk2, ctx->d_error, s));
        CK(cudaMemcpyAsync(phi, d_phi, sizeof(int32_t) * (size_t)ctx->V * ctx->K, cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        cudaFree(d_phi);
        cudaFree(d_nk2);
    }
    if (nk) {
        CK(cudaMemcpyAsync(nk, ctx->d_nk, sizeof(int32_t) * (size_t)ctx->K, cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
    }
    return CULDA_OK;
}

extern "C" int culda_get_theta(culda_ctx *ctx, int16_t *theta_a, int16_t *theta_ja, int32_t *max_ia,
                               int32_t *cur_ia) {
    if (!ctx) return fail(ctx, CULDA_ERR_INVALID_ARG, "culda_get_theta: null context");
    CK(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    if (theta_a || theta_ja) {
        std::vector<ThetaEntry> t((size_t)ctx->theta_cap);
        CK(cudaMemcpyAsync(t.data(), ctx->d_theta, sizeof(ThetaEntry) * t.size(), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        for (size_t i = 0; i < t.size(); ++i) {
            // the reference stores counts as int16 (thetaA): same truncation
            if (theta_a) theta_a[i] = (int16_t)(uint16_t)(t[i] & 0xFFFFu);
            if (theta_ja) theta_ja[i] = (int16_t)(uint16_t)(t[i] >> 18);  // stored as 4 * topic
        }
    }
    if (max_ia) std::copy(ctx->h_max_ia.begin(), ctx->h_max_ia.end(), max_ia);
    if (cur_ia) {
        std::vector<int2> r((size_t)ctx->D);
        CK(cudaMemcpyAsync(r.data(), ctx->d_rows, sizeof(int2) * r.size(), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        for (int32_t d = 0; d < ctx->D; ++d) cur_ia[d] = r[d].y;
    }
    return CULDA_OK;
}

extern "C" int64_t culda_theta_capacity(const culda_ctx *ctx) { return ctx ? ctx->theta_cap : -1; }
extern "C" int64_t culda_num_tokens(const culda_ctx *ctx) { return ctx ? ctx->N : -1; }

extern "C" int culda_sample_snapshot(culda_ctx *ctx, uint32_t iteration, uint16_t *topics_out, double *loglik) {
    if (!ctx) return fail(ctx, CULDA_ERR_INVALID_ARG, "culda_sample_snapshot: null context");
    CK(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    const int cur = ctx->cur, nxt = 1 - cur;
    CK(cudaMemsetAsync(ctx->d_counter, 0, sizeof(int32_t), s));
    if (ctx->num_hot > 0 && !ctx->d_frozen_phi) {
        CK(cudaMemsetAsync(ctx->d_hot_phi, 0, sizeof(int32_t) * (size_t)ctx->num_hot * ctx->K, s));
        CK(launch_hot_rows(ctx->K, ctx->d_hot_items, ctx->num_hot_items, ctx->d_z[cur], ctx->d_hot_phi, ctx->d_error,
                           s));
    }
    CK(launch_uniforms(ctx->N, ctx->params.seed, nullptr, iteration, ctx->d_tok_index, ctx->d_u, s));
    CK(launch_sample(sample_params(ctx, cur, iteration, nullptr), ctx->group_lanes, ctx->sample_blocks,
                     ctx->sample_grid, s));
    CK(launch_finalize_ll(ctx->d_item_ll, ctx->num_items, ctx->d_stats, nullptr, s));
    DevStats h{};
    int32_t e = 0;
    CK(cudaMemcpyAsync(&h, ctx->d_stats, sizeof(DevStats), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(&e, ctx->d_error, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (loglik) *loglik = (h.ll_sum - ctx->doc_term) / (double)ctx->N;
    if (e) return fail(ctx, CULDA_ERR_DEVICE_STATE, "sampler reported device error 0x%x", e);
    return topics_out ? topics_to_host(ctx, ctx->d_z[nxt], topics_out) : CULDA_OK;
}

extern "C" int culda_loglik_joint(culda_ctx *ctx, double *ll) {
    if (!ctx || !ll) return fail(ctx, CULDA_ERR_INVALID_ARG, "culda_loglik_joint: null argument");
    CK(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    const int P = num_sms(ctx->device) * 4;
    double *d_part = nullptr;
    CK(dalloc(&d_part, (size_t)P));
    CK(launch_loglik_joint(ctx->K, ctx->V, ctx->D, ctx->params.alpha, ctx->params.beta, ctx->d_word_ptr,
                           ctx->d_z[ctx->cur], ctx->d_rows, ctx->d_theta, ctx->d_doc_ptr, d_part, P, ctx->d_error,
                           s));
    std::vector<double> part((size_t)P);
    std::vector<int32_t> nk((size_t)ctx->K);
    CK(cudaMemcpyAsync(part.data(), d_part, sizeof(double) * (size_t)P, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(nk.data(), ctx->d_nk, sizeof(int32_t) * (size_t)ctx->K, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    cudaFree(d_part);
    const double a = ctx->params.alpha, b = ctx->params.beta, vb = (double)ctx->V * b, ka = (double)ctx->K * a;
    double sum = 0, comp = 0;
    auto add = [&](double x) {
        const double t = sum + x;
        if (std::fabs(sum) >= std::fabs(x))
            comp += (sum - t) + x;
        else
            comp += (x - t) + sum;
        sum = t;
    };
    for (double x : part) add(x);
    add((double)ctx->K * std::lgamma(vb));
    for (int32_t k : nk) add(-std::lgamma((double)k + vb));
    add((double)ctx->D * std::lgamma(ka));
    *ll = sum + comp;
    return CULDA_OK;
}

extern "C" int culda_get_info(const culda_ctx *ctx, culda_info *info) {
    if (!ctx || !info) return CULDA_ERR_INVALID_ARG;
    info->num_items = ctx->num_items;
    info->num_hot = ctx->num_hot;
    info->num_hot_items = ctx->num_hot_items;
    info->item_tokens = ctx->item_tokens;
    info->group_lanes = ctx->group_lanes;
    info->sample_grid = ctx->sample_grid;
    info->sample_blocks = ctx->sample_blocks;
    info->tuned = ctx->tuned;
    info->tune_ms = ctx->tune_ms;
    info->theta_min_len = ctx->theta_min_len;
    info->theta_long_docs = ctx->theta_long;
    info->theta_tune_ms = ctx->theta_tune_ms;
    info->theta_grid = ctx->theta_grid;
    // hot_rows (when words are split), uniforms, sample, finalize_ll, theta_rebuild, copy_error
    info->kernels_per_iteration = (ctx->num_hot > 0 ? 1 : 0) + 5;
    info->theta_capacity = ctx->theta_cap;
    const int64_t N = ctx->N, D = ctx->D, V = ctx->V, K = ctx->K;
    (void)N;
    (void)D;
    (void)V;
    (void)K;
    info->device_bytes = (int64_t)ctx->block_bytes;
    info->doc_term = ctx->doc_term;
    return CULDA_OK;
}

extern "C" const char *culda_last_error(const culda_ctx *ctx) { return ctx ? ctx->err.c_str() : global_error(); }

extern "C" uint32_t culda_next_iteration(const culda_ctx *ctx) { return ctx ? ctx->next_iteration : 0u; }

extern "C" int culda_set_iteration(culda_ctx *ctx, uint32_t iteration) {
    if (!ctx || iteration == 0u) return fail(ctx, CULDA_ERR_INVALID_ARG, "culda_set_iteration: invalid argument");
    CK(cudaSetDevice(ctx->device));
    CK(cudaStreamSynchronize(ctx->stream));
    CK(cudaMemcpy(ctx->d_iter, &iteration, sizeof(uint32_t), cudaMemcpyHostToDevice));
    ctx->next_iteration = iteration;
    return CULDA_OK;
}

extern "C" void culda_destroy(culda_ctx *ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    free_learned_state(ctx);
    for (int c = 0; c < 2; ++c)
        if (ctx->graph[c]) cudaGraphExecDestroy(ctx->graph[c]);
    if (ctx->d_block) {
        if (ctx->block_pooled) {  // back to the pool, ordered after the stream's work
            cudaFreeAsync(ctx->d_block, ctx->stream);
            cudaStreamSynchronize(ctx->stream);
        } else {
            cudaFree(ctx->d_block);
        }
    }
    if (ctx->h_stats) pinned_stats_put(ctx->h_stats);
    for (cudaEvent_t ev : {ctx->ev0, ctx->ev1, ctx->ev_s0, ctx->ev_s1, ctx->ev_t0, ctx->ev_t1})
        if (ev) cudaEventDestroy(ev);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

extern "C" const char *culda_status_string(int status) {
    switch (status) {
        case CULDA_OK: return "ok";
        case CULDA_ERR_INVALID_ARG: return "invalid argument";
        case CULDA_ERR_IO: return "i/o error";
        case CULDA_ERR_FORMAT: return "format error";
        case CULDA_ERR_CUDA: return "CUDA error";
        case CULDA_ERR_OOM: return "out of memory";
        case CULDA_ERR_UNSUPPORTED: return "unsupported";
        case CULDA_ERR_DEVICE_STATE: return "inconsistent device state";
        case CULDA_ERR_NO_DEVICE: return "no CUDA device";
        default: return "unknown status";
    }
}

namespace culda {
int device_malloc(void **p, size_t bytes) {
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaErrorMemoryAllocation) return (int)e;
    cudaGetLastError();
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kPoolDevices) return (int)e;
    cudaMemPool_t pool = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_pool_mu);
        pool = g_pools[dev];
    }
    if (!pool || cudaMemPoolTrimTo(pool, 0) != cudaSuccess) return (int)e;
    return (int)cudaMalloc(p, bytes);
}
}  // namespace culda

extern "C" int culda_trim_memory(int32_t device) {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) return CULDA_ERR_NO_DEVICE;
    if (device < 0 || device >= ndev) return CULDA_ERR_INVALID_ARG;
    cudaMemPool_t pool = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_pool_mu);
        if (device < kPoolDevices) pool = g_pools[device];
    }
    if (!pool) return CULDA_OK;
    return cudaMemPoolTrimTo(pool, 0) == cudaSuccess ? CULDA_OK : CULDA_ERR_CUDA;
}

extern "C" const char *culda_version(void) { return "culda-b200 0.1 sm_100a"; }
