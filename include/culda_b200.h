/*
 * culda_b200.h — C ABI of the B200-native collapsed-Gibbs LDA sampler.
 *
 * This library is a drop-in for CuLDA_CGS's one-GPU path (`culda -g 1 -c 1`):
 * the per-iteration sample -> log-likelihood -> phi/n_k rebuild -> theta rebuild
 * loop.  Every entry point is `extern "C"`, takes plain pointers and sizes,
 * never throws, never calls exit(), and returns an int status (0 = ok,
 * negative = error; see CULDA_* below).  Host buffers belong to the caller;
 * device buffers created by culda_create belong to the context.
 *
 * Two layers are exported:
 *   1. Context API (culda_create / culda_iterate / culda_get_*): replaces the
 *      reference driver SingleChunkSingleGPU (src_culda/train/SingleChunkSingleGPU.h:5-157)
 *      together with the classes that own device memory there
 *      (DocChunk, ModelPhi/ModelPhiGPU, ModelTheta/ModelThetaChunk).
 *   2. Kernel-level API (culda_update_phi, culda_compute_phi_head,
 *      culda_update_theta, culda_sample, culda_loglik): device pointers owned by
 *      the caller, one entry point per reference kernel API, so a maintainer can
 *      swap them in call by call.  Each cites the reference function it replaces.
 *
 * Layout conventions (all little-endian, device arrays unless stated):
 *   word_ptr  int64[V+1]  token range of each word in word-major order
 *                         (reference: wordIndices, doc_chunk.cpp:118-134)
 *   doc_ids   int32[N]    doc id of every token, word-major, ascending within a
 *                         word (reference: wordTokens, the .word.data payload)
 *   topics    uint16[N]   topic of every token (reference: wordTopics, int16)
 *   doc_ptr   int64[D+1]  token count prefix per doc (reference: docRevIndices)
 *   doc_tok   int32[N]    word-major token index of every token, grouped by doc
 *                         and ascending within a doc (reference: docRevIdx)
 *   theta     uint32[cap] CSR entries, one word each: the count in the low
 *                         16 bits, 4 * topic in the high 16 bits; ascending
 *                         topic inside a row, zero padded (reference: thetaA
 *                         and thetaJA, two int16 arrays,
 *                         lda_theta_kernel.cu:55-58).  The topic is kept as a
 *                         byte offset so the sampler needs one 32-byte load per
 *                         eight entries and one shared-memory load per entry;
 *                         the array must be 32-byte aligned.
 *   theta_rows int32[2*D] {row start, row end} per doc; start is the reference's
 *                         thetaMaxIA[d], end its thetaCurIA[d] = start + roundup32(nnz)
 *   nk        int32[K]    tokens per topic (reference: phiTopic)
 *   phi       int32[V*K]  word-topic counts, row per word (reference: phiTopicWord)
 */
#ifndef CULDA_B200_H_
#define CULDA_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* The library is built with hidden visibility; exactly the entry points
 * declared here are exported. */
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

/* ------------------------------------------------------------------ status */
enum {
    CULDA_OK = 0,
    CULDA_ERR_INVALID_ARG = -1,  /* bad argument or size                       */
    CULDA_ERR_IO = -2,           /* file missing or unreadable                 */
    CULDA_ERR_FORMAT = -3,       /* file contents inconsistent                 */
    CULDA_ERR_CUDA = -4,         /* a CUDA runtime call failed                 */
    CULDA_ERR_OOM = -5,          /* host or device allocation failed           */
    CULDA_ERR_UNSUPPORTED = -6,  /* valid input outside what this build runs   */
    CULDA_ERR_DEVICE_STATE = -7, /* a kernel found an inconsistent state       */
    CULDA_ERR_NO_DEVICE = -8     /* no CUDA device visible                     */
};

/* Human-readable name of a status code (static storage). */
const char *culda_status_string(int status);

/* Library version string, e.g. "culda-b200 0.1 sm_100a". */
const char *culda_version(void);

/* ------------------------------------------------------------------ corpus */
/*
 * Host-side corpus in CuLDA_CGS's word-first format (src_format/format.cpp:64-157,
 * src_format/data_chunk.h:49-67): a doc index, a word index and the word-major
 * doc-id payload.  A corpus returned by culda_corpus_load/generate owns its
 * arrays and is released with culda_corpus_free; a caller may also fill the
 * struct with its own arrays (then it must not call culda_corpus_free on it).
 */
typedef struct culda_corpus {
    int32_t num_docs;   /* D */
    int32_t num_words;  /* V */
    int64_t num_tokens; /* N */
    int64_t *doc_ptr;   /* [D+1], doc_ptr[0] = 0 (the .doc.idx cumulative ends)  */
    int64_t *word_ptr;  /* [V+1], word_ptr[0] = 0 (the .word.idx cumulative ends) */
    int32_t *doc_ids;   /* [N] word-major doc ids (the .word.data payload)        */
    int32_t *word_label;/* [V] or NULL: token string of word v is "w<label>"      */
    int32_t owned;      /* 1 when the arrays belong to the library                */
} culda_corpus;

enum { CULDA_LEN_POISSON = 0, CULDA_LEN_LOGNORMAL = 1, CULDA_LEN_PARETO = 2 };

/* Seeded synthetic LDA corpus (no reference counterpart; stands in for the
 * reference's unnamed datasets).  Topic-word distributions phi_k ~ Dir(word_conc * V * p)
 * with p_r proportional to r^-zipf_s; doc mixtures theta_d ~ Dir(doc_conc) over
 * num_topics; doc lengths from len_law clipped to [len_min, len_max].  Word ids
 * are assigned by first appearance, as src_format/format.cpp:75-76 does. */
typedef struct culda_gen_params {
    int32_t num_words;
    int32_t num_topics;
    int32_t num_docs;
    int32_t len_law;    /* CULDA_LEN_* */
    double zipf_s;
    double word_conc;
    double doc_conc;
    double len_a;       /* poisson: lambda; lognormal: mu; pareto: shape */
    double len_b;       /* lognormal: sigma; pareto: x_m                 */
    int32_t len_min;
    int32_t len_max;
    uint64_t seed;
    int32_t threads;    /* host threads, 0 = all                         */
} culda_gen_params;

int culda_corpus_generate(const culda_gen_params *p, culda_corpus **out);

/* Read `<prefix>.doc.idx`, `.chunk`, `.word.idx`, `.word.data` exactly as
 * Document::loadDocument (src_culda/model/doc.cpp:62-156) and
 * DocChunk::loadChunk (src_culda/model/doc_chunk.cpp:106-223) do.  Only
 * num_chunks == 1 is supported (the one-GPU path); the .chunk file must hold
 * exactly num_chunks rows (doc.cpp:111-114). */
int culda_corpus_load(const char *prefix, int num_chunks, culda_corpus **out);

/* Write the five src_format files for `c` (byte-identical to what
 * src_format/format.cpp writes for the equivalent text corpus). */
int culda_corpus_write(const culda_corpus *c, const char *prefix, int num_chunks);

/* Write the corpus as text, one doc per line "d<id> w<label> w<label> ...",
 * the input format of src_format/format.cpp. */
int culda_corpus_write_text(const culda_corpus *c, const char *path);

void culda_corpus_free(culda_corpus *c);

/* Token strings of a corpus read from text: word w's bytes are
 * bytes[offsets[w] .. offsets[w+1]) (no terminator; any byte but whitespace). */
typedef struct culda_vocab {
    int32_t num_words;
    int64_t *offsets;  /* [V+1] */
    char *bytes;
} culda_vocab;

void culda_vocab_free(culda_vocab *v);

/* Parse a text corpus (one document per line: a title field, then the
 * document's whitespace-separated tokens; lines with no field are skipped) on
 * `threads` host threads (0 = all), with word ids by first appearance.  This is
 * the parsing half of the reference's preprocessing tool, src_format/format.cpp:56-90
 * with src_culda/model/vocab.cpp:24-31.  `vocab` may be NULL.  Empty
 * corpora and title-only documents are accepted, as the reference's tool accepts
 * them. */
int culda_corpus_from_text(const char *path, int32_t threads, culda_corpus **corpus, culda_vocab **vocab);

/* Write the five src_format files for `c`, with the token strings of `vocab`
 * in `.vocab` (NULL: "w<label>"), byte-identical to src_format/format.cpp:92-165
 * and src_format/data_chunk.h:49-67, chunk-id suffixes when num_chunks > 1. */
int culda_format_write(const culda_corpus *c, const culda_vocab *vocab, const char *prefix, int num_chunks);

/* The reference's `format input output_prefix numChunks` tool
 * (src_format/format.cpp:19-165) as one call: culda_corpus_from_text followed
 * by culda_format_write.  An input that cannot be opened returns CULDA_ERR_IO
 * with "<input> open failed" in culda_last_error(NULL). */
int culda_format_text(const char *in_path, const char *out_prefix, int num_chunks, int32_t threads);

/* doc_tok[N] (reference docRevIdx, doc_chunk.cpp:225-255) on the host. */
int culda_corpus_doc_tokens(const culda_corpus *c, int32_t *doc_tok);

/* ------------------------------------------------------------------ context */
typedef struct culda_params {
    int32_t k;            /* topics: multiple of 32, 32..4096 (reference: -k, rounded up to 32 in main.cpp:132-135) */
    float alpha;          /* reference: -a */
    float beta;           /* reference: -b */
    uint64_t seed;        /* Philox key for init and sampling */
    int32_t device;       /* CUDA device ordinal */
    int32_t group_lanes;  /* sampler variant: 0 = auto, CULDA_SAMPLER_FLAT (-1) = the warp-flattened
                             walk, else 1,2,4,8,16,32 lanes per token */
    int32_t item_tokens;  /* max tokens per sampler work item, 0 = auto, at most 65535 */
    int32_t flags;        /* CULDA_FLAG_* */
    int32_t sample_blocks; /* sampler register budget, as resident CTAs per SM: 0 = auto (9
                              for the flat walk, 8 for the group samplers), 8 (<= 64
                              registers), 9 (<= 56 registers; the flat walk only) or 10
                              (<= 48 registers; group_lanes 4, 8, 16) */
    int32_t theta_min_len; /* theta rebuild bins: docs of at least this many tokens are rebuilt
                              by a whole CTA each, the others by one warp each.  0 = auto (N
                              over the rebuild's warps, at least 1024; CULDA_FLAG_AUTOTUNE
                              times candidates), -1 = one warp for every doc, > 0 = this
                              threshold.  No reference counterpart (the reference's rebuild
                              takes a warp per doc, lda_theta_kernel.cu:5-87). */
} culda_params;

/* group_lanes value of the warp-flattened sampler: a warp splits the rows of up
 * to 32 segments evenly over its lanes, builds every row's prefix sums in shared
 * memory, and each lane then draws its own tokens. */
enum { CULDA_SAMPLER_FLAT = -1 };

enum {
    CULDA_FLAG_NO_GRAPH = 1,      /* launch the iteration kernel by kernel instead of one CUDA graph */
    CULDA_FLAG_VERBOSE = 2,       /* print set-up details to stderr */
    CULDA_FLAG_NO_REORDER = 4,    /* keep tokens in input order inside each word (default: by doc length) */
    CULDA_FLAG_AUTOTUNE = 8       /* time the sampler variants (lanes per token x register budget) and
                                     the theta rebuild's bin thresholds on the state before iteration 3
                                     (after two iterations with the defaults) and keep the fastest;
                                     group_lanes, sample_blocks and theta_min_len must be 0.  Results
                                     are cached per (device name, N, D, V, K) in the process and, when
                                     the environment variable CULDA_TUNE_CACHE names a file, in that
                                     file; a cached result applies from the first iteration. */
};

typedef struct culda_iter_stats {
    int32_t iteration;      /* 1-based */
    int32_t status;         /* device error word after the iteration (0 = consistent) */
    double seconds;         /* device time of the iteration (CUDA events) */
    double loglik;          /* mean log((S+Q)/(L_d+K*alpha)) over tokens, pre-sampling snapshot
                               (the reference's printed value, lda_train_kernel.cu:258, without
                               its per-warp int truncation) */
    double tokens_per_sec;  /* N / seconds */
    int64_t row_entries;    /* sum over tokens of the padded theta row length of the rebuilt state */
    int64_t theta_nnz;      /* non-zeros in theta after the rebuild */
    int64_t token_nnz;      /* sum over tokens of the non-zeros in their doc's rebuilt row */
    double sample_seconds;  /* device time of the sampler kernel */
    double rebuild_seconds; /* device time of the theta / n_k rebuild */
    double accept_rate;     /* Metropolis-Hastings iterations: accepted moves / proposals (else 0) */
} culda_iter_stats;

typedef struct culda_ctx culda_ctx;

/* Upload the corpus, build the doc-reverse index, the theta layout and the
 * sampler work list, draw the initial topics (Philox, counter (t, 0, 0, 1))
 * and build the initial counts.  Replaces DocChunk::allocGPU/toGPU
 * (doc_chunk.cpp:277-356), Document::generateTopics (doc_chunk.cpp:259-264),
 * ModelPhi::InitData/UpdatePhiGPU/UpdatePhiHead and ModelTheta::InitData/
 * UpdateThetaGPU (SingleChunkSingleGPU.h:15-41). */
int culda_create(const culda_corpus *c, const culda_params *p, culda_ctx **out);

/* Run n iterations (sample, log-likelihood, rebuild counts), one CUDA graph
 * launch each, writing one culda_iter_stats per iteration into stats (may be
 * NULL).  Replaces the loop body SingleChunkSingleGPU.h:70-127. */
int culda_iterate(culda_ctx *ctx, int n, culda_iter_stats *stats);

/* Replace all topics from a host array and rebuild the counts. */
int culda_set_topics(culda_ctx *ctx, const uint16_t *topics);

/* Checkpoint and resume (no reference counterpart; the reference saves no
 * usable model state, model_phi.cpp:161-189): the state of a chain is its
 * topics (culda_get_topics) and the number of its next iteration, which keys
 * the Philox draws.  A context created with the same corpus, K, alpha, beta
 * and seed, given those topics (culda_set_topics) and that iteration number,
 * continues with exactly the draws the original chain would have made.
 * culda_next_iteration returns the number (1-based), culda_set_iteration sets
 * it (>= 1). */
uint32_t culda_next_iteration(const culda_ctx *ctx);
int culda_set_iteration(culda_ctx *ctx, uint32_t iteration);

/* Copy state back (reference: DocChunk::toCPU, ModelPhi::MasterGPUToCPU,
 * ModelTheta::toCPU, SingleChunkSingleGPU.h:138-148).  Any pointer may be NULL. */
int culda_get_topics(culda_ctx *ctx, uint16_t *topics);
int culda_get_phi(culda_ctx *ctx, int32_t *phi, int32_t *nk);
/* thetaA / thetaJA in the reference's two-int16 layout, plus MaxIA[D+1] and CurIA[D]. */
int culda_get_theta(culda_ctx *ctx, int16_t *theta_a, int16_t *theta_ja, int32_t *max_ia, int32_t *cur_ia);
int64_t culda_theta_capacity(const culda_ctx *ctx);
int64_t culda_num_tokens(const culda_ctx *ctx);

/* One sampling pass over the current snapshot with Philox counter `iteration`,
 * without rebuilding counts or advancing the iteration counter; writes the
 * sampled topics (host, may be NULL) and the snapshot log-likelihood.  Used to
 * compare a single draw with the host oracle on a frozen snapshot. */
int culda_sample_snapshot(culda_ctx *ctx, uint32_t iteration, uint16_t *topics_out, double *loglik);

/* FP64 joint log-likelihood log p(w, z) of the current state (Griffiths and
 * Steyvers 2004, lgamma form).  No reference counterpart. */
int culda_loglik_joint(culda_ctx *ctx, double *ll);

/* Layout and launch facts of a context (no reference counterpart). */
typedef struct culda_info {
    int32_t num_items;          /* sampler work items */
    int32_t num_hot;            /* words split over several items */
    int32_t num_hot_items;
    int32_t item_tokens;        /* largest item */
    int32_t group_lanes;        /* lanes per token in the sampler */
    int32_t sample_grid;        /* persistent sampler CTAs */
    int32_t sample_blocks;      /* the sampler's register budget (resident CTAs per SM) */
    int32_t theta_grid;         /* theta rebuild CTAs */
    int32_t kernels_per_iteration;
    int64_t theta_capacity;     /* theta entries */
    int64_t device_bytes;       /* device memory held by the context */
    double doc_term;            /* sum_d L_d log(L_d + K alpha) */
    int32_t tuned;              /* sampler variant: 0 = given or default (or tuning still pending),
                                   1 = timed, 2 = from the tuning cache */
    float tune_ms;              /* the chosen variant's sampler time when it was timed (tuned != 0) */
    int32_t theta_min_len;      /* theta rebuild bin threshold in tokens (0: every doc by one warp) */
    int32_t theta_long_docs;    /* docs rebuilt by a whole CTA each */
    float theta_tune_ms;        /* the chosen threshold's rebuild time when it was timed, else 0 */
} culda_info;

int culda_get_info(const culda_ctx *ctx, culda_info *info);

const char *culda_last_error(const culda_ctx *ctx);

/* Frees the context.  Its device block goes back to a per-device memory pool
 * that keeps it reserved for the process, so the next culda_create on that
 * device reuses the memory instead of mapping new pages (the reference frees
 * each buffer with cudaFree, e.g. src_culda/model/doc_chunk.cpp:281-289). */
void culda_destroy(culda_ctx *ctx);

/* Returns the pool's unused reserve on `device` to the driver (memory that
 * live contexts hold is untouched).  No reference counterpart. */
int culda_trim_memory(int32_t device);

/* ------------------------------------------------------------- kernel level */
/* A sampler work item: tokens [begin, begin+count) of one word.  Words with
 * more than item_tokens tokens are split into several items (hot words; the
 * reference's slots, doc_chunk.cpp:148-205); `hot` indexes their phi row in
 * the hot-row buffer, -1 for words held by a single item. */
typedef struct culda_item {
    int64_t begin;
    int32_t count;
    int32_t word;
    int32_t hot;
    int32_t first;      /* 1 on the first item of its word */
    int32_t seg_begin;  /* the item's segments are seg_start[seg_begin .. seg_begin+seg_count) */
    int32_t seg_count;
} culda_item;

/* Build the work list for `word_ptr` (host).  Items are ordered largest first.
 * Returns the number of items (<= max_items) or a negative status; with
 * items == NULL only counts.  *num_hot receives the number of hot words. */
int64_t culda_build_items(int32_t num_words, const int64_t *word_ptr, int32_t item_tokens,
                          culda_item *items, int64_t max_items, int32_t *num_hot);

/* Segments of a work list (host): maximal runs of consecutive tokens of one
 * doc inside an item, at most max_len tokens each.  Tokens of one word in one
 * doc share their sampling distribution on a frozen snapshot, so the sampler
 * walks the doc's theta row once per segment.  Fills seg_begin/seg_count of
 * every item and seg_start (the first token of each segment); returns the
 * number of segments or a negative status; with seg_start == NULL only counts. */
int64_t culda_build_segments(int64_t num_tokens, const int32_t *doc_ids, culda_item *items, int32_t num_items,
                             int32_t max_len, int32_t *seg_start, int64_t max_segs);

/* Replaces LDAUpdatePhiAPI (src_culda/kernel/lda_phi_kernel.cu:136-159) and the
 * n_k memset before it (src_culda/model/model_phi_gpu.cpp:79).  Per-word shared
 * memory histograms, no global atomics and no per-warp scratch array; nk is
 * the column sum of phi. */
int culda_update_phi(int32_t k, int32_t num_words, const int64_t *d_word_ptr, const uint16_t *d_topics,
                     int32_t *d_phi, int32_t *d_nk, void *stream);

/* Replaces LDAComputePhiHeadAPI (src_culda/kernel/lda_phi_kernel.cu:49-72):
 * phi_head[w*K+k] = (phi[w*K+k] + beta) / (nk[k] + V*beta) in FP32 (the
 * reference rounds it to FP16).  The sampler computes this on the fly; this
 * entry point exists for callers that want the table. */
int culda_compute_phi_head(int32_t k, float beta, int32_t num_words, const int32_t *d_phi, const int32_t *d_nk,
                           float *d_phi_head, void *stream);

/* Workspace bytes culda_update_theta needs for num_docs documents. */
size_t culda_update_theta_workspace(int32_t k, int32_t num_docs);

/* Replaces LDAUpdateThetaAPI (src_culda/kernel/lda_theta_kernel.cu:89-126) and
 * the two memsets before it (src_culda/model/model_theta_chunk.cpp:114-115).
 * Rebuilds every theta row from the topics of its doc's tokens, writes
 * theta_rows[2d+1] (the row end) and zeroes the part of the old row past the
 * new end; d_nk (optional) receives the topic totals.  d_doc_order lists the
 * docs longest first (length binning); NULL means 0..D-1.  d_stats (optional,
 * int64[3]) receives {sum_d L_d * rowlen_d, sum_d nnz_d, sum_d L_d * nnz_d}. */
int culda_update_theta(int32_t k, int32_t num_docs, const int64_t *d_doc_ptr, const int32_t *d_doc_tok,
                       const uint16_t *d_topics, const int32_t *d_doc_order, int32_t *d_theta_rows,
                       uint32_t *d_theta, int32_t *d_nk, int64_t *d_stats, void *d_workspace,
                       size_t workspace_bytes, void *stream);

typedef struct culda_sample_args {
    int32_t k;
    float alpha;
    float beta;
    int32_t num_docs;
    int32_t num_words;
    int64_t num_tokens;
    const int64_t *word_ptr;     /* [V+1] */
    const int32_t *doc_ids;      /* [N] */
    const uint16_t *topics_in;   /* [N] topics of the snapshot: phi rows are histogrammed from them */
    uint16_t *topics_out;        /* [N] sampled topics (must not alias topics_in) */
    const uint32_t *theta;       /* packed CSR of the snapshot (32-byte aligned) */
    const int32_t *theta_rows;   /* [2*D] */
    const int32_t *nk;           /* [K] of the snapshot */
    const culda_item *items;     /* device copy of the work list (with segments) */
    const int32_t *seg_start;    /* device copy of the segment starts (culda_build_segments) */
    int32_t num_segs;
    int32_t num_items;
    int32_t num_hot;             /* words split over several items */
    const culda_item *hot_items; /* device copy of the items with hot >= 0 (any order) */
    int32_t num_hot_items;
    int64_t theta_capacity;      /* entries in theta (rows are checked against it) */
    uint64_t seed;
    uint32_t iteration;          /* Philox counter word 2 */
    int32_t group_lanes;         /* CULDA_SAMPLER_FLAT or 1,2,4,8,16,32 */
    double *loglik_sum;          /* device double: receives sum over tokens of log(S+Q) */
    int32_t *error;              /* device int32 error word (optional) */
} culda_sample_args;

/* Workspace bytes culda_sample needs (hot phi rows, per-item partial sums). */
size_t culda_sample_workspace(int32_t k, int32_t num_items, int32_t num_hot);

/* Replaces the LDAKernelTrain launch (src_culda/kernel/lda_train_kernel.cu:20-271,
 * launched at src_culda/train/SingleChunkSingleGPU.h:75-100) and the per-token
 * log terms it writes.  For every token t of word w in doc d on the frozen
 * snapshot: S = sum_k theta_dk * phihat_wk over the doc's row, Q = alpha *
 * sum_k phihat_wk, u = Philox4x32-10(key=seed, ctr={t_lo, t_hi, iteration, 0}),
 * draw by inverse CDF over the row (ascending topic) then over 0..K-1. */
int culda_sample(const culda_sample_args *a, void *d_workspace, size_t workspace_bytes, void *stream);

/* Size of the fixed device scratch array behind culda_sample_noalloc (8 MiB,
 * held on every GPU that loads the library until the process exits). */
#define CULDA_NOALLOC_SCRATCH_BYTES (8u << 20)

/* culda_sample without a caller workspace; no counterpart in the reference.
 * For callers that cannot allocate device memory for the sampler: a serving
 * process whose own pool allocator reserved all device memory up front and
 * lets no library call cudaMalloc.  Same arguments, checks and results as
 * culda_sample; the scratch is a fixed device array of
 * CULDA_NOALLOC_SCRATCH_BYTES instead of a workspace, and the call allocates
 * nothing.  Invalid arguments (K, num_items <= 0, num_hot < 0) return
 * CULDA_ERR_INVALID_ARG; a valid work list needing more scratch than the
 * array holds (culda_sample_workspace) is rejected with CULDA_ERR_UNSUPPORTED.
 * Like culda_sample, each call reads the theta range check back to the host,
 * so it returns only after its stream has run the work queued before it.
 * The first call on each device looks up the array's device address (and
 * loads the library's device code there if that has not happened yet): make
 * that first call before any stream capture.  The address is kept for the
 * life of the process, so the library must not be used on a device after a
 * cudaDeviceReset of it.  Every call on a device shares the one array, so
 * calls that may overlap on the GPU (other streams, other host threads) race
 * and must be serialised by the caller. */
int culda_sample_noalloc(const culda_sample_args *a, void *stream);

/* Replaces LDATrainPerplexity (src_culda/kernel/lda_train_kernel.cu:323-356):
 * turns the device sum written by culda_sample into the per-token value the
 * reference prints: (sum - sum_d L_d*log(L_d + K*alpha)) / N, read back to
 * host (synchronises the stream). */
int culda_loglik(const double *d_loglik_sum, double doc_term, int64_t num_tokens, double *loglik, void *stream);

/* ------------------------------------------- tensor-core GEMM (no reference counterpart)
 * The BF16 GEMM the document encoder is built from: C = A * B^T with A
 * [m x k] and B [n x k] row-major BF16 (k contiguous), FP32 accumulation on the
 * tensor cores, and one of the encoder's fused epilogues:
 *   CULDA_GEMM_F32        out_f32[m x n] = alpha * C (+ bias[col] when bias != NULL)
 *   CULDA_GEMM_BIAS_GELU  out_f32 = C + bias (the pre-activation);
 *                         out_bf16[m x n] and out_bf16_t[n x m] = GELU(C + bias)
 *   CULDA_GEMM_GELU_BWD   g = C * GELU'(pre[m x n]); out_bf16 and out_bf16_t = g;
 *                         colsum[col] += sum over rows of g (when colsum != NULL)
 * GELU is x * Phi(x) (the error-function form).  m and n must be multiples of
 * 128, k of 64; lda, ldb multiples of 8 elements; row-major outputs use row
 * stride ldo, the transposed output ld_t.  A device error word (optional)
 * receives bit 16 if a bounded wait inside the kernel gave up. */
enum { CULDA_GEMM_F32 = 0, CULDA_GEMM_BIAS_GELU = 1, CULDA_GEMM_GELU_BWD = 2 };

typedef struct culda_gemm_args {
    int32_t m, n, k;
    const void *a;      /* bf16 [m x lda] */
    int32_t lda;
    const void *b;      /* bf16 [n x ldb] */
    int32_t ldb;
    int32_t epilogue;   /* CULDA_GEMM_* */
    float alpha;        /* CULDA_GEMM_F32 scale */
    float *out_f32;     /* [m x ldo] */
    void *out_bf16;     /* bf16 [m x ldo] */
    void *out_bf16_t;   /* bf16 [n x ld_t] */
    int32_t ldo;
    int32_t ld_t;
    const float *bias;  /* [n] */
    const float *pre;   /* [m x ldo] */
    float *colsum;      /* [n] */
    int32_t *error;     /* device int32 or NULL */
    int32_t k_splits;   /* CULDA_GEMM_F32 only: 0 or 1 = one CTA per output tile; s > 1 cuts k
                           into s slices whose partial products are added into out_f32 with
                           atomics (out_f32 must hold zeros, or what to add to; bias is added
                           once; the sum order, so the last bits, may vary run to run) */
} culda_gemm_args;

int culda_gemm_bf16(const culda_gemm_args *a, void *stream);

/* ------------------------------- document encoder (no reference counterpart)
 * A small network that maps a document's bag of words to a distribution over
 * the K topics, used as an independent Metropolis-Hastings proposal and to
 * warm-start topics of new documents:
 *   x0 = mean over the doc's tokens of E[word]         E: [V x 256]
 *   h1 = GELU(W1 x0 + b1), h2 = GELU(W2 h1 + b2)       W1: [512 x 256], W2: [512 x 512]
 *   q  = softmax(W3 h2 + b3)                           W3: [K x 512]
 * BF16 operands on the tensor cores (culda_gemm_bf16) with FP32 accumulation
 * and FP32 master weights; trained with Adam on the cross-entropy
 * -sum_k target_k log q_k, averaged over the batch.
 * Batches are CSR slices: doc b of a batch is docs[b] (or b when docs is
 * NULL) of the CSR (doc_ptr int64[], words int32[] word ids), all device
 * pointers. */
#define CULDA_ENC_EMBED 256
#define CULDA_ENC_HIDDEN 512

typedef struct culda_encoder culda_encoder;

typedef struct culda_encoder_params {
    int32_t num_words;   /* V */
    int32_t k;           /* topics: a multiple of 128, up to 4096 */
    int32_t max_batch;   /* docs per call, 1..65536 (rounded up to 128 inside) */
    int32_t device;
    uint64_t seed;       /* Philox key of the initial weights */
    float lr;            /* Adam step size (0 = 1e-3) */
    float beta1, beta2;  /* Adam decay rates (0 = 0.9, 0.999) */
    float eps;           /* Adam epsilon (0 = 1e-8) */
} culda_encoder_params;

/* Tensors of the encoder, for culda_encoder_get/set_tensor (FP32, row-major). */
enum {
    CULDA_ENC_E = 0, CULDA_ENC_W1 = 1, CULDA_ENC_B1 = 2, CULDA_ENC_W2 = 3, CULDA_ENC_B2 = 4, CULDA_ENC_W3 = 5,
    CULDA_ENC_B3 = 6,
    CULDA_ENC_GRAD = 16  /* + tensor: its gradient from the last backward pass */
};

int culda_encoder_create(const culda_encoder_params *p, culda_encoder **out);
int culda_encoder_destroy(culda_encoder *e);
int64_t culda_encoder_tensor_size(const culda_encoder *e, int32_t which);  /* elements, < 0 if unknown */
int culda_encoder_get_tensor(culda_encoder *e, int32_t which, float *host);
int culda_encoder_set_tensor(culda_encoder *e, int32_t which, const float *host);  /* weights only */

/* q for a batch: d_probs [batch x K] FP32 (device). */
int culda_encoder_forward(culda_encoder *e, int32_t batch, const int32_t *d_docs, const int64_t *d_doc_ptr,
                          const int32_t *d_words, float *d_probs, void *stream);

/* Forward and backward against d_target [batch x K] (device, rows summing to
 * 1): leaves the gradients in the encoder (CULDA_ENC_GRAD + tensor) and the
 * mean cross-entropy in *loss (host; synchronises the stream). */
int culda_encoder_backward(culda_encoder *e, int32_t batch, const int32_t *d_docs, const int64_t *d_doc_ptr,
                           const int32_t *d_words, const float *d_target, double *loss, void *stream);

/* culda_encoder_backward followed by one Adam step on every weight. */
int culda_encoder_train_step(culda_encoder *e, int32_t batch, const int32_t *d_docs, const int64_t *d_doc_ptr,
                             const int32_t *d_words, const float *d_target, double *loss, void *stream);

/* ----------------------------------- learned proposal (no reference counterpart)
 * Training data, the encoder proposal and Metropolis-Hastings iterations on a
 * context.  The target of every MH step is the plain sampler's conditional on
 * the frozen snapshot of the iteration, p(k) ~ (n_dk + alpha) phihat_wk, so
 * the chain's target is unchanged; plain CGS (culda_iterate) can be mixed in
 * at any point. */

/* Adds the current state's doc-topic counts to the context's training
 * accumulator (D x K FP32, allocated on the first call). */
int culda_accumulate_theta(culda_ctx *ctx);

/* Trains enc on (document, accumulated topic distribution) pairs with target
 * (acc_dk / n + alpha) / (L_d + K alpha), n the accumulated states: `epochs`
 * passes over the docs in a Philox-shuffled order (key `seed`), batches of the
 * encoder's max_batch.  *loss: mean cross-entropy of the last epoch.  The
 * encoder's num_words and k must match the context. */
int culda_train_encoder(culda_ctx *ctx, culda_encoder *enc, int32_t epochs, uint64_t seed, double *loss);

/* Sets enc's word embeddings from the context's current topics: row w is the
 * word's topic profile (n_wk + beta) / (n_w + K beta) projected to 256
 * dimensions by a fixed random matrix (Philox key `seed`, entries of unit
 * variance; a tensor-core GEMM) and scaled to root-mean-square 0.3, so a
 * document's bag mean starts out as a projection of its words' topic
 * profiles.  The other weights are left as they are. */
int culda_encoder_init_from_phi(culda_ctx *ctx, culda_encoder *enc, uint64_t seed);

/* Runs enc over every doc and keeps, per doc, the proposal
 * (1 - mix) q_d + mix / K as an inclusive prefix table (FP32 D x K).  enc NULL
 * drops the proposal.  mix in [0, 1). */
int culda_set_proposal(culda_ctx *ctx, culda_encoder *enc, float mix);

/* The prefix table of culda_set_proposal, D x K FP32 in doc order (host). */
int culda_get_proposal(culda_ctx *ctx, float *cdf);

/* n Metropolis-Hastings iterations: per token `steps` steps (1..64) from its
 * current topic, alternating the doc proposal (n_dk + alpha, acceptance
 * phihat_wk' / phihat_wk) and, when a proposal is set, the encoder proposal
 * (independent, acceptance p(k') q_d(k) / (p(k) q_d(k'))); without one every
 * step uses the doc proposal.  Uniforms: Philox (seed, token, iteration,
 * 16 + step).  The counts are then rebuilt as after a plain iteration.  stats:
 * loglik is NaN (evaluate with culda_sample_snapshot), sample_seconds is the
 * MH kernel, accept_rate is set. */
int culda_iterate_mh(culda_ctx *ctx, int32_t n, int32_t steps, culda_iter_stats *stats);

/* One MH pass of `steps` steps from the current snapshot with Philox
 * iteration `iteration`, leaving the state unchanged; topics to host in input
 * order (topics_out may be NULL). */
int culda_mh_snapshot(culda_ctx *ctx, uint32_t iteration, int32_t steps, uint16_t *topics_out);

/* ------------------------------------------------ fold-in (no reference counterpart)
 * New documents sampled against a trained model: the context's samplers (plain
 * and MH) use the given word-topic counts phi [V x K] and topic totals nk [K]
 * (host arrays over the same vocabulary, e.g. culda_get_phi of the trained
 * context) instead of its own corpus's counts; theta stays the new documents'.
 * The per-iteration log-likelihood is then the held-out per-token value under
 * the frozen model.  phi NULL returns to the context's own counts.  Rows must
 * sum to nk. */
int culda_set_frozen_phi(culda_ctx *ctx, const int32_t *phi, const int32_t *nk);

/* ------------------------------------ doc-chunk data parallelism (one rank per GPU)
 * Replaces the phi exchange of -g N -c N (src_culda/train/MultiChunkMultiGPUequal.h:88-172,
 * MasterGPUCollect/Reduce/Distribute in src_culda/model/model_phi.cpp:105-144).
 * A context created on one chunk of the documents (a doc range, word ids of
 * the whole vocabulary) writes its chunk's word-topic counts [V x K] and topic
 * totals [K] of the current topics into caller-owned device buffers
 * (culda_count_phi, synchronous); the caller sums those over the chunks in
 * place (an all-reduce) and passes the sums to culda_set_shared_phi, after
 * which the samplers read the word rows and totals from those buffers at
 * every iteration (no copy; the caller keeps them alive and refreshed between
 * iterations).  NULL buffers return the context to its own counts.  Theta and
 * the topics stay the chunk's own. */
int culda_count_phi(culda_ctx *ctx, int32_t *d_phi, int32_t *d_nk);
int culda_set_shared_phi(culda_ctx *ctx, int32_t *d_phi, int32_t *d_nk);

/* Warm start from the proposal set by culda_set_proposal: every token's topic
 * is drawn from q_d(k) * phihat_wk (Philox: seed, token, 0, 6), then the
 * counts are rebuilt. */
int culda_warm_start(culda_ctx *ctx);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif

#endif /* CULDA_B200_H_ */
