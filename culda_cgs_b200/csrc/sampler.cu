// sampler.cu — the sm_100a sampling kernel of the one-GPU CGS iteration
// (replaces LDAKernelTrain, src_culda/kernel/lda_train_kernel.cu:20-271).
//
// Persistent CTAs pull work items (one word, or a slice of a hot word).  Per
// item the word's phi row is built as a shared-memory histogram of the
// snapshot topics (no dense V x K phi in HBM), phihat = (n_wk + beta) /
// (n_k + V beta) is formed in FP32 at shared-memory offset 0, and the
// alpha*phihat prefix of the dense bucket is scanned (by the flat sampler
// once per block of 8 topics).  The item's tokens come
// in segments (runs of one doc, at most 32 tokens) that share one walk of the
// doc's theta row and differ only in their Philox uniforms.  Two samplers do
// the walks and draws:
//   sample_flat_kernel (the default): a warp splits the rows of a batch of
//     segments evenly over 8 groups of 4 lanes (one 256-bit load per lane
//     per step, two alternating prefetch buffers), builds every row's prefix
//     sums in shared memory, and each lane then draws its own tokens;
//   sample_kernel<G>: a group of G lanes walks one row with 32-byte loads
//     (8 entries per lane per step), keeps the running sum after every step
//     in shared memory, and draws the segment's tokens one after another.
//
// A theta entry is one 32-bit word: the count in the low 16 bits and 4 * topic
// (the byte offset of the topic's phihat) in the high 16 bits.  The product
// theta_dk * phihat_wk is one shared-memory load at that offset, an exact
// integer-to-float conversion on the integer pipes and one multiply.
#include <cuda_runtime.h>

#include <algorithm>

#include "device_util.cuh"
#include "kernels.cuh"
#include "philox.h"

namespace culda {

__device__ __forceinline__ uint32_t entry_count(uint32_t e) { return e & 0xFFFFu; }
__device__ __forceinline__ int entry_topic(uint32_t e) { return (int)(e >> 18); }

// The count as a float, exactly: 2^23 + c has c in its low mantissa bits.
__device__ __forceinline__ float entry_count_f(uint32_t e) {
    return __fsub_rn(__uint_as_float(0x4B000000u | (e & 0xFFFFu)), 8388608.0f);
}

// theta_dk * phihat_wk for one entry.  The explicit-rounding intrinsics keep
// the compiler from fusing products and sums into different FMAs in the two
// passes: both passes must produce bitwise the same sums.
__device__ __forceinline__ float entry_prob(uint32_t e, const float *ph) {
    return __fmul_rn(entry_count_f(e),
                     *reinterpret_cast<const float *>(reinterpret_cast<const char *>(ph) + (e >> 16)));
}

__device__ __forceinline__ float fsum(float a, float b) { return __fadd_rn(a, b); }

// ------------------------------------------------------------ dense bucket
// Each thread holds the local inclusive sums of its run out[b, e) and their
// total `tot`; adds to the run the totals of all earlier threads (Kogge-Stone
// shuffles inside a warp, then across the warps).  Ends without a barrier.
__device__ __forceinline__ void add_run_offsets(float tot, float *out, int b, int e, float *s_warp) {
    const int T = blockDim.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = T >> 5;
    float incl = tot;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const float t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    float ex = __shfl_up_sync(0xffffffffu, incl, 1);
    if (lane == 0) ex = 0.f;
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        float w = lane < nwarps ? s_warp[lane] : 0.f;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const float t = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += t;
        }
        float wex = __shfl_up_sync(0xffffffffu, w, 1);
        if (lane == 0) wex = 0.f;
        if (lane < nwarps) s_warp[lane] = wex;
    }
    __syncthreads();
    const float base = s_warp[warp] + ex;
    for (int j = b; j < e; ++j) out[j] = base + out[j];
}

// Inclusive prefix qc[j] = alpha * sum_{i<=j} ph[i].  Each thread owns a run of
// ceil(K/T) entries summed with Neumaier compensation; the run totals are
// scanned with Kogge-Stone shuffles, so every prefix carries an error of
// about ten FP32 roundings.
__device__ void dense_bucket_prefix(const float *ph, float *qc, int K, float alpha, float *s_warp) {
    const int T = blockDim.x, tid = threadIdx.x;
    const int per = (K + T - 1) / T;
    const int b = min(tid * per, K), e = min(b + per, K);
    float s = 0.f, c = 0.f;
    for (int j = b; j < e; ++j) {
        neumaier(s, c, alpha * ph[j]);
        qc[j] = s + c;
    }
    add_run_offsets(s + c, qc, b, e, s_warp);
}

// First topic whose dense-bucket prefix exceeds tq (K-1 when none does).
template <int G>
__device__ __forceinline__ int dense_bucket_search(const float *qc, int K, float tq, int gl, unsigned m, int lane) {
    if constexpr (G == 1) {
        int lo = 0, hi = K - 1;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (qc[mid] > tq)
                hi = mid;
            else
                lo = mid + 1;
        }
        return lo;
    } else {
        int lo = 0, size = K;
        while (size > 1) {
            const int step = (size + G - 1) / G;
            const int off = gl * step;
            const int nseg = (size + step - 1) / step;
            bool hit = false;
            if (off < size) hit = qc[lo + min(off + step, size) - 1] > tq;
            const unsigned b = group_ballot<G>(hit, m, lane);
            const int j = b ? (__ffs(b) - 1) : (nseg - 1);
            lo += j * step;
            size = min(step, size - j * step);
        }
        return lo;
    }
}

// ------------------------------------------------------------- row walk
// Theta entries per lane per step: two 16-byte loads.  A group of 4 lanes
// then reads one 128-byte line of a row per step (rows start on 32 entries).
constexpr int kLaneEntries = 8;

template <int G>
struct SampleShape {
    static constexpr int kGroups = kSampleThreads / G;
    static constexpr int kStep = kLaneEntries * G;          // entries per group step
    // running sums kept per group, enough steps for rows of up to 64 G^2
    // entries (1024 at G = 4) to be walked once; longer rows walk again
    static constexpr int kMaxSteps = 64 * G / kLaneEntries;
    static constexpr int kPrefixFloats = kGroups * kMaxSteps;  // 2048 floats for every G
};

struct Step {
    uint32_t e[kLaneEntries];
};

// The 8 entries (32 bytes) at theta + idx in one 256-bit read-only load
// (sm_100's ld.global.v8; theta is 32-byte aligned and idx a multiple of 8):
// a group's step of 4 lanes is then one request per 128-byte line.
__device__ __forceinline__ void load8(const ThetaEntry *__restrict__ theta, int idx, uint32_t e[8]) {
    asm("ld.global.nc.v8.u32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=r"(e[0]), "=r"(e[1]), "=r"(e[2]), "=r"(e[3]), "=r"(e[4]), "=r"(e[5]), "=r"(e[6]), "=r"(e[7])
        : "l"(theta + idx));
}

__device__ __forceinline__ Step load_step(const ThetaEntry *__restrict__ theta, int idx, int re) {
    Step st;
    if (idx < re) {  // rows end on a multiple of 32 entries, idx on a multiple of kLaneEntries
        load8(theta, idx, st.e);
    } else {
#pragma unroll
        for (int j = 0; j < kLaneEntries; ++j) st.e[j] = 0u;
    }
    return st;
}

__device__ __forceinline__ void step_probs(const Step &st, const float *ph, float p[kLaneEntries]) {
#pragma unroll
    for (int j = 0; j < kLaneEntries; ++j) p[j] = entry_prob(st.e[j], ph);
}

// Pairwise sum of the lane's entries.
__device__ __forceinline__ float lane_sum(const float p[kLaneEntries]) {
    float q[kLaneEntries];
#pragma unroll
    for (int i = 0; i < kLaneEntries; ++i) q[i] = p[i];
#pragma unroll
    for (int w = kLaneEntries / 2; w > 0; w >>= 1)
#pragma unroll
        for (int i = 0; i < w; ++i) q[i] = fsum(q[2 * i], q[2 * i + 1]);
    return q[0];
}

// The group's last non-zero entry of a step (-1 when the step is all padding).
template <int G>
__device__ __forceinline__ int step_last_nonzero(const Step &st, unsigned m, int lane) {
    int last = -1;
#pragma unroll
    for (int j = 0; j < kLaneEntries; ++j)
        if (entry_count(st.e[j])) last = entry_topic(st.e[j]);
    const unsigned nb = group_ballot<G>(last >= 0, m, lane);
    return nb ? group_bcast<G>(last, 31 - __clz(nb), m) : -1;
}

// Inside one step: the first entry whose running sum passes T, starting from
// the running sum `base` before the step; the step's last non-zero entry when
// rounding leaves the step short of T.
template <int G>
__device__ __forceinline__ int resolve_step(const Step &st, float base, float T, const float *ph, int gl, unsigned m,
                                            int lane) {
    float p[kLaneEntries];
    step_probs(st, ph, p);
    float cum = base + group_excl<G>(lane_sum(p), gl, m);
    int hit = -1;
#pragma unroll
    for (int i = 0; i < kLaneEntries; ++i) {
        cum += p[i];
        if (hit < 0 && entry_count(st.e[i]) && cum > T) hit = entry_topic(st.e[i]);
    }
    const unsigned hb = group_ballot<G>(hit >= 0, m, lane);
    if (hb) return group_bcast<G>(hit, __ffs(hb) - 1, m);
    return step_last_nonzero<G>(st, m, lane);
}

// Pass 1 over the doc's theta row [rs, re): S as a compensated sum of the
// group's step totals; lane 0 records the running sum after every step.  All
// G lanes of a group see identical sums (butterfly reductions of the same
// values), so they take the same branches and group-masked shuffles are safe.
template <int G>
__device__ __forceinline__ float row_sum(const ThetaEntry *__restrict__ theta, const float *ph, float *pref, int rs,
                                         int re, int gl, unsigned m, int &nst_out) {
    constexpr int kMax = SampleShape<G>::kMaxSteps, kStep = SampleShape<G>::kStep;
    __syncwarp(m);  // the group's previous row is no longer being read from pref
    float s = 0.f, c = 0.f;
    int nst = 0;
    // the next step's entries are loaded before this step is reduced, so two
    // row loads per lane are in flight
    Step st = load_step(theta, rs + kLaneEntries * gl, re);
#pragma unroll 2
    for (int base = rs; base < re; base += kStep, ++nst) {
        const Step nx = load_step(theta, base + kStep + kLaneEntries * gl, re);
        float p[kLaneEntries];
        step_probs(st, ph, p);
        neumaier(s, c, group_sum<G>(lane_sum(p), m));
        if (gl == 0 && nst < kMax) pref[nst] = s + c;
        st = nx;
    }
    __syncwarp(m);  // pref is complete before any lane searches it
    nst_out = nst;
    return s + c;
}

// The topic for target T = u * (S + Q): inverse CDF over the row (ascending
// topic) when T < S, else over alpha * phihat (topics 0..K-1).
template <int G>
__device__ __forceinline__ int draw_topic(const ThetaEntry *__restrict__ theta, const float *ph, const float *qc,
                                          const float *pref, int nst, float S, float T, int K, int rs, int re, int gl,
                                          unsigned m, int lane) {
    constexpr int kMax = SampleShape<G>::kMaxSteps, kStep = SampleShape<G>::kStep;
    if (!(T < S)) return dense_bucket_search<G>(qc, K, T - S, gl, m, lane);
    if (nst <= kMax) {
        // the first step whose running sum passes T (the last one, S, does)
        for (int r = 0; r < nst; r += G) {
            const int j = r + gl;
            const unsigned hb = group_ballot<G>(j < nst && pref[j] > T, m, lane);
            if (hb) {
                const int hs = r + __ffs(hb) - 1;
                const float before = hs > 0 ? pref[hs - 1] : 0.f;
                const Step st = load_step(theta, rs + hs * kStep + kLaneEntries * gl, re);
                return resolve_step<G>(st, before, T, ph, gl, m, lane);
            }
        }
    } else {
        // long row: walk it again with the same arithmetic up to the step
        // that passes T
        float s2 = 0.f, c2 = 0.f;
        for (int base = rs; base < re; base += kStep) {
            const Step st = load_step(theta, base + kLaneEntries * gl, re);
            float p[kLaneEntries];
            step_probs(st, ph, p);
            const float before = s2 + c2;
            neumaier(s2, c2, group_sum<G>(lane_sum(p), m));
            if (s2 + c2 > T) return resolve_step<G>(st, before, T, ph, gl, m, lane);
        }
    }
    // Only reachable when T lies within the rounding of S itself: the token
    // sits on the boundary between the buckets.  Take the row's last
    // non-zero entry (it lies in the final 32-entry block).
    int last = -1;
    for (int i = max(rs, re - 32); i < re; ++i) {
        const ThetaEntry e = __ldg(theta + i);
        if (entry_count(e)) last = entry_topic(e);
    }
    return last;
}

// -------------------------------------------------------------- the kernel
// MINB resident CTAs per SM is the register budget the compiler is held to:
// 8 -> at most 64 registers (32 warps per SM, no spills), 10 -> at most 48
// (40 warps, some spills).
template <int G, int MINB>
__global__ void __launch_bounds__(kSampleThreads, MINB) sample_kernel(const SampleParams p) {
    extern __shared__ float smem[];
    using Shape = SampleShape<G>;
    const int K = p.k, KP = p.kmask + 1;
    float *ph = smem;               // [KP] phihat of the current word (zero past K), at offset 0
    float *inv = smem + KP;         // [K]  1 / (n_k + V beta)
    float *qc = inv + K;            // [K]  dense-bucket prefix (the word histogram before that)
    float *pref_all = qc + K;       // [kPrefixFloats] running sums per group
    int *hist = reinterpret_cast<int *>(qc);
    __shared__ int s_item;
    __shared__ float s_warp[kSampleThreads / 32];
    __shared__ double s_red[kSampleThreads / 32];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int gl = lane & (G - 1);
    const int group = tid / G;
    constexpr int NG = Shape::kGroups;
    float *pref = pref_all + group * Shape::kMaxSteps;
    const unsigned m = group_mask<G>(lane);
    const uint32_t iter = p.iteration_ptr ? *p.iteration_ptr : p.iteration;

    for (int j = tid; j < K; j += blockDim.x) inv[j] = 1.0f / ((float)p.nk[j] + p.vbeta);
    for (int j = K + tid; j < KP; j += blockDim.x) ph[j] = 0.f;

    for (;;) {
        if (tid == 0) s_item = atomicAdd(p.item_counter, 1);
        __syncthreads();
        const int it = s_item;
        if (it >= p.num_items) break;
        const culda_item item = p.items[it];
        const int64_t ibeg = item.begin, iend = item.begin + item.count;
        if (ibeg < 0 || item.count < 0 || iend > p.num_tokens || item.hot >= p.num_hot || item.seg_begin < 0 ||
            item.seg_count < 0 || (int64_t)item.seg_begin + item.seg_count > p.num_segs) {
            if (tid == 0) {
                atomicOr(p.error, kErrRowRange);
                p.item_ll[it] = 0.0;
            }
            __syncthreads();  // s_item is rewritten only after every thread has read it
            continue;
        }

        // phi row of the word
        const int *src;
        if (p.frozen_phi) {
            src = p.frozen_phi + (size_t)item.word * K;
        } else if (item.hot < 0) {
            for (int j = tid; j < K; j += blockDim.x) hist[j] = 0;
            __syncthreads();
            for (int64_t t = ibeg + tid; t < iend; t += blockDim.x) {
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
        dense_bucket_prefix(ph, qc, K, p.alpha, s_warp);
        __syncthreads();
        const float Q = qc[K - 1];

        double ll = 0.0;
        const int sg_end = item.seg_begin + item.seg_count;
        for (int sgb = item.seg_begin + group; sgb < sg_end; sgb += NG * G) {
            // lane gl prefetches segment gl of this batch: its token range,
            // doc and theta row
            const int sgm = sgb + gl * NG;
            int dm = -1, rsm = 0, rem = 0;
            int64_t t0m = 0, t1m = 0;
            if (sgm < sg_end) {
                t0m = __ldg(p.seg_start + sgm);
                t1m = sgm + 1 < sg_end ? (int64_t)__ldg(p.seg_start + sgm + 1) : iend;
                if (t0m < ibeg || t1m > iend || t0m >= t1m) {
                    atomicOr(p.error, kErrRowRange);
                    t0m = t1m = 0;
                } else {
                    const int d = __ldg(p.doc_ids + t0m);
                    if ((unsigned)d < (unsigned)p.num_docs) {
                        const int2 r = __ldg(p.rows + d);
                        if (r.x >= 0 && r.x <= r.y && (int64_t)r.y <= p.theta_cap && ((r.x | r.y) & 31) == 0) {
                            dm = d;
                            rsm = r.x;
                            rem = r.y;
                        } else {
                            atomicOr(p.error, kErrRowRange);
                        }
                    } else {
                        atomicOr(p.error, kErrDocRange);
                    }
                }
            }
#pragma unroll 1
            for (int j = 0; j < G; ++j) {
                if (sgb + j * NG >= sg_end) break;
                const int d = group_bcast<G>(dm, j, m);
                const int rs = group_bcast<G>(rsm, j, m), re = group_bcast<G>(rem, j, m);
                const int64_t t0 = group_bcast<G>(t0m, j, m), t1 = group_bcast<G>(t1m, j, m);
                if (d < 0) continue;
                // every token of the segment shares the doc's row and so S,
                // Q and the running sums; only its uniform differs
                int nst;
                const float S = row_sum<G>(p.theta, ph, pref, rs, re, gl, m, nst);
                const float total = S + Q;
                const double log_total = (double)logf(total);
                for (int64_t tb = t0; tb < t1; tb += G) {
                    // lane gl fetches the uniform of token tb + gl
                    float um = 0.f;
                    if (tb + gl < t1) {
                        if (p.uniforms) {
                            um = __ldg(p.uniforms + tb + gl);
                        } else {
                            const int64_t key = p.tok_index ? (int64_t)__ldg(p.tok_index + tb + gl) : tb + gl;
                            um = uniform_from_bits(philox_token(p.seed, (uint64_t)key, iter, kPurposeSample));
                        }
                    }
                    const int nb = (int)min((int64_t)G, t1 - tb);
#pragma unroll 1
                    for (int i = 0; i < nb; ++i) {
                        const float T = group_bcast<G>(um, i, m) * total;
                        int z = draw_topic<G>(p.theta, ph, qc, pref, nst, S, T, K, rs, re, gl, m, lane);
                        if (gl == 0) {
                            if (z < 0) {
                                atomicOr(p.error, kErrRowRange);
                                z = 0;
                            }
                            p.topics_out[tb + i] = (uint16_t)z;
                            ll += log_total;
                        }
                    }
                }
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) ll += __shfl_down_sync(0xffffffffu, ll, o);
        if (lane == 0) s_red[warp] = ll;
        __syncthreads();
        if (tid == 0) {
            double s = 0.0;
            for (int w = 0; w < kSampleThreads / 32; ++w) s += s_red[w];
            p.item_ll[it] = s;
        }
    }
}

// ------------------------------------------------------ the flat walk
// The warp-flattened sampler (group_lanes = kFlatLanes, -1).  A warp takes up to
// 32 consecutive segments of the item and splits the 8-entry units of their
// rows into 8 contiguous ranges of 4r units (r odd), one per group of 4
// lanes.  Rows start and end on multiples of 32 entries, i.e. of 4 units, so
// a group step (4 units, one 128-byte line) never straddles two rows.  Each
// group walks its range once with a compensated running sum that restarts at
// every row start and stores every unit's running prefix; a segmented scan
// over the groups' last values gives each group the sum carried into its
// range, which completes the prefixes of the units before its first row
// start.  With every unit's inclusive prefix inside its row in shared memory,
// each lane draws its own tokens: a binary search for the first unit whose
// prefix exceeds the target and a sequential pass over that unit's 8 entries.
// All groups stay busy whatever the mix of row lengths, and no lane waits on
// another token's draw.
constexpr int kUnit = kLaneEntries;               // entries per unit: two 16-byte loads
constexpr int kFlatWarps = kSampleThreads / 32;
constexpr int kFlatSegs = 32;                     // segments a warp takes at a time
constexpr int kFlatMeta = 2 * (kFlatSegs + 1) + 4 * kFlatSegs;  // ints of per-warp segment data
constexpr int kWalkLanes = 4;                     // lanes walking one range: 4 units, 128 bytes, per step

// Units of one warp batch: at least a whole row of K entries (K / 8 units).
// 512 (4,096 entries, 2 KB of prefixes per warp) was the fastest of 256, 512
// and 1024 on the 60M-token and the uneven 118M-token workloads.
__host__ __device__ constexpr int flat_unit_budget(int k) { return k / kUnit > 512 ? k / kUnit : 512; }

__device__ __forceinline__ Step load_unit(const ThetaEntry *__restrict__ theta, int idx) {
    Step st;
    load8(theta, idx, st.e);
    return st;
}

// phihat of an entry's topic: the entry's high half is its byte offset.
__device__ __forceinline__ float entry_phihat(uint32_t e, const float *ph) {
    return *reinterpret_cast<const float *>(reinterpret_cast<const char *>(ph) + (e >> 16));
}

// Sum of a unit's 8 products theta_dk * phihat_wk as one chain of fused
// multiply-adds in entry order (8 instructions instead of 8 multiplies and 7
// adds).  The draws' pass over a unit uses the same chain, so its running
// sum after the last entry equals this sum bit for bit.
__device__ __forceinline__ float unit_sum(const Step &st, const float *ph) {
    float s = 0.f;
#pragma unroll
    for (int j = 0; j < kUnit; ++j) s = __fmaf_rn(entry_count_f(st.e[j]), entry_phihat(st.e[j], ph), s);
    return s;
}

// Largest i in [0, n) with a[i] <= x, for non-decreasing a with a[0] <= x.
__device__ __forceinline__ int last_le(const int *a, int n, int x) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (a[mid] <= x)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ int warp_incl_scan(int v, int lane) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

// The first entry of a unit whose running sum, from `prev`, exceeds T; the
// unit's last non-zero entry when rounding leaves the unit short of T (-1 for
// a unit without non-zero entries).
__device__ __forceinline__ int resolve_unit(const Step &st, float prev, float T, const float *ph) {
    float part = 0.f;
    int hit = -1, last = -1;
#pragma unroll
    for (int j = 0; j < kUnit; ++j) {
        part = __fmaf_rn(entry_count_f(st.e[j]), entry_phihat(st.e[j], ph), part);
        const bool nz = entry_count(st.e[j]) != 0u;
        if (nz) last = entry_topic(st.e[j]);
        if (hit < 0 && nz && fsum(prev, part) > T) hit = entry_topic(st.e[j]);
    }
    return hit >= 0 ? hit : last;
}

// The row's last non-zero entry: rows hold their non-zero entries first and
// zero padding after them, up to the next multiple of 32, so it lies in the
// final 32-entry block.
__device__ __forceinline__ int row_last_nonzero(const ThetaEntry *__restrict__ theta, int rs, int re) {
    int last = -1;
    for (int i = max(rs, re - 32); i < re; ++i) {
        const ThetaEntry e = __ldg(theta + i);
        if (entry_count(e)) last = entry_topic(e);
    }
    return last;
}

// One walk group's pass over units [u0, ge) of a batch: the state carried
// from step to step.  step() reduces the step at u0 (its entries in `cur`)
// while the next step's entries load into `nx`, and returns false after the
// range's last step.  The kernel alternates two Step buffers, step(a, b) then
// step(b, a), so the prefetched entries never move between registers.
struct FlatWalk {
    const ThetaEntry *theta;
    const float *ph;
    float *ub;         // the batch's unit prefixes
    const int *m_cum;  // first unit of every segment of the batch
    const int *m_rs;   // row start of every segment
    int ge, wl;
    unsigned wm;
    int sp, nxt, rowu, rbase, u0;  // segment of unit u0, its successor's first unit, its row
    float s, c;                    // compensated running sum of the row
    int gflag;                     // a row started inside the range

    __device__ __forceinline__ bool step(const Step &cur, Step &nx) {
        const int u1 = u0 + kWalkLanes;
        bool reset1 = false;
        if (u1 < ge && u1 == nxt) {
            do {
                ++sp;
                nxt = m_cum[sp + 1];
            } while (nxt == u1);
            rowu = u1;
            rbase = m_rs[sp];
            reset1 = true;
        }
        if (u1 < ge) nx = load_unit(theta, rbase + kUnit * (u1 + wl - rowu));
        float incl = unit_sum(cur, ph);
#pragma unroll
        for (int o = 1; o < kWalkLanes; o <<= 1) {
            const float t = __shfl_up_sync(wm, incl, o, kWalkLanes);
            if (wl >= o) incl = fsum(incl, t);
        }
        const float tot = __shfl_sync(wm, incl, kWalkLanes - 1, kWalkLanes);
        ub[u0 + wl] = fsum(s + c, incl);
        neumaier(s, c, tot);
        if (u1 >= ge) return false;
        if (reset1) {
            s = 0.f;
            c = 0.f;
            gflag = 1;
        }
        u0 = u1;
        return true;
    }
};

// Items of at most kTinyTokens tokens (the long tail of the vocabulary) do not
// rebuild the K-wide phihat row and dense prefix: a CTA keeps the row of a word
// with no tokens, phihat_k = beta / (n_k + V beta), and its dense prefix, and an
// item only writes its own (at most 32) topics' phihat, the same values a full
// build gives, and restores them afterwards.  The dense prefix of the word is
// the base prefix plus the cumulative corrections alpha * (phihat_wk - base_k)
// of its topics, applied during the search.
constexpr int kTinyTokens = 32;

// The flat walk keeps the dense bucket as one prefix per block of 8 topics
// (K is a multiple of 32): qb[b] = alpha * sum of ph[0 .. 8 (b + 1)).  A draw
// finds its block by a binary search of qb and its topic by a pass over the
// block's 8 phihat values.  At K = 4096 that is 2 KB of shared memory instead
// of 16 KB, which lets 7 CTAs share an SM instead of 5.
constexpr int kDenseBlock = 8;

// Each thread takes a run of blocks: a block's total is the running sum a
// draw's pass over the block forms (the same operations, so the same bits),
// the run's prefix is compensated, and add_run_offsets completes it.
__device__ void dense_block_prefix(const float *ph, float *qb, int K, float alpha, float *s_warp) {
    const int T = blockDim.x, nb = K / kDenseBlock, per = (nb + T - 1) / T;
    const int b0 = min((int)threadIdx.x * per, nb), b1 = min(b0 + per, nb);
    float s = 0.f, c = 0.f;
    for (int b = b0; b < b1; ++b) {
        const float4 x = reinterpret_cast<const float4 *>(ph)[2 * b];
        const float4 y = reinterpret_cast<const float4 *>(ph)[2 * b + 1];
        float part = alpha * x.x;
        part = fsum(part, alpha * x.y);
        part = fsum(part, alpha * x.z);
        part = fsum(part, alpha * x.w);
        part = fsum(part, alpha * y.x);
        part = fsum(part, alpha * y.y);
        part = fsum(part, alpha * y.z);
        part = fsum(part, alpha * y.w);
        neumaier(s, c, part);
        qb[b] = s + c;
    }
    add_run_offsets(s + c, qb, b0, b1, s_warp);
    __syncthreads();
}

// Inside block b, from the prefix `base` before it: the first topic whose
// prefix exceeds tq, the block's last topic when rounding leaves it short.
__device__ __forceinline__ int dense_block_scan(const float *ph, int b, float base, float alpha, float tq) {
    const int t0 = b * kDenseBlock;
    float part = 0.f;
#pragma unroll
    for (int i = 0; i < kDenseBlock; ++i) {
        part = i ? fsum(part, alpha * ph[t0 + i]) : alpha * ph[t0];
        if (fsum(base, part) > tq) return t0 + i;
    }
    return t0 + kDenseBlock - 1;
}

// First topic whose dense prefix exceeds tq (K-1 when none does).
__device__ __forceinline__ int dense_search_blocks(const float *ph, const float *qb, int K, float alpha, float tq) {
    int lo = 0, hi = K / kDenseBlock - 1;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (qb[mid] > tq)
            hi = mid;
        else
            lo = mid + 1;
    }
    return dense_block_scan(ph, lo, lo > 0 ? qb[lo - 1] : 0.f, alpha, tq);
}

// The same for a tiny item: qb holds the base row's prefixes and ph the base
// row with the item's own topics patched in, so a block's prefix is qb[b]
// plus the corrections of the item's topics up to the block's end, and the
// pass over the block reads the patched values directly.
__device__ __forceinline__ int dense_search_tiny_blocks(const float *ph, const float *qb, int K, float alpha, float tq,
                                                        const int *tk, const float *dcum, int m) {
    auto corrected = [&](int b) {
        const int last = b * kDenseBlock + kDenseBlock - 1;
        int a = 0, e = m;  // topics of the item up to the block's end
        while (a < e) {
            const int c = (a + e) >> 1;
            if (tk[c] <= last)
                a = c + 1;
            else
                e = c;
        }
        return fsum(qb[b], a > 0 ? dcum[a - 1] : 0.f);
    };
    int lo = 0, hi = K / kDenseBlock - 1;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (corrected(mid) > tq)
            hi = mid;
        else
            lo = mid + 1;
    }
    return dense_block_scan(ph, lo, lo > 0 ? corrected(lo - 1) : 0.f, alpha, tq);
}

template <int MINB>
__global__ void __launch_bounds__(kSampleThreads, MINB) sample_flat_kernel(const SampleParams p) {
    extern __shared__ float smem[];
    const int K = p.k, KP = p.kmask + 1, B = flat_unit_budget(K);
    float *ph = smem;               // [KP] phihat of the current word (zero past K), at offset 0
                                    // (the word histogram before that)
    float *qb = smem + KP;          // [K / 8] dense-bucket prefix at the end of every 8-topic block
    int *hist = reinterpret_cast<int *>(ph);
    __shared__ int s_item, s_chunk;
    __shared__ float s_warp[kSampleThreads / 32];
    __shared__ double s_red[kSampleThreads / 32];
    // tiny items: whether ph / qb hold the base row, and the item's topics
    __shared__ int s_tiny, s_tm;
    __shared__ int s_tk[kTinyTokens];
    __shared__ float s_tdc[kTinyTokens];
    __shared__ float s_tQ;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wl = lane & (kWalkLanes - 1), wg = lane / kWalkLanes;  // lane in its walk group, group
    const unsigned wm = group_mask<kWalkLanes>(lane);
    float *ub = qb + K / kDenseBlock + warp * B;  // [B] unit prefixes of the warp's batch
    int *m_cum = reinterpret_cast<int *>(qb + K / kDenseBlock + kFlatWarps * B) + warp * kFlatMeta;
    int *m_tc = m_cum + (kFlatSegs + 1);  // [n+1] first unit / first token (flat) of each segment
    int *m_rs = m_tc + (kFlatSegs + 1);   // [n] row start (entry index)
    int *m_t0 = m_rs + kFlatSegs;         // [n] first token
    float *m_S = reinterpret_cast<float *>(m_t0 + kFlatSegs);  // [n] S of the row
    float *m_lg = m_S + kFlatSegs;                               // [n] log(S + Q)
    const uint32_t iter = p.iteration_ptr ? *p.iteration_ptr : p.iteration;

    for (int j = K + tid; j < KP; j += blockDim.x) ph[j] = 0.f;
    if (tid == 0) s_tiny = 0;

    for (;;) {
        if (tid == 0) {
            s_item = atomicAdd(p.item_counter, 1);
            s_chunk = 0;
        }
        __syncthreads();
        const int it = s_item;
        if (it >= p.num_items) break;
        const culda_item item = p.items[it];
        const int64_t ibeg = item.begin, iend = item.begin + item.count;
        if (ibeg < 0 || item.count < 0 || iend > p.num_tokens || item.hot >= p.num_hot || item.seg_begin < 0 ||
            item.seg_count < 0 || (int64_t)item.seg_begin + item.seg_count > p.num_segs) {
            if (tid == 0) {
                atomicOr(p.error, kErrRowRange);
                p.item_ll[it] = 0.0;
            }
            __syncthreads();  // s_item is rewritten only after every thread has read it
            continue;
        }

        // phi row of the word
        // (at K = 256 the full build is cheaper than the patch: 16.2 against 15.7 ms per iteration)
        const bool tiny = K >= 512 && !p.frozen_phi && item.hot < 0 && item.count <= kTinyTokens;
        float Q;
        if (tiny) {
            if (!s_tiny) {  // the base row and its dense prefix, once per CTA
                for (int j = tid; j < K; j += blockDim.x)
                    ph[j] = (0.f + p.beta) * (1.0f / ((float)__ldg(p.nk + j) + p.vbeta));
                __syncthreads();
                dense_block_prefix(ph, qb, K, p.alpha, s_warp);
                if (tid == 0) s_tiny = 1;
            }
            if (warp == 0) {
                // the item's distinct topics (match groups), their counts and ranks
                uint32_t z = 0xFFFFFFFFu;
                if (lane < (int)item.count) {
                    z = p.topics_in[ibeg + lane];
                    if (z >= (uint32_t)K) {
                        atomicOr(p.error, kErrTopicRange);
                        z = 0xFFFFFFFFu;
                    }
                }
                const unsigned grp = __match_any_sync(0xffffffffu, z);
                const bool lead = z != 0xFFFFFFFFu && __ffs(grp) - 1 == lane;
                const uint32_t key = lead ? z : 0xFFFFFFFFu;
                int rank = 0;
#pragma unroll 8
                for (int j = 0; j < 32; ++j) rank += __shfl_sync(0xffffffffu, key, j) < key;
                const int m = __popc(__ballot_sync(0xffffffffu, lead));
                float d = 0.f;
                if (lead) {
                    const float v = ((float)__popc(grp) + p.beta) * (1.0f / ((float)__ldg(p.nk + z) + p.vbeta));
                    d = p.alpha * v - p.alpha * ph[z];  // ph[z] holds the base value here
                    ph[z] = v;
                    s_tk[rank] = (int)z;
                    s_tdc[rank] = d;
                }
                // the corrections in topic order, then their running sums
                __syncwarp();
                float dc = lane < m ? s_tdc[lane] : 0.f;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const float t = __shfl_up_sync(0xffffffffu, dc, o);
                    if (lane >= o) dc = fsum(dc, t);
                }
                __syncwarp();
                if (lane < m) s_tdc[lane] = dc;
                const float total = __shfl_sync(0xffffffffu, dc, m > 0 ? m - 1 : 0);
                if (lane == 0) {
                    s_tm = m;
                    s_tQ = fsum(qb[K / kDenseBlock - 1], m > 0 ? total : 0.f);
                }
            }
            __syncthreads();
            Q = s_tQ;
        } else {
            const int *src;
            if (p.frozen_phi) {
                src = p.frozen_phi + (size_t)item.word * K;
            } else if (item.hot < 0) {
                for (int j = tid; j < K; j += blockDim.x) hist[j] = 0;
                __syncthreads();
                for (int64_t t = ibeg + tid; t < iend; t += blockDim.x) {
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
            // 1 / (n_k + V beta) is formed per item (the same operations, so the
            // same bits, as a table would hold), which keeps the table's 4 KB
            // out of each CTA's shared memory
            for (int j = tid; j < K; j += blockDim.x)
                ph[j] = ((float)src[j] + p.beta) * (1.0f / ((float)__ldg(p.nk + j) + p.vbeta));
            __syncthreads();
            dense_block_prefix(ph, qb, K, p.alpha, s_warp);
            Q = qb[K / kDenseBlock - 1];
            if (tid == 0) s_tiny = 0;  // read by every thread before the barrier above
        }

        double ll = 0.0;
        const int sg_end = item.seg_begin + item.seg_count;
        // chunks of a quarter of the item's segments (at most 32), so the four
        // warps share small items too (on the uneven 118M-token workload a
        // floor of 1 segment beat floors of 2, 4, 8 and 16)
        const int cs = min(kFlatSegs, max(1, (item.seg_count + kFlatWarps - 1) / kFlatWarps));
        for (;;) {
            int ch = 0;
            if (lane == 0) ch = atomicAdd(&s_chunk, 1);
            ch = __shfl_sync(0xffffffffu, ch, 0);
            if ((int64_t)ch * cs >= item.seg_count) break;
            const int seg0 = item.seg_begin + ch * cs;
            const int nseg = min(cs, sg_end - seg0);

            // lane s holds segment seg0 + s: its tokens, doc and theta row
            int rs = 0, nu = 0, t0 = 0, tcount = 0;
            if (lane < nseg) {
                const int sg = seg0 + lane;
                const int64_t a0 = __ldg(p.seg_start + sg);
                const int64_t a1 = sg + 1 < sg_end ? (int64_t)__ldg(p.seg_start + sg + 1) : iend;
                if (a0 < ibeg || a1 > iend || a0 >= a1) {
                    atomicOr(p.error, kErrRowRange);
                } else {
                    const int d = __ldg(p.doc_ids + a0);
                    if ((unsigned)d < (unsigned)p.num_docs) {
                        const int2 r = __ldg(p.rows + d);
                        if (r.x >= 0 && r.x <= r.y && (int64_t)r.y <= p.theta_cap && ((r.x | r.y) & 31) == 0 &&
                            r.y - r.x <= kUnit * B) {
                            rs = r.x;
                            nu = (r.y - r.x) / kUnit;
                            t0 = (int)a0;
                            tcount = (int)(a1 - a0);
                        } else {
                            atomicOr(p.error, kErrRowRange);
                        }
                    } else {
                        atomicOr(p.error, kErrDocRange);
                    }
                }
            }

            int done = 0;
            while (done < nseg) {
                // the batch: segments [done, last] whose units fit the budget
                const bool act = lane >= done && lane < nseg;
                const int v = act ? nu : 0;
                const int incl = warp_incl_scan(v, lane);
                const unsigned fm = __ballot_sync(0xffffffffu, act && incl <= B);
                const int last = 31 - __clz(fm);  // lane `done` always fits: nu <= B
                const int n = last - done + 1;
                const bool mine = act && lane <= last;
                const int tc = mine ? tcount : 0;
                const int tincl = warp_incl_scan(tc, lane);
                const int total_u = __shfl_sync(0xffffffffu, incl, last);
                const int total_t = __shfl_sync(0xffffffffu, tincl, last);
                if (mine) {
                    const int i = lane - done;
                    m_cum[i] = incl - v;
                    m_tc[i] = tincl - tc;
                    m_rs[i] = rs;
                    m_t0[i] = t0;
                    if (lane == last) {
                        m_cum[n] = incl;
                        m_tc[n] = tincl;
                    }
                }
                __syncwarp();

                // walk: group g (lanes 4g..4g+3) takes units [gb, ge), 4 per step,
                // a step being one 128-byte line of one row; the running sum
                // restarts at every row start
                const int r = ((total_u + 31) >> 5) | 1;  // odd: the 8 groups' stores hit distinct banks
                const int gb = min(wg * 4 * r, total_u), ge = min(gb + 4 * r, total_u);
                float gv = 0.f;
                int gflag = 0, lead_end = gb;
                if (gb < ge) {
                    const int sp = last_le(m_cum, n, gb);
                    FlatWalk w{p.theta, ph, ub, m_cum, m_rs, ge, wl, wm, sp, m_cum[sp + 1], m_cum[sp], m_rs[sp], gb,
                               0.f, 0.f, 0};
                    w.gflag = gb == w.rowu;
                    lead_end = w.gflag ? gb : min(w.nxt, ge);
                    Step a = load_unit(p.theta, w.rbase + kUnit * (gb + wl - w.rowu)), b;
                    while (w.step(a, b) && w.step(b, a)) {
                    }
                    gflag = w.gflag;
                    gv = w.s + w.c;
                }
                // segmented scan over the groups: the running row sum entering each range
                double vd = (double)gv;
                int fl = gflag;
#pragma unroll
                for (int o = kWalkLanes; o < 32; o <<= 1) {
                    const double vo = __shfl_up_sync(0xffffffffu, vd, o);
                    const int fo = __shfl_up_sync(0xffffffffu, fl, o);
                    if (lane >= o && !fl) {
                        vd += vo;
                        fl = fo;
                    }
                }
                double carry = __shfl_up_sync(0xffffffffu, vd, kWalkLanes);
                if (lane < kWalkLanes) carry = 0.0;
                if (gb < lead_end) {
                    const float cf = (float)carry;
                    for (int u = gb + wl; u < lead_end; u += kWalkLanes) ub[u] = fsum(ub[u], cf);
                }
                __syncwarp();
                if (mine) {
                    const int i = lane - done;
                    const int c0 = m_cum[i], c1 = m_cum[i + 1];
                    const float S = c1 > c0 ? ub[c1 - 1] : 0.f;
                    m_S[i] = S;
                    m_lg[i] = logf(S + Q);
                }
                __syncwarp();

                // draws: lane f takes the batch's tokens f, f + 32, ...
                for (int f = lane; f < total_t; f += 32) {
                    const int i = last_le(m_tc, n, f);
                    const int tok = m_t0[i] + (f - m_tc[i]);
                    float um;
                    if (p.uniforms) {
                        um = __ldg(p.uniforms + tok);
                    } else {
                        const int64_t key = p.tok_index ? (int64_t)__ldg(p.tok_index + tok) : (int64_t)tok;
                        um = uniform_from_bits(philox_token(p.seed, (uint64_t)key, iter, kPurposeSample));
                    }
                    const float S = m_S[i];
                    const float T = um * (S + Q);
                    int z;
                    if (T < S) {
                        const int c0 = m_cum[i];
                        int lo = c0, hi = m_cum[i + 1] - 1;
                        while (lo < hi) {
                            const int mid = (lo + hi) >> 1;
                            if (ub[mid] > T)
                                hi = mid;
                            else
                                lo = mid + 1;
                        }
                        const float prev = lo > c0 ? ub[lo - 1] : 0.f;
                        z = resolve_unit(load_unit(p.theta, m_rs[i] + kUnit * (lo - c0)), prev, T, ph);
                        // a unit of the row's padding: T lies within a rounding of the
                        // prefix where that unit starts (a lane's carried-in sum can round
                        // one unit in the last place above the previous unit's prefix)
                        if (z < 0) z = row_last_nonzero(p.theta, m_rs[i], m_rs[i] + kUnit * (m_cum[i + 1] - c0));
                    } else {
                        z = tiny ? dense_search_tiny_blocks(ph, qb, K, p.alpha, T - S, s_tk, s_tdc, s_tm)
                                 : dense_search_blocks(ph, qb, K, p.alpha, T - S);
                    }
                    if (z < 0) {
                        atomicOr(p.error, kErrRowRange);
                        z = 0;
                    }
                    p.topics_out[tok] = (uint16_t)z;
                    ll += (double)m_lg[i];
                }
                __syncwarp();  // the batch's shared data is read before the next batch writes it
                done = last + 1;
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) ll += __shfl_down_sync(0xffffffffu, ll, o);
        if (lane == 0) s_red[warp] = ll;
        __syncthreads();
        if (tid == 0) {
            double s = 0.0;
            for (int w = 0; w < kSampleThreads / 32; ++w) s += s_red[w];
            p.item_ll[it] = s;
        }
        // a tiny item's topics back to the base row (every draw of it is done)
        if (tiny && tid < s_tm)
            ph[s_tk[tid]] = (0.f + p.beta) * (1.0f / ((float)__ldg(p.nk + s_tk[tid]) + p.vbeta));
    }
}

size_t sample_smem_bytes(int k, int group_lanes) {
    if (group_lanes == kFlatLanes)  // ph[pow2(K)] + qb[K/8] + per warp: unit prefixes and segment data
        return ((size_t)k / kDenseBlock + (size_t)pow2_ceil(k) + (size_t)kFlatWarps * flat_unit_budget(k) +
                (size_t)kFlatWarps * kFlatMeta) *
               sizeof(float);
    // ph[pow2(K)] + inv[K] + qc[K] + the per-group running sums
    return ((size_t)2 * k + (size_t)pow2_ceil(k) + (size_t)SampleShape<1>::kPrefixFloats) * sizeof(float);
}

template <int G, int MINB>
static const void *sample_fn() {
    return reinterpret_cast<const void *>(&sample_kernel<G, MINB>);
}

static const void *sample_kernel_for(int g, int minb) {
    if (g == kFlatLanes) {
        if (minb == kSampleBlocksDefault) return reinterpret_cast<const void *>(&sample_flat_kernel<kSampleBlocksDefault>);
        if (minb == kFlatBlocks) return reinterpret_cast<const void *>(&sample_flat_kernel<kFlatBlocks>);
        return nullptr;
    }
    if (minb == kSampleBlocksDefault) switch (g) {
            case 1: return sample_fn<1, kSampleBlocksDefault>();
            case 2: return sample_fn<2, kSampleBlocksDefault>();
            case 4: return sample_fn<4, kSampleBlocksDefault>();
            case 8: return sample_fn<8, kSampleBlocksDefault>();
            case 16: return sample_fn<16, kSampleBlocksDefault>();
            case 32: return sample_fn<32, kSampleBlocksDefault>();
            default: return nullptr;
        }
    if (minb == kSampleBlocksHigh) switch (g) {
            case 4: return sample_fn<4, kSampleBlocksHigh>();
            case 8: return sample_fn<8, kSampleBlocksHigh>();
            case 16: return sample_fn<16, kSampleBlocksHigh>();
            default: return nullptr;
        }
    return nullptr;
}

bool sample_variant_exists(int group_lanes, int blocks_per_sm) {
    return sample_kernel_for(group_lanes, blocks_per_sm) != nullptr;
}

int sample_blocks_per_sm(int k, int group_lanes, int blocks_per_sm) {
    const void *fn = sample_kernel_for(group_lanes, blocks_per_sm);
    if (!fn) return 0;
    const size_t smem = sample_smem_bytes(k, group_lanes);
    if (allow_smem(fn, smem, nullptr) != cudaSuccess) return 0;
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, kSampleThreads, smem) != cudaSuccess) return 0;
    return n;
}

cudaError_t launch_sample(const SampleParams &p, int group_lanes, int blocks_per_sm, int grid, cudaStream_t s) {
    const size_t smem = sample_smem_bytes(p.k, group_lanes);
    void *args[] = {const_cast<SampleParams *>(&p)};
    const void *fn = sample_kernel_for(group_lanes, blocks_per_sm);
    if (!fn) return cudaErrorInvalidValue;
    cudaError_t e = allow_smem(fn, smem, s);
    if (e != cudaSuccess) return e;
    return cudaLaunchKernel(fn, dim3(grid), dim3(kSampleThreads), args, smem, s);
}

// ----------------------------------------------------------- hot-word rows
// Full phi rows of words split over several work items: each CTA histograms
// one slice in shared memory and adds the non-zero bins to the word's row.
__global__ void __launch_bounds__(256) hot_rows_kernel(int K, const culda_item *__restrict__ hot_items,
                                                       const uint16_t *__restrict__ topics, int32_t *hot_phi,
                                                       int32_t *error) {
    extern __shared__ int hist_s[];
    const culda_item it = hot_items[blockIdx.x];
    for (int j = threadIdx.x; j < K; j += blockDim.x) hist_s[j] = 0;
    __syncthreads();
    for (int64_t t = it.begin + threadIdx.x; t < it.begin + it.count; t += blockDim.x) {
        const uint32_t z = topics[t];
        if (z < (uint32_t)K)
            atomicAdd(&hist_s[z], 1);
        else
            atomicOr(error, kErrTopicRange);
    }
    __syncthreads();
    int32_t *row = hot_phi + (size_t)it.hot * K;
    for (int j = threadIdx.x; j < K; j += blockDim.x)
        if (hist_s[j]) atomicAdd(&row[j], hist_s[j]);
}

cudaError_t launch_hot_rows(int k, const culda_item *hot_items, int num_hot_items, const uint16_t *topics,
                            int32_t *hot_phi, int32_t *error, cudaStream_t s) {
    if (num_hot_items <= 0) return cudaSuccess;
    const size_t smem = (size_t)k * sizeof(int);
    cudaError_t e = allow_smem(reinterpret_cast<const void *>(&hot_rows_kernel), smem, s);
    if (e != cudaSuccess) return e;
    hot_rows_kernel<<<num_hot_items, 256, smem, s>>>(k, hot_items, topics, hot_phi, error);
    return cudaGetLastError();
}

// ------------------------------------------------------------- LL finalize
__global__ void __launch_bounds__(256) finalize_ll_kernel(const double *__restrict__ item_ll, int num_items,
                                                          DevStats *st, uint32_t *iteration_dev) {
    __shared__ double red[256];
    double s = 0.0;
    for (int i = threadIdx.x; i < num_items; i += 256) s += item_ll[i];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        st->ll_sum = red[0];
        if (iteration_dev) {
            st->iteration = *iteration_dev;
            *iteration_dev += 1u;
        }
    }
}

cudaError_t launch_finalize_ll(const double *item_ll, int num_items, DevStats *st, uint32_t *iteration_dev,
                               cudaStream_t s) {
    finalize_ll_kernel<<<1, 256, 0, s>>>(item_ll, num_items, st, iteration_dev);
    return cudaGetLastError();
}

// ------------------------------------------------- theta entry validation
// Every entry of every row must carry a topic below K (as a byte offset) and
// rows must be 32-aligned inside the array: checked before the kernel-level
// entry point samples a caller's theta.
__global__ void check_theta_kernel(int num_docs, int K, const int2 *__restrict__ rows,
                                   const ThetaEntry *__restrict__ theta, int64_t cap, int32_t *error) {
    const int lane = threadIdx.x & 31;
    for (int d = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; d < num_docs; d += (gridDim.x * blockDim.x) >> 5) {
        const int2 r = rows[d];
        if (r.x < 0 || r.y < r.x || (int64_t)r.y > cap || ((r.x | r.y) & 31)) {
            if (lane == 0) atomicOr(error, kErrRowRange);
            continue;
        }
        for (int i = r.x + lane; i < r.y; i += 32) {
            const ThetaEntry e = theta[i];
            if ((e & 0x30000u) || (e >> 18) >= (uint32_t)K) atomicOr(error, kErrTopicRange);
        }
    }
}

cudaError_t launch_check_theta(int num_docs, int k, const int2 *rows, const ThetaEntry *theta, int64_t cap,
                               int32_t *error, cudaStream_t s) {
    check_theta_kernel<<<grid_for((int64_t)num_docs * 32), 256, 0, s>>>(num_docs, k, rows, theta, cap, error);
    return cudaGetLastError();
}

}  // namespace culda
