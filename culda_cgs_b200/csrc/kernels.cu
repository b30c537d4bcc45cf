// kernels.cu — the sm_100a kernels of the one-GPU CGS iteration and the
// kernel-level C entry points that mirror the reference's kernel APIs.
//
// Iteration data flow (all resident in HBM, word-major token order):
//   hot_rows_kernel     topics_in of hot words -> full phi rows of words split
//                       over several work items (shared-memory histograms)
//   sample_kernel<G>    persistent CTAs pull work items (one word or a slice
//                       of a hot word); per item: phi row as a shared-memory
//                       histogram of topics_in (no dense V x K phi in HBM),
//                       phihat = (n_wk + beta) / (n_k + V beta) in FP32, the
//                       alpha*phihat prefix for the dense bucket; per token a
//                       group of G lanes walks the doc's theta row with 16-byte
//                       loads and draws the new topic.
//   finalize_ll_kernel  fixed-order sum of the per-item log terms
//   theta_rebuild_kernel warp per doc (longest first): 16-bit shared-memory
//                       histogram of the doc's new topics, CSR compaction in
//                       ascending topic, zero padding, n_k as a column sum.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>

#include "kernels.cuh"
#include "philox.h"

namespace culda {

// ------------------------------------------------------------------ helpers
__device__ __forceinline__ void neumaier(float &s, float &c, float x) {
    const float t = s + x;
    if (fabsf(s) >= fabsf(x))
        c += (s - t) + x;
    else
        c += (x - t) + s;
    s = t;
}

template <int G>
__device__ __forceinline__ unsigned group_mask(int lane) {
    if constexpr (G == 32)
        return 0xffffffffu;
    else
        return ((1u << G) - 1u) << (lane & ~(G - 1));
}

template <int G>
__device__ __forceinline__ float group_sum(float v, unsigned m) {
    if constexpr (G > 1) {
#pragma unroll
        for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(m, v, o);
    }
    return v;
}

template <int G, class T>
__device__ __forceinline__ T group_bcast(T v, int src, unsigned m) {
    if constexpr (G == 1)
        return v;
    else
        return __shfl_sync(m, v, src, G);
}

// Ballot restricted to the group, bit j = lane j of the group.
template <int G>
__device__ __forceinline__ unsigned group_ballot(bool pred, unsigned m, int lane) {
    const unsigned b = __ballot_sync(m, pred);
    if constexpr (G == 32)
        return b;
    else
        return (b >> (lane & ~(G - 1))) & ((1u << G) - 1u);
}

// Exclusive prefix of v over the group's lanes (Kogge-Stone).
template <int G>
__device__ __forceinline__ float group_excl(float v, int gl, unsigned m) {
    if constexpr (G == 1) {
        return 0.f;
    } else {
        float incl = v;
#pragma unroll
        for (int o = 1; o < G; o <<= 1) {
            const float t = __shfl_up_sync(m, incl, o, G);
            if (gl >= o) incl += t;
        }
        const float ex = __shfl_up_sync(m, incl, 1, G);
        return gl == 0 ? 0.f : ex;
    }
}

// Opt a kernel into more than 48 KB of dynamic shared memory.  Skipped while
// the stream is being captured into a graph: the context sets every attribute
// before it captures.
static cudaError_t allow_smem(const void *fn, size_t smem, cudaStream_t s) {
    if (smem <= 48 * 1024) return cudaSuccess;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone) return cudaSuccess;
    return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

__device__ __forceinline__ float entry_prob(uint32_t e, const float *ph, int kmax) {
    return (float)(e >> 16) * ph[min((int)(e & 0xFFFFu), kmax)];
}

// --------------------------------------------------------------- sampling
// Inclusive prefix qc[j] = alpha * sum_{i<=j} ph[i].  Each thread owns a run of
// ceil(K/T) entries summed with Neumaier compensation; the run totals are
// scanned with Kogge-Stone shuffles, so every prefix has an error of about
// ten FP32 roundings.
__device__ void dense_bucket_prefix(const float *ph, float *qc, int K, float alpha, float *s_warp) {
    const int T = blockDim.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = T >> 5;
    const int per = (K + T - 1) / T;
    const int b = min(tid * per, K), e = min(b + per, K);
    float s = 0.f, c = 0.f;
    for (int j = b; j < e; ++j) {
        neumaier(s, c, alpha * ph[j]);
        qc[j] = s + c;
    }
    const float tot = s + c;
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
    for (int j = b; j < e; ++j) qc[j] = base + qc[j];
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

// One token: S over the doc's theta row [rs, re), the draw, the new topic.
// All G lanes of the group take the same branches (their sums are bitwise
// equal), so group-masked shuffles are safe.
template <int G>
__device__ __forceinline__ int sample_token(const uint32_t *__restrict__ theta, const float *ph, const float *qc,
                                            float Q, int K, int rs, int re, float u, int gl, unsigned m, int lane,
                                            float &total_out) {
    const int kmax = K - 1;
    // pass 1: S as a compensated sum of group chunk totals
    float s = 0.f, c = 0.f;
    for (int base = rs; base < re; base += 4 * G) {
        const int idx = base + 4 * gl;
        uint4 e = make_uint4(0u, 0u, 0u, 0u);
        if (idx < re) e = __ldg(reinterpret_cast<const uint4 *>(theta + idx));
        const float cl = (entry_prob(e.x, ph, kmax) + entry_prob(e.y, ph, kmax)) +
                         (entry_prob(e.z, ph, kmax) + entry_prob(e.w, ph, kmax));
        neumaier(s, c, group_sum<G>(cl, m));
    }
    const float S = s + c;
    const float total = S + Q;
    total_out = total;
    const float T = u * total;
    if (T < S) {
        // pass 2: the same running sum up to the chunk that crosses T
        float s2 = 0.f, c2 = 0.f;
        for (int base = rs; base < re; base += 4 * G) {
            const int idx = base + 4 * gl;
            uint4 e = make_uint4(0u, 0u, 0u, 0u);
            if (idx < re) e = __ldg(reinterpret_cast<const uint4 *>(theta + idx));
            const float p0 = entry_prob(e.x, ph, kmax), p1 = entry_prob(e.y, ph, kmax);
            const float p2 = entry_prob(e.z, ph, kmax), p3 = entry_prob(e.w, ph, kmax);
            const float cl = (p0 + p1) + (p2 + p3);
            const float prev = s2 + c2;
            neumaier(s2, c2, group_sum<G>(cl, m));
            if (s2 + c2 > T) {
                float cum = prev + group_excl<G>(cl, gl, m);
                int hit = -1, lastnz = -1;
                const uint32_t ev[4] = {e.x, e.y, e.z, e.w};
                const float pv[4] = {p0, p1, p2, p3};
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    cum += pv[i];
                    if (ev[i] >> 16) {
                        lastnz = min((int)(ev[i] & 0xFFFFu), kmax);
                        if (hit < 0 && cum > T) hit = lastnz;
                    }
                }
                const unsigned hb = group_ballot<G>(hit >= 0, m, lane);
                if (hb) return group_bcast<G>(hit, __ffs(hb) - 1, m);
                const unsigned nb = group_ballot<G>(lastnz >= 0, m, lane);
                if (nb) return group_bcast<G>(lastnz, 31 - __clz(nb), m);
                return -1;
            }
        }
        return -1;
    }
    return dense_bucket_search<G>(qc, K, T - S, gl, m, lane);
}

template <int G>
__global__ void __launch_bounds__(kSampleThreads) sample_kernel(const SampleParams p) {
    extern __shared__ float smem[];
    const int K = p.k;
    float *inv = smem;          // [K] 1 / (n_k + V beta)
    float *ph = smem + K;       // [K] phihat of the current word
    float *qc = smem + 2 * K;   // [K] dense-bucket prefix (the word histogram before that)
    int *hist = reinterpret_cast<int *>(qc);
    __shared__ int s_item;
    __shared__ float s_warp[kSampleThreads / 32];
    __shared__ double s_red[kSampleThreads / 32];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int gl = lane & (G - 1);
    const int group = tid / G;
    constexpr int NG = kSampleThreads / G;
    const unsigned m = group_mask<G>(lane);
    const uint32_t iter = p.iteration_ptr ? *p.iteration_ptr : p.iteration;

    for (int j = tid; j < K; j += blockDim.x) inv[j] = 1.0f / ((float)p.nk[j] + p.vbeta);

    for (;;) {
        if (tid == 0) s_item = atomicAdd(p.item_counter, 1);
        __syncthreads();
        const int it = s_item;
        if (it >= p.num_items) break;
        const culda_item item = p.items[it];
        const int64_t ibeg = item.begin, iend = item.begin + item.count;
        if (ibeg < 0 || item.count < 0 || iend > p.num_tokens || item.hot >= p.num_hot) {
            if (tid == 0) atomicOr(p.error, kErrRowRange);
            if (tid == 0) p.item_ll[it] = 0.0;
            __syncthreads();  // s_item is rewritten only after every thread has read it
            continue;
        }

        // phi row of the word
        const int *src;
        if (item.hot < 0) {
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
        for (int64_t tb = ibeg + group; tb < iend; tb += (int64_t)NG * G) {
            // lane gl prefetches the gl-th token of this batch
            const int64_t tm = tb + (int64_t)gl * NG;
            int dm = -1, rsm = 0, rem = 0;
            uint32_t xm = 0;
            if (tm < iend) {
                const int d = __ldg(p.doc_ids + tm);
                if ((unsigned)d < (unsigned)p.num_docs) {
                    const int2 r = __ldg(p.rows + d);
                    if (r.x >= 0 && r.x <= r.y && (int64_t)r.y <= p.theta_cap && ((r.x | r.y) & 3) == 0) {
                        dm = d;
                        rsm = r.x;
                        rem = r.y;
                    } else {
                        atomicOr(p.error, kErrRowRange);
                    }
                } else {
                    atomicOr(p.error, kErrDocRange);
                }
                xm = philox_token(p.seed, (uint64_t)tm, iter, kPurposeSample);
            }
#pragma unroll 1
            for (int j = 0; j < G; ++j) {
                const int64_t t = tb + (int64_t)j * NG;
                if (t >= iend) break;
                const int d = group_bcast<G>(dm, j, m);
                const int rs = group_bcast<G>(rsm, j, m), re = group_bcast<G>(rem, j, m);
                const uint32_t x = group_bcast<G>(xm, j, m);
                if (d < 0) continue;
                float total;
                int z = sample_token<G>(p.theta, ph, qc, Q, K, rs, re, uniform_from_bits(x), gl, m, lane, total);
                if (gl == 0) {
                    if (z < 0) {
                        atomicOr(p.error, kErrRowRange);
                        z = 0;
                    }
                    p.topics_out[t] = (uint16_t)z;
                    ll += (double)logf(total);
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

size_t sample_smem_bytes(int k) { return (size_t)3 * (size_t)k * sizeof(float); }

template <int G>
static const void *sample_fn() {
    return reinterpret_cast<const void *>(&sample_kernel<G>);
}

static const void *sample_kernel_for(int g) {
    switch (g) {
        case 1: return sample_fn<1>();
        case 2: return sample_fn<2>();
        case 4: return sample_fn<4>();
        case 8: return sample_fn<8>();
        case 16: return sample_fn<16>();
        case 32: return sample_fn<32>();
        default: return nullptr;
    }
}

int sample_blocks_per_sm(int k, int group_lanes) {
    const void *fn = sample_kernel_for(group_lanes);
    if (!fn) return 0;
    const size_t smem = sample_smem_bytes(k);
    if (smem > 48 * 1024) cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, kSampleThreads, smem) != cudaSuccess) return 0;
    return n;
}

cudaError_t launch_sample(const SampleParams &p, int group_lanes, int grid, cudaStream_t s) {
    const size_t smem = sample_smem_bytes(p.k);
    void *args[] = {const_cast<SampleParams *>(&p)};
    const void *fn = sample_kernel_for(group_lanes);
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
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(hot_rows_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
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

// ---------------------------------------------------------- theta rebuild
// Warp per doc.  Shared memory per warp: K/2 words of packed 16-bit counts
// (a topic can hold at most L_d <= 65535 tokens, so a low half never carries
// into the high half) and K/32 words of a non-zero mask; per block: K n_k
// partial counts.  The compaction walks the mask in ascending topic order, so
// each row comes out sorted as lda_theta_kernel.cu:58-85 leaves it, and only
// the touched count words are cleared again.
__global__ void __launch_bounds__(kThetaWarps * 32) theta_rebuild_kernel(
    int K, int num_docs, const int64_t *__restrict__ doc_ptr, const int32_t *__restrict__ doc_tok,
    const uint16_t *__restrict__ topics, const int32_t *__restrict__ doc_order, int2 *rows, uint32_t *theta,
    int32_t *nk, int64_t *stats, int32_t *error) {
    extern __shared__ uint32_t sm_u32[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int cwords = K >> 1, mwords = K >> 5;
    uint32_t *nk_acc = sm_u32;
    uint32_t *cnt = sm_u32 + K + warp * (cwords + mwords);
    uint32_t *mask = cnt + cwords;
    for (int i = threadIdx.x; i < K; i += blockDim.x) nk_acc[i] = 0u;
    for (int i = lane; i < cwords + mwords; i += 32) cnt[i] = 0u;
    __syncthreads();

    int64_t my_rows = 0, my_nnz = 0, my_tok_nnz = 0;
    const int nw = gridDim.x * kThetaWarps;
    for (int i = blockIdx.x * kThetaWarps + warp; i < num_docs; i += nw) {
        const int d = doc_order ? doc_order[i] : i;
        const int64_t b = doc_ptr[d], e = doc_ptr[d + 1];
        if (e - b > 65535) {
            if (lane == 0) atomicOr(error, kErrLongDoc);
            continue;
        }
        for (int64_t j = b + lane; j < e; j += 32) {
            const uint32_t z = topics[doc_tok[j]];
            if (z >= (uint32_t)K) {
                atomicOr(error, kErrTopicRange);
                continue;
            }
            const uint32_t sh = (z & 1u) << 4;
            const uint32_t old = atomicAdd(&cnt[z >> 1], 1u << sh);
            if (((old >> sh) & 0xFFFFu) == 0u) atomicOr(&mask[z >> 5], 1u << (z & 31u));
        }
        __syncwarp();
        const int2 row = rows[d];
        const int start = row.x, old_end = row.y;
        int nnz = 0;
        for (int mb = 0; mb < mwords; mb += 32) {
            const int mi = mb + lane;
            const uint32_t mw = mi < mwords ? mask[mi] : 0u;
            const int pc = __popc(mw);
            int incl = pc;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int v = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += v;
            }
            const int total = __shfl_sync(0xffffffffu, incl, 31);
            int pos = start + nnz + incl - pc;
            uint32_t bits = mw;
            while (bits) {
                const int bit = __ffs(bits) - 1;
                bits &= bits - 1u;
                const uint32_t z = ((uint32_t)mi << 5) | (uint32_t)bit;
                const uint32_t c = (cnt[z >> 1] >> ((z & 1u) << 4)) & 0xFFFFu;
                theta[pos++] = (c << 16) | z;
                atomicAdd(&nk_acc[z], c);
            }
            __syncwarp();
            bits = mw;
            while (bits) {
                const int bit = __ffs(bits) - 1;
                bits &= bits - 1u;
                cnt[(((uint32_t)mi << 5) | (uint32_t)bit) >> 1] = 0u;
            }
            if (mi < mwords) mask[mi] = 0u;
            nnz += total;
        }
        __syncwarp();
        const int new_end = start + ((nnz + 31) & ~31);
        const int zend = max(new_end, old_end);
        for (int j = start + nnz + lane; j < zend; j += 32) theta[j] = 0u;
        if (lane == 0) {
            rows[d].y = new_end;
            my_rows += (e - b) * (int64_t)(new_end - start);
            my_nnz += nnz;
            my_tok_nnz += (e - b) * (int64_t)nnz;
        }
    }
    __syncthreads();
    if (nk)
        for (int i = threadIdx.x; i < K; i += blockDim.x)
            if (nk_acc[i]) atomicAdd(&nk[i], (int)nk_acc[i]);
    if (lane == 0 && stats) {
        atomicAdd(reinterpret_cast<unsigned long long *>(&stats[0]), (unsigned long long)my_rows);
        atomicAdd(reinterpret_cast<unsigned long long *>(&stats[1]), (unsigned long long)my_nnz);
        atomicAdd(reinterpret_cast<unsigned long long *>(&stats[2]), (unsigned long long)my_tok_nnz);
    }
}

size_t theta_smem_bytes(int k) {
    return ((size_t)k + (size_t)kThetaWarps * (size_t)((k >> 1) + (k >> 5))) * sizeof(uint32_t);
}

int theta_blocks_per_sm(int k) {
    const size_t smem = theta_smem_bytes(k);
    if (smem > 48 * 1024)
        cudaFuncSetAttribute(theta_rebuild_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, theta_rebuild_kernel, kThetaWarps * 32, smem) !=
        cudaSuccess)
        return 0;
    return n;
}

cudaError_t launch_theta_rebuild(int k, int num_docs, const int64_t *doc_ptr, const int32_t *doc_tok,
                                 const uint16_t *topics, const int32_t *doc_order, int2 *rows, uint32_t *theta,
                                 int32_t *nk, int64_t *stats, int32_t *error, int grid, cudaStream_t s) {
    const size_t smem = theta_smem_bytes(k);
    cudaError_t e = allow_smem(reinterpret_cast<const void *>(&theta_rebuild_kernel), smem, s);
    if (e != cudaSuccess) return e;
    theta_rebuild_kernel<<<grid, kThetaWarps * 32, smem, s>>>(k, num_docs, doc_ptr, doc_tok, topics, doc_order, rows,
                                                              theta, nk, stats, error);
    return cudaGetLastError();
}

// ------------------------------------------------------------ init topics
__global__ void init_topics_kernel(int64_t n, int k, uint64_t seed, uint16_t *z) {
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
        z[t] = (uint16_t)bounded_from_bits(philox_token(seed, (uint64_t)t, 0u, kPurposeInit), (uint32_t)k);
}

cudaError_t launch_init_topics(int64_t n, int k, uint64_t seed, uint16_t *z, cudaStream_t s) {
    int blocks = (int)std::min<int64_t>((n + 255) / 256, 148 * 32);
    if (blocks < 1) blocks = 1;
    init_topics_kernel<<<blocks, 256, 0, s>>>(n, k, seed, z);
    return cudaGetLastError();
}

// ------------------------------------------------------ doc id validation
__global__ void doc_check_kernel(int64_t n, int num_docs, const int32_t *__restrict__ doc_ids, int32_t *doc_count,
                                 int32_t *error) {
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        const int d = doc_ids[t];
        if ((unsigned)d < (unsigned)num_docs)
            atomicAdd(&doc_count[d], 1);
        else
            atomicOr(error, kErrDocRange);
    }
}

cudaError_t launch_doc_check(int64_t n, int num_docs, const int32_t *doc_ids, int32_t *doc_count, int32_t *error,
                             cudaStream_t s) {
    int blocks = (int)std::min<int64_t>((n + 255) / 256, 148 * 32);
    if (blocks < 1) blocks = 1;
    doc_check_kernel<<<blocks, 256, 0, s>>>(n, num_docs, doc_ids, doc_count, error);
    return cudaGetLastError();
}

// ------------------------------------------------------- dense phi (API)
// CTA per word (grid-stride): shared-memory histogram of the word's topics,
// one coalesced row store, n_k accumulated per CTA and added once at the end.
__global__ void __launch_bounds__(256) update_phi_kernel(int K, int V, const int64_t *__restrict__ word_ptr,
                                                         const uint16_t *__restrict__ topics, int32_t *phi,
                                                         int32_t *nk, int32_t *error) {
    extern __shared__ int sm_i32[];
    int *hist = sm_i32, *acc = sm_i32 + K;
    for (int j = threadIdx.x; j < K; j += blockDim.x) acc[j] = 0;
    for (int w = blockIdx.x; w < V; w += gridDim.x) {
        for (int j = threadIdx.x; j < K; j += blockDim.x) hist[j] = 0;
        __syncthreads();
        for (int64_t t = word_ptr[w] + threadIdx.x; t < word_ptr[w + 1]; t += blockDim.x) {
            const uint32_t z = topics[t];
            if (z < (uint32_t)K)
                atomicAdd(&hist[z], 1);
            else if (error)
                atomicOr(error, kErrTopicRange);
        }
        __syncthreads();
        int32_t *row = phi + (size_t)w * K;
        for (int j = threadIdx.x; j < K; j += blockDim.x) {
            row[j] = hist[j];
            acc[j] += hist[j];
        }
        __syncthreads();
    }
    for (int j = threadIdx.x; j < K; j += blockDim.x)
        if (acc[j]) atomicAdd(&nk[j], acc[j]);
}

cudaError_t launch_update_phi(int k, int num_words, const int64_t *word_ptr, const uint16_t *topics, int32_t *phi,
                              int32_t *nk, int32_t *error, cudaStream_t s) {
    const size_t smem = (size_t)2 * k * sizeof(int);
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(update_phi_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    int dev = 0;
    cudaGetDevice(&dev);
    const int grid = std::max(1, std::min(num_words, num_sms(dev) * 4));
    update_phi_kernel<<<grid, 256, smem, s>>>(k, num_words, word_ptr, topics, phi, nk, error);
    return cudaGetLastError();
}

// phi_head = (phi + beta) / (n_k + beta * V), the reference's float quotient
// (lda_phi_kernel.cu:26) kept in FP32.
__global__ void phi_head_kernel(int K, float beta, int V, const int32_t *__restrict__ phi,
                                const int32_t *__restrict__ nk, float *out) {
    const int64_t total = (int64_t)K * V;
    const float vb = beta * (float)V;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const int k = (int)(i % K);
        out[i] = __fdiv_rn((float)phi[i] + beta, (float)nk[k] + vb);
    }
}

cudaError_t launch_phi_head(int k, float beta, int num_words, const int32_t *phi, const int32_t *nk, float *out,
                            cudaStream_t s) {
    int dev = 0;
    cudaGetDevice(&dev);
    phi_head_kernel<<<num_sms(dev) * 8, 256, 0, s>>>(k, beta, num_words, phi, nk, out);
    return cudaGetLastError();
}

// ---------------------------------------------------- joint log-likelihood
// Per-CTA FP64 partial sums (fixed word/doc assignment, so the result is
// reproducible):  sum_{w,k: n>0} [lgamma(n_wk + beta) - lgamma(beta)]
//               + sum_{d,k: n>0} [lgamma(n_dk + alpha) - lgamma(alpha)] - sum_d lgamma(L_d + K alpha).
__global__ void __launch_bounds__(256) loglik_joint_kernel(int K, int V, int D, double alpha, double beta,
                                                           const int64_t *__restrict__ word_ptr,
                                                           const uint16_t *__restrict__ topics,
                                                           const int2 *__restrict__ rows,
                                                           const uint32_t *__restrict__ theta,
                                                           const int64_t *__restrict__ doc_ptr, double *partials,
                                                           int32_t *error) {
    extern __shared__ int hist_j[];
    __shared__ double red[256];
    const double lg_b = lgamma(beta), lg_a = lgamma(alpha), ka = (double)K * alpha;
    double s = 0.0, c = 0.0;
    auto add = [&](double x) {
        const double t = s + x;
        if (fabs(s) >= fabs(x))
            c += (s - t) + x;
        else
            c += (x - t) + s;
        s = t;
    };
    for (int w = blockIdx.x; w < V; w += gridDim.x) {
        for (int j = threadIdx.x; j < K; j += blockDim.x) hist_j[j] = 0;
        __syncthreads();
        for (int64_t t = word_ptr[w] + threadIdx.x; t < word_ptr[w + 1]; t += blockDim.x) {
            const uint32_t z = topics[t];
            if (z < (uint32_t)K)
                atomicAdd(&hist_j[z], 1);
            else
                atomicOr(error, kErrTopicRange);
        }
        __syncthreads();
        for (int j = threadIdx.x; j < K; j += blockDim.x)
            if (hist_j[j] > 0) add(lgamma((double)hist_j[j] + beta) - lg_b);
        __syncthreads();
    }
    for (int d = blockIdx.x; d < D; d += gridDim.x) {
        const int2 r = rows[d];
        for (int i = r.x + threadIdx.x; i < r.y; i += blockDim.x) {
            const uint32_t e = theta[i];
            if (e >> 16) add(lgamma((double)(e >> 16) + alpha) - lg_a);
        }
        if (threadIdx.x == 0) add(-lgamma((double)(doc_ptr[d + 1] - doc_ptr[d]) + ka));
    }
    red[threadIdx.x] = s + c;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) partials[blockIdx.x] = red[0];
}

cudaError_t launch_loglik_joint(int k, int num_words, int num_docs, float alpha, float beta, const int64_t *word_ptr,
                                const uint16_t *topics, const int2 *rows, const uint32_t *theta,
                                const int64_t *doc_ptr, const int32_t *nk, double *partials, int num_partials,
                                int32_t *error, cudaStream_t s) {
    (void)nk;
    const size_t smem = (size_t)k * sizeof(int);
    if (smem > 48 * 1024) {
        cudaError_t e =
            cudaFuncSetAttribute(loglik_joint_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    loglik_joint_kernel<<<num_partials, 256, smem, s>>>(k, num_words, num_docs, (double)alpha, (double)beta, word_ptr,
                                                        topics, rows, theta, doc_ptr, partials, error);
    return cudaGetLastError();
}

int num_sms(int device) {
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, device) != cudaSuccess || n <= 0) n = 148;
    return n;
}

}  // namespace culda

// ===================================================== kernel-level C API
using namespace culda;

static int cuda_status(cudaError_t e) {
    if (e == cudaSuccess) return CULDA_OK;
    set_global_error("CUDA error: %s", cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? CULDA_ERR_OOM : CULDA_ERR_CUDA;
}

static bool valid_k(int32_t k) { return k >= 32 && k <= 4096 && (k % 32) == 0; }

extern "C" int culda_update_phi(int32_t k, int32_t num_words, const int64_t *d_word_ptr, const uint16_t *d_topics,
                                int32_t *d_phi, int32_t *d_nk, void *stream) {
    if (!valid_k(k) || num_words <= 0 || !d_word_ptr || !d_topics || !d_phi || !d_nk) {
        set_global_error("culda_update_phi: invalid argument");
        return CULDA_ERR_INVALID_ARG;
    }
    cudaStream_t s = (cudaStream_t)stream;
    int rc = cuda_status(cudaMemsetAsync(d_nk, 0, sizeof(int32_t) * (size_t)k, s));
    if (rc) return rc;
    // topics outside [0, K) are skipped; the caller validates its topic array
    return cuda_status(launch_update_phi(k, num_words, d_word_ptr, d_topics, d_phi, d_nk, nullptr, s));
}

extern "C" int culda_compute_phi_head(int32_t k, float beta, int32_t num_words, const int32_t *d_phi,
                                      const int32_t *d_nk, float *d_phi_head, void *stream) {
    if (!valid_k(k) || num_words <= 0 || !d_phi || !d_nk || !d_phi_head) {
        set_global_error("culda_compute_phi_head: invalid argument");
        return CULDA_ERR_INVALID_ARG;
    }
    return cuda_status(launch_phi_head(k, beta, num_words, d_phi, d_nk, d_phi_head, (cudaStream_t)stream));
}

extern "C" size_t culda_update_theta_workspace(int32_t k, int32_t num_docs) {
    (void)k;
    (void)num_docs;
    return 256;  // the device error word
}

extern "C" int culda_update_theta(int32_t k, int32_t num_docs, const int64_t *d_doc_ptr, const int32_t *d_doc_tok,
                                  const uint16_t *d_topics, const int32_t *d_doc_order, int32_t *d_theta_rows,
                                  uint32_t *d_theta, int32_t *d_nk, int64_t *d_stats, void *d_workspace,
                                  size_t workspace_bytes, void *stream) {
    if (!valid_k(k) || num_docs <= 0 || !d_doc_ptr || !d_doc_tok || !d_topics || !d_theta_rows || !d_theta ||
        !d_workspace || workspace_bytes < culda_update_theta_workspace(k, num_docs)) {
        set_global_error("culda_update_theta: invalid argument");
        return CULDA_ERR_INVALID_ARG;
    }
    cudaStream_t s = (cudaStream_t)stream;
    int32_t *err = (int32_t *)d_workspace;
    int rc = cuda_status(cudaMemsetAsync(err, 0, sizeof(int32_t), s));
    if (!rc && d_nk) rc = cuda_status(cudaMemsetAsync(d_nk, 0, sizeof(int32_t) * (size_t)k, s));
    if (!rc && d_stats) rc = cuda_status(cudaMemsetAsync(d_stats, 0, 3 * sizeof(int64_t), s));
    if (rc) return rc;
    int dev = 0;
    cudaGetDevice(&dev);
    int bps = theta_blocks_per_sm(k);
    if (bps <= 0) bps = 1;
    const int grid = std::max(1, std::min(num_sms(dev) * bps, (num_docs + kThetaWarps - 1) / kThetaWarps));
    return cuda_status(launch_theta_rebuild(k, num_docs, d_doc_ptr, d_doc_tok, d_topics, d_doc_order,
                                            reinterpret_cast<int2 *>(d_theta_rows), d_theta, d_nk, d_stats, err,
                                            grid, s));
}

extern "C" size_t culda_sample_workspace(int32_t k, int32_t num_items, int32_t num_hot) {
    // [counter:256][item_ll: 8*num_items rounded][hot rows: 4*K*num_hot]
    size_t a = 256;
    a += ((size_t)num_items * sizeof(double) + 255) / 256 * 256;
    a += (size_t)num_hot * (size_t)k * sizeof(int32_t);
    return a;
}

extern "C" int culda_sample(const culda_sample_args *a, void *d_workspace, size_t workspace_bytes, void *stream) {
    if (!a || !valid_k(a->k) || a->num_docs <= 0 || a->num_words <= 0 || a->num_tokens <= 0 || !a->word_ptr ||
        !a->doc_ids || !a->topics_in || !a->topics_out || a->topics_in == a->topics_out || !a->theta ||
        !a->theta_rows || !a->nk || !a->items || a->num_items <= 0 || !a->loglik_sum || !d_workspace ||
        (a->num_hot > 0 && (!a->hot_items || a->num_hot_items <= 0)) || a->theta_capacity <= 0 ||
        workspace_bytes < culda_sample_workspace(a->k, a->num_items, a->num_hot) ||
        (a->group_lanes != 1 && a->group_lanes != 2 && a->group_lanes != 4 && a->group_lanes != 8 &&
         a->group_lanes != 16 && a->group_lanes != 32) ||
        ((uintptr_t)a->theta & 15u)) {
        set_global_error("culda_sample: invalid argument");
        return CULDA_ERR_INVALID_ARG;
    }
    cudaStream_t s = (cudaStream_t)stream;
    char *ws = (char *)d_workspace;
    int32_t *counter = (int32_t *)ws;
    double *item_ll = (double *)(ws + 256);
    int32_t *hot_phi = (int32_t *)(ws + 256 + ((size_t)a->num_items * sizeof(double) + 255) / 256 * 256);
    int rc = cuda_status(cudaMemsetAsync(counter, 0, 256, s));
    if (rc) return rc;
    if (a->num_hot > 0) {
        rc = cuda_status(cudaMemsetAsync(hot_phi, 0, (size_t)a->num_hot * a->k * sizeof(int32_t), s));
        if (!rc)
            rc = cuda_status(launch_hot_rows(a->k, a->hot_items, a->num_hot_items, a->topics_in, hot_phi,
                                             a->error ? a->error : counter + 1, s));
        if (rc) return rc;
    }
    SampleParams p{};
    p.k = a->k;
    p.alpha = a->alpha;
    p.beta = a->beta;
    p.vbeta = a->beta * (float)a->num_words;
    p.num_docs = a->num_docs;
    p.num_items = a->num_items;
    p.num_hot = a->num_hot;
    p.num_tokens = a->num_tokens;
    p.theta_cap = a->theta_capacity;
    p.doc_ids = a->doc_ids;
    p.topics_in = a->topics_in;
    p.topics_out = a->topics_out;
    p.theta = a->theta;
    p.rows = reinterpret_cast<const int2 *>(a->theta_rows);
    p.nk = a->nk;
    p.items = a->items;
    p.hot_phi = hot_phi;
    p.item_counter = counter;
    p.item_ll = item_ll;
    p.seed = a->seed;
    p.iteration = a->iteration;
    p.iteration_ptr = nullptr;
    p.error = a->error ? a->error : counter + 1;
    int dev = 0;
    cudaGetDevice(&dev);
    int bps = sample_blocks_per_sm(a->k, a->group_lanes);
    if (bps <= 0) bps = 1;
    const int grid = std::max(1, std::min(a->num_items, num_sms(dev) * bps));
    rc = cuda_status(launch_sample(p, a->group_lanes, grid, s));
    if (rc) return rc;
    // fold the per-item sums into the caller's accumulator
    DevStats *st = (DevStats *)(counter + 8);
    rc = cuda_status(launch_finalize_ll(item_ll, a->num_items, st, nullptr, s));
    if (rc) return rc;
    return cuda_status(cudaMemcpyAsync(a->loglik_sum, &st->ll_sum, sizeof(double), cudaMemcpyDeviceToDevice, s));
}

extern "C" int culda_loglik(const double *d_loglik_sum, double doc_term, int64_t num_tokens, double *loglik,
                            void *stream) {
    if (!d_loglik_sum || !loglik || num_tokens <= 0) return CULDA_ERR_INVALID_ARG;
    double sum = 0;
    cudaStream_t s = (cudaStream_t)stream;
    int rc = cuda_status(cudaMemcpyAsync(&sum, d_loglik_sum, sizeof(double), cudaMemcpyDeviceToHost, s));
    if (!rc) rc = cuda_status(cudaStreamSynchronize(s));
    if (rc) return rc;
    *loglik = (sum - doc_term) / (double)num_tokens;
    return CULDA_OK;
}
