// kernels.cu — the count-rebuild and utility kernels of the one-GPU CGS
// iteration, and the kernel-level C entry points that mirror the reference's
// kernel APIs.  The sampler is in sampler.cu.
//
// Iteration data flow (all resident in HBM; tokens stored word by word, and
// inside a word ordered by their doc's length so neighbouring tokens walk
// theta rows of similar length):
//   uniforms_kernel      one Philox4x32-10 uniform per token
//   hot_rows_kernel      full phi rows of words split over several work items
//   sample_kernel<G>     the draw (sampler.cu)
//   finalize_ll_kernel   fixed-order sum of the per-item log terms
//   theta_rebuild_kernel block per long doc, warp per other doc (longest
//                        first): 16-bit shared-memory histogram of the doc's
//                        new topics (docs of at most 32 tokens: match groups
//                        in registers), CSR compaction in ascending topic,
//                        zero padding, n_k as a column sum.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>

#include "device_util.cuh"
#include "kernels.cuh"
#include "philox.h"

namespace culda {

// ---------------------------------------------------------- theta rebuild
// Two bins in one persistent launch.  The longest documents (the first
// num_long of doc_order, every one at least the bin threshold long) are taken
// one at a time by a whole CTA from an atomic queue: its eight warps count
// the doc's tokens into one shared histogram.  Every other document is taken
// by one warp (static round robin over the rest of doc_order, longest first).
// Shared memory per warp: K/2 words of packed 16-bit counts (a topic can hold
// at most L_d <= 65535 tokens, so a low half never carries into the high half)
// and K/32 words of a non-zero mask; per block: K n_k partial counts.  The
// block bin uses warp 0's histogram.  The compaction walks the mask in
// ascending topic order, so each row comes out sorted as
// lda_theta_kernel.cu:58-85 leaves it, and only the touched count words are
// cleared again.

namespace {

// Counts tokens [b + first, e) with stride `step` into the packed histogram.
__device__ __forceinline__ void theta_count(int K, int64_t b, int64_t e, int first, int step,
                                            const int32_t *__restrict__ doc_tok,
                                            const uint16_t *__restrict__ topics, uint32_t *cnt, uint32_t *mask,
                                            int32_t *error) {
    // eight tokens per thread in flight: the index loads, then the topic
    // loads they address, then the histogram updates
    constexpr int kInFlight = 8;
    for (int64_t j0 = b + first; j0 < e; j0 += (int64_t)step * kInFlight) {
        int32_t idx[kInFlight];
        uint32_t zz[kInFlight];
#pragma unroll
        for (int u = 0; u < kInFlight; ++u) idx[u] = j0 + (int64_t)step * u < e ? doc_tok[j0 + (int64_t)step * u] : -1;
#pragma unroll
        for (int u = 0; u < kInFlight; ++u) zz[u] = idx[u] >= 0 ? (uint32_t)topics[idx[u]] : 0u;
#pragma unroll
        for (int u = 0; u < kInFlight; ++u) {
            if (idx[u] < 0) continue;
            const uint32_t z = zz[u];
            if (z >= (uint32_t)K) {
                atomicOr(error, kErrTopicRange);
                continue;
            }
            const uint32_t sh = (z & 1u) << 4;
            const uint32_t old = atomicAdd(&cnt[z >> 1], 1u << sh);
            if (((old >> sh) & 0xFFFFu) == 0u) atomicOr(&mask[z >> 5], 1u << (z & 31u));
        }
    }
}

// One warp: the doc's row from its histogram (ascending topic), zero padding
// to the row's previous end, the histogram cleared, n_k partial sums.
__device__ __forceinline__ void theta_compact(int K, int d, int64_t len, int lane, uint32_t *cnt, uint32_t *mask,
                                              uint32_t *nk_acc, int2 *rows, ThetaEntry *theta, int64_t &my_rows,
                                              int64_t &my_nnz, int64_t &my_tok_nnz) {
    const int mwords = K >> 5;
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
            theta[pos++] = theta_entry(z, c);
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
        my_rows += len * (int64_t)(new_end - start);
        my_nnz += nnz;
        my_tok_nnz += len * (int64_t)nnz;
    }
}

// One warp, a doc of at most 32 tokens: no histogram.  Each lane holds one
// token's topic; the lanes with equal topics form a match group whose lowest
// lane writes the entry (topic, group size) at its rank among the groups'
// topics, so the row comes out in ascending topic order as theta_compact
// leaves it.
__device__ __forceinline__ void theta_short(int K, int d, int64_t b, int len, int lane,
                                            const int32_t *__restrict__ doc_tok,
                                            const uint16_t *__restrict__ topics, uint32_t *nk_acc, int2 *rows,
                                            ThetaEntry *theta, int64_t &my_rows, int64_t &my_nnz,
                                            int64_t &my_tok_nnz, int32_t *error) {
    uint32_t z = 0xFFFFFFFFu;
    if (lane < len) {
        const uint32_t t = topics[doc_tok[b + lane]];
        if (t < (uint32_t)K)
            z = t;
        else
            atomicOr(error, kErrTopicRange);
    }
    const unsigned grp = __match_any_sync(0xffffffffu, z);
    const bool lead = z != 0xFFFFFFFFu && __ffs(grp) - 1 == lane;
    const int nnz = __popc(__ballot_sync(0xffffffffu, lead));
    const uint32_t key = lead ? z : 0xFFFFFFFFu;
    int rank = 0;
#pragma unroll 8
    for (int j = 0; j < 32; ++j) rank += __shfl_sync(0xffffffffu, key, j) < key;
    const int2 row = rows[d];
    const int start = row.x, old_end = row.y;
    if (lead) {
        const uint32_t c = (uint32_t)__popc(grp);
        theta[start + rank] = theta_entry(z, c);
        atomicAdd(&nk_acc[z], c);
    }
    const int new_end = start + ((nnz + 31) & ~31);
    const int zend = max(new_end, old_end);
    for (int j = start + nnz + lane; j < zend; j += 32) theta[j] = 0u;
    if (lane == 0) {
        rows[d].y = new_end;
        my_rows += (int64_t)len * (new_end - start);
        my_nnz += nnz;
        my_tok_nnz += (int64_t)len * nnz;
    }
}

}  // namespace

__global__ void __launch_bounds__(kThetaWarps * 32) theta_rebuild_kernel(
    int K, int num_docs, const int64_t *__restrict__ doc_ptr, const int32_t *__restrict__ doc_tok,
    const uint16_t *__restrict__ topics, const int32_t *__restrict__ doc_order, int num_long, int32_t *long_queue,
    int2 *rows, ThetaEntry *theta, int32_t *nk, int64_t *stats, int32_t *error) {
    extern __shared__ uint32_t sm_u32[];
    __shared__ int s_next;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int cwords = K >> 1, mwords = K >> 5;
    uint32_t *nk_acc = sm_u32;
    uint32_t *cnt = sm_u32 + K + warp * (cwords + mwords);
    uint32_t *mask = cnt + cwords;
    for (int i = threadIdx.x; i < K; i += blockDim.x) nk_acc[i] = 0u;
    for (int i = lane; i < cwords + mwords; i += 32) cnt[i] = 0u;
    __syncthreads();

    int64_t my_rows = 0, my_nnz = 0, my_tok_nnz = 0;
    // block bin: one long document per CTA at a time
    if (num_long > 0) {
        uint32_t *bcnt = sm_u32 + K;  // warp 0's histogram
        uint32_t *bmask = bcnt + cwords;
        for (;;) {
            if (threadIdx.x == 0) s_next = atomicAdd(long_queue, 1);
            __syncthreads();
            const int i = s_next;
            __syncthreads();  // every thread has read s_next before thread 0 overwrites it
            if (i >= num_long) break;
            const int d = doc_order[i];
            const int64_t b = doc_ptr[d], e = doc_ptr[d + 1];
            if (e - b > 65535) {
                if (threadIdx.x == 0) atomicOr(error, kErrLongDoc);
                continue;
            }
            theta_count(K, b, e, threadIdx.x, kThetaWarps * 32, doc_tok, topics, bcnt, bmask, error);
            __syncthreads();
            if (warp == 0) theta_compact(K, d, e - b, lane, bcnt, bmask, nk_acc, rows, theta, my_rows, my_nnz,
                                         my_tok_nnz);
            __syncthreads();  // the histogram is clear again before the next document
        }
    }
    // warp bin: the remaining documents, one per warp
    const int nw = gridDim.x * kThetaWarps;
    for (int i = num_long + blockIdx.x * kThetaWarps + warp; i < num_docs; i += nw) {
        const int d = doc_order ? doc_order[i] : i;
        const int64_t b = doc_ptr[d], e = doc_ptr[d + 1];
        if (e - b > 65535) {
            if (lane == 0) atomicOr(error, kErrLongDoc);
            continue;
        }
        if (e - b <= 32) {
            theta_short(K, d, b, (int)(e - b), lane, doc_tok, topics, nk_acc, rows, theta, my_rows, my_nnz,
                        my_tok_nnz, error);
            continue;
        }
        theta_count(K, b, e, lane, 32, doc_tok, topics, cnt, mask, error);
        __syncwarp();
        theta_compact(K, d, e - b, lane, cnt, mask, nk_acc, rows, theta, my_rows, my_nnz, my_tok_nnz);
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
    if (allow_smem(reinterpret_cast<const void *>(&theta_rebuild_kernel), smem, nullptr) != cudaSuccess) return 0;
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, theta_rebuild_kernel, kThetaWarps * 32, smem) !=
        cudaSuccess)
        return 0;
    return n;
}

cudaError_t launch_theta_rebuild(int k, int num_docs, const int64_t *doc_ptr, const int32_t *doc_tok,
                                 const uint16_t *topics, const int32_t *doc_order, int2 *rows, ThetaEntry *theta,
                                 int32_t *nk, int64_t *stats, int32_t *error, int grid, cudaStream_t s,
                                 int num_long, int32_t *long_queue) {
    if (num_long > 0 && (!doc_order || !long_queue || num_long > num_docs)) return cudaErrorInvalidValue;
    const size_t smem = theta_smem_bytes(k);
    cudaError_t e = allow_smem(reinterpret_cast<const void *>(&theta_rebuild_kernel), smem, s);
    if (e != cudaSuccess) return e;
    if (num_long > 0) {
        e = cudaMemsetAsync(long_queue, 0, sizeof(int32_t), s);
        if (e != cudaSuccess) return e;
    }
    theta_rebuild_kernel<<<grid, kThetaWarps * 32, smem, s>>>(k, num_docs, doc_ptr, doc_tok, topics, doc_order,
                                                              num_long > 0 ? num_long : 0, long_queue, rows, theta,
                                                              nk, stats, error);
    return cudaGetLastError();
}

// -------------------------------------------------------- small utilities

// z[i] = floor(x0 * K / 2^32), x0 = Philox(seed, {t, 0, 1}) with t the
// token's word-major index.
__global__ void init_topics_kernel(int64_t n, int k, uint64_t seed, const int32_t *__restrict__ tok_index,
                                   uint16_t *z) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t t = tok_index ? (uint64_t)tok_index[i] : (uint64_t)i;
        z[i] = (uint16_t)bounded_from_bits(philox_token(seed, t, 0u, kPurposeInit), (uint32_t)k);
    }
}

cudaError_t launch_init_topics(int64_t n, int k, uint64_t seed, const int32_t *tok_index, uint16_t *z,
                               cudaStream_t s) {
    init_topics_kernel<<<grid_for(n), 256, 0, s>>>(n, k, seed, tok_index, z);
    return cudaGetLastError();
}

// One Philox4x32-10 block per token, computed by all threads in parallel
// (the sampler's groups would otherwise leave most lanes idle while a
// segment's one or two tokens draw theirs).
__global__ void uniforms_kernel(int64_t n, uint64_t seed, const uint32_t *__restrict__ iteration_dev,
                                uint32_t iteration, const int32_t *__restrict__ tok_index, float *u) {
    const uint32_t iter = iteration_dev ? *iteration_dev : iteration;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t t = tok_index ? (uint64_t)tok_index[i] : (uint64_t)i;
        u[i] = uniform_from_bits(philox_token(seed, t, iter, kPurposeSample));
    }
}

cudaError_t launch_uniforms(int64_t n, uint64_t seed, const uint32_t *iteration_dev, uint32_t iteration,
                            const int32_t *tok_index, float *u, cudaStream_t s) {
    uniforms_kernel<<<grid_for(n), 256, 0, s>>>(n, seed, iteration_dev, iteration, tok_index, u);
    return cudaGetLastError();
}

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
    doc_check_kernel<<<grid_for(n), 256, 0, s>>>(n, num_docs, doc_ids, doc_count, error);
    return cudaGetLastError();
}

__global__ void check_topics_kernel(int64_t n, int k, const uint16_t *__restrict__ z, int32_t *error) {
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
        if (z[t] >= (uint32_t)k) atomicOr(error, kErrTopicRange);
}

cudaError_t launch_check_topics(int64_t n, int k, const uint16_t *z, int32_t *error, cudaStream_t s) {
    check_topics_kernel<<<grid_for(n), 256, 0, s>>>(n, k, z, error);
    return cudaGetLastError();
}

// Thread per token: the word is found by binary search of word_ptr (V+1
// ascending offsets, L2-resident), so a Zipf-head word of millions of tokens
// is spread over the whole grid instead of one warp.
__global__ void order_keys_kernel(int num_words, int64_t num_tokens, const int64_t *__restrict__ word_ptr,
                                  const int32_t *__restrict__ doc_ids, const int64_t *__restrict__ doc_ptr,
                                  uint64_t *keys) {
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < num_tokens;
         t += (int64_t)gridDim.x * blockDim.x) {
        int lo = 0, hi = num_words - 1;  // the last word w with word_ptr[w] <= t
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (__ldg(word_ptr + mid) <= t)
                lo = mid;
            else
                hi = mid - 1;
        }
        const int d = doc_ids[t];
        const int64_t len = min(doc_ptr[d + 1] - doc_ptr[d], (int64_t)65535);
        keys[t] = ((uint64_t)lo << 16) | (uint64_t)(65535 - len);
    }
}

cudaError_t launch_order_keys(int num_words, int64_t num_tokens, const int64_t *word_ptr, const int32_t *doc_ids,
                              const int64_t *doc_ptr, uint64_t *keys, cudaStream_t s) {
    if (num_tokens <= 0) return cudaSuccess;
    order_keys_kernel<<<grid_for(num_tokens), 256, 0, s>>>(num_words, num_tokens, word_ptr, doc_ids, doc_ptr, keys);
    return cudaGetLastError();
}

// 32-bit keys for vocabularies of at most 2^24 words: the word above an 8-bit
// log-linear length class, 16 classes per doubling (the position of the
// length's leading one and the 4 bits after it), longest first.  Docs in one
// class keep their input order (the sort is stable), so a doc's tokens inside
// a word stay contiguous.
__global__ void order_keys32_kernel(int num_words, int64_t num_tokens, const int64_t *__restrict__ word_ptr,
                                    const int32_t *__restrict__ doc_ids, const int64_t *__restrict__ doc_ptr,
                                    uint32_t *keys) {
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < num_tokens;
         t += (int64_t)gridDim.x * blockDim.x) {
        int lo = 0, hi = num_words - 1;  // the last word w with word_ptr[w] <= t
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (__ldg(word_ptr + mid) <= t)
                lo = mid;
            else
                hi = mid - 1;
        }
        const int d = doc_ids[t];
        const int64_t l64 = doc_ptr[d + 1] - doc_ptr[d];
        const uint32_t len = l64 < 1 ? 1u : l64 > 65535 ? 65535u : (uint32_t)l64;
        const uint32_t msb = 31u - __clz(len);                         // 0 .. 15
        const uint32_t frac = ((len << (31u - msb)) >> 27) & 15u;      // the 4 bits after the leading one
        keys[t] = ((uint32_t)lo << 8) | (255u - (msb * 16u + frac));
    }
}

cudaError_t launch_order_keys32(int num_words, int64_t num_tokens, const int64_t *word_ptr, const int32_t *doc_ids,
                                const int64_t *doc_ptr, uint32_t *keys, cudaStream_t s) {
    if (num_tokens <= 0) return cudaSuccess;
    if (num_words > (1 << 24)) return cudaErrorInvalidValue;
    order_keys32_kernel<<<grid_for(num_tokens), 256, 0, s>>>(num_words, num_tokens, word_ptr, doc_ids, doc_ptr,
                                                             keys);
    return cudaGetLastError();
}

template <class T>
__global__ void gather_kernel(int64_t n, const int32_t *__restrict__ index, const T *__restrict__ src, T *dst) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        dst[i] = src[index[i]];
}

template <class T>
__global__ void scatter_kernel(int64_t n, const int32_t *__restrict__ index, const T *__restrict__ src, T *dst) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        dst[index[i]] = src[i];
}

template <class T>
cudaError_t launch_gather(int64_t n, const int32_t *index, const T *src, T *dst, cudaStream_t s) {
    gather_kernel<T><<<grid_for(n), 256, 0, s>>>(n, index, src, dst);
    return cudaGetLastError();
}

template <class T>
cudaError_t launch_scatter(int64_t n, const int32_t *index, const T *src, T *dst, cudaStream_t s) {
    scatter_kernel<T><<<grid_for(n), 256, 0, s>>>(n, index, src, dst);
    return cudaGetLastError();
}

template cudaError_t launch_gather<int32_t>(int64_t, const int32_t *, const int32_t *, int32_t *, cudaStream_t);
template cudaError_t launch_gather<uint16_t>(int64_t, const int32_t *, const uint16_t *, uint16_t *, cudaStream_t);
template cudaError_t launch_scatter<uint16_t>(int64_t, const int32_t *, const uint16_t *, uint16_t *, cudaStream_t);

__global__ void iota_kernel(int64_t n, int32_t *v) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        v[i] = (int32_t)i;
}

cudaError_t launch_iota(int64_t n, int32_t *v, cudaStream_t s) {
    iota_kernel<<<grid_for(n), 256, 0, s>>>(n, v);
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
    cudaError_t e = allow_smem(reinterpret_cast<const void *>(&update_phi_kernel), smem, s);
    if (e != cudaSuccess) return e;
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
                                                           const ThetaEntry *__restrict__ theta,
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
            const uint32_t cnt = theta[i] & 0xFFFFu;
            if (cnt > 0u) add(lgamma((double)cnt + alpha) - lg_a);
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
                                const uint16_t *topics, const int2 *rows, const ThetaEntry *theta,
                                const int64_t *doc_ptr, double *partials, int num_partials, int32_t *error,
                                cudaStream_t s) {
    const size_t smem = (size_t)k * sizeof(int);
    cudaError_t e = allow_smem(reinterpret_cast<const void *>(&loglik_joint_kernel), smem, s);
    if (e != cudaSuccess) return e;
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
        !d_workspace || workspace_bytes < culda_update_theta_workspace(k, num_docs) || ((uintptr_t)d_theta & 15u)) {
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
                                            reinterpret_cast<int2 *>(d_theta_rows),
                                            reinterpret_cast<ThetaEntry *>(d_theta), d_nk, d_stats, err, grid, s));
}

extern "C" size_t culda_sample_workspace(int32_t k, int32_t num_items, int32_t num_hot) {
    // [counter, error, stats: 256][item_ll: 8*num_items rounded][hot rows: 4*K*num_hot]
    size_t a = 256;
    a += ((size_t)num_items * sizeof(double) + 255) / 256 * 256;
    a += (size_t)num_hot * (size_t)k * sizeof(int32_t);
    return a;
}

extern "C" int culda_sample(const culda_sample_args *a, void *d_workspace, size_t workspace_bytes, void *stream) {
    if (!a || !valid_k(a->k) || a->num_docs <= 0 || a->num_words <= 0 || a->num_tokens <= 0 || !a->word_ptr ||
        !a->doc_ids || !a->topics_in || !a->topics_out || a->topics_in == a->topics_out || !a->theta ||
        !a->theta_rows || !a->nk || !a->items || a->num_items <= 0 || !a->seg_start || a->num_segs <= 0 ||
        !a->loglik_sum || !d_workspace ||
        a->num_hot < 0 || (a->num_hot > 0 && (!a->hot_items || a->num_hot_items <= 0)) || a->theta_capacity <= 0 ||
        workspace_bytes < culda_sample_workspace(a->k, a->num_items, a->num_hot) ||
        (a->group_lanes != kFlatLanes && a->group_lanes != 1 && a->group_lanes != 2 && a->group_lanes != 4 &&
         a->group_lanes != 8 && a->group_lanes != 16 && a->group_lanes != 32) ||
        ((uintptr_t)a->theta & 31u)) {
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
    // the sampler indexes shared memory with each entry's topic: reject a
    // theta array whose rows or topics are out of range before launching it
    {
        int32_t *flag = counter + 2, bad = 0;
        rc = cuda_status(launch_check_theta(a->num_docs, a->k, reinterpret_cast<const int2 *>(a->theta_rows),
                                            reinterpret_cast<const ThetaEntry *>(a->theta), a->theta_capacity, flag,
                                            s));
        if (!rc) rc = cuda_status(cudaMemcpyAsync(&bad, flag, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
        if (!rc) rc = cuda_status(cudaStreamSynchronize(s));
        if (rc) return rc;
        if (bad) {
            set_global_error("culda_sample: theta rows or topics out of range (flags 0x%x)", bad);
            return CULDA_ERR_INVALID_ARG;
        }
    }
    if (a->num_hot > 0) {
        rc = cuda_status(cudaMemsetAsync(hot_phi, 0, (size_t)a->num_hot * a->k * sizeof(int32_t), s));
        if (!rc)
            rc = cuda_status(launch_hot_rows(a->k, a->hot_items, a->num_hot_items, a->topics_in, hot_phi,
                                             a->error ? a->error : counter + 1, s));
        if (rc) return rc;
    }
    SampleParams p{};
    p.k = a->k;
    p.kmask = pow2_ceil(a->k) - 1;
    p.alpha = a->alpha;
    p.beta = a->beta;
    p.vbeta = a->beta * (float)a->num_words;
    p.num_docs = a->num_docs;
    p.num_items = a->num_items;
    p.num_hot = a->num_hot;
    p.num_tokens = a->num_tokens;
    p.theta_cap = a->theta_capacity;
    p.doc_ids = a->doc_ids;
    p.tok_index = nullptr;
    p.topics_in = a->topics_in;
    p.topics_out = a->topics_out;
    p.theta = reinterpret_cast<const ThetaEntry *>(a->theta);
    p.rows = reinterpret_cast<const int2 *>(a->theta_rows);
    p.nk = a->nk;
    p.items = a->items;
    p.seg_start = a->seg_start;
    p.num_segs = a->num_segs;
    p.hot_phi = hot_phi;
    p.item_counter = counter;
    p.item_ll = item_ll;
    p.seed = a->seed;
    p.iteration = a->iteration;
    p.iteration_ptr = nullptr;
    p.error = a->error ? a->error : counter + 1;
    int dev = 0;
    cudaGetDevice(&dev);
    const int blocks = a->group_lanes == kFlatLanes ? kFlatBlocks : kSampleBlocksDefault;
    int bps = sample_blocks_per_sm(a->k, a->group_lanes, blocks);
    if (bps <= 0) bps = 1;
    const int grid = std::max(1, std::min(a->num_items, num_sms(dev) * bps));
    rc = cuda_status(launch_sample(p, a->group_lanes, blocks, grid, s));
    if (rc) return rc;
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
