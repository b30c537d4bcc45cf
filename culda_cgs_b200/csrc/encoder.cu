// encoder.cu — the document encoder of the learned Metropolis-Hastings
// proposal: embedding bag -> 2 x 512 GELU MLP -> softmax over K topics, its
// backward pass and Adam, on the tensor-core GEMM of gemm.cu; and the C entry
// points of the GEMM and of the encoder.
//
// Per batch of Bp rows (the batch rounded up to 128; rows past the batch are
// zero and carry no gradient):
//   forward   X0 = embbag(E)                         [Bp x 256]  BF16 (+ X0^T)
//             P1 = X0 W1^T + b1, H1 = GELU(P1)       [Bp x 512]  FP32 / BF16 (+ H1^T)
//             P2 = H1 W2^T + b2, H2 = GELU(P2)       [Bp x 512]
//             Z  = H2 W3^T + b3, q = softmax(Z)      [Bp x K]
//   backward  dZ = (q - target) / B                  BF16 (+ dZ^T), db3 = column sums
//             dW3 = dZ^T H2                          GEMM(dZ^T, H2^T)
//             dP2 = (dZ W3) * GELU'(P2)              GEMM(dZ, W3^T), db2 = column sums
//             dW2 = dP2^T H1,  dP1 = (dP2 W2) * GELU'(P1), db1
//             dW1 = dP1^T X0,  dX0 = dP1 W1          FP32
//             dE[w] = sum of dX0[b] / L_b over the tokens of w in the batch
//                   (tokens grouped by word, one write per embedding row)
// The weight gradients split their K range (the batch) over several CTAs
// per tile.  Every GEMM is C = A B^T with both operands K-major, so each weight is kept
// in BF16 twice (W and W^T) and each activation that feeds a weight gradient
// is written transposed by the epilogue that produces it.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "device_util.cuh"
#include "encoder.cuh"
#include "gemm.cuh"
#include "internal.h"
#include "philox.h"

using bf16 = __nv_bfloat16;

namespace culda {
namespace {

constexpr int kE = CULDA_ENC_EMBED, kH = CULDA_ENC_HIDDEN;
constexpr int kNumTensors = 7;

// ------------------------------------------------------------------ kernels
__global__ void init_uniform_kernel(int64_t n, float *dst, float scale, uint64_t seed, uint32_t tensor) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        dst[i] = scale * (2.0f * uniform_from_bits(philox_token(seed, (uint64_t)i, tensor, kPurposeWeights)) - 1.0f);
}

__global__ void to_bf16_kernel(int64_t n, const float *src, bf16 *dst) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        dst[i] = __float2bfloat16_rn(src[i]);
}

// out[c][r] = in[r][c] for an [R x C] matrix, through 32 x 32 shared tiles.
template <class T>
__global__ void transpose_bf16_kernel(int R, int C, const T *in, int ld_in, bf16 *out, int ld_out) {
    __shared__ float tile[32][33];
    const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {
        const int r = r0 + i, c = c0 + threadIdx.x;
        if (r < R && c < C) tile[i][threadIdx.x] = (float)in[(size_t)r * ld_in + c];
    }
    __syncthreads();
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {
        const int c = c0 + i, r = r0 + threadIdx.x;
        if (r < R && c < C) out[(size_t)c * ld_out + r] = __float2bfloat16_rn(tile[threadIdx.x][i]);
    }
}

__device__ __forceinline__ void unpack8(const uint4 &v, float f[8]) {
    const bf16 *h = reinterpret_cast<const bf16 *>(&v);
#pragma unroll
    for (int i = 0; i < 8; ++i) f[i] = __bfloat162float(h[i]);
}

// Warp per batch row; lane l owns embedding columns 8l .. 8l+7.
__global__ void __launch_bounds__(256) embbag_fwd_kernel(int batch, int rows, const int32_t *__restrict__ docs,
                                                         const int64_t *__restrict__ doc_ptr,
                                                         const int32_t *__restrict__ words, int V,
                                                         const bf16 *__restrict__ emb, bf16 *X0, int32_t *error) {
    // one CTA per batch row: its 8 warps take contiguous eighths of the
    // document's tokens (a long document is no longer one warp's serial loop),
    // then the partial sums are added in warp order
    __shared__ float part[8][kE];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int b = blockIdx.x; b < rows; b += gridDim.x) {
        float acc[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        int64_t t0 = 0, t1 = 0;
        if (b < batch) {
            const int d = docs ? docs[b] : b;
            t0 = doc_ptr[d];
            t1 = doc_ptr[d + 1];
            const int64_t per = (t1 - t0 + 7) / 8;
            const int64_t w0 = t0 + per * warp, w1 = min(t1, w0 + per);
            for (int64_t tb = w0; tb < w1; tb += 32) {
                const int wl = tb + lane < w1 ? words[tb + lane] : 0;
                const int n = (int)min((int64_t)32, w1 - tb);
                // eight embedding rows in flight, then added in token order
                for (int j0 = 0; j0 < n; j0 += 8) {
                    uint4 v[8];
                    bool ok[8];
#pragma unroll
                    for (int u = 0; u < 8; ++u) {
                        const int w = __shfl_sync(0xffffffffu, wl, (j0 + u) & 31);
                        const bool in = j0 + u < n;
                        ok[u] = in && (unsigned)w < (unsigned)V;
                        if (in && !ok[u] && lane == 0) atomicOr(error, kErrWordRange);
                        v[u] = ok[u] ? __ldg(reinterpret_cast<const uint4 *>(emb + (size_t)w * kE) + lane)
                                     : make_uint4(0u, 0u, 0u, 0u);
                    }
#pragma unroll
                    for (int u = 0; u < 8; ++u) {
                        if (!ok[u]) continue;
                        float f[8];
                        unpack8(v[u], f);
#pragma unroll
                        for (int i = 0; i < 8; ++i) acc[i] += f[i];
                    }
                }
            }
        }
#pragma unroll
        for (int i = 0; i < 8; ++i) part[warp][8 * lane + i] = acc[i];
        __syncthreads();
        if (warp == 0) {
            float sum[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
            for (int w = 0; w < 8; ++w)
#pragma unroll
                for (int i = 0; i < 8; ++i) sum[i] += part[w][8 * lane + i];
            const float inv = t1 > t0 ? 1.0f / (float)(t1 - t0) : 0.f;
            uint4 q;
            __nv_bfloat162 *h = reinterpret_cast<__nv_bfloat162 *>(&q);
#pragma unroll
            for (int i = 0; i < 4; ++i) h[i] = __floats2bfloat162_rn(sum[2 * i] * inv, sum[2 * i + 1] * inv);
            reinterpret_cast<uint4 *>(X0 + (size_t)b * kE)[lane] = q;
        }
        __syncthreads();  // part is rewritten by the next row
    }
}

// The embedding gradient: the batch's (word, row) pairs are laid out in row
// order (a scan of the row lengths), sorted by word (a radix sort, stable, so
// a word's tokens stay in row order), and the sorted list is cut into chunks
// of 32 tokens.  A warp walks its chunk in order, summing dX0[b] / L_b per
// word in registers.  A word whose tokens all lie in the chunk is written with
// plain stores; a word whose run crosses the chunk's first or last token (the
// frequent ones) adds each chunk's partial sum with one vector atomic per
// lane.  gE holds zeros before the pass; words outside [0, V) sort last under
// the key V and are skipped.

// len[b] = L_b (for the scan of row offsets) and inv_len[b] = 1 / L_b.
__global__ void bag_rows_kernel(int batch, const int32_t *__restrict__ docs, const int64_t *__restrict__ doc_ptr,
                                int32_t *len, float *inv_len) {
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < batch; b += gridDim.x * blockDim.x) {
        const int d = docs ? docs[b] : b;
        const int64_t L = doc_ptr[d + 1] - doc_ptr[d];
        len[b] = (int32_t)L;
        inv_len[b] = L > 0 ? 1.0f / (float)L : 0.f;
    }
}

// key[off[b] + j] = word of the j-th token of row b (V when out of range), val = b.
__global__ void __launch_bounds__(256) bag_pairs_kernel(int batch, const int32_t *__restrict__ docs,
                                                        const int64_t *__restrict__ doc_ptr,
                                                        const int32_t *__restrict__ words, int V,
                                                        const int32_t *__restrict__ off, int32_t *key, int32_t *val) {
    for (int b = blockIdx.x; b < batch; b += gridDim.x) {
        const int d = docs ? docs[b] : b;
        const int64_t t0 = doc_ptr[d], t1 = doc_ptr[d + 1];
        const int o = off[b];
        for (int64_t t = t0 + threadIdx.x; t < t1; t += blockDim.x) {
            const int w = words[t];
            key[o + (t - t0)] = (unsigned)w < (unsigned)V ? w : V;
            val[o + (t - t0)] = b;
        }
    }
}

// Warp per chunk of 32 sorted tokens; each lane holds 8 of the 256 columns.
__global__ void embbag_bwd_grouped_kernel(int64_t n, int V, const int32_t *__restrict__ wid,
                                          const int32_t *__restrict__ rows, const float *__restrict__ inv_len,
                                          const float *__restrict__ dX0, float *gE) {
    const int lane = threadIdx.x & 31;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t c0 = (((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32; c0 < n; c0 += nw * 32) {
        const int cn = (int)min((int64_t)32, n - c0);
        const int my_w = lane < cn ? wid[c0 + lane] : V;
        const int my_b = lane < cn ? rows[c0 + lane] : 0;
        const float my_s = lane < cn ? inv_len[my_b] : 0.f;
        // does the chunk's first (last) run continue from the chunk before (after) it?
        const int w_before = c0 > 0 ? wid[c0 - 1] : -1;
        const int w_after = c0 + cn < n ? wid[c0 + cn] : -1;
        const int first_w = __shfl_sync(0xffffffffu, my_w, 0), last_w = __shfl_sync(0xffffffffu, my_w, cn - 1);
        // the chunk's dX0 rows, 2 x 16 bytes per lane each, loaded 8 at a time ahead of their use
        float4 a0 = make_float4(0.f, 0.f, 0.f, 0.f), a1 = a0;
        float4 r0[8], r1[8];
        for (int j = 0; j < cn; ++j) {
            if ((j & 7) == 0) {
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    const int bj = __shfl_sync(0xffffffffu, my_b, (j + u) & 31);
                    const float4 *q = reinterpret_cast<const float4 *>(dX0 + (size_t)bj * kE) + 2 * lane;
                    const bool in = j + u < cn;
                    r0[u] = in ? q[0] : make_float4(0.f, 0.f, 0.f, 0.f);
                    r1[u] = in ? q[1] : make_float4(0.f, 0.f, 0.f, 0.f);
                }
            }
            const int w = __shfl_sync(0xffffffffu, my_w, j);
            const float sc = __shfl_sync(0xffffffffu, my_s, j);
            float4 g0 = r0[0], g1 = r1[0];
#pragma unroll
            for (int u = 1; u < 8; ++u)
                if ((j & 7) == u) {
                    g0 = r0[u];
                    g1 = r1[u];
                }
            a0.x += g0.x * sc;
            a0.y += g0.y * sc;
            a0.z += g0.z * sc;
            a0.w += g0.w * sc;
            a1.x += g1.x * sc;
            a1.y += g1.y * sc;
            a1.z += g1.z * sc;
            a1.w += g1.w * sc;
            const int wn = __shfl_sync(0xffffffffu, my_w, (j + 1) & 31);
            if (j + 1 == cn || wn != w) {  // the end of this word's run in the chunk
                if (w < V) {
                    float4 *dst = reinterpret_cast<float4 *>(gE + (size_t)w * kE) + 2 * lane;
                    const bool shared = (w == first_w && w == w_before) || (w == last_w && w == w_after);
                    if (!shared) {  // the whole word: no other chunk adds to it
                        dst[0] = a0;
                        dst[1] = a1;
                    } else {
                        atomicAdd(dst, a0);
                        atomicAdd(dst + 1, a1);
                    }
                }
                a0 = make_float4(0.f, 0.f, 0.f, 0.f);
                a1 = a0;
            }
        }
    }
}

// Softmax of each row of Z [rows x K] and, against the target, dZ = (q - t) /
// batch (BF16), the column sums of dZ (db3) and the summed cross-entropy.
// 256 threads = 8 warps per block, kXentRows rows per block; lane l holds
// columns l, l+32, ... of its row; the block's column sums go to db3 with one
// atomic per column.
constexpr int kXentRows = 8;  // one row per warp: Bp / 8 blocks

__global__ void __launch_bounds__(256) softmax_xent_kernel(int batch, int rows, int K, const float *__restrict__ Z,
                                                           EncoderTarget tg, const int32_t *__restrict__ docs,
                                                           const int64_t *__restrict__ doc_ptr, float *probs,
                                                           bf16 *dZ, float *db3, double *loss) {
    extern __shared__ float colsum[];  // [K]
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int k = threadIdx.x; k < K; k += blockDim.x) colsum[k] = 0.f;
    __syncthreads();
    const float inv_batch = 1.0f / (float)batch;
    double my_loss = 0.0;
    const int r_end = min(rows, (int)(blockIdx.x + 1) * kXentRows);
    for (int b = blockIdx.x * kXentRows + warp; b < r_end; b += 8) {
        const float *z = Z + (size_t)b * K;
        if (b >= batch) {  // padding row: no gradient
            if (dZ)
                for (int k = lane; k < K; k += 32) dZ[(size_t)b * K + k] = __float2bfloat16_rn(0.f);
            continue;
        }
        float mx = -INFINITY;
        for (int k = lane; k < K; k += 32) mx = fmaxf(mx, z[k]);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        float se = 0.f;
        for (int k = lane; k < K; k += 32) se += __expf(z[k] - mx);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) se += __shfl_xor_sync(0xffffffffu, se, o);
        const float lse = mx + __logf(se), inv_se = 1.0f / se;
        if (probs)
            for (int k = lane; k < K; k += 32) probs[(size_t)b * K + k] = __expf(z[k] - mx) * inv_se;
        if (!dZ) continue;
        const int d = docs ? docs[b] : b;
        float tscale = 0.f;
        if (!tg.dense) {
            const float L = (float)(doc_ptr[d + 1] - doc_ptr[d]);
            tscale = 1.0f / (L + (float)K * tg.alpha);
        }
        float l = 0.f;
        for (int k = lane; k < K; k += 32) {
            const float t = tg.dense ? tg.dense[(size_t)b * K + k]
                                     : (tg.acc[(size_t)d * K + k] * tg.inv_n + tg.alpha) * tscale;
            const float q = __expf(z[k] - mx) * inv_se;
            const float g = (q - t) * inv_batch;
            dZ[(size_t)b * K + k] = __float2bfloat16_rn(g);
            atomicAdd(&colsum[k], g);
            l += t * (lse - z[k]);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
        if (lane == 0) my_loss += (double)l;
    }
    __syncthreads();
    if (db3)
        for (int k = threadIdx.x; k < K; k += blockDim.x)
            if (colsum[k] != 0.f) atomicAdd(&db3[k], colsum[k]);
    if (lane == 0 && loss && my_loss != 0.0) atomicAdd(loss, my_loss);
}

__global__ void adam_kernel(int64_t n, float *p, const float *g, float *m, float *v, float lr, float b1, float b2,
                            float eps, float c1, float c2) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.0f - b1) * gi;
        const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        p[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + eps);
    }
}

}  // namespace
}  // namespace culda

using namespace culda;

// ------------------------------------------------------------------ object
struct culda_encoder {
    int device = 0;
    int V = 0, K = 0, Bmax = 0;  // Bmax: rows, a multiple of 128
    float lr = 1e-3f, b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    int64_t steps = 0;
    int64_t off[kNumTensors + 1] = {};  // offsets of the tensors in the FP32 blocks
    float *params = nullptr, *grads = nullptr, *adam_m = nullptr, *adam_v = nullptr;
    bf16 *emb_bf = nullptr, *W1 = nullptr, *W1t = nullptr, *W2 = nullptr, *W2t = nullptr, *W3 = nullptr,
         *W3t = nullptr;
    bf16 *X0 = nullptr, *X0t = nullptr, *H1 = nullptr, *H1t = nullptr, *H2 = nullptr, *H2t = nullptr;
    bf16 *dZ = nullptr, *dZt = nullptr, *dP2 = nullptr, *dP2t = nullptr, *dP1 = nullptr, *dP1t = nullptr;
    float *P1 = nullptr, *P2 = nullptr, *Z = nullptr, *dX0 = nullptr;
    double *d_loss = nullptr;
    int32_t *d_error = nullptr;
    // the batch's (word, row) pairs sorted by word, for the embedding gradient
    int32_t *bag_len = nullptr, *bag_off = nullptr;  // [Bmax + 1] row lengths and their exclusive scan
    float *bag_inv_len = nullptr;                    // [Bmax] 1 / L of every batch row
    int32_t *bag_key = nullptr, *bag_val = nullptr;  // [bag_cap] pairs in row order
    int32_t *bag_wid = nullptr, *bag_rows = nullptr; // [bag_cap] the pairs sorted by word
    int64_t bag_cap = 0;
    void *scan_tmp = nullptr, *sort_tmp = nullptr;
    size_t scan_tmp_bytes = 0, sort_tmp_bytes = 0;
    int key_bits = 1;                                // bits of the keys 0..V
    std::vector<void *> allocs;

    float *tensor(int t) { return params + off[t]; }
    float *grad(int t) { return grads + off[t]; }
};

namespace culda {
namespace {

template <class T>
cudaError_t ealloc(culda_encoder *e, T **p, size_t n) {
    const cudaError_t r =
        (cudaError_t)device_malloc(reinterpret_cast<void **>(p), std::max<size_t>(n, 1) * sizeof(T));
    if (r == cudaSuccess) e->allocs.push_back(*p);
    return r;
}

int fail_enc(int code, const char *fmt, const char *what) {
    set_global_error(fmt, what);
    return code;
}

#define ECK(x)                                                                   \
    do {                                                                         \
        cudaError_t _e = (x);                                                    \
        if (_e != cudaSuccess) return fail_enc(CULDA_ERR_CUDA, "encoder: %s", cudaGetErrorString(_e)); \
    } while (0)

cudaError_t transpose_to_bf16(int R, int C, const float *in, bf16 *out, cudaStream_t s) {
    transpose_bf16_kernel<float><<<dim3((C + 31) / 32, (R + 31) / 32), dim3(32, 8), 0, s>>>(R, C, in, C, out, R);
    return cudaGetLastError();
}

cudaError_t transpose_bf16(int R, int C, const bf16 *in, bf16 *out, cudaStream_t s) {
    transpose_bf16_kernel<bf16><<<dim3((C + 31) / 32, (R + 31) / 32), dim3(32, 8), 0, s>>>(R, C, in, C, out, R);
    return cudaGetLastError();
}

// BF16 copies of the weights (and the transposes the backward pass reads).
cudaError_t refresh_bf16(culda_encoder *e, cudaStream_t s) {
    const int64_t ne = (int64_t)e->V * kE;
    to_bf16_kernel<<<grid_for(ne), 256, 0, s>>>(ne, e->tensor(CULDA_ENC_E), e->emb_bf);
    to_bf16_kernel<<<grid_for((int64_t)kH * kE), 256, 0, s>>>((int64_t)kH * kE, e->tensor(CULDA_ENC_W1), e->W1);
    to_bf16_kernel<<<grid_for((int64_t)kH * kH), 256, 0, s>>>((int64_t)kH * kH, e->tensor(CULDA_ENC_W2), e->W2);
    to_bf16_kernel<<<grid_for((int64_t)e->K * kH), 256, 0, s>>>((int64_t)e->K * kH, e->tensor(CULDA_ENC_W3), e->W3);
    cudaError_t r = transpose_to_bf16(kH, kE, e->tensor(CULDA_ENC_W1), e->W1t, s);
    if (r == cudaSuccess) r = transpose_to_bf16(kH, kH, e->tensor(CULDA_ENC_W2), e->W2t, s);
    if (r == cudaSuccess) r = transpose_to_bf16(e->K, kH, e->tensor(CULDA_ENC_W3), e->W3t, s);
    return r;
}

cudaError_t gemm(int M, int N, int K, const bf16 *A, const bf16 *B, int epi, const GemmEpilogue &ep, int32_t *err,
                 cudaStream_t s) {
    return gemm_bf16_nt(M, N, K, A, K, B, K, epi, ep, err, s);
}

// Weight gradients: M x N is a few tiles and K the batch, so the K range is
// cut into slices (at least 4 k-blocks each), as many as fill the two CTAs
// per SM in one wave; the slices add into the zeroed gradient.
cudaError_t gemm_wgrad(int M, int N, int K, const bf16 *A, const bf16 *B, GemmEpilogue ep, int32_t *err,
                       cudaStream_t s) {
    int sms = 148;
    int dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int tiles = (M / 128) * (N / 128);
    const int by_k = std::max(1, (K / 64) / 4);
    ep.k_splits = std::max(1, std::min(by_k, (2 * sms) / tiles));
    return gemm_bf16_nt(M, N, K, A, K, B, K, kEpiF32, ep, err, s);
}

}  // namespace

int encoder_k(const culda_encoder *e) { return e->K; }
int encoder_num_words(const culda_encoder *e) { return e->V; }
float *encoder_tensor(culda_encoder *e, int t) { return e->tensor(t); }
int encoder_refresh(culda_encoder *e, cudaStream_t s) {
    ECK(refresh_bf16(e, s));
    return CULDA_OK;
}
int encoder_max_batch(const culda_encoder *e) { return e->Bmax; }
int32_t *encoder_error_word(culda_encoder *e) { return e->d_error; }

int encoder_pass(culda_encoder *e, int batch, const int32_t *docs, const int64_t *doc_ptr, const int32_t *words,
                 const EncoderTarget *target, bool update, float *probs, cudaStream_t s, int64_t batch_tokens) {
    if (batch <= 0 || batch > e->Bmax || !doc_ptr || !words)
        return fail_enc(CULDA_ERR_INVALID_ARG, "encoder: %s", "batch outside 1..max_batch or null CSR");
    if (target && !target->dense && !target->acc)
        return fail_enc(CULDA_ERR_INVALID_ARG, "encoder: %s", "target without data");
    ECK(cudaSetDevice(e->device));
    const int Bp = (batch + 127) & ~127, K = e->K;
    int32_t *err = e->d_error;
    // forward
    embbag_fwd_kernel<<<std::min(Bp, 148 * 16), 256, 0, s>>>(batch, Bp, docs, doc_ptr, words, e->V, e->emb_bf,
                                                                 e->X0, err);
    ECK(cudaGetLastError());
    GemmEpilogue ep;
    ep.out_f32 = e->P1;
    ep.ldo = kH;
    ep.out_bf16 = e->H1;
    ep.out_bf16_t = e->H1t;
    ep.ld_t = Bp;
    ep.bias = e->tensor(CULDA_ENC_B1);
    ECK(gemm(Bp, kH, kE, e->X0, e->W1, kEpiBiasGelu, ep, err, s));
    ep.out_f32 = e->P2;
    ep.out_bf16 = e->H2;
    ep.out_bf16_t = e->H2t;
    ep.bias = e->tensor(CULDA_ENC_B2);
    ECK(gemm(Bp, kH, kH, e->H1, e->W2, kEpiBiasGelu, ep, err, s));
    GemmEpilogue ez;
    ez.out_f32 = e->Z;
    ez.ldo = K;
    ez.bias = e->tensor(CULDA_ENC_B3);
    ECK(gemm(Bp, K, kH, e->H2, e->W3, kEpiF32, ez, err, s));
    const size_t xsmem = (size_t)K * sizeof(float);
    if (!target) {
        softmax_xent_kernel<<<(Bp + kXentRows - 1) / kXentRows, 256, xsmem, s>>>(
            batch, Bp, K, e->Z, EncoderTarget{}, docs, doc_ptr, probs, nullptr, nullptr, nullptr);
        ECK(cudaGetLastError());
        return CULDA_OK;
    }
    // backward
    ECK(cudaMemsetAsync(e->grads, 0, sizeof(float) * (size_t)e->off[kNumTensors], s));
    softmax_xent_kernel<<<(Bp + kXentRows - 1) / kXentRows, 256, xsmem, s>>>(
        batch, Bp, K, e->Z, *target, docs, doc_ptr, probs, e->dZ, e->grad(CULDA_ENC_B3), e->d_loss);
    ECK(cudaGetLastError());
    ECK(transpose_bf16(Bp, K, e->dZ, e->dZt, s));
    ECK(transpose_bf16(Bp, kE, e->X0, e->X0t, s));
    GemmEpilogue gw;
    gw.ldo = kH;
    gw.out_f32 = e->grad(CULDA_ENC_W3);
    ECK(gemm_wgrad(K, kH, Bp, e->dZt, e->H2t, gw, err, s));  // dW3 = dZ^T H2
    GemmEpilogue gb;
    gb.ldo = kH;
    gb.ld_t = Bp;
    gb.pre = e->P2;
    gb.out_bf16 = e->dP2;
    gb.out_bf16_t = e->dP2t;
    gb.colsum = e->grad(CULDA_ENC_B2);
    ECK(gemm(Bp, kH, K, e->dZ, e->W3t, kEpiGeluBwd, gb, err, s));  // dP2 = (dZ W3) GELU'(P2)
    gw.out_f32 = e->grad(CULDA_ENC_W2);
    ECK(gemm_wgrad(kH, kH, Bp, e->dP2t, e->H1t, gw, err, s));  // dW2 = dP2^T H1
    gb.pre = e->P1;
    gb.out_bf16 = e->dP1;
    gb.out_bf16_t = e->dP1t;
    gb.colsum = e->grad(CULDA_ENC_B1);
    ECK(gemm(Bp, kH, kH, e->dP2, e->W2t, kEpiGeluBwd, gb, err, s));  // dP1 = (dP2 W2) GELU'(P1)
    GemmEpilogue g1;
    g1.ldo = kE;
    g1.out_f32 = e->grad(CULDA_ENC_W1);
    ECK(gemm_wgrad(kH, kE, Bp, e->dP1t, e->X0t, g1, err, s));  // dW1 = dP1^T X0
    g1.out_f32 = e->dX0;
    ECK(gemm(Bp, kE, kH, e->dP1, e->W1t, kEpiF32, g1, err, s));  // dX0 = dP1 W1
    // the batch's (word, row) pairs sorted by word, then one pass over them
    bag_rows_kernel<<<(batch + 255) / 256, 256, 0, s>>>(batch, docs, doc_ptr, e->bag_len, e->bag_inv_len);
    ECK(cudaGetLastError());
    ECK(cub::DeviceScan::ExclusiveSum(e->scan_tmp, e->scan_tmp_bytes, e->bag_len, e->bag_off, batch + 1, s));
    if (batch_tokens < 0) {  // the caller did not count the batch's tokens: read the scan's total
        int32_t n = 0;
        ECK(cudaMemcpyAsync(&n, e->bag_off + batch, sizeof n, cudaMemcpyDeviceToHost, s));
        ECK(cudaStreamSynchronize(s));
        batch_tokens = n;
    }
    if (batch_tokens > e->bag_cap) {
        ECK(cudaStreamSynchronize(s));
        for (void **q : {(void **)&e->bag_key, (void **)&e->bag_val, (void **)&e->bag_wid, (void **)&e->bag_rows,
                         &e->sort_tmp}) {
            if (*q) {
                cudaFree(*q);
                e->allocs.erase(std::find(e->allocs.begin(), e->allocs.end(), *q));
                *q = nullptr;
            }
        }
        const int64_t cap = std::max<int64_t>(batch_tokens, 2 * e->bag_cap);
        ECK(ealloc(e, &e->bag_key, (size_t)cap));
        ECK(ealloc(e, &e->bag_val, (size_t)cap));
        ECK(ealloc(e, &e->bag_wid, (size_t)cap));
        ECK(ealloc(e, &e->bag_rows, (size_t)cap));
        e->sort_tmp_bytes = 0;
        ECK(cub::DeviceRadixSort::SortPairs(nullptr, e->sort_tmp_bytes, e->bag_key, e->bag_wid, e->bag_val,
                                            e->bag_rows, (int)cap, 0, e->key_bits));
        uint8_t *tmp = nullptr;
        ECK(ealloc(e, &tmp, e->sort_tmp_bytes));
        e->sort_tmp = tmp;
        e->bag_cap = cap;
    }
    if (batch_tokens > 0) {
        bag_pairs_kernel<<<std::min(batch, 148 * 16), 256, 0, s>>>(batch, docs, doc_ptr, words, e->V, e->bag_off,
                                                                   e->bag_key, e->bag_val);
        ECK(cudaGetLastError());
        ECK(cub::DeviceRadixSort::SortPairs(e->sort_tmp, e->sort_tmp_bytes, e->bag_key, e->bag_wid, e->bag_val,
                                            e->bag_rows, (int)batch_tokens, 0, e->key_bits, s));
        embbag_bwd_grouped_kernel<<<grid_for(batch_tokens), 256, 0, s>>>(batch_tokens, e->V, e->bag_wid, e->bag_rows,
                                                                         e->bag_inv_len, e->dX0,
                                                                         e->grad(CULDA_ENC_E));
        ECK(cudaGetLastError());
    }
    if (update) {
        e->steps += 1;
        const float c1 = 1.0f / (1.0f - powf(e->b1, (float)e->steps));
        const float c2 = 1.0f / (1.0f - powf(e->b2, (float)e->steps));
        const int64_t n = e->off[kNumTensors];
        adam_kernel<<<grid_for(n), 256, 0, s>>>(n, e->params, e->grads, e->adam_m, e->adam_v, e->lr, e->b1, e->b2,
                                                e->eps, c1, c2);
        ECK(cudaGetLastError());
        ECK(refresh_bf16(e, s));
    }
    return CULDA_OK;
}

int encoder_take_loss(culda_encoder *e, int batch_rows, double *loss, cudaStream_t s) {
    double h = 0.0;
    int32_t err = 0;
    ECK(cudaMemcpyAsync(&h, e->d_loss, sizeof(double), cudaMemcpyDeviceToHost, s));
    ECK(cudaMemcpyAsync(&err, e->d_error, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    ECK(cudaMemsetAsync(e->d_loss, 0, sizeof(double), s));
    ECK(cudaStreamSynchronize(s));
    if (err) {
        cudaMemsetAsync(e->d_error, 0, sizeof(int32_t), s);
        char msg[96];
        snprintf(msg, sizeof msg, "encoder: device error 0x%x", err);
        return fail_enc(CULDA_ERR_DEVICE_STATE, "%s", msg);
    }
    if (loss) *loss = batch_rows > 0 ? h / (double)batch_rows : 0.0;
    return CULDA_OK;
}

}  // namespace culda

// ============================================================ C entry points
extern "C" int culda_gemm_bf16(const culda_gemm_args *a, void *stream) {
    if (!a) {
        set_global_error("culda_gemm_bf16: null arguments");
        return CULDA_ERR_INVALID_ARG;
    }
    GemmEpilogue ep;
    ep.out_f32 = a->out_f32;
    ep.ldo = a->ldo;
    ep.out_bf16 = reinterpret_cast<bf16 *>(a->out_bf16);
    ep.out_bf16_t = reinterpret_cast<bf16 *>(a->out_bf16_t);
    ep.ld_t = a->ld_t;
    ep.bias = a->bias;
    ep.pre = a->pre;
    ep.colsum = a->colsum;
    ep.alpha = a->alpha;
    ep.k_splits = a->k_splits > 0 ? a->k_splits : 1;
    if (const char *why = gemm_check(a->m, a->n, a->k, a->a, a->lda, a->b, a->ldb, a->epilogue, ep)) {
        set_global_error("culda_gemm_bf16: %s", why);
        return CULDA_ERR_INVALID_ARG;
    }
    const cudaError_t e = gemm_bf16_nt(a->m, a->n, a->k, a->a, a->lda, a->b, a->ldb, a->epilogue, ep, a->error,
                                       static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) {
        set_global_error("culda_gemm_bf16: %s", cudaGetErrorString(e));
        return e == cudaErrorNotSupported ? CULDA_ERR_UNSUPPORTED : CULDA_ERR_CUDA;
    }
    return CULDA_OK;
}

extern "C" int culda_encoder_create(const culda_encoder_params *p, culda_encoder **out) {
    if (!p || !out) return fail_enc(CULDA_ERR_INVALID_ARG, "culda_encoder_create: %s", "null argument");
    *out = nullptr;
    if (p->num_words <= 0 || p->k < 128 || p->k > 4096 || p->k % 128 || p->max_batch <= 0 || p->max_batch > 65536)
        return fail_enc(CULDA_ERR_INVALID_ARG, "culda_encoder_create: %s",
                        "num_words > 0, k a multiple of 128 in 128..4096, max_batch in 1..65536");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0)
        return fail_enc(CULDA_ERR_NO_DEVICE, "culda_encoder_create: %s", "no CUDA device");
    if (p->device < 0 || p->device >= ndev)
        return fail_enc(CULDA_ERR_INVALID_ARG, "culda_encoder_create: %s", "device out of range");
    culda_encoder *e = new culda_encoder;
    e->device = p->device;
    e->V = p->num_words;
    e->K = p->k;
    e->Bmax = (p->max_batch + 127) & ~127;
    if (p->lr > 0.f) e->lr = p->lr;
    if (p->beta1 > 0.f) e->b1 = p->beta1;
    if (p->beta2 > 0.f) e->b2 = p->beta2;
    if (p->eps > 0.f) e->eps = p->eps;
    const int64_t sizes[kNumTensors] = {(int64_t)e->V * kE, (int64_t)kH * kE, kH, (int64_t)kH * kH, kH,
                                        (int64_t)e->K * kH, e->K};
    for (int t = 0; t < kNumTensors; ++t) e->off[t + 1] = e->off[t] + sizes[t];
    const size_t np = (size_t)e->off[kNumTensors];
    const size_t B = (size_t)e->Bmax, K = (size_t)e->K;
    auto bail = [&](cudaError_t r) {
        for (void *q : e->allocs) cudaFree(q);
        delete e;
        return fail_enc(r == cudaErrorMemoryAllocation ? CULDA_ERR_OOM : CULDA_ERR_CUDA, "culda_encoder_create: %s",
                        cudaGetErrorString(r));
    };
    cudaError_t r = cudaSetDevice(e->device);
    if (r != cudaSuccess) return bail(r);
#define EALLOC(ptr, n)                 \
    r = ealloc(e, &(ptr), (size_t)(n)); \
    if (r != cudaSuccess) return bail(r)
    EALLOC(e->params, np);
    EALLOC(e->grads, np);
    EALLOC(e->adam_m, np);
    EALLOC(e->adam_v, np);
    EALLOC(e->emb_bf, (size_t)e->V * kE);
    EALLOC(e->W1, kH * kE);
    EALLOC(e->W1t, kH * kE);
    EALLOC(e->W2, kH * kH);
    EALLOC(e->W2t, kH * kH);
    EALLOC(e->W3, K * kH);
    EALLOC(e->W3t, K * kH);
    EALLOC(e->X0, B * kE);
    EALLOC(e->X0t, B * kE);
    EALLOC(e->H1, B * kH);
    EALLOC(e->H1t, B * kH);
    EALLOC(e->H2, B * kH);
    EALLOC(e->H2t, B * kH);
    EALLOC(e->dZ, B * K);
    EALLOC(e->dZt, B * K);
    EALLOC(e->dP2, B * kH);
    EALLOC(e->dP2t, B * kH);
    EALLOC(e->dP1, B * kH);
    EALLOC(e->dP1t, B * kH);
    EALLOC(e->P1, B * kH);
    EALLOC(e->P2, B * kH);
    EALLOC(e->Z, B * K);
    EALLOC(e->dX0, B * kE);
    EALLOC(e->d_loss, 1);
    EALLOC(e->d_error, 1);
    EALLOC(e->bag_len, (size_t)B + 1);
    EALLOC(e->bag_off, (size_t)B + 1);
    EALLOC(e->bag_inv_len, B);
    while ((1u << e->key_bits) <= (unsigned)e->V) ++e->key_bits;  // keys 0..V
    r = cub::DeviceScan::ExclusiveSum(nullptr, e->scan_tmp_bytes, e->bag_len, e->bag_off, B + 1);
    if (r != cudaSuccess) return bail(r);
    {
        uint8_t *tmp = nullptr;
        EALLOC(tmp, e->scan_tmp_bytes);
        e->scan_tmp = tmp;
    }
#undef EALLOC
    cudaStream_t s = nullptr;
    r = cudaMemsetAsync(e->grads, 0, sizeof(float) * np, s);
    if (r == cudaSuccess) r = cudaMemsetAsync(e->adam_m, 0, sizeof(float) * np, s);
    if (r == cudaSuccess) r = cudaMemsetAsync(e->adam_v, 0, sizeof(float) * np, s);
    if (r == cudaSuccess) r = cudaMemsetAsync(e->params, 0, sizeof(float) * np, s);
    if (r == cudaSuccess) r = cudaMemsetAsync(e->d_loss, 0, sizeof(double), s);
    if (r == cudaSuccess) r = cudaMemsetAsync(e->d_error, 0, sizeof(int32_t), s);
    if (r != cudaSuccess) return bail(r);
    // weights: uniform(-a, a) with a = sqrt(6 / (fan_in + fan_out)); embeddings
    // uniform(-0.5, 0.5); biases zero
    const struct {
        int t;
        float a;
    } init[] = {{CULDA_ENC_E, 0.5f},
                {CULDA_ENC_W1, sqrtf(6.0f / (kE + kH))},
                {CULDA_ENC_W2, sqrtf(6.0f / (kH + kH))},
                {CULDA_ENC_W3, sqrtf(6.0f / (float)(kH + e->K))}};
    for (const auto &x : init) {
        const int64_t n = sizes[x.t];
        init_uniform_kernel<<<grid_for(n), 256, 0, s>>>(n, e->tensor(x.t), x.a, p->seed, (uint32_t)x.t);
    }
    r = refresh_bf16(e, s);
    if (r == cudaSuccess) r = cudaStreamSynchronize(s);
    if (r != cudaSuccess) return bail(r);
    *out = e;
    return CULDA_OK;
}

extern "C" int culda_encoder_destroy(culda_encoder *e) {
    if (!e) return CULDA_OK;
    cudaSetDevice(e->device);
    cudaDeviceSynchronize();
    for (void *q : e->allocs) cudaFree(q);
    delete e;
    return CULDA_OK;
}

extern "C" int64_t culda_encoder_tensor_size(const culda_encoder *e, int32_t which) {
    if (!e) return CULDA_ERR_INVALID_ARG;
    const int t = which >= CULDA_ENC_GRAD ? which - CULDA_ENC_GRAD : which;
    if (t < 0 || t >= kNumTensors) return CULDA_ERR_INVALID_ARG;
    return e->off[t + 1] - e->off[t];
}

extern "C" int culda_encoder_get_tensor(culda_encoder *e, int32_t which, float *host) {
    const int64_t n = culda_encoder_tensor_size(e, which);
    if (n < 0 || !host) return fail_enc(CULDA_ERR_INVALID_ARG, "culda_encoder_get_tensor: %s", "bad tensor");
    ECK(cudaSetDevice(e->device));
    const float *src = which >= CULDA_ENC_GRAD ? e->grad(which - CULDA_ENC_GRAD) : e->tensor(which);
    ECK(cudaMemcpy(host, src, sizeof(float) * (size_t)n, cudaMemcpyDeviceToHost));
    return CULDA_OK;
}

extern "C" int culda_encoder_set_tensor(culda_encoder *e, int32_t which, const float *host) {
    const int64_t n = culda_encoder_tensor_size(e, which);
    if (n < 0 || !host || which >= CULDA_ENC_GRAD)
        return fail_enc(CULDA_ERR_INVALID_ARG, "culda_encoder_set_tensor: %s", "bad tensor");
    ECK(cudaSetDevice(e->device));
    ECK(cudaMemcpy(e->tensor(which), host, sizeof(float) * (size_t)n, cudaMemcpyHostToDevice));
    ECK(refresh_bf16(e, nullptr));
    ECK(cudaDeviceSynchronize());
    return CULDA_OK;
}

extern "C" int culda_encoder_forward(culda_encoder *e, int32_t batch, const int32_t *d_docs,
                                     const int64_t *d_doc_ptr, const int32_t *d_words, float *d_probs, void *stream) {
    if (!e || !d_probs) return fail_enc(CULDA_ERR_INVALID_ARG, "culda_encoder_forward: %s", "null argument");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int rc = encoder_pass(e, batch, d_docs, d_doc_ptr, d_words, nullptr, false, d_probs, s);
    if (rc) return rc;
    return encoder_take_loss(e, 0, nullptr, s);
}

static int backward_call(culda_encoder *e, int32_t batch, const int32_t *d_docs, const int64_t *d_doc_ptr,
                         const int32_t *d_words, const float *d_target, double *loss, void *stream, bool update) {
    if (!e || !d_target) return fail_enc(CULDA_ERR_INVALID_ARG, "culda_encoder_backward: %s", "null argument");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    EncoderTarget t;
    t.dense = d_target;
    int rc = encoder_pass(e, batch, d_docs, d_doc_ptr, d_words, &t, update, nullptr, s);
    if (rc) return rc;
    return encoder_take_loss(e, batch, loss, s);
}

extern "C" int culda_encoder_backward(culda_encoder *e, int32_t batch, const int32_t *d_docs,
                                      const int64_t *d_doc_ptr, const int32_t *d_words, const float *d_target,
                                      double *loss, void *stream) {
    return backward_call(e, batch, d_docs, d_doc_ptr, d_words, d_target, loss, stream, false);
}

extern "C" int culda_encoder_train_step(culda_encoder *e, int32_t batch, const int32_t *d_docs,
                                        const int64_t *d_doc_ptr, const int32_t *d_words, const float *d_target,
                                        double *loss, void *stream) {
    return backward_call(e, batch, d_docs, d_doc_ptr, d_words, d_target, loss, stream, true);
}
