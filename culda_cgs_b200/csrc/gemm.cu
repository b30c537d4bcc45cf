// gemm.cu — BF16 GEMM on the sm_100a tensor cores for the document encoder:
// C[M x N] = A[M x K] * B[N x K]^T, both operands K-major (row-major with K
// contiguous), FP32 accumulation in tensor memory, with the encoder's
// epilogues fused: FP32 store, bias + GELU (pre-activation kept, activation
// stored in BF16 both as is and transposed), and the GELU backward (times
// GELU'(pre), BF16 out and transposed, bias-gradient column sums).
//
// One CTA of 128 threads per 128 x 128 output tile (and per K slice when the
// K range is split), two CTAs resident per SM so one tile's epilogue runs
// while the other's MMAs do.  Warp 0 lane 0 streams
// 128 x 64 tiles of A and B into a 3-stage shared-memory ring with TMA
// (128-byte swizzle); warp 1 lane 0 issues tcgen05.mma (M = 128, N = 128,
// K = 16 per instruction) into 128 TMEM columns and frees each stage with
// tcgen05.commit; when the last MMA has landed all four warps read their 32
// TMEM lanes back with tcgen05.ld into a shared-memory copy of the tile, and
// the epilogue writes it out row by row (coalesced) and, for the transposed
// BF16 copy and the column sums, column by column.  Every mbarrier wait
// is bounded: a wait that gives up sets kErrTimeout in the error word and the
// tile is not stored.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <mutex>

#include "gemm.cuh"
#include "internal.h"
#include "umma.cuh"

namespace culda {

namespace {

constexpr int kBM = 128, kBN = 128, kBK = 64, kStages = 3;
constexpr int kTileBytes = kBM * kBK * 2;  // 16 KB; the B tile (kBN rows) is the same size
constexpr int kGemmThreads = 128;
constexpr size_t kGemmSmem = (size_t)kStages * 2 * kTileBytes + 1024;  // + alignment slack

__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }

__device__ __forceinline__ float gelu_grad(float x) {
    const float cdf = 0.5f * (1.0f + erff(x * 0.70710678118654752f));
    const float pdf = 0.39894228040143268f * __expf(-0.5f * x * x);
    return cdf + x * pdf;
}

// The accumulator tile is staged in shared memory (the operand ring is free
// once the last MMA has landed) as S[128][kSP] floats, row = output row; the
// stride of 129 keeps both a lane-per-row write and a lane-per-row column read
// free of bank conflicts.  Phase 1 (rows): each warp takes rows w, w+4, ...,
// each lane 4 consecutive columns, so every global row store or load is one
// 512-byte (FP32) or 256-byte (BF16) run.  Phase 2 (columns, BF16 epilogues):
// each warp takes columns, each lane rows l, l+32, l+64, l+96 of the column,
// for the transposed copy and the bias-gradient column sums.
constexpr int kSP = kBN + 1;

template <int EPI>
__device__ __forceinline__ void epilogue_rows(const GemmEpilogue &ep, float *S, int m0, int n0, int warp, int lane) {
    const int c = 4 * lane;
    constexpr int kRowStep = kGemmThreads / 32, kAhead = 8;
    for (int r0 = warp; r0 < kBM; r0 += kRowStep * kAhead) {
        // the pre-activations of the next 8 rows are loaded before any of them
        // is stored: the stores below could alias them for all the compiler knows
        float4 pv[kAhead];
        if constexpr (EPI == kEpiGeluBwd) {
#pragma unroll
            for (int u = 0; u < kAhead; ++u)
                pv[u] = *reinterpret_cast<const float4 *>(ep.pre + (size_t)(m0 + r0 + kRowStep * u) * ep.ldo + n0 + c);
        }
#pragma unroll
        for (int u = 0; u < kAhead; ++u) {
        const int r = r0 + kRowStep * u;
        float v[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) v[i] = S[r * kSP + c + i];
        const size_t o = (size_t)(m0 + r) * ep.ldo + n0 + c;
        if constexpr (EPI == kEpiF32) {
            const bool with_bias = ep.bias && blockIdx.z == 0;
#pragma unroll
            for (int i = 0; i < 4; ++i) v[i] = v[i] * ep.alpha + (with_bias ? ep.bias[n0 + c + i] : 0.f);
            float4 *d = reinterpret_cast<float4 *>(ep.out_f32 + o);
            if (ep.k_splits > 1)
                atomicAdd(d, make_float4(v[0], v[1], v[2], v[3]));
            else
                *d = make_float4(v[0], v[1], v[2], v[3]);
        } else {
            if constexpr (EPI == kEpiBiasGelu) {
#pragma unroll
                for (int i = 0; i < 4; ++i) v[i] += ep.bias[n0 + c + i];
                *reinterpret_cast<float4 *>(ep.out_f32 + o) = make_float4(v[0], v[1], v[2], v[3]);
#pragma unroll
                for (int i = 0; i < 4; ++i) v[i] = gelu(v[i]);
            } else {  // kEpiGeluBwd
                const float4 pre = pv[u];
                v[0] *= gelu_grad(pre.x);
                v[1] *= gelu_grad(pre.y);
                v[2] *= gelu_grad(pre.z);
                v[3] *= gelu_grad(pre.w);
            }
            uint2 q;
            __nv_bfloat162 *h = reinterpret_cast<__nv_bfloat162 *>(&q);
            h[0] = __floats2bfloat162_rn(v[0], v[1]);
            h[1] = __floats2bfloat162_rn(v[2], v[3]);
            *reinterpret_cast<uint2 *>(ep.out_bf16 + o) = q;
            // the transposed copy and the column sums take the FP32 value: both
            // copies are the same single rounding of it to BF16
#pragma unroll
            for (int i = 0; i < 4; ++i) S[r * kSP + c + i] = v[i];
        }
        }
    }
}

template <int EPI>
__device__ __forceinline__ void epilogue_cols(const GemmEpilogue &ep, const float *S, int m0, int n0, int warp,
                                              int lane) {
    for (int cc = warp; cc < kBN; cc += kGemmThreads / 32) {
        float s = 0.f;
        __nv_bfloat16 *dst = ep.out_bf16_t + (size_t)(n0 + cc) * ep.ld_t + m0;
#pragma unroll
        for (int k = 0; k < kBM / 32; ++k) {
            const int r = lane + 32 * k;
            const float v = S[r * kSP + cc];
            dst[r] = __float2bfloat16_rn(v);
            s += v;
        }
        if (EPI == kEpiGeluBwd && ep.colsum) {
#pragma unroll
            for (int w = 16; w > 0; w >>= 1) s += __shfl_xor_sync(0xffffffffu, s, w);
            if (lane == 0) atomicAdd(ep.colsum + n0 + cc, s);
        }
    }
}

template <int EPI>
__global__ void __launch_bounds__(kGemmThreads, 2)
    gemm_bf16_kernel(const __grid_constant__ CUtensorMap tma_a, const __grid_constant__ CUtensorMap tma_b, int K,
                     const GemmEpilogue ep, int32_t *error) {
    extern __shared__ uint8_t gsm_raw[];
    __shared__ __align__(8) uint64_t full[kStages], empty[kStages], done;
    __shared__ uint32_t tmem_slot;
    __shared__ int abort_flag;

    const uint32_t raw = umma::smem_u32(gsm_raw);
    uint8_t *base = gsm_raw + ((1024u - (raw & 1023u)) & 1023u);  // 1024-byte aligned for the swizzle
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.y * kBM, n0 = blockIdx.x * kBN;
    // this CTA's K slice: k-blocks [kb0, kb0 + nk)
    const int nk_all = K / kBK;
    const int kb0 = (int)(((int64_t)nk_all * blockIdx.z) / gridDim.z);
    const int nk = (int)(((int64_t)nk_all * (blockIdx.z + 1)) / gridDim.z) - kb0;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) {
            umma::mbar_init(&full[s], 1);
            umma::mbar_init(&empty[s], 1);
        }
        umma::mbar_init(&done, 1);
        umma::mbar_fence_init();
        abort_flag = 0;
        umma::tma_prefetch_map(&tma_a);
        umma::tma_prefetch_map(&tma_b);
    }
    if (warp == 0) {
        umma::tmem_alloc(&tmem_slot, kBN);
        umma::tmem_relinquish();
    }
    umma::tc_fence_before();
    __syncthreads();
    umma::tc_fence_after();
    const uint32_t tmem = tmem_slot;

    if (warp == 0) {
        if (lane == 0) {  // TMA producer
            for (int kb = 0; kb < nk; ++kb) {
                const int s = kb % kStages;
                if (kb >= kStages && !umma::mbar_wait(&empty[s], (uint32_t)((kb / kStages) - 1) & 1u)) {
                    if (error) atomicOr(error, kErrTimeout);
                    atomicExch(&abort_flag, 1);
                    break;
                }
                umma::mbar_arrive_expect_tx(&full[s], 2u * kTileBytes);
                umma::tma_load_2d(base + (size_t)s * kTileBytes, &tma_a, (kb0 + kb) * kBK, m0, &full[s]);
                umma::tma_load_2d(base + (size_t)(kStages + s) * kTileBytes, &tma_b, (kb0 + kb) * kBK, n0, &full[s]);
            }
        }
        __syncwarp();
    } else if (warp == 1) {
        if (lane == 0) {  // MMA issuer
            constexpr uint32_t idesc = umma::idesc_bf16_f32(kBM, kBN);
            for (int kb = 0; kb < nk; ++kb) {
                const int s = kb % kStages;
                if (!umma::mbar_wait(&full[s], (uint32_t)(kb / kStages) & 1u)) {
                    if (error) atomicOr(error, kErrTimeout);
                    atomicExch(&abort_flag, 1);
                    break;
                }
                umma::tc_fence_after();
                const uint64_t ad = umma::sdesc_k_sw128(base + (size_t)s * kTileBytes);
                const uint64_t bd = umma::sdesc_k_sw128(base + (size_t)(kStages + s) * kTileBytes);
#pragma unroll
                for (int j = 0; j < kBK / 16; ++j)  // 16 BF16 = 32 bytes = 2 descriptor units per step
                    umma::mma_bf16(tmem, ad + 2u * j, bd + 2u * j, idesc, (kb | j) != 0 ? 1u : 0u);
                umma::mma_commit(&empty[s]);
            }
            umma::mma_commit(&done);  // arrives once every MMA issued above has completed
        }
        __syncwarp();
    }

    // epilogue: warp w owns TMEM lanes 32w .. 32w+31 = output rows m0+32w ..;
    // the decision to store is the same in every thread (barrier, then the flag)
    bool ok = umma::mbar_wait(&done, 0u);
    umma::tc_fence_after();
    if (!__all_sync(0xffffffffu, ok) && lane == 0 && error) atomicOr(error, kErrTimeout);
    const bool go = __syncthreads_and(ok) && !*(volatile int *)&abort_flag;
    if (go) {
        float *S = reinterpret_cast<float *>(base);  // the operand ring, free now: every MMA has landed
        const int r = warp * 32 + lane;
        for (int c = 0; c < kBN; c += 16) {
            float v[16];
            umma::tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c, v);
#pragma unroll
            for (int i = 0; i < 16; ++i) S[r * kSP + c + i] = v[i];
        }
        __syncthreads();
        epilogue_rows<EPI>(ep, S, m0, n0, warp, lane);
        if (EPI != kEpiF32) {
            __syncthreads();
            epilogue_cols<EPI>(ep, S, m0, n0, warp, lane);
        }
    }
    umma::tc_fence_before();
    __syncthreads();
    if (warp == 0) umma::tmem_dealloc(tmem, kBN);
}

// ------------------------------------------------------------ tensor maps
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    });
    return fn;
}

// A row-major BF16 matrix [rows x cols] with row stride ld elements, read in
// boxes of 128 rows x 64 columns with 128-byte swizzle.
cudaError_t make_map(CUtensorMap *map, const void *ptr, int rows, int cols, int ld) {
    EncodeTiledFn fn = encode_fn();
    if (!fn) return cudaErrorNotSupported;
    const cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)ld * 2u};
    const cuuint32_t box[2] = {(cuuint32_t)kBK, (cuuint32_t)kBM};
    const cuuint32_t estr[2] = {1u, 1u};
    const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void *>(ptr), dims, strides, box, estr,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

template <int EPI>
cudaError_t launch(const CUtensorMap &a, const CUtensorMap &b, int M, int N, int K, const GemmEpilogue &ep,
                   int32_t *error, cudaStream_t s) {
    static std::once_flag once;
    static cudaError_t attr = cudaSuccess;
    std::call_once(once, [] {
        attr = cudaFuncSetAttribute(gemm_bf16_kernel<EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)kGemmSmem);
    });
    if (attr != cudaSuccess) return attr;
    gemm_bf16_kernel<EPI><<<dim3(N / kBN, M / kBM, ep.k_splits), kGemmThreads, kGemmSmem, s>>>(a, b, K, ep, error);
    return cudaGetLastError();
}

bool aligned16(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

}  // namespace

const char *gemm_check(int M, int N, int K, const void *A, int lda, const void *B, int ldb, int epi,
                       const GemmEpilogue &ep) {
    if (M <= 0 || N <= 0 || K <= 0 || M % kBM || N % kBN || K % kBK) return "M, N must be multiples of 128, K of 64";
    if (!A || !B || !aligned16(A) || !aligned16(B)) return "A and B must be 16-byte aligned device pointers";
    if (lda < K || ldb < K || lda % 8 || ldb % 8) return "lda, ldb must be >= K and multiples of 8";
    if (ep.ldo < N || ep.ldo % 4) return "ldo must be >= N and a multiple of 4";
    if (ep.k_splits < 1 || ep.k_splits > K / kBK) return "k_splits must be in 1..K/64";
    if (ep.k_splits > 1 && epi != kEpiF32) return "split-K needs the F32 epilogue";
    switch (epi) {
        case kEpiF32:
            if (!ep.out_f32 || !aligned16(ep.out_f32)) return "F32 epilogue needs a 16-byte aligned out_f32";
            break;
        case kEpiBiasGelu:
            if (!ep.out_f32 || !ep.out_bf16 || !ep.out_bf16_t || !ep.bias) return "bias+GELU epilogue: null output";
            if (!aligned16(ep.out_f32) || !aligned16(ep.out_bf16) || ep.ldo % 8) return "bias+GELU epilogue: alignment";
            if (ep.ld_t < M) return "ld_t must be >= M";
            break;
        case kEpiGeluBwd:
            if (!ep.pre || !ep.out_bf16 || !ep.out_bf16_t) return "GELU backward epilogue: null operand";
            if (!aligned16(ep.pre) || !aligned16(ep.out_bf16) || ep.ldo % 8) return "GELU backward epilogue: alignment";
            if (ep.ld_t < M) return "ld_t must be >= M";
            break;
        default:
            return "unknown epilogue";
    }
    return nullptr;
}

cudaError_t gemm_bf16_nt(int M, int N, int K, const void *A, int lda, const void *B, int ldb, int epi,
                         const GemmEpilogue &ep, int32_t *error, cudaStream_t s) {
    if (gemm_check(M, N, K, A, lda, B, ldb, epi, ep)) return cudaErrorInvalidValue;
    CUtensorMap ma, mb;
    cudaError_t e = make_map(&ma, A, M, K, lda);
    if (e != cudaSuccess) return e;
    e = make_map(&mb, B, N, K, ldb);
    if (e != cudaSuccess) return e;
    switch (epi) {
        case kEpiF32: return launch<kEpiF32>(ma, mb, M, N, K, ep, error, s);
        case kEpiBiasGelu: return launch<kEpiBiasGelu>(ma, mb, M, N, K, ep, error, s);
        default: return launch<kEpiGeluBwd>(ma, mb, M, N, K, ep, error, s);
    }
}

}  // namespace culda
