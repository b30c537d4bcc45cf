// device_util.cuh — device helpers shared by the sampler and the rebuild kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace culda {

// Neumaier-compensated accumulation: s + c carries the running sum.  Both
// error terms are formed and one selected, so lanes that take different sides
// do not diverge.
__device__ __forceinline__ void neumaier(float &s, float &c, float x) {
    const float t = s + x;
    const float a = (s - t) + x, b = (x - t) + s;
    c += fabsf(s) >= fabsf(x) ? a : b;
    s = t;
}

// Lanes [g*G, g*G+G) of a warp cooperate on one token ("a group").
template <int G>
__device__ __forceinline__ unsigned group_mask(int lane) {
    if constexpr (G == 32)
        return 0xffffffffu;
    else
        return ((1u << G) - 1u) << (lane & ~(G - 1));
}

// Butterfly sum over the group's lanes; every lane ends with the same bits.
template <int G>
__device__ __forceinline__ float group_sum(float v, unsigned m) {
    if constexpr (G > 1) {
#pragma unroll
        for (int o = G / 2; o > 0; o >>= 1) v = __fadd_rn(v, __shfl_xor_sync(m, v, o));
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

// Opt a kernel into more than the default dynamic shared memory (the
// threshold leaves room for static shared memory).  Skipped while the stream
// is being captured into a graph: the context sets every attribute first.
inline cudaError_t allow_smem(const void *fn, size_t smem, cudaStream_t s) {
    if (smem <= 40 * 1024) return cudaSuccess;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (s && cudaStreamIsCapturing(s, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone) return cudaSuccess;
    return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

inline int grid_for(int64_t n) {
    int64_t b = (n + 255) / 256;
    return (int)(b < 1 ? 1 : (b > 148 * 32 ? 148 * 32 : b));
}

}  // namespace culda
