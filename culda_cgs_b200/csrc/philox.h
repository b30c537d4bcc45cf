// philox.h — Philox4x32-10 counter-based RNG for host and device.
//
// Written from the construction in Salmon, Moraes, Dror and Shaw, "Parallel
// Random Numbers: As Easy as 1, 2, 3" (SC'11): ten rounds of the 4x32 S-box
// (two 32x32->64 multiplies by 0xD2511F53 and 0xCD9E8D57, the high halves
// xored with the other two words and the round key) and a Weyl key schedule
// (+0x9E3779B9, +0xBB67AE85).  Replaces the reference's cuRAND XORWOW states
// (src_culda/kernel/lda_train_kernel.cu:14-18,141), which are seeded from
// clock() and shared by the 32 warps of a block: a counter-based generator
// needs no state, so every token's uniform is a pure function of
// (seed, token, iteration) and runs are replayable.
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define CULDA_HD __host__ __device__ __forceinline__
#else
#define CULDA_HD inline
#endif

namespace culda {

struct u32x4 {
    uint32_t x, y, z, w;
};

CULDA_HD void mul_hi_lo(uint32_t a, uint32_t b, uint32_t &hi, uint32_t &lo) {
#if defined(__CUDA_ARCH__)
    lo = a * b;
    hi = __umulhi(a, b);
#else
    uint64_t p = (uint64_t)a * (uint64_t)b;
    hi = (uint32_t)(p >> 32);
    lo = (uint32_t)p;
#endif
}

CULDA_HD u32x4 philox4x32_10(u32x4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        uint32_t hi0, lo0, hi1, lo1;
        mul_hi_lo(0xD2511F53u, c.x, hi0, lo0);
        mul_hi_lo(0xCD9E8D57u, c.z, hi1, lo1);
        u32x4 n;
        n.x = hi1 ^ c.y ^ k0;
        n.y = lo1;
        n.z = hi0 ^ c.w ^ k1;
        n.w = lo0;
        c = n;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return c;
}

// Counter layout used everywhere in this library:
//   {token index low, token index high, iteration, purpose}
// The counter's last word: one independent stream per use.
enum : uint32_t {
    kPurposeSample = 0u,    // plain CGS draw
    kPurposeInit = 1u,      // initial topics
    kPurposeProposal = 2u,  // Metropolis-Hastings proposals and acceptances
    kPurposeAccept = 3u,
    kPurposeWeights = 4u,   // encoder weight initialisation
    kPurposeShuffle = 5u,   // encoder training batch order
    kPurposeWarm = 6u,      // encoder warm start of new documents' topics
    kPurposeMH = 16u        // Metropolis-Hastings step j of an iteration uses kPurposeMH + j
};

// All four words of one Philox block.
CULDA_HD u32x4 philox_token4(uint64_t seed, uint64_t token, uint32_t iteration, uint32_t purpose) {
    u32x4 c = {(uint32_t)token, (uint32_t)(token >> 32), iteration, purpose};
    return philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
}

CULDA_HD uint32_t philox_token(uint64_t seed, uint64_t token, uint32_t iteration, uint32_t purpose) {
    u32x4 c = {(uint32_t)token, (uint32_t)(token >> 32), iteration, purpose};
    return philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32)).x;
}

// Uniform in (0,1) with 24 significant bits: (2*(x>>9)+1) * 2^-24.  Exact in
// float and double, never 0 or 1.
CULDA_HD float uniform_from_bits(uint32_t x) { return (float)(((x >> 9) << 1) | 1u) * 5.9604644775390625e-08f; }

// floor(x * n / 2^32): an unbiased-for-powers-of-two map of 32 random bits to [0, n).
CULDA_HD uint32_t bounded_from_bits(uint32_t x, uint32_t n) { return (uint32_t)(((uint64_t)x * (uint64_t)n) >> 32); }

}  // namespace culda
