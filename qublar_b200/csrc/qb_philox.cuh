// Philox4x32-10 counter-based generator, written from J. K. Salmon,
// M. A. Moraes, R. O. Dror, D. E. Shaw, "Parallel random numbers: as easy as
// 1, 2, 3", SC'11, section 4 (the Philox S-box: two 32x32->64 multiplies per
// round, the high halves xor-ed with the other counter words and the round
// key, the round key bumped by the Weyl constants between rounds).
//
// The annealer keys it by the branch seed and counts by (bit, sweep): every
// Metropolis draw is a pure function of (seed, bit, sweep), so the parallel
// coloured sweep consumes the same numbers in any launch shape, and a CPU
// restatement can reproduce every decision. The reference instead consumes a
// sequential splitmix64 stream (ising_weighted.hpp:236-252), which ties draws
// to the sweep order.
#pragma once

#include <cstdint>

#ifndef QB_HD
#if defined(__CUDACC__)
#define QB_HD __host__ __device__ __forceinline__
#else
#define QB_HD inline
#endif
#endif

namespace qb {

struct Philox4 {
    uint32_t v[4];
};

QB_HD uint32_t mulhi32(uint32_t a, uint32_t b) {
#if defined(__CUDA_ARCH__)
    return __umulhi(a, b);
#else
    return uint32_t((uint64_t(a) * uint64_t(b)) >> 32);
#endif
}

QB_HD Philox4 philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
    for (int r = 0; r < 10; ++r) {
        const uint32_t hi0 = mulhi32(M0, c0), lo0 = M0 * c0;
        const uint32_t hi1 = mulhi32(M1, c2), lo1 = M1 * c2;
        const uint32_t n0 = hi1 ^ c1 ^ k0;
        const uint32_t n2 = hi0 ^ c3 ^ k1;
        c0 = n0;
        c1 = lo1;
        c2 = n2;
        c3 = lo0;
        k0 += W0;
        k1 += W1;
    }
    Philox4 o;
    o.v[0] = c0; o.v[1] = c1; o.v[2] = c2; o.v[3] = c3;
    return o;
}

// 53-bit uniform integer of the draw (seed, bit, sweep, stream): the top 53
// bits of words 1:0. u = u53 * 2^-53 in [0, 1), the resolution of the
// reference's uniform() (ising_weighted.hpp:242).
QB_HD uint64_t draw_u53(uint64_t seed, uint32_t bit, uint32_t sweep, uint32_t stream) {
    const Philox4 o = philox4x32_10(bit, sweep, stream, 0u, uint32_t(seed), uint32_t(seed >> 32));
    const uint64_t z = (uint64_t(o.v[1]) << 32) | uint64_t(o.v[0]);
    return z >> 11;
}

// Both halves of one draw block: *lo = draw_u53 (words 1:0), *hi = the top 53
// bits of words 3:2. Two replicas that share a key take one half each, so one
// Philox evaluation serves both.
QB_HD void draw_u53_pair(uint64_t seed, uint32_t bit, uint32_t sweep, uint32_t stream, uint64_t* lo, uint64_t* hi) {
    const Philox4 o = philox4x32_10(bit, sweep, stream, 0u, uint32_t(seed), uint32_t(seed >> 32));
    *lo = ((uint64_t(o.v[1]) << 32) | uint64_t(o.v[0])) >> 11;
    *hi = ((uint64_t(o.v[3]) << 32) | uint64_t(o.v[2])) >> 11;
}

// One half of a draw block: words 1:0 (half 0, = draw_u53) or words 3:2 (half 1).
QB_HD uint64_t draw_u53_half(uint64_t seed, uint32_t bit, uint32_t sweep, uint32_t stream, int half) {
    const Philox4 o = philox4x32_10(bit, sweep, stream, 0u, uint32_t(seed), uint32_t(seed >> 32));
    return half ? ((uint64_t(o.v[3]) << 32) | uint64_t(o.v[2])) >> 11
                : ((uint64_t(o.v[1]) << 32) | uint64_t(o.v[0])) >> 11;
}

// Integer-Ising replica pairing: replicas 2k and 2k + 1 of a solve share the
// Philox key base + 2k; 2k takes words 1:0 of each block and 2k + 1 words 3:2.
// A thread that carries both replicas of a pair evaluates one block for the two.
QB_HD uint64_t ising_pair_key(uint64_t base, uint32_t b) { return base + uint64_t(b & ~1u); }
QB_HD int ising_pair_half(uint32_t b) { return int(b & 1u); }

}  // namespace qb
