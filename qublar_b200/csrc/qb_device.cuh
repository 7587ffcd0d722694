// Device helpers shared by the cooperative-grid sweeps: acquire/release
// global accesses and the bounded grid barrier.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace qb {

constexpr unsigned kSpinLimit = 1u << 24;   // polls of a grid barrier before it reports a timeout

__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void red_release_gpu(unsigned* p, unsigned v) {
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Grid barrier of a cooperative launch: arrive, then poll the counter until
// every CTA of barrier round `round` has arrived. A poll limit turns a lost
// CTA into an error flag instead of a hang; every CTA then leaves its loops.
// per_round: arrivals that complete a round (0 = gridDim.x); limit: polls
// before giving up.
__device__ __forceinline__ bool grid_barrier(unsigned* bar, int* err, unsigned round, unsigned per_round = 0,
                                             unsigned limit = kSpinLimit) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned target = round * (per_round ? per_round : gridDim.x);
        red_release_gpu(bar, 1u);
        unsigned spins = 0;
        int ok = 1;
        while (ld_acquire_gpu(bar) < target) {
            if (++spins > limit || *reinterpret_cast<volatile int*>(err)) {
                atomicExch(err, 1);
                ok = 0;
                break;
            }
        }
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// The two halves of grid_barrier, so a CTA can work between its arrival and
// the wait: grid_arrive after the CTA's last write of the phase, grid_wait
// before its first read of the next phase. Every thread calls both.
__device__ __forceinline__ void grid_arrive(unsigned* bar) {
    __syncthreads();
    if (threadIdx.x == 0) red_release_gpu(bar, 1u);
}

__device__ __forceinline__ bool grid_wait(unsigned* bar, int* err, unsigned round, unsigned per_round = 0,
                                          unsigned limit = kSpinLimit) {
    __shared__ int s_ok2;
    if (threadIdx.x == 0) {
        const unsigned target = round * (per_round ? per_round : gridDim.x);
        unsigned spins = 0;
        int ok = 1;
        while (ld_acquire_gpu(bar) < target) {
            if (++spins > limit || *reinterpret_cast<volatile int*>(err)) {
                atomicExch(err, 1);
                ok = 0;
                break;
            }
        }
        s_ok2 = ok;
    }
    __syncthreads();
    return s_ok2 != 0;
}

// grid_wait with two pollers: lane 0 of warp 0 and, 400 ns later, lane 0 of
// warp 1 poll the counter, so the counter is sampled twice per L2 round trip
// and a completed barrier is seen sooner (on a B200 the lockstep pyramid
// sweep went 369 -> 356 ms; three pollers were slower: the polls crowd the
// counter's cache line). The first to see the target writes the round into
// *seen, which ends the other's loop; *seen starts at 0 and *fail at 0 in
// the kernel's prologue. Each poller gives up after `limit` polls.
__device__ __forceinline__ bool grid_wait2(unsigned* bar, int* err, unsigned round, unsigned per_round, unsigned limit,
                                           unsigned* seen, int* fail) {
    const int w = int(threadIdx.x >> 5);
    if ((threadIdx.x & 31) == 0 && w < 2) {
        const unsigned target = round * (per_round ? per_round : gridDim.x);
        if (w > 0) __nanosleep(400u);
        unsigned spins = 0;
        for (;;) {
            if (*reinterpret_cast<volatile unsigned*>(seen) == round) break;
            if (ld_acquire_gpu(bar) >= target) {
                *reinterpret_cast<volatile unsigned*>(seen) = round;
                break;
            }
            if (++spins > limit || *reinterpret_cast<volatile int*>(err)) {
                atomicExch(err, 1);
                *reinterpret_cast<volatile int*>(fail) = 1;
                *reinterpret_cast<volatile unsigned*>(seen) = round;
                break;
            }
        }
    }
    __syncthreads();
    return *reinterpret_cast<volatile int*>(fail) == 0;
}

// The Metropolis test of an uphill move, u53 * 2^-53 < exp(-dE / T) with the
// quotient and the exp in fp64, settled in fp32 when the two sides are far
// apart. With x = fp32(dE) * inv_T (inv_T = fp32 1/T, dE > 0), p =
// __expf(-x) is within a relative (2 + 2.2 x) 2^-23 of exp(-dE / T) wherever
// it is a normal number: the two roundings of the argument cost x 2^-23, and
// __expf's documented error is 2 + 1.173 |x| ulp (an ulp is at most 2^-23 of
// a normal result). u = fp32(hi) * 2^-32 (hi = the draw's top 32 bits) is at
// most 2^-32 + u 2^-24 below u53 * 2^-53 and at most u 2^-24 above it. With
// r = (8 + 4 x) 2^-23, which covers both and the roundings of the tests
// themselves, u + 2^-32 < p (1 - r) proves acceptance and u > p (1 + r)
// proves rejection (also after p underflows: a draw of 2^-32 or more exceeds
// exp(-87)). A zero draw, non-finite values and the narrow band between take
// the fp64 test, so the outcome is always the fp64 test's. The band is narrow
// because a class step waits for the slowest of its warps: a wide band sends
// some warp of nearly every step through the fp64 division and exp.
// The fp32 part: 1 accept, 0 reject, -1 undecided (the fp64 test decides).
__device__ __forceinline__ int uphill_fast(uint64_t u53, float dE, float inv_T) {
    const float u = __uint2float_rn(uint32_t(u53 >> 21)) * 0x1p-32f;
    const float x = dE * inv_T;
    const float p = __expf(-x);
    const float r = __fmaf_rn(4.0f, x, 8.0f) * 0x1p-23f;
    if (u + 0x1p-32f < p * (1.0f - r)) return 1;
    if (u > p * (1.0f + r)) return 0;
    return -1;
}
__device__ __forceinline__ bool uphill_accept(uint64_t u53, double dE, double T, float inv_T) {
    const int f = uphill_fast(u53, float(dE), inv_T);
    return f >= 0 ? f != 0 : double(u53) * 0x1.0p-53 < exp(-dE / T);
}

// ---- compensated residuals of the residual-form sweeps ----------------------------
//
// A branch's state per ray b is the scaled residual rho_b = s_b (sum_v a_bv x_v
// - d_b) with s_b = sqrt|w_b|, carried as an fp32 pair hi + lo. A bit-ray
// entry holds the fp32 coefficient a' = fp32(s_b a) (one rounding of the fp64
// product), so a flip changes rho_b by exactly +-a' and the TwoSum below keeps
// hi + lo equal to the running sum up to the rounding of lo. A bit's data term
// is sum_k sign(w_k) a'_k rho_k = sum_k w_k a_k r_k of local_field_dE
// (src/ising_recon.hpp:105-118) with r = rho / s.

// a' = fp32(sqrt|w| * a), the fp64 product rounded once.
__device__ __forceinline__ float scaled_coef(double sw, float a) { return __double2float_rn(__dmul_rn(sw, double(a))); }

// The fp32 pair (hi, lo) nearest an fp64 value: hi = fp32(v), lo = fp32(v - hi).
__device__ __forceinline__ float2 split_pair(double v) {
    const float hi = __double2float_rn(v);
    return make_float2(hi, __double2float_rn(__dsub_rn(v, double(hi))));
}

// hi + lo += v: TwoSum of hi and v, its rounding error added into lo.
__device__ __forceinline__ float2 two_sum_add(float2 p, float v) {
    const float s = __fadd_rn(p.x, v);
    const float bp = __fsub_rn(s, p.x);
    const float e = __fadd_rn(__fsub_rn(p.x, __fsub_rn(s, bp)), __fsub_rn(v, bp));
    return make_float2(s, __fadd_rn(p.y, e));
}

// Raises a kernel's dynamic shared-memory limit to the device maximum (the
// opt-in per-block size less the kernel's static shared memory). Every launcher
// sets the same value, so planning threads that check occupancy while others
// launch all see one limit; the launch itself passes the bytes it needs.
template <typename K>
inline cudaError_t allow_max_smem(K* kern) {
    int dev = 0, optin = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cudaFuncAttributes fa{};
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, kern);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - int(fa.sharedSizeBytes));
    return e;
}

}  // namespace qb
