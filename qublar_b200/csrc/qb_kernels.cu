// sm_100a kernels of the annealer.
//
// Integer Ising / Max-Cut (replaces anneal_kernel, src/ising_gpu.cuh:166-254):
//   one CTA anneals one replica; its int32 fields and int8 spins sit in shared
//   memory (global scratch for large n). A sweep walks the colour classes; all
//   bits of a class are proposed at once, the accepted ones push
//   f_j -= 2 w_ij s_i to their neighbours (integer shared-memory atomics: the
//   sum is order-free, so the result is deterministic), and the CTA barrier
//   separates classes. Fields and energies stay exact integers as in
//   wising::State (src/ising_weighted.hpp:193-223).
//
// Residual form (replaces anneal_branch, src/ising_recon.hpp:121-144):
//   one thread-block cluster anneals one branch. The branch's weighted
//   residuals rw_b = w_b (sum_v a_bv x_v - d_b) live in the cluster's
//   distributed shared memory (ray b on CTA b % CL), its bits on the CTA that
//   evaluates them. A bit's score is dE = delta (lin + h) + q + lambda (deg -
//   2 unlike) with h = sum_k a_k rw_k (an fmaf chain over its rays in order)
//   and q = 1/2 sum_k w a_k^2 -- the local_field_dE of
//   src/ising_recon.hpp:105-118 regrouped; an accepted flip scatters
//   rw += w a delta. A class never holds two bits of one ray, so the scatter
//   needs no atomics; a cluster barrier separates classes. Residuals are fp32
//   and are recomputed from scratch in fp64 every `refresh` sweeps.
//
// Metropolis (both forms): accept if dE <= 0, else if u < exp(-dE/T) in
// double, u the 53-bit Philox draw of (branch seed, original bit, sweep) --
// the acceptance expression of ising_weighted.hpp:260 / ising_recon.hpp:136.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <algorithm>
#include <cstring>
#include <mutex>
#include <vector>

#include "qb_device.cuh"
#include "qb_kernels.hpp"
#include "qb_philox.cuh"

namespace cg = cooperative_groups;

namespace qb {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kIsingThreads = 512;
constexpr int kResidThreads = 512;
constexpr int kGroup = 8;       // lanes per bit in the residual sweep
constexpr int kHeavy = 64;      // bits with more rays take a full warp
constexpr int kChunkB = 1024;   // stage bits per chunk
constexpr int kChunkE = 4096;   // stage entries per chunk
constexpr int kChunkN = 6144;   // stage neighbour entries per chunk
constexpr uint32_t kSlotBits = 27;
constexpr uint32_t kSlotMask = (1u << kSlotBits) - 1u;

__device__ __forceinline__ bool metropolis(double dE, double T, float inv_T, uint64_t seed, int half, uint32_t bit,
                                           uint32_t sweep) {
    if (dE <= 0.0) return true;
    return uphill_accept(draw_u53_half(seed, bit, sweep, 0u, half), dE, T, inv_T);
}

// ---- integer Ising ----------------------------------------------------------------

struct IsingArgs {
    int n;
    int n_colours;
    int sweeps;
    uint64_t seed0;
    const int32_t* class_ptr;
    const int32_t* row;
    const int32_t* adj;
    const void* w;
    const int32_t* f0;
    const int32_t* order;
    const double* temp;
    int32_t* f_scratch;   // R x n (global-state variant)
    int8_t* s_scratch;    // R x n
    int wide;             // rows long enough that a warp per accepted flip pays for a second barrier
    uint8_t* x_out;       // R x n
    int32_t* f_out;       // R x n
    long long* e_out;     // R
    long long* trace;     // nullable: R x sweeps tracked energies after each sweep (zeroed)
};

// Accepted bits of a class listed for the warp-wide neighbour update, used
// when some bit has at least kWideRow neighbours (a second barrier per class
// then pays for itself).
constexpr int kAccList = 1024;
constexpr int kWideRow = 24;

template <typename WT, bool SMEM>
__global__ void __launch_bounds__(kIsingThreads) ising_anneal_kernel(IsingArgs A) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ long long red[kIsingThreads / 32];
    __shared__ int2 acc_list[kAccList];   // (bit, -2 s_i mod 2^32) of the class's accepted flips
    __shared__ int acc_count[2];          // per class parity
    const int rep = int(blockIdx.x);
    const int n = A.n;
    int32_t* f;
    int8_t* s;
    if (SMEM) {
        f = reinterpret_cast<int32_t*>(smem);
        s = reinterpret_cast<int8_t*>(smem + size_t(n) * sizeof(int32_t));
    } else {
        f = A.f_scratch + size_t(rep) * size_t(n);
        s = A.s_scratch + size_t(rep) * size_t(n);
    }
    for (int i = int(threadIdx.x); i < n; i += blockDim.x) {
        f[i] = A.f0[i];
        s[i] = -1;
    }
    if (threadIdx.x < 2) acc_count[threadIdx.x] = 0;
    __syncthreads();
    const uint64_t seed = ising_pair_key(A.seed0, uint32_t(rep));
    const int half = ising_pair_half(uint32_t(rep));
    const WT* w = static_cast<const WT*>(A.w);
    const int lane = int(threadIdx.x & 31u), warp = int(threadIdx.x >> 5), n_warps = int(blockDim.x >> 5);
    long long E = 0;
    int parity = 0;
    for (int sweep = 0; sweep < A.sweeps; ++sweep) {
        const double T = A.temp[sweep];
        const float inv_T = float(1.0 / T);
        for (int c = 0; c < A.n_colours; ++c, parity ^= 1) {
            const int c1 = A.class_ptr[c + 1];
            // 1. decide every bit of the class; with wide rows, list the
            // accepted flips, else update their neighbours at once
            for (int i = A.class_ptr[c] + int(threadIdx.x); i < c1; i += blockDim.x) {
                const int si = s[i];
                const long long dE = -(long long)si * (long long)f[i];
                if (metropolis(double(dE), T, inv_T, seed, half, uint32_t(A.order[i]), uint32_t(sweep))) {
                    s[i] = int8_t(-si);
                    E += dE;
                    // f_j -= 2 w_ij s_i, in wrap-around uint32 arithmetic: the
                    // final field fits int32 (|f| <= field bound), the term may not
                    const uint32_t ms = si > 0 ? 0xFFFFFFFEu : 2u;   // -2 s_i mod 2^32
                    const int slot = A.wide ? atomicAdd(&acc_count[parity], 1) : kAccList;
                    if (slot < kAccList) {
                        acc_list[slot] = make_int2(i, int(ms));
                    } else {   // narrow rows or a full list: update the neighbours here
                        const int r1 = A.row[i + 1];
                        for (int k = A.row[i]; k < r1; ++k)
                            atomicAdd(reinterpret_cast<unsigned int*>(&f[A.adj[k]]), uint32_t(int32_t(w[k])) * ms);
                    }
                }
            }
            __syncthreads();
            if (!A.wide) continue;
            // 2. a warp per accepted flip, its lanes over the bit's neighbours
            // (integer sums: the order of the atomics does not matter)
            const int na = min(acc_count[parity], kAccList);
            for (int q = warp; q < na; q += n_warps) {
                const int2 e = acc_list[q];
                const int r1 = A.row[e.x + 1];
                for (int k = A.row[e.x] + lane; k < r1; k += 32)
                    atomicAdd(reinterpret_cast<unsigned int*>(&f[A.adj[k]]), uint32_t(int32_t(w[k])) * uint32_t(e.y));
            }
            __syncthreads();
            if (threadIdx.x == 0) acc_count[parity] = 0;   // reused two classes later, after two barriers
        }
        if (A.trace) {   // the tracked energy after this sweep: each warp adds its threads' running sums
            long long Ew = E;
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) Ew += __shfl_xor_sync(kFull, Ew, off);
            if (lane == 0 && Ew != 0)
                atomicAdd(reinterpret_cast<unsigned long long*>(&A.trace[size_t(rep) * A.sweeps + sweep]),
                          (unsigned long long)Ew);
        }
    }
    for (int i = int(threadIdx.x); i < n; i += blockDim.x) {
        const size_t o = size_t(rep) * size_t(n) + size_t(A.order[i]);
        A.x_out[o] = s[i] > 0 ? 1u : 0u;
        A.f_out[o] = f[i];
    }
    // fixed-shape block reduction: the sum of integers is exact anyway
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) E += __shfl_xor_sync(kFull, E, off);
    if ((threadIdx.x & 31u) == 0) red[threadIdx.x >> 5] = E;
    __syncthreads();
    if (threadIdx.x == 0) {
        long long t = 0;
        for (int q = 0; q < int(blockDim.x >> 5); ++q) t += red[q];
        A.e_out[rep] = t;
    }
}

// E = -sum_e w_e [x_u != x_v] per state over the edge list as given: the
// independent count of cut_of (ising_weighted.hpp:173-178) and
// oracle_kernel (ising_gpu.cuh:257-272).
__global__ void ising_energy_kernel(const int32_t* eu, const int32_t* ev, const int32_t* ew, int64_t m,
                                    const uint8_t* X, int n, long long* e) {
    const uint8_t* x = X + size_t(blockIdx.y) * size_t(n);
    long long acc = 0;
    for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < m; k += int64_t(gridDim.x) * blockDim.x)
        if (x[eu[k]] != x[ev[k]]) acc += ew[k];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(kFull, acc, off);
    if ((threadIdx.x & 31u) == 0 && acc != 0)
        atomicAdd(reinterpret_cast<unsigned long long*>(&e[blockIdx.y]), (unsigned long long)(-acc));
}

// ---- residual form ------------------------------------------------------------------

struct ResidArgs {
    int n;
    int n_rays;
    int sweeps;
    int refresh;
    int ray_slots;
    int bit_words;
    float lambda;
    uint64_t seed0;
    const int4* chunks;         // per CTA rank: 2 x int4 per chunk (see ResidualPlan)
    const int32_t* chunk_ptr;   // CL + 1
    const int32_t* row;
    const uint2* ent;           // per bit-ray entry: {ray | (w < 0) << 31, a' = fp32(sqrt|w| a)}
    const float* lin;
    const float* q;
    const int32_t* nbr_ptr;
    const uint32_t* nbr_home;
    const int32_t* order;
    const double* d;
    const double* w64;
    const int32_t* rrow;
    const uint32_t* rbit_home;
    const float* ra;
    const double* temp;
    uint8_t* x_out;
    float* drift;
    unsigned long long* accepts;
    double* trace;              // nullable: R x sweeps, the sum of accepted dE of each sweep
    unsigned long long* phase;  // PHASES builds: per CTA {gather, score, barrier, chunks} clock64 sums
};

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ uint32_t map_rank(uint32_t addr, uint32_t rank) {
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(addr), "r"(rank));
    return r;
}
__device__ __forceinline__ float2 ld_cluster_f32x2(uint32_t addr) {
    float2 v;
    asm volatile("ld.shared::cluster.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "r"(addr));
    return v;
}
__device__ __forceinline__ void st_cluster_f32x2(uint32_t addr, float2 v) {
    asm volatile("st.shared::cluster.v2.f32 [%0], {%1, %2};" ::"r"(addr), "f"(v.x), "f"(v.y));
}
__device__ __forceinline__ uint32_t ld_cluster_u32(uint32_t addr) {
    uint32_t v;
    asm volatile("ld.shared::cluster.u32 %0, [%1];" : "=r"(v) : "r"(addr));
    return v;
}
// The bit at home word h = (cta << 27) | slot, from any CTA of the cluster.
__device__ __forceinline__ uint32_t ld_home_bit(uint32_t xs_base, uint32_t h) {
    const uint32_t slot = h & kSlotMask;
    return (ld_cluster_u32(map_rank(xs_base + (slot >> 5) * 4u, h >> kSlotBits)) >> (slot & 31u)) & 1u;
}

__device__ __forceinline__ void prefetch_l2(const void* p, uint32_t bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// Shared memory of the residual sweep's stage buffers.
struct ResidStage {
    unsigned long long* u;   // kChunkB Philox draws (53-bit)
    float2* rv;              // kChunkE gathered residual pairs (hi, lo)
    int32_t* row;            // kChunkB + 1 entry offsets (chunk-relative)
    int32_t* nbp;            // kChunkB + 1 neighbour offsets (chunk-relative)
    float* lin;              // kChunkB
    float* q;                // kChunkB
    uint8_t* xn;             // kChunkN neighbour bits
};

// Score, decide and (on accept) scatter bit k of the chunk with a group of G
// lanes: lane l sums sign(w) a' * fp32(hi + lo) over entries l, l + G, ... as
// an fmaf chain, an xor butterfly joins the lanes (the oracle mirrors this
// order).
template <int CL, int G>
__device__ __forceinline__ bool score_bit(int k, int gl, unsigned gmask, int leader, const ResidStage& S,
                                          const uint2* ent, uint32_t rw_base, uint32_t* xs, int slot0, float lambda,
                                          double T, float inv_T, double* s_trace) {
    constexpr int kShift = CL == 1 ? 0 : CL == 2 ? 1 : CL == 4 ? 2 : CL == 8 ? 3 : 4;
    const int rs = S.row[k], re = S.row[k + 1], ns = S.nbp[k], ne = S.nbp[k + 1];
    float acc = 0.0f;
    for (int e = rs + gl; e < re; e += G) {
        const uint2 en = __ldg(&ent[e]);
        const float c = (en.x >> 31) ? -__uint_as_float(en.y) : __uint_as_float(en.y);
        acc = fmaf(c, __fadd_rn(S.rv[e].x, S.rv[e].y), acc);
    }
#pragma unroll
    for (int off = G / 2; off > 0; off >>= 1) acc = __fadd_rn(acc, __shfl_xor_sync(gmask, acc, off));
    const int slot = slot0 + k;
    const uint32_t xi = (xs[slot >> 5] >> (slot & 31)) & 1u;
    int unlike = 0;
    for (int j = ns + gl; j < ne; j += G) unlike += S.xn[j] != xi ? 1 : 0;
#pragma unroll
    for (int off = G / 2; off > 0; off >>= 1) unlike += __shfl_xor_sync(gmask, unlike, off);
    int accept = 0;
    if (gl == 0) {
        const float delta = xi ? -1.0f : 1.0f;
        const float t = __fadd_rn(S.lin[k], acc);
        const float prior = __fmul_rn(lambda, float((ne - ns) - 2 * unlike));
        const float dE = __fadd_rn(__fadd_rn(__fmul_rn(delta, t), S.q[k]), prior);
        accept = (dE <= 0.0f || uphill_accept(S.u[k], double(dE), T, inv_T)) ? 1 : 0;
        if (accept && s_trace) atomicAdd(s_trace, double(dE));
    }
    accept = __shfl_sync(gmask, accept, leader);
    if (accept) {
        const float dl = xi ? -1.0f : 1.0f;
        for (int e = rs + gl; e < re; e += G) {
            const uint2 en = __ldg(&ent[e]);
            const uint32_t ray = en.x & 0x7FFFFFFFu;
            const uint32_t ad = map_rank(rw_base + (ray >> kShift) * 8u, ray & (CL - 1));
            st_cluster_f32x2(ad, two_sum_add(S.rv[e], __fmul_rn(dl, __uint_as_float(en.y))));
        }
        if (gl == 0) atomicXor(&xs[slot >> 5], 1u << (slot & 31));
    }
    return accept != 0;
}

// One cluster anneals one branch. A colour class is worked through in chunks
// of this CTA's slice (<= kChunkB bits, <= kChunkE entries, <= kChunkN
// neighbour entries; the planner balances the slices and puts heavy bits
// first); per chunk:
//   1. every thread gathers into shared memory: the chunk's per-bit metadata,
//      the bits' Philox draws (pure arithmetic that overlaps the loads), the
//      entries' rw from the ray owners' shared memory and the neighbours'
//      bits, while the next chunk's entries are prefetched into L2;
//   2. heavy bits take a warp each, the others a kGroup-lane group: sum,
//      score, decide; an accepted bit writes rw + (w a) delta straight back to
//      the owners (no atomics: a class holds at most one bit of a ray) and
//      flips its own bit;
// and a cluster barrier closes the class.
template <int CL, bool PHASES>
__global__ void __launch_bounds__(kResidThreads, 2) resid_anneal_kernel(ResidArgs A) {
    static_assert((CL & (CL - 1)) == 0 && CL <= 16, "cluster size: a power of two <= 16");
    static_assert(kResidThreads % kGroup == 0 && 32 % kGroup == 0, "lane groups tile a warp");
    extern __shared__ __align__(16) unsigned char smem[];
    constexpr int kShift = CL == 1 ? 0 : CL == 2 ? 1 : CL == 4 ? 2 : CL == 8 ? 3 : 4;
    constexpr int kGroups = kResidThreads / kGroup;
    constexpr int kWarps = kResidThreads / 32;
    ResidStage S;
    S.u = reinterpret_cast<unsigned long long*>(smem);
    float2* rw = reinterpret_cast<float2*>(S.u + kChunkB);                   // (hi, lo) of rho per owned ray
    S.rv = rw + A.ray_slots;
    S.row = reinterpret_cast<int32_t*>(S.rv + kChunkE);
    S.nbp = S.row + (kChunkB + 1);
    S.lin = reinterpret_cast<float*>(S.nbp + (kChunkB + 1));
    S.q = S.lin + kChunkB;
    S.xn = reinterpret_cast<uint8_t*>(S.q + kChunkB);
    uint32_t* xs = reinterpret_cast<uint32_t*>(S.xn + kChunkN);             // owned bits, packed
    __shared__ unsigned long long s_acc_count;
    __shared__ double s_trace;   // accepted dE of this CTA's bits in the current sweep
    cg::cluster_group cluster = cg::this_cluster();
    const uint32_t rank = cluster.block_rank();
    const int branch = int(blockIdx.x) / CL;
    const int tid = int(threadIdx.x);
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const int gl = tid % kGroup;
    const int grp = tid / kGroup;
    const unsigned gmask = (kGroup == 32 ? kFull : ((1u << kGroup) - 1u)) << (lane & ~(kGroup - 1));
    const uint64_t seed = A.seed0 + uint64_t(branch);
    const uint32_t rw_base = smem_addr(rw);
    const uint32_t xs_base = smem_addr(xs);
    const int4* chunks = A.chunks + 2 * A.chunk_ptr[rank];
    const int n_chunks = A.chunk_ptr[rank + 1] - A.chunk_ptr[rank];

    for (int sl = tid; sl < A.ray_slots; sl += kResidThreads) {
        const int b = (sl << kShift) + int(rank);
        rw[sl] = b < A.n_rays ? split_pair(-__dmul_rn(sqrt(fabs(A.w64[b])), A.d[b])) : make_float2(0.0f, 0.0f);
    }
    for (int sl = tid; sl < A.bit_words; sl += kResidThreads) xs[sl] = 0u;
    if (tid == 0) {
        s_acc_count = 0;
        s_trace = 0.0;
    }
    cluster.sync();

    unsigned long long my_accepts = 0;
    long long ph_gather = 0, ph_score = 0, ph_bar = 0, ph_chunks = 0, t_ph = 0;
    for (int sweep = 0; sweep < A.sweeps; ++sweep) {
        if (A.refresh > 0 && sweep > 0 && sweep % A.refresh == 0) {
            // fp64 refresh of the owned residuals: rho_b = (sum over the
            // ray's set bits of a', in ray order) - sqrt|w_b| d_b
            float dmax = 0.0f;
            for (int sl = tid; sl < A.ray_slots; sl += kResidThreads) {
                const int b = (sl << kShift) + int(rank);
                if (b >= A.n_rays) continue;
                const double sw = sqrt(fabs(A.w64[b]));
                double acc = 0.0;
                const int k1 = A.rrow[b + 1];
                for (int k = A.rrow[b]; k < k1; ++k)
                    if (ld_home_bit(xs_base, A.rbit_home[k])) acc = __dadd_rn(acc, double(scaled_coef(sw, A.ra[k])));
                const double v = __dsub_rn(acc, __dmul_rn(sw, A.d[b]));
                dmax = fmaxf(dmax, __double2float_rn(fabs(__dsub_rn(__dadd_rn(double(rw[sl].x), double(rw[sl].y)), v))));
                rw[sl] = split_pair(v);
            }
            if (dmax > 0.0f) atomicMax(reinterpret_cast<int*>(&A.drift[branch]), __float_as_int(dmax));
            cluster.sync();
        }
        const double T = A.temp[sweep];
        const float inv_T = float(1.0 / T);
        for (int ci = 0; ci < n_chunks; ++ci) {
            const int4 c0 = chunks[2 * ci];       // b0, b1, slot of b0, last-of-class | heavy bits << 1
            const int4 c1 = chunks[2 * ci + 1];   // e0, e1, n0, n1
            const int nb = c0.y - c0.x;
            if (PHASES) t_ph = clock64();
            if (tid == 0) {   // the next chunk's entries into L2
                // a bulk prefetch starts on a 16-byte boundary and moves a
                // multiple of 16 bytes: whole entry pairs (the table carries
                // one spare pair at its end)
                const int nx = ci + 1 < n_chunks ? ci + 1 : 0;
                const int4 c1n = chunks[2 * nx + 1];
                const int p0 = c1n.x & ~1, p1 = (c1n.y + 1) & ~1;
                if (c1n.y > c1n.x) prefetch_l2(&A.ent[p0], uint32_t(p1 - p0) * 8u);
            }
            // 1. gather
            for (int k = tid; k <= nb; k += kResidThreads) {
                const int i = c0.x + k;
                S.row[k] = A.row[i] - c1.x;
                S.nbp[k] = A.nbr_ptr[i] - c1.z;
                if (k < nb) {
                    S.lin[k] = A.lin[i];
                    S.q[k] = A.q[i];
                    S.u[k] = draw_u53(seed, uint32_t(A.order[i]), uint32_t(sweep), 0u);
                }
            }
            for (int e0 = c1.x + tid; e0 < c1.y; e0 += 4 * kResidThreads) {
                uint32_t ray[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int e = e0 + u * kResidThreads;
                    ray[u] = e < c1.y ? (__ldg(&A.ent[e]).x & 0x7FFFFFFFu) : 0u;
                }
                float2 rv[4];
#pragma unroll
                for (int u = 0; u < 4; ++u)
                    rv[u] = e0 + u * kResidThreads < c1.y
                                ? ld_cluster_f32x2(map_rank(rw_base + (ray[u] >> kShift) * 8u, ray[u] & (CL - 1)))
                                : make_float2(0.0f, 0.0f);
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int e = e0 + u * kResidThreads;
                    if (e < c1.y) S.rv[e - c1.x] = rv[u];
                }
            }
            for (int j = c1.z + tid; j < c1.w; j += kResidThreads)
                S.xn[j - c1.z] = uint8_t(ld_home_bit(xs_base, A.nbr_home[j]));
            __syncthreads();
            if (PHASES) {
                const long long t1 = clock64();
                ph_gather += t1 - t_ph;
                t_ph = t1;
            }
            // 2. score, decide, scatter
            const uint2* ent = A.ent + c1.x;
            const int nh = c0.w >> 1;
            for (int k = warp; k < nh; k += kWarps)
                my_accepts += (score_bit<CL, 32>(k, lane, kFull, 0, S, ent, rw_base, xs, c0.z, A.lambda, T, inv_T,
                                                 A.trace ? &s_trace : nullptr) && lane == 0);
            for (int k = nh + grp; k < nb; k += kGroups)
                my_accepts += (score_bit<CL, kGroup>(k, gl, gmask, lane & ~(kGroup - 1), S, ent, rw_base, xs, c0.z,
                                                     A.lambda, T, inv_T, A.trace ? &s_trace : nullptr) && gl == 0);
            if (PHASES) {
                __syncthreads();
                const long long t1 = clock64();
                ph_score += t1 - t_ph;
                t_ph = t1;
            }
            if (c0.w & 1) cluster.sync();   // class done: its flips become visible cluster-wide
            else __syncthreads();           // stage buffers are reused by the next chunk
            if (PHASES) {
                ph_bar += clock64() - t_ph;
                ++ph_chunks;
            }
        }
        if (A.trace) {   // this CTA's part of the sweep's tracked energy change
            __syncthreads();
            if (tid == 0) {
                if (s_trace != 0.0) atomicAdd(&A.trace[size_t(branch) * A.sweeps + sweep], s_trace);
                s_trace = 0.0;
            }
        }
    }
    if (PHASES && tid == 0) {
        unsigned long long* ph = A.phase + 4 * size_t(blockIdx.x);
        ph[0] = ph_gather; ph[1] = ph_score; ph[2] = ph_bar; ph[3] = ph_chunks;
    }
    // branches out, original bit order
    for (int ci = 0; ci < n_chunks; ++ci) {
        const int4 c0 = chunks[2 * ci];
        for (int k = tid; k < c0.y - c0.x; k += kResidThreads) {
            const int slot = c0.z + k;
            A.x_out[size_t(branch) * size_t(A.n) + size_t(A.order[c0.x + k])] = uint8_t((xs[slot >> 5] >> (slot & 31)) & 1u);
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) my_accepts += __shfl_xor_sync(kFull, my_accepts, off);
    if (lane == 0 && my_accepts) atomicAdd(&s_acc_count, my_accepts);
    __syncthreads();
    if (tid == 0 && s_acc_count) atomicAdd(&A.accepts[branch], s_acc_count);
    cluster.sync();   // no CTA leaves while a peer may still read its shared memory
}

// ---- residual form, all branches in lockstep ------------------------------------------
//
// Every CTA of a co-resident (cooperative) grid takes a balanced slice of
// each colour class; a warp sums one 16-entry segment of a bit for 16 branches
// at once: lane l serves branch l % 16 and entries of parity l / 16, so one
// coalesced 128-byte load of rho[ray][16 branches] (hi, lo pairs) feeds 16
// branches. Residuals and bits live in global memory (L2-resident: 9.7 MB of
// residual pairs and 1.2 MB of bit words for the benchmark pyramid at 16
// branches); a bounded grid barrier closes each class. Branch b of a bit sums
// h = sum over its 16-entry segments in order of (the fmaf chain over the
// segment's even entries + the chain over its odd entries), each term
// c * fp32(hi + lo) with c = sign(w) a' (the oracle's "lockstep" order).

constexpr int kLockThreads = 1024;
constexpr int kLockE = 2048;   // staged entries per chunk
constexpr int kLockB = 256;    // staged bits per chunk
constexpr int kLockN = 1536;   // staged neighbour entries per chunk
constexpr int kSeg = 16;       // entries per segment: one warp, one batch of loads
constexpr int kLockSegs = kLockE / kSeg + kLockB;   // segments a chunk can hold
constexpr int kStageWarps = 2;                       // warps that stage the next chunk
constexpr int kLockMaxNG = 4;  // branch groups of 16 one launch serves (64 branches)
constexpr uint32_t kRayMask = 0x7FFFFFFFu;   // entry word 0: ray | (w < 0) << 31

struct ResidLockArgs {
    int n;
    int n_rays;
    int sweeps;
    int refresh;
    int R;              // branches
    int NG;             // groups of 16 branches
    float lambda;
    uint64_t seed0;
    const int4* chunks;         // per CTA: 2 x int4 per chunk {b0, b1, segments, last} {e0, e1, n0, n1}
    const int32_t* chunk_ptr;   // gridDim + 1
    const uint2* ent;           // {ray | (w < 0) << 31, a'} per bit-ray entry, sweep order
    const uint4* meta;          // per bit, 2 x uint4: {row start, rays, nbr start, nbrs} {lin, q, input index, first segment}
    const int32_t* nbr;         // sweep-order index of each neighbour
    const int32_t* order;
    const double* d;
    const double* w64;
    const int32_t* rrow;
    const int32_t* rbit;        // sweep-order bit of each ray-major entry
    const float* ra;
    const double* temp;
    float2* rp;                 // n_rays x (16 NG): (hi, lo) of every branch's scaled residual
    uint32_t* xb;               // n x NG: bit words, branch 16 g + l at bit l of word g
    unsigned* bar;              // grid barrier counter (zero at launch)
    int* err;                   // 1: a barrier timed out
    int* status;                // nullable: set to QB_ETIMEDOUT when a barrier times out
    unsigned bar_extra;         // arrivals a barrier round waits for beyond the grid (0; test hook)
    unsigned spin_limit;        // polls of a barrier before it gives up
    uint8_t* x_out;
    float* drift;
    unsigned long long* accepts;
    double* trace;              // nullable: R x sweeps, the sum of accepted dE of each sweep
    unsigned long long* phase;  // PHASES builds: per CTA {stage wait, items, barrier, chunks, A, A-C, C} clock64 sums
};

__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async4(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }

struct LockStage {
    uint2* ent;      // kLockE
    uint4* meta;     // 2 kLockB
    int32_t* nbr;    // kLockN
};

// Stage a chunk's entries, bit records and neighbour lists (async copies by
// threads t0, t0 + stride, ...; 16-byte copies for the entries where both ends
// allow, 8-byte ones at a chunk's odd edge).
__device__ __forceinline__ void lock_stage(const ResidLockArgs& A, const int4 c0, const int4 c1, const LockStage& S,
                                           int t0, int stride) {
    const int e0 = c1.x, e1 = c1.y;
    if ((e0 & 1) == 0) {
        for (int e = e0 + 2 * t0; e + 1 < e1; e += 2 * stride) cp_async16(&S.ent[e - e0], &A.ent[e]);
        if (((e1 - e0) & 1) && t0 == 0) cp_async8(&S.ent[e1 - 1 - e0], &A.ent[e1 - 1]);
    } else {
        for (int e = e0 + t0; e < e1; e += stride) cp_async8(&S.ent[e - e0], &A.ent[e]);
    }
    for (int k = 2 * c0.x + t0; k < 2 * c0.y; k += stride) cp_async16(&S.meta[k - 2 * c0.x], &A.meta[k]);
    for (int j = c1.z + t0; j < c1.w; j += stride) cp_async4(&S.nbr[j - c1.z], &A.nbr[j]);
}

// Every CTA of a cooperative grid works its chunk list (a balanced slice of
// each colour class); the next chunk's structure is staged in shared memory
// while the current one runs. Per chunk:
//   A. a warp sums one 16-entry segment of one bit for 16 branches and keeps
//      the (hi, lo) pairs it loaded (its first segment's); other warps count
//      each (bit, group)'s unlike neighbours;
//   B. a warp per (bit, group) adds the bit's segment sums in order, decides,
//      and records which branches flip;
//   C. the warps of phase A add delta a' into the flipped branches' pairs by
//      TwoSum and store them (a class touches a residual at most once, so
//      plain stores suffice and the result is deterministic).
// A bounded grid barrier closes each class.
template <bool PHASES, int NG>
__global__ void __launch_bounds__(kLockThreads, 1) resid_lockstep_kernel(ResidLockArgs A) {
    static_assert(NG >= 1 && NG <= kLockMaxNG, "16-branch groups: 1 .. kLockMaxNG");
    __shared__ unsigned s_seen_round;   // the last class barrier this CTA saw complete
    __shared__ int s_wait_fail;
    extern __shared__ __align__(16) unsigned char smem[];
    const int tid = int(threadIdx.x);
    const int lane = tid & 31;
    const int warp = tid >> 5;
    constexpr int kWarps = kLockThreads / 32;
    const int br = lane & 15;           // branch in the group
    const int half = lane >> 4;         // entry parity
    const int P = int(gridDim.x);
    const int p = int(blockIdx.x);
    const int RP = 16 * NG;           // residual row pitch (pairs)
    constexpr size_t kStageBytes = size_t(kLockE) * 8 + size_t(kLockB) * 32 + size_t(kLockN) * 4;
    // one group of 16 branches: the Philox draws of the next chunk are made
    // while the grid barrier is pending and wait in two 16-branch tables
    unsigned long long* s_draw = reinterpret_cast<unsigned long long*>(smem + 2 * kStageBytes);
    const bool pre_draw = NG == 1;
    float* hseg = reinterpret_cast<float*>(s_draw + (pre_draw ? 2 * size_t(kLockB) * 16 : 0));   // kLockSegs x NG x 16 segment sums
    uint32_t* s_xw = reinterpret_cast<uint32_t*>(hseg + size_t(kLockSegs) * NG * 16);   // kLockB x NG bit words (before)
    uint32_t* s_amask = s_xw + size_t(kLockB) * NG;                                   // kLockB x NG flipped branches
    uint8_t* s_map = reinterpret_cast<uint8_t*>(s_amask + size_t(kLockB) * NG);         // 2 x kLockSegs: bit of each segment
    uint8_t* s_unl = s_map + 2 * kLockSegs;                                            // kLockB x NG x 16 unlike counts
    __shared__ double s_trace[16 * kLockMaxNG];
    // the draws of the chunk that starts at bit b0 with nb bits in sweep `sw`, into table `t`
    auto make_draws = [&](int t, int b0, int nb, int sw) {
        unsigned long long* d = s_draw + size_t(t) * kLockB * 16;
        for (int q = tid; q < nb * 16; q += kLockThreads) {
            const int k = q >> 4, b = q & 15;
            if (b < A.R) d[q] = draw_u53(A.seed0 + uint64_t(b), uint32_t(__ldg(&A.order[b0 + k])), uint32_t(sw), 0u);
        }
    };
    // the segment -> bit map of the chunk staged in buffer b (bits per chunk
    // <= kLockB = 256 fit a byte), built before the chunk runs so that a
    // segment item finds its bit with one shared load
    auto seg_map = [&](int b, const int4 n0) {
        const uint4* meta = reinterpret_cast<const uint4*>(smem + size_t(b) * kStageBytes + size_t(kLockE) * 8);
        uint8_t* m = s_map + b * kLockSegs;
        for (int k = tid; k < n0.y - n0.x; k += kLockThreads) {
            const int s0 = int(meta[2 * k + 1].w), ns = (int(meta[2 * k].y) + kSeg - 1) / kSeg;
            for (int j = 0; j < ns; ++j) m[s0 + j] = uint8_t(k);
        }
    };
    auto stage = [&](int b) {
        LockStage L;
        unsigned char* q = smem + size_t(b) * kStageBytes;
        L.ent = reinterpret_cast<uint2*>(q);
        L.meta = reinterpret_cast<uint4*>(q + size_t(kLockE) * 8);
        L.nbr = reinterpret_cast<int32_t*>(q + size_t(kLockE) * 8 + size_t(kLockB) * 32);
        return L;
    };
    const unsigned per_round = unsigned(P) + A.bar_extra;
    const int4* chunks = A.chunks + 2 * A.chunk_ptr[p];
    const int n_chunks = A.chunk_ptr[p + 1] - A.chunk_ptr[p];
    unsigned round = 0;
    unsigned long long my_accepts = 0;
    __shared__ unsigned long long s_acc_count;
    if (tid == 0) {
        s_acc_count = 0;
        s_seen_round = 0;
        s_wait_fail = 0;
    }
    if (tid < 16 * kLockMaxNG) s_trace[tid] = 0.0;
    // x = 0: rho_b = -sqrt|w_b| d_b for every branch
    for (size_t k = size_t(p) * kLockThreads + tid; k < size_t(A.n_rays) * RP; k += size_t(P) * kLockThreads) {
        const int b = int(k / RP);
        A.rp[k] = split_pair(-__dmul_rn(sqrt(fabs(A.w64[b])), A.d[b]));
    }
    for (size_t k = size_t(p) * kLockThreads + tid; k < size_t(A.n) * NG; k += size_t(P) * kLockThreads) A.xb[k] = 0u;
    if (n_chunks > 0) lock_stage(A, chunks[0], chunks[1], stage(0), tid, kLockThreads);
    cp_async_commit();
    if (pre_draw && n_chunks > 0 && A.sweeps > 0) make_draws(0, chunks[0].x, chunks[0].y - chunks[0].x, 0);
    asm volatile("cp.async.wait_all;" ::: "memory");
    bool ok = grid_barrier(A.bar, A.err, ++round, per_round, A.spin_limit);   // also publishes the first stage
    if (n_chunks > 0) seg_map(0, chunks[0]);
    __syncthreads();
    int gci = 0;   // chunk counter over all sweeps: staging buffer gci & 1
    int4 cur0 = make_int4(0, 0, 0, 0), cur1 = make_int4(0, 0, 0, 0);   // descriptor of the chunk in hand
    if (n_chunks > 0) {
        cur0 = chunks[0];
        cur1 = chunks[1];
    }
    long long ph_wait = 0, ph_items = 0, ph_bar = 0, ph_n = 0, t_ph = 0, ph_a = 0, ph_b = 0, t_a = 0, ph_c = 0;
    for (int sweep = 0; ok && sweep < A.sweeps; ++sweep) {
        if (A.refresh > 0 && sweep > 0 && sweep % A.refresh == 0) {
            // fp64 refresh: thread per (ray, branch), the ray's set bits in
            // order: rho = sum a' - sqrt|w| d, the drift |hi + lo - rho| recorded
            for (size_t k = size_t(p) * kLockThreads + tid; k < size_t(A.n_rays) * RP; k += size_t(P) * kLockThreads) {
                const int b = int(k / RP), j = int(k % RP);
                if (j >= A.R) continue;
                const int g = j >> 4, l = j & 15;
                const double sw = sqrt(fabs(A.w64[b]));
                double acc = 0.0;
                for (int e = A.rrow[b]; e < A.rrow[b + 1]; ++e)
                    if ((__ldcg(&A.xb[size_t(A.rbit[e]) * NG + g]) >> l) & 1u) acc = __dadd_rn(acc, double(scaled_coef(sw, A.ra[e])));
                const double v = __dsub_rn(acc, __dmul_rn(sw, A.d[b]));
                const float2 cur = __ldcg(&A.rp[k]);
                const float dv = __double2float_rn(fabs(__dsub_rn(__dadd_rn(double(cur.x), double(cur.y)), v)));
                if (dv > 0.0f) atomicMax(reinterpret_cast<int*>(&A.drift[j]), __float_as_int(dv));
                __stcg(&A.rp[k], split_pair(v));
            }
            ok = grid_barrier(A.bar, A.err, ++round, per_round, A.spin_limit);
            if (!ok) break;
        }
        const double T = A.temp[sweep];
        const float inv_T = float(1.0 / T);
        for (int ci = 0; ci < n_chunks; ++ci, ++gci) {
            const int4 c0 = cur0, c1 = cur1;
            // the next chunk (wrapping into the next sweep) is staged while this
            // one runs; its descriptor is fetched now and used after this chunk's work
            const int nx = ci + 1 < n_chunks ? ci + 1 : 0;
            const int4 cn0 = __ldg(&chunks[2 * nx]), cn1 = __ldg(&chunks[2 * nx + 1]);
            if (PHASES) t_ph = clock64();
            // this chunk's stage was waited for and published before the
            // previous chunk's block barriers (or the first grid barrier)
            const LockStage St = stage(gci & 1);
            // the other buffer was last read by the previous chunk, which every
            // thread has finished: the CTA's last kStageWarps warps (without
            // phase-A items, mostly: items go to the lowest warps first) stage
            // the next chunk into it now, so no segment item waits behind the
            // copies' issue
            if (tid >= kLockThreads - 32 * kStageWarps)
                lock_stage(A, cn0, cn1, stage((gci + 1) & 1), tid - (kLockThreads - 32 * kStageWarps), 32 * kStageWarps);
            cp_async_commit();
            const int sweep_n = nx == 0 ? sweep + 1 : sweep;
            const int nb = c0.y - c0.x;
            const int nseg = c0.z;                       // segments of the chunk
            if (PHASES) t_a = clock64();
            // A. segment sums, and per (bit, group) the bit word and the
            // unlike-neighbour counts, in one round of loads
            const int nseg_items = nseg * NG;
            float2 held[kSeg / 2];   // the pairs of this warp's first segment item, for phase C
            int held_it = -1;
#pragma unroll
            for (int u = 0; u < kSeg / 2; ++u) held[u] = make_float2(0.0f, 0.0f);
            for (int it = warp; it < nseg_items + nb * NG; it += kWarps) {
                if (it >= nseg_items) {
                    const int k = (it - nseg_items) / NG, g = (it - nseg_items) % NG;
                    const uint4 m0 = St.meta[2 * k];
                    const int ns = int(m0.z) - c1.z, nn = int(m0.w);
                    const uint32_t xw = __ldcg(&A.xb[size_t(c0.x + k) * NG + g]);
                    int unlike = 0;
                    for (int j0 = 0; j0 < nn; j0 += 32) {
                        const uint32_t w = j0 + lane < nn ? __ldcg(&A.xb[size_t(St.nbr[ns + j0 + lane]) * NG + g]) : 0u;
                        const int m = min(32, nn - j0);
                        for (int u = 0; u < m; ++u) {
                            const uint32_t wu = __shfl_sync(kFull, w, u);
                            unlike += ((wu ^ xw) >> br) & 1u;
                        }
                    }
                    if (half == 0) s_unl[(k * NG + g) * 16 + br] = uint8_t(unlike);
                    if (lane == 0) s_xw[k * NG + g] = xw;
                    continue;
                }
                const int sg = it / NG, g = it % NG;
                const int lo = s_map[(gci & 1) * kLockSegs + sg];   // the bit of segment sg
                const uint4 m0 = St.meta[2 * lo];
                const int seg_in_bit = sg - int(St.meta[2 * lo + 1].w);
                const int rs = int(m0.x) - c1.x + seg_in_bit * kSeg;
                const int re = min(int(m0.x) - c1.x + int(m0.y), rs + kSeg);
                float cv[kSeg / 2];
                float2 rv[kSeg / 2];
#pragma unroll
                for (int u = 0; u < kSeg / 2; ++u) {
                    const int e = rs + half + 2 * u;
                    if (e < re) {
                        const uint2 en = St.ent[e];
                        cv[u] = (en.x >> 31) ? -__uint_as_float(en.y) : __uint_as_float(en.y);
                        rv[u] = __ldcg(&A.rp[size_t(en.x & kRayMask) * RP + 16 * g + br]);
                    } else {
                        cv[u] = 0.0f;
                        rv[u] = make_float2(0.0f, 0.0f);
                    }
                }
                float acc = 0.0f;
#pragma unroll
                for (int u = 0; u < kSeg / 2; ++u)
                    if (rs + half + 2 * u < re) acc = fmaf(cv[u], __fadd_rn(rv[u].x, rv[u].y), acc);
                const float other = __shfl_xor_sync(kFull, acc, 16);
                if (half == 0) hseg[(sg * NG + g) * 16 + br] = __fadd_rn(acc, other);
                if (held_it < 0) {
                    held_it = it;
#pragma unroll
                    for (int u = 0; u < kSeg / 2; ++u) held[u] = rv[u];
                }
            }
            __syncthreads();
            if (PHASES) {
                const long long t1 = clock64();
                ph_a += t1 - t_a;
                t_a = t1;
            }
            // B. decide, a warp per (bit, group)
            for (int it = warp; it < nb * NG; it += kWarps) {
                const int k = it / NG, g = it % NG;
                const int branch = 16 * g + br;
                const bool live = branch < A.R && half == 0;
                const uint4 m0 = St.meta[2 * k], m1 = St.meta[2 * k + 1];
                const int i = c0.x + k;
                const int ne = int(m0.w);
                const uint32_t xw = s_xw[k * NG + g];
                const uint32_t xi = (xw >> br) & 1u;
                const int unlike = s_unl[(k * NG + g) * 16 + br];
                const uint64_t u53 = !live ? 0ull
                                     : pre_draw ? s_draw[size_t(gci & 1) * kLockB * 16 + size_t(k) * 16 + br]
                                                : draw_u53(A.seed0 + uint64_t(branch), m1.z, uint32_t(sweep), 0u);
                int flip = 0;
                float dE = 0.0f;
                if (live) {
                    const int nsg = (int(m0.y) + kSeg - 1) / kSeg;
                    const int s0 = int(m1.w);
                    // the first four segment sums loaded together, then every sum
                    // added in order (most bits have at most four segments)
                    float hv[4];
#pragma unroll
                    for (int q = 0; q < 4; ++q) hv[q] = q < nsg ? hseg[((s0 + q) * NG + g) * 16 + br] : 0.0f;
                    float h = 0.0f;
#pragma unroll
                    for (int q = 0; q < 4; ++q)
                        if (q < nsg) h = __fadd_rn(h, hv[q]);
                    for (int q = 4; q < nsg; ++q) h = __fadd_rn(h, hseg[((s0 + q) * NG + g) * 16 + br]);
                    const float delta = xi ? -1.0f : 1.0f;
                    const float t = __fadd_rn(__uint_as_float(m1.x), h);
                    const float prior = __fmul_rn(A.lambda, float(ne - 2 * unlike));
                    dE = __fadd_rn(__fadd_rn(__fmul_rn(delta, t), __uint_as_float(m1.y)), prior);
                    flip = (dE <= 0.0f || uphill_accept(u53, double(dE), T, inv_T)) ? 1 : 0;
                }
                const unsigned amask = __ballot_sync(kFull, flip) & 0xFFFFu;
                if (lane == 0) {
                    s_amask[k * NG + g] = amask;
                    if (amask) {
                        __stcg(&A.xb[size_t(i) * NG + g], xw ^ amask);
                        my_accepts += unsigned(__popc(amask));
                    }
                }
                if (A.trace && flip) atomicAdd(&s_trace[branch], double(dE));
            }
            __syncthreads();
            long long t_c = 0;
            if (PHASES) t_c = clock64();   // phase B ends here; phase C is counted apart
            // the sweep's tracked energy change, once per CTA per sweep
            if (A.trace && ci == n_chunks - 1 && tid < A.R) {
                atomicAdd(&A.trace[size_t(tid) * A.sweeps + sweep], s_trace[tid]);
                s_trace[tid] = 0.0;
            }
            // C. the flipped branches' residuals: rho += delta a' (TwoSum)
            for (int it = warp; it < nseg_items; it += kWarps) {
                const int sg = it / NG, g = it % NG;
                const int k = s_map[(gci & 1) * kLockSegs + sg];
                const uint32_t amask = s_amask[k * NG + g];
                if (!amask) continue;   // warp-uniform
                const bool mine = (amask >> br) & 1u;
                const float dl = ((s_xw[k * NG + g] >> br) & 1u) ? -1.0f : 1.0f;
                const uint4 m0 = St.meta[2 * k];
                const int seg_in_bit = sg - int(St.meta[2 * k + 1].w);
                const int rs = int(m0.x) - c1.x + seg_in_bit * kSeg;
                const int re = min(int(m0.x) - c1.x + int(m0.y), rs + kSeg);
                float2 cur[kSeg / 2];
                if (it == held_it) {
#pragma unroll
                    for (int u = 0; u < kSeg / 2; ++u) cur[u] = held[u];
                } else {
#pragma unroll
                    for (int u = 0; u < kSeg / 2; ++u) {
                        const int e = rs + half + 2 * u;
                        cur[u] = mine && e < re ? __ldcg(&A.rp[size_t(St.ent[e].x & kRayMask) * RP + 16 * g + br])
                                                : make_float2(0.0f, 0.0f);
                    }
                }
                if (mine) {
#pragma unroll
                    for (int u = 0; u < kSeg / 2; ++u) {
                        const int e = rs + half + 2 * u;
                        if (e < re) {
                            const uint2 en = St.ent[e];
                            __stcg(&A.rp[size_t(en.x & kRayMask) * RP + 16 * g + br],
                                   two_sum_add(cur[u], __fmul_rn(dl, __uint_as_float(en.y))));
                        }
                    }
                }
            }
            // no barrier here: the next chunk's first barrier (or the grid
            // barrier's) orders this chunk's shared-memory reads before the
            // next chunk's writes
            if (PHASES) {
                __syncthreads();
                const long long t1 = clock64();
                ph_b += t1 - t_a;
                ph_c += t1 - t_c;
            }
            if (PHASES) {
                const long long t1 = clock64();
                ph_items += t1 - t_ph;
                t_ph = t1;
            }
            // the next chunk's stage (issued at this chunk's start) is complete
            // once every thread's copies are; the block barrier below publishes
            // it, its segment map is built after that, and the closing block
            // barrier publishes the map
            {
                const long long tw = PHASES ? clock64() : 0;
                asm volatile("cp.async.wait_all;" ::: "memory");
                if (PHASES) ph_wait += clock64() - tw;
            }
            if (c0.w & 1) {
                // arrive; build the map and make the next chunk's draws while
                // the others arrive; then wait
                grid_arrive(A.bar);
                seg_map((gci + 1) & 1, cn0);
                if (pre_draw && sweep_n < A.sweeps) make_draws((gci + 1) & 1, cn0.x, cn0.y - cn0.x, sweep_n);
                ok = grid_wait2(A.bar, A.err, ++round, per_round, A.spin_limit, &s_seen_round, &s_wait_fail);
            } else {
                __syncthreads();
                seg_map((gci + 1) & 1, cn0);
                if (pre_draw && sweep_n < A.sweeps) make_draws((gci + 1) & 1, cn0.x, cn0.y - cn0.x, sweep_n);
                __syncthreads();
            }
            cur0 = cn0;
            cur1 = cn1;
            if (!ok) break;
            if (PHASES) {
                ph_bar += clock64() - t_ph;
                ++ph_n;
            }
        }
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
    if (PHASES && tid == 0) {
        unsigned long long* ph = A.phase + 8 * size_t(blockIdx.x);
        ph[0] = ph_wait; ph[1] = ph_items; ph[2] = ph_bar; ph[3] = ph_n; ph[4] = ph_a; ph[5] = ph_b; ph[6] = ph_c;
    }
    if (ok) {
        // branches out, original bit order
        for (size_t k = size_t(p) * kLockThreads + tid; k < size_t(A.n) * A.R; k += size_t(P) * kLockThreads) {
            const int i = int(k % A.n), b = int(k / A.n);
            A.x_out[size_t(b) * A.n + A.order[i]] = uint8_t((__ldcg(&A.xb[size_t(i) * NG + (b >> 4)]) >> (b & 15)) & 1u);
        }
    } else if (tid == 0 && A.status) {
        *reinterpret_cast<volatile int*>(A.status) = int(QB_ETIMEDOUT);
    }
    if (lane == 0 && my_accepts) atomicAdd(&s_acc_count, my_accepts);
    __syncthreads();
    if (tid == 0 && s_acc_count) atomicAdd(&A.accepts[0], s_acc_count);
}

// binary_energy (src/ising_recon.hpp:65-79) of K states in fp64, one CTA per
// state, original bit order; the block sum has a fixed shape.
struct ResidEnergyArgs {
    int n;
    int n_rays;
    double lambda;
    const double* d;
    const double* w;
    const int32_t* rrow;   // ray-major, bits ascending inside a ray
    const int32_t* rbit;
    const float* ra;
    const double* lin;
    const int32_t* nbr_ptr;
    const int32_t* nbr;
    const uint8_t* X;
    double* e;
};

__device__ double block_sum_f64(double v, double* red) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v = v + __shfl_xor_sync(kFull, v, off);
    __syncthreads();
    if ((threadIdx.x & 31u) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int q = 0; q < int(blockDim.x >> 5); ++q) t += red[q];
    return t;
}

// Partial sums of state s over block j's share of the rays (data term) and of
// the bits (prior term); grid = (blocks per state, states), so every SM takes
// part. The partials are added in block order afterwards.
__global__ void __launch_bounds__(256) resid_energy_part_kernel(ResidEnergyArgs A, double* part) {
    __shared__ double red[32];
    const int st = int(blockIdx.y), j = int(blockIdx.x), nb = int(gridDim.x);
    const uint8_t* x = A.X + size_t(st) * size_t(A.n);
    const int r0 = int(int64_t(A.n_rays) * j / nb), r1 = int(int64_t(A.n_rays) * (j + 1) / nb);
    const int i0 = int(int64_t(A.n) * j / nb), i1 = int(int64_t(A.n) * (j + 1) / nb);
    double data = 0.0, prior = 0.0;
    for (int b = r0 + int(threadIdx.x); b < r1; b += blockDim.x) {
        double r = -A.d[b];
        for (int k = A.rrow[b]; k < A.rrow[b + 1]; ++k)
            if (x[A.rbit[k]]) r += double(A.ra[k]);
        data += 0.5 * A.w[b] * r * r;
    }
    for (int i = i0 + int(threadIdx.x); i < i1; i += blockDim.x) {
        prior += A.lin[i] * double(x[i]);
        for (int k = A.nbr_ptr[i]; k < A.nbr_ptr[i + 1]; ++k)
            if (A.nbr[k] > i && x[A.nbr[k]] != x[i]) prior += A.lambda;
    }
    const double sd = block_sum_f64(data, red);
    const double sp = block_sum_f64(prior, red);
    if (threadIdx.x == 0) {
        part[(size_t(st) * size_t(nb) + size_t(j)) * 2] = sd;
        part[(size_t(st) * size_t(nb) + size_t(j)) * 2 + 1] = sp;
    }
}

// e_s = (data partials in block order) + (prior partials in block order).
__global__ void resid_energy_final_kernel(const double* part, int nb, int K, double* e) {
    const int st = int(blockIdx.x * blockDim.x + threadIdx.x);
    if (st >= K) return;
    double sd = 0.0, sp = 0.0;
    for (int j = 0; j < nb; ++j) {
        sd += part[(size_t(st) * size_t(nb) + size_t(j)) * 2];
        sp += part[(size_t(st) * size_t(nb) + size_t(j)) * 2 + 1];
    }
    e[st] = sd + sp;
}

// ---- results ----------------------------------------------------------------------------

// p_v = (sum_b x_bv) / R: the float division of branch_fractions
// (ising_recon.hpp:160-163) on an exact integer count.
__global__ void marginals_kernel(const uint8_t* x, int R, int n, float* p) {
    for (int v = int(blockIdx.x * blockDim.x + threadIdx.x); v < n; v += gridDim.x * blockDim.x) {
        int cnt = 0;
        for (int b = 0; b < R; ++b) cnt += x[size_t(b) * size_t(n) + size_t(v)];
        p[v] = float(cnt) / float(R);
    }
}

// classify (ising_recon.hpp:305-309): NotThere = 1 when p >= hi, Exists = 0
// when p <= lo, Undecided = 2 otherwise.
__global__ void tristate_kernel(const float* p, int n, float lo, float hi, uint8_t* out) {
    for (int v = int(blockIdx.x * blockDim.x + threadIdx.x); v < n; v += gridDim.x * blockDim.x) {
        const float q = p[v];
        out[v] = q >= hi ? 1u : (q <= lo ? 0u : 2u);
    }
}

__global__ void i64_to_f64_kernel(const long long* e, int R, double* out) {
    const int i = int(blockIdx.x * blockDim.x + threadIdx.x);
    if (i < R) out[i] = double(e[i]);
}

int grid_for(int64_t n, int threads) {
    int64_t g = (n + threads - 1) / threads;
    if (g < 1) g = 1;
    if (g > 148 * 16) g = 148 * 16;
    return int(g);
}

}  // namespace

// ---- launchers ------------------------------------------------------------------------

size_t ising_smem_bytes(const IsingPlan& p) {
    const size_t need = size_t(p.n) * (sizeof(int32_t) + sizeof(int8_t));
    return need <= size_t(200) * 1024 ? need : 0;
}

qb_status launch_ising_anneal(const IsingPlan& p, const SolveBuffers& b, int R, int sweeps, uint64_t seed0,
                              cudaStream_t st) {
    IsingArgs A{};
    A.n = p.n;
    A.n_colours = p.col.n_colours();
    A.sweeps = sweeps;
    A.seed0 = seed0;
    A.class_ptr = p.d_class_ptr.as<int32_t>();
    A.row = p.d_row.as<int32_t>();
    A.adj = p.d_adj.as<int32_t>();
    A.w = p.d_w.p;
    A.f0 = p.d_f0.as<int32_t>();
    A.order = p.d_order.as<int32_t>();
    A.temp = b.temp;
    A.x_out = b.x;
    A.f_out = b.f;
    A.e_out = b.e_i64;
    A.trace = reinterpret_cast<long long*>(b.trace);
    int max_deg = 0;
    for (int i = 0; i < p.n; ++i) max_deg = std::max(max_deg, p.row[size_t(i) + 1] - p.row[size_t(i)]);
    A.wide = max_deg >= kWideRow ? 1 : 0;
    const size_t smem = ising_smem_bytes(p);
    if (smem == 0) {
        if (!b.scratch) return fail(QB_EINVAL, "ising sweep: global state needs scratch");
        A.f_scratch = static_cast<int32_t*>(b.scratch);
        A.s_scratch = reinterpret_cast<int8_t*>(A.f_scratch + size_t(R) * size_t(p.n));
    }
    // CTA size: 512 threads while the replicas fit one CTA per SM; with more
    // replicas, 128-thread CTAs, several per SM (measured on the 800-node ER
    // graph: 1,024 replicas take 16.7 ms at 128 threads, 28.1 at 256, 48.8 at
    // 512; 16 replicas 11.8 ms at 512, 13.1 at 128). The decisions do not
    // depend on the CTA size (integer sums are order-free). QB_ISING_THREADS
    // overrides (a multiple of 32, 32..512).
    int threads = kIsingThreads;
    {
        int dev = 0, sms = 148;
        if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (R > sms) threads = 128;
        if (const char* t = std::getenv("QB_ISING_THREADS")) {
            const int v = std::atoi(t);
            if (v >= 32 && v <= kIsingThreads && v % 32 == 0) threads = v;
        }
    }
    const dim3 grid(static_cast<unsigned>(R)), block(static_cast<unsigned>(threads));
    if (smem) {
        if (p.weight_bytes == 1) {
            QB_CUDA(allow_max_smem(ising_anneal_kernel<int8_t, true>));
            ising_anneal_kernel<int8_t, true><<<grid, block, smem, st>>>(A);
        } else {
            QB_CUDA(allow_max_smem(ising_anneal_kernel<int32_t, true>));
            ising_anneal_kernel<int32_t, true><<<grid, block, smem, st>>>(A);
        }
    } else {
        if (p.weight_bytes == 1) ising_anneal_kernel<int8_t, false><<<grid, block, 0, st>>>(A);
        else ising_anneal_kernel<int32_t, false><<<grid, block, 0, st>>>(A);
    }
    QB_CUDA(cudaGetLastError());
    return QB_OK;
}

qb_status launch_ising_energies(const IsingPlan& p, const uint8_t* x, int K, long long* e, cudaStream_t st) {
    QB_CUDA(cudaMemsetAsync(e, 0, sizeof(long long) * size_t(K), st));
    if (p.m == 0 || K == 0) return QB_OK;
    const int threads = 256;
    int gx = int((p.m + threads - 1) / threads);
    if (gx > 64) gx = 64;
    ising_energy_kernel<<<dim3(unsigned(gx), unsigned(K)), threads, 0, st>>>(
        p.d_eu.as<int32_t>(), p.d_ev.as<int32_t>(), p.d_ew.as<int32_t>(), p.m, x, p.n, e);
    QB_CUDA(cudaGetLastError());
    return QB_OK;
}

size_t resid_stage_bytes() {
    return size_t(kChunkB) * 8 + size_t(kChunkE) * 8 + size_t(kChunkB + 1) * 8 + size_t(kChunkB) * 8 + size_t(kChunkN);
}

size_t resid_smem_bytes(const ResidualPlan& p) {
    const size_t words = (size_t(p.bit_slots) + 31) / 32;
    return resid_stage_bytes() + size_t(p.ray_slots) * 8 + words * 4;
}

int resid_chunk_bits() { return kChunkB; }
int resid_group_lanes() { return kGroup; }
int resid_heavy_entries() { return kHeavy; }
int resid_chunk_entries() { return kChunkE; }
int resid_chunk_nbrs() { return kChunkN; }

namespace {
template <int CL>
qb_status resid_launch_cl(const ResidArgs& A, int R, size_t smem, cudaStream_t st, bool check_only) {
    auto kern = A.phase ? resid_anneal_kernel<CL, true> : resid_anneal_kernel<CL, false>;
    QB_CUDA(allow_max_smem(kern));
    if (CL > 8) QB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(unsigned(R * CL));
    cfg.blockDim = dim3(kResidThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = CL;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int clusters = 0;
    QB_CUDA(cudaOccupancyMaxActiveClusters(&clusters, kern, &cfg));
    if (clusters < 1) return fail(QB_ENOTSUP, "residual sweep: a cluster of this size does not fit on the device");
    if (std::getenv("QB_DEBUG"))
        std::fprintf(stderr, "[qublar] residual sweep: cluster %d x %d threads, %zu B shared, %d clusters co-resident, grid %d\n",
                     CL, kResidThreads, smem, clusters, R * CL);
    if (check_only) return QB_OK;
    QB_CUDA(cudaLaunchKernelEx(&cfg, kern, A));
    QB_CUDA(cudaGetLastError());
    return QB_OK;
}
}  // namespace

qb_status launch_resid_anneal(const ResidualPlan& p, const SolveBuffers& b, int R, int sweeps, int refresh,
                              uint64_t seed0, cudaStream_t st) {
    ResidArgs A{};
    A.n = p.n;
    A.n_rays = p.n_rays;
    A.sweeps = sweeps;
    A.refresh = refresh;
    A.ray_slots = p.ray_slots;
    A.bit_words = (p.bit_slots + 31) / 32;
    A.lambda = float(p.lambda);
    A.seed0 = seed0;
    A.chunks = p.d_chunks.as<int4>();
    A.chunk_ptr = p.d_chunk_ptr.as<int32_t>();
    A.row = p.d_row.as<int32_t>();
    A.ent = p.d_ent.as<uint2>();
    A.lin = p.d_lin.as<float>();
    A.q = p.d_q.as<float>();
    A.nbr_ptr = p.d_nbr_ptr.as<int32_t>();
    A.nbr_home = p.d_nbr_home.as<uint32_t>();
    A.order = p.d_order.as<int32_t>();
    A.d = p.d_d.as<double>();
    A.w64 = p.d_w64.as<double>();
    A.rrow = p.d_rrow.as<int32_t>();
    A.rbit_home = p.d_rbit.as<uint32_t>();
    A.ra = p.d_ra.as<float>();
    A.temp = b.temp;
    A.x_out = b.x;
    A.drift = b.drift;
    A.accepts = b.accepts;
    A.trace = b.trace;
    const size_t smem = resid_smem_bytes(p);
    // QB_PHASE_TIMES: per-CTA clock64 sums of the gather, score and barrier
    // phases, printed to stderr after the launch (diagnostics; same work)
    DevBuf phase;
    const bool phases = std::getenv("QB_PHASE_TIMES") != nullptr;
    if (phases) {
        qb_status s = phase.alloc(size_t(R) * size_t(p.CL) * 32);
        if (s != QB_OK) return s;
        QB_CUDA(cudaMemsetAsync(phase.p, 0, phase.bytes, st));
        A.phase = phase.as<unsigned long long>();
    }
    qb_status s;
    switch (p.CL) {
        case 1: s = resid_launch_cl<1>(A, R, smem, st, false); break;
        case 2: s = resid_launch_cl<2>(A, R, smem, st, false); break;
        case 4: s = resid_launch_cl<4>(A, R, smem, st, false); break;
        case 8: s = resid_launch_cl<8>(A, R, smem, st, false); break;
        case 16: s = resid_launch_cl<16>(A, R, smem, st, false); break;
        default: return fail(QB_EINVAL, "residual sweep: cluster size must be 1, 2, 4, 8 or 16");
    }
    if (s == QB_OK && phases) {
        std::vector<unsigned long long> h(size_t(R) * size_t(p.CL) * 4);
        QB_CUDA(cudaMemcpyAsync(h.data(), phase.p, phase.bytes, cudaMemcpyDeviceToHost, st));
        QB_CUDA(cudaStreamSynchronize(st));
        double g = 0, sc = 0, br = 0, ch = 0;
        const size_t ctas = size_t(R) * size_t(p.CL);
        for (size_t c = 0; c < ctas; ++c) { g += h[4 * c]; sc += h[4 * c + 1]; br += h[4 * c + 2]; ch += h[4 * c + 3]; }
        std::fprintf(stderr, "[qublar] phases per CTA: chunks %.0f, cycles per chunk: gather %.0f, score %.0f, barrier %.0f\n",
                     ch / ctas, g / ch, sc / ch, br / ch);
    }
    return s;
}

qb_status resid_check_fit(const ResidualPlan& p) {
    ResidArgs A{};
    const size_t smem = resid_smem_bytes(p);
    if (smem > size_t(227) * 1024) return fail(QB_ENOTSUP, "residual sweep: state exceeds the cluster's shared memory");
    switch (p.CL) {
        case 1: return resid_launch_cl<1>(A, 1, smem, nullptr, true);
        case 2: return resid_launch_cl<2>(A, 1, smem, nullptr, true);
        case 4: return resid_launch_cl<4>(A, 1, smem, nullptr, true);
        case 8: return resid_launch_cl<8>(A, 1, smem, nullptr, true);
        case 16: return resid_launch_cl<16>(A, 1, smem, nullptr, true);
        default: return fail(QB_EINVAL, "residual sweep: cluster size must be 1, 2, 4, 8 or 16");
    }
}

size_t resid_lockstep_smem(int NG) {
    return 2 * (size_t(kLockE) * 8 + size_t(kLockB) * 32 + size_t(kLockN) * 4) + (NG == 1 ? 2 * size_t(kLockB) * 16 * 8 : 0) +
           size_t(kLockSegs) * NG * 16 * 4 + size_t(kLockB) * NG * (4 + 4 + 16) + 2 * size_t(kLockSegs);
}
// The largest of those over the branch-group counts one launch serves.
size_t resid_lockstep_smem_max() {
    size_t m = 0;
    for (int g = 1; g <= kLockMaxNG; ++g) m = std::max(m, resid_lockstep_smem(g));
    return m;
}
// The lockstep kernel for ng groups of 16 branches (the group count is a
// compile-time constant of each instance, so the item index arithmetic is
// shifts and multiplies).
template <bool PHASES>
const void* lockstep_kernel(int ng) {
    switch (ng) {
        case 1: return reinterpret_cast<const void*>(resid_lockstep_kernel<PHASES, 1>);
        case 2: return reinterpret_cast<const void*>(resid_lockstep_kernel<PHASES, 2>);
        case 3: return reinterpret_cast<const void*>(resid_lockstep_kernel<PHASES, 3>);
        default: return reinterpret_cast<const void*>(resid_lockstep_kernel<PHASES, 4>);
    }
}

// Raises the dynamic shared-memory limit of every lockstep instance.
cudaError_t allow_lockstep_smem() {
    for (int ng = 1; ng <= kLockMaxNG; ++ng) {
        cudaError_t e = cudaFuncSetAttribute(lockstep_kernel<false>(ng), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             int(resid_lockstep_smem_max()));
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(lockstep_kernel<true>(ng), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     int(resid_lockstep_smem_max()));
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

int resid_lockstep_max_branches() { return 16 * kLockMaxNG; }
int resid_lockstep_segment() { return kSeg; }
int resid_lockstep_chunk_segments() { return kLockSegs; }
int resid_lockstep_chunk_bits() { return kLockB; }
int resid_lockstep_chunk_entries() { return kLockE; }
int resid_lockstep_chunk_nbrs() { return kLockN; }

int resid_lockstep_grid() {
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return 0;
    if (allow_lockstep_smem() != cudaSuccess) return 0;
    // every instance needs one co-resident CTA per SM
    for (int ng = 1; ng <= kLockMaxNG; ++ng) {
        int per_sm = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, lockstep_kernel<false>(ng), kLockThreads,
                                                          resid_lockstep_smem_max()) != cudaSuccess ||
            per_sm < 1)
            return 0;
    }
    int per_sm = 1;
    return per_sm >= 1 ? sms : 0;
}

// The scratch of a lockstep solve starts with a control block: the barrier
// counter and, at +16, the timeout flag.
constexpr size_t kLockCtl = 256;

size_t resid_lockstep_scratch(const ResidualPlan& p, int R) {
    const int NG = (R + 15) / 16;
    return size_t(p.n_rays) * 16 * NG * 8 + size_t(p.n) * NG * 4 + kLockCtl;
}

// QB_TEST_BARRIER_STALL=k (tests only): every grid barrier of the lockstep
// sweep also waits for one arrival that never comes and gives up after k
// polls, so the timeout path runs to its status without a fault or a hang.
void lock_barrier_settings(ResidLockArgs& A) {
    A.bar_extra = 0;
    A.spin_limit = kSpinLimit;
    const char* v = std::getenv("QB_TEST_BARRIER_STALL");
    if (v && std::atoi(v) > 0) {
        A.bar_extra = 1;
        A.spin_limit = unsigned(std::atoi(v));
    }
}


qb_status launch_resid_lockstep(const ResidualPlan& p, const SolveBuffers& b, int R, int sweeps, int refresh,
                                uint64_t seed0, cudaStream_t st) {
    ResidLockArgs A{};
    A.n = p.n;
    A.n_rays = p.n_rays;
    A.sweeps = sweeps;
    A.refresh = refresh;
    A.R = R;
    A.NG = (R + 15) / 16;
    A.lambda = float(p.lambda);
    A.seed0 = seed0;
    A.chunks = p.d_chunks.as<int4>();
    A.chunk_ptr = p.d_chunk_ptr.as<int32_t>();
    A.ent = p.d_ent.as<uint2>();
    A.meta = p.d_meta.as<uint4>();
    A.nbr = p.d_nbr_new.as<int32_t>();
    A.order = p.d_order.as<int32_t>();
    A.d = p.d_d.as<double>();
    A.w64 = p.d_w64.as<double>();
    A.rrow = p.d_rrow.as<int32_t>();
    A.rbit = p.d_rbit_new.as<int32_t>();
    A.ra = p.d_ra.as<float>();
    A.temp = b.temp;
    // scratch: control block (barrier counter, timeout flag at +16), residual pairs, bit words
    char* sc = static_cast<char*>(b.scratch);
    A.bar = reinterpret_cast<unsigned*>(sc);
    A.err = reinterpret_cast<int*>(sc + 16);
    A.rp = reinterpret_cast<float2*>(sc + kLockCtl);
    A.xb = reinterpret_cast<uint32_t*>(sc + kLockCtl + size_t(p.n_rays) * 16 * A.NG * 8);
    A.x_out = b.x;
    A.drift = b.drift;
    A.accepts = b.accepts;
    A.trace = b.trace;
    lock_barrier_settings(A);
    // the barrier counters restart per launch; the timeout flag (+16) is
    // zeroed once per solve by the caller, so a timeout of any launch shows
    QB_CUDA(cudaMemsetAsync(A.bar, 0, 16, st));
    const int grid = p.lock_grid;
    if (grid < 1) return fail(QB_ENOTSUP, "residual lockstep sweep: no co-resident grid");
    DevBuf phase;
    const bool phases = std::getenv("QB_PHASE_TIMES") != nullptr;
    if (phases) {
        qb_status s = phase.alloc(size_t(grid) * 64);
        if (s != QB_OK) return s;
        QB_CUDA(cudaMemsetAsync(phase.p, 0, phase.bytes, st));
        A.phase = phase.as<unsigned long long>();
    }
    const void* kern = phases ? lockstep_kernel<true>(A.NG) : lockstep_kernel<false>(A.NG);
    void* args[] = {&A};
    QB_CUDA(cudaLaunchCooperativeKernel(kern, dim3(unsigned(grid)), dim3(kLockThreads), args, resid_lockstep_smem(A.NG), st));
    if (phases) {
        std::vector<unsigned long long> h(size_t(grid) * 8);
        QB_CUDA(cudaMemcpyAsync(h.data(), phase.p, phase.bytes, cudaMemcpyDeviceToHost, st));
        QB_CUDA(cudaStreamSynchronize(st));
        double w = 0, it = 0, br = 0, ch = 0, pa = 0, pb = 0, pc = 0, itmax = 0;
        for (int c = 0; c < grid; ++c) {
            w += h[8 * c]; it += h[8 * c + 1]; br += h[8 * c + 2]; ch += h[8 * c + 3]; pa += h[8 * c + 4]; pb += h[8 * c + 5];
            pc += h[8 * c + 6];
            itmax = std::max(itmax, double(h[8 * c + 1]) / std::max(1.0, double(h[8 * c + 3])));
        }
        std::fprintf(stderr, "[qublar] lockstep phases per CTA: chunks %.0f, cycles per chunk: items %.0f "
                     "(A %.0f, B %.0f, C %.0f; slowest CTA's mean %.0f), barrier %.0f (of which the next stage's wait %.0f)\n",
                     ch / grid, it / ch, pa / ch, (pb - pc) / ch, pc / ch, itmax, br / ch, w / ch);
    }
    return QB_OK;
}

// Diagnostics of the Metropolis test (qb_metropolis_check): per move the
// fp32 verdict, the sweeps' outcome and the plain fp64 test, with dE rounded
// to fp32 and inv_T = fp32(1/T) as the sweeps have them.
__global__ void metropolis_check_kernel(const uint64_t* u53, const double* dE, const double* T, int n, uint8_t* fast,
                                        uint8_t* accept, uint8_t* exact) {
    for (int k = int(blockIdx.x * blockDim.x + threadIdx.x); k < n; k += int(gridDim.x * blockDim.x)) {
        const float d = __double2float_rn(dE[k]);
        const double t = T[k];
        const float inv_t = float(1.0 / t);
        const int f = uphill_fast(u53[k], d, inv_t);
        fast[k] = f < 0 ? 255u : uint8_t(f);
        accept[k] = uphill_accept(u53[k], double(d), t, inv_t) ? 1u : 0u;
        exact[k] = double(u53[k]) * 0x1.0p-53 < exp(-double(d) / t) ? 1u : 0u;
    }
}

qb_status launch_metropolis_check(const uint64_t* u53, const double* dE, const double* T, int n, uint8_t* fast,
                                  uint8_t* accept, uint8_t* exact, cudaStream_t st) {
    if (n <= 0) return QB_OK;
    metropolis_check_kernel<<<std::min((n + 255) / 256, 4096), 256, 0, st>>>(u53, dE, T, n, fast, accept, exact);
    QB_CUDA(cudaGetLastError());
    return QB_OK;
}

qb_status launch_resid_energies(const ResidualPlan& p, const uint8_t* x, int K, double* e, cudaStream_t st) {
    if (K == 0) return QB_OK;
    ResidEnergyArgs A{};
    A.n = p.n;
    A.n_rays = p.n_rays;
    A.lambda = p.lambda;
    A.d = p.d_d.as<double>();
    A.w = p.d_w64.as<double>();
    A.rrow = p.d_rrow.as<int32_t>();   // the ray-major offsets and a are shared with the refresh
    A.rbit = p.d_o_rbit.as<int32_t>();
    A.ra = p.d_ra.as<float>();
    A.lin = p.d_o_lin.as<double>();
    A.nbr_ptr = p.d_o_nbr_ptr.as<int32_t>();
    A.nbr = p.d_o_nbr.as<int32_t>();
    A.X = x;
    A.e = e;
    // blocks per state: about four CTAs of work per SM in all
    int dev = 0, sms = 148;
    QB_CUDA(cudaGetDevice(&dev));
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int nb = std::max(1, std::min(256, (4 * sms + K - 1) / K));
    const size_t bytes = size_t(K) * size_t(nb) * 2 * sizeof(double);
    double* part = nullptr;
    cudaMemPool_t pool = library_pool(dev);
    if (pool) QB_CUDA(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&part), bytes, pool, st));
    else QB_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&part), bytes, st));
    resid_energy_part_kernel<<<dim3(unsigned(nb), unsigned(K)), 256, 0, st>>>(A, part);
    cudaError_t err = cudaGetLastError();
    if (err == cudaSuccess) {
        resid_energy_final_kernel<<<unsigned((K + 127) / 128), 128, 0, st>>>(part, nb, K, e);
        err = cudaGetLastError();
    }
    cudaFreeAsync(part, st);
    QB_CUDA(err);
    return QB_OK;
}

qb_status launch_marginals(const uint8_t* x, int R, int n, float* p, cudaStream_t st) {
    marginals_kernel<<<grid_for(n, 256), 256, 0, st>>>(x, R, n, p);
    QB_CUDA(cudaGetLastError());
    return QB_OK;
}

qb_status launch_tristate(const float* p, int n, float lo, float hi, uint8_t* out, cudaStream_t st) {
    tristate_kernel<<<grid_for(n, 256), 256, 0, st>>>(p, n, lo, hi, out);
    QB_CUDA(cudaGetLastError());
    return QB_OK;
}

qb_status launch_i64_to_f64(const long long* e, int R, double* out, cudaStream_t st) {
    i64_to_f64_kernel<<<(R + 255) / 256, 256, 0, st>>>(e, R, out);
    QB_CUDA(cudaGetLastError());
    return QB_OK;
}


// ---- residual solve without allocation ------------------------------------------------
//
// Some callers must not allocate device memory on their hot path: a host
// framework that owns every byte of device memory through its own pool, a
// plugin whose host forbids cudaMalloc/cudaFree while it runs (they
// synchronise the device and can stall other work), or a latency-bound loop
// that allocated once at start-up. qb_solve_residual_noalloc serves them: it
// runs the lockstep residual sweep with its per-solve scratch (the branches'
// residuals and bit words, the grid-barrier counter, the temperature table,
// the drift and accept tallies) in one static device array that the library
// carries, and writes the branches into a device buffer the caller owns.
//
// The array costs every GPU that loads the library QB_NOALLOC_SCRATCH_BYTES of
// device memory until the process exits. Calls share it and it keeps the last
// call's contents, so the entry point clears what must start at zero (the
// barrier counter, the error flag, the tallies) and the kernel writes the
// rest before reading it. Two calls whose work overlaps on the GPU (other
// streams, other host threads) race on the array: serialise them.

static __device__ __align__(256) unsigned char g_noalloc_scratch[QB_NOALLOC_SCRATCH_BYTES];

namespace {

constexpr int kNoAllocDevices = 64;
std::mutex g_noalloc_mu;
void* g_noalloc_addr[kNoAllocDevices] = {};

// The array's device address on the current device. In host code the name
// g_noalloc_scratch is a host-side stand-in, not a device address: the first
// call on a device looks the address up with cudaGetSymbolAddress and keeps it.
qb_status noalloc_scratch(int dev, unsigned char** out) {
    if (dev < 0 || dev >= kNoAllocDevices) return fail(QB_ENOTSUP, "qb_solve_residual_noalloc: device ordinal above 63");
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
        void* addr = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&addr, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_scratch)", __FILE__, __LINE__);
        g_noalloc_addr[dev] = addr;
    }
    *out = static_cast<unsigned char*>(g_noalloc_addr[dev]);
    return QB_OK;
}

size_t align256(size_t v) { return (v + 255) & ~size_t(255); }

}  // namespace

}  // namespace qb

extern "C" qb_status qb_solve_residual_noalloc(const qb_problem* p, const qb_schedule* s, uint32_t n_branches,
                                               uint64_t seed_offset, uint8_t* x_out, int32_t* status, void* stream) {
    using namespace qb;
    return guarded("qb_solve_residual_noalloc", [&]() -> qb_status {
        if (!p || !s || !x_out || !status) return fail(QB_EINVAL, "qb_solve_residual_noalloc: null argument");
        if (p->kind != QB_KIND_RESIDUAL) return fail(QB_EINVAL, "qb_solve_residual_noalloc: residual problems only");
        const ResidualPlan& P = p->resid;
        if (P.variant != QB_RESID_LOCKSTEP || P.lock_grid < 1)
            return fail(QB_ENOTSUP, "qb_solve_residual_noalloc: the problem is not planned for the lockstep sweep");
        if (!p->uploaded)
            return fail(QB_EINVAL, "qb_solve_residual_noalloc: the problem is not on the device (deferred upload)");
        const int R = int(n_branches);
        if (n_branches < 1 || R > 16 * kLockMaxNG)
            return fail(QB_EINVAL, "qb_solve_residual_noalloc: n_branches must be in [1, 64]");
        if (s->anneal_sweeps < 0 || s->hold_sweeps < 0 || s->anneal_sweeps + s->hold_sweeps < 1 || !(s->t_hot > 0.0) ||
            !(s->t_cold > 0.0) || s->refresh_sweeps < 0)
            return fail(QB_EINVAL, "qb_solve_residual_noalloc: bad schedule");
        const int sweeps = s->anneal_sweeps + s->hold_sweeps;
        const int NG = (R + 15) / 16;
        // scratch layout: residual pairs | bit words | barrier counter + error
        // flag | temperatures | drift | accepts
        const size_t off_xb = align256(size_t(P.n_rays) * 16 * NG * 8);
        const size_t off_bar = off_xb + align256(size_t(P.n) * NG * 4);
        const size_t off_temp = off_bar + kLockCtl;
        const size_t off_drift = off_temp + align256(size_t(sweeps) * 8);
        const size_t off_acc = off_drift + align256(size_t(R) * 4);
        const size_t need = off_acc + 256;
        if (need > QB_NOALLOC_SCRATCH_BYTES) {
            char msg[256];
            std::snprintf(msg, sizeof msg,
                          "qb_solve_residual_noalloc: %zu bytes of scratch needed, the static scratch holds %zu "
                          "(fewer rays, bits, branches or sweeps; or use qb_solve)",
                          need, size_t(QB_NOALLOC_SCRATCH_BYTES));
            return fail(QB_ENOMEM, msg);
        }
        QB_CUDA(cudaSetDevice(p->device));
        unsigned char* base = nullptr;
        qb_status st = noalloc_scratch(p->device, &base);
        if (st != QB_OK) return st;
        cudaStream_t cs = static_cast<cudaStream_t>(stream);
        // the table is copied from pageable memory: the copy has taken the
        // bytes by the time the call returns, so the vector may go
        const std::vector<double> temp = temperatures(*s);
        QB_CUDA(cudaMemcpyAsync(base + off_temp, temp.data(), temp.size() * 8, cudaMemcpyHostToDevice, cs));
        QB_CUDA(cudaMemsetAsync(base + off_bar, 0, kLockCtl, cs));
        QB_CUDA(cudaMemsetAsync(base + off_drift, 0, size_t(R) * 4, cs));
        QB_CUDA(cudaMemsetAsync(base + off_acc, 0, 8, cs));
        QB_CUDA(cudaMemsetAsync(status, 0, sizeof(int32_t), cs));   // QB_OK unless a barrier times out
        ResidLockArgs A{};
        A.n = P.n;
        A.n_rays = P.n_rays;
        A.sweeps = sweeps;
        A.refresh = s->refresh_sweeps;
        A.R = R;
        A.NG = NG;
        A.lambda = float(P.lambda);
        A.seed0 = 1 + seed_offset;
        A.chunks = P.d_chunks.as<int4>();
        A.chunk_ptr = P.d_chunk_ptr.as<int32_t>();
        A.ent = P.d_ent.as<uint2>();
        A.meta = P.d_meta.as<uint4>();
        A.nbr = P.d_nbr_new.as<int32_t>();
        A.order = P.d_order.as<int32_t>();
        A.d = P.d_d.as<double>();
        A.w64 = P.d_w64.as<double>();
        A.rrow = P.d_rrow.as<int32_t>();
        A.rbit = P.d_rbit_new.as<int32_t>();
        A.ra = P.d_ra.as<float>();
        A.temp = reinterpret_cast<const double*>(base + off_temp);
        A.rp = reinterpret_cast<float2*>(base);
        A.xb = reinterpret_cast<uint32_t*>(base + off_xb);
        A.bar = reinterpret_cast<unsigned*>(base + off_bar);
        A.err = reinterpret_cast<int*>(base + off_bar + 16);
        A.status = status;
        A.x_out = x_out;
        A.drift = reinterpret_cast<float*>(base + off_drift);
        A.accepts = reinterpret_cast<unsigned long long*>(base + off_acc);
        A.trace = nullptr;
        A.phase = nullptr;
        lock_barrier_settings(A);
        QB_CUDA(allow_lockstep_smem());
        void* args[] = {&A};
        QB_CUDA(cudaLaunchCooperativeKernel(lockstep_kernel<false>(A.NG),
                                            dim3(unsigned(P.lock_grid)), dim3(kLockThreads), args,
                                            resid_lockstep_smem(A.NG), cs));
        return QB_OK;
    });
}

