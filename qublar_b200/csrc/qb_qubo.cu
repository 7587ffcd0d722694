// Weighted QUBO sweep with compensated fp32 local fields (the general real
// QUBO E(x) = offset + sum_i h_i x_i + sum_{i<j} J_ij x_i x_j, x in {0,1},
// of qubo_energy, src/check_ree_qubo.cu:158-163, which the reference anneals
// only through its pair-ray encoding into anneal_branch, :172-192).
//
// All replicas (up to 64 per launch) of one problem run in lockstep on a
// cooperative grid. A warp visits one bit for every replica: lane l serves
// replicas l and l + 32. The state lives in global memory, L2-resident:
//   xf[i].x -- 64-bit word, bit r = x_i of replica r;
//   xf[i].y -- 64-bit word, bit r = "replica r flipped x_i at its latest visit"
//             (one 16-byte pair, so a neighbour's value and flips arrive in one load);
//   L[i][r] -- the local field L_i = h_i + sum_j J_ij x_j as an unevaluated
//             sum hi + lo of two fp32 numbers (a float2).
// Incremental fields, deterministically: when bit i is visited, every
// neighbour j has been visited exactly once since i's previous visit (colour
// classes in a fixed order, no two bits of a class coupled), so xf[j].y names
// exactly the changes i has not seen. The visit adds their deltas +-J_ij to
// L_i in CSR order with the TwoSum error carried in lo (compensated
// summation), scores dE = (1 - 2 x_i)(hi + lo), decides, and publishes its
// own flips in xf[i].y. Pushing deltas with atomics instead would make fp32
// results depend on arrival order; pulling them keeps every bit reproducible.
// Every `refresh` sweeps a visit also recomputes L_i from scratch in fp64,
// records |fp32 - fp64| (the drift) and restarts hi + lo from it. The final
// energies are recomputed in fp64 from scratch by a separate kernel.
// Acceptance: dE <= 0, else u53 * 2^-53 < exp(-dE / T) in double, u53 a
// half of the Philox block of (key, original bit, sweep): of the 64 replicas
// of a launch, replica r < 32 takes words 1:0 of key seed0 + r and replica
// r + 32 words 3:2 of the same key (branch b of a solve: key seed_base + b -
// 32 [b mod 64 >= 32]), so one evaluation serves both replicas of a lane;
// uphill_accept settles most draws in fp32 with the same outcome.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "qb_device.cuh"
#include "qb_internal.hpp"
#include "qb_philox.cuh"
#include "qb_qubo.hpp"

namespace qb {

namespace {

constexpr unsigned kFullMask = 0xffffffffu;
constexpr int kQThreads = 1024;

struct QuboArgs {
    int n;
    int n_colours;
    int sweeps;
    int refresh;
    int R;
    uint64_t seed0;
    const int32_t* class_ptr;
    const int32_t* row;
    const int32_t* adj;
    const float* J;
    const float* h;
    const int32_t* order;
    const double* temp;
    float2* L;                     // n x 64 (hi, lo)
    ulonglong2* xf;                // n (value word, flip word)
    unsigned* bar;
    int* err;
    uint8_t* x_out;                // R x n, original order
    float* drift;                  // R
    double* e_track;               // R: sum of accepted dE (E - offset)
    unsigned long long* accepts;   // R
    double* trace;                 // nullable: R x sweeps, the sum of accepted dE of each sweep
};

// 32 x 32 bit transpose across the warp: lane p returns the word whose bit q
// is bit p of lane q's w (five rounds of block swaps between lanes l, l ^ j).
__device__ __forceinline__ unsigned warp_transpose32(unsigned w, int lane) {
#pragma unroll
    for (int j = 16; j >= 1; j >>= 1) {
        const unsigned L = j == 16 ? 0x0000FFFFu : j == 8 ? 0x00FF00FFu : j == 4 ? 0x0F0F0F0Fu : j == 2 ? 0x33333333u
                                                                                                  : 0x55555555u;
        const unsigned o = __shfl_xor_sync(kFullMask, w, j);
        w = (lane & j) ? ((w & ~L) | ((o & ~L) >> j)) : ((w & L) | ((o & L) << j));
    }
    return w;
}

// hi + lo += v, the rounding error of the fp32 add carried into lo (Knuth's
// TwoSum; no fused operations).
__device__ __forceinline__ void two_sum_acc(float& hi, float& lo, float v) {
    const float s = __fadd_rn(hi, v);
    const float bp = __fsub_rn(s, hi);
    const float e = __fadd_rn(__fsub_rn(hi, __fsub_rn(s, bp)), __fsub_rn(v, bp));
    hi = s;
    lo = __fadd_rn(lo, e);
}

__global__ void __launch_bounds__(kQThreads, 1) qubo_lockstep_kernel(QuboArgs A) {
    const int lane = int(threadIdx.x & 31u);
    const int wpc = int(blockDim.x >> 5);
    const int gw = int(blockIdx.x) * wpc + int(threadIdx.x >> 5);
    const int tw = int(gridDim.x) * wpc;
    const int r0 = lane, r1 = lane + 32;
    const bool has0 = r0 < A.R, has1 = r1 < A.R;
    const uint64_t key = A.seed0 + uint64_t(r0);   // replicas r0 and r1 share the draw block
    float eh0 = 0.0f, el0 = 0.0f, eh1 = 0.0f, el1 = 0.0f;
    unsigned long long acc_a = 0, acc_b = 0;
    float dr0 = 0.0f, dr1 = 0.0f;
    double tr0 = 0.0, tr1 = 0.0;   // this sweep's accepted dE (traced solves)
    __shared__ double s_tr[64];
    if (threadIdx.x < 64) s_tr[threadIdx.x] = 0.0;
    unsigned round = 0;

    for (int j = gw; j < A.n; j += tw) {
        const float hj = A.h[j];
        const size_t base = size_t(j) * 64;
        A.L[base + r0] = make_float2(hj, 0.0f);
        A.L[base + r1] = make_float2(hj, 0.0f);
        if (lane == 0) A.xf[j] = make_ulonglong2(0ull, 0ull);
    }
    bool ok = grid_barrier(A.bar, A.err, ++round);
    for (int sweep = 0; sweep < A.sweeps && ok; ++sweep) {
        const double T = A.temp[sweep];
        const float inv_T = float(1.0 / T);
        const bool refresh = A.refresh > 0 && sweep > 0 && sweep % A.refresh == 0;
        for (int c = 0; c < A.n_colours && ok; ++c) {
            const int c1 = A.class_ptr[c + 1];
            for (int j = A.class_ptr[c] + gw; j < c1; j += tw) {
                const size_t base = size_t(j) * 64;
                const float2 l0 = __ldcg(A.L + base + r0), l1 = __ldcg(A.L + base + r1);
                const unsigned long long xj = __ldcg(A.xf + j).x;
                float hi0 = l0.x, lo0 = l0.y, hi1 = l1.x, lo1 = l1.y;
                double a0 = 0.0, a1 = 0.0;
                if (refresh) a0 = a1 = double(__ldg(A.h + j));
                const int k0 = __ldg(A.row + j), k1 = __ldg(A.row + j + 1);
                for (int kb = k0; kb < k1; kb += 32) {
                    // lane q fetches neighbour kb + q, then the warp walks them in order
                    const int k = kb + lane;
                    float Jk = 0.0f;
                    unsigned long long f = 0ull, x = 0ull;
                    if (k < k1) {
                        const int nb = __ldg(A.adj + k);
                        Jk = __ldg(A.J + k);
                        const ulonglong2 w = __ldcg(A.xf + nb);
                        x = w.x;
                        f = w.y;
                    }
                    if (!refresh) {
                        // each lane walks, in CSR order, the neighbours that one of its two
                        // replicas flipped: bit q of F0 (F1) = neighbour kb + q flipped in
                        // replica r0 (r1), so the warp iterates over the busiest lane's
                        // flips instead of every neighbour that any replica flipped
                        if (__ballot_sync(kFullMask, f != 0ull) == 0u) continue;
                        const unsigned F0 = warp_transpose32(uint32_t(f), lane);
                        const unsigned F1 = warp_transpose32(uint32_t(f >> 32), lane);
                        const unsigned xlo = uint32_t(x), xhi = uint32_t(x >> 32);
                        // each replica walks its own flipped neighbours (ascending: CSR
                        // order), two steps of both lists per iteration, so the warp runs
                        // max(flips of r0, flips of r1) of its busiest lane, not their union
                        unsigned t0 = F0, t1 = F1;
                        while (__any_sync(kFullMask, (t0 | t1) != 0u)) {
                            unsigned b0[2], b1[2];
                            float J0[2], J1[2];
                            unsigned xl[2], xh[2];
#pragma unroll
                            for (int u = 0; u < 2; ++u) {
                                b0[u] = t0 & (0u - t0);
                                t0 ^= b0[u];
                                b1[u] = t1 & (0u - t1);
                                t1 ^= b1[u];
                            }
#pragma unroll
                            for (int u = 0; u < 2; ++u) {
                                const int q0 = b0[u] ? __ffs(b0[u]) - 1 : 0, q1 = b1[u] ? __ffs(b1[u]) - 1 : 0;
                                J0[u] = __shfl_sync(kFullMask, Jk, q0);
                                J1[u] = __shfl_sync(kFullMask, Jk, q1);
                                xl[u] = __shfl_sync(kFullMask, xlo, q0);
                                xh[u] = __shfl_sync(kFullMask, xhi, q1);
                            }
#pragma unroll
                            for (int u = 0; u < 2; ++u) {
                                if (b0[u]) two_sum_acc(hi0, lo0, ((xl[u] >> lane) & 1u) ? J0[u] : -J0[u]);
                                if (b1[u]) two_sum_acc(hi1, lo1, ((xh[u] >> lane) & 1u) ? J1[u] : -J1[u]);
                            }
                        }
                        continue;
                    }
                    // refresh sweep: walk every neighbour in CSR order (the fp64 sum needs
                    // every x), applying the flips' deltas as above
                    unsigned todo = __ballot_sync(kFullMask, k < k1);
                    while (todo) {
                        const int q = __ffs(todo) - 1;
                        todo &= todo - 1u;
                        const unsigned long long fq = __shfl_sync(kFullMask, f, q);
                        const unsigned long long xq = __shfl_sync(kFullMask, x, q);
                        const float Jq = __shfl_sync(kFullMask, Jk, q);
                        if ((fq >> r0) & 1ull) two_sum_acc(hi0, lo0, ((xq >> r0) & 1ull) ? Jq : -Jq);
                        if ((fq >> r1) & 1ull) two_sum_acc(hi1, lo1, ((xq >> r1) & 1ull) ? Jq : -Jq);
                        if (refresh) {
                            if ((xq >> r0) & 1ull) a0 += double(Jq);
                            if ((xq >> r1) & 1ull) a1 += double(Jq);
                        }
                    }
                }
                if (refresh) {
                    if (has0) dr0 = fmaxf(dr0, float(fabs(double(__fadd_rn(hi0, lo0)) - a0)));
                    if (has1) dr1 = fmaxf(dr1, float(fabs(double(__fadd_rn(hi1, lo1)) - a1)));
                    hi0 = float(a0);
                    lo0 = float(a0 - double(hi0));
                    hi1 = float(a1);
                    lo1 = float(a1 - double(hi1));
                }
                const bool b0 = (xj >> r0) & 1ull, b1 = (xj >> r1) & 1ull;
                const float L0 = __fadd_rn(hi0, lo0), L1 = __fadd_rn(hi1, lo1);
                const float dE0 = b0 ? -L0 : L0, dE1 = b1 ? -L1 : L1;
                const uint32_t oj = uint32_t(__ldg(A.order + j));
                const bool up0 = has0 && !(dE0 <= 0.0f), up1 = has1 && !(dE1 <= 0.0f);   // uphill (or NaN: rejected)
                uint64_t u0 = 0, u1 = 0;
                if (up0 || up1) draw_u53_pair(key, oj, uint32_t(sweep), 0u, &u0, &u1);
                const bool acc0 = has0 && (!up0 || uphill_accept(u0, double(dE0), T, inv_T));
                const bool acc1 = has1 && (!up1 || uphill_accept(u1, double(dE1), T, inv_T));
                const unsigned m0 = __ballot_sync(kFullMask, acc0), m1 = __ballot_sync(kFullMask, acc1);
                const unsigned long long mask = (unsigned long long)m0 | ((unsigned long long)m1 << 32);
                if (lane == 0) {
                    A.xf[j] = make_ulonglong2(xj ^ mask, mask);
                }
                if (acc0) {
                    two_sum_acc(eh0, el0, dE0);
                    tr0 += double(dE0);
                    ++acc_a;
                }
                if (acc1) {
                    two_sum_acc(eh1, el1, dE1);
                    tr1 += double(dE1);
                    ++acc_b;
                }
                A.L[base + r0] = make_float2(hi0, lo0);
                A.L[base + r1] = make_float2(hi1, lo1);
            }
            ok = grid_barrier(A.bar, A.err, ++round);
        }
        if (A.trace) {   // the sweep's accepted dE: lanes -> shared memory -> one add per CTA and replica
            if (has0 && tr0 != 0.0) atomicAdd(&s_tr[r0], tr0);
            if (has1 && tr1 != 0.0) atomicAdd(&s_tr[r1], tr1);
            tr0 = tr1 = 0.0;
            __syncthreads();
            if (int(threadIdx.x) < A.R) {
                if (s_tr[threadIdx.x] != 0.0) atomicAdd(&A.trace[size_t(threadIdx.x) * A.sweeps + sweep], s_tr[threadIdx.x]);
                s_tr[threadIdx.x] = 0.0;
            }
        }
    }
    if (ok) {
        for (int j = gw; j < A.n; j += tw) {
            const unsigned long long xj = __ldcg(A.xf + j).x;
            const size_t o = size_t(__ldg(A.order + j));
            if (has0) A.x_out[size_t(r0) * size_t(A.n) + o] = uint8_t((xj >> r0) & 1ull);
            if (has1) A.x_out[size_t(r1) * size_t(A.n) + o] = uint8_t((xj >> r1) & 1ull);
        }
    }
    if (has0) {
        if (dr0 > 0.0f) atomicMax(reinterpret_cast<int*>(&A.drift[r0]), __float_as_int(dr0));
        if (acc_a) atomicAdd(&A.accepts[r0], acc_a);
        atomicAdd(&A.e_track[r0], double(eh0) + double(el0));
    }
    if (has1) {
        if (dr1 > 0.0f) atomicMax(reinterpret_cast<int*>(&A.drift[r1]), __float_as_int(dr1));
        if (acc_b) atomicAdd(&A.accepts[r1], acc_b);
        atomicAdd(&A.e_track[r1], double(eh1) + double(el1));
    }
}

// E(x) = offset + sum_i h_i x_i + sum_e J_e x_u x_v in fp64 from scratch
// (qubo_energy, src/check_ree_qubo.cu:158-163). Grid = (blocks per state,
// states): block j of state st sums its share of the bits (linear terms) and
// of the edges into part[st * nb + j]; qubo_energy_final_kernel adds the
// partials in block order. The shape is fixed by (K, SM count), so the sums
// are deterministic.
__global__ void __launch_bounds__(256) qubo_energy_part_kernel(const int32_t* eu, const int32_t* ev, const float* ew,
                                                               int64_t m, const float* h, int n, const uint8_t* X,
                                                               double* part) {
    __shared__ double red[256 / 32];
    const int st = int(blockIdx.y), j = int(blockIdx.x), nb = int(gridDim.x);
    const uint8_t* x = X + size_t(st) * size_t(n);
    const int i0 = int(int64_t(n) * j / nb), i1 = int(int64_t(n) * (j + 1) / nb);
    const int64_t k0 = m * j / nb, k1 = m * (j + 1) / nb;
    double acc = 0.0;
    for (int i = i0 + int(threadIdx.x); i < i1; i += int(blockDim.x))
        if (x[i]) acc += double(h[i]);
    for (int64_t k = k0 + threadIdx.x; k < k1; k += blockDim.x)
        if (x[eu[k]] && x[ev[k]]) acc += double(ew[k]);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(kFullMask, acc, off);
    if ((threadIdx.x & 31u) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int q = 0; q < int(blockDim.x >> 5); ++q) t += red[q];
        part[size_t(st) * size_t(nb) + size_t(j)] = t;
    }
}

// e_st = offset + the partials of state st in block order.
__global__ void qubo_energy_final_kernel(const double* part, int nb, int K, double offset, double* e) {
    const int st = int(blockIdx.x * blockDim.x + threadIdx.x);
    if (st >= K) return;
    double t = offset;
    for (int j = 0; j < nb; ++j) t += part[size_t(st) * size_t(nb) + size_t(j)];
    e[st] = t;
}

}  // namespace

int qubo_lockstep_grid() {
    int dev = 0, sms = 0, occ = 0, coop = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    if (cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) != cudaSuccess || !coop) return 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, qubo_lockstep_kernel, kQThreads, 0) != cudaSuccess) return 0;
    return occ * sms;
}

int qubo_max_branches() { return 64; }

size_t qubo_scratch(const QuboPlan& p) { return 64 + size_t(p.n) * 64 * 4 * 2 + size_t(p.n) * 16; }

qb_status launch_qubo_lockstep(const QuboPlan& p, const QuboBuffers& b, int R, int sweeps, int refresh, uint64_t seed0,
                               cudaStream_t st, int ctas) {
    if (R < 1 || R > 64) return fail(QB_EINVAL, "qubo sweep: 1 to 64 replicas per launch");
    const int full = qubo_lockstep_grid();
    if (full < 1) return fail(QB_ENOTSUP, "qubo sweep: no co-resident grid on this device");
    const int grid = ctas > 0 ? std::min(ctas, full) : full;
    QuboArgs A{};
    A.n = p.n;
    A.n_colours = p.col.n_colours();
    A.sweeps = sweeps;
    A.refresh = refresh;
    A.R = R;
    A.seed0 = seed0;
    A.class_ptr = p.d_class_ptr.as<int32_t>();
    A.row = p.d_row.as<int32_t>();
    A.adj = p.d_adj.as<int32_t>();
    A.J = p.d_J.as<float>();
    A.h = p.d_h.as<float>();
    A.order = p.d_order.as<int32_t>();
    A.temp = b.temp;
    // scratch: control block (barrier counter, timeout flag at +16), fields, words
    char* sc = static_cast<char*>(b.scratch);
    A.bar = reinterpret_cast<unsigned*>(sc);
    A.err = reinterpret_cast<int*>(sc + 16);
    A.L = reinterpret_cast<float2*>(sc + 64);
    A.xf = reinterpret_cast<ulonglong2*>(A.L + size_t(p.n) * 64);
    A.x_out = b.x;
    A.drift = b.drift;
    A.e_track = b.e_track;
    A.trace = b.trace;
    A.accepts = b.accepts;
    QB_CUDA(cudaMemsetAsync(A.bar, 0, 16, st));   // the timeout flag is zeroed once per solve by the caller
    void* args[] = {&A};
    QB_CUDA(cudaLaunchCooperativeKernel(reinterpret_cast<void*>(qubo_lockstep_kernel), dim3(unsigned(grid)),
                                        dim3(kQThreads), args, 0, st));
    return QB_OK;
}

qb_status launch_qubo_energies(const QuboPlan& p, const uint8_t* x, int K, double* e, cudaStream_t st) {
    if (K == 0) return QB_OK;
    // blocks per state: about four CTAs of work per SM in all
    int dev = 0, sms = 148;
    QB_CUDA(cudaGetDevice(&dev));
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int nb = std::max(1, std::min(256, (4 * sms + K - 1) / K));
    const size_t bytes = size_t(K) * size_t(nb) * sizeof(double);
    double* part = nullptr;
    cudaMemPool_t pool = library_pool(dev);
    if (pool) QB_CUDA(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&part), bytes, pool, st));
    else QB_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&part), bytes, st));
    qubo_energy_part_kernel<<<dim3(unsigned(nb), unsigned(K)), 256, 0, st>>>(
        p.d_eu.as<int32_t>(), p.d_ev.as<int32_t>(), p.d_ew.as<float>(), p.m, p.d_ho.as<float>(), p.n, x, part);
    cudaError_t err = cudaGetLastError();
    if (err == cudaSuccess) {
        qubo_energy_final_kernel<<<unsigned((K + 127) / 128), 128, 0, st>>>(part, nb, K, p.offset, e);
        err = cudaGetLastError();
    }
    cudaFreeAsync(part, st);
    QB_CUDA(err);
    return QB_OK;
}

}  // namespace qb
