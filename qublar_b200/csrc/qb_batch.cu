// Packed integer Ising sweep: many instances and replica groups of uneven size
// in one persistent launch.
//
// Each CTA takes the next work item from a device counter (items arrive
// sorted by estimated cost, largest first), anneals its G replicas of one
// instance over its sweep range, and takes another. The item's fields (int32)
// and spins (int8) sit in the CTA's shared memory, laid out bit-major with the
// replica fastest. A thread carries replicas 2h and 2h + 1 of one bit (items
// of G >= 2), so a warp covers 64 / G consecutive bits of a class for all G
// replicas: the two replicas share one Philox block and one walk of the bit's
// CSR row, and neighbour updates of one accepted bit land in G consecutive
// words. Items too large for shared memory run in place on their global
// state.
//
// The decisions are those of the single-instance sweep (qb_kernels.cu): colour
// classes in order, dE = -s_i f_i, accept if dE <= 0, else if u53 * 2^-53 <
// exp(-dE / T) with u53 the Philox draw of (replica key, original bit, sweep),
// words 1:0 or 3:2 of the block as the replica is even or odd
// (ising_pair_key). For |dE| <= 256 the comparison uses a per-sweep table of
// ceil(exp(-k / T) * 2^53), which is the same test on the integer u53 (the
// scaling by 2^53 is exact), so a replica's trajectory does not depend on the
// item it falls in, the launch shape, or the other instances of the batch.
#include <cuda_runtime.h>

#include <cstdint>

#include "qb_batch.hpp"
#include "qb_device.cuh"
#include "qb_philox.cuh"

namespace qb {

namespace {

constexpr int kThrMax = 256;
constexpr int kClassMax = 512;   // class boundaries kept in shared memory
constexpr int kBatchThreadsMax = 1024;

static_assert(sizeof(IsingItem) % 8 == 0, "IsingItem is copied as 8-byte words");

__device__ __forceinline__ unsigned long long accept_threshold(int k, double T) {
    const double p = exp(-double(k) / T);
    return (unsigned long long)ceil(p * 0x1.0p53);
}

// The item's outputs (kItemFinal: x and f in original bit order) and its kept
// state (kItemKeep).
template <bool GLOBAL>
__device__ __forceinline__ void ising_item_out(const IsingItem& it, const int32_t* f, const int8_t* s, int tid, int bs) {
    const int n = it.n, lg = it.log2g, G = 1 << lg, NG = n << lg;
    if (it.flags & kItemFinal) {
        for (int p = tid; p < NG; p += bs) {
            const int i = p >> lg;
            const size_t o = size_t(p & (G - 1)) * size_t(n) + size_t(it.order[i]);
            it.x_out[o] = s[p] > 0 ? 1u : 0u;
            it.f_out[o] = f[p];
        }
    }
    if (!GLOBAL && (it.flags & kItemKeep)) {
        for (int p = tid; p < NG; p += bs) {
            it.f_state[p] = f[p];
            it.s_state[p] = s[p];
        }
    }
}

template <typename WT, bool GLOBAL>
__device__ __forceinline__ void ising_item(const IsingItem& it, unsigned char* smem, unsigned long long* thr,
                                           unsigned long long* e_sh, int* cls) {
    const int n = it.n;
    const int lg = it.log2g;
    const int G = 1 << lg;
    const int NG = n << lg;
    const int tid = int(threadIdx.x);
    const int bs = int(blockDim.x);
    const int flags = it.flags;
    const int32_t* __restrict__ class_ptr = it.class_ptr;
    const int32_t* __restrict__ order = it.order;
    const double* __restrict__ temp = it.temp;
    const int n_colours = it.n_colours;
    const int bound = it.bound;
    const int sweep0 = it.sweep0, sweep1 = it.sweep1;
    int32_t* f;
    int8_t* s;
    if (GLOBAL) {
        f = it.f_state;
        s = it.s_state;
    } else {
        f = reinterpret_cast<int32_t*>(smem);
        s = reinterpret_cast<int8_t*>(smem + size_t(NG) * 4);
    }
    const bool init = (flags & kItemInit) != 0;
    if (init) {
        for (int p = tid; p < NG; p += bs) {
            f[p] = it.f0[p >> lg];
            s[p] = -1;
        }
    } else if (!GLOBAL) {
        for (int p = tid; p < NG; p += bs) {
            f[p] = it.f_state[p];
            s[p] = it.s_state[p];
        }
    }
    // class boundaries on chip (most instances have far fewer classes)
    const bool cls_sh = n_colours <= kClassMax;
    if (cls_sh)
        for (int c = tid; c <= n_colours; c += bs) cls[c] = class_ptr[c];
    if (tid < G) e_sh[tid] = 0ull;
    __syncthreads();
    const bool table = bound <= kThrMax;
    // the item's replica r is replica r0 + r of the solve: it draws from key
    // ising_pair_key(base, r0 + r) = seed0 - m + ((m + r) & ~1), m = r0 & 1,
    // the words of half (m + r) & 1
    const int m = (flags & kItemOddBase) ? 1 : 0;
    if (lg >= 1 && m == 0) {
        // pairs: a thread carries replicas 2h and 2h + 1 of one bit, which
        // share one Philox block (G / 2 threads per bit, the pair fastest).
        // Threads of odd bit slots take replica 2h + 1 first, so the field
        // accesses of two consecutive bits start on banks of opposite parity.
        // The item's tables are read from the shared descriptor where they are
        // used, to keep the registers for the two replicas' state. (Energy
        // changes added to the replicas' shared sums at each flip instead of
        // in registers made the sweep 1.4x slower: the lanes of different
        // bits that carry the same replica hit one shared word.)
        const int lh = lg - 1;
        const int par = (tid >> lh) & 1;
        const int ra = ((tid & ((G >> 1) - 1)) << 1) + par, rb = ra ^ 1;
        long long Ea = 0, Eb = 0;
        for (int sweep = sweep0; sweep < sweep1; ++sweep) {
            const double T = it.temp[sweep];
            if (table) {
                for (int k = tid + 1; k <= bound; k += bs) thr[k] = accept_threshold(k, T);
                __syncthreads();
            }
            for (int c = 0; c < n_colours; ++c) {
                const int q0 = (cls_sh ? cls[c] : it.class_ptr[c]) << lh;
                const int q1 = (cls_sh ? cls[c + 1] : it.class_ptr[c + 1]) << lh;
                for (int q = q0 + tid; q < q1; q += bs) {
                    const int i = q >> lh;
                    const uint32_t oi = uint32_t(__ldg(order + i));
                    const int pa = (i << lg) + ra, pb = (i << lg) + rb;
                    const int sa = s[pa], sb = s[pb];
                    const int dEa = -sa * f[pa], dEb = -sb * f[pb];
                    bool acca = dEa <= 0, accb = dEb <= 0;
                    unsigned long long ta = 0ull, tb = 0ull;
                    if (!acca) {
                        ta = table ? thr[dEa] : accept_threshold(dEa, T);
                        acca = ta >= (1ull << 53);
                    }
                    if (!accb) {
                        tb = table ? thr[dEb] : accept_threshold(dEb, T);
                        accb = tb >= (1ull << 53);
                    }
                    const bool needa = !acca && ta != 0ull, needb = !accb && tb != 0ull;
                    if (needa || needb) {
                        uint64_t lo, hi;
                        draw_u53_pair(it.seed0 + uint64_t(ra & ~1), oi, uint32_t(sweep), 0u, &lo, &hi);
                        if (needa) acca = (par ? hi : lo) < ta;
                        if (needb) accb = (par ? lo : hi) < tb;
                    }
                    if (acca) {
                        s[pa] = int8_t(-sa);
                        Ea += dEa;
                    }
                    if (accb) {
                        s[pb] = int8_t(-sb);
                        Eb += dEb;
                    }
                    if (acca || accb) {
                        // f_j -= 2 w_ij s_i per flipped replica, wrap-around uint32
                        const uint32_t msa = sa > 0 ? 0xFFFFFFFEu : 2u, msb = sb > 0 ? 0xFFFFFFFEu : 2u;
                        const int32_t* __restrict__ row = it.row;
                        const int32_t* __restrict__ adj = it.adj;
                        const WT* __restrict__ w = static_cast<const WT*>(it.w);
                        int k = __ldg(row + i);
                        const int k1 = __ldg(row + i + 1);
                        for (; k + 4 <= k1; k += 4) {
                            int j[4];
                            uint32_t d[4];
#pragma unroll
                            for (int u = 0; u < 4; ++u) {
                                j[u] = __ldg(adj + k + u) << lg;
                                d[u] = uint32_t(int32_t(__ldg(w + k + u)));
                            }
                            if (acca) {
#pragma unroll
                                for (int u = 0; u < 4; ++u)
                                    atomicAdd(reinterpret_cast<unsigned int*>(&f[j[u] + ra]), d[u] * msa);
                            }
                            if (accb) {
#pragma unroll
                                for (int u = 0; u < 4; ++u)
                                    atomicAdd(reinterpret_cast<unsigned int*>(&f[j[u] + rb]), d[u] * msb);
                            }
                        }
                        for (; k < k1; ++k) {
                            const int j = __ldg(adj + k) << lg;
                            const uint32_t d = uint32_t(int32_t(__ldg(w + k)));
                            if (acca) atomicAdd(reinterpret_cast<unsigned int*>(&f[j + ra]), d * msa);
                            if (accb) atomicAdd(reinterpret_cast<unsigned int*>(&f[j + rb]), d * msb);
                        }
                    }
                }
                __syncthreads();
            }
        }
        atomicAdd(&e_sh[ra], (unsigned long long)Ea);
        atomicAdd(&e_sh[rb], (unsigned long long)Eb);
        __syncthreads();
        if (tid < G) {
            const long long prev = init ? 0ll : it.e_acc[tid];
            it.e_acc[tid] = prev + (long long)e_sh[tid];
        }
        ising_item_out<GLOBAL>(it, f, s, tid, bs);
        return;
    }
    // one replica per thread (groups of one replica): bs is a multiple of G,
    // so this thread always serves replica r
    const int r = tid & (G - 1);
    const uint64_t seed = it.seed0 - uint64_t(m) + uint64_t((m + r) & ~1);
    const int half = (m + r) & 1;
    long long E = 0;
    for (int sweep = sweep0; sweep < sweep1; ++sweep) {
        const double T = temp[sweep];
        if (table) {
            for (int k = tid + 1; k <= bound; k += bs) thr[k] = accept_threshold(k, T);
            __syncthreads();
        }
        for (int c = 0; c < n_colours; ++c) {
            const int p0 = (cls_sh ? cls[c] : class_ptr[c]) << lg;
            const int p1 = (cls_sh ? cls[c + 1] : class_ptr[c + 1]) << lg;
            for (int p = p0 + tid; p < p1; p += bs) {
                const int i = p >> lg;
                const uint32_t oi = uint32_t(__ldg(order + i));   // issued before the state loads
                const int si = s[p];
                const int dE = -si * f[p];
                bool acc = dE <= 0;
                if (!acc) {
                    const unsigned long long t = table ? thr[dE] : accept_threshold(dE, T);
                    if (t >= (1ull << 53)) acc = true;
                    else if (t != 0ull) acc = draw_u53_half(seed, oi, uint32_t(sweep), 0u, half) < t;
                }
                if (acc) {
                    s[p] = int8_t(-si);
                    E += dE;
                    // f_j -= 2 w_ij s_i in wrap-around uint32 arithmetic (the final
                    // field fits int32, a partial term may not)
                    const uint32_t ms = si > 0 ? 0xFFFFFFFEu : 2u;
                    // the CSR pointers are read from the shared descriptor here, at
                    // the (rarer) accepted flip, to keep them out of the registers
                    const int32_t* __restrict__ row = it.row;
                    const int32_t* __restrict__ adj = it.adj;
                    const WT* __restrict__ w = static_cast<const WT*>(it.w);
                    int k = __ldg(row + i);
                    const int k1 = __ldg(row + i + 1);
                    // four neighbours per step: their loads issue before the atomics
                    for (; k + 4 <= k1; k += 4) {
                        int j[4];
                        uint32_t d[4];
#pragma unroll
                        for (int q = 0; q < 4; ++q) {
                            j[q] = __ldg(adj + k + q);
                            d[q] = uint32_t(int32_t(__ldg(w + k + q))) * ms;
                        }
#pragma unroll
                        for (int q = 0; q < 4; ++q)
                            atomicAdd(reinterpret_cast<unsigned int*>(&f[(j[q] << lg) + r]), d[q]);
                    }
                    for (; k < k1; ++k)
                        atomicAdd(reinterpret_cast<unsigned int*>(&f[(__ldg(adj + k) << lg) + r]),
                                  uint32_t(int32_t(__ldg(w + k))) * ms);
                }
            }
            __syncthreads();
        }
    }
    atomicAdd(&e_sh[r], (unsigned long long)E);
    __syncthreads();
    if (tid < G) {
        const long long prev = init ? 0ll : it.e_acc[tid];
        it.e_acc[tid] = prev + (long long)e_sh[tid];
    }
    ising_item_out<GLOBAL>(it, f, s, tid, bs);
}

// items are handed out by ctl[0]; their count is n_items, or ctl[1] when
// n_items < 0 (a launch replayed from a graph reads it from device memory).
// MAXT: the largest CTA the instance serves, one CTA per SM (the item state
// fills the shared memory): 1024 threads get 64 registers each, 512 up to
// 128, room for the two-replica threads' state.
template <int MAXT>
__global__ void __launch_bounds__(MAXT, 1) ising_batch_kernel(const IsingItem* __restrict__ items, int n_items,
                                                                      int* ctl) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ unsigned long long thr[kThrMax + 1];
    __shared__ unsigned long long e_sh[kBatchMaxGroup];
    __shared__ __align__(16) IsingItem it;
    __shared__ int next;
    __shared__ int cls[kClassMax + 1];
    const int total = n_items >= 0 ? n_items : ctl[1];
    for (;;) {
        if (threadIdx.x == 0) next = atomicAdd(ctl, 1);
        __syncthreads();
        const int k = next;
        if (k >= total) return;
        constexpr int kWords = int(sizeof(IsingItem) / 8);
        if (threadIdx.x < kWords)
            reinterpret_cast<uint64_t*>(&it)[threadIdx.x] = reinterpret_cast<const uint64_t*>(items + k)[threadIdx.x];
        __syncthreads();
        const bool global = (it.flags & kItemGlobal) != 0;
        if (it.wbytes == 1) {
            if (global) ising_item<int8_t, true>(it, smem, thr, e_sh, cls);
            else ising_item<int8_t, false>(it, smem, thr, e_sh, cls);
        } else {
            if (global) ising_item<int32_t, true>(it, smem, thr, e_sh, cls);
            else ising_item<int32_t, false>(it, smem, thr, e_sh, cls);
        }
        __syncthreads();
    }
}

// Per-bit fraction of branches with x = 1 for every instance of a batch: the
// float division of branch_fractions (ising_recon.hpp:160-163) on exact counts.
__global__ void batch_marginals_kernel(const uint8_t* __restrict__ x, const BatchInstDev* __restrict__ inst, int n_inst,
                                       int64_t total, float* __restrict__ p) {
    for (int64_t g = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; g < total; g += int64_t(gridDim.x) * blockDim.x) {
        int lo = 0, hi = n_inst - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (inst[mid].p_off <= g) lo = mid;
            else hi = mid - 1;
        }
        const BatchInstDev d = inst[lo];
        const int64_t i = g - d.p_off;
        int cnt = 0;
        for (int r = 0; r < d.R; ++r) cnt += x[d.x_off + int64_t(r) * d.n + i];
        p[g] = float(cnt) / float(d.R);
    }
}

using BatchKernel = void (*)(const IsingItem*, int, int*);

BatchKernel batch_kernel(int threads) {
    return threads > 512 ? ising_batch_kernel<kBatchThreadsMax> : ising_batch_kernel<512>;
}

}  // namespace

qb_status launch_ising_batch_ctl(const IsingItem* d_items, int* d_ctl, const BatchShape& sh, cudaStream_t st) {
    if (sh.ctas <= 0) return fail(QB_EINVAL, "batch: the launch needs its CTA count");
    batch_kernel(sh.threads)<<<dim3(unsigned(sh.ctas)), dim3(unsigned(sh.threads)), size_t(sh.smem_bytes), st>>>(d_items, -1,
                                                                                                        d_ctl);
    QB_CUDA(cudaGetLastError());
    return QB_OK;
}

qb_status launch_batch_marginals(const uint8_t* x, const BatchInstDev* inst, int n_inst, int64_t total, float* p,
                                 cudaStream_t st) {
    if (total <= 0) return QB_OK;
    int64_t blocks = (total + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    batch_marginals_kernel<<<dim3(unsigned(blocks)), 256, 0, st>>>(x, inst, n_inst, total, p);
    QB_CUDA(cudaGetLastError());
    return QB_OK;
}

int batch_max_smem() {
    int dev = 0, optin = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) return 0;
    cudaFuncAttributes fa{};
    // both instances have the same static shared memory
    if (cudaFuncGetAttributes(&fa, ising_batch_kernel<kBatchThreadsMax>) != cudaSuccess) return 0;
    return optin - int(fa.sharedSizeBytes);
}

qb_status batch_ctas(const BatchShape& sh, int* ctas) {
    int dev = 0, sms = 0, occ = 0;
    QB_CUDA(cudaGetDevice(&dev));
    QB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    if (sh.threads < 32 || sh.threads > kBatchThreadsMax || sh.threads % kBatchMaxGroup)
        return fail(QB_EINVAL, "batch: threads must be a multiple of 32 in [32, 1024]");
    QB_CUDA(allow_max_smem(batch_kernel(sh.threads)));
    QB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, batch_kernel(sh.threads), sh.threads,
                                                          size_t(sh.smem_bytes)));
    if (occ < 1) return fail(QB_EREFUSED, "batch: the launch shape does not fit an SM");
    *ctas = occ * sms;
    return QB_OK;
}

qb_status launch_ising_batch(const IsingItem* d_items, int n_items, int* d_counter, const BatchShape& sh,
                             cudaStream_t st) {
    int ctas = sh.ctas;
    if (ctas <= 0) {
        qb_status s = batch_ctas(sh, &ctas);
        if (s != QB_OK) return s;
    } else {
        QB_CUDA(allow_max_smem(batch_kernel(sh.threads)));
    }
    if (n_items <= 0) return QB_OK;
    if (ctas > n_items) ctas = n_items;
    QB_CUDA(cudaMemsetAsync(d_counter, 0, sizeof(int), st));
    batch_kernel(sh.threads)<<<dim3(unsigned(ctas)), dim3(unsigned(sh.threads)), size_t(sh.smem_bytes), st>>>(d_items, n_items,
                                                                                                      d_counter);
    QB_CUDA(cudaGetLastError());
    return QB_OK;
}

}  // namespace qb
