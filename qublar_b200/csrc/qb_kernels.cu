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
//   evaluates them. A warp scores a bit with a lane-strided gather over its
//   rays, dE = delta (lin + sum_k a_k rw_k) + q + lambda (deg - 2 unlike),
//   q = 1/2 sum_k w a_k^2 (the local_field_dE of src/ising_recon.hpp:105-118
//   regrouped), and scatters rw += w a delta on accept. A class never holds
//   two bits of one ray, so the scatter needs no atomics; a cluster barrier
//   separates classes. Residuals are fp32 and are recomputed from scratch in
//   fp64 every `refresh` sweeps.
//
// Metropolis (both forms): accept if dE <= 0, else if u < exp(-dE/T) in
// double, u the 53-bit Philox draw of (branch seed, original bit, sweep) --
// the acceptance expression of ising_weighted.hpp:260 / ising_recon.hpp:136.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "qb_kernels.hpp"
#include "qb_philox.cuh"

namespace cg = cooperative_groups;

namespace qb {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kIsingThreads = 512;
constexpr int kResidThreads = 256;
constexpr uint32_t kSlotBits = 27;
constexpr uint32_t kSlotMask = (1u << kSlotBits) - 1u;

__device__ __forceinline__ bool metropolis(double dE, double T, uint64_t seed, uint32_t bit, uint32_t sweep) {
    if (dE <= 0.0) return true;
    const uint64_t u53 = draw_u53(seed, bit, sweep, 0u);
    return double(u53) * 0x1.0p-53 < exp(-dE / T);
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
    uint8_t* x_out;       // R x n
    int32_t* f_out;       // R x n
    long long* e_out;     // R
};

template <typename WT, bool SMEM>
__global__ void __launch_bounds__(kIsingThreads) ising_anneal_kernel(IsingArgs A) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ long long red[kIsingThreads / 32];
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
    __syncthreads();
    const uint64_t seed = A.seed0 + uint64_t(rep);
    const WT* w = static_cast<const WT*>(A.w);
    long long E = 0;
    for (int sweep = 0; sweep < A.sweeps; ++sweep) {
        const double T = A.temp[sweep];
        for (int c = 0; c < A.n_colours; ++c) {
            const int c1 = A.class_ptr[c + 1];
            for (int i = A.class_ptr[c] + int(threadIdx.x); i < c1; i += blockDim.x) {
                const int si = s[i];
                const long long dE = -(long long)si * (long long)f[i];
                if (metropolis(double(dE), T, seed, uint32_t(A.order[i]), uint32_t(sweep))) {
                    s[i] = int8_t(-si);
                    E += dE;
                    const int r1 = A.row[i + 1];
                    // f_j -= 2 w_ij s_i, in wrap-around uint32 arithmetic: the
                    // final field fits int32 (|f| <= field bound), the term may not
                    const uint32_t ms = si > 0 ? 0xFFFFFFFEu : 2u;   // -2 s_i mod 2^32
                    for (int k = A.row[i]; k < r1; ++k)
                        atomicAdd(reinterpret_cast<unsigned int*>(&f[A.adj[k]]), uint32_t(int32_t(w[k])) * ms);
                }
            }
            __syncthreads();
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
    int n_colours;
    int sweeps;
    int refresh;
    int ray_slots;
    int bit_slots;
    float lambda;
    uint64_t seed0;
    const int32_t* class_ptr;
    const int32_t* slot_base;   // n_colours * CL
    const int32_t* row;
    const int32_t* ray;
    const float* a;
    const float* lin;
    const float* q;
    const int32_t* nbr_ptr;
    const uint32_t* nbr_home;
    const int32_t* order;
    const double* d;
    const double* w64;
    const float* wf;
    const int32_t* rrow;
    const uint32_t* rbit_home;
    const float* ra;
    const double* temp;
    uint8_t* x_out;
    float* drift;
};

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ uint32_t map_rank(uint32_t addr, uint32_t rank) {
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(addr), "r"(rank));
    return r;
}
__device__ __forceinline__ float2 ld_cluster_f2(uint32_t addr) {
    float2 v;
    asm volatile("ld.shared::cluster.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "r"(addr) : "memory");
    return v;
}
__device__ __forceinline__ void st_cluster_f32(uint32_t addr, float v) {
    asm volatile("st.shared::cluster.f32 [%0], %1;" ::"r"(addr), "f"(v) : "memory");
}
__device__ __forceinline__ uint32_t ld_cluster_u8(uint32_t addr) {
    uint32_t v;
    asm volatile("ld.shared::cluster.u8 %0, [%1];" : "=r"(v) : "r"(addr) : "memory");
    return v;
}

template <int CL>
__global__ void __launch_bounds__(kResidThreads) resid_anneal_kernel(ResidArgs A) {
    static_assert((CL & (CL - 1)) == 0 && CL <= 16, "cluster size: a power of two <= 16");
    extern __shared__ __align__(16) unsigned char smem[];
    float2* rw = reinterpret_cast<float2*>(smem);                        // (w r, w) per owned ray
    uint8_t* xs = smem + size_t(A.ray_slots) * sizeof(float2);         // owned bits
    cg::cluster_group cluster = cg::this_cluster();
    const uint32_t rank = cluster.block_rank();
    const int branch = int(blockIdx.x) / CL;
    const int lane = int(threadIdx.x & 31u);
    const int warp = int(threadIdx.x >> 5);
    constexpr int kWarps = kResidThreads / 32;
    constexpr int kShift = CL == 1 ? 0 : CL == 2 ? 1 : CL == 4 ? 2 : CL == 8 ? 3 : 4;
    const uint64_t seed = A.seed0 + uint64_t(branch);
    const uint32_t rw_base = smem_addr(rw);
    const uint32_t xs_base = smem_addr(xs);

    for (int sl = int(threadIdx.x); sl < A.ray_slots; sl += kResidThreads) {
        const int b = (sl << kShift) + int(rank);
        float2 v = make_float2(0.0f, 0.0f);
        if (b < A.n_rays) {
            v.x = float(A.w64[b] * (-A.d[b]));
            v.y = A.wf[b];
        }
        rw[sl] = v;
    }
    for (int sl = int(threadIdx.x); sl < A.bit_slots; sl += kResidThreads) xs[sl] = 0;
    cluster.sync();

    for (int sweep = 0; sweep < A.sweeps; ++sweep) {
        if (A.refresh > 0 && sweep > 0 && sweep % A.refresh == 0) {
            // fp64 refresh of the owned residuals: r_b = sum_{v on b, x_v} a - d_b
            float dmax = 0.0f;
            for (int sl = warp; sl < A.ray_slots; sl += kWarps) {
                const int b = (sl << kShift) + int(rank);
                if (b >= A.n_rays) continue;
                double acc = 0.0;
                for (int k = A.rrow[b] + lane; k < A.rrow[b + 1]; k += 32) {
                    const uint32_t h = A.rbit_home[k];
                    if (ld_cluster_u8(map_rank(xs_base + (h & kSlotMask), h >> kSlotBits))) acc += double(A.ra[k]);
                }
#pragma unroll
                for (int off = 16; off > 0; off >>= 1) acc = acc + __shfl_xor_sync(kFull, acc, off);
                if (lane == 0) {
                    const float nv = float(A.w64[b] * (acc - A.d[b]));
                    dmax = fmaxf(dmax, fabsf(nv - rw[sl].x));
                    rw[sl].x = nv;
                }
            }
            if (lane == 0 && dmax > 0.0f) atomicMax(reinterpret_cast<int*>(&A.drift[branch]), __float_as_int(dmax));
            cluster.sync();
        }
        const double T = A.temp[sweep];
        for (int c = 0; c < A.n_colours; ++c) {
            const int cs = A.class_ptr[c], ce = A.class_ptr[c + 1];
            const int chunk = (ce - cs + CL - 1) / CL;
            const int b0 = cs + int(rank) * chunk;
            const int b1 = min(b0 + chunk, ce);
            const int slot0 = A.slot_base[c * CL + int(rank)];
            for (int i = b0 + warp; i < b1; i += kWarps) {
                const int rs = A.row[i], re = A.row[i + 1];
                float acc = 0.0f;
                for (int k = rs + lane; k < re; k += 32) {
                    const int rb = A.ray[k];
                    const float2 v = ld_cluster_f2(map_rank(rw_base + uint32_t(rb >> kShift) * 8u, uint32_t(rb & (CL - 1))));
                    acc = fmaf(A.a[k], v.x, acc);
                }
#pragma unroll
                for (int off = 16; off > 0; off >>= 1) acc = __fadd_rn(acc, __shfl_xor_sync(kFull, acc, off));
                const int slot = slot0 + (i - b0);
                const uint32_t xi = xs[slot];
                const int np0 = A.nbr_ptr[i], np1 = A.nbr_ptr[i + 1];
                int unlike = 0;
                for (int k = np0 + lane; k < np1; k += 32) {
                    const uint32_t h = A.nbr_home[k];
                    unlike += ld_cluster_u8(map_rank(xs_base + (h & kSlotMask), h >> kSlotBits)) != xi ? 1 : 0;
                }
                unlike = __reduce_add_sync(kFull, unlike);
                const float delta = xi ? -1.0f : 1.0f;
                int accept = 0;
                if (lane == 0) {
                    const float t = __fadd_rn(A.lin[i], acc);
                    const float prior = __fmul_rn(A.lambda, float((np1 - np0) - 2 * unlike));
                    const float dE = __fadd_rn(__fadd_rn(__fmul_rn(delta, t), A.q[i]), prior);
                    accept = metropolis(double(dE), T, seed, uint32_t(A.order[i]), uint32_t(sweep)) ? 1 : 0;
                }
                accept = __shfl_sync(kFull, accept, 0);
                if (accept) {
                    for (int k = rs + lane; k < re; k += 32) {
                        const int rb = A.ray[k];
                        const uint32_t ad = map_rank(rw_base + uint32_t(rb >> kShift) * 8u, uint32_t(rb & (CL - 1)));
                        const float2 v = ld_cluster_f2(ad);
                        const float upd = __fmul_rn(v.y, A.a[k]);
                        st_cluster_f32(ad, xi ? __fsub_rn(v.x, upd) : __fadd_rn(v.x, upd));
                    }
                    if (lane == 0) xs[slot] = uint8_t(xi ^ 1u);
                }
            }
            cluster.sync();
        }
    }
    // branches out, original bit order
    for (int c = 0; c < A.n_colours; ++c) {
        const int cs = A.class_ptr[c], ce = A.class_ptr[c + 1];
        const int chunk = (ce - cs + CL - 1) / CL;
        const int b0 = cs + int(rank) * chunk;
        const int b1 = min(b0 + chunk, ce);
        const int slot0 = A.slot_base[c * CL + int(rank)];
        for (int i = b0 + int(threadIdx.x); i < b1; i += kResidThreads)
            A.x_out[size_t(branch) * size_t(A.n) + size_t(A.order[i])] = xs[slot0 + (i - b0)];
    }
    cluster.sync();   // no CTA leaves while a peer may still read its shared memory
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

__global__ void __launch_bounds__(1024) resid_energy_kernel(ResidEnergyArgs A) {
    __shared__ double red[32];
    const uint8_t* x = A.X + size_t(blockIdx.x) * size_t(A.n);
    double data = 0.0, prior = 0.0;
    for (int b = int(threadIdx.x); b < A.n_rays; b += blockDim.x) {
        double r = -A.d[b];
        for (int k = A.rrow[b]; k < A.rrow[b + 1]; ++k)
            if (x[A.rbit[k]]) r += double(A.ra[k]);
        data += 0.5 * A.w[b] * r * r;
    }
    for (int i = int(threadIdx.x); i < A.n; i += blockDim.x) {
        prior += A.lin[i] * double(x[i]);
        for (int k = A.nbr_ptr[i]; k < A.nbr_ptr[i + 1]; ++k)
            if (A.nbr[k] > i && x[A.nbr[k]] != x[i]) prior += A.lambda;
    }
    const double sd = block_sum_f64(data, red);
    const double sp = block_sum_f64(prior, red);
    if (threadIdx.x == 0) A.e[blockIdx.x] = sd + sp;
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
    const size_t smem = ising_smem_bytes(p);
    if (smem == 0) {
        if (!b.scratch) return fail(QB_EINVAL, "ising sweep: global state needs scratch");
        A.f_scratch = static_cast<int32_t*>(b.scratch);
        A.s_scratch = reinterpret_cast<int8_t*>(A.f_scratch + size_t(R) * size_t(p.n));
    }
    const dim3 grid(static_cast<unsigned>(R)), block(kIsingThreads);
    if (smem) {
        if (p.weight_bytes == 1) {
            QB_CUDA(cudaFuncSetAttribute(ising_anneal_kernel<int8_t, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
            ising_anneal_kernel<int8_t, true><<<grid, block, smem, st>>>(A);
        } else {
            QB_CUDA(cudaFuncSetAttribute(ising_anneal_kernel<int32_t, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
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

size_t resid_smem_bytes(const ResidualPlan& p) {
    return size_t(p.ray_slots) * sizeof(float2) + size_t(p.bit_slots);
}

namespace {
template <int CL>
qb_status resid_launch_cl(const ResidArgs& A, int R, size_t smem, cudaStream_t st, bool check_only) {
    auto kern = resid_anneal_kernel<CL>;
    QB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
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
    A.n_colours = p.col.n_colours();
    A.sweeps = sweeps;
    A.refresh = refresh;
    A.ray_slots = p.ray_slots;
    A.bit_slots = p.bit_slots;
    A.lambda = float(p.lambda);
    A.seed0 = seed0;
    A.class_ptr = p.d_class_ptr.as<int32_t>();
    A.slot_base = p.d_slot_base.as<int32_t>();
    A.row = p.d_row.as<int32_t>();
    A.ray = p.d_ray.as<int32_t>();
    A.a = p.d_a.as<float>();
    A.lin = p.d_lin.as<float>();
    A.q = p.d_q.as<float>();
    A.nbr_ptr = p.d_nbr_ptr.as<int32_t>();
    A.nbr_home = p.d_nbr_home.as<uint32_t>();
    A.order = p.d_order.as<int32_t>();
    A.d = p.d_d.as<double>();
    A.w64 = p.d_w64.as<double>();
    A.wf = p.d_wf.as<float>();
    A.rrow = p.d_rrow.as<int32_t>();
    A.rbit_home = p.d_rbit.as<uint32_t>();
    A.ra = p.d_ra.as<float>();
    A.temp = b.temp;
    A.x_out = b.x;
    A.drift = b.drift;
    const size_t smem = resid_smem_bytes(p);
    switch (p.CL) {
        case 4: return resid_launch_cl<4>(A, R, smem, st, false);
        case 8: return resid_launch_cl<8>(A, R, smem, st, false);
        case 16: return resid_launch_cl<16>(A, R, smem, st, false);
        default: return fail(QB_EINVAL, "residual sweep: cluster size must be 4, 8 or 16");
    }
}

qb_status resid_check_fit(const ResidualPlan& p) {
    ResidArgs A{};
    const size_t smem = resid_smem_bytes(p);
    if (smem > size_t(227) * 1024) return fail(QB_ENOTSUP, "residual sweep: state exceeds the cluster's shared memory");
    switch (p.CL) {
        case 4: return resid_launch_cl<4>(A, 1, smem, nullptr, true);
        case 8: return resid_launch_cl<8>(A, 1, smem, nullptr, true);
        case 16: return resid_launch_cl<16>(A, 1, smem, nullptr, true);
        default: return fail(QB_EINVAL, "residual sweep: cluster size must be 4, 8 or 16");
    }
}

qb_status launch_resid_energies(const ResidualPlan& p, const uint8_t* x, int K, double* e, cudaStream_t st) {
    if (K == 0) return QB_OK;
    ResidEnergyArgs A{};
    A.n = p.n;
    A.n_rays = p.n_rays;
    A.lambda = p.lambda;
    A.d = p.d_d.as<double>();
    A.w = p.d_w64.as<double>();
    A.rrow = p.d_o_rrow.as<int32_t>();
    A.rbit = p.d_o_rbit.as<int32_t>();
    A.ra = p.d_o_ra.as<float>();
    A.lin = p.d_o_lin.as<double>();
    A.nbr_ptr = p.d_o_nbr_ptr.as<int32_t>();
    A.nbr = p.d_o_nbr.as<int32_t>();
    A.X = x;
    A.e = e;
    resid_energy_kernel<<<unsigned(K), 1024, 0, st>>>(A);
    QB_CUDA(cudaGetLastError());
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

}  // namespace qb
