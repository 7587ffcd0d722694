// Device assembly of a residual plan's large tables from the problem's own
// bit-major CSR (row_ptr, ray, a): the sweep-order entry table and the
// ray-major CSR with its three bit columns. The host plans the colouring,
// the slices and the per-bit tables; only the O(nnz) tables are built here,
// so the upload moves the 8 bytes per entry the caller already holds instead
// of 24 bytes per entry built on the host.
//
// The arrays are the host build's to the bit:
//   ent[h_row[k] + q] = {ray | (w[ray] < 0) << 31, fp32(sqrt|w[ray]| * a)} for
//     the q-th entry of the bit at sweep position k (the fp64 product rounded
//     once, as the host computes it);
//   the ray-major CSR lists every ray's bits in ascending input order (the
//     fp64 energy verifier and the residual refresh sum in that order): the
//     entries are scattered to their rays with atomics, then each ray's
//     segment is sorted by (bit, entry) keys, which are distinct.
#include <cuda_runtime.h>

#include <cstdint>

#include "qb_build.hpp"
#include "qb_internal.hpp"

namespace qb {

namespace {

constexpr int kBuildWarps = 8;          // warps per CTA of the entry and scatter kernels
constexpr int kSortWarps = 4;           // warps per CTA of the segment sort
constexpr int kScanThreads = 1024;

__global__ void __launch_bounds__(kBuildWarps * 32) build_entries_kernel(ResidBuildArgs A) {
    const int lane = int(threadIdx.x & 31u);
    const int warps = int(gridDim.x) * kBuildWarps;
    for (int k = int(blockIdx.x) * kBuildWarps + int(threadIdx.x >> 5); k < A.n; k += warps) {
        const int i = A.order[k];
        const int e0 = A.row_ptr[i], len = A.row_ptr[i + 1] - e0;
        const int dst = A.h_row[k];
        for (int q = lane; q < len; q += 32) {
            const int r = A.ray[e0 + q];
            const double w = A.w[r];
            const float ap = __double2float_rn(__dmul_rn(sqrt(fabs(w)), double(A.a[e0 + q])));
            A.ent[dst + q] = make_uint2(uint32_t(r) | (w < 0.0 ? 0x80000000u : 0u), __float_as_uint(ap));
            atomicAdd(&A.rcount[r], 1);
        }
    }
}

// rrow = exclusive prefix sum of rcount (one CTA: each thread sums a
// contiguous run, the run totals are scanned in shared memory, then each
// thread writes its run); cursor = rrow, the scatter's slot counters.
__global__ void __launch_bounds__(kScanThreads) ray_offsets_kernel(ResidBuildArgs A) {
    __shared__ int32_t part[kScanThreads];
    const int t = int(threadIdx.x);
    const int per = (A.n_rays + kScanThreads - 1) / kScanThreads;
    const int b0 = t * per, b1 = min(A.n_rays, b0 + per);
    int32_t s = 0;
    for (int b = b0; b < b1; ++b) s += A.rcount[b];
    part[t] = s;
    __syncthreads();
    for (int off = 1; off < kScanThreads; off <<= 1) {   // Hillis-Steele inclusive scan
        const int32_t v = t >= off ? part[t - off] : 0;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    int32_t run = part[t] - s;
    for (int b = b0; b < b1; ++b) {
        A.rrow[b] = run;
        A.cursor[b] = run;
        run += A.rcount[b];
    }
    if (t == kScanThreads - 1) A.rrow[A.n_rays] = part[t];
}

__global__ void __launch_bounds__(kBuildWarps * 32) scatter_rays_kernel(ResidBuildArgs A) {
    const int lane = int(threadIdx.x & 31u);
    const int warps = int(gridDim.x) * kBuildWarps;
    for (int i = int(blockIdx.x) * kBuildWarps + int(threadIdx.x >> 5); i < A.n; i += warps) {
        const int e0 = A.row_ptr[i], e1 = A.row_ptr[i + 1];
        for (int e = e0 + lane; e < e1; e += 32) {
            const int slot = atomicAdd(&A.cursor[A.ray[e]], 1);
            A.rkey[slot] = (static_cast<unsigned long long>(uint32_t(i)) << 32) | uint32_t(e);
        }
    }
}

// One warp per ray: bitonic sort of the segment's keys in shared memory
// (padded to a power of two with all-ones keys), then the bit columns.
__global__ void __launch_bounds__(kSortWarps * 32) sort_rays_kernel(ResidBuildArgs A) {
    extern __shared__ unsigned long long sk[];
    const int lane = int(threadIdx.x & 31u), wid = int(threadIdx.x >> 5);
    unsigned long long* s = sk + size_t(wid) * kRaySortMax;
    const int warps = int(gridDim.x) * kSortWarps;
    for (int r = int(blockIdx.x) * kSortWarps + wid; r < A.n_rays; r += warps) {
        const int s0 = A.rrow[r], len = A.rrow[r + 1] - s0;
        if (len == 0) continue;
        int P = 1;
        while (P < len) P <<= 1;
        for (int t = lane; t < P; t += 32) s[t] = t < len ? A.rkey[s0 + t] : ~0ull;
        __syncwarp();
        for (int k = 2; k <= P; k <<= 1)
            for (int j = k >> 1; j > 0; j >>= 1) {
                for (int t = lane; t < P; t += 32) {
                    const int u = t ^ j;
                    if (u > t) {
                        const unsigned long long x = s[t], y = s[u];
                        const bool up = (t & k) == 0;
                        if ((x > y) == up) {
                            s[t] = y;
                            s[u] = x;
                        }
                    }
                }
                __syncwarp();
            }
        for (int t = lane; t < len; t += 32) {
            const unsigned long long key = s[t];
            const int i = int(key >> 32), e = int(uint32_t(key));
            const int kpos = A.inverse[i];
            A.rbit_o[s0 + t] = i;
            A.rbit_n[s0 + t] = kpos;
            A.rbit_h[s0 + t] = A.bit_home[kpos];
            A.ra[s0 + t] = A.a[e];
        }
        __syncwarp();
    }
}

int grid_for(int items, int per_cta) {
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int want = (items + per_cta - 1) / per_cta;
    return want < 1 ? 1 : (want < sms * 8 ? want : sms * 8);
}

}  // namespace

size_t resid_sort_smem() { return size_t(kSortWarps) * kRaySortMax * sizeof(unsigned long long); }

qb_status launch_resid_build(const ResidBuildArgs& A, cudaStream_t st) {
    if (A.n_rays > 0) QB_CUDA(cudaMemsetAsync(A.rcount, 0, size_t(A.n_rays) * 4, st));
    if (A.n > 0) {
        build_entries_kernel<<<grid_for(A.n, kBuildWarps), kBuildWarps * 32, 0, st>>>(A);
        QB_CUDA(cudaGetLastError());
    }
    ray_offsets_kernel<<<1, kScanThreads, 0, st>>>(A);
    QB_CUDA(cudaGetLastError());
    if (A.n > 0) {
        scatter_rays_kernel<<<grid_for(A.n, kBuildWarps), kBuildWarps * 32, 0, st>>>(A);
        QB_CUDA(cudaGetLastError());
    }
    if (A.n_rays > 0) {
        const size_t smem = resid_sort_smem();
        QB_CUDA(cudaFuncSetAttribute(sort_rays_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
        sort_rays_kernel<<<grid_for(A.n_rays, kSortWarps), kSortWarps * 32, smem, st>>>(A);
        QB_CUDA(cudaGetLastError());
    }
    return QB_OK;
}

}  // namespace qb
