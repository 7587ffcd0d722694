// Exact local posterior of a region of interest.
//
// qb_roi_qubo builds the conditional QUBO of a region R of a residual-form
// problem with every other bit held at x_bar (roi_qubo,
// src/ising_recon.hpp:240-300): expanding 1/2 w (r + sum a x)^2 with x^2 = x,
// the linear field, the bonds inside R and the bonds to fixed neighbours
// gives E(x_R) - E(0_R) = sum_i h_i x_i + sum_{i<j} J_ij x_i x_j. It is host
// code that accumulates in the reference's order, so h and J are the
// reference's to the last bit.
//
// qb_enumerate_qubo visits all 2^n states of such a dense QUBO on the device
// (the reference stops at exporting it): each thread walks a block of
// consecutive Gray-code indices, so consecutive states differ in one bit and
// the energy and every bit's field update in O(n); it keeps a running minimum
// m, the sums of exp(-(E - m)/T) overall, per set bit and weighted by E, and
// rescales them when m drops. The partial sums are combined on the host in a
// fixed order: log Z, the exact marginals p(x_i = 1), the mean energy and the
// ground state, in fp64 and reproducible.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "qb_internal.hpp"

namespace qb {
namespace {

constexpr int kEnumMaxN = 34;
constexpr int kEnumThreads = 256;

// Per-thread partial: m, s0 (sum of weights), sE (sum of E * weight),
// e_min, x_min (as double bits), then s_i for i < n.
constexpr int kPartHead = 5;

__global__ void __launch_bounds__(kEnumThreads) enumerate_kernel(int n, const double* __restrict__ h,
                                                                 const double* __restrict__ Jsym, double inv_T,
                                                                 uint64_t per_thread, uint64_t total,
                                                                 double* __restrict__ part) {
    __shared__ double sJ[kEnumMaxN * kEnumMaxN];
    __shared__ double sh[kEnumMaxN];
    for (int k = int(threadIdx.x); k < n * n; k += kEnumThreads) sJ[k] = Jsym[k];
    for (int k = int(threadIdx.x); k < n; k += kEnumThreads) sh[k] = h[k];
    __syncthreads();
    const uint64_t t = uint64_t(blockIdx.x) * kEnumThreads + threadIdx.x;
    const uint64_t s_begin = t * per_thread;
    if (s_begin >= total) return;
    const uint64_t s_end = s_begin + per_thread < total ? s_begin + per_thread : total;
    uint64_t x = s_begin ^ (s_begin >> 1);   // Gray code of the first index
    double f[kEnumMaxN];                      // f_i = h_i + sum_j J_ij x_j
    double E = 0.0;
    for (int i = 0; i < n; ++i) {
        double fi = sh[i];
        for (int j = 0; j < n; ++j)
            if (j != i && ((x >> j) & 1ull)) fi += sJ[i * n + j];
        f[i] = fi;
    }
    for (int i = 0; i < n; ++i)
        if ((x >> i) & 1ull) {
            E += sh[i];
            for (int j = i + 1; j < n; ++j)
                if ((x >> j) & 1ull) E += sJ[i * n + j];
        }
    double m = E, s0 = 0.0, sE = 0.0, e_min = E;
    uint64_t x_min = x;
    double si[kEnumMaxN];
    for (int i = 0; i < n; ++i) si[i] = 0.0;
    for (uint64_t s = s_begin;; ) {
        if (E < m) {   // a new minimum: rescale what was summed
            const double c = exp(-(m - E) * inv_T);
            s0 *= c;
            sE *= c;
            for (int i = 0; i < n; ++i) si[i] *= c;
            m = E;
        }
        if (E < e_min) {
            e_min = E;
            x_min = x;
        }
        const double wgt = exp(-(E - m) * inv_T);
        s0 += wgt;
        sE += wgt * E;
        for (int i = 0; i < n; ++i)
            if ((x >> i) & 1ull) si[i] += wgt;
        if (++s >= s_end) break;
        // next Gray state: flip the bit of the lowest set bit of s
        const int b = __ffsll((long long)s) - 1;
        const double delta = ((x >> b) & 1ull) ? -1.0 : 1.0;
        E += delta * f[b];
        x ^= 1ull << b;
        for (int j = 0; j < n; ++j)
            if (j != b) f[j] += delta * sJ[j * n + b];
    }
    double* o = part + size_t(t) * size_t(kPartHead + n);
    o[0] = m;
    o[1] = s0;
    o[2] = sE;
    o[3] = e_min;
    o[4] = __longlong_as_double((long long)x_min);
    for (int i = 0; i < n; ++i) o[kPartHead + i] = si[i];
}

}  // namespace
}  // namespace qb

extern "C" qb_status qb_roi_qubo(const qb_residual_desc* p, const int32_t* roi, int32_t n_roi, const uint8_t* x_bar,
                                 double* h, double* J) {
    return qb::guarded("qb_roi_qubo", [&]() -> qb_status {
        using qb::fail;
        if (!p || !roi || !x_bar || !h || !J || n_roi < 0) return fail(QB_EINVAL, "qb_roi_qubo: null argument");
        const int nv = p->n_vars, nr = p->n_rays, n = n_roi;
        std::vector<int32_t> pos(static_cast<size_t>(nv), -1);
        for (int i = 0; i < n; ++i) {
            if (roi[i] < 0 || roi[i] >= nv) return fail(QB_EINVAL, "qb_roi_qubo: region index out of range");
            if (pos[size_t(roi[i])] >= 0) return fail(QB_EINVAL, "qb_roi_qubo: a bit appears twice in the region");
            pos[size_t(roi[i])] = i;
        }
        std::fill(h, h + n, 0.0);
        std::fill(J, J + size_t(n) * size_t(n), 0.0);
        // residuals with the region switched off
        std::vector<double> r(static_cast<size_t>(nr));
        for (int b = 0; b < nr; ++b) r[size_t(b)] = -p->d[b];
        for (int v = 0; v < nv; ++v)
            if (x_bar[v] && pos[size_t(v)] < 0)
                for (int k = p->row_ptr[v]; k < p->row_ptr[v + 1]; ++k) r[size_t(p->ray[k])] += p->a[k];
        // data terms through the rays the region touches (in ray order for the couplings)
        std::vector<std::vector<std::pair<int, double>>> on_ray;
        std::vector<int32_t> slot(static_cast<size_t>(nr), -1);
        std::vector<int32_t> touched;
        for (int i = 0; i < n; ++i)
            for (int k = p->row_ptr[roi[i]]; k < p->row_ptr[roi[i] + 1]; ++k) {
                const int b = p->ray[k];
                const double a = p->a[k];
                h[i] += p->w[b] * (r[size_t(b)] * a + 0.5 * a * a);
                if (slot[size_t(b)] < 0) {
                    slot[size_t(b)] = int32_t(on_ray.size());
                    on_ray.emplace_back();
                    touched.push_back(b);
                }
                on_ray[size_t(slot[size_t(b)])].push_back({i, a});
            }
        std::sort(touched.begin(), touched.end());
        for (int b : touched) {
            const auto& L = on_ray[size_t(slot[size_t(b)])];
            for (size_t u = 0; u < L.size(); ++u)
                for (size_t v = u + 1; v < L.size(); ++v) {
                    int i = L[u].first, j = L[v].first;
                    if (i > j) std::swap(i, j);
                    J[size_t(i) * size_t(n) + size_t(j)] += p->w[b] * L[u].second * L[v].second;
                }
        }
        // the prior: the linear field, bonds inside the region, bonds to fixed neighbours
        for (int i = 0; i < n; ++i) {
            const int vi = roi[i];
            h[i] += p->field ? p->field[vi] : p->kappa;
            for (int k = p->nbr_ptr[vi]; k < p->nbr_ptr[vi + 1]; ++k) {
                const int vj = p->nbr[k];
                const int pj = pos[size_t(vj)];
                if (pj >= 0) {
                    if (pj > i) {
                        h[i] += p->lambda;
                        h[pj] += p->lambda;
                        J[size_t(i) * size_t(n) + size_t(pj)] -= 2.0 * p->lambda;
                    }
                } else {
                    h[i] += p->lambda * (x_bar[vj] ? -1.0 : 1.0);
                }
            }
        }
        return QB_OK;
    });
}

extern "C" qb_status qb_enumerate_qubo(int32_t n, const double* h, const double* J, double T, const qb_opts* opts,
                                       qb_enum_result* out, double* marginals) {
    return qb::guarded("qb_enumerate_qubo", [&]() -> qb_status {
        using namespace qb;
        if (!h || !J || !out || !marginals) return fail(QB_EINVAL, "qb_enumerate_qubo: null argument");
        if (n < 1 || n > kEnumMaxN) return fail(QB_EINVAL, "qb_enumerate_qubo: n must be in [1, 34]");
        if (!(T > 0.0) || !std::isfinite(T)) return fail(QB_EINVAL, "qb_enumerate_qubo: T must be positive");
        for (int i = 0; i < n; ++i) {
            if (!std::isfinite(h[i])) return fail(QB_EINVAL, "qb_enumerate_qubo: non-finite h");
            for (int j = i + 1; j < n; ++j)
                if (!std::isfinite(J[size_t(i) * size_t(n) + size_t(j)])) return fail(QB_EINVAL, "qb_enumerate_qubo: non-finite J");
        }
        cudaStream_t st = opts ? static_cast<cudaStream_t>(opts->stream) : nullptr;
        if (opts && opts->device >= 0) QB_CUDA(cudaSetDevice(opts->device));
        // the upper triangle as a symmetric matrix with a zero diagonal
        std::vector<double> Js(size_t(n) * size_t(n), 0.0);
        for (int i = 0; i < n; ++i)
            for (int j = i + 1; j < n; ++j) Js[size_t(i) * n + j] = Js[size_t(j) * n + i] = J[size_t(i) * n + j];
        const uint64_t total = uint64_t(1) << n;
        const uint64_t max_threads = uint64_t(148) * 4 * kEnumThreads;
        uint64_t per = 1;
        while (total / per > max_threads) per <<= 1;
        const uint64_t threads = (total + per - 1) / per;
        const unsigned blocks = unsigned((threads + kEnumThreads - 1) / kEnumThreads);
        DevBuf d_h, d_J, d_part;
        qb_status s;
        if ((s = upload(d_h, h, size_t(n) * 8, st))) return s;
        if ((s = upload(d_J, Js.data(), Js.size() * 8, st))) return s;
        const size_t stride = size_t(kPartHead + n);
        if ((s = d_part.alloc(size_t(threads) * stride * 8))) return s;
        enumerate_kernel<<<blocks, kEnumThreads, 0, st>>>(n, d_h.as<double>(), d_J.as<double>(), 1.0 / T, per, total,
                                                          d_part.as<double>());
        QB_CUDA(cudaGetLastError());
        std::vector<double> part(size_t(threads) * stride);
        QB_CUDA(cudaMemcpyAsync(part.data(), d_part.p, part.size() * 8, cudaMemcpyDeviceToHost, st));
        QB_CUDA(cudaStreamSynchronize(st));
        // combine in thread order
        double m = INFINITY, e_min = INFINITY;
        for (uint64_t t = 0; t < threads; ++t) m = std::min(m, part[size_t(t) * stride]);
        double z = 0.0, ze = 0.0;
        uint64_t x_min = 0;
        std::vector<double> zi(static_cast<size_t>(n), 0.0);
        for (uint64_t t = 0; t < threads; ++t) {
            const double* o = &part[size_t(t) * stride];
            const double c = std::exp(-(o[0] - m) / T);
            z += o[1] * c;
            ze += o[2] * c;
            for (int i = 0; i < n; ++i) zi[size_t(i)] += o[kPartHead + i] * c;
            if (o[3] < e_min) {
                e_min = o[3];
                std::memcpy(&x_min, &o[4], 8);
            }
        }
        out->log_z = std::log(z) - m / T;
        out->e_min = e_min;
        out->x_min = x_min;
        out->mean_energy = ze / z;
        out->states = total;
        for (int i = 0; i < n; ++i) marginals[i] = zi[size_t(i)] / z;
        return QB_OK;
    });
}
