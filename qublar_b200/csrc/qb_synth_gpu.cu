// The tomography builder's ray march on the device: one thread per sky bin
// walks the bin's S x S sub-rays through the voxel grid in the host's order
// (Amanatides-Woo, as in qb_synth.cpp) and accumulates the optical depths and
// every reached bit's averaged chord in the host's operation order. Every
// floating-point step is an explicit round-to-nearest intrinsic, so nothing
// is contracted into a fused multiply-add, and the directions come from the
// host's cos/sin tables: the depths, chords and bit orders equal the host
// march's bit for bit. A bin dedups its bits with an open-addressing table in
// global memory; the Poisson draws, the ray selection and the CSR stay on the
// host (one sequential stream).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "qb_internal.hpp"
#include "qb_synth_march.hpp"

namespace qb {

namespace {

constexpr int kBinCap = 512;     // distinct bits one sky bin may reach
constexpr int kHashCap = 1024;   // open-addressing slots per bin (a power of two)
constexpr int kMarchThreads = 128;

struct MarchArgs {
    double lo[3];
    double v;
    int n[3];
    const int32_t* cell;       // per cell: its bit (>= 0), -1 rock without a bit, -2 not rock
    const uint8_t* is_void;
    double det[12];
    int n_theta, n_phi, S, n_bins;
    double inv_s2, mu_rock, mu_air;
    const double* cth;
    const double* sth;
    const double* cph;
    const double* sph;
    double* tau0;              // n_bins
    double* tau;               // n_bins
    int32_t* cnt;              // n_bins; -1: the bin overflowed its list
    int32_t* bits;             // n_bins x kBinCap
    double* len;               // n_bins x kBinCap
    unsigned long long* hash;  // n_bins x kHashCap: (bit + 1) << 32 | slot, 0 = empty
};

__global__ void __launch_bounds__(kMarchThreads) synth_march_kernel(MarchArgs A) {
    for (int b = int(blockIdx.x * blockDim.x + threadIdx.x); b < A.n_bins; b += int(gridDim.x * blockDim.x)) {
        const int k = b / (A.n_theta * A.n_phi), it = (b / A.n_phi) % A.n_theta, ip = b % A.n_phi;
        const double o[3] = {A.det[3 * k], A.det[3 * k + 1], A.det[3 * k + 2]};
        int32_t* bits = A.bits + size_t(b) * kBinCap;
        double* len = A.len + size_t(b) * kBinCap;
        unsigned long long* hs = A.hash + size_t(b) * kHashCap;
        double tau0 = 0.0, tau = 0.0;
        int cnt = 0;
        bool over = false;
        const double rock_w = __dmul_rn(A.inv_s2, A.mu_rock), air_w = __dmul_rn(A.inv_s2, A.mu_air);
        for (int su = 0; su < A.S; ++su)
            for (int sv = 0; sv < A.S; ++sv) {
                const double cs = A.cth[it * A.S + su], ss = A.sth[it * A.S + su];
                const int pi = (k * A.n_phi + ip) * A.S + sv;
                const double d[3] = {__dmul_rn(ss, A.cph[pi]), __dmul_rn(ss, A.sph[pi]), cs};
                const double under = __ddiv_rn(__dmul_rn(rock_w, -o[2]), cs);   // rock under the base
                tau0 = __dadd_rn(tau0, under);
                tau = __dadd_rn(tau, under);
                // slab entry and exit of the grid
                double t0 = 0.0, t1 = INFINITY;
                bool miss = false;
                for (int a = 0; a < 3; ++a) {
                    const double lo = A.lo[a], hi = __dadd_rn(A.lo[a], __dmul_rn(A.v, double(A.n[a])));
                    if (fabs(d[a]) < 1e-15) {
                        if (o[a] < lo || o[a] > hi) miss = true;
                        continue;
                    }
                    double ta = __ddiv_rn(__dsub_rn(lo, o[a]), d[a]), tb = __ddiv_rn(__dsub_rn(hi, o[a]), d[a]);
                    if (ta > tb) {
                        const double x = ta;
                        ta = tb;
                        tb = x;
                    }
                    t0 = t0 < ta ? ta : t0;
                    t1 = tb < t1 ? tb : t1;
                }
                if (miss || !(t0 < t1)) continue;
                int c[3], step[3];
                double tmax[3], tdel[3];
                for (int a = 0; a < 3; ++a) {
                    const double p = __dadd_rn(o[a], __dmul_rn(d[a], __dadd_rn(t0, 1e-9)));
                    int ci = int(floor(__ddiv_rn(__dsub_rn(p, A.lo[a]), A.v)));
                    ci = min(max(ci, 0), A.n[a] - 1);
                    c[a] = ci;
                    if (d[a] > 0) {
                        step[a] = 1;
                        tmax[a] = __ddiv_rn(__dsub_rn(__dadd_rn(A.lo[a], __dmul_rn(double(ci + 1), A.v)), o[a]), d[a]);
                        tdel[a] = __ddiv_rn(A.v, d[a]);
                    } else if (d[a] < 0) {
                        step[a] = -1;
                        tmax[a] = __ddiv_rn(__dsub_rn(__dadd_rn(A.lo[a], __dmul_rn(double(ci), A.v)), o[a]), d[a]);
                        tdel[a] = __ddiv_rn(-A.v, d[a]);
                    } else {
                        step[a] = 0;
                        tmax[a] = INFINITY;
                        tdel[a] = INFINITY;
                    }
                }
                double t = t0;
                for (;;) {
                    int ax = 0;
                    if (tmax[1] < tmax[ax]) ax = 1;
                    if (tmax[2] < tmax[ax]) ax = 2;
                    const double tn = t1 < tmax[ax] ? t1 : tmax[ax];
                    const double seg = __dsub_rn(tn, t);
                    if (seg > 0.0) {
                        const int64_t cell = (int64_t(c[2]) * A.n[1] + c[1]) * A.n[0] + c[0];
                        const int32_t cb = A.cell[cell];
                        if (cb != -2) {
                            tau0 = __dadd_rn(tau0, __dmul_rn(rock_w, seg));
                            tau = __dadd_rn(tau, __dmul_rn(A.is_void[cell] ? air_w : rock_w, seg));
                            if (cb >= 0 && !over) {
                                uint32_t h = (uint32_t(cb) * 2654435761u) >> (32 - 10);
                                int slot = -1;
                                for (;;) {
                                    const unsigned long long e = hs[h];
                                    if (e == 0ull) {
                                        if (cnt == kBinCap) break;
                                        slot = cnt++;
                                        hs[h] = (static_cast<unsigned long long>(uint32_t(cb) + 1u) << 32) | uint32_t(slot);
                                        bits[slot] = cb;
                                        len[slot] = 0.0;
                                        break;
                                    }
                                    if (uint32_t(e >> 32) == uint32_t(cb) + 1u) {
                                        slot = int(uint32_t(e));
                                        break;
                                    }
                                    h = (h + 1u) & uint32_t(kHashCap - 1);
                                }
                                if (slot < 0) over = true;
                                else len[slot] = __dadd_rn(len[slot], __dmul_rn(A.inv_s2, seg));
                            }
                        }
                    }
                    t = tn;
                    if (t >= t1) break;
                    c[ax] += step[ax];
                    if (c[ax] < 0 || c[ax] >= A.n[ax]) break;
                    tmax[ax] = __dadd_rn(tmax[ax], tdel[ax]);
                }
            }
        A.tau0[b] = tau0;
        A.tau[b] = tau;
        A.cnt[b] = over ? -1 : cnt;
    }
}

// The bins' lists packed in bin order: bit and fp32(mu_rock * chord), the
// host's rounding of the coefficient.
__global__ void synth_pack_kernel(const int32_t* __restrict__ cnt, const int64_t* __restrict__ off, int n_bins,
                                  const int32_t* __restrict__ bits, const double* __restrict__ len, double mu_rock,
                                  int32_t* __restrict__ e_bit, float* __restrict__ e_a) {
    const int lane = int(threadIdx.x & 31u);
    const int warps = int(gridDim.x * blockDim.x) >> 5;
    for (int b = int((blockIdx.x * blockDim.x + threadIdx.x) >> 5); b < n_bins; b += warps) {
        const int64_t o = off[b];
        for (int j = lane; j < cnt[b]; j += 32) {
            e_bit[o + j] = bits[size_t(b) * kBinCap + j];
            e_a[o + j] = __double2float_rn(__dmul_rn(mu_rock, len[size_t(b) * kBinCap + j]));
        }
    }
}

}  // namespace

qb_status synth_march_device(const SynthMarch& M, const qb_opts* opts, std::vector<BinMarch>& bins,
                             std::vector<int32_t>& e_bit, std::vector<float>& e_a) {
    int dev = opts && opts->device >= 0 ? opts->device : 0;
    if (!opts || opts->device < 0) QB_CUDA(cudaGetDevice(&dev));
    QB_CUDA(cudaSetDevice(dev));
    cudaStream_t st = opts ? static_cast<cudaStream_t>(opts->stream) : nullptr;
    const int n_bins = M.n_det * M.n_theta * M.n_phi;
    const int64_t ncell = M.g.cells();
    std::vector<int32_t> cell(static_cast<size_t>(ncell));
    for (int64_t c = 0; c < ncell; ++c) cell[size_t(c)] = M.rock[size_t(c)] ? M.cell_bit[size_t(c)] : -2;
    DevBuf d_cell, d_void, d_cth, d_sth, d_cph, d_sph, d_tau0, d_tau, d_cnt, d_bits, d_len, d_hash, d_off, d_ebit, d_ea;
    qb_status s;
    if ((s = upload_vec(d_cell, cell, st))) return s;
    if ((s = upload_vec(d_void, M.is_void, st))) return s;
    if ((s = upload_vec(d_cth, M.cth, st))) return s;
    if ((s = upload_vec(d_sth, M.sth, st))) return s;
    if ((s = upload_vec(d_cph, M.cph, st))) return s;
    if ((s = upload_vec(d_sph, M.sph, st))) return s;
    if ((s = d_tau0.alloc(size_t(n_bins) * 8))) return s;
    if ((s = d_tau.alloc(size_t(n_bins) * 8))) return s;
    if ((s = d_cnt.alloc(size_t(n_bins) * 4))) return s;
    if ((s = d_bits.alloc(size_t(n_bins) * kBinCap * 4))) return s;
    if ((s = d_len.alloc(size_t(n_bins) * kBinCap * 8))) return s;
    if ((s = d_hash.alloc(size_t(n_bins) * kHashCap * 8))) return s;
    QB_CUDA(cudaMemsetAsync(d_hash.p, 0, d_hash.bytes, st));
    MarchArgs A{};
    for (int a = 0; a < 3; ++a) {
        A.lo[a] = M.g.lo[a];
        A.n[a] = M.g.n[a];
    }
    A.v = M.g.v;
    A.cell = d_cell.as<int32_t>();
    A.is_void = d_void.as<uint8_t>();
    std::memcpy(A.det, M.det, sizeof A.det);
    A.n_theta = M.n_theta;
    A.n_phi = M.n_phi;
    A.S = M.S;
    A.n_bins = n_bins;
    A.inv_s2 = M.inv_s2;
    A.mu_rock = M.mu_rock;
    A.mu_air = M.mu_air;
    A.cth = d_cth.as<double>();
    A.sth = d_sth.as<double>();
    A.cph = d_cph.as<double>();
    A.sph = d_sph.as<double>();
    A.tau0 = d_tau0.as<double>();
    A.tau = d_tau.as<double>();
    A.cnt = d_cnt.as<int32_t>();
    A.bits = d_bits.as<int32_t>();
    A.len = d_len.as<double>();
    A.hash = d_hash.as<unsigned long long>();
    synth_march_kernel<<<unsigned((n_bins + kMarchThreads - 1) / kMarchThreads), kMarchThreads, 0, st>>>(A);
    QB_CUDA(cudaGetLastError());
    std::vector<double> tau0(static_cast<size_t>(n_bins)), tau(static_cast<size_t>(n_bins));
    std::vector<int32_t> cnt(static_cast<size_t>(n_bins));
    QB_CUDA(cudaMemcpyAsync(tau0.data(), d_tau0.p, tau0.size() * 8, cudaMemcpyDeviceToHost, st));
    QB_CUDA(cudaMemcpyAsync(tau.data(), d_tau.p, tau.size() * 8, cudaMemcpyDeviceToHost, st));
    QB_CUDA(cudaMemcpyAsync(cnt.data(), d_cnt.p, cnt.size() * 4, cudaMemcpyDeviceToHost, st));
    QB_CUDA(cudaStreamSynchronize(st));
    bins.assign(static_cast<size_t>(n_bins), BinMarch{});
    std::vector<int64_t> off(static_cast<size_t>(n_bins));
    int64_t total = 0;
    for (int b = 0; b < n_bins; ++b) {
        if (cnt[size_t(b)] < 0)
            return fail(QB_ENOTSUP, "qb_synth_tomography_device: a sky bin reaches more than 512 bits "
                                    "(qb_synth_tomography builds it on the host)");
        bins[size_t(b)] = BinMarch{tau0[size_t(b)], tau[size_t(b)], total, cnt[size_t(b)]};
        off[size_t(b)] = total;
        total += cnt[size_t(b)];
    }
    e_bit.resize(size_t(total));
    e_a.resize(size_t(total));
    if (total > 0) {
        if ((s = upload_vec(d_off, off, st))) return s;
        if ((s = d_ebit.alloc(size_t(total) * 4))) return s;
        if ((s = d_ea.alloc(size_t(total) * 4))) return s;
        synth_pack_kernel<<<unsigned(std::min(n_bins / 8 + 1, 148 * 16)), 256, 0, st>>>(
            d_cnt.as<int32_t>(), d_off.as<int64_t>(), n_bins, d_bits.as<int32_t>(), d_len.as<double>(), M.mu_rock,
            d_ebit.as<int32_t>(), d_ea.as<float>());
        QB_CUDA(cudaGetLastError());
        QB_CUDA(cudaMemcpyAsync(e_bit.data(), d_ebit.p, size_t(total) * 4, cudaMemcpyDeviceToHost, st));
        QB_CUDA(cudaMemcpyAsync(e_a.data(), d_ea.p, size_t(total) * 4, cudaMemcpyDeviceToHost, st));
    }
    QB_CUDA(cudaStreamSynchronize(st));
    return QB_OK;
}

}  // namespace qb
