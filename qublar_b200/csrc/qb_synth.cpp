// Synthetic muon-tomography QUBO of a square-base pyramid (known truth).
//
// The construction follows the reference's problem builder in structure:
//   bits      = grid cells in the domain, x-fastest, 6-neighbour adjacency
//               (BitField::grid, src/engine.hpp:61-85)
//   rows      = one straight ray per populated sky bin of each detector:
//               d = tau0 - t, w = max(N_det, 1), a = mu_rock * chord
//               (muon_rows, src/op_muon.hpp:22-51)
//   CSR       = entries grouped by bit (assemble, src/engine.hpp:120-149;
//               here the order inside a bit is by ray, deterministically)
// The geometry is this project's own: detectors sit below the base and look
// up through the pyramid across zenith bins; chords come from an
// Amanatides-Woo voxel walk (J. Amanatides, A. Woo, "A fast voxel traversal
// algorithm for ray tracing", Eurographics 1987); counts are Poisson with
// Beer-Lambert transmission, the void being air.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <new>
#include <vector>

#include "qb_internal.hpp"
#include "qb_synth_march.hpp"
#include "qublar_synth.h"

namespace {

uint64_t splitmix_next(uint64_t& s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
double uniform01(uint64_t& s) { return double(splitmix_next(s) >> 11) * 0x1.0p-53; }

// Poisson(lam): Knuth's product of uniforms below 30, a rounded normal
// (Box-Muller) above; deterministic in the stream.
int64_t poisson(double lam, uint64_t& s) {
    if (lam <= 0.0) return 0;
    if (lam < 30.0) {
        const double L = std::exp(-lam);
        int64_t k = 0;
        double p = 1.0;
        do { ++k; p *= uniform01(s); } while (p > L);
        return k - 1;
    }
    double u1 = uniform01(s);
    const double u2 = uniform01(s);
    if (u1 < 1e-300) u1 = 1e-300;
    const double z = std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * M_PI * u2);
    const double v = std::floor(lam + std::sqrt(lam) * z + 0.5);
    return v < 0.0 ? 0 : int64_t(v);
}

using qb::BinMarch;
using qb::Grid;
using qb::SynthMarch;

// Voxel walk: visit(cell, chord) for every cell the ray crosses, in order.
template <class Visit>
void march(const Grid& g, const double o[3], const double d[3], Visit visit) {
    double t0 = 0.0, t1 = std::numeric_limits<double>::infinity();
    for (int a = 0; a < 3; ++a) {
        const double lo = g.lo[a], hi = g.lo[a] + g.v * g.n[a];
        if (std::fabs(d[a]) < 1e-15) {
            if (o[a] < lo || o[a] > hi) return;
            continue;
        }
        double ta = (lo - o[a]) / d[a], tb = (hi - o[a]) / d[a];
        if (ta > tb) std::swap(ta, tb);
        t0 = std::max(t0, ta);
        t1 = std::min(t1, tb);
    }
    if (!(t0 < t1)) return;
    int c[3], step[3];
    double tmax[3], tdel[3];
    for (int a = 0; a < 3; ++a) {
        const double p = o[a] + d[a] * (t0 + 1e-9);
        int ci = int(std::floor((p - g.lo[a]) / g.v));
        ci = std::min(std::max(ci, 0), g.n[a] - 1);
        c[a] = ci;
        if (d[a] > 0) {
            step[a] = 1;
            tmax[a] = (g.lo[a] + (ci + 1) * g.v - o[a]) / d[a];
            tdel[a] = g.v / d[a];
        } else if (d[a] < 0) {
            step[a] = -1;
            tmax[a] = (g.lo[a] + ci * g.v - o[a]) / d[a];
            tdel[a] = -g.v / d[a];
        } else {
            step[a] = 0;
            tmax[a] = std::numeric_limits<double>::infinity();
            tdel[a] = std::numeric_limits<double>::infinity();
        }
    }
    double t = t0;
    for (;;) {
        int ax = 0;
        if (tmax[1] < tmax[ax]) ax = 1;
        if (tmax[2] < tmax[ax]) ax = 2;
        const double tn = std::min(tmax[ax], t1);
        const double seg = tn - t;
        if (seg > 0.0) visit((int64_t(c[2]) * g.n[1] + c[1]) * g.n[0] + c[0], seg);
        t = tn;
        if (t >= t1) break;
        c[ax] += step[ax];
        if (c[ax] < 0 || c[ax] >= g.n[ax]) break;
        tmax[ax] += tdel[ax];
    }
}

// Every sky bin's row on the host: chords averaged over the S x S sub-rays
// spread over the bin's solid angle (S = 1: the bin's centre line), bits in
// the order the sub-rays first reach them.
qb_status march_host(const SynthMarch& M, std::vector<BinMarch>& bins, std::vector<int32_t>& e_bit,
                     std::vector<float>& e_a) {
    const int S = M.S;
    bins.assign(size_t(M.n_det) * M.n_theta * M.n_phi, BinMarch{});
    std::vector<int64_t> stamp(size_t(M.n_bits), -1);
    std::vector<int32_t> slot(size_t(M.n_bits), 0);
    std::vector<double> e_len;
    int64_t stamp_id = 0;
    for (int k = 0; k < M.n_det; ++k) {
        const double* o = &M.det[3 * k];
        for (int it = 0; it < M.n_theta; ++it)
            for (int ip = 0; ip < M.n_phi; ++ip) {
                BinMarch& B = bins[(size_t(k) * M.n_theta + it) * M.n_phi + ip];
                double tau0 = 0.0, tau = 0.0;
                const int64_t first = int64_t(e_bit.size());
                for (int su = 0; su < S; ++su)
                    for (int sv = 0; sv < S; ++sv) {
                        const double cs = M.cth[size_t(it) * S + su], ss = M.sth[size_t(it) * S + su];
                        const size_t pi = (size_t(k) * M.n_phi + ip) * S + sv;
                        const double dir[3] = {ss * M.cph[pi], ss * M.sph[pi], cs};
                        tau0 += M.inv_s2 * M.mu_rock * (-o[2]) / cs;   // rock under the base
                        tau += M.inv_s2 * M.mu_rock * (-o[2]) / cs;
                        march(M.g, o, dir, [&](int64_t c, double seg) {
                            if (!M.rock[size_t(c)]) return;
                            tau0 += M.inv_s2 * M.mu_rock * seg;
                            tau += M.inv_s2 * (M.is_void[size_t(c)] ? M.mu_air : M.mu_rock) * seg;
                            const int b = M.cell_bit[size_t(c)];
                            if (b < 0) return;
                            if (stamp[size_t(b)] != stamp_id) {
                                stamp[size_t(b)] = stamp_id;
                                slot[size_t(b)] = int32_t(int64_t(e_bit.size()) - first);
                                e_bit.push_back(b);
                                e_len.push_back(0.0);
                            }
                            e_len[size_t(slot[size_t(b)])] += M.inv_s2 * seg;
                        });
                    }
                ++stamp_id;
                for (double len : e_len) e_a.push_back(float(M.mu_rock * len));
                e_len.clear();
                B.tau0 = tau0;
                B.tau = tau;
                B.first = first;
                B.cnt = int64_t(e_bit.size()) - first;
            }
    }
    return QB_OK;
}

}  // namespace

struct qb_tomo {
    int32_t dims[3] = {0, 0, 0};      // the voxel grid, x fastest
    std::vector<int64_t> bit_cell;    // the grid cell of every bit
    std::vector<double> d, w;
    std::vector<int32_t> row_ptr, ray;
    std::vector<float> a;
    std::vector<int32_t> nbr_ptr, nbr;
    std::vector<uint8_t> truth;
    double lambda = 0.0, kappa = 0.0;
};

extern "C" void qb_tomo_params_default(qb_tomo_params* p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    // A Khufu-proportioned pyramid (height / half base = 139 / 115): 87 m
    // half base, 105.16 m high, voxelised to 1.5 m cubes; the first 306,328
    // cells (x fastest, from the base up) are the bits, the apex is rock.
    p->target_bits = 306328;
    p->target_rays = 75594;
    p->voxel = 1.5;
    p->half_base = 87.0;
    p->height = 87.0 * 139.0 / 115.0;
    // Three detectors in galleries 2 m under the base, near the rim, each
    // looking inward across the pyramid at low elevation (zenith 50-88
    // degrees, +-70 degrees of azimuth around the axis): long chords. With
    // chords averaged over 4 x 4 sub-rays a row holds about 148 cells.
    p->n_detectors = 3;
    const double R = 0.80 * p->half_base;
    for (int k = 0; k < 3; ++k) {
        const double ang = 2.0 * M_PI * k / 3.0 + M_PI / 6.0;
        p->det[3 * k + 0] = R * std::cos(ang);
        p->det[3 * k + 1] = R * std::sin(ang);
        p->det[3 * k + 2] = -2.0;
    }
    p->n_theta = 70;
    p->n_phi = 360;
    p->theta_min = 50.0 * M_PI / 180.0;
    p->theta_max = 88.0 * M_PI / 180.0;
    p->phi_half = 70.0 * M_PI / 180.0;
    p->mu_rock = 0.046;
    p->void_center[0] = 6.0;
    p->void_center[1] = -4.0;
    p->void_center[2] = 30.0;
    p->void_side = 30.0;
    p->exposure = 2.0e9;
    p->min_open = 30.0;
    p->sub_rays = 4;
    p->room_radius = 12.0;   // every ray of a detector fans out of its room
    p->lambda = 2.0;
    p->kappa = std::log(999.0);   // prior void fraction 1e-3
    p->seed = 20260929ull;
}

namespace {

qb_status synth_tomography(const qb_tomo_params* p, bool on_device, const qb_opts* opts, qb_tomo** out) {
    if (!p || !out) return qb::fail(QB_EINVAL, "qb_synth_tomography: null argument");
    *out = nullptr;
    if (p->voxel <= 0 || p->half_base <= 0 || p->height <= 0 || p->n_detectors < 1 || p->n_detectors > 4 ||
        p->n_theta < 1 || p->n_phi < 1 || p->theta_max <= p->theta_min || p->theta_max >= M_PI / 2)
        return qb::fail(QB_EINVAL, "qb_synth_tomography: bad geometry");
    Grid g;
    g.v = p->voxel;
    const int nxy = int(std::ceil(2.0 * p->half_base / p->voxel - 1e-9));
    const int nz = int(std::ceil(p->height / p->voxel - 1e-9));
    g.n[0] = g.n[1] = nxy;
    g.n[2] = nz;
    g.lo[0] = g.lo[1] = -0.5 * nxy * p->voxel;
    g.lo[2] = 0.0;
    const int64_t ncell = g.cells();
    auto centre = [&](int64_t c, double q[3]) {
        const int i = int(c % nxy), j = int((c / nxy) % nxy), k = int(c / (int64_t(nxy) * nxy));
        q[0] = g.lo[0] + (i + 0.5) * g.v;
        q[1] = g.lo[1] + (j + 0.5) * g.v;
        q[2] = g.lo[2] + (k + 0.5) * g.v;
    };
    std::vector<uint8_t> rock(size_t(ncell), 0), is_void(size_t(ncell), 0);
    std::vector<int32_t> cell_bit(size_t(ncell), -1);
    std::vector<int64_t> bit_cell;
    const double hv = 0.5 * p->void_side;
    for (int64_t c = 0; c < ncell; ++c) {
        double q[3];
        centre(c, q);
        const double wz = p->half_base * (1.0 - q[2] / p->height);
        if (q[2] < p->height && std::fabs(q[0]) <= wz && std::fabs(q[1]) <= wz) {
            rock[size_t(c)] = 1;
            // detector rooms are surveyed, not inferred: cells within
            // room_radius of a detector carry no bit (check_ising.cu:179-199)
            bool room = false;
            for (int k = 0; k < p->n_detectors; ++k) {
                const double dx = q[0] - p->det[3 * k], dy = q[1] - p->det[3 * k + 1], dz = q[2] - p->det[3 * k + 2];
                room |= dx * dx + dy * dy + dz * dz < p->room_radius * p->room_radius;
            }
            if (room) continue;
            if (std::fabs(q[0] - p->void_center[0]) <= hv && std::fabs(q[1] - p->void_center[1]) <= hv &&
                std::fabs(q[2] - p->void_center[2]) <= hv)
                is_void[size_t(c)] = 1;
            if (p->target_bits <= 0 || int64_t(bit_cell.size()) < p->target_bits) {
                cell_bit[size_t(c)] = int32_t(bit_cell.size());
                bit_cell.push_back(c);
            }
        }
    }
    if (p->target_bits > 0 && int64_t(bit_cell.size()) < p->target_bits)
        return qb::fail(QB_EINVAL, "qb_synth_tomography: the pyramid holds fewer cells than target_bits");
    const int n = int(bit_cell.size());
    qb_tomo* t = new (std::nothrow) qb_tomo();
    if (!t) return qb::fail(QB_ENOMEM, "qb_synth_tomography: out of host memory");
    t->lambda = p->lambda;
    t->kappa = p->kappa;
    t->dims[0] = t->dims[1] = nxy;
    t->dims[2] = nz;
    t->bit_cell = bit_cell;
    // prior adjacency, BitField::grid's candidate order
    t->nbr_ptr.assign(size_t(n) + 1, 0);
    t->truth.assign(size_t(n), 0);
    for (int b = 0; b < n; ++b) {
        const int64_t c = bit_cell[size_t(b)];
        t->truth[size_t(b)] = is_void[size_t(c)];
        const int x = int(c % nxy), y = int((c / nxy) % nxy), z = int(c / (int64_t(nxy) * nxy));
        const int cand[6][3] = {{x - 1, y, z}, {x + 1, y, z}, {x, y - 1, z}, {x, y + 1, z}, {x, y, z - 1}, {x, y, z + 1}};
        for (const auto& q : cand) {
            if (q[0] < 0 || q[0] >= nxy || q[1] < 0 || q[1] >= nxy || q[2] < 0 || q[2] >= nz) continue;
            const int u = cell_bit[size_t((int64_t(q[2]) * nxy + q[1]) * nxy + q[0])];
            if (u >= 0) t->nbr.push_back(u);
        }
        t->nbr_ptr[size_t(b) + 1] = int32_t(t->nbr.size());
    }
    // rays: march every sky bin (host or device), then draw the counts bin
    // by bin from one stream
    SynthMarch M;
    M.g = g;
    M.rock = std::move(rock);
    M.is_void = std::move(is_void);
    M.cell_bit = std::move(cell_bit);
    M.n_det = p->n_detectors;
    std::memcpy(M.det, p->det, sizeof M.det);
    M.n_theta = p->n_theta;
    M.n_phi = p->n_phi;
    M.S = p->sub_rays > 0 ? p->sub_rays : 1;
    M.n_bits = n;
    M.inv_s2 = 1.0 / double(M.S * M.S);
    M.mu_rock = p->mu_rock;
    M.mu_air = p->mu_rock * (1.2 / 2700.0);
    const double dth = (p->theta_max - p->theta_min) / p->n_theta;
    const double dph = 2.0 * p->phi_half / p->n_phi;
    // sub-ray angles: th_s depends on (zenith bin, su), ph_s on (detector, azimuth bin, sv)
    M.cth.resize(size_t(p->n_theta) * M.S);
    M.sth.resize(M.cth.size());
    for (int it = 0; it < p->n_theta; ++it) {
        const double th = p->theta_min + (it + 0.5) * dth;
        for (int su = 0; su < M.S; ++su) {
            const double th_s = th + ((su + 0.5) / M.S - 0.5) * dth;
            M.cth[size_t(it) * M.S + su] = std::cos(th_s);
            M.sth[size_t(it) * M.S + su] = std::sin(th_s);
        }
    }
    M.cph.resize(size_t(p->n_detectors) * p->n_phi * M.S);
    M.sph.resize(M.cph.size());
    for (int k = 0; k < p->n_detectors; ++k) {
        const double* o = &p->det[3 * k];
        const double axis_phi = std::atan2(-o[1], -o[0]);
        for (int ip = 0; ip < p->n_phi; ++ip) {
            const double ph = axis_phi - p->phi_half + (ip + 0.5) * dph;
            for (int sv = 0; sv < M.S; ++sv) {
                const double ph_s = ph + ((sv + 0.5) / M.S - 0.5) * dph;
                M.cph[(size_t(k) * p->n_phi + ip) * M.S + sv] = std::cos(ph_s);
                M.sph[(size_t(k) * p->n_phi + ip) * M.S + sv] = std::sin(ph_s);
            }
        }
    }
    std::vector<BinMarch> bins;
    std::vector<int32_t> e_bit;
    std::vector<float> e_a;
#ifdef QB_SYNTH_HOST_ONLY   // the host-only build of the builder (no device march linked in)
    qb_status ms = on_device ? qb::fail(QB_ENOTSUP, "qb_synth_tomography_device: host-only build")
                             : march_host(M, bins, e_bit, e_a);
#else
    qb_status ms = on_device ? qb::synth_march_device(M, opts, bins, e_bit, e_a) : march_host(M, bins, e_bit, e_a);
#endif
    if (ms != QB_OK) {
        delete t;
        return ms;
    }
    struct RayRec { double d, w, open; int64_t first, count; };
    std::vector<RayRec> rays;
    uint64_t rs = p->seed;
    for (int k = 0; k < p->n_detectors; ++k)
        for (int it = 0; it < p->n_theta; ++it) {
            const double th = p->theta_min + (it + 0.5) * dth;
            const double ct = std::cos(th), st = std::sin(th);
            for (int ip = 0; ip < p->n_phi; ++ip) {
                const BinMarch& B = bins[(size_t(k) * p->n_theta + it) * p->n_phi + ip];
                const double lam_open = p->exposure * ct * ct * st * dth * dph;
                const int64_t n_open = poisson(lam_open, rs);
                const int64_t n_det = poisson(double(n_open) * std::exp(-B.tau), rs);
                if (B.cnt == 0 || double(n_open) < p->min_open) continue;
                const double det = std::max(double(n_det), 1.0);
                const double tt = -std::log(det / double(n_open));
                rays.push_back({B.tau0 - tt, det, double(n_open), B.first, B.cnt});
            }
        }
    // keep target_rays: the most-exposed rays, original order preserved
    std::vector<uint8_t> keep(rays.size(), 1);
    if (p->target_rays > 0) {
        if (int64_t(rays.size()) < p->target_rays) {
            delete t;
            return qb::fail(QB_EINVAL, "qb_synth_tomography: fewer populated rays than target_rays");
        }
        std::vector<int32_t> idx(rays.size());
        for (size_t i = 0; i < rays.size(); ++i) idx[i] = int32_t(i);
        std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return rays[size_t(a)].open > rays[size_t(b)].open; });
        for (size_t i = size_t(p->target_rays); i < idx.size(); ++i) keep[size_t(idx[i])] = 0;
    }
    std::vector<int32_t> cnt_bit(size_t(n) + 1, 0);
    int32_t nr = 0;
    std::vector<int32_t> ray_id(rays.size(), -1);
    for (size_t r = 0; r < rays.size(); ++r) {
        if (!keep[r]) continue;
        ray_id[r] = nr++;
        t->d.push_back(rays[r].d);
        t->w.push_back(rays[r].w);
        for (int64_t e = rays[r].first; e < rays[r].first + rays[r].count; ++e) cnt_bit[size_t(e_bit[size_t(e)]) + 1]++;
    }
    t->row_ptr.assign(size_t(n) + 1, 0);
    for (int b = 0; b < n; ++b) t->row_ptr[size_t(b) + 1] = t->row_ptr[size_t(b)] + cnt_bit[size_t(b) + 1];
    const int64_t nnz = t->row_ptr[size_t(n)];
    t->ray.assign(size_t(nnz), 0);
    t->a.assign(size_t(nnz), 0.0f);
    std::vector<int32_t> fill(t->row_ptr.begin(), t->row_ptr.end() - 1);
    for (size_t r = 0; r < rays.size(); ++r) {
        if (ray_id[r] < 0) continue;
        for (int64_t e = rays[r].first; e < rays[r].first + rays[r].count; ++e) {
            const int b = e_bit[size_t(e)];
            const int32_t k = fill[size_t(b)]++;
            t->ray[size_t(k)] = ray_id[r];
            t->a[size_t(k)] = e_a[size_t(e)];
        }
    }
    *out = t;
    return QB_OK;
}

}  // namespace

extern "C" qb_status qb_synth_tomography(const qb_tomo_params* p, qb_tomo** out) {
    return qb::guarded("qb_synth_tomography", [&]() -> qb_status {
        return synth_tomography(p, false, nullptr, out);
    });
}

extern "C" qb_status qb_synth_tomography_device(const qb_tomo_params* p, const qb_opts* opts, qb_tomo** out) {
    return qb::guarded("qb_synth_tomography_device", [&]() -> qb_status {
        return synth_tomography(p, true, opts, out);
    });
}

extern "C" qb_status qb_tomo_sizes(const qb_tomo* t, int32_t* n_vars, int32_t* n_rays, int64_t* nnz, int64_t* n_nbr) {
    if (!t) return qb::fail(QB_EINVAL, "qb_tomo_sizes: null tomography");
    if (n_vars) *n_vars = int32_t(t->row_ptr.size()) - 1;
    if (n_rays) *n_rays = int32_t(t->d.size());
    if (nnz) *nnz = int64_t(t->ray.size());
    if (n_nbr) *n_nbr = int64_t(t->nbr.size());
    return QB_OK;
}

extern "C" qb_status qb_tomo_arrays(const qb_tomo* t, double* d, double* w, int32_t* row_ptr, int32_t* ray, float* a,
                                    int32_t* nbr_ptr, int32_t* nbr, uint8_t* truth) {
    if (!t) return qb::fail(QB_EINVAL, "qb_tomo_arrays: null tomography");
    auto cp = [](void* dst, const void* src, size_t bytes) { if (dst && bytes) std::memcpy(dst, src, bytes); };
    cp(d, t->d.data(), t->d.size() * sizeof(double));
    cp(w, t->w.data(), t->w.size() * sizeof(double));
    cp(row_ptr, t->row_ptr.data(), t->row_ptr.size() * sizeof(int32_t));
    cp(ray, t->ray.data(), t->ray.size() * sizeof(int32_t));
    cp(a, t->a.data(), t->a.size() * sizeof(float));
    cp(nbr_ptr, t->nbr_ptr.data(), t->nbr_ptr.size() * sizeof(int32_t));
    cp(nbr, t->nbr.data(), t->nbr.size() * sizeof(int32_t));
    cp(truth, t->truth.data(), t->truth.size());
    return QB_OK;
}

extern "C" qb_status qb_tomo_cells(const qb_tomo* t, int32_t* dims, int64_t* bit_cell) {
    if (!t) return qb::fail(QB_EINVAL, "qb_tomo_cells: null tomography");
    if (dims) std::memcpy(dims, t->dims, sizeof t->dims);
    if (bit_cell && !t->bit_cell.empty()) std::memcpy(bit_cell, t->bit_cell.data(), t->bit_cell.size() * sizeof(int64_t));
    return QB_OK;
}

extern "C" qb_status qb_tomo_desc(const qb_tomo* t, qb_residual_desc* desc) {
    if (!t || !desc) return qb::fail(QB_EINVAL, "qb_tomo_desc: null argument");
    desc->n_vars = int32_t(t->row_ptr.size()) - 1;
    desc->n_rays = int32_t(t->d.size());
    desc->d = t->d.data();
    desc->w = t->w.data();
    desc->row_ptr = t->row_ptr.data();
    desc->ray = t->ray.data();
    desc->a = t->a.data();
    desc->nbr_ptr = t->nbr_ptr.data();
    desc->nbr = t->nbr.data();
    desc->lambda = t->lambda;
    desc->kappa = t->kappa;
    desc->field = nullptr;
    return QB_OK;
}

extern "C" void qb_tomo_destroy(qb_tomo* t) { delete t; }
