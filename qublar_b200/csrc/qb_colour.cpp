// Greedy colourings that turn a sequential Metropolis sweep into a sequence
// of conflict-free parallel steps.
//
// The reference sweeps bits in index order (ising_weighted.hpp:258,
// ising_recon.hpp:132) and parallelises only across replicas, or speculates
// on a 32-spin window (ising_gpu.cuh:207-246). Here every bit of a class can
// be updated at once because no two of them share a coupling (Ising) or a ray
// or a prior bond (residual form): the dE each one sees is exact.
#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <cstring>

#include <omp.h>

#include "qb_internal.hpp"

namespace qb {

namespace {
constexpr int kColourWords = 8;   // 64-colour words per ray row at the start: one cache line
}  // namespace

void finish_colouring(Colouring& c, int n) {
    int nc = 0;
    for (int i = 0; i < n; ++i) nc = std::max(nc, c.colour[size_t(i)] + 1);
    c.class_ptr.assign(size_t(nc) + 1, 0);
    for (int i = 0; i < n; ++i) c.class_ptr[size_t(c.colour[size_t(i)]) + 1]++;
    for (int k = 0; k < nc; ++k) c.class_ptr[size_t(k) + 1] += c.class_ptr[size_t(k)];
    std::vector<int32_t> fill(c.class_ptr.begin(), c.class_ptr.end() - 1);
    c.order.assign(size_t(n), 0);
    c.inverse.assign(size_t(n), 0);
    for (int i = 0; i < n; ++i) {   // stable: original order inside a class
        const int k = fill[size_t(c.colour[size_t(i)])]++;
        c.order[size_t(k)] = i;
        c.inverse[size_t(i)] = k;
    }
}

Colouring colour_graph(int n, const std::vector<int64_t>& row, const std::vector<int32_t>& col) {
    Colouring c;
    c.colour.assign(size_t(n), -1);
    // Largest degree first (Welsh-Powell order), ties by index: fewer classes
    // than index order on irregular graphs, identical on regular ones; then
    // the classes are balanced (below). A stable counting sort by decreasing
    // degree.
    auto deg = [&](int i) { return int(row[size_t(i) + 1] - row[size_t(i)]); };
    int maxdeg = 0;
    for (int i = 0; i < n; ++i) maxdeg = std::max(maxdeg, deg(i));
    std::vector<int32_t> vis(static_cast<size_t>(n));
    {
        std::vector<int32_t> start(size_t(maxdeg) + 2, 0);
        for (int i = 0; i < n; ++i) start[size_t(maxdeg - deg(i)) + 1]++;
        for (int d = 0; d <= maxdeg; ++d) start[size_t(d) + 1] += start[size_t(d)];
        for (int i = 0; i < n; ++i) vis[size_t(start[size_t(maxdeg - deg(i))]++)] = i;
    }
    // Each bit takes the smallest colour none of its neighbours holds, so no
    // colour exceeds the largest degree. mark[colour + 1] == i: a neighbour of
    // i holds that colour; slot 0 collects the uncoloured neighbours.
    std::vector<int32_t> mark(size_t(maxdeg) + 2, -1);
    for (size_t v = 0; v < vis.size(); ++v) {
        const int i = vis[v];
        // prefetches in stages, as in the residual first fit: the offsets of
        // the bit 12 visits ahead, its neighbour list 6 ahead, the neighbours'
        // colours 2 ahead
        if (v + 12 < vis.size()) __builtin_prefetch(row.data() + vis[v + 12]);
        if (v + 6 < vis.size()) {
            const int i6 = vis[v + 6];
            for (int64_t k = row[size_t(i6)]; k < row[size_t(i6) + 1]; k += 16) __builtin_prefetch(col.data() + k);
        }
        if (v + 2 < vis.size()) {
            const int i2 = vis[v + 2];
            for (int64_t k = row[size_t(i2)]; k < row[size_t(i2) + 1]; ++k)
                __builtin_prefetch(c.colour.data() + col[size_t(k)]);
        }
        for (int64_t k = row[size_t(i)]; k < row[size_t(i) + 1]; ++k)
            mark[size_t(c.colour[size_t(col[size_t(k)])] + 1)] = i;
        int cc = 0;
        while (mark[size_t(cc) + 1] == i) ++cc;
        c.colour[size_t(i)] = cc;
    }
    // Balance the classes: a sweep of a class costs ceil(size / workers)
    // passes, so lopsided greedy classes (27k bits down to 14 on the weighted
    // lattice) waste passes. Bits of classes above ceil(n / K), in index order,
    // move to the smallest class below that size that holds none of their
    // neighbours (the class count does not change).
    // (QB_GRAPH_BALANCE=0 keeps the greedy classes)
    const char* bal = std::getenv("QB_GRAPH_BALANCE");
    int K = 0;
    for (int i = 0; i < n; ++i) K = std::max(K, c.colour[size_t(i)] + 1);
    if (K > 1 && !(bal && std::strcmp(bal, "0") == 0)) {
        const int target = (n + K - 1) / K;
        std::vector<int32_t> size(static_cast<size_t>(K), 0), seen(static_cast<size_t>(K), -1);
        for (int i = 0; i < n; ++i) size[size_t(c.colour[size_t(i)])]++;
        for (int i = 0; i < n; ++i) {
            const int ci = c.colour[size_t(i)];
            if (size[size_t(ci)] <= target) continue;
            for (int64_t k = row[size_t(i)]; k < row[size_t(i) + 1]; ++k) seen[size_t(c.colour[size_t(col[size_t(k)])])] = i;
            int best = -1;
            for (int q = 0; q < K; ++q)
                if (q != ci && size[size_t(q)] < target && seen[size_t(q)] != i &&
                    (best < 0 || size[size_t(q)] < size[size_t(best)]))
                    best = q;
            if (best >= 0) {
                c.colour[size_t(i)] = best;
                size[size_t(ci)]--;
                size[size_t(best)]++;
            }
        }
    }
    finish_colouring(c, n);
    return c;
}

Colouring colour_residual(int n, int n_rays, int* max_ray_len, const int32_t* row_ptr, const int32_t* ray,
                          const int32_t* nbr_ptr, const int32_t* nbr) {
    Colouring c;
    c.colour.assign(size_t(n), -1);
    // Per-ray bitset of the colours already on the ray: `words` 64-colour
    // words per ray, one 64-byte cache line at the start (512 colours), grown
    // when a bit runs out of free colours. The rows start on a cache line.
    int words = kColourWords;
    std::vector<uint64_t> store;
    uint64_t* used = nullptr;
    auto alloc_rows = [&](int w) {
        std::vector<uint64_t> g(size_t(std::max(n_rays, 1)) * size_t(w) + 8, 0);
        uint64_t* base = g.data();
        while (reinterpret_cast<uintptr_t>(base) % 64) ++base;
        if (used)
            for (int b = 0; b < n_rays; ++b)
                std::memcpy(base + size_t(b) * size_t(w), used + size_t(b) * size_t(words), sizeof(uint64_t) * size_t(words));
        store.swap(g);
        used = base;
        words = w;
    };
    alloc_rows(kColourWords);
    // Visit bits by their conflict degree counted with multiplicity (the sum
    // of the lengths of their rays), largest first (Welsh-Powell order), ties
    // by index: long conflict lists get the low colours, which keeps the class
    // count near the longest ray (340 classes on the 306,328-bit pyramid whose
    // longest ray crosses 288 bits; ordering by ray count gives 349).
    std::vector<int32_t> raylen(static_cast<size_t>(std::max(n_rays, 1)), 0);
    const int nnz = row_ptr[n];
    const int T = omp_get_max_threads();
    if (T > 1 && nnz >= (1 << 20) && int64_t(T) * n_rays <= (int64_t(1) << 24)) {
        // per-thread counts over slices of the entries, then summed per ray
        std::vector<int32_t> part(size_t(T) * size_t(n_rays), 0);
#pragma omp parallel num_threads(T)
        {
            int32_t* cnt = part.data() + size_t(omp_get_thread_num()) * size_t(n_rays);
#pragma omp for schedule(static)
            for (int k = 0; k < nnz; ++k) cnt[ray[k]]++;
#pragma omp for schedule(static)
            for (int r = 0; r < n_rays; ++r) {
                int32_t s = 0;
                for (int t = 0; t < T; ++t) s += part[size_t(t) * size_t(n_rays) + size_t(r)];
                raylen[size_t(r)] = s;
            }
        }
    } else {
        for (int k = 0; k < nnz; ++k) raylen[size_t(ray[k])]++;
    }
    if (max_ray_len) *max_ray_len = n_rays > 0 ? *std::max_element(raylen.begin(), raylen.begin() + n_rays) : 0;
    std::vector<int64_t> conf(static_cast<size_t>(n), 0);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
        int64_t s = 0;
        for (int k = row_ptr[i]; k < row_ptr[i + 1]; ++k) s += raylen[size_t(ray[k])];
        conf[size_t(i)] = s;
    }
    // stable counting sort by decreasing conflict degree
    int64_t cmax = 0;
    for (int i = 0; i < n; ++i) cmax = std::max(cmax, conf[size_t(i)]);
    std::vector<int32_t> vis(static_cast<size_t>(n));
    if (cmax <= int64_t(16) * n + (1 << 20)) {
        std::vector<int32_t> start(size_t(cmax) + 2, 0);
        for (int i = 0; i < n; ++i) start[size_t(cmax - conf[size_t(i)]) + 1]++;
        for (int64_t v = 0; v <= cmax; ++v) start[size_t(v) + 1] += start[size_t(v)];
        for (int i = 0; i < n; ++i) vis[size_t(start[size_t(cmax - conf[size_t(i)])]++)] = i;
    } else {
        for (int i = 0; i < n; ++i) vis[size_t(i)] = i;
        std::stable_sort(vis.begin(), vis.end(), [&](int a, int b) { return conf[size_t(a)] > conf[size_t(b)]; });
    }
    // First fit: the lowest colour on none of the bit's rays and on none of its
    // prior neighbours.
    // the ray and neighbour lists gathered into visit order (in parallel), so
    // that the first-fit loop streams them instead of fetching every bit's
    // lists from a random place of the caller's arrays
    std::vector<int64_t> vrow(size_t(n) + 1, 0), vnb(size_t(n) + 1, 0);
    for (int v = 0; v < n; ++v) {
        const int i = vis[size_t(v)];
        vrow[size_t(v) + 1] = vrow[size_t(v)] + (row_ptr[i + 1] - row_ptr[i]);
        vnb[size_t(v) + 1] = vnb[size_t(v)] + (nbr_ptr[i + 1] - nbr_ptr[i]);
    }
    RawVec<int32_t> vray(size_t(vrow[size_t(n)]) + 1), vnbr(size_t(vnb[size_t(n)]) + 1);
#pragma omp parallel for schedule(static, 1024)
    for (int v = 0; v < n; ++v) {
        const int i = vis[size_t(v)];
        std::memcpy(vray.data() + vrow[size_t(v)], ray + row_ptr[i], sizeof(int32_t) * size_t(row_ptr[i + 1] - row_ptr[i]));
        std::memcpy(vnbr.data() + vnb[size_t(v)], nbr + nbr_ptr[i], sizeof(int32_t) * size_t(nbr_ptr[i + 1] - nbr_ptr[i]));
    }
    std::vector<uint64_t> forbid;
    for (size_t v = 0; v < vis.size(); ++v) {
        const int i = vis[v];
        const int32_t* rl = vray.data() + vrow[v];
        const int nrl = int(vrow[v + 1] - vrow[v]);
        const int32_t* nl = vnbr.data() + vnb[v];
        const int nnl = int(vnb[v + 1] - vnb[v]);
        // the rows (random rays) and neighbour colours of the bit 3 visits ahead
        if (v + 3 < vis.size()) {
            for (int64_t k = vrow[v + 3]; k < vrow[v + 4]; ++k) __builtin_prefetch(used + size_t(vray[size_t(k)]) * size_t(words), 1);
            for (int64_t k = vnb[v + 3]; k < vnb[v + 4]; ++k) __builtin_prefetch(c.colour.data() + vnbr[size_t(k)]);
        }
        int cc = -1;
        if (words == kColourWords) {
            uint64_t f[kColourWords] = {};
            for (int k = 0; k < nrl; ++k) {
                const uint64_t* u = used + size_t(rl[k]) * kColourWords;
                for (int q = 0; q < kColourWords; ++q) f[q] |= u[q];
            }
            for (int k = 0; k < nnl; ++k) {
                const int cj = c.colour[size_t(nl[k])];
                if (cj >= 0) f[cj >> 6] |= uint64_t(1) << (cj & 63);
            }
            for (int q = 0; q < kColourWords && cc < 0; ++q)
                if (~f[q]) cc = 64 * q + __builtin_ctzll(~f[q]);
            if (cc < 0) alloc_rows(2 * kColourWords);   // all 512 taken: continue with wider rows
        }
        while (cc < 0) {
            forbid.assign(size_t(words), 0);
            for (int k = 0; k < nrl; ++k) {
                const uint64_t* u = used + size_t(rl[k]) * size_t(words);
                for (int q = 0; q < words; ++q) forbid[size_t(q)] |= u[q];
            }
            for (int k = 0; k < nnl; ++k) {
                const int cj = c.colour[size_t(nl[k])];
                if (cj >= 0) forbid[size_t(cj >> 6)] |= uint64_t(1) << (cj & 63);
            }
            for (int q = 0; q < words && cc < 0; ++q)
                if (~forbid[size_t(q)]) cc = 64 * q + __builtin_ctzll(~forbid[size_t(q)]);
            if (cc < 0) alloc_rows(words * 2);
        }
        c.colour[size_t(i)] = cc;
        for (int k = 0; k < nrl; ++k) used[size_t(rl[k]) * size_t(words) + size_t(cc >> 6)] |= uint64_t(1) << (cc & 63);
    }
    finish_colouring(c, n);
    return c;
}

bool colouring_valid_graph(const Colouring& c, const std::vector<int64_t>& row, const std::vector<int32_t>& col) {
    const int n = int(c.colour.size());
    for (int i = 0; i < n; ++i)
        for (int64_t k = row[size_t(i)]; k < row[size_t(i) + 1]; ++k)
            if (c.colour[size_t(col[size_t(k)])] == c.colour[size_t(i)]) return false;
    return true;
}

}  // namespace qb
