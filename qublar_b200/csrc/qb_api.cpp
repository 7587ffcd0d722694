// The C ABI (include/qublar.h): validation, planning, upload, solve, results.
#include <algorithm>
#include <cstdio>
#include <chrono>
#include <climits>
#include <functional>
#ifdef _OPENMP
#include <omp.h>
#endif
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "qb_build.hpp"
#include "qb_batch.hpp"
#include "qb_internal.hpp"
#include "qb_kernels.hpp"
#include "qb_qubo.hpp"

using namespace qb;

namespace {

cudaStream_t stream_of(const qb_opts* o) { return o ? static_cast<cudaStream_t>(o->stream) : nullptr; }

qb_status select_device(const qb_opts* o, int* dev_out) {
    int dev = 0;
    if (o && o->device >= 0) {
        QB_CUDA(cudaSetDevice(o->device));
        dev = o->device;
    } else {
        QB_CUDA(cudaGetDevice(&dev));
    }
    *dev_out = dev;
    return QB_OK;
}

// Stream-ordered allocation for per-solve buffers: no device-wide
// synchronisation inside a timed loop.
qb_status alloc_async(DevBuf& b, size_t bytes, cudaStream_t st) {
    b.release();
    if (bytes == 0) return QB_OK;
    int dev = 0;
    QB_CUDA(cudaGetDevice(&dev));
    cudaMemPool_t pool = library_pool(dev);
    if (pool) QB_CUDA(cudaMallocFromPoolAsync(&b.p, bytes, pool, st));
    else QB_CUDA(cudaMallocAsync(&b.p, bytes, st));
    b.bytes = bytes;
    b.pooled = true;
    b.pool_stream = st;
    return QB_OK;
}

// Stream-ordered release of a stream-ordered allocation; a buffer taken from
// a plain allocation (the packed-replica arenas) is freed plainly.
void free_async(DevBuf& b, cudaStream_t st) {
    if (b.p) {
        if (b.pooled) cudaFreeAsync(b.p, st);
        else cudaFree(b.p);
    }
    b.p = nullptr;
    b.bytes = 0;
    b.pooled = false;
}

}  // namespace

// The temperature of every sweep by the reference's expression
// (ising_recon.hpp:129-131, ising_weighted.hpp:255-257); `volatile` keeps the
// double rounding of gising::temperatures (ising_gpu.cuh:114-124).
std::vector<double> qb::temperatures(const qb_schedule& s) {
    const int total = s.anneal_sweeps + s.hold_sweeps;
    std::vector<double> t(size_t(total), 0.0);
    for (int sweep = 0; sweep < total; ++sweep) {
        const double frac = std::min(1.0, double(sweep) / std::max(1, s.anneal_sweeps - 1));
        volatile double temp = sweep < s.anneal_sweeps ? s.t_hot * std::pow(s.t_cold / s.t_hot, frac) : s.t_cold;
        t[size_t(sweep)] = temp;
    }
    return t;
}

namespace {

// Slices per class the host-only planner assumes for the lockstep sweep (the
// SM count of a B200); the order inside a class does not change results.
constexpr int kHostLockSlices = 148;

int env_int(const char* name, int dflt) {
    const char* v = std::getenv(name);
    return v && *v ? std::atoi(v) : dflt;
}

// Stage times of a planner, printed to stderr at the end when QB_PLAN_TIMES is set.
class PlanMarks {
public:
    PlanMarks() : on_(std::getenv("QB_PLAN_TIMES") != nullptr) { (*this)("start"); }
    void operator()(const char* what) {
        if (on_) marks_.emplace_back(what, std::chrono::steady_clock::now());
    }
    void print() const {
        for (size_t k = 1; k < marks_.size(); ++k)
            std::fprintf(stderr, "[qb plan]   %s %.1f ms\n", marks_[k].first,
                         std::chrono::duration<double, std::milli>(marks_[k].second - marks_[k - 1].second).count());
    }

private:
    bool on_;
    std::vector<std::pair<const char*, std::chrono::steady_clock::time_point>> marks_;
};

// Symmetric CSR of an edge list in edge order: edge (a, b) appends b to row a
// and a to row b, as parse_rudy builds its adjacency (ising_weighted.hpp:135-147).
// With threads, each takes a contiguous slice of the edges: it counts its
// slice's endpoints per vertex, the counts are turned into write positions
// (a row holds slice 0's entries, then slice 1's, ...), and it writes its
// slice in edge order, so every row is in edge order. When threads x vertices
// counters would not fit in 2^26 words, each thread instead owns a range of
// rows and scans the whole edge list. Indices must be in range; 2m < 2^31.
template <class W>
void sym_csr(int n, int64_t m, const int32_t* eu, const int32_t* ev, const W* ew, std::vector<int64_t>& row,
             std::vector<int32_t>& col, std::vector<W>& w) {
    const int T = m >= (int64_t(1) << 16) ? std::max(1, omp_get_max_threads()) : 1;
    row.assign(size_t(n) + 1, 0);
    col.resize(size_t(2 * m));
    w.resize(size_t(2 * m));
    if (T > 1 && int64_t(T) * n <= (int64_t(1) << 26)) {
        RawVec<int32_t> at(size_t(T) * size_t(n));   // [slice][vertex]: counts, then write positions
#pragma omp parallel num_threads(T)
        {
            const int t = omp_get_thread_num(), nt = omp_get_num_threads();
            int32_t* cnt = at.data() + size_t(t) * size_t(n);
            std::fill(cnt, cnt + n, 0);
            const int64_t e0 = m * t / nt, e1 = m * (t + 1) / nt;
            for (int64_t e = e0; e < e1; ++e) {
                cnt[eu[e]]++;
                cnt[ev[e]]++;
            }
#pragma omp barrier
            // degrees, then write positions, in blocks of vertices so each
            // slice's counters are read in order
            constexpr int kBlock = 2048;
#pragma omp for schedule(static)
            for (int vb = 0; vb < n; vb += kBlock) {
                const int ve = std::min(n, vb + kBlock);
                for (int q = 0; q < nt; ++q) {
                    const int32_t* cq = at.data() + size_t(q) * size_t(n);
                    for (int v = vb; v < ve; ++v) row[size_t(v) + 1] += cq[v];
                }
            }
#pragma omp single
            for (int v = 0; v < n; ++v) row[size_t(v) + 1] += row[size_t(v)];
#pragma omp for schedule(static)
            for (int vb = 0; vb < n; vb += kBlock) {
                const int ve = std::min(n, vb + kBlock);
                int32_t pos[kBlock];
                for (int v = vb; v < ve; ++v) pos[v - vb] = int32_t(row[size_t(v)]);
                for (int q = 0; q < nt; ++q) {
                    int32_t* cq = at.data() + size_t(q) * size_t(n);
                    for (int v = vb; v < ve; ++v) {
                        const int32_t k = cq[v];
                        cq[v] = pos[v - vb];
                        pos[v - vb] += k;
                    }
                }
            }
            for (int64_t e = e0; e < e1; ++e) {
                const int32_t a = eu[e], b = ev[e];
                int32_t k = cnt[a]++;
                col[size_t(k)] = b;
                w[size_t(k)] = ew[e];
                k = cnt[b]++;
                col[size_t(k)] = a;
                w[size_t(k)] = ew[e];
            }
        }
        return;
    }
#pragma omp parallel num_threads(T)
    {
        const int t = omp_get_thread_num(), nt = omp_get_num_threads();
        const uint32_t lo = uint32_t(int64_t(n) * t / nt), span = uint32_t(int64_t(n) * (t + 1) / nt) - lo;
        int64_t* r = row.data() + 1;
        for (int64_t e = 0; e < m; ++e) {
            const uint32_t a = uint32_t(eu[e]), b = uint32_t(ev[e]);
            if (a - lo < span) r[a]++;
            if (b - lo < span) r[b]++;
        }
    }
    for (int i = 0; i < n; ++i) row[size_t(i) + 1] += row[size_t(i)];
    std::vector<int64_t> fill(row.begin(), row.end() - 1);
#pragma omp parallel num_threads(T)
    {
        // rows split by entry count
        const int t = omp_get_thread_num(), nt = omp_get_num_threads();
        auto first_row = [&](int q) {
            return uint32_t(std::lower_bound(row.begin(), row.end() - 1, 2 * m * q / nt) - row.begin());
        };
        const uint32_t lo = t == 0 ? 0u : first_row(t), hi = t + 1 == nt ? uint32_t(n) : first_row(t + 1);
        const uint32_t span = hi - lo;
        for (int64_t e = 0; e < m; ++e) {
            const uint32_t a = uint32_t(eu[e]), b = uint32_t(ev[e]);
            if (a - lo < span) {
                const int64_t k = fill[a]++;
                col[size_t(k)] = int32_t(b);
                w[size_t(k)] = ew[e];
            }
            if (b - lo < span) {
                const int64_t k = fill[b]++;
                col[size_t(k)] = int32_t(a);
                w[size_t(k)] = ew[e];
            }
        }
    }
}

// The first edge for which bad(e) holds, or m (a parallel scan for the lowest
// index, so the reason reported is the one a sequential scan finds).
template <class F>
int64_t first_bad_edge(int64_t m, F bad) {
    int64_t first = m;
#pragma omp parallel for schedule(static) reduction(min : first) if (m >= (int64_t(1) << 16))
    for (int64_t e = 0; e < m; ++e)
        if (bad(e)) first = std::min(first, e);
    return first;
}

// True when some row of a symmetric CSR lists a neighbour twice: an edge given
// twice, in either orientation.
bool has_duplicate_edge(int n, const std::vector<int64_t>& row, const std::vector<int32_t>& col) {
    bool dup = false;
#pragma omp parallel reduction(|| : dup) if (row[size_t(n)] >= (int64_t(1) << 16))
    {
        std::vector<int32_t> buf;
#pragma omp for schedule(dynamic, 2048)
        for (int i = 0; i < n; ++i) {
            buf.assign(col.begin() + row[size_t(i)], col.begin() + row[size_t(i) + 1]);
            std::sort(buf.begin(), buf.end());
            if (std::adjacent_find(buf.begin(), buf.end()) != buf.end()) dup = true;
        }
    }
    return dup;
}

// Row offsets of the sweep-order CSR: row k holds the neighbours of bit order[k].
void sweep_rows(const Colouring& C, const std::vector<int64_t>& row, std::vector<int32_t>& out) {
    const size_t n = C.order.size();
    out.assign(n + 1, 0);
    for (size_t k = 0; k < n; ++k) {
        const size_t i = size_t(C.order[k]);
        out[k + 1] = out[k] + int32_t(row[i + 1] - row[i]);
    }
}

// ---- ising planning -------------------------------------------------------------------

qb_status plan_ising(const qb_ising_desc* g, IsingPlan& P) {
    const int n = g->n;
    const int64_t m = g->m;
    if (n <= 0) return fail(QB_EINVAL, "ising: n must be positive");
    if (m < 0) return fail(QB_EINVAL, "ising: m must be non-negative");
    if (m > 0 && (!g->eu || !g->ev || !g->ew)) return fail(QB_EINVAL, "ising: null edge arrays");
    if (2 * m >= (int64_t(1) << 31)) return fail(QB_EREFUSED, "ising: more than 2^30 edges");
    // loader refusals of parse_rudy (ising_weighted.hpp:113-133)
    PlanMarks mark;
    auto out_of_range = [&](int64_t e) {
        const int32_t u = g->eu[e], v = g->ev[e];
        return u < 0 || u >= n || v < 0 || v >= n;
    };
    const int64_t bad = first_bad_edge(m, [&](int64_t e) { return out_of_range(e) || g->eu[e] == g->ev[e]; });
    if (bad < m) return fail(QB_EINVAL, out_of_range(bad) ? "ising: vertex index out of range" : "ising: self-loop");
    // symmetric CSR in edge order, as parse_rudy builds it (ising_weighted.hpp:135-147)
    std::vector<int64_t> row;
    std::vector<int32_t> col, w;
    sym_csr(n, m, g->eu, g->ev, g->ew, row, col, w);
    mark("csr");
    if (has_duplicate_edge(n, row, col)) return fail(QB_EINVAL, "ising: duplicate edge");
    mark("duplicates");
    P.n = n;
    P.m = m;
    P.nnz = 2 * m;
    // plan figures of gising::make_plan (ising_gpu.cuh:74-101)
    double sum_w2 = 0.0;
    P.w_min = 0;
    P.max_w = 0;
    for (int64_t e = 0; e < m; ++e) {
        const int64_t a = std::llabs(int64_t(g->ew[e]));
        sum_w2 += double(a) * double(a);
        P.max_w = std::max(P.max_w, a);
        if (a != 0 && (P.w_min == 0 || a < P.w_min)) P.w_min = a;
    }
    P.B = 0;
    for (int i = 0; i < n; ++i) {
        int64_t acc = 0;
        for (int64_t k = row[size_t(i)]; k < row[size_t(i) + 1]; ++k) acc += std::llabs(int64_t(w[size_t(k)]));
        P.B = std::max(P.B, acc);
    }
    if (P.B > 2147483647LL) return fail(QB_EREFUSED, "ising: field bound exceeds int32");
    P.sigma = std::sqrt(2.0 * sum_w2 / double(n));
    P.weight_bytes = P.max_w <= 127 ? 1 : 4;
    mark("figures");
    P.col = colour_graph(n, row, col);
    mark("colour");
    // sweep-order CSR
    const Colouring& C = P.col;
    sweep_rows(C, row, P.row);
    P.adj.resize(size_t(2 * m));
    P.wgt.resize(size_t(2 * m));
    P.f0.assign(size_t(n), 0);
#pragma omp parallel for schedule(dynamic, 4096) if (m >= (int64_t(1) << 16))
    for (int i = 0; i < n; ++i) {   // in the caller's bit order: the adjacency streams
        const int k = C.inverse[size_t(i)];
        int32_t pos = P.row[size_t(k)];
        int64_t acc = 0;
        for (int64_t e = row[size_t(i)]; e < row[size_t(i) + 1]; ++e) {
            P.adj[size_t(pos)] = C.inverse[size_t(col[size_t(e)])];
            P.wgt[size_t(pos)] = w[size_t(e)];
            acc -= w[size_t(e)];
            ++pos;
        }
        P.f0[size_t(k)] = int32_t(acc);   // x = 0: s = -1 everywhere (wising::State, ising_weighted.hpp:199-208)
    }
    mark("arrays");
    mark.print();
    return QB_OK;
}

// Device bytes upload_ising will take.
int64_t ising_device_bytes(const IsingPlan& P) {
    return int64_t(P.row.size() + P.adj.size() + P.f0.size() + P.col.order.size() + P.col.class_ptr.size()) * 4 +
           int64_t(P.wgt.size()) * P.weight_bytes + P.m * 12;
}

qb_status upload_ising(IsingPlan& P, const qb_ising_desc* g, cudaStream_t st, int64_t* bytes) {
    qb_status s;
    if ((s = upload_vec(P.d_row, P.row, st))) return s;
    if ((s = upload_vec(P.d_adj, P.adj, st))) return s;
    if (P.weight_bytes == 1) {
        std::vector<int8_t> w8(P.wgt.size());
        for (size_t k = 0; k < w8.size(); ++k) w8[k] = int8_t(P.wgt[k]);
        if ((s = upload_vec(P.d_w, w8, st))) return s;
        QB_CUDA(cudaStreamSynchronize(st));   // w8 is a local
    } else if ((s = upload_vec(P.d_w, P.wgt, st))) {
        return s;
    }
    if ((s = upload_vec(P.d_f0, P.f0, st))) return s;
    if ((s = upload_vec(P.d_order, P.col.order, st))) return s;
    if ((s = upload_vec(P.d_class_ptr, P.col.class_ptr, st))) return s;
    if ((s = upload(P.d_eu, g->eu, size_t(P.m) * 4, st))) return s;
    if ((s = upload(P.d_ev, g->ev, size_t(P.m) * 4, st))) return s;
    if ((s = upload(P.d_ew, g->ew, size_t(P.m) * 4, st))) return s;
    QB_CUDA(cudaStreamSynchronize(st));
    *bytes = int64_t(P.d_row.bytes + P.d_adj.bytes + P.d_w.bytes + P.d_f0.bytes + P.d_order.bytes +
                     P.d_class_ptr.bytes + P.d_eu.bytes + P.d_ev.bytes + P.d_ew.bytes);
    return QB_OK;
}

// ---- weighted qubo planning ---------------------------------------------------------------

qb_status plan_qubo(const qb_qubo_desc* g, QuboPlan& P) {
    const int n = g->n;
    const int64_t m = g->m;
    if (n <= 0) return fail(QB_EINVAL, "qubo: n must be positive");
    if (m < 0) return fail(QB_EINVAL, "qubo: m must be non-negative");
    if (m > 0 && (!g->eu || !g->ev || !g->ew)) return fail(QB_EINVAL, "qubo: null edge arrays");
    if (2 * m >= (int64_t(1) << 31)) return fail(QB_EREFUSED, "qubo: more than 2^30 edges");
    if (!std::isfinite(g->offset)) return fail(QB_EINVAL, "qubo: offset must be finite");
    PlanMarks mark;
    auto out_of_range = [&](int64_t e) {
        const int32_t u = g->eu[e], v = g->ev[e];
        return u < 0 || u >= n || v < 0 || v >= n;
    };
    const int64_t bad = first_bad_edge(
        m, [&](int64_t e) { return out_of_range(e) || g->eu[e] == g->ev[e] || !std::isfinite(g->ew[e]); });
    if (bad < m) {
        if (out_of_range(bad)) return fail(QB_EINVAL, "qubo: vertex index out of range");
        if (g->eu[bad] == g->ev[bad]) return fail(QB_EINVAL, "qubo: self-loop (put diagonal terms in h)");
        return fail(QB_EINVAL, "qubo: coupling is not finite");
    }
    // symmetric CSR, edge order per vertex
    std::vector<int64_t> row;
    std::vector<int32_t> col;
    std::vector<float> w;
    sym_csr(n, m, g->eu, g->ev, g->ew, row, col, w);
    mark("csr");
    if (has_duplicate_edge(n, row, col)) return fail(QB_EINVAL, "qubo: duplicate edge");
    if (g->h)
        for (int i = 0; i < n; ++i)
            if (!std::isfinite(g->h[i])) return fail(QB_EINVAL, "qubo: linear term is not finite");
    mark("duplicates");
    P.n = n;
    P.m = m;
    P.nnz = 2 * m;
    P.offset = g->offset;
    P.col = colour_graph(n, row, col);
    mark("colour");
    const Colouring& C = P.col;
    sweep_rows(C, row, P.row);
    P.adj.resize(size_t(2 * m));
    P.J.resize(size_t(2 * m));
    P.h.assign(size_t(n), 0.0f);
#pragma omp parallel for schedule(dynamic, 4096) if (m >= (int64_t(1) << 16))
    for (int i = 0; i < n; ++i) {   // in the caller's bit order: the adjacency streams
        const int k = C.inverse[size_t(i)];
        int32_t pos = P.row[size_t(k)];
        for (int64_t e = row[size_t(i)]; e < row[size_t(i) + 1]; ++e) {
            P.adj[size_t(pos)] = C.inverse[size_t(col[size_t(e)])];
            P.J[size_t(pos)] = w[size_t(e)];
            ++pos;
        }
        P.h[size_t(k)] = g->h ? g->h[i] : 0.0f;
    }
    mark("arrays");
    mark.print();
    return QB_OK;
}

int64_t qubo_device_bytes(const QuboPlan& P) {
    return int64_t(P.row.size() + P.adj.size() + P.J.size() + P.h.size() + P.col.order.size() +
                   P.col.class_ptr.size()) * 4 + P.m * 12 + int64_t(P.n) * 4;
}

qb_status upload_qubo(QuboPlan& P, const qb_qubo_desc* g, cudaStream_t st, int64_t* bytes) {
    qb_status s;
    if ((s = upload_vec(P.d_row, P.row, st))) return s;
    if ((s = upload_vec(P.d_adj, P.adj, st))) return s;
    if ((s = upload_vec(P.d_J, P.J, st))) return s;
    if ((s = upload_vec(P.d_h, P.h, st))) return s;
    if ((s = upload_vec(P.d_order, P.col.order, st))) return s;
    if ((s = upload_vec(P.d_class_ptr, P.col.class_ptr, st))) return s;
    if ((s = upload(P.d_eu, g->eu, size_t(P.m) * 4, st))) return s;
    if ((s = upload(P.d_ev, g->ev, size_t(P.m) * 4, st))) return s;
    if ((s = upload(P.d_ew, g->ew, size_t(P.m) * 4, st))) return s;
    std::vector<float> ho(size_t(P.n), 0.0f);
    if (g->h) std::memcpy(ho.data(), g->h, size_t(P.n) * 4);
    if ((s = upload_vec(P.d_ho, ho, st))) return s;
    QB_CUDA(cudaStreamSynchronize(st));   // `ho` is a local
    *bytes = int64_t(P.d_row.bytes + P.d_adj.bytes + P.d_J.bytes + P.d_h.bytes + P.d_order.bytes +
                     P.d_class_ptr.bytes + P.d_eu.bytes + P.d_ev.bytes + P.d_ew.bytes + P.d_ho.bytes);
    return QB_OK;
}

// ---- residual planning ------------------------------------------------------------------

qb_status check_residual(const qb_residual_desc* d) {
    if (d->n_vars <= 0) return fail(QB_EINVAL, "residual: n_vars must be positive");
    if (d->n_rays < 0) return fail(QB_EINVAL, "residual: n_rays must be non-negative");
    if (!d->row_ptr || !d->nbr_ptr) return fail(QB_EINVAL, "residual: null CSR offsets");
    if (d->n_rays > 0 && (!d->d || !d->w)) return fail(QB_EINVAL, "residual: null d or w");
    const int n = d->n_vars;
    if (d->row_ptr[0] != 0 || d->nbr_ptr[0] != 0) return fail(QB_EINVAL, "residual: CSR offsets must start at 0");
    for (int i = 0; i < n; ++i) {
        if (d->row_ptr[i + 1] < d->row_ptr[i]) return fail(QB_EINVAL, "residual: row_ptr decreases");
        if (d->nbr_ptr[i + 1] < d->nbr_ptr[i]) return fail(QB_EINVAL, "residual: nbr_ptr decreases");
    }
    const int64_t nnz = d->row_ptr[n];
    if (nnz > 0 && (!d->ray || !d->a)) return fail(QB_EINVAL, "residual: null ray or a");
    if (d->nbr_ptr[n] > 0 && !d->nbr) return fail(QB_EINVAL, "residual: null nbr");
    // Bits are checked in parallel; the reported failure is the one of the
    // lowest failing bit (its first failing entry), as a sequential scan finds.
    static const char* const kWhy[] = {nullptr, "residual: ray index out of range",
                                       "residual: a bit lists a ray twice", "residual: non-finite a",
                                       "residual: neighbour index out of range",
                                       "residual: the neighbour lists are not symmetric"};
    int first_bad = n, why = 0;
#pragma omp parallel
    {
        std::vector<int32_t> stamp(size_t(std::max(d->n_rays, 1)), -1);
        int my_bad = n, my_why = 0;
#pragma omp for schedule(static, 2048)
        for (int i = 0; i < n; ++i) {
            if (i > my_bad) continue;
            int w = 0;
            for (int k = d->row_ptr[i]; k < d->row_ptr[i + 1] && !w; ++k) {
                const int b = d->ray[k];
                if (b < 0 || b >= d->n_rays) w = 1;
                else if (stamp[size_t(b)] == i) w = 2;
                else if (!std::isfinite(d->a[k])) w = 3;
                else stamp[size_t(b)] = i;
            }
            for (int k = d->nbr_ptr[i]; k < d->nbr_ptr[i + 1] && !w; ++k) {
                const int j = d->nbr[k];
                if (j < 0 || j >= n || j == i) {
                    w = 4;
                } else {
                    bool back = false;
                    for (int q = d->nbr_ptr[j]; q < d->nbr_ptr[j + 1]; ++q) back |= d->nbr[q] == i;
                    if (!back) w = 5;
                }
            }
            if (w && i < my_bad) {
                my_bad = i;
                my_why = w;
            }
        }
#pragma omp critical
        if (my_bad < first_bad) {
            first_bad = my_bad;
            why = my_why;
        }
    }
    if (why) return fail(QB_EINVAL, kWhy[why]);
    for (int b = 0; b < d->n_rays; ++b)
        if (!std::isfinite(d->d[b]) || !std::isfinite(d->w[b])) return fail(QB_EINVAL, "residual: non-finite d or w");
    return QB_OK;
}

// Host plan of a residual problem: colour classes, each class split into CL
// slices of about equal work (longest-processing-time first over bit-ray
// entries), heavy bits (more than resid_heavy_entries() rays) first inside a
// slice, slices cut into chunks that fit the kernel's stage buffers, and every
// device array in sweep order. Reordering bits inside a class changes no
// result: a class holds no two interacting bits.
qb_status plan_residual(const qb_residual_desc* d, ResidualPlan& P, int lock_slices) {
    const int n = d->n_vars, nr = d->n_rays;
    P.n = n;
    P.n_rays = nr;
    P.nnz = d->row_ptr[n];
    P.n_nbr = d->nbr_ptr[n];
    P.lambda = d->lambda;
    P.e0 = 0.0;
    for (int b = 0; b < nr; ++b) P.e0 += 0.5 * d->w[b] * d->d[b] * d->d[b];
    PlanMarks mark;
    P.col = colour_residual(n, nr, &P.max_ray_len, d->row_ptr, d->ray, d->nbr_ptr, d->nbr);
    mark("colour");
    Colouring& C = P.col;
    const int nc = C.n_colours();
    auto deg = [&](int i) { return d->row_ptr[i + 1] - d->row_ptr[i]; };
    // variant: lockstep unless QB_RESID_KERNEL=cluster or no cooperative grid
    const char* kv = std::getenv("QB_RESID_KERNEL");
    const bool want_cluster = kv && std::strcmp(kv, "cluster") == 0;
    P.variant = (lock_slices > 0 && !want_cluster) ? QB_RESID_LOCKSTEP : QB_RESID_CLUSTER;
    P.lock_grid = P.variant == QB_RESID_LOCKSTEP ? lock_slices : 0;
    // cluster size: the smallest whose shared memory holds one branch
    // (QB_RESID_CLUSTER overrides)
    int CL = env_int("QB_RESID_CLUSTER", 0);
    const int candidates[5] = {1, 2, 4, 8, 16};
    for (int t = 0; t < 5 && CL == 0; ++t) {
        const int c = candidates[t];
        const size_t bytes = size_t((nr + c - 1) / c) * 8 + size_t(n / c + nc + 64) / 8 + resid_stage_bytes();
        if (bytes <= size_t(112) * 1024) CL = c;
    }
    if (P.variant == QB_RESID_CLUSTER) {
        if (CL == 0) return fail(QB_ENOTSUP, "residual: the problem exceeds one cluster's shared memory");
        if (CL != 1 && CL != 2 && CL != 4 && CL != 8 && CL != 16)
            return fail(QB_EINVAL, "residual: cluster size must be 1, 2, 4, 8 or 16");
    }
    if (CL == 0) CL = 16;
    P.CL = CL;
    P.ray_slots = (nr + CL - 1) / CL;
    const int S = P.variant == QB_RESID_LOCKSTEP ? P.lock_grid : CL;   // slices per class
    const int heavy = resid_heavy_entries();
    // balanced slices: per class, longest-processing-time first onto the
    // least-loaded slice (a min-heap of loads); classes are independent
    std::vector<int32_t> slice_ptr(size_t(nc) * size_t(S + 1), 0);   // per class: S + 1 offsets
#pragma omp parallel
    {
        std::vector<int32_t> mem;
        std::vector<std::vector<int32_t>> slices(static_cast<size_t>(S));
        std::vector<std::pair<int64_t, int>> heap;
#pragma omp for schedule(dynamic, 1)
        for (int c = 0; c < nc; ++c) {
            const int cs = C.class_ptr[size_t(c)], ce = C.class_ptr[size_t(c) + 1];
            mem.assign(C.order.begin() + cs, C.order.begin() + ce);
            std::stable_sort(mem.begin(), mem.end(), [&](int a, int b) { return deg(a) > deg(b); });
            for (auto& v : slices) v.clear();
            heap.clear();
            for (int t = 0; t < S; ++t) heap.emplace_back(0, t);   // (load, slice): smallest first
            std::make_heap(heap.begin(), heap.end(), std::greater<std::pair<int64_t, int>>());
            for (int i : mem) {
                std::pop_heap(heap.begin(), heap.end(), std::greater<std::pair<int64_t, int>>());
                auto& top = heap.back();
                slices[size_t(top.second)].push_back(i);
                top.first += deg(i) + 8;
                std::push_heap(heap.begin(), heap.end(), std::greater<std::pair<int64_t, int>>());
            }
            int pos = cs;
            for (int t = 0; t < S; ++t) {
                auto& v = slices[size_t(t)];
                std::stable_sort(v.begin(), v.end(), [&](int a, int b) {
                    const bool ha = deg(a) > heavy, hb = deg(b) > heavy;
                    return ha != hb ? ha : a < b;
                });
                slice_ptr[size_t(c) * (S + 1) + size_t(t)] = pos;
                for (int i : v) C.order[size_t(pos++)] = i;
            }
            slice_ptr[size_t(c) * (S + 1) + size_t(S)] = pos;
        }
    }
    for (int k = 0; k < n; ++k) C.inverse[size_t(C.order[size_t(k)])] = k;
    mark("slices");
    const bool lock = P.variant == QB_RESID_LOCKSTEP;
    // homes (cluster variant): bit k of slice t of class c -> (t << 27) |
    // running slot of CTA t
    P.slot_base.assign(size_t(nc) * size_t(S), 0);
    P.bit_home.assign(size_t(n), 0);
    std::vector<int32_t> used(size_t(S), 0);
    for (int c = 0; c < nc; ++c)
        for (int t = 0; t < S; ++t) {
            P.slot_base[size_t(c) * S + size_t(t)] = used[size_t(t)];
            const int b0 = slice_ptr[size_t(c) * (S + 1) + size_t(t)], b1 = slice_ptr[size_t(c) * (S + 1) + size_t(t) + 1];
            for (int i = b0; i < b1; ++i) {
                if (!lock) P.bit_home[size_t(i)] = (uint32_t(t) << 27) | uint32_t(used[size_t(t)]);
                used[size_t(t)]++;
            }
        }
    P.bit_slots = *std::max_element(used.begin(), used.end());
    if (!lock && P.bit_slots >= (1 << 27)) return fail(QB_EREFUSED, "residual: too many bits per CTA");
    // sweep-order per-bit arrays (the entry table itself is assembled at upload)
    P.h_row.assign(size_t(n) + 1, 0);
    P.h_nbr_ptr.assign(size_t(n) + 1, 0);
#pragma omp parallel for schedule(static, 4096)
    for (int k = 0; k < n; ++k) {   // the degrees gathered in sweep order, then summed
        const int i = C.order[size_t(k)];
        P.h_row[size_t(k) + 1] = d->row_ptr[i + 1] - d->row_ptr[i];
        P.h_nbr_ptr[size_t(k) + 1] = d->nbr_ptr[i + 1] - d->nbr_ptr[i];
    }
    for (int k = 0; k < n; ++k) {
        P.h_row[size_t(k) + 1] += P.h_row[size_t(k)];
        P.h_nbr_ptr[size_t(k) + 1] += P.h_nbr_ptr[size_t(k)];
    }
    P.h_lin.resize(size_t(n));
    P.h_q.resize(size_t(n));
    P.h_nbr_home.resize(size_t(P.n_nbr));
    P.h_nbr_new.resize(size_t(P.n_nbr));
#pragma omp parallel for schedule(static, 1024)
    for (int i = 0; i < n; ++i) {   // in the caller's bit order: the entries stream
        const int k = C.inverse[size_t(i)];
        // q = 1/2 sum sign(w) a'^2 over the bit's entries, a' = fp32(sqrt|w| a):
        // the flip's own term of the data energy in the sweep's coefficients
        double qd = 0.0;
        for (int e = d->row_ptr[i]; e < d->row_ptr[i + 1]; ++e) {
            const double w = d->w[d->ray[e]];
            const double ap = double(ray_coef(w, d->a[e]));
            qd += (w < 0.0 ? -0.5 : 0.5) * ap * ap;
        }
        P.h_q[size_t(k)] = float(qd);
        P.h_lin[size_t(k)] = float(d->field ? d->field[i] : d->kappa);
        int32_t np = P.h_nbr_ptr[size_t(k)];
        for (int e = d->nbr_ptr[i]; e < d->nbr_ptr[i + 1]; ++e) {
            P.h_nbr_new[size_t(np)] = C.inverse[size_t(d->nbr[e])];
            P.h_nbr_home[size_t(np++)] = P.bit_home[size_t(C.inverse[size_t(d->nbr[e])])];
        }
    }
    if (lock) {
        P.h_meta.assign(size_t(n) * 8, 0u);
#pragma omp parallel for schedule(static, 4096)
        for (int k = 0; k < n; ++k) {
            uint32_t* m = &P.h_meta[size_t(k) * 8];
            m[0] = uint32_t(P.h_row[size_t(k)]);
            m[1] = uint32_t(P.h_row[size_t(k) + 1] - P.h_row[size_t(k)]);
            m[2] = uint32_t(P.h_nbr_ptr[size_t(k)]);
            m[3] = uint32_t(P.h_nbr_ptr[size_t(k) + 1] - P.h_nbr_ptr[size_t(k)]);
            std::memcpy(&m[4], &P.h_lin[size_t(k)], 4);
            std::memcpy(&m[5], &P.h_q[size_t(k)], 4);
            m[6] = uint32_t(C.order[size_t(k)]);
        }
    }
    mark("arrays");
    // chunk table of every CTA (see ResidualPlan)
    const int kB = lock ? resid_lockstep_chunk_bits() : resid_chunk_bits();
    const int kE = lock ? resid_lockstep_chunk_entries() : resid_chunk_entries();
    const int kN = lock ? resid_lockstep_chunk_nbrs() : resid_chunk_nbrs();
    const std::vector<int32_t>& row = P.h_row;
    const std::vector<int32_t>& nbp = P.h_nbr_ptr;
    const int kSeg = lock ? resid_lockstep_segment() : 1;
    const int kS = lock ? resid_lockstep_chunk_segments() : INT32_MAX;
    auto segs = [&](int k) { return (row[size_t(k) + 1] - row[size_t(k)] + kSeg - 1) / kSeg; };
    P.chunks.clear();
    P.chunk_ptr.assign(size_t(S) + 1, 0);
    // each slice's chunks on its own thread, joined in slice order
    std::vector<std::vector<int32_t>> per(static_cast<size_t>(S));
    int too_big = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(| : too_big)
    for (int t = 0; t < S; ++t) {
        std::vector<int32_t>& out = per[size_t(t)];
        for (int c = 0; c < nc && !too_big; ++c) {
            const int b0 = slice_ptr[size_t(c) * (S + 1) + size_t(t)], b1 = slice_ptr[size_t(c) * (S + 1) + size_t(t) + 1];
            const int slot0 = P.slot_base[size_t(c) * S + size_t(t)];
            int s0 = b0;
            do {
                int e = s0, nseg = 0;
                while (e < b1 && e - s0 < kB && row[size_t(e) + 1] - row[size_t(s0)] <= kE &&
                       nbp[size_t(e) + 1] - nbp[size_t(s0)] <= kN && (!lock || nseg + segs(e) <= kS)) {
                    if (lock) P.h_meta[size_t(e) * 8 + 7] = uint32_t(nseg);   // first segment of the bit
                    nseg += lock ? segs(e) : 0;
                    ++e;
                }
                if (e == s0 && s0 < b1) {
                    too_big = 1;
                    break;
                }
                int nh = 0;
                while (s0 + nh < e && row[size_t(s0 + nh) + 1] - row[size_t(s0 + nh)] > heavy) ++nh;
                const int32_t rec[8] = {s0, e, lock ? nseg : slot0 + (s0 - b0), (e == b1 ? 1 : 0) | (nh << 1),
                                        row[size_t(s0)], row[size_t(e)], nbp[size_t(s0)], nbp[size_t(e)]};
                out.insert(out.end(), rec, rec + 8);
                s0 = e;
            } while (s0 < b1);
        }
    }
    if (too_big) return fail(QB_ENOTSUP, "residual: a bit has more rays or neighbours than a chunk holds");
    for (int t = 0; t < S; ++t) {
        P.chunks.insert(P.chunks.end(), per[size_t(t)].begin(), per[size_t(t)].end());
        P.chunk_ptr[size_t(t) + 1] = int32_t(P.chunks.size() / 8);
    }
    mark("chunks");
    mark.print();
    return QB_OK;
}

// Bytes after the last bit-ray entry: the cluster sweep's bulk L2 prefetch
// moves whole 16-byte entry pairs and may reach one entry past the end.
constexpr size_t kEntPad = 16;

// Device bytes upload_residual will take.
int64_t residual_device_bytes(const ResidualPlan& P) {
    const int64_t n = P.n, nr = P.n_rays, nnz = P.nnz;
    int64_t b = int64_t(P.nnz * 2 + int64_t(P.h_row.size()) + P.h_lin.size() + P.h_q.size() + P.h_nbr_ptr.size() +
                        P.h_nbr_home.size() + P.col.order.size() + P.col.class_ptr.size() + P.chunks.size() +
                        P.chunk_ptr.size()) * 4;
    b += (nr + 1) * 4 + nnz * 12 + n * 8 + nr * 16 + (n + 1) * 4 + P.n_nbr * 4;   // ray-major CSR (two bit orders)
    if (P.variant == QB_RESID_LOCKSTEP) b += int64_t(P.h_meta.size() + P.h_nbr_new.size()) * 4 + nnz * 4;
    return b;
}

// The sweep-order entry table and the ray-major CSR on the host: the same
// arrays as the device assembly (qb_build.cu), for rays too long for its sort.
static void host_build_residual(const ResidualPlan& P, const qb_residual_desc* d, RawVec<uint32_t>& ent,
                                std::vector<int32_t>& rrow, RawVec<int32_t>& rbit_o, RawVec<uint32_t>& rbit_h,
                                RawVec<int32_t>& rbit_n, RawVec<float>& ra) {
    const int n = P.n, nr = P.n_rays;
    const Colouring& C = P.col;
    ent.resize(size_t(P.nnz) * 2 + kEntPad / 4);
    for (size_t k = size_t(P.nnz) * 2; k < ent.size(); ++k) ent[k] = 0u;
#pragma omp parallel for schedule(static, 1024)
    for (int k = 0; k < n; ++k) {
        const int i = C.order[size_t(k)];
        int32_t pos = P.h_row[size_t(k)];
        for (int e = d->row_ptr[i]; e < d->row_ptr[i + 1]; ++e, ++pos) {
            const double w = d->w[d->ray[e]];
            const float ap = ray_coef(w, d->a[e]);   // the residual's exact step
            uint32_t* en = &ent[size_t(pos) * 2];
            en[0] = uint32_t(d->ray[e]) | (w < 0.0 ? 0x80000000u : 0u);
            std::memcpy(&en[1], &ap, 4);
        }
    }
    // ray-major CSR, bits ascending in input order inside a ray: a counting
    // sort by ray split over threads by contiguous bit ranges (each thread
    // counts its bits per ray, the counts are prefix-summed across threads,
    // and each thread fills its own slots)
    rrow.assign(size_t(nr) + 1, 0);
    rbit_o.resize(size_t(P.nnz));
    rbit_h.resize(size_t(P.nnz));
    rbit_n.resize(size_t(P.nnz));
    ra.resize(size_t(P.nnz));
    int T = 1;
#ifdef _OPENMP
    T = std::max(1, std::min(omp_get_max_threads(), 32));
#endif
    std::vector<std::vector<int32_t>> cnt(static_cast<size_t>(T));
    auto bits_of = [&](int t, int* i0, int* i1) {
        *i0 = int(int64_t(n) * t / T);
        *i1 = int(int64_t(n) * (t + 1) / T);
    };
#pragma omp parallel for num_threads(T) schedule(static, 1)
    for (int t = 0; t < T; ++t) {
        int i0, i1;
        bits_of(t, &i0, &i1);
        auto& c = cnt[size_t(t)];
        c.assign(size_t(nr), 0);
        for (int e = d->row_ptr[i0]; e < d->row_ptr[i1]; ++e) c[size_t(d->ray[e])]++;
    }
    for (int b = 0; b < nr; ++b) {
        int32_t run = rrow[size_t(b)];
        for (int t = 0; t < T; ++t) {
            const int32_t v = cnt[size_t(t)][size_t(b)];
            cnt[size_t(t)][size_t(b)] = run;   // this thread's first slot on ray b
            run += v;
        }
        rrow[size_t(b) + 1] = run;
    }
#pragma omp parallel for num_threads(T) schedule(static, 1)
    for (int t = 0; t < T; ++t) {
        int i0, i1;
        bits_of(t, &i0, &i1);
        auto& fill = cnt[size_t(t)];
        for (int i = i0; i < i1; ++i)
            for (int e = d->row_ptr[i]; e < d->row_ptr[i + 1]; ++e) {
                const int32_t k = fill[size_t(d->ray[e])]++;
                rbit_o[size_t(k)] = i;
                rbit_h[size_t(k)] = P.bit_home[size_t(C.inverse[size_t(i)])];
                rbit_n[size_t(k)] = C.inverse[size_t(i)];
                ra[size_t(k)] = d->a[e];
            }
    }
}

qb_status upload_residual(ResidualPlan& P, const qb_residual_desc* d, cudaStream_t st, int64_t* bytes) {
    const int n = P.n, nr = P.n_rays;
    const Colouring& C = P.col;
    const bool lock = P.variant == QB_RESID_LOCKSTEP;
    qb_status s;
    // the O(nnz) tables: assembled on the device from the caller's CSR unless a
    // ray is too long for the device sort (QB_RESID_BUILD=host forces the host)
    const char* bv = std::getenv("QB_RESID_BUILD");
    const bool on_device = P.max_ray_len <= kRaySortMax && !(bv && std::strcmp(bv, "host") == 0);
    RawVec<uint32_t> ent;
    std::vector<int32_t> rrow;
    RawVec<int32_t> rbit_o, rbit_n;
    RawVec<uint32_t> rbit_h;
    RawVec<float> ra;
    DevBuf t_row_ptr, t_ray, t_a, t_inverse, t_home, t_rcount, t_cursor, t_rkey, t_rbit_n;
    if (on_device) {
        if ((s = upload(t_row_ptr, d->row_ptr, (size_t(n) + 1) * 4, st))) return s;
        if ((s = upload(t_ray, d->ray, size_t(P.nnz) * 4, st))) return s;
        if ((s = upload(t_a, d->a, size_t(P.nnz) * 4, st))) return s;
        if ((s = upload_vec(t_inverse, C.inverse, st))) return s;
        if ((s = upload_vec(t_home, P.bit_home, st))) return s;
        if ((s = upload_vec(P.d_row, P.h_row, st))) return s;
        if ((s = upload_vec(P.d_order, C.order, st))) return s;
        if ((s = upload(P.d_w64, d->w, size_t(nr) * 8, st))) return s;
        if ((s = P.d_ent.alloc(size_t(P.nnz) * 8 + kEntPad))) return s;
        if ((s = P.d_rrow.alloc((size_t(nr) + 1) * 4))) return s;
        if ((s = P.d_o_rbit.alloc(size_t(P.nnz) * 4))) return s;
        if ((s = P.d_rbit.alloc(size_t(P.nnz) * 4))) return s;
        if ((s = P.d_ra.alloc(size_t(P.nnz) * 4))) return s;
        DevBuf& rbn = lock ? P.d_rbit_new : t_rbit_n;   // sweep positions: kept by the lockstep sweep only
        if ((s = rbn.alloc(size_t(P.nnz) * 4))) return s;
        if ((s = t_rcount.alloc(size_t(std::max(nr, 1)) * 4))) return s;
        if ((s = t_cursor.alloc(size_t(std::max(nr, 1)) * 4))) return s;
        if ((s = t_rkey.alloc(size_t(P.nnz) * 8))) return s;
        ResidBuildArgs A{};
        A.n = n;
        A.n_rays = nr;
        A.row_ptr = t_row_ptr.as<int32_t>();
        A.ray = t_ray.as<int32_t>();
        A.a = t_a.as<float>();
        A.w = P.d_w64.as<double>();
        A.order = P.d_order.as<int32_t>();
        A.inverse = t_inverse.as<int32_t>();
        A.h_row = P.d_row.as<int32_t>();
        A.bit_home = t_home.as<uint32_t>();
        A.ent = P.d_ent.as<uint2>();
        A.rrow = P.d_rrow.as<int32_t>();
        A.rbit_o = P.d_o_rbit.as<int32_t>();
        A.rbit_n = rbn.as<int32_t>();
        A.rbit_h = P.d_rbit.as<uint32_t>();
        A.ra = P.d_ra.as<float>();
        A.rcount = t_rcount.as<int32_t>();
        A.cursor = t_cursor.as<int32_t>();
        A.rkey = t_rkey.as<unsigned long long>();
        if ((s = launch_resid_build(A, st))) return s;
    } else {
        host_build_residual(P, d, ent, rrow, rbit_o, rbit_h, rbit_n, ra);
    }
    std::vector<double> o_lin(static_cast<size_t>(n));
    for (int i = 0; i < n; ++i) o_lin[size_t(i)] = d->field ? d->field[i] : d->kappa;
#define QB_UP(buf, vec) if ((s = upload_vec(P.buf, vec, st))) return s
    if (!on_device) {
        QB_UP(d_ent, ent); QB_UP(d_row, P.h_row); QB_UP(d_order, C.order);
        QB_UP(d_rrow, rrow); QB_UP(d_rbit, rbit_h); QB_UP(d_ra, ra); QB_UP(d_o_rbit, rbit_o);
        if (lock) QB_UP(d_rbit_new, rbit_n);
        if ((s = upload(P.d_w64, d->w, size_t(nr) * 8, st))) return s;
    }
    QB_UP(d_lin, P.h_lin); QB_UP(d_q, P.h_q);
    QB_UP(d_nbr_ptr, P.h_nbr_ptr); QB_UP(d_nbr_home, P.h_nbr_home);
    QB_UP(d_class_ptr, C.class_ptr); QB_UP(d_chunks, P.chunks); QB_UP(d_chunk_ptr, P.chunk_ptr);
    QB_UP(d_o_lin, o_lin);
    if (lock) {
        QB_UP(d_meta, P.h_meta); QB_UP(d_nbr_new, P.h_nbr_new);
    }
#undef QB_UP
    if ((s = upload(P.d_d, d->d, size_t(nr) * 8, st))) return s;
    if ((s = upload(P.d_o_nbr_ptr, d->nbr_ptr, (size_t(n) + 1) * 4, st))) return s;
    if ((s = upload(P.d_o_nbr, d->nbr, size_t(P.n_nbr) * 4, st))) return s;
    QB_CUDA(cudaStreamSynchronize(st));   // the host vectors and device scratch above are locals
    const DevBuf* all[] = {&P.d_row, &P.d_ent, &P.d_lin, &P.d_q, &P.d_nbr_ptr, &P.d_nbr_home, &P.d_order,
                           &P.d_class_ptr, &P.d_chunks, &P.d_chunk_ptr, &P.d_d, &P.d_w64, &P.d_rrow, &P.d_rbit,
                           &P.d_ra, &P.d_o_rbit, &P.d_o_nbr_ptr, &P.d_o_nbr, &P.d_o_lin,
                           &P.d_meta, &P.d_nbr_new, &P.d_rbit_new};
    int64_t tot = 0;
    for (const DevBuf* b : all) tot += int64_t(b->bytes);
    *bytes = tot;
    return QB_OK;
}

qb_status check_schedule(const qb_schedule* s) {
    if (!s) return fail(QB_EINVAL, "schedule: null");
    if (s->anneal_sweeps < 0 || s->hold_sweeps < 0 || s->anneal_sweeps + s->hold_sweeps < 1)
        return fail(QB_EINVAL, "schedule: needs at least one sweep");
    if (!(s->t_hot > 0.0) || !(s->t_cold > 0.0) || !std::isfinite(s->t_hot) || !std::isfinite(s->t_cold))
        return fail(QB_EINVAL, "schedule: temperatures must be positive and finite");
    if (s->refresh_sweeps < 0) return fail(QB_EINVAL, "schedule: refresh_sweeps must be non-negative");
    return QB_OK;
}

qb_status wait(qb_result* r) {
    if (!r->synced) {
        QB_CUDA(cudaStreamSynchronize(r->stream));
        r->synced = true;
    }
    if (r->d_err) {
        int e = 0;
        QB_CUDA(cudaMemcpy(&e, r->d_err, sizeof(int), cudaMemcpyDeviceToHost));
        if (e) return fail(QB_ETIMEDOUT, "a grid barrier of the sweep timed out: the results are not valid");
    }
    return QB_OK;
}

qb_status download(qb_result* r, void* dst, const DevBuf& src, size_t bytes) {
    if (!dst) return fail(QB_EINVAL, "result: null output buffer");
    if (!src.p || src.bytes < bytes) return fail(QB_EINVAL, "result: this output is not available for the problem kind");
    QB_CUDA(cudaSetDevice(r->device));
    QB_CUDA(cudaMemcpyAsync(dst, src.p, bytes, cudaMemcpyDeviceToHost, r->stream));
    QB_CUDA(cudaStreamSynchronize(r->stream));
    r->synced = true;
    return wait(r);
}

}  // namespace

// ---- problems ------------------------------------------------------------------------------

qb_status qb::problem_upload(qb_problem* p, cudaStream_t st) {
    if (p->uploaded) return QB_OK;
    const bool gone = p->kind == QB_KIND_ISING   ? p->host.eu.empty() && p->ising.m > 0
                      : p->kind == QB_KIND_QUBO ? p->host.eu.empty() && p->qubo.m > 0
                                                : p->host.row_ptr.empty();
    if (gone)
        return fail(QB_EINVAL, "problem: its device memory was released and it was not created with deferred upload");
    QB_CUDA(cudaSetDevice(p->device));
    HostDesc& h = p->host;
    qb_status s;
    if (p->kind == QB_KIND_ISING) {
        const qb_ising_desc d{p->ising.n, p->ising.m, h.eu.data(), h.ev.data(), h.ew.data()};
        s = upload_ising(p->ising, &d, st, &p->device_bytes);
    } else if (p->kind == QB_KIND_QUBO) {
        const qb_qubo_desc d{p->qubo.n, p->qubo.m, h.eu.data(), h.ev.data(), h.wf.data(),
                             h.hf.empty() ? nullptr : h.hf.data(), h.offset};
        s = upload_qubo(p->qubo, &d, st, &p->device_bytes);
    } else {
        const qb_residual_desc d{p->resid.n, p->resid.n_rays, h.d.data(), h.w.data(), h.row_ptr.data(), h.ray.data(),
                                 h.a.data(), h.nbr_ptr.data(), h.nbr.data(), h.lambda, h.kappa,
                                 h.has_field ? h.field.data() : nullptr};
        s = upload_residual(p->resid, &d, st, &p->device_bytes);
    }
    if (s != QB_OK) return s;
    p->uploaded = true;   // host copies stay: the problem can go to the device again after a release
    return QB_OK;
}

qb_status qb::replan_residual(qb_problem* p, int slices) {
    if (p->kind != QB_KIND_RESIDUAL || p->resid.variant != QB_RESID_LOCKSTEP) return QB_OK;
    if (p->resid.lock_grid == slices) return QB_OK;
    HostDesc& h = p->host;
    if (h.row_ptr.empty()) return fail(QB_EINVAL, "replan: the problem keeps no host copy (create it with QB_OPT_DEFER_UPLOAD)");
    if (p->uploaded) problem_release_device(p);
    const qb_residual_desc d{p->resid.n, p->resid.n_rays, h.d.data(), h.w.data(), h.row_ptr.data(), h.ray.data(),
                             h.a.data(), h.nbr_ptr.data(), h.nbr.data(), h.lambda, h.kappa,
                             h.has_field ? h.field.data() : nullptr};
    ResidualPlan fresh;
    qb_status s = plan_residual(&d, fresh, slices);
    if (s != QB_OK) return s;
    if (fresh.variant != QB_RESID_LOCKSTEP) return fail(QB_ENOTSUP, "replan: the lockstep plan was not kept");
    p->resid = std::move(fresh);
    p->device_bytes = residual_device_bytes(p->resid);
    return QB_OK;
}

void qb::problem_release_device(qb_problem* p) {
    IsingPlan& I = p->ising;
    ResidualPlan& R = p->resid;
    QuboPlan& Q = p->qubo;
    DevBuf* all[] = {&I.d_row, &I.d_adj, &I.d_w, &I.d_f0, &I.d_order, &I.d_class_ptr, &I.d_eu, &I.d_ev, &I.d_ew,
                     &R.d_row, &R.d_ent, &R.d_lin, &R.d_q, &R.d_nbr_ptr, &R.d_nbr_home, &R.d_order, &R.d_class_ptr,
                     &R.d_chunks, &R.d_chunk_ptr, &R.d_d, &R.d_w64, &R.d_rrow, &R.d_rbit, &R.d_ra, &R.d_meta,
                     &R.d_nbr_new, &R.d_rbit_new, &R.d_o_row, &R.d_o_ray, &R.d_o_a, &R.d_o_nbr_ptr, &R.d_o_nbr,
                     &R.d_o_lin, &R.d_o_rbit,
                     &Q.d_row, &Q.d_adj, &Q.d_J, &Q.d_h, &Q.d_order, &Q.d_class_ptr, &Q.d_eu, &Q.d_ev, &Q.d_ew, &Q.d_ho,
                     &p->d_temp};
    // buffers of the plain create path go back to the pool on the legacy
    // stream: no queued work may still read them
    bool wait = false;
    for (DevBuf* b : all) wait |= b->sync_free;
    if (wait) cudaDeviceSynchronize();
    for (DevBuf* b : all) b->release();
    p->uploaded = false;
}

extern "C" qb_status qb_problem_create_ising(const qb_ising_desc* desc, const qb_opts* opts, qb_problem** out) {
    return qb::guarded("qb_problem_create_ising", [&]() -> qb_status {
        if (!desc || !out) return fail(QB_EINVAL, "qb_problem_create_ising: null argument");
        *out = nullptr;
        qb_problem* p = new (std::nothrow) qb_problem();
        if (!p) return fail(QB_ENOMEM, "qb_problem_create_ising: out of host memory");
        p->kind = QB_KIND_ISING;
        const bool defer = opts && (opts->flags & QB_OPT_DEFER_UPLOAD);
        qb_status s = plan_ising(desc, p->ising);
        if (s == QB_OK && p->ising.w_min == 0) s = fail(QB_EREFUSED, "ising: all weights are zero");   // ising_gpu.cuh:94
        if (s == QB_OK) s = select_device(opts, &p->device);
        if (s == QB_OK && defer) {
            const size_t m = size_t(desc->m);
            p->host.eu.assign(desc->eu, desc->eu + m);
            p->host.ev.assign(desc->ev, desc->ev + m);
            p->host.ew.assign(desc->ew, desc->ew + m);
            p->device_bytes = ising_device_bytes(p->ising);
        } else if (s == QB_OK) {
            AsyncAllocScope pool(stream_of(opts), true);   // returned at destroy, after a device synchronise
            s = upload_ising(p->ising, desc, stream_of(opts), &p->device_bytes);
            p->uploaded = s == QB_OK;
        }
        if (s != QB_OK) {
            qb_problem_destroy(p);   // waits for any copy the failed upload queued
            return s;
        }
        *out = p;
        return QB_OK;
    });
}

extern "C" qb_status qb_problem_create_residual(const qb_residual_desc* desc, const qb_opts* opts, qb_problem** out) {
    return qb::guarded("qb_problem_create_residual", [&]() -> qb_status {
        if (!desc || !out) return fail(QB_EINVAL, "qb_problem_create_residual: null argument");
        *out = nullptr;
        // QB_PLAN_TIMES=1 prints the host check, plan and upload times to stderr
        const bool times = std::getenv("QB_PLAN_TIMES") != nullptr;
        auto now = [] { return std::chrono::steady_clock::now(); };
        auto ms = [](std::chrono::steady_clock::time_point a, std::chrono::steady_clock::time_point b) {
            return std::chrono::duration<double, std::milli>(b - a).count();
        };
        const auto t0 = now();
        qb_status s = check_residual(desc);
        if (s != QB_OK) return s;
        qb_problem* p = new (std::nothrow) qb_problem();
        if (!p) return fail(QB_ENOMEM, "qb_problem_create_residual: out of host memory");
        p->kind = QB_KIND_RESIDUAL;
        const bool defer = opts && (opts->flags & QB_OPT_DEFER_UPLOAD);
        const bool cluster = opts && (opts->flags & QB_OPT_RESID_CLUSTER);
        s = select_device(opts, &p->device);
        const auto t1 = now();
        if (s == QB_OK) s = plan_residual(desc, p->resid, cluster ? 0 : resid_lockstep_grid());
        if (s == QB_OK && p->resid.variant == QB_RESID_CLUSTER) s = resid_check_fit(p->resid);
        const auto t2 = now();
        if (s == QB_OK && defer) {
            HostDesc& h = p->host;
            const int n = desc->n_vars, nr = desc->n_rays;
            const size_t nnz = size_t(desc->row_ptr[n]), nn = size_t(desc->nbr_ptr[n]);
            h.d.assign(desc->d, desc->d + nr);
            h.w.assign(desc->w, desc->w + nr);
            h.row_ptr.assign(desc->row_ptr, desc->row_ptr + n + 1);
            h.ray.assign(desc->ray, desc->ray + nnz);
            h.a.assign(desc->a, desc->a + nnz);
            h.nbr_ptr.assign(desc->nbr_ptr, desc->nbr_ptr + n + 1);
            h.nbr.assign(desc->nbr, desc->nbr + nn);
            h.has_field = desc->field != nullptr;
            if (h.has_field) h.field.assign(desc->field, desc->field + n);
            h.lambda = desc->lambda;
            h.kappa = desc->kappa;
            p->device_bytes = residual_device_bytes(p->resid);
        } else if (s == QB_OK) {
            AsyncAllocScope pool(stream_of(opts), true);   // returned at destroy, after a device synchronise
            s = upload_residual(p->resid, desc, stream_of(opts), &p->device_bytes);
            p->uploaded = s == QB_OK;
        }
        if (times)
            std::fprintf(stderr, "[qb plan] check %.1f ms, plan %.1f ms, upload %.1f ms\n", ms(t0, t1), ms(t1, t2),
                         ms(t2, now()));
        if (s != QB_OK) {
            qb_problem_destroy(p);   // waits for any copy the failed upload queued
            return s;
        }
        *out = p;
        return QB_OK;
    });
}

extern "C" qb_status qb_problem_create_qubo(const qb_qubo_desc* desc, const qb_opts* opts, qb_problem** out) {
    return qb::guarded("qb_problem_create_qubo", [&]() -> qb_status {
        if (!desc || !out) return fail(QB_EINVAL, "qb_problem_create_qubo: null argument");
        *out = nullptr;
        qb_problem* p = new (std::nothrow) qb_problem();
        if (!p) return fail(QB_ENOMEM, "qb_problem_create_qubo: out of host memory");
        p->kind = QB_KIND_QUBO;
        const bool defer = opts && (opts->flags & QB_OPT_DEFER_UPLOAD);
        qb_status s = plan_qubo(desc, p->qubo);
        if (s == QB_OK) s = select_device(opts, &p->device);
        if (s == QB_OK && defer) {
            const size_t m = size_t(desc->m);
            HostDesc& h = p->host;
            h.eu.assign(desc->eu, desc->eu + m);
            h.ev.assign(desc->ev, desc->ev + m);
            h.wf.assign(desc->ew, desc->ew + m);
            if (desc->h) h.hf.assign(desc->h, desc->h + desc->n);
            h.offset = desc->offset;
            p->device_bytes = qubo_device_bytes(p->qubo);
        } else if (s == QB_OK) {
            AsyncAllocScope pool(stream_of(opts), true);   // returned at destroy, after a device synchronise
            s = upload_qubo(p->qubo, desc, stream_of(opts), &p->device_bytes);
            p->uploaded = s == QB_OK;
        }
        if (s != QB_OK) {
            qb_problem_destroy(p);   // waits for any copy the failed upload queued
            return s;
        }
        *out = p;
        return QB_OK;
    });
}

extern "C" void qb_problem_destroy(qb_problem* p) {
    if (!p) return;
    cudaSetDevice(p->device);
    // the problem's buffers go back to the library's pool: no work that reads
    // them may still be queued (cudaFree used to wait for the device the same way)
    cudaDeviceSynchronize();
    delete p;
}

extern "C" qb_status qb_problem_info_get(const qb_problem* p, qb_problem_info* info) {
    if (!p || !info) return fail(QB_EINVAL, "qb_problem_info_get: null argument");
    std::memset(info, 0, sizeof(*info));
    info->kind = p->kind;
    info->device_bytes = p->device_bytes;
    const Colouring& C = p->kind == QB_KIND_ISING ? p->ising.col : p->kind == QB_KIND_QUBO ? p->qubo.col : p->resid.col;
    info->n_colours = C.n_colours();
    for (int k = 0; k < C.n_colours(); ++k)
        info->max_class = std::max(info->max_class, C.class_ptr[size_t(k) + 1] - C.class_ptr[size_t(k)]);
    if (p->kind == QB_KIND_ISING) {
        const IsingPlan& P = p->ising;
        info->n = P.n;
        info->nnz = P.nnz;
        info->field_bytes = 4;
        info->weight_bytes = P.weight_bytes;
        info->sigma = P.sigma;
        info->w_min = double(P.w_min);
        info->field_bound = P.B;
    } else if (p->kind == QB_KIND_QUBO) {
        info->n = p->qubo.n;
        info->nnz = p->qubo.nnz;
        info->field_bytes = 8;    // fp32 hi + lo
        info->weight_bytes = 4;
    } else {
        const ResidualPlan& P = p->resid;
        info->n = P.n;
        info->nnz = P.nnz;
        info->n_rays = P.n_rays;
        info->field_bytes = 4;
        info->weight_bytes = 4;
        info->variant = P.variant;
    }
    return QB_OK;
}

extern "C" qb_status qb_problem_colouring(const qb_problem* p, int32_t* order, int32_t* class_ptr, int32_t* n_colours) {
    if (!p) return fail(QB_EINVAL, "qb_problem_colouring: null problem");
    const Colouring& C = p->kind == QB_KIND_ISING ? p->ising.col : p->kind == QB_KIND_QUBO ? p->qubo.col : p->resid.col;
    if (order) std::memcpy(order, C.order.data(), C.order.size() * sizeof(int32_t));
    if (class_ptr) std::memcpy(class_ptr, C.class_ptr.data(), C.class_ptr.size() * sizeof(int32_t));
    if (n_colours) *n_colours = C.n_colours();
    return QB_OK;
}

extern "C" qb_status qb_colour_ising(const qb_ising_desc* desc, int32_t* order, int32_t* class_ptr, int32_t* n_colours) {
    return qb::guarded("qb_colour_ising", [&]() -> qb_status {
        if (!desc) return fail(QB_EINVAL, "qb_colour_ising: null descriptor");
        IsingPlan P;
        qb_status s = plan_ising(desc, P);
        if (s != QB_OK) return s;
        if (order) std::memcpy(order, P.col.order.data(), P.col.order.size() * sizeof(int32_t));
        if (class_ptr) std::memcpy(class_ptr, P.col.class_ptr.data(), P.col.class_ptr.size() * sizeof(int32_t));
        if (n_colours) *n_colours = P.col.n_colours();
        return QB_OK;
    });
}

extern "C" qb_status qb_colour_residual(const qb_residual_desc* desc, int32_t* order, int32_t* class_ptr, int32_t* n_colours) {
    return qb::guarded("qb_colour_residual", [&]() -> qb_status {
        if (!desc) return fail(QB_EINVAL, "qb_colour_residual: null descriptor");
        qb_status s = check_residual(desc);
        if (s != QB_OK) return s;
        ResidualPlan P;
        if ((s = plan_residual(desc, P, kHostLockSlices)) != QB_OK) return s;
        const Colouring& c = P.col;
        if (order) std::memcpy(order, c.order.data(), c.order.size() * sizeof(int32_t));
        if (class_ptr) std::memcpy(class_ptr, c.class_ptr.data(), c.class_ptr.size() * sizeof(int32_t));
        if (n_colours) *n_colours = c.n_colours();
        return QB_OK;
    });
}

extern "C" qb_status qb_schedule_scaled(const qb_problem* p, int32_t anneal_sweeps, int32_t hold_sweeps, qb_schedule* out) {
    if (!p || !out) return fail(QB_EINVAL, "qb_schedule_scaled: null argument");
    if (p->kind != QB_KIND_ISING) return fail(QB_EINVAL, "qb_schedule_scaled: ising problems only");
    out->t_hot = p->ising.sigma;
    out->t_cold = 0.1 * double(p->ising.w_min);
    out->anneal_sweeps = anneal_sweeps;
    out->hold_sweeps = hold_sweeps;
    out->refresh_sweeps = 0;
    return QB_OK;
}

// ---- solve ---------------------------------------------------------------------------------------

extern "C" qb_status qb_solve(qb_problem* p, const qb_schedule* sch, uint32_t n_branches, uint64_t seed_offset,
                              const qb_opts* opts, qb_result** out) {
    return qb::guarded("qb_solve", [&]() -> qb_status {
        if (!p || !out) return fail(QB_EINVAL, "qb_solve: null argument");
        *out = nullptr;
        qb_status s = check_schedule(sch);
        if (s != QB_OK) return s;
        if (n_branches < 1 || n_branches > (1u << 20)) return fail(QB_EINVAL, "qb_solve: n_branches must be in [1, 2^20]");
        QB_CUDA(cudaSetDevice(p->device));
        cudaStream_t st = stream_of(opts);
        if ((s = problem_upload(p, st)) != QB_OK) return s;
        qb_result* r = new (std::nothrow) qb_result();
        if (!r) return fail(QB_ENOMEM, "qb_solve: out of host memory");
        r->prob = p;
        r->device = p->device;
        r->stream = st;
        r->R = int(n_branches);
        r->sweeps = sch->anneal_sweeps + sch->hold_sweeps;
        const int R = r->R;
        const int n = p->kind == QB_KIND_ISING ? p->ising.n : p->kind == QB_KIND_QUBO ? p->qubo.n : p->resid.n;
        r->n = n;
        const uint64_t seed0 = 1 + seed_offset;   // branch b: seed b + 1 + offset (ising_recon.hpp:157)
        auto bail = [&](qb_status e) {
            qb_result_destroy(r);
            return e;
        };
        const bool same = p->d_temp.p && p->temp_sched.t_hot == sch->t_hot && p->temp_sched.t_cold == sch->t_cold &&
                          p->temp_sched.anneal_sweeps == sch->anneal_sweeps && p->temp_sched.hold_sweeps == sch->hold_sweeps;
        if (!same) {
            const std::vector<double> temp = temperatures(*sch);
            QB_CUDA(cudaStreamSynchronize(st));   // a solve in flight may still read the old table
            if ((s = upload_vec(p->d_temp, temp, st))) return bail(s);
            QB_CUDA(cudaStreamSynchronize(st));
            p->temp_sched = *sch;
        }
        if ((s = alloc_async(r->d_x, size_t(R) * size_t(n), st))) return bail(s);
        if ((s = alloc_async(r->d_e_f64, size_t(R) * sizeof(double), st))) return bail(s);
        if ((s = alloc_async(r->d_p, size_t(n) * sizeof(float), st))) return bail(s);
        if (cudaEventCreate(&r->ev0) != cudaSuccess || cudaEventCreate(&r->ev1) != cudaSuccess ||
            cudaEventCreate(&r->ev2) != cudaSuccess)
            return bail(cuda_fail(cudaGetLastError(), "cudaEventCreate", __FILE__, __LINE__));
        SolveBuffers b;
        b.x = r->d_x.as<uint8_t>();
        b.e_f64 = r->d_e_f64.as<double>();
        b.p = r->d_p.as<float>();
        b.temp = p->d_temp.as<double>();
        if (opts && (opts->flags & QB_OPT_TRACE)) {
            const size_t tb = size_t(R) * size_t(r->sweeps) * 8;
            if ((s = alloc_async(r->d_trace, tb, st))) return bail(s);
            QB_CUDA(cudaMemsetAsync(r->d_trace.p, 0, tb, st));
            b.trace = r->d_trace.as<double>();
            r->trace_base = p->kind == QB_KIND_RESIDUAL ? p->resid.e0 : p->kind == QB_KIND_QUBO ? p->qubo.offset : 0.0;
        }
        if (p->kind == QB_KIND_ISING && !b.trace && packed_replicas_fit(p->ising, R)) {
            // many replicas: groups of them as work items of the packed kernel
            // (the same branches, fields and energies as one CTA per replica)
            const IsingPlan& P = p->ising;
            r->d_x.release();
            r->d_p.release();
            cudaEventRecord(r->ev0, st);
            if ((s = packed_replicas(p, *sch, R, seed_offset, opts, &r->packed, r->d_x, r->d_f, r->d_e_i64, r->d_p)))
                return bail(s);
            cudaEventRecord(r->ev1, st);
            b.x = r->d_x.as<uint8_t>();
            if ((s = alloc_async(r->d_e_scr, size_t(R) * 8, st))) return bail(s);
            if ((s = launch_ising_energies(P, b.x, R, r->d_e_scr.as<long long>(), st))) return bail(s);
            if ((s = launch_i64_to_f64(r->d_e_scr.as<long long>(), R, b.e_f64, st))) return bail(s);
            r->launches = 2 + 2;   // packed anneal + its marginals, energies, conversion
            cudaEventRecord(r->ev2, st);
            *out = r;
            return QB_OK;
        }
        if (p->kind == QB_KIND_ISING) {
            const IsingPlan& P = p->ising;
            if ((s = alloc_async(r->d_f, size_t(R) * size_t(n) * 4, st))) return bail(s);
            if ((s = alloc_async(r->d_e_i64, size_t(R) * 8, st))) return bail(s);
            if ((s = alloc_async(r->d_e_scr, size_t(R) * 8, st))) return bail(s);
            if (ising_smem_bytes(P) == 0 && (s = alloc_async(r->d_scratch, size_t(R) * size_t(n) * 5, st))) return bail(s);
            b.f = r->d_f.as<int32_t>();
            b.e_i64 = r->d_e_i64.as<long long>();
            b.scratch = r->d_scratch.p;
            cudaEventRecord(r->ev0, st);
            if ((s = launch_ising_anneal(P, b, R, r->sweeps, seed0, st))) return bail(s);
            cudaEventRecord(r->ev1, st);
            if ((s = launch_ising_energies(P, b.x, R, r->d_e_scr.as<long long>(), st))) return bail(s);
            if ((s = launch_i64_to_f64(r->d_e_scr.as<long long>(), R, b.e_f64, st))) return bail(s);
            r->launches = 3;
        } else if (p->kind == QB_KIND_QUBO) {
            const QuboPlan& P = p->qubo;
            if ((s = alloc_async(r->d_drift, size_t(R) * sizeof(float), st))) return bail(s);
            if ((s = alloc_async(r->d_accepts, size_t(R) * 8, st))) return bail(s);
            if ((s = alloc_async(r->d_e_track, size_t(R) * 8, st))) return bail(s);
            if ((s = alloc_async(r->d_scratch, qubo_scratch(P), st))) return bail(s);
            if (cudaMemsetAsync(r->d_drift.p, 0, size_t(R) * sizeof(float), st) != cudaSuccess ||
                cudaMemsetAsync(r->d_accepts.p, 0, size_t(R) * 8, st) != cudaSuccess ||
                cudaMemsetAsync(r->d_e_track.p, 0, size_t(R) * 8, st) != cudaSuccess ||
                cudaMemsetAsync(r->d_scratch.p, 0, 64, st) != cudaSuccess)
                return bail(cuda_fail(cudaGetLastError(), "cudaMemsetAsync", __FILE__, __LINE__));
            r->d_err = reinterpret_cast<const int*>(static_cast<const char*>(r->d_scratch.p) + 16);
            const int RB = qubo_max_branches();
            cudaEventRecord(r->ev0, st);
            int anneal_launches = 0;
            for (int b0 = 0; b0 < R && s == QB_OK; b0 += RB, ++anneal_launches) {
                QuboBuffers qbuf;
                qbuf.x = b.x + size_t(b0) * size_t(n);
                qbuf.temp = b.temp;
                qbuf.drift = r->d_drift.as<float>() + b0;
                qbuf.e_track = r->d_e_track.as<double>() + b0;
                qbuf.accepts = r->d_accepts.as<unsigned long long>() + b0;
                qbuf.trace = b.trace ? b.trace + size_t(b0) * size_t(r->sweeps) : nullptr;
                qbuf.scratch = r->d_scratch.p;
                s = launch_qubo_lockstep(P, qbuf, std::min(RB, R - b0), r->sweeps, sch->refresh_sweeps,
                                         seed0 + uint64_t(b0), st);
            }
            if (s != QB_OK) return bail(s);
            cudaEventRecord(r->ev1, st);
            if ((s = launch_qubo_energies(P, b.x, R, b.e_f64, st))) return bail(s);
            r->launches = anneal_launches + 1;
        } else {
            const ResidualPlan& P = p->resid;
            if ((s = alloc_async(r->d_drift, size_t(R) * sizeof(float), st))) return bail(s);
            if ((s = alloc_async(r->d_accepts, size_t(R) * 8, st))) return bail(s);
            if (cudaMemsetAsync(r->d_drift.p, 0, size_t(R) * sizeof(float), st) != cudaSuccess ||
                cudaMemsetAsync(r->d_accepts.p, 0, size_t(R) * 8, st) != cudaSuccess)
                return bail(cuda_fail(cudaGetLastError(), "cudaMemsetAsync", __FILE__, __LINE__));
            b.drift = r->d_drift.as<float>();
            b.accepts = r->d_accepts.as<unsigned long long>();
            const int RB = std::min(R, resid_lockstep_max_branches());   // branches per lockstep launch
            if (P.variant == QB_RESID_LOCKSTEP) {
                if ((s = alloc_async(r->d_scratch, resid_lockstep_scratch(P, RB), st))) return bail(s);
                b.scratch = r->d_scratch.p;
                QB_CUDA(cudaMemsetAsync(r->d_scratch.p, 0, 64, st));   // control block, timeout flag included
                r->d_err = reinterpret_cast<const int*>(static_cast<const char*>(r->d_scratch.p) + 16);
            }
            cudaEventRecord(r->ev0, st);
            int anneal_launches = 0;
            if (P.variant == QB_RESID_LOCKSTEP) {
                // blocks of at most RB branches, one cooperative launch each
                for (int b0 = 0; b0 < R && s == QB_OK; b0 += RB, ++anneal_launches) {
                    SolveBuffers bb = b;
                    bb.x = b.x + size_t(b0) * size_t(n);
                    bb.drift = b.drift + b0;
                    if (b.trace) bb.trace = b.trace + size_t(b0) * size_t(r->sweeps);
                    s = launch_resid_lockstep(P, bb, std::min(RB, R - b0), r->sweeps, sch->refresh_sweeps,
                                              seed0 + uint64_t(b0), st);
                }
            } else {
                s = launch_resid_anneal(P, b, R, r->sweeps, sch->refresh_sweeps, seed0, st);
                anneal_launches = 1;
            }
            if (s != QB_OK) return bail(s);
            cudaEventRecord(r->ev1, st);
            if ((s = launch_resid_energies(P, b.x, R, b.e_f64, st))) return bail(s);
            r->launches = anneal_launches + 1;
        }
        if ((s = launch_marginals(b.x, R, n, b.p, st))) return bail(s);
        r->launches += 1;
        cudaEventRecord(r->ev2, st);
        *out = r;
        return QB_OK;
    });
}

extern "C" qb_status qb_result_info_get(qb_result* r, qb_result_info* info) {
    if (!r || !info) return fail(QB_EINVAL, "qb_result_info_get: null argument");
    QB_CUDA(cudaSetDevice(r->device));
    qb_status s = wait(r);
    if (s != QB_OK) return s;
    std::memset(info, 0, sizeof(*info));
    info->n = r->n;
    info->n_branches = r->R;
    info->sweeps = r->sweeps;
    info->launches = r->launches;
    info->attempts = int64_t(r->R) * int64_t(r->sweeps) * int64_t(r->n);
    QB_CUDA(cudaEventElapsedTime(&info->anneal_ms, r->ev0, r->ev1));
    QB_CUDA(cudaEventElapsedTime(&info->total_ms, r->ev0, r->ev2));
    if (r->prob->kind == QB_KIND_QUBO) {
        std::vector<double> et(static_cast<size_t>(r->R)), ef(static_cast<size_t>(r->R));
        QB_CUDA(cudaMemcpy(et.data(), r->d_e_track.p, et.size() * 8, cudaMemcpyDeviceToHost));
        QB_CUDA(cudaMemcpy(ef.data(), r->d_e_f64.p, ef.size() * 8, cudaMemcpyDeviceToHost));
        for (size_t k = 0; k < et.size(); ++k)
            info->max_energy_error = std::max(info->max_energy_error, std::fabs(r->prob->qubo.offset + et[k] - ef[k]));
    }
    if (r->prob->kind == QB_KIND_RESIDUAL && r->d_trace.p) {
        // a traced residual solve: E(x = 0) plus the accepted dE against the fp64 energy
        std::vector<double> tr(size_t(r->R) * size_t(r->sweeps)), ef(static_cast<size_t>(r->R));
        QB_CUDA(cudaMemcpy(tr.data(), r->d_trace.p, tr.size() * 8, cudaMemcpyDeviceToHost));
        QB_CUDA(cudaMemcpy(ef.data(), r->d_e_f64.p, ef.size() * 8, cudaMemcpyDeviceToHost));
        for (int k = 0; k < r->R; ++k) {
            double e = r->trace_base;
            for (int t = 0; t < r->sweeps; ++t) e += tr[size_t(k) * size_t(r->sweeps) + size_t(t)];
            info->max_energy_error = std::max(info->max_energy_error, std::fabs(e - ef[size_t(k)]));
        }
    }
    if (r->prob->kind == QB_KIND_RESIDUAL || r->prob->kind == QB_KIND_QUBO) {
        std::vector<float> dr(static_cast<size_t>(r->R));
        QB_CUDA(cudaMemcpy(dr.data(), r->d_drift.p, dr.size() * sizeof(float), cudaMemcpyDeviceToHost));
        for (float v : dr) info->max_drift = std::max(info->max_drift, double(v));
        std::vector<unsigned long long> ac(size_t(r->R));
        QB_CUDA(cudaMemcpy(ac.data(), r->d_accepts.p, ac.size() * 8, cudaMemcpyDeviceToHost));
        for (unsigned long long v : ac) info->accepted += int64_t(v);
    }
    return QB_OK;
}

extern "C" qb_status qb_result_branches(qb_result* r, uint8_t* x) {
    if (!r) return fail(QB_EINVAL, "qb_result_branches: null result");
    return download(r, x, r->d_x, size_t(r->R) * size_t(r->n));
}

extern "C" qb_status qb_result_energies_i64(qb_result* r, int64_t* e) {
    if (!r) return fail(QB_EINVAL, "qb_result_energies_i64: null result");
    if (r->prob->kind != QB_KIND_ISING) return fail(QB_EINVAL, "qb_result_energies_i64: ising problems only");
    return download(r, e, r->d_e_i64, size_t(r->R) * 8);
}

extern "C" qb_status qb_result_fields_i64(qb_result* r, int64_t* f) {
    if (!r || !f) return fail(QB_EINVAL, "qb_result_fields_i64: null argument");
    if (r->prob->kind != QB_KIND_ISING) return fail(QB_EINVAL, "qb_result_fields_i64: ising problems only");
    std::vector<int32_t> f32(size_t(r->R) * size_t(r->n));
    qb_status s = download(r, f32.data(), r->d_f, f32.size() * 4);
    if (s != QB_OK) return s;
    for (size_t k = 0; k < f32.size(); ++k) f[k] = f32[k];
    return QB_OK;
}

extern "C" qb_status qb_result_energies_f64(qb_result* r, double* e) {
    if (!r) return fail(QB_EINVAL, "qb_result_energies_f64: null result");
    return download(r, e, r->d_e_f64, size_t(r->R) * 8);
}

extern "C" qb_status qb_result_energy_trace(qb_result* r, double* trace) {
    return qb::guarded("qb_result_energy_trace", [&]() -> qb_status {
        if (!r || !trace) return fail(QB_EINVAL, "qb_result_energy_trace: null argument");
        if (!r->d_trace.p) return fail(QB_EINVAL, "qb_result_energy_trace: the solve was not made with QB_OPT_TRACE");
        const size_t R = size_t(r->R), S = size_t(r->sweeps);
        if (r->prob->kind == QB_KIND_ISING) {
            std::vector<long long> t(R * S);
            qb_status s = download(r, t.data(), r->d_trace, t.size() * 8);
            if (s != QB_OK) return s;
            for (size_t k = 0; k < t.size(); ++k) trace[k] = double(t[k]);
            return QB_OK;
        }
        // per-sweep sums of accepted dE, accumulated from the energy of x = 0
        // (residual) or the offset (qubo) in sweep order
        std::vector<double> t(R * S);
        qb_status s = download(r, t.data(), r->d_trace, t.size() * 8);
        if (s != QB_OK) return s;
        for (size_t k = 0; k < R; ++k) {
            double e = r->trace_base;
            for (size_t q = 0; q < S; ++q) {
                e += t[k * S + q];
                trace[k * S + q] = e;
            }
        }
        return QB_OK;
    });
}

extern "C" qb_status qb_result_marginals(qb_result* r, float* p) {
    if (!r) return fail(QB_EINVAL, "qb_result_marginals: null result");
    return download(r, p, r->d_p, size_t(r->n) * 4);
}

extern "C" qb_status qb_result_tristate(qb_result* r, float lo, float hi, uint8_t* bits) {
    if (!r || !bits) return fail(QB_EINVAL, "qb_result_tristate: null argument");
    if (!(lo <= hi)) return fail(QB_EINVAL, "qb_result_tristate: needs lo <= hi");
    QB_CUDA(cudaSetDevice(r->device));
    DevBuf tmp;
    qb_status s = alloc_async(tmp, size_t(r->n), r->stream);
    if (s != QB_OK) return s;
    s = launch_tristate(r->d_p.as<float>(), r->n, lo, hi, tmp.as<uint8_t>(), r->stream);
    if (s == QB_OK) s = download(r, bits, tmp, size_t(r->n));
    free_async(tmp, r->stream);
    return s;
}

extern "C" void qb_result_destroy(qb_result* r) {
    if (!r) return;
    cudaSetDevice(r->device);
    cudaStream_t st = r->stream;
    DevBuf* all[] = {&r->d_x, &r->d_f, &r->d_e_i64, &r->d_e_scr, &r->d_e_f64, &r->d_p, &r->d_temp, &r->d_drift,
                     &r->d_accepts, &r->d_e_track, &r->d_scratch, &r->d_trace};
    if (r->packed) qb_batch_destroy(r->packed);   // waits for the stream: its tables are in use until then
    for (DevBuf* b : all) free_async(*b, st);
    if (r->ev0) cudaEventDestroy(r->ev0);
    if (r->ev1) cudaEventDestroy(r->ev1);
    if (r->ev2) cudaEventDestroy(r->ev2);
    delete r;
}

// ---- evaluators -------------------------------------------------------------------------------

extern "C" qb_status qb_energies_ising(const qb_problem* p, const uint8_t* x, int32_t k, int64_t* e) {
    return qb::guarded("qb_energies_ising", [&]() -> qb_status {
        if (!p || (!x && k > 0) || (!e && k > 0) || k < 0) return fail(QB_EINVAL, "qb_energies_ising: bad argument");
        if (p->kind != QB_KIND_ISING) return fail(QB_EINVAL, "qb_energies_ising: ising problems only");
        if (!p->uploaded) return fail(QB_EINVAL, "qb_energies_ising: the problem is not on the device");
        if (k == 0) return QB_OK;
        QB_CUDA(cudaSetDevice(p->device));
        DevBuf dx, de;
        qb_status s;
        if ((s = upload(dx, x, size_t(k) * size_t(p->ising.n), nullptr))) return s;
        if ((s = de.alloc(size_t(k) * 8))) return s;
        if ((s = launch_ising_energies(p->ising, dx.as<uint8_t>(), k, de.as<long long>(), nullptr))) return s;
        QB_CUDA(cudaMemcpy(e, de.p, size_t(k) * 8, cudaMemcpyDeviceToHost));
        return QB_OK;
    });
}

extern "C" qb_status qb_energies_qubo(const qb_problem* p, const uint8_t* x, int32_t k, double* e) {
    return qb::guarded("qb_energies_qubo", [&]() -> qb_status {
        if (!p || (!x && k > 0) || (!e && k > 0) || k < 0) return fail(QB_EINVAL, "qb_energies_qubo: bad argument");
        if (p->kind != QB_KIND_QUBO) return fail(QB_EINVAL, "qb_energies_qubo: weighted qubo problems only");
        if (!p->uploaded) return fail(QB_EINVAL, "qb_energies_qubo: the problem is not on the device");
        if (k == 0) return QB_OK;
        QB_CUDA(cudaSetDevice(p->device));
        DevBuf dx, de;
        qb_status s;
        if ((s = upload(dx, x, size_t(k) * size_t(p->qubo.n), nullptr))) return s;
        if ((s = de.alloc(size_t(k) * 8))) return s;
        if ((s = launch_qubo_energies(p->qubo, dx.as<uint8_t>(), k, de.as<double>(), nullptr))) return s;
        QB_CUDA(cudaMemcpy(e, de.p, size_t(k) * 8, cudaMemcpyDeviceToHost));
        return QB_OK;
    });
}

extern "C" qb_status qb_energies_residual(const qb_problem* p, const uint8_t* x, int32_t k, double* e) {
    return qb::guarded("qb_energies_residual", [&]() -> qb_status {
        if (!p || (!x && k > 0) || (!e && k > 0) || k < 0) return fail(QB_EINVAL, "qb_energies_residual: bad argument");
        if (p->kind != QB_KIND_RESIDUAL) return fail(QB_EINVAL, "qb_energies_residual: residual problems only");
        if (!p->uploaded) return fail(QB_EINVAL, "qb_energies_residual: the problem is not on the device");
        if (k == 0) return QB_OK;
        QB_CUDA(cudaSetDevice(p->device));
        DevBuf dx, de;
        qb_status s;
        if ((s = upload(dx, x, size_t(k) * size_t(p->resid.n), nullptr))) return s;
        if ((s = de.alloc(size_t(k) * 8))) return s;
        if ((s = launch_resid_energies(p->resid, dx.as<uint8_t>(), k, de.as<double>(), nullptr))) return s;
        QB_CUDA(cudaMemcpy(e, de.p, size_t(k) * 8, cudaMemcpyDeviceToHost));
        return QB_OK;
    });
}

extern "C" qb_status qb_metropolis_check(const uint64_t* u53, const double* dE, const double* T, int32_t n,
                                         int32_t device, uint8_t* fast, uint8_t* accept, uint8_t* exact) {
    return guarded("metropolis_check", [&]() -> qb_status {
        if (n < 0) return fail(QB_EINVAL, "metropolis_check: n must be non-negative");
        if (n > 0 && (!u53 || !dE || !T || !fast || !accept || !exact))
            return fail(QB_EINVAL, "metropolis_check: null array");
        if (n == 0) return QB_OK;
        QB_CUDA(cudaSetDevice(device));
        DevBuf du, de, dt, dout;
        qb_status s;
        if ((s = upload(du, u53, size_t(n) * 8, nullptr)) || (s = upload(de, dE, size_t(n) * 8, nullptr)) ||
            (s = upload(dt, T, size_t(n) * 8, nullptr)) || (s = dout.alloc(size_t(n) * 3)))
            return s;
        uint8_t* o = dout.as<uint8_t>();
        if ((s = launch_metropolis_check(du.as<uint64_t>(), de.as<double>(), dt.as<double>(), n, o, o + n, o + 2 * size_t(n),
                                         nullptr)))
            return s;
        QB_CUDA(cudaMemcpy(fast, o, size_t(n), cudaMemcpyDeviceToHost));
        QB_CUDA(cudaMemcpy(accept, o + n, size_t(n), cudaMemcpyDeviceToHost));
        QB_CUDA(cudaMemcpy(exact, o + 2 * size_t(n), size_t(n), cudaMemcpyDeviceToHost));
        return QB_OK;
    });
}

extern "C" qb_status qb_device_trim(int32_t device) {
    return guarded("qb_device_trim", [&]() -> qb_status {
        QB_CUDA(cudaSetDevice(device));
        QB_CUDA(cudaDeviceSynchronize());
        if (cudaMemPool_t pool = library_pool(device)) QB_CUDA(cudaMemPoolTrimTo(pool, 0));
        return QB_OK;
    });
}
