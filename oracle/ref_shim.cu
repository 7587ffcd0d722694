// ref_shim.cu -- TEST INFRASTRUCTURE ONLY. A C interface over the reference's
// own annealing code, compiled unchanged from QuBLAR's sources (the include
// path points into the reference tree; nothing is copied). Built by
// oracle/Makefile into oracle/_ref/libqbref.so; host code only, no kernel of the
// reference is launched.
//
// Wrapped: argos::wising::parse_rudy / anneal / cut_of / energy_scratch
// (src/ising_weighted.hpp:83-267), argos::binary_energy / local_field_dE /
// anneal_branch / branch_fractions (src/ising_recon.hpp:65-166),
// argos::BitField::grid / assemble (src/engine.hpp:61-149).
#include <chrono>
#include <cstdint>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "engine.hpp"
#include "ising_recon.hpp"
#include "ising_weighted.hpp"

namespace wi = argos::wising;

extern "C" {

// ---- integer engine ---------------------------------------------------------------------

void* ref_graph_parse(const char* text, size_t len, char* err, int errlen) {
    auto* g = new wi::WeightedGraph();
    std::string e;
    if (!wi::parse_rudy(text, len, *g, e)) {
        if (err && errlen > 0) {
            std::strncpy(err, e.c_str(), size_t(errlen - 1));
            err[errlen - 1] = 0;
        }
        delete g;
        return nullptr;
    }
    return g;
}

void ref_graph_free(void* h) { delete static_cast<wi::WeightedGraph*>(h); }

void ref_graph_sizes(void* h, int* n, long long* m, long long* sum_w) {
    const auto* g = static_cast<wi::WeightedGraph*>(h);
    *n = g->n;
    *m = g->m;
    *sum_w = g->sum_w;
}

long long ref_cut_of(void* h, const uint8_t* x) {
    const auto* g = static_cast<wi::WeightedGraph*>(h);
    return wi::cut_of(*g, std::vector<uint8_t>(x, x + g->n));
}

long long ref_energy_scratch(void* h, const uint8_t* x) {
    const auto* g = static_cast<wi::WeightedGraph*>(h);
    return wi::energy_scratch(*g, std::vector<uint8_t>(x, x + g->n));
}

// wi::anneal for seeds seed0 .. seed0+R-1 on a pool of n_threads; X: R x n, E: R.
double ref_wising_anneal_many(void* h, double t_hot, double t_cold, int anneal, int hold, uint64_t seed0, int R,
                              int n_threads, uint8_t* X, long long* E) {
    const auto* g = static_cast<wi::WeightedGraph*>(h);
    wi::Budget b;
    b.t_hot = t_hot;
    b.t_cold = t_cold;
    b.anneal_sweeps = anneal;
    b.hold_sweeps = hold;
    const auto t0 = std::chrono::steady_clock::now();
    std::vector<std::thread> pool;
    for (int t = 0; t < n_threads; ++t)
        pool.emplace_back([&, t] {
            for (int r = t; r < R; r += n_threads) {
                const wi::RunOut o = wi::anneal(*g, b, seed0 + uint64_t(r));
                if (X) std::memcpy(X + size_t(r) * size_t(g->n), o.x.data(), size_t(g->n));
                if (E) E[r] = o.energy_tracked;
            }
        });
    for (auto& th : pool) th.join();
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// wi::anneal's loop, instrumented: the tracked energy after each sweep (the
// precedent of check_ree_qubo.cu:195-216), through the reference's own State,
// Budget schedule and uniform().
long long ref_wising_trace(void* h, double t_hot, double t_cold, int anneal, int hold, uint64_t seed, uint8_t* x,
                           double* trace) {
    const auto* g = static_cast<wi::WeightedGraph*>(h);
    wi::State st(*g);
    uint64_t state = seed * 0x2545F4914F6CDD1Dull + 1;
    const int total = anneal + hold;
    for (int sweep = 0; sweep < total; ++sweep) {
        const double frac = std::min(1.0, double(sweep) / std::max(1, anneal - 1));
        const double temp = sweep < anneal ? t_hot * std::pow(t_cold / t_hot, frac) : t_cold;
        for (int i = 0; i < g->n; ++i) {
            const double dE = double(st.dE(i));
            if (dE <= 0.0 || wi::detail::uniform(state) < std::exp(-dE / temp)) st.flip(i);
        }
        trace[sweep] = double(st.energy);
    }
    const std::vector<uint8_t> xo = st.x();
    std::memcpy(x, xo.data(), xo.size());
    return st.energy;
}

// ---- float / residual engine ------------------------------------------------------------------

struct RefResidDesc {   // the layout of qb_residual_desc
    int32_t n_vars, n_rays;
    const double *d, *w;
    const int32_t *row_ptr, *ray;
    const float* a;
    const int32_t *nbr_ptr, *nbr;
    double lambda, kappa;
    const double* field;
};

void* ref_problem_new(const RefResidDesc* s) {
    auto* p = new argos::BinaryProblem();
    const int n = s->n_vars;
    p->var_voxel.resize(size_t(n));
    for (int i = 0; i < n; ++i) p->var_voxel[size_t(i)] = i;
    p->voxel_var = p->var_voxel;
    p->d.assign(s->d, s->d + s->n_rays);
    p->w.assign(s->w, s->w + s->n_rays);
    p->row_ptr.assign(s->row_ptr, s->row_ptr + n + 1);
    p->ray.assign(s->ray, s->ray + s->row_ptr[n]);
    p->a.assign(s->a, s->a + s->row_ptr[n]);
    p->nbr_ptr.assign(s->nbr_ptr, s->nbr_ptr + n + 1);
    p->nbr.assign(s->nbr, s->nbr + s->nbr_ptr[n]);
    p->lambda = s->lambda;
    p->kappa = s->kappa;
    if (s->field) p->field.assign(s->field, s->field + n);
    return p;
}

void ref_problem_free(void* h) { delete static_cast<argos::BinaryProblem*>(h); }

double ref_binary_energy(void* h, const uint8_t* x) {
    const auto* p = static_cast<argos::BinaryProblem*>(h);
    return argos::binary_energy(*p, std::vector<uint8_t>(x, x + p->n_vars()));
}

double ref_local_field_dE(void* h, const uint8_t* x, const double* r, int i) {
    const auto* p = static_cast<argos::BinaryProblem*>(h);
    return argos::local_field_dE(*p, std::vector<uint8_t>(x, x + p->n_vars()),
                                 std::vector<double>(r, r + p->n_rays()), i);
}

void ref_anneal_branch(void* h, double t_hot, double t_cold, int anneal, int hold, uint64_t seed, uint8_t* x) {
    const auto* p = static_cast<argos::BinaryProblem*>(h);
    argos::Schedule s;
    s.t_hot = t_hot;
    s.t_cold = t_cold;
    s.anneal_sweeps = anneal;
    s.hold_sweeps = hold;
    const std::vector<uint8_t> o = argos::anneal_branch(*p, s, seed);
    std::memcpy(x, o.data(), o.size());
}

// branch_fractions with its own thread pool; returns the wall seconds.
double ref_branch_fractions(void* h, double t_hot, double t_cold, int anneal, int hold, int n_branches,
                            unsigned n_threads, uint64_t seed_offset, float* frac, uint8_t* X) {
    const auto* p = static_cast<argos::BinaryProblem*>(h);
    argos::Schedule s;
    s.t_hot = t_hot;
    s.t_cold = t_cold;
    s.anneal_sweeps = anneal;
    s.hold_sweeps = hold;
    std::vector<std::vector<uint8_t>> keep;
    const auto t0 = std::chrono::steady_clock::now();
    const std::vector<float> f = argos::branch_fractions(*p, s, n_branches, n_threads, X ? &keep : nullptr, seed_offset);
    const double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (frac) std::memcpy(frac, f.data(), f.size() * sizeof(float));
    if (X)
        for (size_t b = 0; b < keep.size(); ++b) std::memcpy(X + b * size_t(p->n_vars()), keep[b].data(), keep[b].size());
    return wall;
}

// anneal_branch's loop, instrumented with binary_energy after each sweep
// (check_ree_qubo.cu:195-216: an instrumented copy, identical arithmetic).
void ref_anneal_branch_trace(void* h, double t_hot, double t_cold, int anneal, int hold, uint64_t seed, uint8_t* xo,
                             double* trace) {
    const auto* p = static_cast<argos::BinaryProblem*>(h);
    std::vector<uint8_t> x(size_t(p->n_vars()), 0);
    std::vector<double> r(size_t(p->n_rays()));
    for (int b = 0; b < p->n_rays(); ++b) r[size_t(b)] = -p->d[size_t(b)];
    uint64_t state = seed * 0x2545F4914F6CDD1Dull + 1;
    const int total = anneal + hold;
    for (int sweep = 0; sweep < total; ++sweep) {
        const double frac = std::min(1.0, double(sweep) / std::max(1, anneal - 1));
        const double temp = sweep < anneal ? t_hot * std::pow(t_cold / t_hot, frac) : t_cold;
        for (int i = 0; i < p->n_vars(); ++i) {
            const double delta = x[size_t(i)] ? -1.0 : 1.0;
            const double dE = argos::local_field_dE(*p, x, r, i);
            if (dE <= 0.0 || argos::detail::uniform(state) < std::exp(-dE / temp)) {
                x[size_t(i)] ^= 1u;
                for (int k = p->row_ptr[size_t(i)]; k < p->row_ptr[size_t(i) + 1]; ++k)
                    r[size_t(p->ray[size_t(k)])] += p->a[size_t(k)] * delta;
            }
        }
        trace[sweep] = argos::binary_energy(*p, x);
    }
    std::memcpy(xo, x.data(), x.size());
}

// freeze_provable_rock (ising_recon.hpp:187-234): returns the kept count and
// fills kept (reduced -> original), the reduced field and neighbour CSR.
int ref_freeze(void* h, double margin, int32_t* kept, double* field, int32_t* nbr_ptr, int32_t* nbr, int* rounds) {
    const auto* p = static_cast<argos::BinaryProblem*>(h);
    const argos::FreezeResult fr = argos::freeze_provable_rock(*p, margin);
    const int nk = int(fr.kept.size());
    std::memcpy(kept, fr.kept.data(), size_t(nk) * 4);
    std::memcpy(field, fr.reduced.field.data(), size_t(nk) * 8);
    std::memcpy(nbr_ptr, fr.reduced.nbr_ptr.data(), size_t(nk + 1) * 4);
    std::memcpy(nbr, fr.reduced.nbr.data(), fr.reduced.nbr.size() * 4);
    *rounds = fr.rounds;
    return nk;
}

// roi_qubo (ising_recon.hpp:251-300): h (n) and J (n x n, upper triangle) of
// the region `roi` with the rest held at x_bar.
void ref_roi_qubo(void* h, const int32_t* roi, int n_roi, const uint8_t* x_bar, double* h_out, double* J_out) {
    const auto* p = static_cast<argos::BinaryProblem*>(h);
    const argos::RoiQubo q = argos::roi_qubo(*p, std::vector<int>(roi, roi + n_roi),
                                             std::vector<uint8_t>(x_bar, x_bar + p->n_vars()));
    std::memcpy(h_out, q.h.data(), size_t(n_roi) * 8);
    std::memcpy(J_out, q.J.data(), size_t(n_roi) * size_t(n_roi) * 8);
}

// ---- problem assembly -------------------------------------------------------------------

// BitField::grid over the domain mask (nx x ny x nz, x fastest) and assemble
// (src/engine.hpp:61-149) of one sensor's rows given as entries (bit, row, a)
// in row order, with the prior (lambda, kappa). Outputs sized by the caller:
// var_voxel (n bits), row_ptr (n + 1), ray and a (n_entries), nbr_ptr (n + 1),
// nbr (6 n at most); returns the bit count, *n_nbr the neighbour entries.
int ref_grid_assemble(int nx, int ny, int nz, const uint8_t* domain, int n_rows, const double* d, const double* w,
                      long long n_entries, const int32_t* e_bit, const int32_t* e_row, const float* e_a,
                      double lambda, double kappa, int32_t* var_voxel, int32_t* row_ptr, int32_t* ray, float* a,
                      int32_t* nbr_ptr, int32_t* nbr, long long* n_nbr) {
    const std::vector<char> dom(domain, domain + size_t(nx) * ny * nz);
    const argos::BitField f = argos::BitField::grid(nx, ny, nz, dom);
    argos::OperatorRows op;
    op.d.assign(d, d + n_rows);
    op.w.assign(w, w + n_rows);
    for (long long k = 0; k < n_entries; ++k) op.entries.push_back({e_bit[k], e_row[k], e_a[k]});
    argos::IsingPrior prior;
    prior.lambda = lambda;
    prior.kappa = kappa;
    const argos::BinaryProblem p = argos::assemble(f, {&op}, prior);
    const int n = p.n_vars();
    std::memcpy(var_voxel, p.var_voxel.data(), size_t(n) * 4);
    std::memcpy(row_ptr, p.row_ptr.data(), size_t(n + 1) * 4);
    std::memcpy(ray, p.ray.data(), p.ray.size() * 4);
    std::memcpy(a, p.a.data(), p.a.size() * 4);
    std::memcpy(nbr_ptr, p.nbr_ptr.data(), size_t(n + 1) * 4);
    std::memcpy(nbr, p.nbr.data(), p.nbr.size() * 4);
    *n_nbr = (long long)p.nbr.size();
    return n;
}

}  // extern "C"
