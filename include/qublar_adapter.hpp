// qublar_adapter.hpp -- the reference's C++ call shapes over the C ABI.
//
// A QuBLAR caller swaps one function name and keeps its arguments:
//
//   argos::branch_fractions(prob, sched, n, threads, &keep, off)   (src/ising_recon.hpp:148-166)
//     -> qublar::compat::branch_fractions(prob, sched, n, threads, &keep, off)
//   argos::anneal_branch(prob, sched, seed)                         (src/ising_recon.hpp:121-144)
//     -> qublar::compat::anneal_branch(prob, sched, seed)
//   argos::wising::anneal(graph, budget, seed)                      (src/ising_weighted.hpp:250-267)
//     -> qublar::compat::anneal<argos::wising::RunOut>(graph, budget, seed)
//   argos::gising::run_batch(dg, budget, seed_base, R)              (src/ising_gpu.cuh:396-458)
//     -> qublar::compat::run_batch(graph, budget, seed_base, R)
//
// The templates read the reference types by member name (BinaryProblem:
// var_voxel, d, w, row_ptr, ray, a, nbr_ptr, nbr, lambda, kappa, field;
// WeightedGraph: n, m, eu, ev, ew; Schedule/Budget: t_hot, t_cold,
// anneal_sweeps, hold_sweeps), so this header needs none of the reference's
// headers. Failures throw std::runtime_error with the library's message; the
// C ABI underneath never throws or exits. n_threads is accepted and ignored
// (the GPU replaces the thread pool).
#pragma once

#include <algorithm>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "qublar.h"

namespace qublar {
namespace compat {

inline void check(qb_status s, const char* what) {
    if (s != QB_OK)
        throw std::runtime_error(std::string(what) + ": " + qb_status_string(s) + ": " + qb_last_error());
}

// RAII over the C handles.
struct Problem {
    qb_problem* h = nullptr;
    Problem() = default;
    Problem(const Problem&) = delete;
    Problem& operator=(const Problem&) = delete;
    ~Problem() { qb_problem_destroy(h); }
};
struct Result {
    qb_result* h = nullptr;
    Result() = default;
    Result(const Result&) = delete;
    Result& operator=(const Result&) = delete;
    ~Result() { qb_result_destroy(h); }
};

// Residual refresh cadence used by the adapter (fp64 recompute of the fp32
// residuals every this many sweeps).
constexpr int32_t kRefreshSweeps = 50;

// The C ABI reads as many entries as the offsets say; the vectors know their
// lengths, so an inconsistent problem is refused here before any call.
inline void require(bool ok, const char* why) {
    if (!ok) throw std::runtime_error(std::string("qublar adapter: ") + why);
}

template <class BinaryProblemT>
qb_residual_desc residual_desc(const BinaryProblemT& p) {
    const size_t n = p.var_voxel.size();
    require(p.row_ptr.size() == n + 1 && p.nbr_ptr.size() == n + 1, "row_ptr and nbr_ptr need n_vars + 1 entries");
    require(p.w.size() == p.d.size(), "d and w differ in length");
    require(p.row_ptr.back() >= 0 && size_t(p.row_ptr.back()) <= std::min(p.ray.size(), p.a.size()),
            "row_ptr[n_vars] exceeds the length of ray or a");
    require(p.nbr_ptr.back() >= 0 && size_t(p.nbr_ptr.back()) <= p.nbr.size(),
            "nbr_ptr[n_vars] exceeds the length of nbr");
    require(p.field.empty() || p.field.size() >= n, "field is shorter than n_vars");
    qb_residual_desc d{};
    d.n_vars = int32_t(p.var_voxel.size());
    d.n_rays = int32_t(p.d.size());
    d.d = p.d.data();
    d.w = p.w.data();
    d.row_ptr = p.row_ptr.data();
    d.ray = p.ray.data();
    d.a = p.a.data();
    d.nbr_ptr = p.nbr_ptr.data();
    d.nbr = p.nbr.data();
    d.lambda = p.lambda;
    d.kappa = p.kappa;
    d.field = p.field.empty() ? nullptr : p.field.data();
    return d;
}

template <class ScheduleT>
qb_schedule schedule_of(const ScheduleT& s, int32_t refresh = kRefreshSweeps) {
    qb_schedule q{};
    q.t_hot = s.t_hot;
    q.t_cold = s.t_cold;
    q.anneal_sweeps = int32_t(s.anneal_sweeps);
    q.hold_sweeps = int32_t(s.hold_sweeps);
    q.refresh_sweeps = refresh;
    return q;
}

// argos::branch_fractions: per-bit fraction of n_branches annealed branches
// with x = 1; branch b uses seed b + 1 + seed_offset; keep receives the branches.
template <class BinaryProblemT, class ScheduleT>
std::vector<float> branch_fractions(const BinaryProblemT& p, const ScheduleT& s, int n_branches, unsigned n_threads,
                                    std::vector<std::vector<uint8_t>>* keep = nullptr, uint64_t seed_offset = 0) {
    (void)n_threads;
    const qb_residual_desc d = residual_desc(p);
    Problem prob;
    check(qb_problem_create_residual(&d, nullptr, &prob.h), "qb_problem_create_residual");
    const qb_schedule q = schedule_of(s);
    Result res;
    check(qb_solve(prob.h, &q, uint32_t(n_branches), seed_offset, nullptr, &res.h), "qb_solve");
    std::vector<float> frac(static_cast<size_t>(d.n_vars));
    check(qb_result_marginals(res.h, frac.data()), "qb_result_marginals");
    if (keep) {
        std::vector<uint8_t> X(size_t(n_branches) * size_t(d.n_vars));
        check(qb_result_branches(res.h, X.data()), "qb_result_branches");
        keep->assign(size_t(n_branches), std::vector<uint8_t>());
        for (int b = 0; b < n_branches; ++b)
            (*keep)[size_t(b)].assign(X.begin() + size_t(b) * size_t(d.n_vars), X.begin() + size_t(b + 1) * size_t(d.n_vars));
    }
    return frac;
}

// argos::anneal_branch: one branch with seed `seed`.
template <class BinaryProblemT, class ScheduleT>
std::vector<uint8_t> anneal_branch(const BinaryProblemT& p, const ScheduleT& s, uint64_t seed) {
    std::vector<std::vector<uint8_t>> keep;
    branch_fractions(p, s, 1, 1u, &keep, seed - 1);
    return keep[0];
}

template <class WeightedGraphT>
qb_ising_desc ising_desc(const WeightedGraphT& g) {
    require(g.m >= 0 && g.eu.size() == size_t(g.m) && g.ev.size() == size_t(g.m) && g.ew.size() == size_t(g.m),
            "eu, ev and ew need m entries each");
    qb_ising_desc d{};
    d.n = int32_t(g.n);
    d.m = int64_t(g.m);
    d.eu = g.eu.data();
    d.ev = g.ev.data();
    d.ew = g.ew.data();
    return d;
}

// wising::anneal: one replica with seed `seed`; RunOutT has members x
// (std::vector<uint8_t>) and energy_tracked (E = -cut, exact).
template <class RunOutT, class WeightedGraphT, class BudgetT>
RunOutT anneal(const WeightedGraphT& g, const BudgetT& b, uint64_t seed) {
    const qb_ising_desc d = ising_desc(g);
    Problem prob;
    check(qb_problem_create_ising(&d, nullptr, &prob.h), "qb_problem_create_ising");
    const qb_schedule q = schedule_of(b, 0);
    Result res;
    check(qb_solve(prob.h, &q, 1u, seed - 1, nullptr, &res.h), "qb_solve");
    RunOutT out;
    out.x.assign(size_t(d.n), 0);
    check(qb_result_branches(res.h, out.x.data()), "qb_result_branches");
    int64_t e = 0;
    check(qb_result_energies_i64(res.h, &e), "qb_result_energies_i64");
    out.energy_tracked = e;
    return out;
}

// gising::BatchOut's fields (ising_gpu.cuh:345-359): spins +-1 as R x n_pad
// int8 with n_pad = n here, tracked energies, timing; x(r) gives 0/1.
struct BatchOut {
    int R = 0, n = 0, n_pad = 0;
    std::vector<int8_t> s;
    std::vector<long long> energy;
    double wall_s = 0.0;
    double kernel_ms = 0.0;
    int launches = 0;
    int sweeps_per_launch = 0;
    std::vector<uint8_t> x(int r) const {
        std::vector<uint8_t> out(static_cast<size_t>(n));
        for (int i = 0; i < n; ++i) out[size_t(i)] = s[size_t(r) * size_t(n_pad) + size_t(i)] > 0 ? 1u : 0u;
        return out;
    }
};

// gising::run_batch: replicas with seeds seed_base .. seed_base + R - 1.
template <class WeightedGraphT, class BudgetT>
BatchOut run_batch(const WeightedGraphT& g, const BudgetT& b, uint64_t seed_base, int R) {
    const qb_ising_desc d = ising_desc(g);
    Problem prob;
    check(qb_problem_create_ising(&d, nullptr, &prob.h), "qb_problem_create_ising");
    const qb_schedule q = schedule_of(b, 0);
    Result res;
    check(qb_solve(prob.h, &q, uint32_t(R), seed_base - 1, nullptr, &res.h), "qb_solve");
    qb_result_info info{};
    check(qb_result_info_get(res.h, &info), "qb_result_info_get");
    BatchOut out;
    out.R = R;
    out.n = out.n_pad = d.n;
    std::vector<uint8_t> X(size_t(R) * size_t(d.n));
    check(qb_result_branches(res.h, X.data()), "qb_result_branches");
    out.s.resize(X.size());
    for (size_t k = 0; k < X.size(); ++k) out.s[k] = X[k] ? int8_t(1) : int8_t(-1);
    std::vector<int64_t> e(static_cast<size_t>(R));
    check(qb_result_energies_i64(res.h, e.data()), "qb_result_energies_i64");
    out.energy.assign(e.begin(), e.end());
    out.kernel_ms = info.anneal_ms;
    out.launches = info.launches;
    out.sweeps_per_launch = info.sweeps;
    return out;
}

// argos::classify (src/ising_recon.hpp:305-309): 1 NotThere, 0 Exists, 2 Undecided.
inline uint8_t classify(float p_void, float lo = 0.1f, float hi = 0.9f) {
    if (p_void >= hi) return 1;
    if (p_void <= lo) return 0;
    return 2;
}

}  // namespace compat
}  // namespace qublar
