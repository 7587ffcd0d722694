// Drives include/qublar_adapter.hpp the way a QuBLAR caller would, with
// stand-in types that carry the reference's member names (BinaryProblem,
// Schedule, WeightedGraph, Budget, RunOut), so no reference header is needed;
// compiled with -DQB_REAL_TYPES against the reference's headers it uses the
// reference's own types instead (oracle/Makefile: oracle/_ref/adapter_real).
//
//   adapter_check <dir> cpu   -> a call without a device must throw cleanly
//   adapter_check <dir> gpu   -> branch_fractions / anneal / run_batch results
//                                are written to <dir> for the test to compare
//   adapter_check <dir> lengths -> problems whose vectors are shorter than
//                                their offsets say are refused by the adapter,
//                                before any call into the library
// <dir> holds the problem as raw little-endian arrays written by the test.
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "qublar_adapter.hpp"

#ifdef QB_REAL_TYPES
// Built by oracle/Makefile against the reference's own headers (include path
// into the reference tree): the adapter is driven with the real types.
#include "ising_recon.hpp"
#include "ising_weighted.hpp"
using argos::BinaryProblem;
using argos::Schedule;
using argos::wising::Budget;
using argos::wising::RunOut;
using argos::wising::WeightedGraph;
#else
struct BinaryProblem {   // the members of argos::BinaryProblem (src/engine.hpp:30-49)
    std::vector<int> var_voxel, voxel_var;
    std::vector<double> d, w;
    std::vector<int> row_ptr, ray;
    std::vector<float> a;
    std::vector<int> nbr_ptr, nbr;
    double lambda = 0.0, kappa = 0.0;
    std::vector<double> field;
};
struct Schedule {        // argos::Schedule (src/ising_recon.hpp:81-86)
    double t_hot = 50.0, t_cold = 1.0;
    int anneal_sweeps = 200, hold_sweeps = 50;
};
struct WeightedGraph {   // argos::wising::WeightedGraph (src/ising_weighted.hpp:35-42)
    int n = 0;
    int64_t m = 0;
    std::vector<int32_t> eu, ev, ew;
};
struct Budget {          // argos::wising::Budget (src/ising_weighted.hpp:227-232)
    double t_hot = 5.0, t_cold = 1e-3;
    int anneal_sweeps = 400, hold_sweeps = 20;
};
struct RunOut {          // argos::wising::RunOut (src/ising_weighted.hpp:245-248)
    std::vector<uint8_t> x;
    int64_t energy_tracked = 0;
};
#endif

template <class T>
static std::vector<T> load(const std::string& path) {
    std::ifstream f(path, std::ios::binary | std::ios::ate);
    const std::streamsize bytes = f.tellg();
    f.seekg(0);
    std::vector<T> v(size_t(bytes) / sizeof(T));
    f.read(reinterpret_cast<char*>(v.data()), bytes);
    return v;
}
template <class T>
static void save(const std::string& path, const std::vector<T>& v) {
    std::ofstream f(path, std::ios::binary);
    f.write(reinterpret_cast<const char*>(v.data()), std::streamsize(v.size() * sizeof(T)));
}

int main(int argc, char** argv) {
    if (argc < 3) return 2;
    const std::string dir = argv[1], mode = argv[2];
    BinaryProblem p;
    p.d = load<double>(dir + "/d.bin");
    p.w = load<double>(dir + "/w.bin");
    p.row_ptr = load<int>(dir + "/row_ptr.bin");
    p.ray = load<int>(dir + "/ray.bin");
    p.a = load<float>(dir + "/a.bin");
    p.nbr_ptr = load<int>(dir + "/nbr_ptr.bin");
    p.nbr = load<int>(dir + "/nbr.bin");
    const std::vector<double> prior = load<double>(dir + "/prior.bin");   // lambda, kappa
    p.lambda = prior[0];
    p.kappa = prior[1];
    p.var_voxel.resize(p.row_ptr.size() - 1);
    for (size_t i = 0; i < p.var_voxel.size(); ++i) p.var_voxel[i] = int(i);
    p.voxel_var = p.var_voxel;
    WeightedGraph g;
    g.eu = load<int32_t>(dir + "/eu.bin");
    g.ev = load<int32_t>(dir + "/ev.bin");
    g.ew = load<int32_t>(dir + "/ew.bin");
    g.m = int64_t(g.eu.size());
    g.n = load<int32_t>(dir + "/gn.bin")[0];
    Schedule s;
    s.anneal_sweeps = 40;
    s.hold_sweeps = 10;
    Budget b;
    b.anneal_sweeps = 100;
    b.hold_sweeps = 10;
    if (mode == "lengths") {
        int refused = 0, cases = 0;
        auto expect_refusal = [&](auto call) {
            ++cases;
            try {
                call();
            } catch (const std::runtime_error& e) {
                if (std::string(e.what()).rfind("qublar adapter: ", 0) == 0) ++refused;
            }
        };
        auto fractions = [&](const BinaryProblem& q) { return [&q, &s] { qublar::compat::branch_fractions(q, s, 1, 1u); }; };
        BinaryProblem q = p;
        q.nbr_ptr.back() = int(q.nbr.size()) + 1;
        expect_refusal(fractions(q));
        q = p;
        q.a.pop_back();
        expect_refusal(fractions(q));
        q = p;
        q.row_ptr.pop_back();
        expect_refusal(fractions(q));
        q = p;
        q.w.pop_back();
        expect_refusal(fractions(q));
        q = p;
        q.field.assign(2, 0.0);
        expect_refusal(fractions(q));
        WeightedGraph h = g;
        h.ew.pop_back();
        expect_refusal([&] { qublar::compat::anneal<RunOut>(h, b, 1); });
        h = g;
        h.m += 1;
        expect_refusal([&] { qublar::compat::run_batch(h, b, 1, 2); });
        std::printf("refused %d of %d\n", refused, cases);
        return refused == cases ? 0 : 1;
    }
    try {
        std::vector<std::vector<uint8_t>> keep;
        const std::vector<float> frac = qublar::compat::branch_fractions(p, s, 4, 16u, &keep, 5);
        std::vector<uint8_t> X;
        for (const auto& x : keep) X.insert(X.end(), x.begin(), x.end());
        const RunOut r = qublar::compat::anneal<RunOut>(g, b, 3);
        const qublar::compat::BatchOut bo = qublar::compat::run_batch(g, b, 1, 4);
        std::vector<uint8_t> BX;
        for (int k = 0; k < bo.R; ++k) {
            const auto x = bo.x(k);
            BX.insert(BX.end(), x.begin(), x.end());
        }
        if (mode == "cpu") {
            std::printf("unexpected success without a device\n");
            return 1;
        }
        save(dir + "/frac.bin", frac);
        save(dir + "/branches.bin", X);
        save(dir + "/anneal_x.bin", r.x);
        save(dir + "/anneal_e.bin", std::vector<int64_t>{r.energy_tracked});
        save(dir + "/batch_x.bin", BX);
        save(dir + "/batch_e.bin", std::vector<long long>(bo.energy.begin(), bo.energy.end()));
        std::printf("adapter ok\n");
        return 0;
    } catch (const std::exception& e) {
        std::printf("exception: %s\n", e.what());
        return mode == "cpu" ? 0 : 1;
    }
}
