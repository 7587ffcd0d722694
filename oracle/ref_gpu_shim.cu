// ref_gpu_shim.cu -- TEST INFRASTRUCTURE ONLY. A C interface over the
// reference's own GPU annealer, compiled unchanged from QuBLAR's sources for
// sm_100a (the include path points into the reference tree; nothing is
// copied): argos::gising::make_plan, DeviceGraph and run_batch
// (src/ising_gpu.cuh:74-101, 278-343, 396-458), the existing-kernel comparator
// for the integer configurations. Built by oracle/Makefile into
// oracle/_ref/libqbref_gpu.so, apart from the host-only libqbref.so; only GPU
// tests load it.
//
// The reference ends the process (exit 3) on any CUDA error
// (src/ising_gpu.cuh:44-52); this shim keeps that behaviour.
#include <cstdint>
#include <cstring>
#include <string>

#include "ising_gpu.cuh"

namespace gi = argos::gising;
namespace wi = argos::wising;

namespace {

struct RefGpuGraph {
    wi::WeightedGraph g;
    gi::Plan plan;
    gi::DeviceGraph* dg = nullptr;
};

void set_err(char* err, int errlen, const std::string& e) {
    if (err && errlen > 0) {
        std::strncpy(err, e.c_str(), size_t(errlen - 1));
        err[errlen - 1] = 0;
    }
}

}  // namespace

extern "C" {

// parse_rudy + make_plan + DeviceGraph (the stock path of tools/gpu_anneal.cu:136-137).
void* refgpu_graph_new(const char* text, size_t len, int force_global, char* err, int errlen) {
    auto* h = new RefGpuGraph();
    std::string e;
    if (!wi::parse_rudy(text, len, h->g, e)) {
        set_err(err, errlen, e);
        delete h;
        return nullptr;
    }
    h->plan = gi::make_plan(h->g, force_global != 0);
    if (!h->plan.refused.empty()) {
        set_err(err, errlen, h->plan.refused);
        delete h;
        return nullptr;
    }
    h->dg = new gi::DeviceGraph(h->g, h->plan);
    return h;
}

void refgpu_graph_free(void* p) {
    auto* h = static_cast<RefGpuGraph*>(p);
    if (!h) return;
    delete h->dg;
    delete h;
}

// The plan's storage choices: field bytes, weight bytes, dense, shared state.
void refgpu_plan(void* p, int* field_bytes, int* weight_bytes, int* dense, int* shared_state) {
    const auto* h = static_cast<RefGpuGraph*>(p);
    *field_bytes = h->plan.field_bytes;
    *weight_bytes = h->plan.weight_bytes;
    *dense = h->plan.dense ? 1 : 0;
    *shared_state = h->plan.shared_state ? 1 : 0;
}

// run_batch for seeds seed_base .. seed_base+R-1; X: R x n (0/1), E: R tracked
// energies. Returns the reference's wall time in seconds (launches, then the
// copies back); kernel_ms is its event time over the launches.
double refgpu_run_batch(void* p, double t_hot, double t_cold, int anneal, int hold, uint64_t seed_base, int R,
                        uint8_t* X, long long* E, double* kernel_ms, int* launches) {
    const auto* h = static_cast<RefGpuGraph*>(p);
    wi::Budget b;
    b.t_hot = t_hot;
    b.t_cold = t_cold;
    b.anneal_sweeps = anneal;
    b.hold_sweeps = hold;
    const gi::BatchOut o = gi::run_batch(*h->dg, b, seed_base, R);
    for (int r = 0; r < R; ++r) {
        if (X) {
            const std::vector<uint8_t> x = o.x(r);
            std::memcpy(X + size_t(r) * size_t(o.n), x.data(), size_t(o.n));
        }
        if (E) E[r] = o.energy[size_t(r)];
    }
    if (kernel_ms) *kernel_ms = o.kernel_ms;
    if (launches) *launches = o.launches;
    return o.wall_s;
}

}  // extern "C"
