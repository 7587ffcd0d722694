// Launchers of the weighted-QUBO sweep (qb_qubo.cu), called by the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "qb_internal.hpp"

namespace qb {

struct QuboBuffers {
    uint8_t* x = nullptr;                    // R x n, original order
    const double* temp = nullptr;
    float* drift = nullptr;                  // R
    double* e_track = nullptr;               // R (zeroed by the caller)
    unsigned long long* accepts = nullptr;   // R (zeroed by the caller)
    double* trace = nullptr;                 // R x sweeps per-sweep sums of accepted dE (zeroed), or null
    void* scratch = nullptr;                 // qubo_scratch bytes
};

// CTAs of the cooperative grid (0: the device cannot run it).
int qubo_lockstep_grid();
// Replicas one launch serves.
int qubo_max_branches();
// Scratch of one launch: a 64-byte control block (barrier counter, timeout
// flag at +16, which the caller zeroes once per solve), fields, bit words.
size_t qubo_scratch(const QuboPlan& p);
// ctas: the cooperative grid (0 = the whole device; fewer CTAs leave the rest
// of the device to other work; the branches do not depend on it).
qb_status launch_qubo_lockstep(const QuboPlan& p, const QuboBuffers& b, int R, int sweeps, int refresh, uint64_t seed0,
                               cudaStream_t st, int ctas = 0);
qb_status launch_qubo_energies(const QuboPlan& p, const uint8_t* x, int K, double* e, cudaStream_t st);

}  // namespace qb
