// Launchers of the sm_100a kernels (qb_kernels.cu), called by the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "qb_internal.hpp"

namespace qb {

// Cluster size of the residual sweep: one cluster anneals one branch, its
// residuals spread over the cluster's shared memory.
constexpr int kResidClusterDefault = 8;

struct SolveBuffers {
    uint8_t* x = nullptr;        // R x n, original order
    int32_t* f = nullptr;        // R x n fields (ising)
    long long* e_i64 = nullptr;  // R
    double* e_f64 = nullptr;     // R
    float* p = nullptr;          // n
    const double* temp = nullptr;
    float* drift = nullptr;      // R
    unsigned long long* accepts = nullptr;   // R accepted flips (residual)
    double* trace = nullptr;     // R x sweeps per-sweep sums of accepted dE (zeroed), or null: no trace
    void* scratch = nullptr;     // ising: R x n x 5 bytes when the state does not fit on chip
};

// Dynamic shared memory of one CTA of the ising sweep, 0 when the state lives
// in global scratch.
size_t ising_smem_bytes(const IsingPlan& p);
qb_status launch_ising_anneal(const IsingPlan& p, const SolveBuffers& b, int R, int sweeps, uint64_t seed0,
                              cudaStream_t st);
qb_status launch_ising_energies(const IsingPlan& p, const uint8_t* x, int K, long long* e, cudaStream_t st);

size_t resid_smem_bytes(const ResidualPlan& p);
// Chunk limits of the residual sweep: bits, bit-ray entries, neighbour entries.
int resid_chunk_bits();
// Lanes that share one bit's sum in the residual sweep (its summation order):
// resid_group_lanes() for a bit with at most resid_heavy_entries() rays, a
// full warp (32) for a heavier bit.
int resid_group_lanes();
int resid_heavy_entries();
// Shared memory of the kernel's stage buffers (excluding residual slots and bits).
size_t resid_stage_bytes();
int resid_chunk_entries();
int resid_chunk_nbrs();
qb_status resid_check_fit(const ResidualPlan& p);
qb_status launch_resid_anneal(const ResidualPlan& p, const SolveBuffers& b, int R, int sweeps, int refresh,
                              uint64_t seed0, cudaStream_t st);
// All branches in lockstep on a cooperative grid: the grid size the device
// runs (0 when it cannot), the scratch a solve of R branches needs, the launch.
int resid_lockstep_grid();
int resid_lockstep_chunk_bits();
int resid_lockstep_chunk_entries();
int resid_lockstep_chunk_nbrs();
int resid_lockstep_chunk_segments();
int resid_lockstep_segment();        // entries per segment (the summation order)
int resid_lockstep_max_branches();   // branches one lockstep solve serves
size_t resid_lockstep_scratch(const ResidualPlan& p, int R);
// The scratch starts with a 64-byte control block: the barrier counter, then
// (at +16) the timeout flag, which the caller zeroes once per solve.
qb_status launch_resid_lockstep(const ResidualPlan& p, const SolveBuffers& b, int R, int sweeps, int refresh,
                                uint64_t seed0, cudaStream_t st);
qb_status launch_resid_energies(const ResidualPlan& p, const uint8_t* x, int K, double* e, cudaStream_t st);
qb_status launch_metropolis_check(const uint64_t* u53, const double* dE, const double* T, int n, uint8_t* fast,
                                  uint8_t* accept, uint8_t* exact, cudaStream_t st);

qb_status launch_marginals(const uint8_t* x, int R, int n, float* p, cudaStream_t st);
qb_status launch_tristate(const float* p, int n, float lo, float hi, uint8_t* out, cudaStream_t st);
qb_status launch_i64_to_f64(const long long* e, int R, double* out, cudaStream_t st);

}  // namespace qb
