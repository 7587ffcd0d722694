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
    void* scratch = nullptr;     // ising: R x n x 5 bytes when the state does not fit on chip
};

// Dynamic shared memory of one CTA of the ising sweep, 0 when the state lives
// in global scratch.
size_t ising_smem_bytes(const IsingPlan& p);
qb_status launch_ising_anneal(const IsingPlan& p, const SolveBuffers& b, int R, int sweeps, uint64_t seed0,
                              cudaStream_t st);
qb_status launch_ising_energies(const IsingPlan& p, const uint8_t* x, int K, long long* e, cudaStream_t st);

size_t resid_smem_bytes(const ResidualPlan& p);
qb_status resid_check_fit(const ResidualPlan& p);
qb_status launch_resid_anneal(const ResidualPlan& p, const SolveBuffers& b, int R, int sweeps, int refresh,
                              uint64_t seed0, cudaStream_t st);
qb_status launch_resid_energies(const ResidualPlan& p, const uint8_t* x, int K, double* e, cudaStream_t st);

qb_status launch_marginals(const uint8_t* x, int R, int n, float* p, cudaStream_t st);
qb_status launch_tristate(const float* p, int n, float lo, float hi, uint8_t* out, cudaStream_t st);
qb_status launch_i64_to_f64(const long long* e, int R, double* out, cudaStream_t st);

}  // namespace qb
