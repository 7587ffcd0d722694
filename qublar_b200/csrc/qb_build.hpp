// Device assembly of a residual plan's O(nnz) tables (qb_build.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "qublar.h"

namespace qb {

// Longest ray whose segment the device sort holds in shared memory; a problem
// with a longer ray is assembled on the host.
constexpr int kRaySortMax = 4096;

struct ResidBuildArgs {
    int n;
    int n_rays;
    const int32_t* row_ptr;    // n + 1, input order
    const int32_t* ray;        // nnz, input order
    const float* a;            // nnz, input order
    const double* w;           // n_rays
    const int32_t* order;      // sweep position -> input bit
    const int32_t* inverse;    // input bit -> sweep position
    const int32_t* h_row;      // n + 1 sweep-order entry offsets
    const uint32_t* bit_home;  // sweep position -> home word (cluster sweep)
    uint2* ent;                // nnz sweep-order entries {ray | (w < 0) << 31, fp32(sqrt|w| a)}
    int32_t* rrow;             // n_rays + 1 ray-major offsets
    int32_t* rbit_o;           // nnz: input bit
    int32_t* rbit_n;           // nnz: sweep position
    uint32_t* rbit_h;          // nnz: home word
    float* ra;                 // nnz: a
    int32_t* rcount;           // scratch: n_rays
    int32_t* cursor;           // scratch: n_rays
    unsigned long long* rkey;  // scratch: nnz
};

size_t resid_sort_smem();
qb_status launch_resid_build(const ResidBuildArgs& A, cudaStream_t st);

}  // namespace qb
