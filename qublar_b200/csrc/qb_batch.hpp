// Packed integer Ising work: many instances and replica groups of uneven size
// in one persistent launch (the batched form of qb_solve on ising problems).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "qb_internal.hpp"

namespace qb {

// One unit of work: G = 2^log2g replicas of one instance over sweeps
// [sweep0, sweep1). Its state is laid out bit-major with the replica fastest
// (f[i * G + r], s[i * G + r]) so the lanes of a warp are the replicas of one
// bit, or G-wide groups of consecutive bits.
struct IsingItem {
    const int32_t* class_ptr;   // n_colours + 1
    const int32_t* row;         // sweep-order CSR
    const int32_t* adj;
    const void* w;              // int8 or int32 per wbytes
    const int32_t* f0;          // fields of x = 0
    const int32_t* order;       // sweep position -> original bit
    const double* temp;         // temperature of every sweep of the schedule
    int32_t* f_state;           // n x G: where the state lives (kItemGlobal) or is kept between slices
    int8_t* s_state;
    long long* e_acc;           // G tracked energies, accumulated over slices
    uint8_t* x_out;             // G x n, original order (kItemFinal)
    int32_t* f_out;             // G x n
    uint64_t seed0;             // seed of the item's first replica
    int32_t n;
    int32_t n_colours;
    int32_t log2g;
    int32_t sweep0;
    int32_t sweep1;
    int32_t flags;
    int32_t bound;              // max_i sum_j |w_ij|: |dE| <= bound
    int32_t wbytes;             // 1 or 4
};

constexpr int kItemInit = 1;     // start from x = 0 (s = -1, f = f0, E = 0)
constexpr int kItemGlobal = 2;   // the state stays in f_state/s_state (too large for shared memory)
constexpr int kItemFinal = 4;    // write x_out, f_out at the end
constexpr int kItemKeep = 8;     // write the shared-memory state back to f_state/s_state at the end
// bit 8 of flags: the parity of the item's first replica r0 (its replicas'
// Philox key pairing, ising_pair_key); seed0 is the solve's base + r0
constexpr int kItemOddBase = 1 << 8;
inline int item_rbase_flags(int r0) { return (r0 & 1) ? kItemOddBase : 0; }

constexpr int kBatchMaxGroup = 32;

// Launch shape of the packed kernel.
struct BatchShape {
    int threads = 512;
    int smem_bytes = 0;    // dynamic shared memory per CTA (state of one item)
    int ctas = 0;          // persistent CTAs (0: as many as fit)
};

// Shared memory one item of n bits and G replicas needs.
inline size_t batch_item_smem(int n, int G) { return size_t(n) * size_t(G) * 5; }

// Largest dynamic shared memory a CTA of the packed kernel can take.
int batch_max_smem();
// Persistent CTAs that fit the device at this shape.
qb_status batch_ctas(const BatchShape& sh, int* ctas);
// Runs items [0, n_items) on `ctas` persistent CTAs; counter is one device int
// the launch uses to hand out items (zeroed on the stream first).
qb_status launch_ising_batch(const IsingItem* d_items, int n_items, int* d_counter, const BatchShape& sh,
                             cudaStream_t st);

// The same kernel with its item count in device memory: ctl[0] must be 0 and
// ctl[1] the item count when it starts (a launch a graph can replay).
// sh.ctas must be set; the shared-memory attribute must have been set by
// batch_ctas for this shape.
qb_status launch_ising_batch_ctl(const IsingItem* d_items, int* d_ctl, const BatchShape& sh, cudaStream_t st);

// Where one instance's outputs sit in the batch arenas.
struct BatchInstDev {
    int64_t x_off;   // first byte of its R x n branches
    int64_t p_off;   // first entry of its n marginals (the sum of the n before it)
    int32_t n;
    int32_t R;
};
qb_status launch_batch_marginals(const uint8_t* x, const BatchInstDev* inst, int n_inst, int64_t total, float* p,
                                 cudaStream_t st);

// qb_solve of many replicas of one ising problem through the packed kernel:
// groups of G replicas (G the smallest power of two that keeps the groups
// within the CTAs the device runs at once), each group a work item. The
// branches, fields, tracked energies and marginals are those of the
// CTA-per-replica sweep (the packed kernel's draws and arithmetic are the
// same); the arenas are handed over in x, f, e, pm and the batch, which holds
// the launch's tables, in *keep (destroy it after the stream's work).
qb_status packed_replicas(qb_problem* p, const qb_schedule& s, int R, uint64_t seed_offset, const qb_opts* opts,
                          qb_batch** keep, DevBuf& x, DevBuf& f, DevBuf& e, DevBuf& pm);
// Whether packed_replicas serves R replicas of this plan (asked for with
// QB_PACKED_REPLICAS=1, R >= 128, and a group's state fits a CTA's shared
// memory).
bool packed_replicas_fit(const IsingPlan& P, int R);

}  // namespace qb
