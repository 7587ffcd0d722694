// Internal host-side types of the B200 annealer: problem plans, device
// buffers, error plumbing. Nothing here crosses the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <exception>
#include <memory>
#include <new>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "qublar.h"

namespace qb {

// ---- errors ------------------------------------------------------------------

void set_error(const std::string& msg);
qb_status fail(qb_status s, const std::string& msg);

// Runs the body of a C ABI entry point: an exception (a failed host
// allocation above all, for sizes the caller chose) becomes a status instead
// of crossing the C ABI and ending the caller's process.
template <typename F>
qb_status guarded(const char* name, F&& body) noexcept {
    try {
        return body();
    } catch (const std::bad_alloc&) {
        return fail(QB_ENOMEM, std::string(name) + ": out of host memory");
    } catch (const std::exception& e) {
        return fail(QB_EINVAL, std::string(name) + ": " + e.what());
    } catch (...) {
        return fail(QB_EINVAL, std::string(name) + ": unexpected failure");
    }
}
qb_status cuda_fail(cudaError_t e, const char* what, const char* file, int line);

#define QB_CUDA(call)                                                              \
    do {                                                                           \
        cudaError_t e_ = (call);                                                   \
        if (e_ != cudaSuccess) return ::qb::cuda_fail(e_, #call, __FILE__, __LINE__); \
    } while (0)

// ---- device buffer (RAII, library-owned) -------------------------------------

// Allocations of a DevBuf are stream-ordered (from the library's pool on
// stream st, returned with cudaFreeAsync) while an AsyncAllocScope is open on
// the allocating thread: a server thread takes and returns request memory
// without the device-wide synchronisation of cudaMalloc/cudaFree, so work on
// other streams keeps running, and repeated problems reuse the pool's memory
// instead of mapping it afresh. free_on_legacy: the buffers are returned on the
// legacy default stream (for buffers that outlive the caller's stream; their
// owner synchronises the device first).
struct AsyncAllocScope {
    explicit AsyncAllocScope(cudaStream_t st, bool free_on_legacy = false);
    ~AsyncAllocScope();
    AsyncAllocScope(const AsyncAllocScope&) = delete;
    AsyncAllocScope& operator=(const AsyncAllocScope&) = delete;
    cudaStream_t prev;
    bool prev_on;
    bool prev_legacy;
};

// The library's stream-ordered memory pool of a device (created on first use;
// it keeps freed memory for reuse until qb_device_trim), or null if the device
// has none.
cudaMemPool_t library_pool(int dev);

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    bool pooled = false;              // from cudaMallocAsync: returned with cudaFreeAsync
    bool sync_free = false;           // returned on the legacy stream: its owner waits for the device first
    cudaStream_t pool_stream = nullptr;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    DevBuf(DevBuf&& o) noexcept
        : p(o.p), bytes(o.bytes), pooled(o.pooled), sync_free(o.sync_free), pool_stream(o.pool_stream) {
        o.p = nullptr;
        o.bytes = 0;
        o.pooled = false;
        o.sync_free = false;
    }
    DevBuf& operator=(DevBuf&& o) noexcept {
        if (this != &o) {
            release();
            p = o.p;
            bytes = o.bytes;
            pooled = o.pooled;
            sync_free = o.sync_free;
            pool_stream = o.pool_stream;
            o.p = nullptr;
            o.bytes = 0;
            o.pooled = false;
            o.sync_free = false;
        }
        return *this;
    }
    ~DevBuf() { release(); }
    void release() {
        if (p) {
            if (pooled) cudaFreeAsync(p, pool_stream);
            else cudaFree(p);
        }
        pooled = false;
        sync_free = false;
        p = nullptr;
        bytes = 0;
    }
    qb_status alloc(size_t n);
    template <typename T>
    T* as() const { return static_cast<T*>(p); }
};

qb_status upload(DevBuf& dst, const void* src, size_t bytes, cudaStream_t st);

template <typename T, typename A>
qb_status upload_vec(DevBuf& dst, const std::vector<T, A>& v, cudaStream_t st) {
    return upload(dst, v.data(), v.size() * sizeof(T), st);
}

// An allocator whose value-initialisation leaves elements uninitialised, for
// large host tables that a parallel loop fills right after sizing: the
// single-threaded zero fill is skipped and the filling threads touch the
// pages first.
template <typename T>
struct NoInitAlloc : std::allocator<T> {
    template <typename U>
    struct rebind {
        using other = NoInitAlloc<U>;
    };
    NoInitAlloc() = default;
    template <typename U>
    NoInitAlloc(const NoInitAlloc<U>&) noexcept {}
    template <typename U>
    void construct(U* p) noexcept(std::is_nothrow_default_constructible<U>::value) {
        ::new (static_cast<void*>(p)) U;
    }
    template <typename U, typename... Args>
    void construct(U* p, Args&&... args) {
        ::new (static_cast<void*>(p)) U(std::forward<Args>(args)...);
    }
};
template <typename T>
using RawVec = std::vector<T, NoInitAlloc<T>>;

// The residual sweeps' fp32 coefficient of a bit-ray entry: a' = fp32(sqrt|w| a),
// the fp64 product rounded once (the device's scaled_coef, qb_device.cuh).
inline float ray_coef(double w, float a) { return float(std::sqrt(std::fabs(w)) * double(a)); }

// The temperature of every sweep of a schedule (host, double).
std::vector<double> temperatures(const qb_schedule& s);

// ---- colouring ----------------------------------------------------------------

// A sweep order: bits grouped by colour class. order[k] is the original index
// of the k-th bit of the sweep; class c occupies order[class_ptr[c] ..
// class_ptr[c+1]). No two bits of one class interact.
struct Colouring {
    std::vector<int32_t> colour;      // per original bit
    std::vector<int32_t> order;       // new -> old
    std::vector<int32_t> inverse;     // old -> new
    std::vector<int32_t> class_ptr;   // n_colours + 1
    int n_colours() const { return int(class_ptr.size()) - 1; }
};

// Greedy first-fit distance-1 colouring of a symmetric graph given in CSR.
Colouring colour_graph(int n, const std::vector<int64_t>& row, const std::vector<int32_t>& col);

// Colouring of the residual conflict graph: bits conflict when they share a
// ray or are neighbours in the prior. Rays are cliques, handled with per-ray
// used-colour bitsets (no explicit conflict graph is built).
Colouring colour_residual(int n, int n_rays, int* max_ray_len, const int32_t* row_ptr, const int32_t* ray,
                          const int32_t* nbr_ptr, const int32_t* nbr);

void finish_colouring(Colouring& c, int n);

// True when no class holds two interacting bits (test hook).
bool colouring_valid_graph(const Colouring& c, const std::vector<int64_t>& row, const std::vector<int32_t>& col);

// ---- problems -----------------------------------------------------------------

struct IsingPlan {
    int n = 0;
    int64_t m = 0;
    int64_t nnz = 0;          // 2m
    int64_t B = 0;            // max_i sum_j |w_ij|
    int64_t max_w = 0;
    int64_t w_min = 0;
    double sigma = 0.0;
    int weight_bytes = 4;     // 1 (int8) or 4
    Colouring col;
    // host copies in sweep (new) order
    std::vector<int32_t> row;    // n + 1 (int32 offsets: nnz < 2^31 is required)
    std::vector<int32_t> adj;    // nnz, new indices
    std::vector<int32_t> wgt;    // nnz
    std::vector<int32_t> f0;     // fields of x = 0, new order
    // device
    DevBuf d_row, d_adj, d_w, d_f0, d_order, d_class_ptr;
    DevBuf d_eu, d_ev, d_ew;     // edge list as given (energy verifier)
};

struct ResidualPlan {
    int variant = 1;                  // QB_RESID_LOCKSTEP or QB_RESID_CLUSTER
    int lock_grid = 0;                // lockstep: CTAs of the cooperative grid (= slices per class)
    int n = 0;
    int n_rays = 0;
    int64_t nnz = 0;
    int64_t n_nbr = 0;
    double lambda = 0.0;
    double e0 = 0.0;                  // energy of x = 0: 1/2 sum_b w_b d_b^2 (fp64, ray order)
    Colouring col;
    // cluster decomposition of one branch: CL CTAs; ray b lives on CTA b % CL,
    // slot b / CL; bit k of class c belongs to CTA t = (k - class start) / chunk(c)
    int CL = 8;
    int ray_slots = 0;
    int bit_slots = 0;
    std::vector<int32_t> slot_base;   // n_colours * CL: first slot of (class, CTA)
    std::vector<uint32_t> bit_home;   // new bit -> (cta << 27) | slot
    // chunk table: CTA t works chunks [chunk_ptr[t], chunk_ptr[t+1]), each two
    // int4 {b0, b1, slot of b0, last chunk of its class} {e0, e1, n0, n1}
    // (bits, bit-ray entries and neighbour entries of the chunk, sweep order)
    std::vector<int32_t> chunks;
    std::vector<int32_t> chunk_ptr;
    std::vector<int32_t> h_nbr_new;   // neighbours as sweep-order indices
    std::vector<uint32_t> h_meta;     // lockstep: per bit 8 words {row start, rays, nbr start, nbrs, lin, q, index, 0}
    // host copies of the sweep-order arrays (h_ent is released after upload)
    std::vector<int32_t> h_row, h_nbr_ptr;
    int max_ray_len = 0;              // most bits on one ray
    std::vector<uint32_t> h_nbr_home;
    std::vector<float> h_lin, h_q;
    // device arrays in sweep order
    DevBuf d_row, d_ent, d_lin, d_q, d_nbr_ptr, d_nbr_home, d_order, d_class_ptr, d_chunks, d_chunk_ptr;
    DevBuf d_d, d_w64;                // per ray
    DevBuf d_rrow, d_rbit, d_ra;      // ray-major CSR for refresh (bit as home word)
    DevBuf d_meta, d_nbr_new, d_rbit_new;   // lockstep tables
    // energy verifier (original order)
    DevBuf d_o_row, d_o_ray, d_o_a, d_o_nbr_ptr, d_o_nbr, d_o_lin;
    DevBuf d_o_rbit;                  // ray-major bits in input order (offsets and a: d_rrow, d_ra)
};

// Weighted QUBO E(x) = offset + sum_i h_i x_i + sum_e J_e x_u x_v with fp32
// couplings and linear terms, planned for the compensated lockstep sweep.
struct QuboPlan {
    int n = 0;
    int64_t m = 0;
    int64_t nnz = 0;          // 2m
    double offset = 0.0;
    Colouring col;
    // sweep order: neighbours of the bit at position p are adj[row[p] ..
    // row[p+1]) as sweep positions, in the order of the symmetric CSR built
    // from the edge list (edge order per vertex)
    std::vector<int32_t> row, adj;
    std::vector<float> J, h;
    DevBuf d_row, d_adj, d_J, d_h, d_order, d_class_ptr;
    DevBuf d_eu, d_ev, d_ew, d_ho;   // edge list and h as given (fp64 evaluator)
};

// Host copies of a problem's input arrays, kept when its upload is deferred
// (QB_OPT_DEFER_UPLOAD) so that the problem can go to the device later.
struct HostDesc {
    std::vector<int32_t> eu, ev, ew;                       // ising (eu, ev also qubo)
    std::vector<float> wf, hf;                             // qubo couplings and linear terms
    double offset = 0.0;
    std::vector<double> d, w, field;                       // residual
    std::vector<int32_t> row_ptr, ray, nbr_ptr, nbr;
    std::vector<float> a;
    double lambda = 0.0, kappa = 0.0;
    bool has_field = false;
};

}  // namespace qb

struct qb_problem {
    int kind = 0;
    int device = 0;
    qb::IsingPlan ising;
    qb::ResidualPlan resid;
    qb::QuboPlan qubo;
    int64_t device_bytes = 0;     // device memory the problem holds (or will hold once uploaded)
    bool uploaded = false;
    qb::HostDesc host;            // filled while the upload is deferred
    // temperature table of the last schedule solved (reused while unchanged:
    // no pageable upload, hence no stream synchronisation, per solve)
    qb_schedule temp_sched{};
    qb::DevBuf d_temp;
};

namespace qb {
// Upload of a problem created with QB_OPT_DEFER_UPLOAD (no-op when already on
// the device), and the release of its device memory.
qb_status problem_upload(qb_problem* p, cudaStream_t st);
void problem_release_device(qb_problem* p);
// Plans a lockstep residual problem again for a cooperative grid of `slices`
// CTAs, from the host copies a deferred problem keeps (its device copy, if
// any, is released; the next upload follows the new plan). The colouring is
// the same, so the branches are too.
qb_status replan_residual(qb_problem* p, int slices);
}  // namespace qb

struct qb_result {
    qb_problem* prob = nullptr;
    int device = 0;
    cudaStream_t stream = nullptr;
    int n = 0;
    int R = 0;
    int sweeps = 0;
    int launches = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev2 = nullptr;   // start, anneal end, solve end
    qb::DevBuf d_x;          // R x n uint8, original order
    qb::DevBuf d_f;          // R x n int32 fields (ising), original order
    qb::DevBuf d_e_i64;      // R tracked energies (ising)
    qb::DevBuf d_e_scr;      // R energies from scratch over the edge list (ising)
    qb::DevBuf d_e_f64;      // R energies from scratch
    qb::DevBuf d_p;          // n marginals
    qb::DevBuf d_temp;       // sweeps temperatures
    qb::DevBuf d_drift;      // R floats
    qb::DevBuf d_accepts;    // R accepted-flip counts (residual, qubo)
    qb::DevBuf d_e_track;    // R tracked energies minus offset (qubo)
    qb::DevBuf d_scratch;    // per-branch state that does not fit on chip
    qb::DevBuf d_trace;      // R x sweeps: ising int64 tracked energies; residual, qubo fp64 per-sweep dE sums
    double trace_base = 0.0; // residual: energy of x = 0; qubo: the offset
    const int* d_err = nullptr;   // timeout flag of a cooperative sweep (inside d_scratch), or null
    qb_batch* packed = nullptr;   // many replicas solved by the packed kernel: its launch tables
    bool synced = false;
};
