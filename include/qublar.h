/*
 * qublar.h -- C ABI of the B200 simulated-annealing QUBO/Ising solver.
 *
 * The boundary replaces the annealing path of QuBLAR:
 *   - argos::wising::WeightedGraph / anneal / cut_of / energy_scratch
 *       (src/ising_weighted.hpp:35-42, :173-189, :250-267)
 *   - argos::gising::make_plan / scaled_budget / run_batch / device_energies
 *       (src/ising_gpu.cuh:74-111, :396-458, :461-475)
 *   - argos::BinaryProblem / Schedule / binary_energy / anneal_branch /
 *     branch_fractions / classify
 *       (src/engine.hpp:30-49, src/ising_recon.hpp:65-166, :302-309)
 *
 * A QUBO goes in (integer Max-Cut graph or residual-form BinaryProblem),
 * annealed branches, exact energies, per-bit void fractions and the tri-state
 * map come out. Plain pointers and sizes only; the library owns device memory,
 * the caller owns host buffers, and no call throws or exits: every failure is
 * a qb_status with a thread-local message (qb_last_error).
 *
 * Differences from the reference that a caller can observe, by design:
 *   - sweeps visit the bits in colour-class order (a greedy distance-1
 *     colouring of the conflict graph), not in index order;
 *   - the Metropolis draw of (branch, bit, sweep) is Philox4x32-10 keyed by the
 *     branch seed, not the reference's sequential splitmix64 stream; two
 *     branches share a key and take one half of each Philox block each
 *     (integer Ising: branches 2k and 2k + 1; weighted QUBO: branches r and
 *     r + 32 of every 64).
 * Energies and fields of any returned configuration are exact (integer) or
 * fp64 from scratch; trajectories agree with the reference statistically.
 */
#ifndef QUBLAR_H
#define QUBLAR_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define QUBLAR_ABI_VERSION 1

/* Status codes. The reference exits the process on a CUDA error
 * (GISING_CUDA, src/ising_gpu.cuh:44-52) and refuses plans through a string
 * (Plan::refused, src/ising_gpu.cuh:93-94); both become codes here. */
typedef enum qb_status {
    QB_OK = 0,
    QB_EINVAL = 1,      /* malformed input (the refusals of parse_rudy, ising_weighted.hpp:89-123) */
    QB_ENOMEM = 2,      /* allocation failed or the request exceeds the device budget */
    QB_EREFUSED = 3,    /* the planner refuses the instance (field bound, all-zero weights, size) */
    QB_ETIMEDOUT = 4,   /* a bounded wait ran out */
    QB_ECUDA = 5,       /* a CUDA runtime error; qb_last_error names the call */
    QB_ENOTSUP = 6,     /* a request this build does not serve */
    QB_ECANCELLED = 7,  /* a served request was cancelled */
    QB_EBUSY = 8        /* the result is not ready yet */
} qb_status;

/* Problem kinds reported by qb_problem_info_get. */
#define QB_KIND_ISING 1     /* integer-weighted Max-Cut / Ising, E = -cut */
#define QB_KIND_RESIDUAL 2  /* residual-form QUBO (rays + 6-neighbour prior) */
#define QB_KIND_QUBO 3      /* weighted QUBO with fp32 couplings and linear terms */

/* Text of a status code (static storage). */
const char* qb_status_string(qb_status s);
/* Detail of the last failure on this host thread (thread-local storage). */
const char* qb_last_error(void);
/* QUBLAR_ABI_VERSION of the loaded library. */
int32_t qb_abi_version(void);
/* Number of CUDA devices visible, or -1 with qb_last_error set. */
int32_t qb_device_count(void);

typedef struct qb_problem qb_problem;
typedef struct qb_result qb_result;

/* Integer-weighted graph; replaces argos::wising::WeightedGraph
 * (src/ising_weighted.hpp:35-42). Edges are 0-based (u, v, w), u != v, no
 * duplicates in either orientation, w in int32. E(x) = -sum_e w_e [x_u != x_v]. */
typedef struct qb_ising_desc {
    int32_t n;
    int64_t m;
    const int32_t* eu;
    const int32_t* ev;
    const int32_t* ew;
} qb_ising_desc;

/* A graph read from rudy / G-set text: the input format of the reference's
 * integer engine. qb_parse_rudy replaces parse_rudy
 * (src/ising_weighted.hpp:83-149): header "n m", then m lines "u v [w]",
 * 1-based, w = +1 when absent; it refuses what parse_rudy refuses, with the
 * same reason in qb_last_error (bad header, a token that is not an integer, a
 * weight outside int32, a trailing token, a vertex out of range, a self-loop,
 * an edge count that differs from the header, a duplicate edge).
 * qb_graph_desc points a descriptor at the graph's arrays (valid until
 * qb_graph_destroy) for qb_problem_create_ising. Host only. */
typedef struct qb_graph qb_graph;
qb_status qb_parse_rudy(const char* text, size_t size, qb_graph** out);
qb_status qb_graph_desc(const qb_graph* g, qb_ising_desc* desc);
void qb_graph_destroy(qb_graph* g);

/* Residual-form QUBO; replaces argos::BinaryProblem (src/engine.hpp:30-49):
 *   E(x) = 1/2 sum_b w_b (sum_v a_bv x_v - d_b)^2
 *        + lambda sum_<uv> [x_u != x_v] + sum_v lin_v x_v,
 * lin_v = field[v] when field != NULL, else kappa (BinaryProblem::lin). The
 * bit->ray CSR (row_ptr, ray, a) and the symmetric neighbour CSR (nbr_ptr, nbr)
 * use int32 offsets like the reference. */
typedef struct qb_residual_desc {
    int32_t n_vars;
    int32_t n_rays;
    const double* d;        /* n_rays */
    const double* w;        /* n_rays */
    const int32_t* row_ptr; /* n_vars + 1 */
    const int32_t* ray;     /* row_ptr[n_vars] */
    const float* a;         /* row_ptr[n_vars] */
    const int32_t* nbr_ptr; /* n_vars + 1 */
    const int32_t* nbr;     /* nbr_ptr[n_vars] */
    double lambda;
    double kappa;
    const double* field;    /* n_vars, or NULL */
} qb_residual_desc;

/* Weighted QUBO with real couplings, x in {0,1}:
 *   E(x) = offset + sum_i h_i x_i + sum_e J_e x_{u_e} x_{v_e},
 * the Model of src/check_ree_qubo.cu (offset, Qd, Qo; evaluated by
 * qubo_energy, :158-163), which the reference anneals only through its
 * pair-ray encoding into a BinaryProblem (to_engine, :172-192). Couplings and
 * linear terms are fp32; edges are 0-based, u != v, no duplicates in either
 * orientation; h may be NULL (all zero). */
typedef struct qb_qubo_desc {
    int32_t n;
    int64_t m;
    const int32_t* eu;
    const int32_t* ev;
    const float* ew;
    const float* h;
    double offset;
} qb_qubo_desc;

/* Geometric schedule: T(s) = t_hot (t_cold/t_hot)^min(1, s/max(1, A-1)) for
 * s < A, then t_cold for `hold_sweeps` more sweeps -- the expression of
 * ising_recon.hpp:129-131 and ising_weighted.hpp:255-257. Replaces
 * argos::Schedule (ising_recon.hpp:81-86) and wising::Budget (:227-232).
 * refresh_sweeps: residual instances recompute their fp32 residuals from
 * scratch in fp64 every this many sweeps (0 = at the start only); weighted
 * QUBO instances recompute their compensated fp32 local fields in fp64 every
 * this many sweeps (0 = never). */
typedef struct qb_schedule {
    double t_hot;
    double t_cold;
    int32_t anneal_sweeps;
    int32_t hold_sweeps;
    int32_t refresh_sweeps;
} qb_schedule;

/* Per-call options. stream: a cudaStream_t (NULL = the legacy default
 * stream); device: CUDA ordinal (-1 = current); flags: QB_OPT_* below. */
typedef struct qb_opts {
    void* stream;
    int32_t device;
    uint32_t flags;
} qb_opts;

/* qb_opts.flags of qb_problem_create_*:
 *   QB_OPT_DEFER_UPLOAD  plan on the host now, copy the inputs, and take
 *                        device memory only when the problem is first solved
 *                        or admitted by a server (qb_problem_info.device_bytes
 *                        reports what it will take); the host copies stay, so
 *                        a server can release the device copy when a request
 *                        finishes and the problem can be submitted again;
 *   QB_OPT_RESID_CLUSTER plan a residual problem for the cluster sweep (one
 *                        thread-block cluster per branch, which runs beside
 *                        other kernels) instead of the whole-device lockstep
 *                        sweep. */
#define QB_OPT_DEFER_UPLOAD 1u
#define QB_OPT_RESID_CLUSTER 2u
/* qb_opts.flags of qb_solve: QB_OPT_TRACE records every branch's energy after
 * every sweep (qb_result_energy_trace). */
#define QB_OPT_TRACE 4u

/* Upload an integer graph and plan it (colouring, field width).
 * Replaces gising::make_plan + DeviceGraph (src/ising_gpu.cuh:74-101, :278-336). */
qb_status qb_problem_create_ising(const qb_ising_desc* desc, const qb_opts* opts, qb_problem** out);
/* Upload a residual-form problem and plan it (conflict colouring of bits that
 * share a ray or a neighbour bond). Replaces passing a BinaryProblem to
 * branch_fractions (src/ising_recon.hpp:148). */
qb_status qb_problem_create_residual(const qb_residual_desc* desc, const qb_opts* opts, qb_problem** out);
/* Plan a weighted QUBO for the compensated-field sweep: all replicas of a
 * launch (up to 64) in lockstep on a cooperative grid, local fields carried
 * as fp32 hi + lo sums, refreshed in fp64 every schedule.refresh_sweeps.
 * Replaces annealing the pair-ray encoding of the Model through
 * anneal_branch (src/check_ree_qubo.cu:172-192, src/ising_recon.hpp:121-144). */
qb_status qb_problem_create_qubo(const qb_qubo_desc* desc, const qb_opts* opts, qb_problem** out);
void qb_problem_destroy(qb_problem* p);

/* The device memory of problems and solves comes from a stream-ordered pool
 * the library keeps per device: destroyed problems and results return their
 * buffers to it, and later ones reuse them without mapping memory afresh
 * (qb_problem_destroy waits for the device before it returns them). This call
 * waits for `device` and hands the memory the pool holds back to the driver. */
qb_status qb_device_trim(int32_t device);

typedef struct qb_problem_info {
    int32_t kind;           /* QB_KIND_* */
    int32_t n;              /* bits */
    int64_t nnz;            /* directed couplings (ising) or bit-ray entries (residual) */
    int32_t n_rays;         /* residual only */
    int32_t n_colours;      /* colour classes of the sweep */
    int32_t max_class;      /* largest class */
    int32_t field_bytes;    /* ising: 4 (int32 fields) */
    int32_t weight_bytes;   /* ising: 1 or 4 */
    int64_t device_bytes;   /* device memory held by the problem */
    double sigma;           /* ising: sqrt(2 sum w^2 / n) (ising_gpu.cuh:99) */
    double w_min;           /* ising: min |w| over w != 0 */
    int64_t field_bound;    /* ising: max_i sum_j |w_ij| (ising_gpu.cuh:87-92) */
    int32_t variant;        /* residual: QB_RESID_LOCKSTEP or QB_RESID_CLUSTER */
} qb_problem_info;

/* Residual sweep variants (qb_problem_info.variant). LOCKSTEP: every branch
 * on one cooperative grid, residuals in L2, a bounded grid barrier per colour
 * class; a bit's sum is the even-entry fmaf chain plus the odd-entry chain.
 * CLUSTER: one thread-block cluster per branch, residuals in distributed
 * shared memory; a bit's sum is 8 (or, above 64 rays, 32) lane-strided fmaf
 * chains joined by an xor butterfly. */
#define QB_RESID_LOCKSTEP 1
#define QB_RESID_CLUSTER 2
qb_status qb_problem_info_get(const qb_problem* p, qb_problem_info* info);

/* The sweep order of the plan: order[k] is the bit (input index) visited k-th
 * in a sweep, class c is order[class_ptr[c] .. class_ptr[c+1]). Either output
 * may be NULL; *n_colours receives the class count. */
qb_status qb_problem_colouring(const qb_problem* p, int32_t* order, int32_t* class_ptr, int32_t* n_colours);

/* Plan only, on the host (no device is touched): the colour-class sweep order
 * qb_problem_create_* would use for this input. order: n entries; class_ptr:
 * room for n + 1 entries (the first n_colours + 1 are written). Validates the
 * input like the create calls. */
qb_status qb_colour_ising(const qb_ising_desc* desc, int32_t* order, int32_t* class_ptr, int32_t* n_colours);
qb_status qb_colour_residual(const qb_residual_desc* desc, int32_t* order, int32_t* class_ptr, int32_t* n_colours);

/* T_hot = sigma, T_cold = 0.1 w_min: the reference's scaled budget
 * (gising::scaled_budget, src/ising_gpu.cuh:104-111). Ising problems only. */
qb_status qb_schedule_scaled(const qb_problem* p, int32_t anneal_sweeps, int32_t hold_sweeps, qb_schedule* out);

/* Anneal n_branches branches; branch b uses seed b + 1 + seed_offset, the
 * reference's convention (ising_recon.hpp:157, gpu_anneal.cu:143), except
 * that the branches sharing a Philox key (above) use the seed of the first of
 * them: integer-Ising branch b draws words 1:0 (b even) or 3:2 (b odd) of the
 * block of seed (b & ~1) + 1 + seed_offset. Every
 * branch starts from x = 0. The kernels are queued on opts->stream; the call
 * returns without waiting for them. Replaces anneal_branch /
 * branch_fractions (ising_recon.hpp:121-166), wising::anneal
 * (ising_weighted.hpp:250) and gising::run_batch (ising_gpu.cuh:396). */
qb_status qb_solve(qb_problem* p, const qb_schedule* s, uint32_t n_branches, uint64_t seed_offset,
                   const qb_opts* opts, qb_result** out);

typedef struct qb_result_info {
    int32_t n;
    int32_t n_branches;
    int32_t sweeps;
    int32_t launches;       /* kernels this solve launched */
    float anneal_ms;        /* CUDA-event time of the anneal kernels (on the solve's stream) */
    float total_ms;         /* CUDA-event time of the whole solve */
    int64_t attempts;       /* n_branches * sweeps * n */
    double max_drift;       /* residual: max |fp32 residual - fp64 residual| seen at refreshes;
                               qubo: max |compensated fp32 field - fp64 field| seen at refreshes */
    int64_t accepted;       /* residual, qubo: accepted flips over all branches and sweeps */
    double max_energy_error;   /* qubo: max over branches of |offset + sum of accepted dE - fp64 energy from scratch| */
} qb_result_info;
/* Waits for the solve. */
qb_status qb_result_info_get(qb_result* r, qb_result_info* info);
/* Branches as 0/1 bytes, n_branches x n, bit order of the input. Waits. */
qb_status qb_result_branches(qb_result* r, uint8_t* x);
/* Ising: tracked energies E = -cut of every branch (RunOut::energy_tracked). */
qb_status qb_result_energies_i64(qb_result* r, int64_t* e);
/* Ising: maintained local fields f_i = sum_j w_ij s_j, n_branches x n (wising::State::f). */
qb_status qb_result_fields_i64(qb_result* r, int64_t* f);
/* Energies from scratch in fp64 (binary_energy for residual problems, -cut for ising). */
qb_status qb_result_energies_f64(qb_result* r, double* e);
/* Per-bit fraction of branches with x = 1 (branch_fractions, ising_recon.hpp:160-163). */
qb_status qb_result_marginals(qb_result* r, float* p);
/* The energy of every branch after every sweep, n_branches x sweeps, for a
 * solve made with QB_OPT_TRACE: the per-sweep energy the reference's
 * instrumented annealers record (check_ree_qubo.cu:195-216 anneal_trace; the
 * tracked State::energy of ising_weighted.hpp:209-217). Ising: the exact
 * tracked integer energy. Residual: the fp64 energy of x = 0 plus the
 * accepted fp32 dE summed in fp64 (the sum's order across CTAs is not fixed,
 * so the last bits may vary from run to run). QUBO: offset plus the accepted
 * dE summed in fp64 in a fixed order. */
qb_status qb_result_energy_trace(qb_result* r, double* trace);
/* Tri-state per bit: 1 = NotThere (p >= hi), 0 = Exists (p <= lo), 2 = Undecided
 * (argos::classify, ising_recon.hpp:302-309; defaults lo = 0.1, hi = 0.9). */
qb_status qb_result_tristate(qb_result* r, float lo, float hi, uint8_t* bits);
void qb_result_destroy(qb_result* r);

/* Size of the static device scratch of qb_solve_residual_noalloc: held by
 * every GPU that loads the library, from its first use until the process
 * exits (16 MiB: the 306,328-bit, 75,594-ray pyramid at 16 branches needs
 * about 11 MB). */
#define QB_NOALLOC_SCRATCH_BYTES (16u << 20)

/* A residual solve that allocates nothing, for callers that must not call
 * cudaMalloc/cudaFree while they run: a host that owns all device memory
 * through its own pool, a plugin host that forbids allocation calls (they
 * synchronise the device), a loop that allocated everything at start-up.
 * This entry point has no counterpart in the reference. It runs the lockstep
 * sweep of qb_solve for one block of at most 64 branches and writes the
 * branches (n_branches x n bytes, 0/1, input bit order) into x_out, a device
 * buffer the caller owns; the branches equal qb_solve's for the same
 * arguments. status is a device int32 the caller owns: the call sets it to
 * QB_OK on `stream`, and the sweep sets it to QB_ETIMEDOUT when one of its
 * bounded grid barriers gives up, in which case x_out is not written; read it
 * after the stream's work is done. Its per-solve scratch lives in one static
 * device array of QB_NOALLOC_SCRATCH_BYTES; problems that need more return
 * QB_ENOMEM with the size. The first call on a device looks up that array's
 * device address; make it before any stream capture. Calls share the array:
 * calls whose work overlaps on the GPU race, so serialise them. The problem
 * must come from qb_problem_create_residual with the lockstep plan
 * (qb_problem_info.variant == QB_RESID_LOCKSTEP). Returns once the work is
 * queued on `stream` (cudaStream_t, NULL = legacy default stream). */
qb_status qb_solve_residual_noalloc(const qb_problem* p, const qb_schedule* s, uint32_t n_branches,
                                    uint64_t seed_offset, uint8_t* x_out, int32_t* status, void* stream);

/* Diagnostics: the sweeps' Metropolis test of n uphill moves, run on `device`.
 * Move k draws u53[k] (53 bits) against dE[k] > 0 at temperature T[k]; dE is
 * rounded to fp32 as the sweeps hold it. fast[k] = the fp32 verdict (1
 * accept, 0 reject, 255 left to fp64), accept[k] = the sweeps' outcome,
 * exact[k] = the plain fp64 test u53 * 2^-53 < exp(-dE / T); accept always
 * equals exact. Host arrays of n entries; synchronous. */
qb_status qb_metropolis_check(const uint64_t* u53, const double* dE, const double* T, int32_t n, int32_t device,
                              uint8_t* fast, uint8_t* accept, uint8_t* exact);

/* ---- batches: many ising instances in one persistent launch ----------------
 *
 * The reference anneals one instance per launch (gising::run_batch,
 * src/ising_gpu.cuh:396-458, driven per graph by tools/gpu_anneal.cu:139).
 * qb_solve_batch packs many ising problems of uneven size, each with its own
 * schedule, branch count and seeds, into work items (one instance x a group
 * of replicas) that one persistent kernel drains largest first. Every branch
 * is identical to what qb_solve returns for its problem with the same
 * schedule and seeds, whatever the batch holds and whatever the launch shape. */
typedef struct qb_batch qb_batch;

typedef struct qb_batch_item {
    qb_problem* problem;     /* an ising problem (qb_problem_create_ising), on the batch's device */
    qb_schedule schedule;    /* this instance's schedule */
    uint32_t n_branches;     /* branch b uses seed b + 1 + seed_offset */
    uint64_t seed_offset;
} qb_batch_item;

/* Launch shape of the packed kernel; zeros take the defaults (512 threads,
 * 96 KiB of state per CTA, groups of up to 32 replicas). */
typedef struct qb_batch_config {
    int32_t threads;         /* per CTA: a multiple of 32 in [32, 1024] */
    int32_t smem_bytes;      /* shared memory for one item's state (n x group x 5 bytes) */
    int32_t max_group;       /* replicas per work item: a power of two in [1, 32] */
    int32_t ctas;            /* persistent CTAs; 0 = as many as fit the device */
} qb_batch_config;

/* Times candidate shapes on the batch itself with its schedules sampled at
 * sample_sweeps evenly spaced sweeps (0 = 8), times the three fastest again
 * on a sample four times longer, and returns the fastest of those. The
 * answer is kept per process for batches of the same shape (instance count,
 * total bits, total edges, total branches) and returned at once next time.
 * Results do not depend on the shape. */
qb_status qb_batch_autotune(const qb_batch_item* items, int32_t count, int32_t sample_sweeps, const qb_opts* opts,
                            qb_batch_config* out);

/* Queues the packed anneal on opts->stream and returns. cfg may be NULL. */
qb_status qb_solve_batch(const qb_batch_item* items, int32_t count, const qb_batch_config* cfg, const qb_opts* opts,
                         qb_batch** out);

typedef struct qb_batch_info {
    int32_t items;           /* instances */
    int32_t work_items;      /* instance x replica-group units */
    int32_t global_items;    /* units whose state did not fit shared memory */
    int32_t threads;
    int32_t smem_bytes;
    int32_t max_group;
    int32_t ctas;
    int32_t launches;        /* kernels the batch launched */
    int64_t attempts;        /* sum over instances of branches x sweeps x n */
    float anneal_ms;         /* CUDA-event time of the packed anneal */
    float total_ms;          /* ... of the whole batch (anneal + marginals) */
} qb_batch_info;
/* Waits for the batch. */
qb_status qb_batch_info_get(qb_batch* b, qb_batch_info* info);
/* Instance `item`'s branches (n_branches x n, 0/1, input bit order). Waits. */
qb_status qb_batch_branches(qb_batch* b, int32_t item, uint8_t* x);
/* Instance `item`'s tracked energies E = -cut (n_branches). */
qb_status qb_batch_energies_i64(qb_batch* b, int32_t item, int64_t* e);
/* Instance `item`'s maintained fields (n_branches x n). */
qb_status qb_batch_fields_i64(qb_batch* b, int32_t item, int64_t* f);
/* Instance `item`'s per-bit fraction of branches with x = 1. */
qb_status qb_batch_marginals(qb_batch* b, int32_t item, float* p);
void qb_batch_destroy(qb_batch* b);

/* ---- serving: a persistent request loop with continuous batching ----------
 *
 * The reference has no server: each solve is a blocking call on stream 0
 * (gising::run_batch, src/ising_gpu.cuh:396-458; branch_fractions,
 * src/ising_recon.hpp:148-166). A qb_server owns one device and a worker
 * thread. Requests (a problem, a schedule, branches, a seed offset) are
 * admitted in arrival order while the device-memory budget and the active
 * limit allow; a problem created with QB_OPT_DEFER_UPLOAD goes to the device
 * only then, and leaves it when its request finishes.
 *   - ising requests advance together in ticks: one launch of the packed
 *     kernel (replayed from a CUDA graph) moves every admitted request forward
 *     by a slice of its sweeps, its spins and fields staying on the device in
 *     between; a request admitted while a tick runs joins the next tick;
 *   - residual requests (planned with QB_OPT_RESID_CLUSTER) run as one
 *     cluster launch each on a pool of streams, beside the ticks;
 *   - lockstep residual and weighted QUBO requests run as cooperative grids
 *     sized to their problems (enough CTAs for about one round of work per
 *     colour class, at most half the device), several side by side and beside
 *     the ticks; a deferred lockstep residual problem is planned again for
 *     its grid when it is submitted (the same colouring and branches), one
 *     without a host copy runs alone on the whole device.
 * A request's branches equal those of qb_solve on its own with the same
 * schedule and seeds, whatever else the server runs. All calls are
 * thread-safe. */
typedef struct qb_server qb_server;

typedef struct qb_server_config {
    int32_t device;              /* CUDA ordinal (-1 = current) */
    int64_t hbm_budget_bytes;    /* admission budget: problems + working memory + unreleased results (0 = 150 GB,
                                    capped at 90% of the free memory at creation) */
    int32_t max_active;          /* requests on the device at once (0 = 4096) */
    int32_t residual_streams;    /* streams for residual requests (0 = 8) */
    int32_t tick_target_us;      /* ising slices are sized so a tick item takes about this long (0 = 20000) */
    int32_t use_graph;           /* 0: launch ticks directly; otherwise replay a captured CUDA graph */
    qb_batch_config batch;       /* packed-kernel shape (zeros = defaults) */
    int32_t max_pending;         /* requests waiting for admission at most; a submit beyond returns QB_EBUSY
                                    (0 = no limit) */
    int32_t coop_parts;          /* cooperative sweeps (lockstep residual, weighted QUBO) run side by side, up
                                    to this many at once, each on a grid sized to its problem (at most half the
                                    device; the grids together within what the device holds at once)
                                    (0 = 4; 1 = each alone on the whole device) */
} qb_server_config;

/* Request states reported by qb_server_poll. */
#define QB_REQ_PENDING 0
#define QB_REQ_RUNNING 1
#define QB_REQ_DONE 2
#define QB_REQ_FAILED 3
#define QB_REQ_CANCELLED 4

typedef struct qb_request_info {
    int32_t state;               /* QB_REQ_* */
    int32_t status;              /* qb_status of a failed request */
    int32_t kind;                /* QB_KIND_* */
    int32_t n;
    int32_t n_branches;
    int32_t sweeps;
    int64_t attempts;            /* n_branches x sweeps x n */
    int64_t device_bytes;        /* budget charged at admission */
    double t_submit;             /* host steady-clock seconds */
    double t_admit;
    double t_done;
} qb_request_info;

typedef struct qb_server_stats {
    int64_t submitted;
    int64_t completed;
    int64_t failed;
    int64_t cancelled;
    int64_t pending;
    int64_t active;
    int64_t ticks;
    int64_t bytes_in_use;
    int64_t peak_bytes;
    int64_t budget_bytes;
    int64_t attempts_done;
} qb_server_stats;

qb_status qb_server_create(const qb_server_config* cfg, qb_server** out);
/* Queues a request and returns its id at once (QB_EBUSY when max_pending
 * requests already wait). The problem must stay alive until the request is
 * finished or cancelled; one problem serves one request at a time. */
qb_status qb_server_submit(qb_server* s, qb_problem* problem, const qb_schedule* sched, uint32_t n_branches,
                           uint64_t seed_offset, uint64_t* id);
/* Current state (QB_REQ_*) of a request. */
qb_status qb_server_poll(qb_server* s, uint64_t id, int32_t* state);
/* Waits until the request is finished (QB_OK), failed (its status), cancelled
 * (QB_ECANCELLED) or timeout_ms passes (QB_ETIMEDOUT; timeout_ms < 0 waits
 * without limit). */
qb_status qb_server_wait(qb_server* s, uint64_t id, int32_t timeout_ms);
/* Cancels a request that has not finished: a pending one leaves the queue, a
 * running ising request leaves at the next tick, a running residual request
 * finishes its launch and is then dropped. */
qb_status qb_server_cancel(qb_server* s, uint64_t id);
qb_status qb_server_request_info(qb_server* s, uint64_t id, qb_request_info* info);
/* Results of a finished request (layouts as the qb_result getters). */
qb_status qb_server_result_branches(qb_server* s, uint64_t id, uint8_t* x);
qb_status qb_server_result_marginals(qb_server* s, uint64_t id, float* p);
/* Ising: tracked energies (int64); residual: fp64 energies from scratch. */
qb_status qb_server_result_energies_i64(qb_server* s, uint64_t id, int64_t* e);
qb_status qb_server_result_energies_f64(qb_server* s, uint64_t id, double* e);
/* Frees a finished request's results and returns their memory to the budget. */
qb_status qb_server_release(qb_server* s, uint64_t id);
qb_status qb_server_stats_get(qb_server* s, qb_server_stats* st);
/* Cancels what is pending, waits for what runs, stops the worker. */
void qb_server_destroy(qb_server* s);

/* ---- provable-rock freezing --------------------------------------------------
 *
 * freeze_provable_rock (src/ising_recon.hpp:168-235) on the device: every bit
 * whose 0 -> 1 flip costs at least `margin` whatever the other bits do
 * (bound: sum_b w_b a (a/2 - d_b) + lin + lambda (#frozen - #free
 * neighbours)) is fixed at 0, repeated to a fixpoint; the reduced problem
 * keeps the other bits (in order) with the bonds to frozen rock folded into
 * their field. The frozen set and the reduced problem equal the reference's
 * (the fixpoint does not depend on the visiting order when lambda >= 0, which
 * is required); `rounds` counts the device's parallel rounds. The reduced
 * problem's arrays live in the handle (valid until qb_freeze_destroy); pass
 * them to qb_problem_create_residual and map results back through `kept`
 * (reduced bit -> original bit; every other bit is 0). */
typedef struct qb_freeze qb_freeze;
qb_status qb_freeze_rock(const qb_residual_desc* desc, double margin, const qb_opts* opts, qb_freeze** out);
qb_status qb_freeze_info(const qb_freeze* f, int32_t* n_kept, int32_t* rounds);
qb_status qb_freeze_kept(const qb_freeze* f, int32_t* kept);
qb_status qb_freeze_reduced(const qb_freeze* f, qb_residual_desc* reduced);
void qb_freeze_destroy(qb_freeze* f);

/* ---- exact local posterior of a region ------------------------------------
 *
 * qb_roi_qubo: the conditional QUBO of the region roi[0..n_roi) of a
 * residual-form problem, every other bit held at x_bar (roi_qubo,
 * src/ising_recon.hpp:240-300): E(x_R) - E(0_R) = sum_i h_i x_i +
 * sum_{i<j} J_ij x_i x_j, h of n_roi and J of n_roi x n_roi (upper triangle
 * used), equal to the reference's bit for bit. Host only.
 * qb_enumerate_qubo: every one of the 2^n states (n <= 34) of a dense QUBO
 * on the device, at temperature T: log Z, the exact marginals p(x_i = 1)
 * (into marginals[n]), the mean energy and the ground state (bit i of x_min =
 * x_i; the first found on ties). The reference exports the region's QUBO for
 * other tools; here it is enumerated. */
typedef struct qb_enum_result {
    double log_z;
    double e_min;
    uint64_t x_min;
    double mean_energy;
    uint64_t states;
} qb_enum_result;
qb_status qb_roi_qubo(const qb_residual_desc* p, const int32_t* roi, int32_t n_roi, const uint8_t* x_bar, double* h,
                      double* J);
qb_status qb_enumerate_qubo(int32_t n, const double* h, const double* J, double T, const qb_opts* opts,
                            qb_enum_result* out, double* marginals);

/* The machine export of a tomography solve; replaces the export block of
 * src/check_ising.cu:507-525 and the masks of tools/export_machine_map.py
 * (:47-55, :130-145). In directory `dir` it writes
 *   ising_out_pvoid.bin          float32 nx^3, C order (z, y, x): the p_void of
 *                                the voxel's bit, -1 outside the unknown domain;
 *   ising_out_pvoid_noprior.bin  the same for p_void_noprior (when not NULL);
 *   ising_out_truth.bin          uint8 nx^3, as given (when truth is not NULL);
 *   ising_out_branches.bin       n_branches x n_vars bytes, branch-major (when not NULL);
 *   ising_out.meta               text: nx, voxel, lo, branches, vars, lambda, kappa;
 *   ising_out_tristate.bin       uint8 nx^3: 0 Exists (p <= 0.1), 1 NotThere
 *                                (p >= 0.9), 2 Undecided (argos::classify,
 *                                ising_recon.hpp:305-309, in fp32), 255 outside;
 *   ising_out_traversable.bin    uint8 nx^3: 1 only where Exists;
 *   ising_out_machine.meta       the loader keys of the two masks.
 * var_voxel[i] is bit i's voxel index in nx^3 (nx <= 1024); two bits on one
 * voxel are refused. Host only. */
typedef struct qb_export_desc {
    int32_t nx;
    double voxel;
    double lo[3];
    int32_t n_vars;
    const int32_t* var_voxel;
    const float* p_void;
    const float* p_void_noprior;   /* may be NULL */
    const uint8_t* truth;          /* nx^3, may be NULL */
    const uint8_t* branches;       /* n_branches x n_vars, may be NULL */
    int32_t n_branches;
    double lambda;
    double kappa;
} qb_export_desc;
qb_status qb_write_ising_out(const char* dir, const qb_export_desc* d);

/* A region's QUBO as text for tensor tooling; replaces the writers of
 * build/ising_out_roi.txt and ising_out_roi_uncertain.txt
 * (src/check_ising.cu:568-591): line 1 n; n lines "voxel p truth h"; then the
 * n x n matrix J row by row (qb_roi_qubo fills the upper triangle), every value
 * followed by a space; reals with 17 significant digits. truth may be NULL
 * (written as 0). Host only. */
qb_status qb_write_roi_text(const char* path, int32_t n, const int32_t* voxel, const float* p, const uint8_t* truth,
                            const double* h, const double* J);

/* General QUBO text, the format the reference writes for its sequencing QUBOs
 * (src/check_ree_qubo.cu:277-283, read by tools/ree_neal.py):
 *   line 1: n m offset P optimum
 *   n lines: i Qd_i c_i           (i = 0..n-1 in order; c = cost / P)
 *   m lines: i j Qo_ij            (0 <= i < j < n, ascending (i, j))
 * with E(x) = offset + sum_i Qd_i x_i + sum Qo_ij x_i x_j and reals as %.17g.
 * qb_parse_qubo_text refuses a bad header, a malformed or short line, linear
 * lines out of order, a pair with i >= j or out of range, pairs out of order or
 * repeated, non-finite values and trailing text (reason in qb_last_error).
 * qb_qubo_text_arrays copies the fp64 data into caller buffers (n, n, m, m, m
 * elements; any may be NULL); qb_qubo_text_desc points a weighted-QUBO
 * descriptor at fp32 copies (Qd -> h, Qo -> J, the offset) for
 * qb_problem_create_qubo, valid until qb_qubo_text_destroy. qb_write_qubo_text
 * writes the format. Host only. */
typedef struct qb_qubo_text qb_qubo_text;
qb_status qb_parse_qubo_text(const char* text, size_t size, qb_qubo_text** out);
qb_status qb_qubo_text_info(const qb_qubo_text* q, int32_t* n, int64_t* m, double* offset, double* penalty,
                            double* optimum);
qb_status qb_qubo_text_arrays(const qb_qubo_text* q, double* qd, double* cost, int32_t* eu, int32_t* ev, double* qo);
qb_status qb_qubo_text_desc(const qb_qubo_text* q, qb_qubo_desc* d);
void qb_qubo_text_destroy(qb_qubo_text* q);
qb_status qb_write_qubo_text(const char* path, int32_t n, int64_t m, double offset, double penalty, double optimum,
                             const double* qd, const double* cost, const int32_t* eu, const int32_t* ev,
                             const double* qo);

/* Device energies of k caller states (k x n bytes, 0/1) by an independent
 * edge-list kernel: gising::device_energies (src/ising_gpu.cuh:461-475). */
qb_status qb_energies_ising(const qb_problem* p, const uint8_t* x, int32_t k, int64_t* e);
/* Device fp64 energies of k caller states for a weighted QUBO problem
 * (qubo_energy, src/check_ree_qubo.cu:158-163). */
qb_status qb_energies_qubo(const qb_problem* p, const uint8_t* x, int32_t k, double* e);
/* Device fp64 energies of k caller states for a residual problem
 * (binary_energy, src/ising_recon.hpp:65-79). */
qb_status qb_energies_residual(const qb_problem* p, const uint8_t* x, int32_t k, double* e);

#ifdef __cplusplus
}
#endif

#endif /* QUBLAR_H */
