// The serving loop of the C ABI (qb_server_*): admission by a device-memory
// budget, ising requests advanced together in ticks of the packed kernel
// (one CUDA-graph replay per tick, state resident between ticks), residual
// requests as cluster launches on a stream pool beside the ticks, and the
// cooperative sweeps (lockstep residual, weighted QUBO) side by side on equal
// partitions of the device's SMs, one cooperative grid per request.
//
// One worker thread owns every device call of the loop. It never holds the
// server mutex across a CUDA call that waits, and it polls completion events
// (no host callbacks), so client threads only ever wait on the mutex briefly.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "qb_batch.hpp"
#include "qb_internal.hpp"
#include "qb_kernels.hpp"
#include "qb_qubo.hpp"

using namespace qb;

namespace {

using Clock = std::chrono::steady_clock;

double now_s() { return std::chrono::duration<double>(Clock::now().time_since_epoch()).count(); }

constexpr int64_t kDefaultBudget = int64_t(150) * 1000 * 1000 * 1000;
constexpr int kDefaultActive = 4096;
constexpr int kDefaultResidStreams = 8;
constexpr int kDefaultTickUs = 20000;
constexpr size_t kTickHeader = 64;   // ctl words before the items
constexpr int kDefaultParts = 4;     // SM partitions for cooperative sweeps

int floor_pow2(int v) {
    int g = 1;
    while (g * 2 <= v) g *= 2;
    return g;
}

int log2i(int v) {
    int l = 0;
    while ((1 << l) < v) ++l;
    return l;
}

struct Group {
    int r0 = 0;
    int G = 1;
    bool global = false;
    int64_t state_off = 0;   // bytes into the request's state arena
};

struct Request {
    uint64_t id = 0;
    qb_problem* prob = nullptr;
    qb_schedule sched{};
    int kind = 0;
    int R = 0;
    int n = 0;
    int sweeps = 0;
    uint64_t seed0 = 0;
    int state = QB_REQ_PENDING;
    qb_status status = QB_OK;
    std::string error;
    double t_submit = 0.0, t_admit = 0.0, t_done = 0.0;
    int64_t charge_work = 0;      // problem + working memory: returned when the request finishes
    int64_t charge_results = 0;   // results: returned when the client releases them
    bool cancel = false;
    bool coop = false;            // a cooperative sweep (lockstep residual or weighted QUBO)
    bool exclusive = false;       // ... on the whole device, with nothing beside it (no partition plan)
    int part = -1;                // the stream a side-by-side cooperative sweep runs on
    int ctas = 0;                 // ... and its grid (CTAs taken from the device's cooperative budget)
    // device memory (stream-ordered allocations)
    DevBuf d_x, d_f, d_e, d_p, d_temp, d_state, d_drift, d_accepts, d_ef64, d_etrack;
    // ising progress
    std::vector<Group> groups;
    int cursor = 0;       // next sweep
    int slice = 1;        // sweeps per tick
    // residual
    cudaEvent_t done_ev = nullptr;
};

}  // namespace

struct qb_server {
    qb_server_config cfg{};
    int device = 0;
    int64_t budget = 0;
    std::thread worker;
    std::mutex mu;
    std::condition_variable cv_work;   // submissions, cancellations, stop
    std::condition_variable cv_done;   // a request finished
    bool stop = false;
    bool kick = false;
    uint64_t next_id = 1;
    std::deque<uint64_t> pending;
    std::map<uint64_t, std::unique_ptr<Request>> reqs;
    int64_t bytes_in_use = 0, peak_bytes = 0;
    int64_t submitted = 0, completed = 0, failed = 0, cancelled = 0, ticks = 0, attempts_done = 0;
    int active = 0;
    // worker-owned device state
    cudaStream_t upload_stream = nullptr, tick_stream = nullptr;
    std::vector<cudaStream_t> resid_streams;
    int next_resid_stream = 0;
    cudaEvent_t upload_ev = nullptr, tick_ev = nullptr;
    BatchShape shape;
    DevBuf d_tick;
    unsigned char* h_tick = nullptr;
    size_t tick_cap = 0;   // items the tick buffers hold
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaGraphNode_t copy_node = nullptr;
    std::vector<Request*> running_ising;
    std::vector<Request*> running_resid;
    Request* exclusive_run = nullptr;
    // cooperative sweeps side by side: up to `parts` at once, each on its own
    // stream with a grid sized to its problem, their grids together within the
    // CTAs the device holds at once (coop_budget), one grid at most coop_cap
    int parts = 1;
    int coop_budget = 0, coop_cap = 0, coop_used = 0;
    int full_resid = 0, full_qubo = 0;
    std::vector<cudaStream_t> part_streams;
    std::vector<Request*> part_run;
    std::vector<qb_problem*> submitting;   // problems being planned for a partition by a submitting thread
    bool tick_inflight = false;
    std::vector<std::pair<Request*, int>> tick_members;   // request, sweep end of its slice
    std::string fatal;
    int64_t admissions = 0;
    int64_t fail_admission = 0;   // QB_SERVER_FAIL_ADMIT=k: the k-th admission fails (host-side fault injection)
};

namespace {

// ---- small helpers (worker thread) ---------------------------------------------------------

void finish_locked(qb_server* S, Request* r, int state, qb_status st, const std::string& msg) {
    r->state = state;
    r->status = st;
    r->error = msg;
    r->t_done = now_s();
    if (state == QB_REQ_DONE) {
        ++S->completed;
        S->attempts_done += int64_t(r->R) * r->sweeps * r->n;
    } else if (state == QB_REQ_FAILED) {
        ++S->failed;
    } else if (state == QB_REQ_CANCELLED) {
        ++S->cancelled;
    }
    S->cv_done.notify_all();
}

// Frees what a request held while it ran (its problem's device copy, state,
// temperatures); results stay until the client releases them.
void drop_work(qb_server* S, Request* r) {
    problem_release_device(r->prob);
    r->d_state.release();
    r->d_temp.release();
    r->d_drift.release();
    r->d_accepts.release();
    r->d_etrack.release();
    if (r->done_ev) {
        cudaEventDestroy(r->done_ev);
        r->done_ev = nullptr;
    }
    std::lock_guard<std::mutex> lk(S->mu);
    S->bytes_in_use -= r->charge_work;
    r->charge_work = 0;
    --S->active;
}

void drop_results(Request* r) {
    DevBuf* all[] = {&r->d_x, &r->d_f, &r->d_e, &r->d_p, &r->d_ef64};
    for (DevBuf* b : all) b->release();
}

int64_t ising_work_bytes(const qb_problem* p, int R, int sweeps) {
    const int64_t n = p->ising.n;
    return p->device_bytes + n * R * 5 + int64_t(sweeps) * 8;
}
int64_t ising_result_bytes(int n, int R) { return int64_t(n) * R * 5 + int64_t(R) * 8 + int64_t(n) * 4; }
int64_t resid_work_bytes(const qb_problem* p, int R, int sweeps) {
    int64_t b = p->device_bytes + int64_t(sweeps) * 8 + int64_t(R) * 12;
    if (p->kind == QB_KIND_RESIDUAL && p->resid.variant == QB_RESID_LOCKSTEP)
        b += int64_t(resid_lockstep_scratch(p->resid, std::min(R, resid_lockstep_max_branches())));
    if (p->kind == QB_KIND_QUBO) b += int64_t(qubo_scratch(p->qubo)) + int64_t(R) * 8;
    return b;
}
int64_t resid_result_bytes(int n, int R) { return int64_t(n) * R + int64_t(R) * 8 + int64_t(n) * 4; }

// Splits an ising request into replica groups for the packed kernel and sizes
// its slice so one item of a tick does about target_attempts attempts.
void plan_groups(qb_server* S, Request* r, double target_attempts) {
    const int cap = S->shape.smem_bytes;
    const int maxg = S->cfg.batch.max_group;
    int64_t off = 0;
    int gmax = 1;
    for (int r0 = 0; r0 < r->R;) {
        const int G0 = std::min(maxg, floor_pow2(r->R - r0));
        int G = G0;
        while (G > 1 && batch_item_smem(r->n, G) > size_t(cap)) G /= 2;
        Group g;
        g.r0 = r0;
        g.global = batch_item_smem(r->n, G) > size_t(cap);
        if (g.global) {
            // a global-state item of one big instance: narrow groups keep its
            // per-tick work near the target and spread it over more CTAs
            G = G0;
            while (G > 1 && double(r->n) * G > target_attempts / 8.0) G /= 2;
        }
        g.G = G;
        g.state_off = off;
        off += int64_t(batch_item_smem(r->n, G) + 255) / 256 * 256;
        gmax = std::max(gmax, G);
        r->groups.push_back(g);
        r0 += G;
    }
    const double per_sweep = double(r->n) * gmax;
    r->slice = int(std::max(1.0, std::min(double(r->sweeps), std::floor(target_attempts / per_sweep))));
}

// The grid of a cooperative request that runs beside others: enough CTAs
// that a colour class gives each of them about one round of warp items (a
// residual bit takes about nnz / (16 n) + 1.5 items, a QUBO bit one warp
// visit), at least 16, at most half the device.
int coop_grid(const qb_server* S, const qb_problem* p) {
    double per_class = 0.0, items_per_bit = 1.0, per_cta = 32.0;
    int full = S->full_qubo;
    if (p->kind == QB_KIND_RESIDUAL) {
        const ResidualPlan& P = p->resid;
        per_class = double(P.n) / std::max(1, P.col.n_colours());
        items_per_bit = double(P.nnz) / std::max(1, P.n) / 16.0 + 1.5;
        per_cta = 28.0;
        full = S->full_resid;
    } else {
        per_class = double(p->qubo.n) / std::max(1, p->qubo.col.n_colours());
    }
    const int want = int(std::ceil(per_class * items_per_bit / per_cta));
    return std::max(std::min(16, full), std::min({want, S->coop_cap, full}));
}

// ---- admission ---------------------------------------------------------------------------------

qb_status admit_ising(qb_server* S, Request* r) {
    qb_status s;
    AsyncAllocScope scope(S->upload_stream);
    if ((s = problem_upload(r->prob, S->upload_stream)) != QB_OK) return s;
    const std::vector<double> temp = temperatures(r->sched);
    if ((s = upload_vec(r->d_temp, temp, S->upload_stream))) return s;
    double target = double(S->cfg.tick_target_us) * 1e-6 * 4e8;   // attempts one CTA does in the target time
    plan_groups(S, r, target);
    int64_t state = 0;
    for (const Group& g : r->groups) state += int64_t(batch_item_smem(r->n, g.G) + 255) / 256 * 256;
    if ((s = r->d_state.alloc(size_t(state)))) return s;
    if ((s = r->d_x.alloc(size_t(r->R) * size_t(r->n)))) return s;
    if ((s = r->d_f.alloc(size_t(r->R) * size_t(r->n) * 4))) return s;
    if ((s = r->d_e.alloc(size_t(r->R) * 8))) return s;
    if ((s = r->d_p.alloc(size_t(r->n) * 4))) return s;
    QB_CUDA(cudaStreamSynchronize(S->upload_stream));   // `temp` is a local
    return QB_OK;
}

qb_status launch_resid(qb_server* S, Request* r) {
    qb_status s;
    cudaStream_t st = S->resid_streams[size_t(S->next_resid_stream)];
    S->next_resid_stream = (S->next_resid_stream + 1) % int(S->resid_streams.size());
    {
        AsyncAllocScope scope(S->upload_stream);
        if ((s = problem_upload(r->prob, S->upload_stream)) != QB_OK) return s;
        const std::vector<double> temp = temperatures(r->sched);
        if ((s = upload_vec(r->d_temp, temp, S->upload_stream))) return s;
        if ((s = r->d_x.alloc(size_t(r->R) * size_t(r->n)))) return s;
        if ((s = r->d_drift.alloc(size_t(r->R) * 4))) return s;
        if ((s = r->d_accepts.alloc(size_t(r->R) * 8))) return s;
        if ((s = r->d_ef64.alloc(size_t(r->R) * 8))) return s;
        if ((s = r->d_p.alloc(size_t(r->n) * 4))) return s;
        QB_CUDA(cudaMemsetAsync(r->d_drift.p, 0, r->d_drift.bytes, S->upload_stream));
        QB_CUDA(cudaMemsetAsync(r->d_accepts.p, 0, r->d_accepts.bytes, S->upload_stream));
        QB_CUDA(cudaStreamSynchronize(S->upload_stream));   // `temp` is a local
    }
    const ResidualPlan& P = r->prob->resid;
    SolveBuffers b;
    b.x = r->d_x.as<uint8_t>();
    b.temp = r->d_temp.as<double>();
    b.drift = r->d_drift.as<float>();
    b.accepts = r->d_accepts.as<unsigned long long>();
    b.e_f64 = r->d_ef64.as<double>();
    b.p = r->d_p.as<float>();
    if ((s = launch_resid_anneal(P, b, r->R, r->sweeps, r->sched.refresh_sweeps, r->seed0, st))) return s;
    if ((s = launch_resid_energies(P, b.x, r->R, b.e_f64, st))) return s;
    if ((s = launch_marginals(b.x, r->R, r->n, b.p, st))) return s;
    QB_CUDA(cudaEventCreateWithFlags(&r->done_ev, cudaEventDisableTiming));
    QB_CUDA(cudaEventRecord(r->done_ev, st));
    return QB_OK;
}

// A cooperative sweep (lockstep residual or weighted QUBO) on stream `st`:
// the whole device (exclusive requests) or one partition's grid; its scratch
// lives in d_state.
qb_status launch_coop(qb_server* S, Request* r, cudaStream_t st, int qubo_ctas) {
    qb_status s;
    const bool qubo = r->kind == QB_KIND_QUBO;
    {
        AsyncAllocScope scope(S->upload_stream);
        if ((s = problem_upload(r->prob, S->upload_stream)) != QB_OK) return s;
        const std::vector<double> temp = temperatures(r->sched);
        if ((s = upload_vec(r->d_temp, temp, S->upload_stream))) return s;
        const size_t scratch = qubo ? qubo_scratch(r->prob->qubo)
                                    : resid_lockstep_scratch(r->prob->resid, std::min(r->R, resid_lockstep_max_branches()));
        if ((s = r->d_state.alloc(scratch))) return s;
        if ((s = r->d_x.alloc(size_t(r->R) * size_t(r->n)))) return s;
        if ((s = r->d_drift.alloc(size_t(r->R) * 4))) return s;
        if ((s = r->d_accepts.alloc(size_t(r->R) * 8))) return s;
        if ((s = r->d_ef64.alloc(size_t(r->R) * 8))) return s;
        if ((s = r->d_p.alloc(size_t(r->n) * 4))) return s;
        if (qubo && (s = r->d_etrack.alloc(size_t(r->R) * 8))) return s;
        QB_CUDA(cudaMemsetAsync(r->d_drift.p, 0, r->d_drift.bytes, S->upload_stream));
        QB_CUDA(cudaMemsetAsync(r->d_accepts.p, 0, r->d_accepts.bytes, S->upload_stream));
        if (qubo) QB_CUDA(cudaMemsetAsync(r->d_etrack.p, 0, r->d_etrack.bytes, S->upload_stream));
        QB_CUDA(cudaMemsetAsync(r->d_state.p, 0, 64, S->upload_stream));   // barrier counter and timeout flag
        QB_CUDA(cudaStreamSynchronize(S->upload_stream));   // `temp` is a local
    }
    uint8_t* x = r->d_x.as<uint8_t>();
    if (qubo) {
        const int RB = qubo_max_branches();
        for (int b0 = 0; b0 < r->R; b0 += RB) {
            QuboBuffers qb;
            qb.x = x + size_t(b0) * size_t(r->n);
            qb.temp = r->d_temp.as<double>();
            qb.drift = r->d_drift.as<float>() + b0;
            qb.e_track = r->d_etrack.as<double>() + b0;
            qb.accepts = r->d_accepts.as<unsigned long long>() + b0;
            qb.scratch = r->d_state.p;
            if ((s = launch_qubo_lockstep(r->prob->qubo, qb, std::min(RB, r->R - b0), r->sweeps,
                                          r->sched.refresh_sweeps, r->seed0 + uint64_t(b0), st, qubo_ctas)))
                return s;
        }
        if ((s = launch_qubo_energies(r->prob->qubo, x, r->R, r->d_ef64.as<double>(), st))) return s;
    } else {
        const ResidualPlan& P = r->prob->resid;
        const int RB = resid_lockstep_max_branches();
        for (int b0 = 0; b0 < r->R; b0 += RB) {
            SolveBuffers b;
            b.x = x + size_t(b0) * size_t(r->n);
            b.temp = r->d_temp.as<double>();
            b.drift = r->d_drift.as<float>() + b0;
            b.accepts = r->d_accepts.as<unsigned long long>() + b0;
            b.scratch = r->d_state.p;
            if ((s = launch_resid_lockstep(P, b, std::min(RB, r->R - b0), r->sweeps, r->sched.refresh_sweeps,
                                           r->seed0 + uint64_t(b0), st)))
                return s;
        }
        if ((s = launch_resid_energies(P, x, r->R, r->d_ef64.as<double>(), st))) return s;
    }
    if ((s = launch_marginals(x, r->R, r->n, r->d_p.as<float>(), st))) return s;
    QB_CUDA(cudaEventCreateWithFlags(&r->done_ev, cudaEventDisableTiming));
    QB_CUDA(cudaEventRecord(r->done_ev, st));
    return QB_OK;
}

// Admits pending requests in arrival order while the budget and the active
// limit allow (a request larger than the whole budget fails). An exclusive
// request waits at the head until the device is idle and holds back those
// behind it while it runs.
void admit_pending(qb_server* S) {
    for (;;) {
        Request* r = nullptr;
        {
            std::lock_guard<std::mutex> lk(S->mu);
            while (!S->pending.empty()) {
                auto it = S->reqs.find(S->pending.front());
                Request* q = it == S->reqs.end() ? nullptr : it->second.get();
                if (!q || q->cancel) {
                    S->pending.pop_front();
                    if (q) finish_locked(S, q, QB_REQ_CANCELLED, QB_ECANCELLED, "cancelled before admission");
                    continue;
                }
                break;
            }
            if (S->pending.empty() || S->stop) return;
            Request* q = S->reqs[S->pending.front()].get();
            const int64_t need = q->charge_work + q->charge_results;
            if (need > S->budget) {
                S->pending.pop_front();
                finish_locked(S, q, QB_REQ_FAILED, QB_ENOMEM, "the request needs more device memory than the whole budget");
                continue;
            }
            if (S->bytes_in_use + need > S->budget || S->active >= S->cfg.max_active) return;
            if (S->exclusive_run) return;
            bool parts_busy = false;
            for (Request* pr : S->part_run) parts_busy |= pr != nullptr;
            if (q->exclusive && (S->tick_inflight || !S->running_ising.empty() || !S->running_resid.empty() || parts_busy))
                return;
            if (q->coop && !q->exclusive) {   // a free stream and room for its grid, or wait at the head
                int slot = -1;
                for (int k = 0; k < int(S->part_run.size()) && slot < 0; ++k)
                    if (!S->part_run[size_t(k)]) slot = k;
                if (slot < 0 || S->coop_used + q->ctas > S->coop_budget) return;
                q->part = slot;
                S->coop_used += q->ctas;
            }
            S->pending.pop_front();
            S->bytes_in_use += need;
            S->peak_bytes = std::max(S->peak_bytes, S->bytes_in_use);
            ++S->active;
            q->state = QB_REQ_RUNNING;
            q->t_admit = now_s();
            r = q;
        }
        ++S->admissions;
        const qb_status s = S->admissions == S->fail_admission
                                ? fail(QB_ENOMEM, "injected admission failure (QB_SERVER_FAIL_ADMIT)")
                            : r->exclusive ? launch_coop(S, r, S->tick_stream, 0)
                            : r->coop      ? launch_coop(S, r, S->part_streams[size_t(r->part)], r->ctas)
                            : r->kind == QB_KIND_ISING ? admit_ising(S, r)
                                                       : launch_resid(S, r);
        if (s != QB_OK) {
            const std::string msg = qb_last_error();
            if (r->coop && !r->exclusive) S->coop_used -= r->ctas;   // its grid never ran
            drop_work(S, r);
            drop_results(r);
            std::lock_guard<std::mutex> lk(S->mu);
            S->bytes_in_use -= r->charge_results;
            r->charge_results = 0;
            finish_locked(S, r, QB_REQ_FAILED, s, msg);
            continue;
        }
        if (r->exclusive) S->exclusive_run = r;
        else if (r->coop) S->part_run[size_t(r->part)] = r;
        else if (r->kind == QB_KIND_ISING) S->running_ising.push_back(r);
        else S->running_resid.push_back(r);
    }
}

// ---- ticks -----------------------------------------------------------------------------------

qb_status ensure_tick_capacity(qb_server* S, size_t items) {
    if (items <= S->tick_cap && S->h_tick) return QB_OK;
    size_t cap = std::max<size_t>(1024, S->tick_cap);
    while (cap < items) cap *= 2;
    if (S->exec) {
        cudaGraphExecDestroy(S->exec);
        S->exec = nullptr;
    }
    if (S->graph) {
        cudaGraphDestroy(S->graph);
        S->graph = nullptr;
    }
    if (S->h_tick) cudaFreeHost(S->h_tick);
    S->h_tick = nullptr;
    const size_t bytes = kTickHeader + cap * sizeof(IsingItem);
    QB_CUDA(cudaStreamSynchronize(S->tick_stream));
    QB_CUDA(cudaMallocHost(&S->h_tick, bytes));
    qb_status s = S->d_tick.alloc(bytes);
    if (s != QB_OK) return s;
    S->tick_cap = cap;
    if (S->cfg.use_graph) {
        // one tick: header + items up, then the packed kernel over them
        QB_CUDA(cudaStreamBeginCapture(S->tick_stream, cudaStreamCaptureModeThreadLocal));
        cudaMemcpyAsync(S->d_tick.p, S->h_tick, bytes, cudaMemcpyHostToDevice, S->tick_stream);
        const qb_status ls = launch_ising_batch_ctl(
            reinterpret_cast<const IsingItem*>(S->d_tick.as<unsigned char>() + kTickHeader), S->d_tick.as<int>(),
            S->shape, S->tick_stream);
        cudaGraph_t g = nullptr;
        const cudaError_t ce = cudaStreamEndCapture(S->tick_stream, &g);
        if (ls != QB_OK) return ls;
        if (ce != cudaSuccess) return cuda_fail(ce, "cudaStreamEndCapture", __FILE__, __LINE__);
        S->graph = g;
        QB_CUDA(cudaGraphInstantiate(&S->exec, S->graph, 0));
        size_t nn = 0;
        QB_CUDA(cudaGraphGetNodes(S->graph, nullptr, &nn));
        std::vector<cudaGraphNode_t> nodes(nn);
        QB_CUDA(cudaGraphGetNodes(S->graph, nodes.data(), &nn));
        S->copy_node = nullptr;
        for (cudaGraphNode_t nd : nodes) {
            cudaGraphNodeType t;
            QB_CUDA(cudaGraphNodeGetType(nd, &t));
            if (t == cudaGraphNodeTypeMemcpy) S->copy_node = nd;
        }
        if (!S->copy_node) return fail(QB_ECUDA, "server: the captured tick has no copy node");
    }
    return QB_OK;
}

qb_status launch_tick(qb_server* S) {
    std::vector<IsingItem> items;
    S->tick_members.clear();
    for (Request* r : S->running_ising) {
        if (r->cancel) continue;
        const IsingPlan& P = r->prob->ising;
        const int s0 = r->cursor, s1 = std::min(r->sweeps, r->cursor + r->slice);
        for (const Group& g : r->groups) {
            IsingItem it;
            std::memset(&it, 0, sizeof(it));
            it.class_ptr = P.d_class_ptr.as<int32_t>();
            it.row = P.d_row.as<int32_t>();
            it.adj = P.d_adj.as<int32_t>();
            it.w = P.d_w.p;
            it.f0 = P.d_f0.as<int32_t>();
            it.order = P.d_order.as<int32_t>();
            it.temp = r->d_temp.as<double>();
            unsigned char* base = r->d_state.as<unsigned char>() + g.state_off;
            it.f_state = reinterpret_cast<int32_t*>(base);
            it.s_state = reinterpret_cast<int8_t*>(base + size_t(r->n) * size_t(g.G) * 4);
            it.e_acc = r->d_e.as<long long>() + g.r0;
            it.x_out = r->d_x.as<uint8_t>() + size_t(g.r0) * size_t(r->n);
            it.f_out = r->d_f.as<int32_t>() + size_t(g.r0) * size_t(r->n);
            it.seed0 = r->seed0 + uint64_t(g.r0);
            it.n = r->n;
            it.n_colours = P.col.n_colours();
            it.log2g = log2i(g.G);
            it.sweep0 = s0;
            it.sweep1 = s1;
            it.flags = (s0 == 0 ? kItemInit : 0) | (s1 == r->sweeps ? kItemFinal : 0) |
                       (g.global ? kItemGlobal : (s1 < r->sweeps ? kItemKeep : 0)) | item_rbase_flags(g.r0);
            it.bound = int32_t(P.B);
            it.wbytes = P.weight_bytes;
            items.push_back(it);
        }
        S->tick_members.emplace_back(r, s1);
    }
    if (items.empty()) return QB_OK;
    // largest first, as in a batch
    std::stable_sort(items.begin(), items.end(), [](const IsingItem& a, const IsingItem& b) {
        return double(a.n) * (1 << a.log2g) * (a.sweep1 - a.sweep0) > double(b.n) * (1 << b.log2g) * (b.sweep1 - b.sweep0);
    });
    qb_status s = ensure_tick_capacity(S, items.size());
    if (s != QB_OK) return s;
    // the uploads of newly admitted requests come first
    QB_CUDA(cudaEventRecord(S->upload_ev, S->upload_stream));
    QB_CUDA(cudaStreamWaitEvent(S->tick_stream, S->upload_ev, 0));
    int* ctl = reinterpret_cast<int*>(S->h_tick);
    ctl[0] = 0;
    ctl[1] = int(items.size());
    std::memcpy(S->h_tick + kTickHeader, items.data(), items.size() * sizeof(IsingItem));
    const size_t bytes = kTickHeader + items.size() * sizeof(IsingItem);
    if (S->cfg.use_graph) {
        QB_CUDA(cudaGraphExecMemcpyNodeSetParams1D(S->exec, S->copy_node, S->d_tick.p, S->h_tick, bytes,
                                                   cudaMemcpyHostToDevice));
        QB_CUDA(cudaGraphLaunch(S->exec, S->tick_stream));
    } else {
        QB_CUDA(cudaMemcpyAsync(S->d_tick.p, S->h_tick, bytes, cudaMemcpyHostToDevice, S->tick_stream));
        if ((s = launch_ising_batch_ctl(reinterpret_cast<const IsingItem*>(S->d_tick.as<unsigned char>() + kTickHeader),
                                        S->d_tick.as<int>(), S->shape, S->tick_stream)))
            return s;
    }
    for (auto& m : S->tick_members)
        if (m.second == m.first->sweeps) {
            Request* r = m.first;
            if ((s = launch_marginals(r->d_x.as<uint8_t>(), r->R, r->n, r->d_p.as<float>(), S->tick_stream))) return s;
        }
    QB_CUDA(cudaEventRecord(S->tick_ev, S->tick_stream));
    S->tick_inflight = true;
    return QB_OK;
}

void fail_all_running(qb_server* S, qb_status st, const std::string& msg) {
    std::vector<Request*> all(S->running_ising);
    all.insert(all.end(), S->running_resid.begin(), S->running_resid.end());
    S->running_ising.clear();
    S->running_resid.clear();
    S->tick_inflight = false;
    for (Request* r : all) {
        drop_work(S, r);
        drop_results(r);
        std::lock_guard<std::mutex> lk(S->mu);
        S->bytes_in_use -= r->charge_results;
        r->charge_results = 0;
        finish_locked(S, r, QB_REQ_FAILED, st, msg);
    }
}

void poll_tick(qb_server* S) {
    if (!S->tick_inflight) return;
    const cudaError_t e = cudaEventQuery(S->tick_ev);
    if (e == cudaErrorNotReady) return;
    S->tick_inflight = false;
    if (e != cudaSuccess) {
        cuda_fail(e, "tick", __FILE__, __LINE__);
        S->fatal = qb_last_error();
        fail_all_running(S, QB_ECUDA, S->fatal);
        return;
    }
    {
        std::lock_guard<std::mutex> lk(S->mu);
        ++S->ticks;
    }
    std::vector<Request*> keep;
    for (auto& m : S->tick_members) m.first->cursor = m.second;
    for (Request* r : S->running_ising) {
        if (r->cancel) {
            drop_work(S, r);
            drop_results(r);
            std::lock_guard<std::mutex> lk(S->mu);
            S->bytes_in_use -= r->charge_results;
            r->charge_results = 0;
            finish_locked(S, r, QB_REQ_CANCELLED, QB_ECANCELLED, "cancelled while running");
        } else if (r->cursor >= r->sweeps) {
            drop_work(S, r);
            std::lock_guard<std::mutex> lk(S->mu);
            finish_locked(S, r, QB_REQ_DONE, QB_OK, "");
        } else {
            keep.push_back(r);
        }
    }
    S->running_ising.swap(keep);
}

void poll_resid(qb_server* S) {
    std::vector<Request*> keep;
    for (Request* r : S->running_resid) {
        const cudaError_t e = cudaEventQuery(r->done_ev);
        if (e == cudaErrorNotReady) {
            keep.push_back(r);
            continue;
        }
        if (e != cudaSuccess) {
            cuda_fail(e, "residual request", __FILE__, __LINE__);
            S->fatal = qb_last_error();
        }
        const bool cancelled = r->cancel;
        drop_work(S, r);
        std::lock_guard<std::mutex> lk(S->mu);
        if (e != cudaSuccess || cancelled) {
            drop_results(r);
            S->bytes_in_use -= r->charge_results;
            r->charge_results = 0;
            if (cancelled) finish_locked(S, r, QB_REQ_CANCELLED, QB_ECANCELLED, "cancelled while running");
            else finish_locked(S, r, QB_REQ_FAILED, QB_ECUDA, S->fatal);
        } else {
            finish_locked(S, r, QB_REQ_DONE, QB_OK, "");
        }
    }
    S->running_resid.swap(keep);
}

// A finished cooperative sweep: its timeout flag, then its results. Returns
// false while it runs.
bool poll_coop(qb_server* S, Request* r) {
    cudaError_t e = cudaEventQuery(r->done_ev);
    if (e == cudaErrorNotReady) return false;
    int timed_out = 0;
    if (e == cudaSuccess) {
        const cudaError_t c = cudaMemcpy(&timed_out, static_cast<const char*>(r->d_state.p) + 16, sizeof(int),
                                         cudaMemcpyDeviceToHost);
        if (c != cudaSuccess) e = c;
    }
    std::string msg;
    if (e != cudaSuccess) {
        cuda_fail(e, "cooperative request", __FILE__, __LINE__);
        msg = qb_last_error();
        S->fatal = msg;
    }
    const bool cancelled = r->cancel;
    drop_work(S, r);
    std::lock_guard<std::mutex> lk(S->mu);
    if (e != cudaSuccess || timed_out || cancelled) {
        drop_results(r);
        S->bytes_in_use -= r->charge_results;
        r->charge_results = 0;
        if (e != cudaSuccess) finish_locked(S, r, QB_REQ_FAILED, QB_ECUDA, msg);
        else if (timed_out)
            finish_locked(S, r, QB_REQ_FAILED, QB_ETIMEDOUT, "a grid barrier of the sweep timed out: no results");
        else finish_locked(S, r, QB_REQ_CANCELLED, QB_ECANCELLED, "cancelled while running");
    } else {
        finish_locked(S, r, QB_REQ_DONE, QB_OK, "");
    }
    return true;
}

void poll_exclusive(qb_server* S) {
    if (S->exclusive_run && poll_coop(S, S->exclusive_run)) S->exclusive_run = nullptr;
    for (Request*& r : S->part_run)
        if (r && poll_coop(S, r)) {
            S->coop_used -= r->ctas;
            r = nullptr;
        }
}

// Cancelled ising requests leave between ticks.
void reap_cancelled_ising(qb_server* S) {
    std::vector<Request*> keep;
    for (Request* r : S->running_ising) {
        if (!r->cancel) {
            keep.push_back(r);
            continue;
        }
        drop_work(S, r);
        drop_results(r);
        std::lock_guard<std::mutex> lk(S->mu);
        S->bytes_in_use -= r->charge_results;
        r->charge_results = 0;
        finish_locked(S, r, QB_REQ_CANCELLED, QB_ECANCELLED, "cancelled while running");
    }
    S->running_ising.swap(keep);
}

void worker_main(qb_server* S) {
    cudaSetDevice(S->device);
    for (;;) {
        try {
            poll_resid(S);
            poll_tick(S);
            poll_exclusive(S);
            if (!S->tick_inflight) reap_cancelled_ising(S);
            admit_pending(S);
            if (!S->tick_inflight && !S->running_ising.empty() && S->fatal.empty()) {
                if (launch_tick(S) != QB_OK) {
                    S->fatal = qb_last_error();
                    fail_all_running(S, QB_ECUDA, S->fatal);
                }
            }
        } catch (const std::exception& e) {
            // a failed host allocation (or any exception) must not end the
            // caller's process: let the device's work end (every kernel's waits
            // are bounded), then fail the running requests with the reason
            cudaDeviceSynchronize();
            S->fatal = dynamic_cast<const std::bad_alloc*>(&e) ? std::string("server worker: out of host memory")
                                                               : std::string("server worker: ") + e.what();
            fail_all_running(S, QB_ENOMEM, S->fatal);
        }
        std::unique_lock<std::mutex> lk(S->mu);
        bool parts_busy = false;
        for (Request* pr : S->part_run) parts_busy |= pr != nullptr;
        const bool busy = S->tick_inflight || !S->running_resid.empty() || S->exclusive_run != nullptr || parts_busy;
        if (S->stop && !busy && S->running_ising.empty()) break;
        if (busy) S->cv_work.wait_for(lk, std::chrono::microseconds(50), [&] { return S->kick; });
        else S->cv_work.wait(lk, [&] { return S->kick || S->stop; });
        S->kick = false;
    }
}

Request* find_locked(qb_server* S, uint64_t id) {
    auto it = S->reqs.find(id);
    return it == S->reqs.end() ? nullptr : it->second.get();
}

}  // namespace

// ---- C ABI -------------------------------------------------------------------------------------

extern "C" qb_status qb_server_create(const qb_server_config* cfg, qb_server** out) {
    return qb::guarded("qb_server_create", [&]() -> qb_status {
        if (!out) return fail(QB_EINVAL, "qb_server_create: null output");
        *out = nullptr;
        qb_server_config c{};
        if (cfg) c = *cfg;
        if (c.max_active == 0) c.max_active = kDefaultActive;
        if (c.residual_streams == 0) c.residual_streams = kDefaultResidStreams;
        if (c.tick_target_us == 0) c.tick_target_us = kDefaultTickUs;
        if (c.hbm_budget_bytes < 0 || c.max_active < 0 || c.residual_streams < 0 || c.residual_streams > 64 ||
            c.tick_target_us < 0 || c.max_pending < 0 || c.coop_parts < 0 || c.coop_parts > 64)
            return fail(QB_EINVAL, "qb_server_create: negative or out-of-range setting");
        if (c.batch.threads == 0) c.batch.threads = 512;
        if (c.batch.smem_bytes == 0) c.batch.smem_bytes = 96 * 1024;
        if (c.batch.max_group == 0) c.batch.max_group = 32;
        if (c.batch.threads < 32 || c.batch.threads > 1024 || c.batch.threads % 32 || c.batch.max_group < 1 ||
            c.batch.max_group > 32 || (c.batch.max_group & (c.batch.max_group - 1)))
            return fail(QB_EINVAL, "qb_server_create: bad packed-kernel shape");
        int dev = c.device;
        if (dev < 0) QB_CUDA(cudaGetDevice(&dev));
        QB_CUDA(cudaSetDevice(dev));
        std::unique_ptr<qb_server> S(new (std::nothrow) qb_server());
        if (!S) return fail(QB_ENOMEM, "qb_server_create: out of host memory");
        S->device = dev;
        size_t free_b = 0, total_b = 0;
        QB_CUDA(cudaMemGetInfo(&free_b, &total_b));
        int64_t budget = c.hbm_budget_bytes ? c.hbm_budget_bytes : kDefaultBudget;
        if (c.hbm_budget_bytes == 0) budget = std::min<int64_t>(budget, int64_t(double(free_b) * 0.9));
        S->budget = budget;
        const int cap = batch_max_smem();
        if (cap <= 0) return fail(QB_ECUDA, "qb_server_create: cannot read the shared-memory limit");
        c.batch.smem_bytes = std::min(c.batch.smem_bytes, cap);
        S->cfg = c;
        S->shape.threads = c.batch.threads;
        S->shape.smem_bytes = c.batch.smem_bytes;
        qb_status s = batch_ctas(S->shape, &S->shape.ctas);
        if (s != QB_OK) return s;
        if (c.batch.ctas > 0) S->shape.ctas = std::min(S->shape.ctas, c.batch.ctas);
        QB_CUDA(cudaStreamCreateWithFlags(&S->upload_stream, cudaStreamNonBlocking));
        QB_CUDA(cudaStreamCreateWithFlags(&S->tick_stream, cudaStreamNonBlocking));
        for (int k = 0; k < c.residual_streams; ++k) {
            cudaStream_t st;
            QB_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
            S->resid_streams.push_back(st);
        }
        QB_CUDA(cudaEventCreateWithFlags(&S->upload_ev, cudaEventDisableTiming));
        QB_CUDA(cudaEventCreateWithFlags(&S->tick_ev, cudaEventDisableTiming));
        // partitions of the SMs for cooperative sweeps (QB_SERVER_PARTS overrides)
        int parts = c.coop_parts > 0 ? c.coop_parts : kDefaultParts;
        if (const char* ev = std::getenv("QB_SERVER_PARTS")) parts = std::max(1, std::atoi(ev));
        const int full_resid = resid_lockstep_grid(), full_qubo = qubo_lockstep_grid();
        parts = std::max(1, std::min(parts, std::min(full_resid, full_qubo)));
        S->parts = parts;
        S->full_resid = full_resid;
        S->full_qubo = full_qubo;
        S->coop_budget = std::min(full_resid, full_qubo);
        S->coop_cap = std::max(1, S->coop_budget / 2);
        if (parts > 1) {
            for (int k = 0; k < parts; ++k) {
                cudaStream_t st;
                QB_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
                S->part_streams.push_back(st);
            }
            S->part_run.assign(size_t(parts), nullptr);
        }
        if (const char* fa = std::getenv("QB_SERVER_FAIL_ADMIT")) S->fail_admission = std::atoll(fa);
        qb_server* raw = S.release();
        raw->worker = std::thread(worker_main, raw);
        *out = raw;
        return QB_OK;
    });
}

extern "C" qb_status qb_server_submit(qb_server* S, qb_problem* p, const qb_schedule* sch, uint32_t n_branches,
                                      uint64_t seed_offset, uint64_t* id) {
    return qb::guarded("qb_server_submit", [&]() -> qb_status {
        if (!S || !p || !sch || !id) return fail(QB_EINVAL, "qb_server_submit: null argument");
        if (p->device != S->device) return fail(QB_EINVAL, "qb_server_submit: the problem is on another device");
        if (n_branches < 1 || n_branches > (1u << 20)) return fail(QB_EINVAL, "qb_server_submit: n_branches must be in [1, 2^20]");
        if (sch->anneal_sweeps < 0 || sch->hold_sweeps < 0 || sch->anneal_sweeps + sch->hold_sweeps < 1 ||
            !(sch->t_hot > 0.0) || !(sch->t_cold > 0.0) || !std::isfinite(sch->t_hot) || !std::isfinite(sch->t_cold) ||
            sch->refresh_sweeps < 0)
            return fail(QB_EINVAL, "qb_server_submit: bad schedule");

        std::unique_ptr<Request> r(new (std::nothrow) Request());
        if (!r) return fail(QB_ENOMEM, "qb_server_submit: out of host memory");
        r->prob = p;
        r->sched = *sch;
        r->kind = p->kind;
        r->R = int(n_branches);
        r->n = p->kind == QB_KIND_ISING ? p->ising.n : p->kind == QB_KIND_QUBO ? p->qubo.n : p->resid.n;
        r->coop = p->kind == QB_KIND_QUBO || (p->kind == QB_KIND_RESIDUAL && p->resid.variant == QB_RESID_LOCKSTEP);
        r->exclusive = r->coop && S->parts == 1;
        if (r->coop && !r->exclusive && p->kind == QB_KIND_QUBO) r->ctas = coop_grid(S, p);
        r->sweeps = sch->anneal_sweeps + sch->hold_sweeps;
        if (r->coop && !r->exclusive && p->kind == QB_KIND_RESIDUAL) {
            // a lockstep residual problem runs on one partition: plan it for
            // that grid (same colouring, same branches) from its host copy;
            // one without a host copy runs on the whole device
            {
                std::lock_guard<std::mutex> lk(S->mu);
                for (auto& kv : S->reqs)
                    if (kv.second->prob == p && (kv.second->state == QB_REQ_PENDING || kv.second->state == QB_REQ_RUNNING))
                        return fail(QB_EBUSY, "qb_server_submit: the problem already has a request in flight");
                if (std::find(S->submitting.begin(), S->submitting.end(), p) != S->submitting.end())
                    return fail(QB_EBUSY, "qb_server_submit: the problem is being submitted by another thread");
                S->submitting.push_back(p);
            }
            qb_status ps = QB_OK;
            if (p->host.row_ptr.empty()) r->exclusive = true;
            else ps = replan_residual(p, r->ctas = coop_grid(S, p));
            std::lock_guard<std::mutex> lk(S->mu);
            S->submitting.erase(std::find(S->submitting.begin(), S->submitting.end(), p));
            if (ps != QB_OK) return ps;
        }
        r->seed0 = 1 + seed_offset;
        if (p->kind == QB_KIND_ISING) {
            r->charge_work = ising_work_bytes(p, r->R, r->sweeps);
            r->charge_results = ising_result_bytes(r->n, r->R);
        } else {
            r->charge_work = resid_work_bytes(p, r->R, r->sweeps);
            r->charge_results = resid_result_bytes(r->n, r->R);
        }
        r->t_submit = now_s();
        std::lock_guard<std::mutex> lk(S->mu);
        if (S->stop) return fail(QB_EINVAL, "qb_server_submit: the server is stopping");
        if (S->cfg.max_pending > 0 && int64_t(S->pending.size()) >= S->cfg.max_pending)
            return fail(QB_EBUSY, "qb_server_submit: the queue is full");
        for (auto& kv : S->reqs)
            if (kv.second->prob == p && (kv.second->state == QB_REQ_PENDING || kv.second->state == QB_REQ_RUNNING))
                return fail(QB_EBUSY, "qb_server_submit: the problem already has a request in flight");
        r->id = S->next_id++;
        *id = r->id;
        S->pending.push_back(r->id);
        S->reqs[r->id] = std::move(r);
        ++S->submitted;
        S->kick = true;
        S->cv_work.notify_one();
        return QB_OK;
    });
}

extern "C" qb_status qb_server_poll(qb_server* S, uint64_t id, int32_t* state) {
    if (!S || !state) return fail(QB_EINVAL, "qb_server_poll: null argument");
    std::lock_guard<std::mutex> lk(S->mu);
    Request* r = find_locked(S, id);
    if (!r) return fail(QB_EINVAL, "qb_server_poll: unknown request");
    *state = r->state;
    return QB_OK;
}

extern "C" qb_status qb_server_wait(qb_server* S, uint64_t id, int32_t timeout_ms) {
    if (!S) return fail(QB_EINVAL, "qb_server_wait: null server");
    std::unique_lock<std::mutex> lk(S->mu);
    Request* r = find_locked(S, id);
    if (!r) return fail(QB_EINVAL, "qb_server_wait: unknown request");
    auto done = [&] { return r->state >= QB_REQ_DONE; };
    if (timeout_ms < 0) S->cv_done.wait(lk, done);
    else if (!S->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), done))
        return fail(QB_ETIMEDOUT, "qb_server_wait: the request is not finished");
    if (r->state == QB_REQ_DONE) return QB_OK;
    if (r->state == QB_REQ_CANCELLED) return fail(QB_ECANCELLED, "qb_server_wait: the request was cancelled");
    return fail(r->status, r->error);
}

extern "C" qb_status qb_server_cancel(qb_server* S, uint64_t id) {
    if (!S) return fail(QB_EINVAL, "qb_server_cancel: null server");
    std::lock_guard<std::mutex> lk(S->mu);
    Request* r = find_locked(S, id);
    if (!r) return fail(QB_EINVAL, "qb_server_cancel: unknown request");
    if (r->state >= QB_REQ_DONE) return fail(QB_EINVAL, "qb_server_cancel: the request has finished");
    r->cancel = true;
    S->kick = true;
    S->cv_work.notify_one();
    return QB_OK;
}

extern "C" qb_status qb_server_request_info(qb_server* S, uint64_t id, qb_request_info* info) {
    if (!S || !info) return fail(QB_EINVAL, "qb_server_request_info: null argument");
    std::lock_guard<std::mutex> lk(S->mu);
    Request* r = find_locked(S, id);
    if (!r) return fail(QB_EINVAL, "qb_server_request_info: unknown request");
    std::memset(info, 0, sizeof(*info));
    info->state = r->state;
    info->status = r->status;
    info->kind = r->kind;
    info->n = r->n;
    info->n_branches = r->R;
    info->sweeps = r->sweeps;
    info->attempts = int64_t(r->R) * r->sweeps * r->n;
    info->device_bytes = r->charge_work + r->charge_results;
    info->t_submit = r->t_submit;
    info->t_admit = r->t_admit;
    info->t_done = r->t_done;
    return QB_OK;
}

namespace {
qb_status result_copy(qb_server* S, uint64_t id, void* dst, const char* what, int which) {
    if (!S || !dst) return fail(QB_EINVAL, std::string(what) + ": null argument");
    const void* src = nullptr;
    size_t bytes = 0;
    int dev = 0;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        Request* r = find_locked(S, id);
        if (!r) return fail(QB_EINVAL, std::string(what) + ": unknown request");
        if (r->state != QB_REQ_DONE) return fail(QB_EBUSY, std::string(what) + ": the request has not finished");
        dev = S->device;
        switch (which) {
            case 0: src = r->d_x.p; bytes = size_t(r->R) * size_t(r->n); break;
            case 1: src = r->d_p.p; bytes = size_t(r->n) * 4; break;
            case 2:
                if (r->kind != QB_KIND_ISING) return fail(QB_EINVAL, std::string(what) + ": ising requests only");
                src = r->d_e.p; bytes = size_t(r->R) * 8; break;
            default:
                if (r->kind == QB_KIND_ISING) return fail(QB_EINVAL, std::string(what) + ": residual or qubo requests only");
                src = r->d_ef64.p; bytes = size_t(r->R) * 8; break;
        }
        if (!src) return fail(QB_EINVAL, std::string(what) + ": the results were released");
    }
    // results of a finished request are immutable until released (which this
    // thread's caller must not race with its own reads)
    QB_CUDA(cudaSetDevice(dev));
    QB_CUDA(cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost));
    return QB_OK;
}
}  // namespace

extern "C" qb_status qb_server_result_branches(qb_server* S, uint64_t id, uint8_t* x) {
    return result_copy(S, id, x, "qb_server_result_branches", 0);
}
extern "C" qb_status qb_server_result_marginals(qb_server* S, uint64_t id, float* p) {
    return result_copy(S, id, p, "qb_server_result_marginals", 1);
}
extern "C" qb_status qb_server_result_energies_i64(qb_server* S, uint64_t id, int64_t* e) {
    return result_copy(S, id, e, "qb_server_result_energies_i64", 2);
}
extern "C" qb_status qb_server_result_energies_f64(qb_server* S, uint64_t id, double* e) {
    return result_copy(S, id, e, "qb_server_result_energies_f64", 3);
}

extern "C" qb_status qb_server_release(qb_server* S, uint64_t id) {
    if (!S) return fail(QB_EINVAL, "qb_server_release: null server");
    std::unique_ptr<Request> r;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        auto it = S->reqs.find(id);
        if (it == S->reqs.end()) return fail(QB_EINVAL, "qb_server_release: unknown request");
        if (it->second->state < QB_REQ_DONE) return fail(QB_EBUSY, "qb_server_release: the request has not finished");
        S->bytes_in_use -= it->second->charge_results;
        it->second->charge_results = 0;
        r = std::move(it->second);
        S->reqs.erase(it);
        S->kick = true;
        S->cv_work.notify_one();
    }
    cudaSetDevice(S->device);
    drop_results(r.get());
    return QB_OK;
}

extern "C" qb_status qb_server_stats_get(qb_server* S, qb_server_stats* st) {
    if (!S || !st) return fail(QB_EINVAL, "qb_server_stats_get: null argument");
    std::lock_guard<std::mutex> lk(S->mu);
    std::memset(st, 0, sizeof(*st));
    st->submitted = S->submitted;
    st->completed = S->completed;
    st->failed = S->failed;
    st->cancelled = S->cancelled;
    st->pending = int64_t(S->pending.size());
    st->active = S->active;
    st->ticks = S->ticks;
    st->bytes_in_use = S->bytes_in_use;
    st->peak_bytes = S->peak_bytes;
    st->budget_bytes = S->budget;
    st->attempts_done = S->attempts_done;
    return QB_OK;
}

extern "C" void qb_server_destroy(qb_server* S) {
    if (!S) return;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stop = true;
        for (uint64_t id : S->pending) {
            Request* r = find_locked(S, id);
            if (r && r->state == QB_REQ_PENDING) finish_locked(S, r, QB_REQ_CANCELLED, QB_ECANCELLED, "server stopped");
        }
        S->pending.clear();
        S->kick = true;
        S->cv_work.notify_one();
    }
    if (S->worker.joinable()) S->worker.join();
    cudaSetDevice(S->device);
    for (auto& kv : S->reqs) drop_results(kv.second.get());
    S->reqs.clear();
    if (S->exec) cudaGraphExecDestroy(S->exec);
    if (S->graph) cudaGraphDestroy(S->graph);
    if (S->tick_stream) cudaStreamSynchronize(S->tick_stream);
    if (S->h_tick) cudaFreeHost(S->h_tick);
    S->d_tick.release();
    for (cudaStream_t st : S->resid_streams) {
        cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
    }
    for (cudaStream_t st : S->part_streams) {
        cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
    }
    if (S->upload_stream) {
        cudaStreamSynchronize(S->upload_stream);
        cudaStreamDestroy(S->upload_stream);
    }
    if (S->tick_stream) cudaStreamDestroy(S->tick_stream);
    if (S->upload_ev) cudaEventDestroy(S->upload_ev);
    if (S->tick_ev) cudaEventDestroy(S->tick_ev);
    delete S;
}
