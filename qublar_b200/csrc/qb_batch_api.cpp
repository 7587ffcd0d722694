// Batch entry points of the C ABI: packing many ising problems into work
// items for the persistent kernel, the output arenas, and the autotuner.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <tuple>
#include <vector>

#include "qb_batch.hpp"
#include "qb_internal.hpp"

using namespace qb;

struct qb_batch {
    struct Inst {
        qb_problem* prob = nullptr;
        int n = 0;
        int R = 0;
        int sweeps = 0;
        uint64_t seed0 = 0;
        int64_t x_off = 0;     // bytes into d_x (and entries into d_f)
        int64_t e_off = 0;     // entries into d_e
        int64_t p_off = 0;     // entries into d_p
        int64_t temp_off = 0;  // entries into d_temp
        qb_schedule sched{};
    };
    int device = 0;
    cudaStream_t stream = nullptr;
    std::vector<Inst> inst;
    qb_batch_config cfg{};
    int work_items = 0;
    int global_items = 0;
    int ctas = 0;
    int launches = 0;
    int64_t attempts = 0;
    int64_t total_bits = 0;
    int64_t total_x = 0;
    int64_t total_r = 0;
    int64_t total_nnz = 0;
    std::vector<IsingItem> h_items;
    std::vector<BatchInstDev> h_inst;
    DevBuf d_items, d_counter, d_x, d_f, d_e, d_p, d_temp, d_state, d_inst;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev2 = nullptr;
    bool synced = false;
};

namespace {

constexpr int kDefaultThreads = 512;
constexpr int kDefaultSmem = 96 * 1024;
constexpr int kDefaultGroup = 32;

bool pow2(int v) { return v > 0 && (v & (v - 1)) == 0; }

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

qb_status check_sched(const qb_schedule& s) {
    if (s.anneal_sweeps < 0 || s.hold_sweeps < 0 || s.anneal_sweeps + s.hold_sweeps < 1)
        return fail(QB_EINVAL, "batch: a schedule needs at least one sweep");
    if (!(s.t_hot > 0.0) || !(s.t_cold > 0.0) || !std::isfinite(s.t_hot) || !std::isfinite(s.t_cold))
        return fail(QB_EINVAL, "batch: temperatures must be positive and finite");
    return QB_OK;
}

qb_status resolve_config(const qb_batch_config* in, qb_batch_config* out) {
    qb_batch_config c{};
    if (in) c = *in;
    if (c.threads == 0) c.threads = kDefaultThreads;
    if (c.smem_bytes == 0) c.smem_bytes = kDefaultSmem;
    if (c.max_group == 0) c.max_group = kDefaultGroup;
    if (c.threads < 32 || c.threads > 1024 || c.threads % 32)
        return fail(QB_EINVAL, "batch: threads must be a multiple of 32 in [32, 1024]");
    if (!pow2(c.max_group) || c.max_group > kBatchMaxGroup)
        return fail(QB_EINVAL, "batch: max_group must be a power of two in [1, 32]");
    if (c.smem_bytes < 0) return fail(QB_EINVAL, "batch: smem_bytes must be non-negative");
    if (c.ctas < 0) return fail(QB_EINVAL, "batch: ctas must be non-negative");
    *out = c;
    return QB_OK;
}

// Host-side checks of the items, before any device call.
qb_status check_items(const qb_batch_item* items, int32_t count) {
    if (!items || count < 1) return fail(QB_EINVAL, "batch: needs at least one item");
    for (int32_t k = 0; k < count; ++k) {
        const qb_batch_item& it = items[k];
        if (!it.problem) return fail(QB_EINVAL, "batch: null problem");
        if (it.problem->kind != QB_KIND_ISING) return fail(QB_EINVAL, "batch: ising problems only");
        if (it.problem->device != items[0].problem->device) return fail(QB_EINVAL, "batch: problems on different devices");
        if (it.n_branches < 1 || it.n_branches > (1u << 20)) return fail(QB_EINVAL, "batch: n_branches must be in [1, 2^20]");
        qb_status s = check_sched(it.schedule);
        if (s != QB_OK) return s;
    }
    return QB_OK;
}

// Validates the instances and lays out the output arenas and temperature
// tables (identical schedules share one table).
qb_status prepare(const qb_batch_item* items, int32_t count, const qb_opts* opts, qb_batch* b) {
    qb_status s0 = check_items(items, count);
    if (s0 != QB_OK) return s0;
    b->stream = opts ? static_cast<cudaStream_t>(opts->stream) : nullptr;
    b->device = items[0].problem ? items[0].problem->device : 0;
    b->inst.resize(size_t(count));
    std::vector<std::pair<std::tuple<double, double, int, int>, int64_t>> tables;
    std::vector<double> temps;
    int64_t x_off = 0, e_off = 0, p_off = 0;
    for (int32_t k = 0; k < count; ++k) {
        const qb_batch_item& it = items[k];
        qb_batch::Inst& I = b->inst[size_t(k)];
        I.prob = it.problem;
        I.n = it.problem->ising.n;
        I.R = int(it.n_branches);
        I.sweeps = it.schedule.anneal_sweeps + it.schedule.hold_sweeps;
        I.seed0 = 1 + it.seed_offset;
        I.sched = it.schedule;
        I.x_off = x_off;
        I.e_off = e_off;
        I.p_off = p_off;
        x_off += int64_t(I.R) * I.n;
        e_off += I.R;
        p_off += I.n;
        b->attempts += int64_t(I.R) * I.sweeps * I.n;
        b->total_nnz += it.problem->ising.nnz;
        const auto key = std::make_tuple(it.schedule.t_hot, it.schedule.t_cold, it.schedule.anneal_sweeps,
                                         it.schedule.hold_sweeps);
        int64_t off = -1;
        for (const auto& t : tables)
            if (t.first == key) off = t.second;
        if (off < 0) {
            off = int64_t(temps.size());
            const std::vector<double> t = temperatures(it.schedule);
            temps.insert(temps.end(), t.begin(), t.end());
            tables.emplace_back(key, off);
        }
        I.temp_off = off;
    }
    b->total_x = x_off;
    b->total_r = e_off;
    b->total_bits = p_off;
    QB_CUDA(cudaSetDevice(b->device));
    qb_status s;
    for (auto& I : b->inst)
        if ((s = problem_upload(I.prob, b->stream)) != QB_OK) return s;
    if ((s = b->d_x.alloc(size_t(x_off)))) return s;
    if ((s = b->d_f.alloc(size_t(x_off) * 4))) return s;
    if ((s = b->d_e.alloc(size_t(e_off) * 8))) return s;
    if ((s = b->d_p.alloc(size_t(p_off) * 4))) return s;
    if ((s = b->d_counter.alloc(sizeof(int)))) return s;
    if ((s = upload_vec(b->d_temp, temps, b->stream))) return s;
    b->h_inst.resize(b->inst.size());
    for (size_t k = 0; k < b->inst.size(); ++k)
        b->h_inst[k] = BatchInstDev{b->inst[k].x_off, b->inst[k].p_off, b->inst[k].n, b->inst[k].R};
    if ((s = upload_vec(b->d_inst, b->h_inst, b->stream))) return s;
    QB_CUDA(cudaStreamSynchronize(b->stream));
    return QB_OK;
}

struct Unit {
    int inst;
    int r0;
    int G;
    bool global;
    int64_t state_off;   // bytes into the global-state arena
    double cost;
};

// Splits every instance into replica groups for the shape `c`, sorts the
// units largest first and writes their descriptors. sample > 0 replaces each
// schedule by `sample` of its sweeps, evenly spaced (autotuning), read from
// sample_temp (one table of `sample` entries per instance).
qb_status build_items(qb_batch* b, const qb_batch_config& c, int sample, const double* sample_temp,
                      std::vector<IsingItem>& out) {
    std::vector<Unit> units;
    int64_t state_bytes = 0;
    for (size_t k = 0; k < b->inst.size(); ++k) {
        const qb_batch::Inst& I = b->inst[k];
        const IsingPlan& P = I.prob->ising;
        int r0 = 0;
        while (r0 < I.R) {
            const int G0 = std::min(c.max_group, floor_pow2(I.R - r0));
            int G = G0;
            while (G > 1 && batch_item_smem(I.n, G) > size_t(c.smem_bytes)) G /= 2;
            const bool global = batch_item_smem(I.n, G) > size_t(c.smem_bytes);
            if (global) G = G0;   // in global memory a wide group keeps the state accesses coalesced
            Unit u{int(k), r0, G, global, 0, 0.0};
            if (global) {
                u.state_off = state_bytes;
                state_bytes += int64_t(batch_item_smem(I.n, G) + 256) / 256 * 256;
            }
            const int sweeps = sample > 0 ? sample : I.sweeps;
            u.cost = double(G) * double(sweeps) * (double(I.n) + 0.25 * double(P.nnz)) * (global ? 3.0 : 1.0);
            units.push_back(u);
            r0 += G;
        }
    }
    std::stable_sort(units.begin(), units.end(), [](const Unit& a, const Unit& z) { return a.cost > z.cost; });
    if (state_bytes > int64_t(b->d_state.bytes)) {
        qb_status s = b->d_state.alloc(size_t(state_bytes));
        if (s != QB_OK) return s;
    }
    out.resize(units.size());
    int n_global = 0;
    for (size_t q = 0; q < units.size(); ++q) {
        const Unit& u = units[q];
        const qb_batch::Inst& I = b->inst[size_t(u.inst)];
        const IsingPlan& P = I.prob->ising;
        IsingItem& it = out[q];
        std::memset(&it, 0, sizeof(it));
        it.class_ptr = P.d_class_ptr.as<int32_t>();
        it.row = P.d_row.as<int32_t>();
        it.adj = P.d_adj.as<int32_t>();
        it.w = P.d_w.p;
        it.f0 = P.d_f0.as<int32_t>();
        it.order = P.d_order.as<int32_t>();
        it.temp = sample > 0 ? sample_temp + size_t(u.inst) * size_t(sample) : b->d_temp.as<double>() + I.temp_off;
        it.e_acc = b->d_e.as<long long>() + I.e_off + u.r0;
        it.x_out = b->d_x.as<uint8_t>() + I.x_off + int64_t(u.r0) * I.n;
        it.f_out = b->d_f.as<int32_t>() + I.x_off + int64_t(u.r0) * I.n;
        it.seed0 = I.seed0 + uint64_t(u.r0);
        it.n = I.n;
        it.n_colours = P.col.n_colours();
        it.log2g = log2i(u.G);
        it.sweep0 = 0;
        it.sweep1 = sample > 0 ? sample : I.sweeps;
        it.flags = kItemInit | kItemFinal | item_rbase_flags(u.r0);
        if (u.global) {
            unsigned char* base = b->d_state.as<unsigned char>() + u.state_off;
            it.f_state = reinterpret_cast<int32_t*>(base);
            it.s_state = reinterpret_cast<int8_t*>(base + size_t(I.n) * size_t(u.G) * 4);
            it.flags |= kItemGlobal;
            ++n_global;
        }
        it.bound = int32_t(P.B);
        it.wbytes = P.weight_bytes;
    }
    b->global_items = n_global;
    return QB_OK;
}

qb_status run_items(qb_batch* b, const qb_batch_config& c, const std::vector<IsingItem>& items) {
    qb_status s;
    if ((s = b->d_items.alloc(items.size() * sizeof(IsingItem)))) return s;
    QB_CUDA(cudaMemcpyAsync(b->d_items.p, items.data(), items.size() * sizeof(IsingItem), cudaMemcpyHostToDevice,
                            b->stream));
    BatchShape sh;
    sh.threads = c.threads;
    sh.smem_bytes = c.smem_bytes;
    sh.ctas = c.ctas;
    if (sh.ctas <= 0 && (s = batch_ctas(sh, &sh.ctas))) return s;
    b->ctas = std::min<int>(sh.ctas, int(items.size()));
    return launch_ising_batch(b->d_items.as<IsingItem>(), int(items.size()), b->d_counter.as<int>(), sh, b->stream);
}

qb_status wait(qb_batch* b) {
    if (!b->synced) {
        QB_CUDA(cudaSetDevice(b->device));
        QB_CUDA(cudaStreamSynchronize(b->stream));
        b->synced = true;
    }
    return QB_OK;
}

qb_status item_of(qb_batch* b, int32_t item, const void* dst) {
    if (!b) return fail(QB_EINVAL, "batch: null batch");
    if (!dst) return fail(QB_EINVAL, "batch: null output buffer");
    if (item < 0 || size_t(item) >= b->inst.size()) return fail(QB_EINVAL, "batch: item index out of range");
    return wait(b);
}

std::mutex g_tune_mu;
std::map<std::tuple<int, int64_t, int64_t, int64_t, int>, qb_batch_config> g_tuned;

}  // namespace

extern "C" qb_status qb_batch_autotune(const qb_batch_item* items, int32_t count, int32_t sample_sweeps,
                                       const qb_opts* opts, qb_batch_config* out) {
    return qb::guarded("qb_batch_autotune", [&]() -> qb_status {
        if (!out) return fail(QB_EINVAL, "qb_batch_autotune: null output");
        if (sample_sweeps < 0) return fail(QB_EINVAL, "qb_batch_autotune: sample_sweeps must be non-negative");
        qb_status s0 = check_items(items, count);
        if (s0 != QB_OK) return s0;
        QB_CUDA(cudaSetDevice(items[0].problem->device));
        const int S = sample_sweeps ? sample_sweeps : 8;
        qb_batch* b = new (std::nothrow) qb_batch();
        if (!b) return fail(QB_ENOMEM, "qb_batch_autotune: out of host memory");
        qb_status s = prepare(items, count, opts, b);
        if (s != QB_OK) {
            qb_batch_destroy(b);
            return s;
        }
        const auto key = std::make_tuple(count, b->total_bits, b->total_nnz, b->total_r, b->device);
        {
            std::lock_guard<std::mutex> lk(g_tune_mu);
            auto hit = g_tuned.find(key);
            if (hit != g_tuned.end()) {
                *out = hit->second;
                qb_batch_destroy(b);
                return QB_OK;
            }
        }
        // each instance's schedule sampled at S evenly spaced sweeps
        std::vector<double> st(b->inst.size() * size_t(S));
        for (size_t k = 0; k < b->inst.size(); ++k) {
            const std::vector<double> t = temperatures(b->inst[k].sched);
            for (int j = 0; j < S; ++j) st[k * size_t(S) + size_t(j)] = t[size_t(int64_t(j) * int64_t(t.size()) / S)];
        }
        DevBuf d_st;
        if ((s = upload_vec(d_st, st, b->stream))) {
            qb_batch_destroy(b);
            return s;
        }
        const int cap = batch_max_smem();
        const int threads_c[] = {256, 512, 1024};
        const int smem_c[] = {48 * 1024, 96 * 1024, cap};
        const int group_c[] = {8, 16, 32};
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        // time one shape on `its`; < 0 when it does not fit an SM
        auto time_shape = [&](const qb_batch_config& c, const std::vector<IsingItem>& its, float* ms) -> qb_status {
            *ms = -1.0f;
            BatchShape sh{c.threads, c.smem_bytes, 0};
            int ctas = 0;
            if (batch_ctas(sh, &ctas) != QB_OK) return QB_OK;   // shape does not fit an SM
            cudaEventRecord(e0, b->stream);
            qb_status r = run_items(b, c, its);
            if (r != QB_OK) return r;
            cudaEventRecord(e1, b->stream);
            if (cudaEventSynchronize(e1) != cudaSuccess)
                return cuda_fail(cudaGetLastError(), "cudaEventSynchronize", __FILE__, __LINE__);
            cudaEventElapsedTime(ms, e0, e1);
            return QB_OK;
        };
        // every shape on the short sample, then the three fastest again on a
        // sample four times longer (short samples cannot separate close shapes)
        std::vector<std::pair<float, qb_batch_config>> timed;
        for (int th : threads_c)
            for (int sm : smem_c)
                for (int g : group_c) {
                    qb_batch_config c{th, std::min(sm, cap), g, 0};
                    std::vector<IsingItem> its;
                    if ((s = build_items(b, c, S, d_st.as<double>(), its)) != QB_OK) break;
                    float ms = 0.0f;
                    if ((s = time_shape(c, its, &ms)) != QB_OK) break;
                    if (ms >= 0.0f) timed.emplace_back(ms, c);
                }
        float best = -1.0f;
        qb_batch_config best_c{};
        if (s == QB_OK && !timed.empty()) {
            std::stable_sort(timed.begin(), timed.end(),
                             [](const std::pair<float, qb_batch_config>& a, const std::pair<float, qb_batch_config>& b_) {
                                 return a.first < b_.first;
                             });
            const int S4 = 4 * S;
            std::vector<double> st4(b->inst.size() * size_t(S4));
            for (size_t k = 0; k < b->inst.size(); ++k) {
                const std::vector<double> t = temperatures(b->inst[k].sched);
                for (int j = 0; j < S4; ++j)
                    st4[k * size_t(S4) + size_t(j)] = t[size_t(int64_t(j) * int64_t(t.size()) / S4)];
            }
            DevBuf d_st4;
            s = upload_vec(d_st4, st4, b->stream);
            for (size_t q = 0; s == QB_OK && q < std::min<size_t>(3, timed.size()); ++q) {
                std::vector<IsingItem> its;
                if ((s = build_items(b, timed[q].second, S4, d_st4.as<double>(), its)) != QB_OK) break;
                float ms = 0.0f;
                if ((s = time_shape(timed[q].second, its, &ms)) != QB_OK) break;
                if (ms >= 0.0f && (best < 0.0f || ms < best)) {
                    best = ms;
                    best_c = timed[q].second;
                }
            }
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        qb_batch_destroy(b);
        if (s != QB_OK) return s;
        if (best < 0.0f) return fail(QB_EREFUSED, "qb_batch_autotune: no candidate shape fits the device");
        {
            std::lock_guard<std::mutex> lk(g_tune_mu);
            g_tuned[key] = best_c;
        }
        *out = best_c;
        return QB_OK;
    });
}

extern "C" qb_status qb_solve_batch(const qb_batch_item* items, int32_t count, const qb_batch_config* cfg,
                                    const qb_opts* opts, qb_batch** out) {
    return qb::guarded("qb_solve_batch", [&]() -> qb_status {
        if (!out) return fail(QB_EINVAL, "qb_solve_batch: null output");
        *out = nullptr;
        qb_status s = check_items(items, count);
        if (s != QB_OK) return s;
        qb_batch_config c{};
        if ((s = resolve_config(cfg, &c)) != QB_OK) return s;
        QB_CUDA(cudaSetDevice(items[0].problem->device));
        const int cap = batch_max_smem();
        if (cap <= 0) return fail(QB_ECUDA, "batch: cannot read the device's shared-memory limit");
        c.smem_bytes = std::min(c.smem_bytes, cap);
        qb_batch* b = new (std::nothrow) qb_batch();
        if (!b) return fail(QB_ENOMEM, "qb_solve_batch: out of host memory");
        auto bail = [&](qb_status e) {
            qb_batch_destroy(b);
            return e;
        };
        if ((s = prepare(items, count, opts, b)) != QB_OK) return bail(s);
        b->cfg = c;
        if ((s = build_items(b, c, 0, nullptr, b->h_items)) != QB_OK) return bail(s);
        b->work_items = int(b->h_items.size());
        if (cudaEventCreate(&b->ev0) != cudaSuccess || cudaEventCreate(&b->ev1) != cudaSuccess ||
            cudaEventCreate(&b->ev2) != cudaSuccess)
            return bail(cuda_fail(cudaGetLastError(), "cudaEventCreate", __FILE__, __LINE__));
        // the descriptors go up before the timed region
        if ((s = b->d_items.alloc(b->h_items.size() * sizeof(IsingItem)))) return bail(s);
        QB_CUDA(cudaMemcpyAsync(b->d_items.p, b->h_items.data(), b->h_items.size() * sizeof(IsingItem),
                                cudaMemcpyHostToDevice, b->stream));
        BatchShape sh{c.threads, c.smem_bytes, c.ctas};
        if (sh.ctas <= 0 && (s = batch_ctas(sh, &sh.ctas))) return bail(s);
        b->ctas = std::min<int>(sh.ctas, b->work_items);
        cudaEventRecord(b->ev0, b->stream);
        if ((s = launch_ising_batch(b->d_items.as<IsingItem>(), b->work_items, b->d_counter.as<int>(), sh, b->stream)))
            return bail(s);
        cudaEventRecord(b->ev1, b->stream);
        if ((s = launch_batch_marginals(b->d_x.as<uint8_t>(), b->d_inst.as<BatchInstDev>(), int(b->inst.size()),
                                        b->total_bits, b->d_p.as<float>(), b->stream)))
            return bail(s);
        cudaEventRecord(b->ev2, b->stream);
        b->launches = 2;
        *out = b;
        return QB_OK;
    });
}

extern "C" qb_status qb_batch_info_get(qb_batch* b, qb_batch_info* info) {
    if (!b || !info) return fail(QB_EINVAL, "qb_batch_info_get: null argument");
    qb_status s = wait(b);
    if (s != QB_OK) return s;
    std::memset(info, 0, sizeof(*info));
    info->items = int32_t(b->inst.size());
    info->work_items = b->work_items;
    info->global_items = b->global_items;
    info->threads = b->cfg.threads;
    info->smem_bytes = b->cfg.smem_bytes;
    info->max_group = b->cfg.max_group;
    info->ctas = b->ctas;
    info->launches = b->launches;
    info->attempts = b->attempts;
    QB_CUDA(cudaEventElapsedTime(&info->anneal_ms, b->ev0, b->ev1));
    QB_CUDA(cudaEventElapsedTime(&info->total_ms, b->ev0, b->ev2));
    return QB_OK;
}

extern "C" qb_status qb_batch_branches(qb_batch* b, int32_t item, uint8_t* x) {
    qb_status s = item_of(b, item, x);
    if (s != QB_OK) return s;
    const qb_batch::Inst& I = b->inst[size_t(item)];
    QB_CUDA(cudaMemcpy(x, b->d_x.as<uint8_t>() + I.x_off, size_t(I.R) * size_t(I.n), cudaMemcpyDeviceToHost));
    return QB_OK;
}

extern "C" qb_status qb_batch_energies_i64(qb_batch* b, int32_t item, int64_t* e) {
    qb_status s = item_of(b, item, e);
    if (s != QB_OK) return s;
    const qb_batch::Inst& I = b->inst[size_t(item)];
    QB_CUDA(cudaMemcpy(e, b->d_e.as<long long>() + I.e_off, size_t(I.R) * 8, cudaMemcpyDeviceToHost));
    return QB_OK;
}

extern "C" qb_status qb_batch_fields_i64(qb_batch* b, int32_t item, int64_t* f) {
    qb_status s = item_of(b, item, f);
    if (s != QB_OK) return s;
    const qb_batch::Inst& I = b->inst[size_t(item)];
    std::vector<int32_t> f32(size_t(I.R) * size_t(I.n));
    QB_CUDA(cudaMemcpy(f32.data(), b->d_f.as<int32_t>() + I.x_off, f32.size() * 4, cudaMemcpyDeviceToHost));
    for (size_t k = 0; k < f32.size(); ++k) f[k] = f32[k];
    return QB_OK;
}

extern "C" qb_status qb_batch_marginals(qb_batch* b, int32_t item, float* p) {
    qb_status s = item_of(b, item, p);
    if (s != QB_OK) return s;
    const qb_batch::Inst& I = b->inst[size_t(item)];
    QB_CUDA(cudaMemcpy(p, b->d_p.as<float>() + I.p_off, size_t(I.n) * 4, cudaMemcpyDeviceToHost));
    return QB_OK;
}

extern "C" void qb_batch_destroy(qb_batch* b) {
    if (!b) return;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    else cudaDeviceSynchronize();
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->ev2) cudaEventDestroy(b->ev2);
    delete b;
}

namespace qb {

namespace {
constexpr int kPackedMinReplicas = 128;
constexpr int kPackedThreads = 256;

void take(DevBuf& dst, DevBuf& src) {
    dst.release();
    dst.p = src.p;
    dst.bytes = src.bytes;
    dst.pooled = src.pooled;
    dst.pool_stream = src.pool_stream;
    src.p = nullptr;
    src.bytes = 0;
    src.pooled = false;
}
}  // namespace

bool packed_replicas_fit(const IsingPlan& P, int R) {
    // opt-in (QB_PACKED_REPLICAS=1): on dense small graphs one CTA per replica
    // with smaller CTAs is the faster form
    const char* on = std::getenv("QB_PACKED_REPLICAS");
    if (R < kPackedMinReplicas || !on || std::atoi(on) == 0) return false;
    const int cap = batch_max_smem();
    return cap > 0 && batch_item_smem(P.n, 1) <= size_t(std::min(cap, kDefaultSmem));
}

qb_status packed_replicas(qb_problem* p, const qb_schedule& s, int R, uint64_t seed_offset, const qb_opts* opts,
                          qb_batch** keep, DevBuf& x, DevBuf& f, DevBuf& e, DevBuf& pm) {
    *keep = nullptr;
    BatchShape sh{kPackedThreads, std::min(batch_max_smem(), kDefaultSmem), 0};
    qb_status st = batch_ctas(sh, &sh.ctas);
    if (st != QB_OK) return st;
    // the smallest group that keeps every item on a CTA of the first wave
    int G = 1;
    while (G < kBatchMaxGroup && (R + G - 1) / G > sh.ctas) G *= 2;
    while (G > 1 && batch_item_smem(p->ising.n, G) > size_t(sh.smem_bytes)) G /= 2;
    const qb_batch_item item{p, s, uint32_t(R), seed_offset};
    qb_batch_config cfg{kPackedThreads, sh.smem_bytes, G, 0};
    qb_batch* b = nullptr;
    if ((st = qb_solve_batch(&item, 1, &cfg, opts, &b)) != QB_OK) return st;
    take(x, b->d_x);
    take(f, b->d_f);
    take(e, b->d_e);
    take(pm, b->d_p);
    *keep = b;
    return QB_OK;
}

}  // namespace qb
