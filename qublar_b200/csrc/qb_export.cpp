// On-disk formats around the annealer: the machine export of a tomography
// solve (the ising_out_* files), a region's QUBO as text, and the general
// QUBO text of the reference's sequencing study. Host only. Numbers are
// formatted and parsed with std::to_chars / std::from_chars, so the files do
// not depend on the process locale: %.17g-equivalent (17 significant digits,
// general format) where the reference prints 17 digits, and 6 significant
// digits where it uses the iostream default.
#include <charconv>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <memory>
#include <new>
#include <string>
#include <system_error>
#include <utility>
#include <vector>

#include "qb_internal.hpp"

namespace {

using qb::fail;

std::string num(double v, int digits) {
    char buf[64];
    const auto r = std::to_chars(buf, buf + sizeof buf, v, std::chars_format::general, digits);
    return std::string(buf, r.ptr);
}

// Writes `size` bytes; reports the file in the error.
qb_status write_file(const std::string& path, const void* data, size_t size) {
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) return fail(QB_EINVAL, ("cannot open " + path + " for writing").c_str());
    const size_t w = size ? std::fwrite(data, 1, size, f) : 0;
    const bool ok = w == size && std::fclose(f) == 0;
    if (!ok) return fail(QB_EINVAL, ("short write to " + path).c_str());
    return QB_OK;
}

qb_status write_text(const std::string& path, const std::string& s) { return write_file(path, s.data(), s.size()); }

std::string join(const char* dir, const char* name) {
    std::string p(dir);
    if (!p.empty() && p.back() != '/') p += '/';
    return p + name;
}

}  // namespace

// ---- the machine export (src/check_ising.cu:507-525, tools/export_machine_map.py:47-55,130-145) ----

extern "C" qb_status qb_write_ising_out(const char* dir, const qb_export_desc* d) {
    return qb::guarded("qb_write_ising_out", [&]() -> qb_status {
        if (!dir || !d || !d->var_voxel || !d->p_void) return fail(QB_EINVAL, "qb_write_ising_out: null argument");
        if (d->nx <= 0 || d->nx > 1024) return fail(QB_EINVAL, "qb_write_ising_out: nx must be in [1, 1024]");
        if (d->n_vars < 0) return fail(QB_EINVAL, "qb_write_ising_out: n_vars must be non-negative");
        if (d->branches && d->n_branches <= 0) return fail(QB_EINVAL, "qb_write_ising_out: branches given without a count");
        const size_t cells = size_t(d->nx) * size_t(d->nx) * size_t(d->nx);
        std::vector<float> grid(cells, -1.0f), grid_d;
        std::vector<uint8_t> taken(cells, 0);
        for (int i = 0; i < d->n_vars; ++i) {
            const int32_t v = d->var_voxel[i];
            if (v < 0 || size_t(v) >= cells) return fail(QB_EINVAL, "qb_write_ising_out: voxel index out of range");
            if (taken[size_t(v)]) return fail(QB_EINVAL, "qb_write_ising_out: two bits map to one voxel");
            taken[size_t(v)] = 1;
            grid[size_t(v)] = d->p_void[i];
        }
        qb_status s;
        if ((s = write_file(join(dir, "ising_out_pvoid.bin"), grid.data(), cells * 4)) != QB_OK) return s;
        if (d->p_void_noprior) {
            grid_d.assign(cells, -1.0f);
            for (int i = 0; i < d->n_vars; ++i) grid_d[size_t(d->var_voxel[i])] = d->p_void_noprior[i];
            if ((s = write_file(join(dir, "ising_out_pvoid_noprior.bin"), grid_d.data(), cells * 4)) != QB_OK) return s;
        }
        if (d->truth && (s = write_file(join(dir, "ising_out_truth.bin"), d->truth, cells)) != QB_OK) return s;
        if (d->branches && (s = write_file(join(dir, "ising_out_branches.bin"), d->branches,
                                             size_t(d->n_branches) * size_t(d->n_vars))) != QB_OK)
            return s;
        const std::string voxel = num(d->voxel, 6);
        const std::string lo = num(d->lo[0], 6) + " " + num(d->lo[1], 6) + " " + num(d->lo[2], 6);
        const std::string meta = "nx " + std::to_string(d->nx) + "\nvoxel " + voxel + "\nlo " + lo + "\nbranches " +
                                 std::to_string(d->n_branches) + "\nvars " + std::to_string(d->n_vars) + "\nlambda " +
                                 num(d->lambda, 6) + "\nkappa " + num(d->kappa, 6) + "\n";
        if ((s = write_text(join(dir, "ising_out.meta"), meta)) != QB_OK) return s;
        // the two masks: classify (ising_recon.hpp:305-309) at 0.1 / 0.9 in fp32,
        // 255 outside; only Exists is traversable
        std::vector<uint8_t> tri(cells, 255), trav(cells, 0);
        for (size_t c = 0; c < cells; ++c) {
            if (!taken[c]) continue;
            const float p = grid[c];
            tri[c] = p >= 0.9f ? 1 : (p <= 0.1f ? 0 : 2);
            trav[c] = tri[c] == 0 ? 1 : 0;
        }
        if ((s = write_file(join(dir, "ising_out_tristate.bin"), tri.data(), cells)) != QB_OK) return s;
        if ((s = write_file(join(dir, "ising_out_traversable.bin"), trav.data(), cells)) != QB_OK) return s;
        const std::string machine =
            "nx " + std::to_string(d->nx) + "\nvoxel " + voxel + "\nlo " + lo +
            "\norder zyx_C\npvoid ising_out_pvoid.bin float32\n"
            "tristate ising_out_tristate.bin uint8 0=Exists 1=NotThere 2=Undecided 255=outside\n"
            "traversable ising_out_traversable.bin uint8 1=Exists_only\nclassify_lo 0.1\nclassify_hi 0.9\n"
            "policy Exists=traversable; Undecided|NotThere|outside=block\n"
            "note does_not_include_evidence_budget; see check_ising / RESULTS\n";
        return write_text(join(dir, "ising_out_machine.meta"), machine);
    });
}

// ---- a region's QUBO as text (src/check_ising.cu:568-591) ----

extern "C" qb_status qb_write_roi_text(const char* path, int32_t n, const int32_t* voxel, const float* p,
                                       const uint8_t* truth, const double* h, const double* J) {
    return qb::guarded("qb_write_roi_text", [&]() -> qb_status {
        if (!path || n < 0 || (n > 0 && (!voxel || !p || !h || !J))) return fail(QB_EINVAL, "qb_write_roi_text: bad argument");
        std::string s = std::to_string(n) + "\n";
        for (int i = 0; i < n; ++i)
            s += std::to_string(voxel[i]) + " " + num(double(p[i]), 17) + " " + std::to_string(truth ? int(truth[i]) : 0) +
                 " " + num(h[i], 17) + "\n";
        for (int i = 0; i < n; ++i) {
            for (int j = 0; j < n; ++j) s += num(J[size_t(i) * size_t(n) + size_t(j)], 17) + " ";
            s += "\n";
        }
        return write_text(path, s);
    });
}

// ---- general QUBO text (src/check_ree_qubo.cu:277-283) ----

struct qb_qubo_text {
    int32_t n = 0;
    double offset = 0.0, penalty = 0.0, optimum = 0.0;
    std::vector<double> qd, cost, qo;
    std::vector<int32_t> eu, ev;
    std::vector<float> hf, wf;   // the fp32 descriptor's arrays
};

namespace {

// A cursor over the text: tokens separated by blanks, lines by '\n'.
struct Cursor {
    const char* p;
    const char* end;
    void blanks() {
        while (p < end && (*p == ' ' || *p == '\t' || *p == '\r')) ++p;
    }
    bool at_eol() {
        blanks();
        return p == end || *p == '\n';
    }
    bool next_line() {   // past the end of the current line, which must hold nothing more
        if (!at_eol()) return false;
        if (p < end) ++p;
        return true;
    }
    template <typename T>
    bool take(T& v) {
        blanks();
        const char* s = p;
        while (p < end && *p != ' ' && *p != '\t' && *p != '\r' && *p != '\n') ++p;
        if (s == p) return false;
        const auto r = std::from_chars(s, p, v);
        return r.ec == std::errc() && r.ptr == p;
    }
};

}  // namespace

extern "C" qb_status qb_parse_qubo_text(const char* text, size_t size, qb_qubo_text** out) {
    return qb::guarded("qb_parse_qubo_text", [&]() -> qb_status {
        if (!text || !out) return fail(QB_EINVAL, "qb_parse_qubo_text: null argument");
        *out = nullptr;
        std::unique_ptr<qb_qubo_text> q(new (std::nothrow) qb_qubo_text());
        if (!q) return fail(QB_ENOMEM, "qb_parse_qubo_text: out of host memory");
        Cursor c{text, text + size};
        int64_t m = 0;
        if (!c.take(q->n) || !c.take(m) || !c.take(q->offset) || !c.take(q->penalty) || !c.take(q->optimum) || !c.next_line())
            return fail(QB_EINVAL, "qubo text: bad header (want \"n m offset P optimum\")");
        if (q->n < 1 || m < 0 || m > int64_t(q->n) * (int64_t(q->n) - 1) / 2)
            return fail(QB_EINVAL, "qubo text: header counts out of range");
        if (int64_t(q->n) + m > int64_t(size / 6))   // every following line takes at least 6 bytes
            return fail(QB_EINVAL, "qubo text: the header counts more lines than the text holds");
        if (!std::isfinite(q->offset) || !std::isfinite(q->penalty) || !std::isfinite(q->optimum))
            return fail(QB_EINVAL, "qubo text: non-finite header value");
        q->qd.resize(size_t(q->n));
        q->cost.resize(size_t(q->n));
        for (int i = 0; i < q->n; ++i) {
            int32_t idx = -1;
            if (!c.take(idx) || !c.take(q->qd[size_t(i)]) || !c.take(q->cost[size_t(i)]) || !c.next_line())
                return fail(QB_EINVAL, "qubo text: bad linear line (want \"i Qd c\")");
            if (idx != i) return fail(QB_EINVAL, "qubo text: linear lines out of order");
            if (!std::isfinite(q->qd[size_t(i)]) || !std::isfinite(q->cost[size_t(i)]))
                return fail(QB_EINVAL, "qubo text: non-finite linear value");
        }
        q->eu.resize(size_t(m));
        q->ev.resize(size_t(m));
        q->qo.resize(size_t(m));
        for (int64_t k = 0; k < m; ++k) {
            int32_t i = -1, j = -1;
            if (!c.take(i) || !c.take(j) || !c.take(q->qo[size_t(k)]) || !c.next_line())
                return fail(QB_EINVAL, "qubo text: bad pair line (want \"i j Qo\")");
            if (i < 0 || j >= q->n || i >= j) return fail(QB_EINVAL, "qubo text: pair index out of range (want 0 <= i < j < n)");
            if (k > 0 && (i < q->eu[size_t(k) - 1] || (i == q->eu[size_t(k) - 1] && j <= q->ev[size_t(k) - 1])))
                return fail(QB_EINVAL, "qubo text: pairs not in ascending (i, j) order or repeated");
            if (!std::isfinite(q->qo[size_t(k)])) return fail(QB_EINVAL, "qubo text: non-finite coupling");
            q->eu[size_t(k)] = i;
            q->ev[size_t(k)] = j;
        }
        for (;;) {   // only blank lines may follow
            if (c.p == c.end) break;
            if (!c.next_line()) return fail(QB_EINVAL, "qubo text: trailing text after the last pair");
        }
        q->hf.assign(q->qd.begin(), q->qd.end());
        q->wf.assign(q->qo.begin(), q->qo.end());
        for (size_t k = 0; k < q->wf.size(); ++k)
            if (!std::isfinite(q->wf[k])) return fail(QB_EINVAL, "qubo text: a coupling overflows fp32");
        for (size_t k = 0; k < q->hf.size(); ++k)
            if (!std::isfinite(q->hf[k])) return fail(QB_EINVAL, "qubo text: a linear term overflows fp32");
        *out = q.release();
        return QB_OK;
    });
}

extern "C" qb_status qb_qubo_text_info(const qb_qubo_text* q, int32_t* n, int64_t* m, double* offset, double* penalty,
                                       double* optimum) {
    if (!q) return fail(QB_EINVAL, "qb_qubo_text_info: null handle");
    if (n) *n = q->n;
    if (m) *m = int64_t(q->qo.size());
    if (offset) *offset = q->offset;
    if (penalty) *penalty = q->penalty;
    if (optimum) *optimum = q->optimum;
    return QB_OK;
}

extern "C" qb_status qb_qubo_text_arrays(const qb_qubo_text* q, double* qd, double* cost, int32_t* eu, int32_t* ev,
                                         double* qo) {
    if (!q) return fail(QB_EINVAL, "qb_qubo_text_arrays: null handle");
    if (qd) std::memcpy(qd, q->qd.data(), q->qd.size() * 8);
    if (cost) std::memcpy(cost, q->cost.data(), q->cost.size() * 8);
    if (eu && !q->eu.empty()) std::memcpy(eu, q->eu.data(), q->eu.size() * 4);
    if (ev && !q->ev.empty()) std::memcpy(ev, q->ev.data(), q->ev.size() * 4);
    if (qo && !q->qo.empty()) std::memcpy(qo, q->qo.data(), q->qo.size() * 8);
    return QB_OK;
}

extern "C" qb_status qb_qubo_text_desc(const qb_qubo_text* q, qb_qubo_desc* d) {
    if (!q || !d) return fail(QB_EINVAL, "qb_qubo_text_desc: null argument");
    d->n = q->n;
    d->m = int64_t(q->qo.size());
    d->eu = q->eu.data();
    d->ev = q->ev.data();
    d->ew = q->wf.data();
    d->h = q->hf.data();
    d->offset = q->offset;
    return QB_OK;
}

extern "C" void qb_qubo_text_destroy(qb_qubo_text* q) { delete q; }

extern "C" qb_status qb_write_qubo_text(const char* path, int32_t n, int64_t m, double offset, double penalty,
                                        double optimum, const double* qd, const double* cost, const int32_t* eu,
                                        const int32_t* ev, const double* qo) {
    return qb::guarded("qb_write_qubo_text", [&]() -> qb_status {
        if (!path || n < 1 || m < 0 || !qd || !cost || (m > 0 && (!eu || !ev || !qo)))
            return fail(QB_EINVAL, "qb_write_qubo_text: bad argument");
        for (int64_t k = 0; k < m; ++k) {
            if (eu[k] < 0 || ev[k] >= n || eu[k] >= ev[k])
                return fail(QB_EINVAL, "qb_write_qubo_text: pair index out of range (want 0 <= i < j < n)");
            if (k > 0 && (eu[k] < eu[k - 1] || (eu[k] == eu[k - 1] && ev[k] <= ev[k - 1])))
                return fail(QB_EINVAL, "qb_write_qubo_text: pairs not in ascending (i, j) order or repeated");
        }
        std::string s = std::to_string(n) + " " + std::to_string(m) + " " + num(offset, 17) + " " + num(penalty, 17) + " " +
                        num(optimum, 17) + "\n";
        for (int i = 0; i < n; ++i) s += std::to_string(i) + " " + num(qd[i], 17) + " " + num(cost[i], 17) + "\n";
        for (int64_t k = 0; k < m; ++k)
            s += std::to_string(eu[k]) + " " + std::to_string(ev[k]) + " " + num(qo[k], 17) + "\n";
        return write_text(path, s);
    });
}
